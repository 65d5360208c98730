"""CPU oracle for the elastic velocity-strain path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only as the checker / the timed CPU baseline.  The
product (``stfwi_b200``) never imports it.

The wave-equation parts live in ``stfwi_oracle.c`` (built by ``Makefile`` into
``liboracle.so``); this module binds them with ctypes and restates, in NumPy,
the host-side pieces of the reference that sit around them:

* ``ricker``                     fwi/forward.py:25-28
* ``cosine_taper_end``           fwi/filters.py:26-32
* ``sosfilt`` / ``sosfilt_T``    fwi/filters.py:14-40 (biquad direct form I,
  normalised by a0) and its transpose (time-reversed cascade)
* ``shot_misfit_and_cotangent``  fwi/gradient.py:139-156 (+ jax.grad of it)
* ``gaussian_smooth_2d``         fwi/loss.py:17-30
* ``crop`` / chain rules         fwi/imaging.py:156-167, and the exact
  (M, L, L2M, B) -> (Vs, Vp, rho) chain of fwi/forward.py:222-227
* ``compute_gradient``           fwi/gradient.py:48-99, backends ``'ad'``
  (exact discrete gradient, what the reference gets from JAX AD) and
  ``'adjoint'`` (forward -> hand adjoint -> imaging condition)
* ``compute_illumination``       fwi/illumination.py:18-48
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None
_lock = threading.Lock()


class OracleDesc(ct.Structure):
    _fields_ = [
        ("nz_dom", ct.c_int32), ("nx_dom", ct.c_int32), ("pad", ct.c_int32),
        ("fd_order", ct.c_int32), ("free_surface", ct.c_int32), ("nt", ct.c_int32),
        ("nrec", ct.c_int32), ("d0_f32", ct.c_int32),
        ("dx", ct.c_double), ("dz", ct.c_double), ("dt", ct.c_double), ("fc", ct.c_double),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_FAST_PATH = os.path.join(_HERE, "liboracle_fast.so")
_fast = None


def build_fast() -> str:
    """Compile liboracle_fast.so (FP32, -march=native, FP contraction, OpenMP
    over shots) for THIS host: it is rebuilt on every call, as a copy made on
    another machine may target another instruction set."""
    subprocess.run(["make", "-s", "-B", "-C", _HERE, "fast"], check=True)
    return _FAST_PATH


def _bind(L, prefixes):
    P = ct.POINTER
    dp, ip = P(ct.c_double), P(ct.c_int32)
    for pre in prefixes:
        f = getattr(L, pre + "forward")
        f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ct.c_int32, ct.c_int32, dp,
                      ip, ip, dp, ct.c_int32, dp, ct.c_int32, dp]
        f.restype = ct.c_int
        f = getattr(L, pre + "adjoint")
        f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ct.c_int32, ct.c_int32, dp,
                      ip, ip, dp, dp, dp, dp, ct.c_int32, dp, ct.c_int32]
        f.restype = ct.c_int
        f = getattr(L, pre + "forward_batch")
        f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ip, dp, ip, ip, dp]
        f.restype = ct.c_int
        f = getattr(L, pre + "gradient_batch")
        f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ip, dp, ip, ip, dp, dp, dp,
                      ct.c_int32]
        f.restype = ct.c_int
        f = getattr(L, pre + "pml_profiles")
        f.argtypes = [P(OracleDesc), dp, dp]
        f.restype = ct.c_int
    return L


def lib_fast():
    """The tuned timing build (symbols oraclefast_*), built here on first use."""
    global _fast
    with _lock:
        if _fast is None:
            build_fast()
            _fast = _bind(ct.CDLL(_FAST_PATH), ("oraclefast_",))
        return _fast


def _entry(name, precision):
    """Entry point `name` of the FP64 (64), FP32 (32) or tuned FP32 ('fast') build."""
    if precision == "fast":
        return getattr(lib_fast(), "oraclefast_" + name)
    return getattr(lib(), f"oracle{precision}_{name}")


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH):
                build()
            L = ct.CDLL(_LIB_PATH)
            P = ct.POINTER
            dp, ip = P(ct.c_double), P(ct.c_int32)
            for pre in ("oracle64_", "oracle32_"):
                f = getattr(L, pre + "forward")
                f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ct.c_int32, ct.c_int32, dp,
                              ip, ip, dp, ct.c_int32, dp, ct.c_int32, dp]
                f.restype = ct.c_int
                f = getattr(L, pre + "adjoint")
                f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ct.c_int32, ct.c_int32, dp,
                              ip, ip, dp, dp, dp, dp, ct.c_int32, dp, ct.c_int32]
                f.restype = ct.c_int
                f = getattr(L, pre + "forward_batch")
                f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ip, dp, ip, ip, dp]
                f.restype = ct.c_int
                f = getattr(L, pre + "gradient_batch")
                f.argtypes = [P(OracleDesc), dp, dp, dp, ct.c_int32, ip, dp, ip, ip, dp, dp, dp,
                              ct.c_int32]
                f.restype = ct.c_int
                f = getattr(L, pre + "pml_profiles")
                f.argtypes = [P(OracleDesc), dp, dp]
                f.restype = ct.c_int
            _lib = L
        return _lib


def _dptr(a):
    return None if a is None else a.ctypes.data_as(ct.POINTER(ct.c_double))


def _iptr(a):
    return None if a is None else a.ctypes.data_as(ct.POINTER(ct.c_int32))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


SRC_TYPES = {"force": 0, "moment": 1}
FIELD_BITS = {"vx": 0, "vz": 1, "ex": 2, "ez": 3, "es": 4}


def grid_shape(nz_dom, nx_dom, pad, free_surface):
    """(nz_t, nx_t) of the padded grid, fwi/forward.py:185-190."""
    return (nz_dom + pad if free_surface else nz_dom + 2 * pad), nx_dom + 2 * pad


def make_desc(nz_dom, nx_dom, pad, fd_order, free_surface, nt, nrec, dx, dz, dt, fc, d0_f32=False):
    return OracleDesc(int(nz_dom), int(nx_dom), int(pad), int(fd_order), int(bool(free_surface)),
                      int(nt), int(nrec), int(bool(d0_f32)), float(dx), float(dz), float(dt), float(fc))


# ----------------------------------------------------------------------------- wave equation

def forward(Vs, Vp, rho, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt, fc, pad,
            src_wavelet, fd_order=2, free_surface=True, src_type="force", full=(), energy=(),
            d0_f32=None, precision=64):
    """One shot of fwi/forward.py:forward_jax.

    Returns ``(rec, full_frames, energy)``: ``rec`` is the (vx, vz, ex, ez)
    tuple of (nt, nrec) receiver traces; ``full_frames`` maps each name in
    ``full`` to its (nt, nz_t, nx_t) history; ``energy`` maps each name in
    ``energy`` to Sum_t field**2 on the padded grid.  ``d0_f32`` defaults to
    "Vp arrived as float32", which is how the reference's JAX promotion builds
    the PML profile (fwi/forward.py:48).
    """
    if fd_order not in (2, 4, 8):
        raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
    if src_type not in SRC_TYPES:
        raise NotImplementedError(f"src_type={src_type!r} not supported (use 'force' or 'moment').")
    if d0_f32 is None:
        d0_f32 = np.asarray(Vp).dtype == np.float32
    rec_x, rec_z = _i32(rec_x), _i32(rec_z)
    nrec = rec_x.size
    d = make_desc(nz_dom, nx_dom, pad, fd_order, free_surface, nt, nrec, dx, dz, dt, fc, d0_f32)
    nz, nx = grid_shape(nz_dom, nx_dom, pad, free_surface)
    rec = np.zeros((4, nt, nrec))
    fmask = 0
    for k in full:
        fmask |= 1 << FIELD_BITS[k]
    emask = 0
    for k in energy:
        emask |= 1 << FIELD_BITS[k]
    fnames = [k for k in ("vx", "vz", "ex", "ez", "es") if fmask >> FIELD_BITS[k] & 1]
    enames = [k for k in ("vx", "vz", "ex", "ez", "es") if emask >> FIELD_BITS[k] & 1]
    fout = np.zeros((len(fnames), nt, nz, nx)) if fnames else None
    eout = np.zeros((len(enames), nz, nx)) if enames else None
    fn = getattr(lib(), f"oracle{precision}_forward")
    rc = fn(ct.byref(d), _dptr(_f64(Vs)), _dptr(_f64(Vp)), _dptr(_f64(rho)), int(src_x), int(src_z),
            SRC_TYPES[src_type], _dptr(_f64(src_wavelet)), _iptr(rec_x), _iptr(rec_z), _dptr(rec),
            fmask, _dptr(fout), emask, _dptr(eout))
    if rc:
        raise ValueError(f"oracle forward failed (code {rc})")
    full_frames = {k: fout[i] for i, k in enumerate(fnames)}
    en = {k: eout[i] for i, k in enumerate(enames)}
    return tuple(rec), full_frames, en


def adjoint(Vs, Vp, rho, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt, fc, pad,
            rec_vx_a, rec_vz_a, rec_ex_a, rec_ez_a, fd_order=2, free_surface=False,
            src_type="force", src_wavelet=None, want=("src",), hist=(), ckpt=25, d0_f32=None,
            precision=64):
    """One shot of fwi/adjoint_jax_kernel.py:adjoint_jax, plus optional model
    gradients.

    ``want`` may hold ``"src"`` (source-wavelet adjoint, (nt,)), ``"gmat"``
    (exact dJ/d(M, L, L2M, B) on the padded grid, [4, nz_t, nx_t]) and
    ``"img"`` ((g_lam, g_mu, g_rho_lame) of fwi/imaging.py on the padded
    grid; g_rho_lame is the density term of fwi/imaging.py:145-154).  The
    last two need ``src_wavelet`` to recompute the forward.
    """
    if fd_order not in (2, 4, 8):
        raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
    if src_type not in SRC_TYPES:
        raise NotImplementedError(f"src_type={src_type!r} not supported (use 'force' or 'moment').")
    if d0_f32 is None:
        d0_f32 = np.asarray(Vp).dtype == np.float32
    rec_x, rec_z = _i32(rec_x), _i32(rec_z)
    nrec = rec_x.size
    d = make_desc(nz_dom, nx_dom, pad, fd_order, free_surface, nt, nrec, dx, dz, dt, fc, d0_f32)
    nz, nx = grid_shape(nz_dom, nx_dom, pad, free_surface)
    ra = np.ascontiguousarray(np.stack([_f64(rec_vx_a), _f64(rec_vz_a), _f64(rec_ex_a), _f64(rec_ez_a)]))
    src_a = np.zeros(nt) if "src" in want else None
    gmat = np.zeros((4, nz, nx)) if "gmat" in want else None
    img = np.zeros((3, nz, nx)) if "img" in want else None
    hmask = 0
    hb = {"U_a": 0, "V_a": 1, "ex_a": 2, "ez_a": 3, "es_a": 4}
    for k in hist:
        hmask |= 1 << hb[k]
    hnames = [k for k in ("U_a", "V_a", "ex_a", "ez_a", "es_a") if hmask >> hb[k] & 1]
    hout = np.zeros((len(hnames), nt, nz, nx)) if hnames else None
    if (gmat is not None or img is not None) and src_wavelet is None:
        raise ValueError("model gradients need src_wavelet")
    wav = _f64(src_wavelet) if src_wavelet is not None else None
    fn = getattr(lib(), f"oracle{precision}_adjoint")
    rc = fn(ct.byref(d), _dptr(_f64(Vs)), _dptr(_f64(Vp)), _dptr(_f64(rho)), int(src_x), int(src_z),
            SRC_TYPES[src_type], _dptr(wav), _iptr(rec_x), _iptr(rec_z), _dptr(ra), _dptr(src_a),
            _dptr(gmat), _dptr(img), hmask, _dptr(hout), int(ckpt))
    if rc:
        raise ValueError(f"oracle adjoint failed (code {rc})")
    out = {"src": src_a, "gmat": gmat, "img": img}
    for i, k in enumerate(hnames):
        out[k] = hout[i]
    return out


def pml_profiles(nz_dom, nx_dom, pad, free_surface, dx, dt, fc, Vp, d0_f32=None):
    """(kx, kz, bx, bz, ax, az) on the padded grid, fwi/forward.py:35-104."""
    if d0_f32 is None:
        d0_f32 = np.asarray(Vp).dtype == np.float32
    d = make_desc(nz_dom, nx_dom, pad, 2, free_surface, 1, 0, dx, dx, dt, fc, d0_f32)
    nz, nx = grid_shape(nz_dom, nx_dom, pad, free_surface)
    out = np.zeros((6, nz, nx))
    rc = lib().oracle64_pml_profiles(ct.byref(d), _dptr(_f64(Vp)), _dptr(out))
    if rc:
        raise ValueError(f"oracle pml_profiles failed (code {rc})")
    return tuple(out)


# ----------------------------------------------------------------------------- host-side pieces

def ricker(t, fc, t0, scaling_factor=1.0):
    """fwi/forward.py:25-28."""
    arg = (np.pi * fc * (np.asarray(t, dtype=np.float64) - t0)) ** 2
    return scaling_factor * (1.0 - 2.0 * arg) * np.exp(-arg)


def cosine_taper_end(x, n_taper):
    """fwi/filters.py:26-32: taper the last n_taper samples of axis 0 (1 -> 0)."""
    x = np.array(x, dtype=np.float64, copy=True)
    n_taper = min(int(n_taper), x.shape[0])
    if n_taper <= 0:
        return x
    taper = (np.cos(np.arange(1, n_taper + 1) / n_taper * np.pi) + 1) / 2
    x[-n_taper:] *= taper.reshape((-1,) + (1,) * (x.ndim - 1))
    return x


def _biquad(x, b0, b1, b2, a1, a2):
    """fwi/filters.py:14-23, direct form I along axis 0."""
    y = np.zeros_like(x)
    x1 = np.zeros_like(x[0]); x2 = np.zeros_like(x[0])
    y1 = np.zeros_like(x[0]); y2 = np.zeros_like(x[0])
    for i in range(x.shape[0]):
        xi = x[i]
        yi = b0 * xi + b1 * x1 + b2 * x2 - a1 * y1 - a2 * y2
        y[i] = yi
        x2, x1, y2, y1 = x1, xi, y1, yi
    return y


def sosfilt(x, sos):
    """fwi/filters.py:35-40: cascade of biquads, each normalised by a0."""
    x = np.asarray(x, dtype=np.float64)
    for s in np.asarray(sos, dtype=np.float64):
        x = _biquad(x, s[0] / s[3], s[1] / s[3], s[2] / s[3], s[4] / s[3], s[5] / s[3])
    return x


def sosfilt_T(y, sos):
    """Transpose of ``sosfilt`` along axis 0: reverse time, run the sections
    in reverse order, reverse back (each section is causal LTI)."""
    y = np.asarray(y, dtype=np.float64)[::-1]
    for s in np.asarray(sos, dtype=np.float64)[::-1]:
        y = _biquad(y, s[0] / s[3], s[1] / s[3], s[2] / s[3], s[4] / s[3], s[5] / s[3])
    return np.ascontiguousarray(y[::-1])


def shot_misfit_and_cotangent(pred, obs, sos, n_taper, scale, n_shots):
    """fwi/gradient.py:139-156 and the jax.grad of it w.r.t. ``pred``:
    misfit_k = (scale/n_shots) * mean((F T pred - F T obs)**2),
    cotangent = (2 scale / (n_shots N)) T^T F^T (F T pred - F T obs)."""
    est = np.asarray(pred, dtype=np.float64)
    obs_p = np.asarray(obs, dtype=np.float64)
    if n_taper > 0:
        est = cosine_taper_end(est, n_taper)
        obs_p = cosine_taper_end(obs_p, n_taper)
    if sos is not None:
        est = sosfilt(est, sos)
        obs_p = sosfilt(obs_p, sos)
    r = est - obs_p
    misfit = (scale / n_shots) * np.mean(r ** 2)
    g = (2.0 * scale / (n_shots * r.size)) * r
    if sos is not None:
        g = sosfilt_T(g, sos)
    if n_taper > 0:
        g = cosine_taper_end(g, n_taper)
    return float(misfit), g


def gaussian_smooth_2d(field, sigma, truncate=3.0):
    """fwi/loss.py:17-30: normalised 2-D Gaussian, 'same' zero-padded convolution."""
    from scipy.signal import convolve2d
    radius = int(truncate * sigma + 0.5)
    x = np.arange(2 * radius + 1) - radius
    g1 = np.exp(-0.5 * (x / sigma) ** 2)
    k = np.outer(g1, g1)
    k = k / k.sum()
    return convolve2d(np.asarray(field, dtype=np.float64), k, mode="same")


def crop(full, pad, free_surface, nz_dom, nx_dom):
    """Physical domain of a padded-grid array (fwi/imaging.py:157-162)."""
    z0 = 0 if free_surface else pad
    return full[..., z0:z0 + nz_dom, pad:pad + nx_dom]


def chain_exact(gmat_phys, Vs, Vp, rho):
    """(dJ/dM, dJ/dL, dJ/dL2M, dJ/dB) -> (dJ/dVs, dJ/dVp, dJ/drho) with
    M = rho Vs^2, L2M = rho Vp^2, L = L2M - 2M, B = 1/rho (fwi/forward.py:222-227)."""
    gM, gL, gL2M, gB = gmat_phys
    Vs = np.asarray(Vs, np.float64); Vp = np.asarray(Vp, np.float64); rho = np.asarray(rho, np.float64)
    g_vs = 2.0 * rho * Vs * (gM - 2.0 * gL)
    g_vp = 2.0 * rho * Vp * (gL2M + gL)
    g_rho = Vs ** 2 * gM + Vp ** 2 * gL2M + (Vp ** 2 - 2.0 * Vs ** 2) * gL - gB / rho ** 2
    return g_vs, g_vp, g_rho


def chain_imaging(g_lam, g_mu, Vs, Vp, rho, g_rho_lame=None):
    """fwi/imaging.py:165-167."""
    Vs = np.asarray(Vs, np.float64); Vp = np.asarray(Vp, np.float64); rho = np.asarray(rho, np.float64)
    if g_rho_lame is None:
        g_rho_lame = np.zeros_like(g_lam)
    g_vs = 2.0 * rho * Vs * (g_mu - 2.0 * g_lam)
    g_vp = 2.0 * rho * Vp * g_lam
    g_rho = (Vp ** 2 - 2.0 * Vs ** 2) * g_lam + Vs ** 2 * g_mu + g_rho_lame
    return g_vs, g_vp, g_rho


_COMP = {0: "vx", 1: "vz", 2: "ex", 3: "ez"}


def forward_batch(Vs, Vp, rho, src_x, src_z, src_types, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt,
                  fc, pad, src_wavelet, fd_order=2, free_surface=True, d0_f32=None, precision=64):
    """Receiver traces of many shots, OpenMP over shots: [nshot, 4, nt, nrec]."""
    if d0_f32 is None:
        d0_f32 = np.asarray(Vp).dtype == np.float32
    rec_x, rec_z = _i32(rec_x), _i32(rec_z)
    ns = len(src_x)
    src = _i32(np.stack([np.asarray(src_x).reshape(-1), np.asarray(src_z).reshape(-1),
                         [SRC_TYPES[t] for t in src_types]], axis=1))
    d = make_desc(nz_dom, nx_dom, pad, fd_order, free_surface, nt, rec_x.size, dx, dz, dt, fc, d0_f32)
    out = np.zeros((ns, 4, nt, rec_x.size))
    fn = _entry("forward_batch", precision)
    rc = fn(ct.byref(d), _dptr(_f64(Vs)), _dptr(_f64(Vp)), _dptr(_f64(rho)), ns, _iptr(src),
            _dptr(_f64(src_wavelet)), _iptr(rec_x), _iptr(rec_z), _dptr(out))
    if rc:
        raise ValueError(f"oracle forward_batch failed (code {rc})")
    return out


def gradient_batch(Vs, Vp, rho, src_x, src_z, src_types, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt,
                   nt, fc, pad, src_wavelet, rec_adj, fd_order=2, free_surface=True, mode="gmat",
                   ckpt=25, d0_f32=None, precision=64):
    """Per-shot model gradients, OpenMP over shots.  ``mode='gmat'``: exact
    dJ/d(M, L, L2M, B) [nshot, 4, nz_t, nx_t]; ``mode='img'``: (g_lam, g_mu,
    g_rho_lame) of fwi/imaging.py [nshot, 3, nz_t, nx_t]."""
    if d0_f32 is None:
        d0_f32 = np.asarray(Vp).dtype == np.float32
    rec_x, rec_z = _i32(rec_x), _i32(rec_z)
    ns = len(src_x)
    src = _i32(np.stack([np.asarray(src_x).reshape(-1), np.asarray(src_z).reshape(-1),
                         [SRC_TYPES[t] for t in src_types]], axis=1))
    d = make_desc(nz_dom, nx_dom, pad, fd_order, free_surface, nt, rec_x.size, dx, dz, dt, fc, d0_f32)
    nz, nx = grid_shape(nz_dom, nx_dom, pad, free_surface)
    gm = np.zeros((ns, 4, nz, nx)) if mode == "gmat" else None
    im = np.zeros((ns, 3, nz, nx)) if mode == "img" else None
    fn = _entry("gradient_batch", precision)
    rc = fn(ct.byref(d), _dptr(_f64(Vs)), _dptr(_f64(Vp)), _dptr(_f64(rho)), ns, _iptr(src),
            _dptr(_f64(src_wavelet)), _iptr(rec_x), _iptr(rec_z), _dptr(_f64(rec_adj)), _dptr(gm),
            _dptr(im), int(ckpt))
    if rc:
        raise ValueError(f"oracle gradient_batch failed (code {rc})")
    return gm if mode == "gmat" else im


def compute_gradient(backend, *, Vs, Vp, rho, src_x, src_z, src_wavelet, observed, rec_x, rec_z,
                     nx_dom, nz_dom, dx, dz, dt, nt, fc, pad, component=2, invert="vs", scale=1.0,
                     sos=None, n_taper=0, fd_order=2, free_surface=False, src_type="force",
                     grad_smooth_sigma=None, source_taper=None, illumination=None, src_types=None,
                     ckpt=25, d0_f32=None, return_parts=False):
    """fwi/gradient.py:48-99 with backends ``'ad'`` (exact discrete gradient,
    the hand derivation standing in for JAX AD) and ``'adjoint'`` (hand
    adjoint + imaging condition).  ``src_types`` (per-shot list) overrides
    ``src_type`` for mixed force/moment batches; the same source type is used
    in the forward and the adjoint of each shot."""
    if backend not in ("ad", "adjoint"):
        raise ValueError(f"unknown backend {backend!r}; use 'ad' or 'adjoint'")
    if invert not in ("vs", "vs_vp", "all"):
        raise ValueError(f"invert={invert!r}; use 'vs', 'vs_vp', or 'all'")
    src_x = np.asarray(src_x).reshape(-1)
    src_z = np.asarray(src_z).reshape(-1)
    n_shots = len(src_x)
    if src_types is None:
        src_types = [src_type] * n_shots
    geo = dict(rec_x=rec_x, rec_z=rec_z, nx_dom=nx_dom, nz_dom=nz_dom, dx=dx, dz=dz, dt=dt, nt=nt,
               fc=fc, pad=pad, src_wavelet=src_wavelet, fd_order=fd_order,
               free_surface=free_surface, d0_f32=d0_f32)
    rec = forward_batch(Vs, Vp, rho, src_x, src_z, src_types, **geo)
    loss = 0.0
    rec_adj = np.zeros_like(rec)
    for k in range(n_shots):
        mis, cot = shot_misfit_and_cotangent(rec[k, component], observed[k], sos, n_taper, scale,
                                             n_shots)
        loss += mis
        rec_adj[k, component] = cot
    parts = gradient_batch(Vs, Vp, rho, src_x, src_z, src_types, rec_adj=rec_adj,
                           mode="gmat" if backend == "ad" else "img", ckpt=ckpt, **geo)
    tot = crop(parts.sum(axis=0), pad, free_surface, nz_dom, nx_dom)
    if backend == "ad":
        g_vs, g_vp, g_rho = chain_exact(tot, Vs, Vp, rho)
    else:
        g_vs, g_vp, g_rho = chain_imaging(tot[0], tot[1], Vs, Vp, rho, g_rho_lame=tot[2])
    if invert == "vs":
        g_vp = np.zeros_like(g_vp); g_rho = np.zeros_like(g_rho)
    elif invert == "vs_vp":
        g_rho = np.zeros_like(g_rho)
    grads = [g_vs, g_vp, g_rho]
    if grad_smooth_sigma is not None:
        grads = [gaussian_smooth_2d(g, grad_smooth_sigma) for g in grads]
    if source_taper is not None:
        grads = [g * np.asarray(source_taper) for g in grads]
    if illumination is not None:
        grads = [g * np.asarray(illumination) for g in grads]
    if return_parts:
        return tuple(grads), float(loss), {"rec": rec, "rec_adj": rec_adj, "parts": tot}
    return tuple(grads), float(loss)


def compute_illumination(nz, nx, dx, dz, dt, nt, f_c, pad, rec_x, rec_z, fd_order, component,
                         Vs, Vp, rho, src_x, src_z, src_wavelet, eps=0.001, free_surface=True,
                         src_type="force", d0_f32=None):
    """fwi/illumination.py:18-48 (the reference always runs it with a free
    surface, because build_forward_fn defaults to it, and crops ``Ws[:nz]``)."""
    name = _COMP[component]
    nz_t, nx_t = grid_shape(nz, nx, pad, free_surface)
    Ws = np.zeros((nz_t, nx_t))
    for i in range(len(src_x)):
        _, _, en = forward(Vs, Vp, rho, src_x[i], src_z[i], rec_x, rec_z, nx, nz, dx, dz, dt, nt,
                           f_c, pad, src_wavelet, fd_order, free_surface, src_type, energy=(name,),
                           d0_f32=d0_f32)
        Ws += en[name]
    Ws = Ws[:nz, pad:pad + nx]
    lamda = eps * np.max(Ws)
    H_inv = 1.0 / (Ws + lamda)
    return H_inv / np.max(H_inv), Ws


# ---------------------------------------------------------------- host pieces around the gradient

def project_velocity(Vs, Vp, rho, K_margin=0.04, vp_cap=None, vs_floor=1e-3, rho_floor=1e-3):
    """fwi/projections.py:67-117: Vp <= vp_cap, Vs <= Vp / ((1 + K) 2/sqrt 3),
    floors on Vs and rho (FP64 copies)."""
    vp = np.asarray(Vp, dtype=np.float64).copy()
    vs = np.asarray(Vs, dtype=np.float64).copy()
    rh = np.asarray(rho, dtype=np.float64).copy()
    r = (1.0 + float(K_margin)) * (2.0 / np.sqrt(3.0))
    if vp_cap is not None:
        vp = np.minimum(vp, float(vp_cap))
    vs = np.maximum(np.minimum(vs, vp / r), float(vs_floor))
    rh = np.maximum(rh, float(rho_floor))
    return vs, vp, rh


def illumination_inverse(Ws_padded, nz_dom, nx_dom, pad, eps):
    """fwi/illumination.py:44-47 on a forward energy of the padded grid
    (free surface: rows from 0)."""
    Ws = np.asarray(Ws_padded)[:nz_dom, pad:pad + nx_dom]
    h = 1.0 / (Ws + eps * np.max(Ws))
    return h / np.max(h)


def eprecond3_multiplier(Ws_padded, rec_x, rec_z, dx, dz, free_surface, pad, nz_dom, nx_dom, eps):
    """fwi/preconditioning.py:65-139 (We on the padded grid) followed by
    fwi/optim_lbfgsb.py:95-99 (crop, 1/We, normalised to max 1)."""
    Ws = np.asarray(Ws_padded, dtype=np.float64)
    nz_t, nx_t = Ws.shape
    z0 = 0 if free_surface else pad
    cz, cx = np.meshgrid((np.arange(nz_t) - z0) * dz, (np.arange(nx_t) - pad) * dx, indexing="ij")
    rec_x, rec_z = np.asarray(rec_x), np.asarray(rec_z)
    if np.std(rec_x) >= np.std(rec_z):
        lo, hi, perp, c_perp, c_line, sp = np.min(rec_x) * dx, np.max(rec_x) * dx, rec_z[0] * dz, cz, cx, dz
    else:
        lo, hi, perp, c_perp, c_line, sp = np.min(rec_z) * dz, np.max(rec_z) * dz, rec_x[0] * dx, cx, cz, dx
    y = np.maximum(np.abs(c_perp - perp), sp)
    We = np.abs(np.sqrt(Ws) * (np.arcsinh((hi - c_line) / y) - np.arcsinh((lo - c_line) / y)))
    We = We + eps * np.max(We)
    p = 1.0 / We[z0:z0 + nz_dom, pad:pad + nx_dom]
    return p / np.max(p)


def imaging_condition(Vs, Vp, rho, ex_hist, ez_hist, es_hist, U_a_hist, V_a_hist, dx, dz, dt, pad,
                      free_surface, nz_dom, nx_dom, vx_hist=None, vz_hist=None):
    """fwi/imaging.py:83-169 in NumPy FP64 on full histories (nt, nz_t, nx_t):
    B of the nearest-neighbour extension of rho (:56-80, :113-114), periodic
    centred differences of B U_a and B V_a (np.roll, :47-53), the Lame sums
    (:125-141), the density term with the centred time derivative (:145-154),
    the crop and the chain rule (:157-167).  Returns (g_Vs, g_Vp, g_rho,
    g_lam, g_mu, g_rho_lame)."""
    z0 = 0 if free_surface else pad
    nz, nx = grid_shape(nz_dom, nx_dom, pad, free_surface)
    ii = np.clip(np.arange(nz) - z0, 0, nz_dom - 1)
    jj = np.clip(np.arange(nx) - pad, 0, nx_dom - 1)
    B = 1.0 / np.asarray(rho, dtype=np.float64)[np.ix_(ii, jj)]
    ua, va = np.asarray(U_a_hist, np.float64), np.asarray(V_a_hist, np.float64)
    BU, BV = B * ua, B * va

    def cd(f, h, ax):
        return (np.roll(f, -1, axis=ax) - np.roll(f, 1, axis=ax)) / (2.0 * h)

    dxBU, dzBV, dzBU, dxBV = cd(BU, dx, 2), cd(BV, dz, 1), cd(BU, dz, 1), cd(BV, dx, 2)
    ex, ez, es = (np.asarray(a, np.float64) for a in (ex_hist, ez_hist, es_hist))
    g_lam = -dt * np.sum((ex + ez) * (dxBU + dzBV), axis=0)
    g_mu = -dt * np.sum(2.0 * ex * dxBU + 2.0 * ez * dzBV + es * (dzBU + dxBV), axis=0)
    g_rl = np.zeros((nz, nx))
    if vx_hist is not None:
        vx, vz = np.asarray(vx_hist, np.float64), np.asarray(vz_hist, np.float64)
        dua = (ua[2:] - ua[:-2]) / (2.0 * dt)
        dva = (va[2:] - va[:-2]) / (2.0 * dt)
        g_rl = -dt * np.sum(vx[1:-1] * dua + vz[1:-1] * dva, axis=0)
    sl = (slice(z0, z0 + nz_dom), slice(pad, pad + nx_dom))
    g_lam, g_mu, g_rl = g_lam[sl], g_mu[sl], g_rl[sl]
    Vs, Vp, r = (np.asarray(a, np.float64) for a in (Vs, Vp, rho))
    g_Vs = 2.0 * r * Vs * (g_mu - 2.0 * g_lam)
    g_Vp = 2.0 * r * Vp * g_lam
    g_rho = (Vp ** 2 - 2.0 * Vs ** 2) * g_lam + Vs ** 2 * g_mu + g_rl
    return g_Vs, g_Vp, g_rho, g_lam, g_mu, g_rl
