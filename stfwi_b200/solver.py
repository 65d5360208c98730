"""Host-side handle over the C ABI: one padded grid, one shot batch, one GPU.

Arrays may be NumPy (host) or torch tensors (host or CUDA); the C ABI copies
with cudaMemcpyDefault, so device tensors never leave the GPU.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _native as N

SRC_TYPES = {"force": N.SRC_FORCE, "moment": N.SRC_MOMENT}


def _torch():
    try:
        import torch
        return torch
    except ImportError:  # pragma: no cover
        return None


def _as_buffer(x, dtype):
    """(pointer, keep-alive) for a host or device array of the given dtype."""
    t = _torch()
    if t is not None and isinstance(x, t.Tensor):
        tdt = {np.float32: t.float32, np.float64: t.float64, np.int32: t.int32}[dtype]
        x = x.detach().to(tdt).contiguous()
        return x.data_ptr(), x
    a = np.ascontiguousarray(np.asarray(x, dtype=dtype))
    return a.ctypes.data, a


def _stream():
    t = _torch()
    if t is not None and t.cuda.is_available() and t.cuda.is_initialized():
        return ct.c_void_p(t.cuda.current_stream().cuda_stream)
    return None


def _want_gradient(want_gradient, density):
    """stfwi_desc.want_gradient: 0 none, 1 stress history, 2 stress and
    velocity history (the density gradient g_rho needs the velocities)."""
    if not want_gradient:
        return 0
    return 2 if density else 1


class Solver:
    """Batch of shots on one model; mirrors the arguments of the reference's
    forward_jax / build_forward_fn (fwi/forward.py:119-123, :508-509).

    ``density=True`` keeps the forward velocities in the gradient history so
    that ``gradient()`` also returns g_rho (the reference's invert='all'):
    dJ/drho of the exact gradient, and the imaging formula's density term."""

    def __init__(self, nz_dom, nx_dom, dx, dz, dt, nt, fc, pad, nrec, max_shots, fd_order=2,
                 free_surface=True, want_gradient=True, shot_group=0, mem_budget_gb=0.0,
                 kernel_variant=0, ckpt_interval=0, density=False):
        if fd_order not in (2, 4, 8):
            raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
        self.lib = N.load()
        self.density = bool(density and want_gradient)
        self.desc = N.StfwiDesc(int(nz_dom), int(nx_dom), int(pad), int(fd_order),
                                int(bool(free_surface)), int(nt), int(nrec), int(max_shots),
                                float(dx), float(dz), float(dt), float(fc),
                                _want_gradient(want_gradient, density),
                                int(shot_group), float(mem_budget_gb), int(kernel_variant),
                                int(ckpt_interval))
        h = ct.c_void_p()
        st = self.lib.stfwi_create(ct.byref(self.desc), ct.byref(h))
        if st == N.STFWI_ERR_UNSUPPORTED:
            raise NotImplementedError(f"stfwi_create: unsupported configuration {self.shape_desc()}")
        if st == N.STFWI_ERR_INVALID:
            raise ValueError(f"stfwi_create: invalid descriptor {self.shape_desc()}")
        if st != N.STFWI_OK:
            raise N.StfwiError(st, f"stfwi_create failed for {self.shape_desc()}")
        self.h = h
        self.nz_dom, self.nx_dom, self.nt, self.nrec = int(nz_dom), int(nx_dom), int(nt), int(nrec)
        self.pad, self.free_surface, self.fd_order = int(pad), bool(free_surface), int(fd_order)
        nzt, nxt = ct.c_int32(), ct.c_int32()
        self.lib.stfwi_grid_shape(ct.byref(self.desc), ct.byref(nzt), ct.byref(nxt))
        self.nz, self.nx = nzt.value, nxt.value
        self.nshot = 0

    def shape_desc(self):
        d = self.desc
        return (f"grid {d.nz_dom}x{d.nx_dom} pad {d.pad} fd{d.fd_order} nt {d.nt} nrec {d.nrec} "
                f"shots {d.max_shots}")

    @staticmethod
    def workspace_bytes(**kw):
        lib = N.load()
        d = N.StfwiDesc(kw["nz_dom"], kw["nx_dom"], kw["pad"], kw.get("fd_order", 2),
                        int(kw.get("free_surface", True)), kw["nt"], kw["nrec"], kw["max_shots"],
                        kw["dx"], kw["dz"], kw["dt"], kw["fc"],
                        _want_gradient(kw.get("want_gradient", True), kw.get("density", False)),
                        kw.get("shot_group", 0), kw.get("mem_budget_gb", 0.0),
                        kw.get("kernel_variant", 0), kw.get("ckpt_interval", 0))
        return int(lib.stfwi_workspace_bytes(ct.byref(d)))

    # ------------------------------------------------------------------ helpers
    def _ok(self, st, what):
        if st != N.STFWI_OK:
            msg = self.lib.stfwi_last_error(self.h).decode()
            if st == N.STFWI_ERR_UNSUPPORTED:
                raise NotImplementedError(f"{what}: {msg}")
            if st == N.STFWI_ERR_INVALID:
                raise ValueError(f"{what}: {msg}")
            raise N.StfwiError(st, f"{what}: {msg}")

    def check(self):
        self._ok(self.lib.stfwi_check(self.h, _stream()), "stfwi_check")

    def close(self):
        if getattr(self, "h", None):
            self.lib.stfwi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ set-up
    def set_model(self, Vs, Vp, rho):
        for name, a in (("Vs", Vs), ("Vp", Vp), ("rho", rho)):
            if tuple(a.shape) != (self.nz_dom, self.nx_dom):
                raise ValueError(f"{name} has shape {tuple(a.shape)}, expected {(self.nz_dom, self.nx_dom)}")
        p1, k1 = _as_buffer(Vs, np.float32)
        p2, k2 = _as_buffer(Vp, np.float32)
        p3, k3 = _as_buffer(rho, np.float32)
        self._ok(self.lib.stfwi_set_model(self.h, p1, p2, p3, _stream()), "set_model")
        self._model_keep = (k1, k2, k3)

    def set_receivers(self, rec_x, rec_z):
        rx = np.ascontiguousarray(np.asarray(rec_x, dtype=np.int32).reshape(-1))
        rz = np.ascontiguousarray(np.asarray(rec_z, dtype=np.int32).reshape(-1))
        if rx.size != self.nrec or rz.size != self.nrec:
            raise ValueError(f"expected {self.nrec} receivers, got {rx.size}/{rz.size}")
        self._ok(self.lib.stfwi_set_receivers(self.h, self.nrec, rx.ctypes.data, rz.ctypes.data),
                 "set_receivers")

    def set_shots(self, src_x, src_z, src_types, wavelets):
        sx = np.asarray(src_x, dtype=np.int64).reshape(-1)
        sz = np.asarray(src_z, dtype=np.int64).reshape(-1)
        if isinstance(src_types, str):
            src_types = [src_types] * sx.size
        try:
            ty = [SRC_TYPES[t] if isinstance(t, str) else int(t) for t in src_types]
        except KeyError as e:
            raise NotImplementedError(f"src_type={e.args[0]!r} not supported (use 'force' or 'moment').")
        src = np.ascontiguousarray(np.stack([sx, sz, np.asarray(ty)], axis=1).astype(np.int32))
        w = wavelets
        if getattr(w, "ndim", 1) == 1:
            w = np.broadcast_to(np.asarray(w, dtype=np.float32), (sx.size, self.nt))
        if tuple(w.shape) != (sx.size, self.nt):
            raise ValueError(f"wavelets have shape {tuple(w.shape)}, expected {(sx.size, self.nt)}")
        pw, kw = _as_buffer(w, np.float32)
        self._ok(self.lib.stfwi_set_shots(self.h, int(sx.size), src.ctypes.data, pw, _stream()),
                 "set_shots")
        self._shots_keep = (src, kw)
        self.nshot = int(sx.size)

    # ------------------------------------------------------------------ passes
    def forward(self, store=False):
        self._ok(self.lib.stfwi_forward(self.h, N.FWD_STORE if store else 0, _stream()), "forward")

    def records(self, out=None):
        """[nshot, 4, nt, nrec] float32 receiver traces (vx, vz, exx, ezz)."""
        if out is None:
            out = np.empty((self.nshot, 4, self.nt, self.nrec), dtype=np.float32)
        p, keep = _as_buffer(out, np.float32) if not isinstance(out, np.ndarray) else (out.ctypes.data, out)
        self._ok(self.lib.stfwi_get_records(self.h, p, _stream()), "get_records")
        self.check()
        return keep if not isinstance(out, np.ndarray) else out

    def misfit(self, obs, component, scale=1.0, sos=None, n_taper=0, nshot_norm=0, out=None, sync=True):
        """Per-shot misfit terms (FP64) and, inside the handle, the adjoint
        sources.  ``out`` may be a device tensor of nshot float64."""
        po, ko = _as_buffer(obs, np.float32)
        sos_a = None if sos is None else np.ascontiguousarray(np.asarray(sos, dtype=np.float64))
        m = N.StfwiMisfitDesc(int(component), int(n_taper), 0 if sos_a is None else sos_a.shape[0],
                              int(nshot_norm), float(scale),
                              None if sos_a is None else sos_a.ctypes.data_as(ct.POINTER(ct.c_double)))
        if out is None:
            out = np.zeros(self.nshot, dtype=np.float64)
        ptr = out.ctypes.data if isinstance(out, np.ndarray) else out.data_ptr()
        self._ok(self.lib.stfwi_misfit(self.h, po, ct.byref(m), ptr, _stream()), "misfit")
        if sync:
            self.check()
        self._obs_keep = ko
        return out

    def set_adjoint_sources(self, rec_adj):
        p, keep = _as_buffer(rec_adj, np.float32)
        self._ok(self.lib.stfwi_set_adjoint_sources(self.h, p, _stream()), "set_adjoint_sources")
        self.check()
        del keep

    def gradient(self, exact=True, imaging=False, src=False, out=None, sync=True):
        """Adjoint sweep.  Returns a dict with 'exact' / 'imaging' ->
        (g_Vs, g_Vp, g_rho) FP64 arrays and 'src' -> [nshot, nt] float32.
        The exact g_rho is zero unless the solver was made with density=True;
        the imaging g_rho then includes the density (velocity) term.
        ``out`` may be a device tensor [n_modes, 3, nz_dom, nx_dom] float64."""
        mode = (N.GRAD_EXACT if exact else 0) | (N.GRAD_IMAGING if imaging else 0) | (N.GRAD_SRC if src else 0)
        nmat = int(exact) + int(imaging)
        g = out if out is not None else np.zeros((max(nmat, 1), 3, self.nz_dom, self.nx_dom), dtype=np.float64)
        gptr = g.ctypes.data if isinstance(g, np.ndarray) else g.data_ptr()
        sa = np.zeros((max(self.nshot, 1), self.nt), dtype=np.float32)
        self._ok(self.lib.stfwi_gradient(self.h, mode, gptr if nmat else None,
                                         sa.ctypes.data if src else None, _stream()), "gradient")
        if sync or src:
            self.check()
        out = {}
        k = 0
        if exact:
            out["exact"] = tuple(g[k]); k += 1
        if imaging:
            out["imaging"] = tuple(g[k]); k += 1
        if src:
            out["src"] = sa
        return out

    def _frames_buffer(self, nf):
        """Host buffer for [nshot, nf, nt, nz_t, nx_t] float32 frames: page-locked
        when torch can provide it (the per-step copies then run asynchronously)."""
        shape = (self.nshot, nf, self.nt, self.nz, self.nx)
        t = _torch()
        if t is not None and t.cuda.is_available():
            try:
                buf = t.empty(shape, dtype=t.float32, pin_memory=True)
                return buf.numpy(), buf
            except RuntimeError:
                pass
        a = np.empty(shape, dtype=np.float32)
        return a, a

    @staticmethod
    def _field_mask(fields):
        mask = 0
        for f in fields:
            if f not in N.FRAME_BITS:
                raise ValueError(f"unknown field {f!r}; use {sorted(N.FRAME_BITS)}")
            mask |= N.FRAME_BITS[f]
        return mask

    def forward_frames(self, fields=("vx", "vz", "ex", "ez", "es"), out=None):
        """Forward run that also returns full padded-grid wavefields: a dict
        field -> [nshot, nt, nz_t, nx_t] float32 (frame n = after step n), in
        the order of ``fields`` ('vx', 'vz', 'ex', 'ez', 'es').  The receiver
        traces of the run are available from ``records()`` as usual."""
        mask = self._field_mask(fields)
        order = [f for f in N.FRAME_BITS if mask & N.FRAME_BITS[f]]
        arr, keep = (out, out) if out is not None else self._frames_buffer(len(order))
        ptr = arr.ctypes.data if isinstance(arr, np.ndarray) else arr.data_ptr()
        self._ok(self.lib.stfwi_forward_frames(self.h, mask, ptr, _stream()), "forward_frames")
        self.check()
        return {f: arr[:, order.index(f)] for f in fields}, keep

    def adjoint_frames(self, fields=("vx", "vz", "ex", "ez", "es"), out=None):
        """Source-wavelet adjoint sweep that also returns the adjoint
        wavefields (U_a, V_a, ex_a, ez_a, es_a by the names 'vx' .. 'es'):
        ([nshot, nt] src_wav_a, dict field -> [nshot, nt, nz_t, nx_t]), frame n
        = the carry out of adjoint step n, in forward-time order."""
        mask = self._field_mask(fields)
        order = [f for f in N.FRAME_BITS if mask & N.FRAME_BITS[f]]
        arr, keep = (out, out) if out is not None else self._frames_buffer(len(order))
        ptr = arr.ctypes.data if isinstance(arr, np.ndarray) else arr.data_ptr()
        sa = np.zeros((max(self.nshot, 1), self.nt), dtype=np.float32)
        self._ok(self.lib.stfwi_adjoint_frames(self.h, mask, ptr, sa.ctypes.data, _stream()), "adjoint_frames")
        self.check()
        return sa, {f: arr[:, order.index(f)] for f in fields}, keep

    def set_wait_limit(self, polls=-1):
        """Polls of a tile-copy wait before a kernel gives up with
        STFWI_ERR_TIMEOUT (-1: the default; 0: every wait gives up at once)."""
        self._ok(self.lib.stfwi_set_wait_limit(self.h, int(polls)), "set_wait_limit")

    KERNELS = ("fwd_vel", "fwd_str", "adj_a", "adj_b")

    def profile(self, every):
        """Sample a CUDA-event pair around each kernel of every `every`-th step."""
        self._ok(self.lib.stfwi_profile(self.h, int(every)), "profile")

    def kernel_times(self):
        """{kernel: (total ms, launches)} of the sampled launches since the last call."""
        out = np.zeros(8, dtype=np.float64)
        self._ok(self.lib.stfwi_kernel_times(self.h, out.ctypes.data), "kernel_times")
        return {k: (float(out[2 * i]), int(out[2 * i + 1])) for i, k in enumerate(self.KERNELS)}

    def autotune(self, steps=20):
        """Pick the tile shapes and the shots per block of each stencil kernel
        by timing `steps` forward and adjoint steps per candidate; returns
        {kernel: shots per block} (``tile_rows()`` gives the shapes).
        Overwrites the state: call before the forward of a gradient."""
        out = np.zeros(4, dtype=np.int32)
        self._ok(self.lib.stfwi_autotune(self.h, int(steps), out.ctypes.data, _stream()), "autotune")
        return dict(zip(self.KERNELS, (int(v) for v in out)))

    def tile_rows(self):
        """(rows of the fwd_vel/fwd_str/adj_a tiles, rows of the adj_b tiles); tiles are 64 columns wide."""
        out = np.zeros(2, dtype=np.int32)
        self._ok(self.lib.stfwi_tile_rows(self.h, out.ctypes.data), "tile_rows")
        return int(out[0]), int(out[1])

    def set_chains(self, chains):
        """Chains (1-4) a pass may be split into over the shot groups; see stfwi_set_chains."""
        self._ok(self.lib.stfwi_set_chains(self.h, int(chains)), "set_chains")

    def set_tile_rows(self, rows_a, rows_b):
        """Tile heights (8 or 16 rows) of fwd_vel/fwd_str/adj_a and of adj_b."""
        self._ok(self.lib.stfwi_set_tile_rows(self.h, int(rows_a), int(rows_b)), "set_tile_rows")

    def set_postprocess(self, grad_smooth_sigma=None, source_taper=None, illumination=None):
        """Post-processing applied on the device to the gradients that
        ``gradient()`` returns (fwi/gradient.py:266-277): Gaussian smoothing,
        then the source-taper and illumination products.  None disables a
        part; the setting stays for later calls."""
        shp = (self.nz_dom, self.nx_dom)
        keep = []
        ptrs = []
        for a in (source_taper, illumination):
            if a is None:
                ptrs.append(None)
                continue
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), shp))
            keep.append(a)
            ptrs.append(a.ctypes.data)
        sigma = 0.0 if grad_smooth_sigma is None else float(grad_smooth_sigma)
        self._ok(self.lib.stfwi_set_postprocess(self.h, sigma, ptrs[0], ptrs[1], _stream()), "set_postprocess")

    def preconditioner(self, kind="illum", component=1, eps=1e-3):
        """[nz_dom, nx_dom] FP64 gradient multiplier in [0, 1] from the forward
        energy of the current model and shots: 'illum' (1 / (Ws + eps max Ws),
        fwi/illumination.py:18-48) or 'eprecond3' (fwi/preconditioning.py)."""
        k = {"illum": N.PRECOND_ILLUM, "eprecond3": N.PRECOND_EPRECOND3}.get(kind)
        if k is None:
            raise ValueError(f"unknown precon={kind!r}; use 'illum' or 'eprecond3'")
        out = np.zeros((self.nz_dom, self.nx_dom), dtype=np.float64)
        self._ok(self.lib.stfwi_preconditioner(self.h, k, int(component), float(eps), out.ctypes.data, _stream()),
                 "preconditioner")
        self.check()
        return out

    def illumination(self, component):
        """Sum over shots and steps of field**2 on the padded grid (FP64)."""
        ws = np.zeros((self.nz, self.nx), dtype=np.float64)
        self._ok(self.lib.stfwi_illumination(self.h, int(component), ws.ctypes.data, _stream()),
                 "illumination")
        self.check()
        return ws


def imaging_condition_device(Vs, Vp, rho, ex_hist, ez_hist, es_hist, U_a_hist, V_a_hist, dx, dz, dt, pad,
                             free_surface, nz_dom, nx_dom, vx_hist=None, vz_hist=None, time_chunk=64):
    """fwi/imaging.py:83-169 through stfwi_imaging_condition: histories
    [nt, nz_t, nx_t] (NumPy or torch, host or CUDA; cast to float32), FP64
    time sums on the GPU.  Returns six [nz_dom, nx_dom] FP64 arrays (g_Vs,
    g_Vp, g_rho, g_lam, g_mu, g_rho_lame)."""
    lib = N.load()
    if (vx_hist is None) != (vz_hist is None):
        raise ValueError("give both vx_hist and vz_hist, or neither")
    nt = int(U_a_hist.shape[0])
    nz_t = nz_dom + pad if free_surface else nz_dom + 2 * pad
    for name, h in (("ex_hist", ex_hist), ("ez_hist", ez_hist), ("es_hist", es_hist), ("U_a_hist", U_a_hist),
                    ("V_a_hist", V_a_hist), ("vx_hist", vx_hist), ("vz_hist", vz_hist)):
        if h is not None and tuple(h.shape) != (nt, nz_t, nx_dom + 2 * pad):
            raise ValueError(f"{name} has shape {tuple(h.shape)}, expected {(nt, nz_t, nx_dom + 2 * pad)}")
    bufs = [_as_buffer(a, np.float32) for a in (Vs, Vp, rho, ex_hist, ez_hist, es_hist, U_a_hist, V_a_hist)]
    vel = [(None, None) if a is None else _as_buffer(a, np.float32) for a in (vx_hist, vz_hist)]
    d = N.StfwiImagingDesc(int(nz_dom), int(nx_dom), int(pad), int(bool(free_surface)), nt, int(time_chunk),
                           float(dx), float(dz), float(dt))
    g = np.zeros((6, nz_dom, nx_dom), dtype=np.float64)
    st = lib.stfwi_imaging_condition(ct.byref(d), *[b[0] for b in bufs], vel[0][0], vel[1][0], g.ctypes.data,
                                     _stream())
    if st == N.STFWI_ERR_INVALID:
        raise ValueError("stfwi_imaging_condition: invalid arguments (see stderr)")
    if st != N.STFWI_OK:
        raise N.StfwiError(st, "stfwi_imaging_condition failed (see stderr)")
    t = _torch()
    if t is not None and t.cuda.is_available() and t.cuda.is_initialized():
        t.cuda.current_stream().synchronize()
    del bufs, vel
    return tuple(g)


def project_velocity_device(Vs, Vp, rho, K_margin=0.04, vp_cap=None, vs_floor=1e-3, rho_floor=1e-3):
    """fwi/projections.py:67-117 in place on CUDA float64 tensors (torch)."""
    import torch
    for name, t in (("Vs", Vs), ("Vp", Vp), ("rho", rho)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous CUDA float64 tensor")
    n = Vs.numel()
    if Vp.numel() != n or rho.numel() != n:
        raise ValueError("Vs, Vp and rho differ in size")
    lib = N.load()
    cap = -1.0 if vp_cap is None else float(vp_cap)
    st = lib.stfwi_project_velocity(n, Vs.data_ptr(), Vp.data_ptr(), rho.data_ptr(), float(K_margin), cap,
                                    float(vs_floor), float(rho_floor), _stream())
    if st != N.STFWI_OK:
        raise N.StfwiError(st, "stfwi_project_velocity failed")
    return Vs, Vp, rho
