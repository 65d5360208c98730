"""The oracle pinned against the reference's own tests and known answers (CPU)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C


@pytest.mark.parametrize("fd,fs,st", C.CONFIGS)
def test_dot_product_adjoint(fd, fs, st):
    """test_adjoint_kernel.py:61-114 in FP64: <L s, y> == <s, L^T y>."""
    vs, vp, rho = C.model()
    sx, sz, rx, rz = C.acquisition(fs, st)
    s_in, ys = C.random_vectors()
    rec, _, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC,
                          C.PAD, s_in, fd, fs, st)
    a = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                  fd_order=fd, free_surface=fs, src_type=st)
    lhs = sum(float(np.sum(r * y)) for r, y in zip(rec, ys))
    rhs = float(np.sum(s_in * a["src"]))
    rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300)
    assert rel < 1e-12, (lhs, rhs, rel)


def test_unsupported_config_raises():
    vs, vp, rho = C.model()
    with pytest.raises(NotImplementedError):
        O.forward(vs, vp, rho, 5, 5, [1], [1], C.NX, C.NZ, C.DX, C.DZ, C.DT, 4, C.FC, C.PAD,
                  np.zeros(4), 6, True, "force")
    with pytest.raises(NotImplementedError):
        O.adjoint(vs, vp, rho, 5, 5, [1], [1], C.NX, C.NZ, C.DX, C.DZ, C.DT, 4, C.FC, C.PAD,
                  *[np.zeros((4, 1))] * 4, fd_order=4, src_type="dipole")


def test_pml_profiles_interior_identity():
    """_pml_coefficients: k=1, b=1, a=0 outside the strips (psi stays 0)."""
    vs, vp, rho = C.model()
    kx, kz, bx, bz, ax, az = O.pml_profiles(C.NZ, C.NX, C.PAD, True, C.DX, C.DT, C.FC, vp)
    inner = (slice(0, C.NZ), slice(C.PAD, C.PAD + C.NX))
    assert np.all(kx[inner] == 1) and np.all(bx[inner] == 1) and np.all(ax[inner] == 0)
    assert np.all(kz[inner] == 1) and np.all(bz[inner] == 1) and np.all(az[inner] == 0)
    # strips: the profile depends on the column (x) / row (z) only
    assert np.all(bx == bx[0:1, :]) and np.all(bz == bz[:, 0:1])


def test_sosfilt_transpose_is_adjoint():
    from scipy.signal import butter
    rng = np.random.default_rng(3)
    sos = butter(6, 3.0, fs=1 / 0.002, output="sos")
    x = rng.standard_normal((300, 5))
    y = rng.standard_normal((300, 5))
    lhs = np.sum(O.sosfilt(x, sos) * y)
    rhs = np.sum(x * O.sosfilt_T(y, sos))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_cotangent_matches_finite_difference():
    """The receiver cotangent is d(misfit)/d(pred) with filter + taper."""
    from scipy.signal import butter
    rng = np.random.default_rng(4)
    sos = butter(6, 5.0, fs=1 / 0.002, output="sos")
    pred = rng.standard_normal((200, 3))
    obs = rng.standard_normal((200, 3))
    _, g = O.shot_misfit_and_cotangent(pred, obs, sos, 20, 3.0, 2)
    d = rng.standard_normal(pred.shape)
    h = 1e-6
    fp, _ = O.shot_misfit_and_cotangent(pred + h * d, obs, sos, 20, 3.0, 2)
    fm, _ = O.shot_misfit_and_cotangent(pred - h * d, obs, sos, 20, 3.0, 2)
    assert abs((fp - fm) / (2 * h) - np.sum(g * d)) < 1e-7 * abs(np.sum(g * d))


def _edge_free_perturbation(phase=0.3):
    """A smooth field that is zero on the domain edges the reference copies
    into the PML (those copies are stop-gradient, fwi/forward.py:217-219)."""
    zz, xx = np.meshgrid(np.arange(C.NZ), np.arange(C.NX), indexing="ij")
    return (np.sin(np.pi * zz / (C.NZ - 1)) * np.sin(np.pi * xx / (C.NX - 1))
            * (1.0 + 0.5 * np.cos(2 * np.pi * xx / C.NX + phase)))


def _fd_check(param, fs, st, fd_order, comp, rel_tol=1e-6):
    vs, vp, rho = C.model()
    nt = 120
    sx, sz, rx, rz = C.acquisition(fs, st)
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=nt,
               fc=C.FC, pad=C.PAD, fd_order=fd_order, free_surface=fs)
    obs = O.forward_batch(vs * 1.03, vp * 0.99, rho * 1.01, [sx], [sz], [st], src_wavelet=wav,
                          **geo)[:, comp]
    pert = _edge_free_perturbation()
    model = {"vs": vs, "vp": vp, "rho": rho}
    amp = {"vs": 40.0, "vp": 30.0, "rho": 20.0}[param]
    d = amp * pert
    if param == "vp":
        # Vp_max is stop-gradient: keep max(Vp) unchanged (it is attained
        # at more than one cell of this model)
        d[vp > vp.max() - 1.0] = 0.0
    kw = dict(src_x=[sx], src_z=[sz], src_wavelet=wav, observed=obs, src_types=[st],
              component=comp, scale=1.0, invert="all", **geo)
    g = O.compute_gradient("ad", Vs=vs, Vp=vp, rho=rho, **kw)[0][("vs", "vp", "rho").index(param)]
    h = 1e-3
    vals = []
    for sgn in (1, -1):
        m = dict(model)
        m[param] = model[param] + sgn * h * d
        vals.append(O.compute_gradient("ad", Vs=m["vs"], Vp=m["vp"], rho=m["rho"], **kw)[1])
    fd = (vals[0] - vals[1]) / (2 * h)
    an = float(np.sum(g * d))
    assert abs(fd - an) < rel_tol * abs(an), (param, fd, an)


@pytest.mark.parametrize("fs,st,fd", [(True, "force", 8), (True, "moment", 8), (False, "force", 4),
                                      (False, "moment", 2)])
def test_exact_gradient_vs_finite_difference(fs, st, fd):
    """Central differences of the FP64 misfit along a smooth Vs perturbation
    agree with the exact model gradient (incl. the free-surface ratio and the
    moment-source factor, both of which depend on Vs)."""
    _fd_check("vs", fs, st, fd, comp=0)


@pytest.mark.parametrize("param", ["vp", "rho"])
def test_exact_gradient_vp_rho_finite_difference(param):
    """The Vp and rho chains (invert='all'), incl. the buoyancy term."""
    _fd_check(param, True, "force", 4, comp=1)


@pytest.mark.parametrize("ckpt", [7, 100])
def test_imaging_density_term_matches_history_formula(ckpt):
    """The density term of the imaging condition (third imaging plane) is
    fwi/imaging.py:145-154 applied to the forward velocity history and the
    adjoint velocity history, also when the recompute runs in checkpoint
    segments that do not divide nt."""
    vs, vp, rho = C.model()
    nt, fs, st, fd = 40, True, "force", 4
    sx, sz, rx, rz = C.acquisition(fs, st)
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    rng = np.random.default_rng(8)
    ys = [rng.standard_normal((nt, len(rx))) for _ in range(4)]
    _, full, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD,
                           wav, fd, fs, st, full=("vx", "vz"))
    a = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, *ys,
                  fd_order=fd, free_surface=fs, src_type=st, src_wavelet=wav, want=("img",),
                  hist=("U_a", "V_a"), ckpt=ckpt)
    vx, vz, ua, va = full["vx"], full["vz"], a["U_a"], a["V_a"]
    ref = np.zeros_like(vx[0])
    for n in range(1, nt - 1):
        ref -= C.DT * (vx[n] * (ua[n + 1] - ua[n - 1]) + vz[n] * (va[n + 1] - va[n - 1])) / (2 * C.DT)
    assert np.abs(ref).max() > 0
    np.testing.assert_allclose(a["img"][2], ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.slow
def test_known_answers_gradient_compare(known_answers):
    """Results_gradient/gradient_compare.npz (compute_gradient_handcoded.py):
    FP64 auto_scale, loss_AD, the exact gradient g_Vs_AD (JAX AD) and the
    imaging gradient g_Vs_HC."""
    K = known_answers
    nt, pad, fd = int(K["gc_nt"]), int(K["gc_pad"]), int(K["gc_fd_order"])
    dt, fc, comp = float(K["gc_dt"]), float(K["gc_f_c"]), int(K["gc_component"])
    nz, nx = K["Vs_true"].shape
    wav = O.ricker(np.arange(nt) * dt, fc, 1.5 / fc)
    geo = dict(rec_x=K["gc_rec_x"], rec_z=K["gc_rec_z"], nx_dom=nx, nz_dom=nz, dx=20.0, dz=20.0,
               dt=dt, nt=nt, fc=fc, pad=pad, fd_order=fd, free_surface=True)
    ns = len(K["gc_src_x"])
    obs = O.forward_batch(K["Vs_true"], K["Vp_true"], K["rho_true"], K["gc_src_x"], K["gc_src_z"],
                          ["force"] * ns, src_wavelet=wav, **geo)[:, comp]
    auto = 1.0 / (np.mean(obs ** 2) + 1e-45)
    assert abs(auto / K["gc_auto_scale"] - 1) < 1e-10
    kw = dict(Vs=K["Vs_init"], Vp=K["Vp_init"], rho=K["rho_init"], src_x=K["gc_src_x"],
              src_z=K["gc_src_z"], src_wavelet=wav, observed=obs, component=comp,
              scale=float(K["gc_auto_scale"]), **geo)
    (g_ad, _, _), loss = O.compute_gradient("ad", **kw)
    assert abs(loss / K["gc_loss_AD"] - 1) < 1e-10
    ref = K["gc_g_Vs_AD"].astype(np.float64)
    assert np.linalg.norm(g_ad - ref) / np.linalg.norm(ref) < 1e-7
    (g_hc, _, _), loss_hc = O.compute_gradient("adjoint", **kw)
    assert abs(loss_hc / K["gc_loss_HC"] - 1) < 1e-10
    ref = K["gc_g_Vs_HC"].astype(np.float64)
    assert np.linalg.norm(g_hc - ref) / np.linalg.norm(ref) < 1e-7


@pytest.mark.parametrize("fs", [True, False])
def test_history_imaging_formula_matches_fused_sums(fs):
    """oracle.imaging_condition (fwi/imaging.py:83-169 on full histories, with
    np.roll) against the imaging sums fused into the oracle's adjoint sweep:
    the two restatements of the same formula agree to FP64 rounding."""
    vs, vp, rho = C.model()
    nt, st, fd = 30, "moment", 8
    sx, sz, rx, rz = C.acquisition(fs, st)
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    rng = np.random.default_rng(5)
    ys = [rng.standard_normal((nt, len(rx))) for _ in range(4)]
    _, full, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, wav, fd, fs,
                           st, full=("vx", "vz", "ex", "ez", "es"))
    a = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, *ys, fd_order=fd,
                  free_surface=fs, src_type=st, src_wavelet=wav, want=("img",), hist=("U_a", "V_a"))
    g = O.imaging_condition(vs, vp, rho, full["ex"], full["ez"], full["es"], a["U_a"], a["V_a"], C.DX, C.DZ, C.DT,
                            C.PAD, fs, C.NZ, C.NX, vx_hist=full["vx"], vz_hist=full["vz"])
    for k, p in enumerate(a["img"]):
        ref = O.crop(p, C.PAD, fs, C.NZ, C.NX)
        np.testing.assert_allclose(g[3 + k], ref, rtol=0, atol=1e-11 * np.abs(ref).max())
