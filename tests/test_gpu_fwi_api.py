"""The reference-signature API (stfwi_b200.fwi) on the GPU against the oracle
and against the reference's stored results (B200)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _small_case(fs=True, fd=8, nt=150):
    vs, vp, rho = C.model()
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.zeros_like(rx) if fs else np.full_like(rx, 3)
    sx, sz = np.array([5, 16, 27]), np.array([1, 4, 2])
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=nt, fc=C.FC,
               pad=C.PAD, fd_order=fd, free_surface=fs)
    return vs, vp, rho, sx, sz, wav, geo


@pytest.mark.parametrize("invert", ["vs_vp", "all"])
@pytest.mark.parametrize("backend,ref", [("cuda", "ad"), ("cuda_imaging", "adjoint")])
def test_compute_gradient_matches_oracle(backend, ref, invert):
    from scipy.signal import butter
    from stfwi_b200 import fwi
    vs, vp, rho, sx, sz, wav, geo = _small_case()
    types = ["force", "moment", "force"]
    obs = O.forward_batch(vs * 1.02, vp, rho, sx, sz, types, src_wavelet=wav, d0_f32=True, **geo)[:, 1]
    sos = butter(6, 40.0, fs=1.0 / C.DT, output="sos")
    zz, xx = np.meshgrid(np.arange(C.NZ), np.arange(C.NX), indexing="ij")
    illum = 0.5 + 0.5 * np.cos(np.pi * zz / C.NZ) ** 2
    taper = np.clip(xx / 5.0, 0, 1)
    kw = dict(Vs=vs, Vp=vp, rho=rho, src_x=sx, src_z=sz, src_wavelet=wav, observed=obs, component=1,
              invert=invert, scale=3.0, sos=sos, n_taper=15, grad_smooth_sigma=1.0, source_taper=taper,
              illumination=illum, src_types=types, **geo)
    (g_vs, g_vp, g_rho), loss = fwi.compute_gradient(backend, **kw)
    (r_vs, r_vp, r_rho), r_loss = O.compute_gradient(ref, d0_f32=True, **kw)
    rec = O.forward_batch(vs, vp, rho, sx, sz, types, src_wavelet=wav, d0_f32=True, **geo)[:, 1]
    amp = float(np.linalg.norm(rec) / np.linalg.norm(rec - obs))
    tol = 2e-5 * max(amp, 1.0)
    errs = (abs(loss / r_loss - 1), _rel(g_vs, r_vs), _rel(g_vp, r_vp))
    assert max(errs) < tol, (errs, tol)
    if invert == "all":
        assert _rel(g_rho, r_rho) < tol, (_rel(g_rho, r_rho), tol)
    else:
        assert np.all(g_rho == 0)


def test_forward_and_adjoint_signatures_match_oracle():
    from stfwi_b200 import fwi
    vs, vp, rho = C.model()
    sx, sz, rx, rz = C.acquisition(False, "moment")
    s_in, ys = C.random_vectors()
    rec = fwi.forward_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in,
                          fd_order=4, free_surface=False, src_type="moment")
    ref, _, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in,
                          4, False, "moment", d0_f32=True)
    assert len(rec) == 4 and rec[0].shape == (C.NT, len(rx))
    assert max(_rel(a, b) for a, b in zip(rec, ref)) < 1e-5
    sa = fwi.adjoint_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                         fd_order=4, free_surface=False, src_type="moment")
    ra = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                   fd_order=4, free_surface=False, src_type="moment", d0_f32=True)["src"]
    assert _rel(sa, ra) < 1e-5
    run_shot = fwi.build_forward_fn(C.NZ, C.NX, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, 100, rx, rz, fd_order=8,
                                    return_vars=["vz", "ex"], free_surface=True)
    vz, ex = run_shot(vs, vp, rho, sx, 0, s_in)
    ref, _, _ = O.forward(vs, vp, rho, sx, 0, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in, 8,
                          True, "force", d0_f32=True)
    assert _rel(vz, ref[1]) < 1e-5 and _rel(ex, ref[2]) < 1e-5
    with pytest.raises(ValueError):
        fwi.build_forward_fn(C.NZ, C.NX, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, 100, rx, rz, return_vars=["vy_full"])
    with pytest.raises(NotImplementedError):
        fwi.adjoint_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                        fd_order=6)
    with pytest.raises(ValueError):
        fwi.compute_gradient("jax", Vs=vs, Vp=vp, rho=rho, src_x=[sx], src_z=[sz], src_wavelet=s_in,
                             observed=np.zeros((1, C.NT, len(rx))), rec_x=rx, rec_z=rz, nx_dom=C.NX,
                             nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=C.NT, fc=C.FC, pad=C.PAD)


def test_illumination_matches_oracle():
    from stfwi_b200 import fwi
    vs, vp, rho, sx, sz, wav, geo = _small_case(nt=100)
    for comp in (0, 2):
        H, Ws = fwi.compute_illumination_for_stage(C.NZ, C.NX, C.DX, C.DZ, C.DT, 100, C.FC, C.PAD, 100,
                                                   geo["rec_x"], geo["rec_z"], 8, comp, vs, vp, rho, sx, sz,
                                                   wav, eps=1e-3, return_ws=True)
        Hr, Wr = O.compute_illumination(C.NZ, C.NX, C.DX, C.DZ, C.DT, 100, C.FC, C.PAD, geo["rec_x"],
                                        geo["rec_z"], 8, comp, vs, vp, rho, sx, sz, wav, eps=1e-3, d0_f32=True)
        assert _rel(Ws, Wr) < 1e-5 and _rel(H, Hr) < 1e-5


def test_build_loss_fn_is_value_and_grad():
    from stfwi_b200 import fwi
    vs, vp, rho, sx, sz, wav, geo = _small_case(nt=120)
    run_shot = fwi.build_forward_fn(C.NZ, C.NX, C.DX, C.DZ, C.DT, 120, C.FC, C.PAD, 60, geo["rec_x"],
                                    geo["rec_z"], fd_order=8, free_surface=True)
    obs = np.stack([run_shot(vs * 1.03, vp, rho, s, sz[0], wav)[1] for s in sx])
    loss_fn = fwi.build_loss_fn(run_shot, obs, sx, sz, wav, component=1, scale=1.0, invert="vs",
                                tikhonov_alpha=1e-3)
    loss, (g_vs, g_vp, g_rho) = loss_fn((vs, vp, rho))
    (r_vs, _, _), r_loss = O.compute_gradient("ad", Vs=vs, Vp=vp, rho=rho, src_x=sx, src_z=np.full(3, sz[0]),
                                              src_wavelet=wav, observed=obs, component=1, scale=1.0,
                                              d0_f32=True, **geo)
    d0, d1 = np.diff(vs.astype(np.float64), axis=0), np.diff(vs.astype(np.float64), axis=1)
    reg = np.sum(d0 ** 2) + np.sum(d1 ** 2)
    assert abs(loss / (r_loss * (1 + 1e-3)) - 1) < 1e-4
    assert np.all(g_vp == 0) and np.all(g_rho == 0)
    # the Tikhonov term adds alpha * (loss/reg) * d(reg)/dVs
    greg = np.zeros_like(d0, shape=vs.shape)
    greg[1:] += 2 * d0; greg[:-1] -= 2 * d0; greg[:, 1:] += 2 * d1; greg[:, :-1] -= 2 * d1
    assert _rel(g_vs, r_vs + 1e-3 * (r_loss / reg) * greg) < 1e-3


def test_reference_first_gradient_34_shots(known_answers):
    """Results_first_gradient/first_gradient.npz (compute_first_gradient.py):
    34 shots x 2890 steps, fd8, free surface, exx misfit after a 3 Hz
    Butterworth and a 10 % taper, sigma=1 smoothing.  FP32 GPU against the
    reference's FP64 loss_AD and its two preconditioned gradients."""
    from scipy.signal import butter
    from stfwi_b200 import fwi
    K = known_answers
    nt, dt, fc = int(K["fg_nt"]), float(K["fg_dt"]), float(K["fg_f_c"])
    nz, nx = K["Vs_true"].shape
    rx, rz, sx, sz = K["fg_rec_x"], K["fg_rec_z"], K["fg_src_x"], K["fg_src_z"]
    wav = fwi.ricker_jax(np.arange(nt) * dt, fc, 1.5 / fc)
    run_obs = fwi.build_forward_fn(nz, nx, 20.0, 20.0, dt, nt, fc, 30, 200, rx, rz, fd_order=8, free_surface=True)
    observed = run_obs.batch(K["Vs_true"], K["Vp_true"], K["rho_true"], sx, sz, wav)[2]
    auto = float(1.0 / (np.mean(observed.astype(np.float64) ** 2) + 1e-45))
    sos = butter(6, float(K["fg_cutoff"]), fs=1.0 / dt, output="sos")
    common = dict(Vs=K["Vs_init"], Vp=K["Vp_init"], rho=K["rho_init"], src_x=sx, src_z=sz, src_wavelet=wav,
                  observed=observed, rec_x=rx, rec_z=rz, nx_dom=nx, nz_dom=nz, dx=20.0, dz=20.0, dt=dt, nt=nt,
                  fc=fc, pad=30, component=2, invert="vs", scale=auto, sos=sos, n_taper=int(0.1 * nt),
                  fd_order=8, free_surface=True, grad_smooth_sigma=1.0)
    H_inv = fwi.compute_illumination_for_stage(nz, nx, 20.0, 20.0, dt, nt, fc, 30, 200, rx, rz, 8, 2,
                                               K["Vs_init"], K["Vp_init"], K["rho_init"], sx, sz, wav,
                                               eps=float(K["fg_illumination_eps"]))
    (g_ad, _, _), loss = fwi.compute_gradient("cuda", illumination=H_inv, **common)
    (g_hc, _, _), loss_hc = fwi.compute_gradient("cuda_imaging", illumination=K["fg_illumination_eprecond3"],
                                                 **common)
    e = {"auto_scale": abs(auto / K["fg_auto_scale"] - 1), "loss_AD": abs(loss / K["fg_loss_AD"] - 1),
         "loss_HC": abs(loss_hc / K["fg_loss_HC"] - 1), "g_Vs_AD": _rel(g_ad, K["fg_g_Vs_AD"]),
         "g_Vs_HC": _rel(g_hc, K["fg_g_Vs_HC"])}
    print("first gradient (34 shots x 2890 steps):", {k: f"{v:.2e}" for k, v in e.items()})
    # measured on a B200: auto_scale 2.8e-7, losses 7.5e-7 / 1.6e-7, g_Vs_HC
    # 6.9e-7 (FP32 stencils against the reference's FP64 run); bounds about 3x
    assert e["auto_scale"] < 1e-6 and e["loss_AD"] < 3e-6 and e["loss_HC"] < 1e-6
    assert e["g_Vs_HC"] < 2e-6
    # g_Vs_AD was scaled by an illumination multiplier that the reference did
    # not store; ours is rebuilt from its recipe (1.3e-3 measured), so this
    # comparison carries that reconstruction, not the kernels' error
    assert e["g_Vs_AD"] < 3e-3
