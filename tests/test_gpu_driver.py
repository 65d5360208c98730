"""The work around the gradient that runs on the device (projection,
post-processing, preconditioners) and the multiscale L-BFGS-B driver
(fwi/optim_lbfgsb.py) on the CUDA path, against the oracle and the
reference's stored preconditioner (B200)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_projection_on_the_device_is_bit_exact():
    """fwi/projections.py:67-117 in FP64 on the device gives the host's
    values bit for bit, with and without the CFL cap."""
    import torch
    from stfwi_b200.fwi import project_velocity_device
    rng = np.random.default_rng(2)
    vs = rng.uniform(-50.0, 3000.0, (37, 53))
    vp = rng.uniform(100.0, 5000.0, (37, 53))
    rho = rng.uniform(-5.0, 2600.0, (37, 53))
    for cap in (None, 3600.0):
        t = [torch.tensor(a, device="cuda") for a in (vs, vp, rho)]
        project_velocity_device(*t, K_margin=0.04, vp_cap=cap)
        ref = O.project_velocity(vs, vp, rho, K_margin=0.04, vp_cap=cap)
        for a, b in zip(t, ref):
            assert np.array_equal(a.cpu().numpy(), b)


def _solver_case(nt=120):
    from stfwi_b200 import Solver
    vs, vp, rho = C.model()
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.zeros_like(rx)
    sx, sz = np.array([5, 16, 27]), np.array([1, 4, 2])
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    S = Solver(C.NZ, C.NX, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, len(rx), 3, fd_order=8, free_surface=True,
               want_gradient=True)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, "force", wav)
    return S, rx, rz


def test_postprocess_on_the_device_matches_host_arithmetic():
    """Smoothing, taper and illumination products applied by stfwi_gradient
    equal the host post-processing (fwi/gradient.py:266-277) of the raw
    gradients of the same handle."""
    S, rx, rz = _solver_case()
    obs = np.random.default_rng(1).standard_normal((3, S.nt, len(rx))).astype(np.float32) * 1e-9
    zz, xx = np.meshgrid(np.arange(C.NZ), np.arange(C.NX), indexing="ij")
    taper = np.clip(xx / 7.0, 0, 1)
    illum = 0.3 + 0.7 * np.cos(np.pi * zz / (2 * C.NZ))
    S.forward(store=True)
    S.misfit(obs, 1, 1.0)
    raw = S.gradient(exact=True, imaging=True)
    for sigma in (1.0, 2.5):
        S.set_postprocess(sigma, taper, illum)
        got = S.gradient(exact=True, imaging=True)
        for k in ("exact", "imaging"):
            for a, b in zip(got[k], raw[k]):
                ref = O.gaussian_smooth_2d(b, sigma) * taper * illum
                assert _rel(a, ref) < 1e-12, (k, sigma, _rel(a, ref))
    S.set_postprocess(None, None, None)
    again = S.gradient(exact=True)
    assert _rel(again["exact"][0], raw["exact"][0]) == 0.0
    S.close()


@pytest.mark.parametrize("kind", ["illum", "eprecond3"])
def test_preconditioners_match_host_formulas(kind):
    """The device preconditioners from the handle's forward energy equal the
    reference's host formulas applied to the same energy."""
    S, rx, rz = _solver_case()
    Ws = S.illumination(2)
    got = S.preconditioner(kind, 2, 5e-3)
    if kind == "illum":
        ref = O.illumination_inverse(Ws, C.NZ, C.NX, C.PAD, 5e-3)
    else:
        ref = O.eprecond3_multiplier(Ws, rx, rz, C.DX, C.DZ, True, C.PAD, C.NZ, C.NX, 5e-3)
    assert abs(got.max() - 1.0) < 1e-15
    assert _rel(got, ref) < 1e-12, _rel(got, ref)
    S.close()


def test_eprecond3_matches_the_reference_first_gradient(known_answers):
    """Results_first_gradient/first_gradient.npz stores the eprecond3
    multiplier the reference used (34 force shots x 2890 steps on the initial
    Marmousi model, exx energy, free surface): the device preconditioner
    from the FP32 forward energy matches it."""
    from stfwi_b200 import Solver, fwi
    K = known_answers
    nt, dt, fc = int(K["fg_nt"]), float(K["fg_dt"]), float(K["fg_f_c"])
    nz, nx = K["Vs_true"].shape
    rx, rz, sx, sz = K["fg_rec_x"], K["fg_rec_z"], K["fg_src_x"], K["fg_src_z"]
    wav = fwi.ricker_jax(np.arange(nt) * dt, fc, 1.5 / fc)
    S = Solver(nz, nx, 20.0, 20.0, dt, nt, fc, 30, len(rx), len(sx), fd_order=8, free_surface=True,
               want_gradient=False)
    S.set_model(K["Vs_init"], K["Vp_init"], K["rho_init"])
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, "force", np.asarray(wav, dtype=np.float32))
    got = S.preconditioner("eprecond3", 2, float(K["fg_illumination_eps"]))
    S.close()
    err = _rel(got, K["fg_illumination_eprecond3"])
    print(f"eprecond3 vs the reference's stored multiplier: rel-L2 {err:.2e}")
    assert err < 1e-4, err


def test_multiscale_driver_matches_oracle_driven_run(monkeypatch):
    """fwi.run_multiscale_fwi on the device (projection, gradient,
    post-processing, preconditioner) against the same L-BFGS-B loop fed
    with FP64 oracle gradients and host projections: two stages (Vs, then
    Vs + Vp with an illumination preconditioner and smoothing) give the same
    loss histories to FP32 accuracy and the misfit drops."""
    from stfwi_b200 import fwi
    from stfwi_b200.fwi import optim_lbfgsb as D
    vs_t, vp_t, rho = C.model()
    nt = 150
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.zeros_like(rx)
    sx, sz = np.array([5, 16, 27]), np.array([1, 1, 1])
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=nt, pad=C.PAD,
               fd_order=8, free_surface=True)
    wav = O.ricker(np.arange(nt) * C.DT, 20.0, 1.5 / 20.0)
    obs = O.forward_batch(vs_t, vp_t, rho, sx, sz, ["force"] * 3, src_wavelet=wav, fc=20.0, d0_f32=True,
                          **geo)[:, 2]
    vs0, vp0 = np.full_like(vs_t, vs_t.mean()), np.full_like(vp_t, vp_t.mean())
    stages = [dict(f_c=20.0, cutoff=30.0, n_iters=3, invert="vs", n_taper_pct=0.1),
              dict(f_c=20.0, cutoff=None, n_iters=3, invert="vs_vp", illumination_eps=1e-2,
                   grad_smooth_sigma=1.0)]
    kw = dict(Vs_init=vs0, Vp_init=vp0, rho_init=rho, src_x=sx, src_z=sz, observed=obs, stages=stages,
              component=2, backend="ad", K_margin=0.04, verbose=False, **geo)
    _, h_gpu = fwi.run_multiscale_fwi(**kw)

    def oracle_gradient(backend, **a):
        a = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in a.items()}
        a.pop("block_size", None)
        return O.compute_gradient("ad", d0_f32=True, **a)

    def host_project(self, model):   # the oracle's projection on the host, written back
        import torch
        p = O.project_velocity(*(a.cpu().numpy() for a in model), K_margin=self.K_margin, vp_cap=self.vp_cap)
        model.copy_(torch.as_tensor(np.stack(p), device=model.device))
        return model

    def oracle_illum(nz, nx, dx, dz, dt, nt_, f_c, pad, block_size, rec_x, rec_z, fd_order, component, Vs, Vp,
                     rho_, src_x, src_z, src_wavelet, eps):
        ws = np.zeros((nz + pad, nx + 2 * pad))
        for k in range(len(src_x)):
            _, _, e = O.forward(Vs, Vp, rho_, src_x[k], src_z[k], rec_x, rec_z, nx, nz, dx, dz, dt, nt_, f_c, pad,
                                src_wavelet, fd_order, True, "force", energy=("ex",), d0_f32=True)
            ws += e["ex"]
        return O.illumination_inverse(ws, nz, nx, pad, eps)

    monkeypatch.setattr(D, "compute_gradient", oracle_gradient)
    monkeypatch.setattr(D.MultiscaleDriver, "_project", host_project)
    monkeypatch.setattr(D, "compute_illumination_for_stage", oracle_illum)
    _, h_ref = fwi.run_multiscale_fwi(**kw)
    for a, b in zip(h_gpu, h_ref):
        la, lb = a["loss_history"], b["loss_history"]
        n = min(len(la), len(lb))
        assert n >= 3
        err = np.max(np.abs(la[:n] / lb[:n] - 1))
        print(f"stage {a['stage']}: {n} evaluations, loss rel diff {err:.2e}, {la[0]:.4e} -> {la[n - 1]:.4e}")
        assert err < 1e-3, err
    assert h_gpu[-1]["loss_history"].min() < 0.9 * h_gpu[0]["loss_history"][0]


def test_uneven_batch_equals_models_run_alone():
    """Two grids of different size and step count, their launches
    interleaved on two streams (stfwi_b200.batch.UnevenBatch), give each
    model's own misfit and gradient."""
    import torch
    from stfwi_b200 import Solver
    from stfwi_b200 import models as Mo
    from stfwi_b200.batch import UnevenBatch
    specs = []
    for nz, nx, dx, nt, ns, fd in ((40, 90, 20.0, 120, 3, 4), (64, 150, 10.0, 200, 4, 8)):
        vs, vp, rho = Mo.layered_fault_model(nz, nx, seed=3)
        dt = 1.5e-3 * dx / 20.0
        specs.append(dict(nz_dom=nz, nx_dom=nx, dx=dx, dz=dx, dt=dt, nt=nt, fc=12.0, pad=10, fd_order=fd,
                          free_surface=True, src_x=np.linspace(5, nx - 6, ns).astype(np.int64),
                          src_z=np.full(ns, 2), src_types=["force", "moment"] * (ns // 2) + ["force"] * (ns % 2),
                          wavelet=Mo.ricker(np.arange(nt) * dt, 12.0, 1.5 / 12.0), rec_x=np.arange(0, nx, 3),
                          rec_z=np.ones(len(range(0, nx, 3)), dtype=np.int64), mem_budget_gb=4.0,
                          true=(vs, vp, rho), init=Mo.smooth_initial(vs, vp, rho, 4.0)))
    B = UnevenBatch(specs)
    obs = [r[:, 1].contiguous() for r in B.records([s["true"] for s in specs])]
    res = B.gradient([s["init"] for s in specs], obs)
    B.close()
    for s, o, (mis, g) in zip(specs, obs, res):
        S = Solver(s["nz_dom"], s["nx_dom"], s["dx"], s["dz"], s["dt"], s["nt"], s["fc"], s["pad"], len(s["rec_x"]),
                   len(s["src_x"]), fd_order=s["fd_order"], free_surface=True, want_gradient=True)
        S.set_receivers(s["rec_x"], s["rec_z"])
        S.set_shots(s["src_x"], s["src_z"], s["src_types"], np.asarray(s["wavelet"], dtype=np.float32))
        S.set_model(*s["init"])
        S.forward(store=True)
        m1 = S.misfit(o, 1, 1.0)
        g1 = S.gradient(exact=True)["exact"]
        S.close()
        assert _rel(mis.cpu().numpy(), m1) < 1e-12
        for c in range(2):
            assert _rel(g[c].cpu().numpy(), g1[c]) < 1e-12, c
