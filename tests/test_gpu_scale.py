"""Differentiation at scale on the 608 x 2000 grid (dx = 5 m, fd 8) on the
B200.  In every GPU run: the dot-product identity of the FP32 forward and
adjoint on the full grid (2000 steps); a short run (2 shots x 300 steps)
against the FP64 oracle; the exact gradient through the
torch.autograd.Function with checkpoints every 200 steps against central
finite differences along 4 seeded smooth Vs perturbations (4 shots, 2000
steps).  With STFWI_SCALE=1 also the full configuration: 32 shots x 10000
steps, 16 perturbations (about 15 minutes of GPU time and 140 GB of device
memory; python -m pytest tests/test_gpu_scale.py -m gpu -s).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu]
full_scale = pytest.mark.skipif(os.environ.get("STFWI_SCALE") != "1", reason="full scale: set STFWI_SCALE=1")

NZ, NX, DX, DT, FC, PAD, FD = 608, 2000, 5.0, 3.75e-4, 15.0, 20, 8


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _geometry(nshot):
    from stfwi_b200 import models as Mo
    vs, vp, rho = Mo.layered_fault_model(NZ, NX, seed=7)
    vs0, vp0, rho0 = Mo.smooth_initial(vs, vp, rho, 10.0)
    sx = np.linspace(40, NX - 41, nshot).astype(np.int64)
    sz = np.full(nshot, 4)
    types = ["force", "moment"] * (nshot // 2) + ["force"] * (nshot % 2)
    rx = np.arange(2, NX - 2, 4, dtype=np.int32)
    rz = np.full_like(rx, 4)
    return (vs, vp, rho), (vs0, vp0, rho0), sx, sz, types, rx, rz


def _smooth_perturbation(rng, z_range=(150, NZ - 150)):
    """Three Gaussian bumps (sigma 40-80 cells) away from the edges, zero on
    the domain boundary (the C-PML copies of the model are stop-gradient);
    centres at depths in `z_range` (cells)."""
    zz, xx = np.meshgrid(np.arange(NZ), np.arange(NX), indexing="ij")
    d = np.zeros((NZ, NX))
    for _ in range(3):
        s = rng.uniform(40, 80)
        z0, x0 = rng.uniform(*z_range), rng.uniform(300, NX - 300)
        d += rng.choice([-1.0, 1.0]) * np.exp(-((zz - z0) ** 2 + (xx - x0) ** 2) / (2 * s * s))
    return d * np.sin(np.pi * zz / (NZ - 1)) * np.sin(np.pi * xx / (NX - 1))


@full_scale
def test_gradient_at_scale_vs_finite_differences():
    """The full configuration: 32 shots x 10000 steps, 16 perturbations."""
    _finite_difference_check(nt=10000, ns=32, n_pert=16, z_range=(150, NZ - 150))


def test_gradient_at_scale_vs_finite_differences_short():
    """The same check in every GPU run: 4 shots x 2000 steps (0.75 s of
    propagation, so the perturbations sit in the upper 100 cells, which the
    reflected waves reach and leave within the record), 4 perturbations."""
    _finite_difference_check(nt=2000, ns=4, n_pert=4, z_range=(20, 100))


def _finite_difference_check(nt, ns, n_pert, z_range):
    import torch
    from scipy.signal import butter
    from stfwi_b200 import Solver, autograd
    from stfwi_b200 import models as Mo
    true, init, sx, sz, types, rx, rz = _geometry(ns)
    wav = Mo.ricker(np.arange(nt) * DT, FC, 1.5 / FC).astype(np.float32)
    S = Solver(NZ, NX, DX, DX, DT, nt, FC, PAD, len(rx), ns, fd_order=FD, free_surface=True,
               want_gradient=True, ckpt_interval=200)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    S.set_model(*true)
    S.forward()
    obs = torch.empty((ns, 4, nt, len(rx)), dtype=torch.float32, device="cuda")
    S.records(out=obs)
    obs = obs[:, 1].contiguous()
    scale = float(1.0 / (obs.double().pow(2).mean().item() + 1e-45))
    sos = butter(6, 10.0, fs=1.0 / DT, output="sos")
    n_taper = nt // 10
    vs = torch.tensor(init[0], dtype=torch.float64, device="cuda", requires_grad=True)
    vp = torch.tensor(init[1], dtype=torch.float64, device="cuda")
    rho = torch.tensor(init[2], dtype=torch.float64, device="cuda")
    loss = autograd.elastic_misfit(vs, vp, rho, S, obs, 1, scale, sos, n_taper)
    loss.backward()
    g = vs.grad.cpu().numpy()

    def misfit(v):
        S.set_model(v, init[1], init[2])
        S.forward()
        return float(S.misfit(obs, 1, scale, sos, n_taper).sum())

    # FP32 traces make the misfit itself noisy at ~1e-6 of its value (the
    # rounding differs between two nearby models): each comparison allows
    # 1 % of <g, d> plus that floor, 2e-6 J, divided by the step 2h
    J = float(loss)
    rng = np.random.default_rng(2026)
    worst = 0.0
    for k in range(n_pert):
        d = _smooth_perturbation(rng, z_range)
        h = 20.0 / np.abs(d).max()   # at most 20 m/s (about 1 % of Vs)
        fd = (misfit(init[0] + h * d) - misfit(init[0] - h * d)) / (2 * h)
        an = float(np.sum(g * d))
        allow = 1e-2 * abs(an) + 2e-6 * J / (2 * h)
        worst = max(worst, abs(fd - an) / allow)
        print(f"perturbation {k:2d}: FD {fd:+.6e}  <g, d> {an:+.6e}  rel {abs(fd - an) / abs(an):.2e}  "
              f"(error / allowance {abs(fd - an) / allow:.2f})")
    S.close()
    print(f"loss {J:.6e}; worst error / allowance {worst:.2f}")
    assert worst < 1.0, worst


def test_dot_product_identity_at_scale():
    """<L s, y> = <s, L^T y> for the FP32 kernels on the full grid (2000
    steps, one force and one moment shot)."""
    from stfwi_b200 import Solver
    nt = 2000
    true, _, _, _, _, rx, rz = _geometry(2)
    rng = np.random.default_rng(9)
    for st in ("force", "moment"):
        s_in = rng.standard_normal(nt).astype(np.float32)
        ys = rng.standard_normal((1, 4, nt, len(rx))).astype(np.float32)
        S = Solver(NZ, NX, DX, DX, DT, nt, FC, PAD, len(rx), 1, fd_order=FD, free_surface=True,
                   want_gradient=False)
        S.set_model(*true)
        S.set_receivers(rx, rz)
        S.set_shots([NX // 3], [40], [st], s_in)
        S.forward()
        rec = S.records()
        S.set_adjoint_sources(ys)
        src_a = S.gradient(exact=False, src=True)["src"][0]
        S.close()
        lhs = float(np.sum(rec.astype(np.float64) * ys))
        rhs = float(np.sum(s_in.astype(np.float64) * src_a))
        rel = abs(lhs - rhs) / abs(lhs)
        print(f"dot product {st}: <Ls,y> {lhs:+.8e}  <s,L^T y> {rhs:+.8e}  rel {rel:.2e}")
        assert rel < 1e-4, rel


def test_short_gradient_at_scale_vs_oracle():
    """Two shots, 300 steps on the full grid: the traces and the exact
    gradient against the FP64 oracle (observed data from Vs x 1.05, so that
    the residual is not a difference of nearly equal traces)."""
    from stfwi_b200 import Solver
    from stfwi_b200 import models as Mo
    nt = 300
    true, init, _, _, _, rx, rz = _geometry(2)
    sx, sz, types = np.array([700, 1300]), np.array([4, 30]), ["force", "moment"]
    wav = Mo.ricker(np.arange(nt) * DT, FC, 0.06)
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=NX, nz_dom=NZ, dx=DX, dz=DX, dt=DT, nt=nt, fc=FC, pad=PAD,
               fd_order=FD, free_surface=True, d0_f32=True)
    ref_rec = O.forward_batch(*init, sx, sz, types, src_wavelet=wav, **geo)
    obs = O.forward_batch(init[0] * 1.05, init[1], init[2], sx, sz, types, src_wavelet=wav, **geo)[:, 1]
    kw = dict(src_x=sx, src_z=sz, src_wavelet=wav, observed=obs, src_types=types, component=1, scale=1.0,
              invert="vs", **geo)
    (g_ref, _, _), loss = O.compute_gradient("ad", Vs=init[0], Vp=init[1], rho=init[2], **kw)
    S = Solver(NZ, NX, DX, DX, DT, nt, FC, PAD, len(rx), 2, fd_order=FD, free_surface=True, want_gradient=True)
    S.set_model(*init)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav.astype(np.float32))
    S.forward(store=True)
    rec = S.records()
    mis = S.misfit(obs.astype(np.float32), 1, 1.0)
    g = S.gradient(exact=True)["exact"][0]
    S.close()
    amp = float(np.linalg.norm(rec[:, 1]) / np.linalg.norm(rec[:, 1] - obs))
    e_rec = max(_rel(rec[k, c], ref_rec[k, c]) for k in range(2) for c in range(4))
    e = (abs(mis.sum() / loss - 1), _rel(g, g_ref))
    print(f"short run on the full grid: traces rel-L2 {e_rec:.2e}, amplification {amp:.1f}, "
          f"misfit rel {e[0]:.2e}, g_Vs rel-L2 {e[1]:.2e}")
    assert e_rec < 1e-5, e_rec
    tol = 2e-5 * max(amp, 1.0)
    assert e[0] < tol and e[1] < tol, (e, tol)
