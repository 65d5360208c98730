"""torch.autograd bindings on the GPU against finite differences and the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _setup(nt=110):
    import torch
    from stfwi_b200 import Solver
    vs, vp, rho = C.model(np.float32)
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.ones_like(rx)
    sx, sz, types = np.array([8, 22]), np.array([2, 4]), ["force", "moment"]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    S = Solver(C.NZ, C.NX, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, len(rx), 2, fd_order=8, free_surface=True,
               want_gradient=True)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(a, device=dev)
    return S, t(vs), t(vp), t(rho), rx, rz, sx, sz, types, wav


def test_forward_function_vjp_matches_oracle_gradient():
    """sum(w * traces) backpropagated = the exact gradient with w as the
    receiver adjoint sources (checked against the FP64 oracle)."""
    import torch
    from stfwi_b200.autograd import elastic_forward
    S, vs, vp, rho, rx, rz, sx, sz, types, wav = _setup()
    vs.requires_grad_(True); vp.requires_grad_(True)
    rec = elastic_forward(vs, vp, rho, S)
    w = torch.randn(rec.shape, generator=torch.Generator(device="cuda").manual_seed(0), device="cuda") * 1e-3
    (rec * w).sum().backward()
    wn = w.double().cpu().numpy()
    gm = O.gradient_batch(C.model()[0], C.model()[1], C.model()[2], sx, sz, types, rec_x=rx, rec_z=rz,
                          nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=rec.shape[2], fc=C.FC,
                          pad=C.PAD, src_wavelet=wav.astype(np.float64), rec_adj=wn, fd_order=8,
                          free_surface=True, mode="gmat", d0_f32=True).sum(axis=0)
    gvs, gvp, _ = O.chain_exact(O.crop(gm, C.PAD, True, C.NZ, C.NX), *C.model())
    e1 = np.linalg.norm(vs.grad.double().cpu().numpy() - gvs) / np.linalg.norm(gvs)
    e2 = np.linalg.norm(vp.grad.double().cpu().numpy() - gvp) / np.linalg.norm(gvp)
    assert e1 < 1e-4 and e2 < 1e-4, (e1, e2)
    S.close()


def test_misfit_function_gradient_vs_finite_differences():
    """The fused-misfit Function's Vs gradient along a smooth perturbation
    that vanishes on the PML-copied edges, against central differences of
    the GPU misfit itself (FP32 forward, FP64 sums)."""
    import torch
    from stfwi_b200.autograd import elastic_misfit
    S, vs, vp, rho, rx, rz, sx, sz, types, wav = _setup()
    with torch.no_grad():
        obs = torch.zeros((2, S.nt, S.nrec), device="cuda")
        S.set_model(vs * 1.04, vp, rho)
        S.forward()
        r = torch.empty((2, 4, S.nt, S.nrec), device="cuda")
        S.records(out=r)
        obs.copy_(r[:, 1])
    vs.requires_grad_(True)
    loss = elastic_misfit(vs, vp, rho, S, obs, component=1, scale=1e6)
    loss.backward()
    zz, xx = np.meshgrid(np.arange(C.NZ), np.arange(C.NX), indexing="ij")
    d = torch.tensor(30.0 * np.sin(np.pi * zz / (C.NZ - 1)) * np.sin(np.pi * xx / (C.NX - 1)),
                     dtype=torch.float32, device="cuda")
    an = float((vs.grad.double() * d.double()).sum())
    h = 1.0
    with torch.no_grad():
        lp = float(elastic_misfit(vs + h * d, vp, rho, S, obs, component=1, scale=1e6))
        lm = float(elastic_misfit(vs - h * d, vp, rho, S, obs, component=1, scale=1e6))
    fd = (lp - lm) / (2 * h)
    assert abs(fd - an) < 2e-3 * abs(an), (fd, an)
    with pytest.raises(NotImplementedError):
        elastic_misfit(vs, vp, rho.clone().requires_grad_(True), S, obs)
    S.close()
