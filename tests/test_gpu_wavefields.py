"""Full wavefields and the history-based imaging condition (B200): the
reference's forward_jax return_vars '*_full' / return_wavefields,
adjoint_jax(return_wavefields=...) and imaging_condition
(fwi/forward.py:449-463, fwi/adjoint_jax_kernel.py:470-483,
fwi/imaging.py:83-169), against the FP64 oracle.

Tolerances: frames of the FP32 kernels against the FP64 oracle, rel-L2 per
field <= 1e-5 (the seismogram bound of the other parity tests; these are
the same states); the imaging sums on FP32 copies of FP64 histories against
the FP64 formula, rel-L2 <= 1e-6 (FP32 rounding of the inputs only).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu

FIELDS = ("vx", "vz", "ex", "ez", "es")


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("fd,fs,st", [(8, True, "force"), (4, False, "moment"), (2, True, "moment")])
def test_forward_frames_match_oracle(fd, fs, st):
    from stfwi_b200 import fwi
    vs, vp, rho = C.model()
    sx, sz, rx, rz = C.acquisition(fs, st)
    s_in, _ = C.random_vectors()
    out = fwi.forward_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in,
                          return_vars=["vz"] + [f + "_full" for f in FIELDS], fd_order=fd, free_surface=fs,
                          src_type=st)
    rec, full, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in,
                             fd, fs, st, full=FIELDS, d0_f32=True)
    assert _rel(out[0], rec[1]) < 1e-5
    errs = {f: _rel(out[1 + k], full[f]) for k, f in enumerate(FIELDS)}
    print(f"forward frames fd{fd} fs={fs} {st}:", {k: f"{v:.1e}" for k, v in errs.items()})
    assert all(e < 1e-5 for e in errs.values()), errs
    # return_wavefields=True: the receiver tuple, then the U, V, ex, ez frames
    w = fwi.forward_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, s_in,
                        return_wavefields=True, fd_order=fd, free_surface=fs, src_type=st)
    assert len(w) == 8 and w[4].shape == full["vx"].shape
    assert max(_rel(w[4 + k], full[f]) for k, f in enumerate(FIELDS[:4])) < 1e-5


@pytest.mark.parametrize("fd,fs,st", [(8, True, "force"), (4, False, "moment")])
def test_adjoint_frames_match_oracle(fd, fs, st):
    from stfwi_b200 import fwi
    vs, vp, rho = C.model()
    sx, sz, rx, rz = C.acquisition(fs, st)
    _, ys = C.random_vectors()
    out = fwi.adjoint_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                          fd_order=fd, free_surface=fs, src_type=st, return_wavefields=True)
    names = ("U_a", "V_a", "ex_a", "ez_a", "es_a")
    ref = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                    fd_order=fd, free_surface=fs, src_type=st, hist=names, d0_f32=True)
    assert len(out) == 6
    assert _rel(out[0], ref["src"]) < 1e-5
    errs = {k: _rel(out[1 + i], ref[k]) for i, k in enumerate(names)}
    print(f"adjoint frames fd{fd} fs={fs} {st}:", {k: f"{v:.1e}" for k, v in errs.items()})
    assert all(e < 1e-5 for e in errs.values()), errs
    vel = fwi.adjoint_jax(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, C.NT, C.FC, C.PAD, *ys,
                          fd_order=fd, free_surface=fs, src_type=st, return_wavefields="velocity")
    assert len(vel) == 3 and _rel(vel[1], ref["U_a"]) < 1e-5 and _rel(vel[2], ref["V_a"]) < 1e-5


@pytest.mark.parametrize("fs", [True, False])
def test_imaging_condition_on_histories(fs):
    """fwi.imaging_condition on the oracle's FP64 histories (cast to FP32,
    given once as host arrays and once as CUDA tensors, with a chunk that
    does not divide nt) against the reference's formula in FP64, and against
    the oracle's fused imaging sums."""
    import torch
    from stfwi_b200 import fwi
    vs, vp, rho = C.model()
    st, fd, nt = "force", 4, 45
    sx, sz, rx, rz = C.acquisition(fs, st)
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    rng = np.random.default_rng(3)
    ys = [rng.standard_normal((nt, len(rx))) for _ in range(4)]
    _, full, _ = O.forward(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, wav, fd, fs,
                           st, full=FIELDS, d0_f32=True)
    a = O.adjoint(vs, vp, rho, sx, sz, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, *ys, fd_order=fd,
                  free_surface=fs, src_type=st, src_wavelet=wav, want=("img",), hist=("U_a", "V_a"), d0_f32=True)
    h32 = {k: full[k].astype(np.float32) for k in FIELDS}
    ua, va = a["U_a"].astype(np.float32), a["V_a"].astype(np.float32)
    geo = (C.DX, C.DZ, C.DT, C.PAD, fs, C.NZ, C.NX)
    ref = O.imaging_condition(vs, vp, rho, h32["ex"], h32["ez"], h32["es"], ua, va, *geo, vx_hist=h32["vx"],
                              vz_hist=h32["vz"])
    got = fwi.imaging_condition(vs, vp, rho, h32["ex"], h32["ez"], h32["es"], ua, va, *geo, vx_hist=h32["vx"],
                                vz_hist=h32["vz"], time_chunk=7)
    errs = [_rel(g, r) for g, r in zip(got, ref)]
    print(f"imaging condition fs={fs} (host histories):", [f"{e:.1e}" for e in errs])
    assert max(errs) < 1e-6, errs
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in h32.items()}
    got_d = fwi.imaging_condition(vs, vp, rho, dev["ex"], dev["ez"], dev["es"], torch.as_tensor(ua, device="cuda"),
                                  torch.as_tensor(va, device="cuda"), *geo, vx_hist=dev["vx"], vz_hist=dev["vz"])
    assert max(_rel(g, r) for g, r in zip(got_d, ref)) < 1e-6
    # the oracle's own imaging sums (fused into its adjoint, FP64 histories)
    lam, mu, rl = (O.crop(p, C.PAD, fs, C.NZ, C.NX) for p in a["img"])
    assert _rel(got[3], lam) < 1e-5 and _rel(got[4], mu) < 1e-5 and _rel(got[5], rl) < 1e-5
    # without the forward velocities the density term is zero
    nov = fwi.imaging_condition(vs, vp, rho, h32["ex"], h32["ez"], h32["es"], ua, va, *geo)
    assert np.all(nov[5] == 0) and _rel(nov[3], ref[3]) < 1e-6
