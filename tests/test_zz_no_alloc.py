"""The misfit entry point that allocates nothing (stfwi_misfit_noalloc).

Some callers cannot call cudaMalloc: a custom call made from inside a
framework that has reserved most of the device for its own memory pool (the
JAX drivers of this workload preallocate 90 % of it), where one more
allocation can fail or fragment that pool.  stfwi_misfit_noalloc serves them
with a fixed, file-scope device scratch array instead of a handle's
workspace.  These tests call it through the C ABI and check it against the
handle-based stfwi_misfit on the same traces, twice in a row (the scratch
keeps the previous call's contents): once with a low-pass filter and the
call's own shot count, once without a filter and with a larger shot count
for the normalisation (a shard of a bigger batch).  This file is collected
last on purpose.
"""
import ctypes as ct

import numpy as np
import pytest

from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _desc(N, component, scale, sos, n_taper, nshot_norm):
    if sos is None:
        return N.StfwiMisfitDesc(component, n_taper, 0, nshot_norm, scale, None), None
    sos_a = np.ascontiguousarray(np.asarray(sos, dtype=np.float64))
    d = N.StfwiMisfitDesc(component, n_taper, sos_a.shape[0], nshot_norm, scale,
                          sos_a.ctypes.data_as(ct.POINTER(ct.c_double)))
    return d, sos_a


def test_noalloc_misfit_matches_handle_path_twice():
    import torch
    from scipy.signal import butter

    from oracle import oracle as O
    from stfwi_b200 import Solver
    from stfwi_b200 import _native as N

    torch.cuda.init()
    lib = N.load()
    vs, vp, rho = C.model()
    nt, fd, fs = 120, 4, True
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.ones_like(rx)
    sx, sz, types = np.array([4, 15, 26]), np.array([2, 4, 3]), ["force", "moment", "force"]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    S = Solver(C.NZ, C.NX, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, len(rx), 3, fd_order=fd, free_surface=fs,
               want_gradient=False)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    S.forward()
    pred = torch.empty((3, 4, nt, len(rx)), dtype=torch.float32, device="cuda")
    S.records(out=pred)
    sos = butter(4, 30.0, fs=1.0 / C.DT, output="sos")
    comp, scale, n_taper = 1, 2.5, 12
    rng = np.random.default_rng(11)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (filt, nnorm) in enumerate(((sos, 0), (None, 7))):
        obs = torch.tensor(rng.standard_normal((3, nt, len(rx))) * 1e-9, dtype=torch.float32, device="cuda")
        # handle path
        mis_ref = S.misfit(obs, comp, scale, filt, n_taper, nshot_norm=nnorm)
        src_ref = S.gradient(exact=False, src=True)["src"]
        # no-allocation path: device inputs and outputs owned by the caller
        rec_adj = torch.full((3, 4, nt, len(rx)), float("nan"), dtype=torch.float32, device="cuda")
        mis = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        d, sos_keep = _desc(N, comp, scale, filt, n_taper, nnorm)
        st = lib.stfwi_misfit_noalloc(3, nt, len(rx), pred.data_ptr(), obs.data_ptr(), ct.byref(d),
                                      rec_adj.data_ptr(), mis.data_ptr(), stream)
        assert st == 0
        torch.cuda.synchronize()
        m = mis.cpu().numpy()
        assert np.all(np.isfinite(m))
        np.testing.assert_allclose(m, mis_ref, rtol=1e-12, atol=0.0)
        # the adjoint sources: fed through the handle's adjoint they give the
        # same source-wavelet adjoint as the handle's own
        assert torch.isfinite(rec_adj).all()
        S.set_adjoint_sources(rec_adj)
        src = S.gradient(exact=False, src=True)["src"]
        err = np.linalg.norm(src - src_ref) / np.linalg.norm(src_ref)
        assert err < 1e-6, (call, err)
    S.close()


def test_noalloc_rejects_oversized_batches():
    import torch

    from stfwi_b200 import _native as N

    torch.cuda.init()
    lib = N.load()
    d = N.StfwiMisfitDesc(1, 0, 0, 0, 1.0, None)
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    too_many = N.NOALLOC_MAX_TRACES // 100 + 1
    st = lib.stfwi_misfit_noalloc(100, 10, too_many, buf.data_ptr(), buf.data_ptr(), ct.byref(d),
                                  buf.data_ptr(), buf.data_ptr(), None)
    assert st == N.STFWI_ERR_INVALID
