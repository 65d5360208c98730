"""Failure detection on the GPU without a GPU fault (B200).

* A tile-copy wait that runs out: the wait limit set to zero polls makes
  every kernel give up at its first wait; it records STFWI_ERR_TIMEOUT,
  drains its own copies in flight and returns, the context stays usable, and
  the same handle then computes the right answer with the default limit.
* A NaN in the host model: the receiver check reports STFWI_ERR_NONFINITE
  instead of returning NaN traces, and the handle recovers with a clean model.
* The sharded CUDA path (stfwi_b200.parallel with the real per-rank GPU
  gradient) on two gloo ranks sharing the GPU: the reduced gradient and
  misfit equal one process over all shots.  The ranks' kernels never wait on
  each other; the only exchange is the host all-reduce.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as O
from tests import dot_case as C

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _small_solver(nt=60, nshot=3, want_gradient=False):
    from stfwi_b200 import Solver
    vs, vp, rho = C.model()
    rx = np.arange(1, C.NX - 1, 2, dtype=np.int32)
    rz = np.ones_like(rx)
    sx, sz, types = np.array([4, 15, 26])[:nshot], np.array([2, 4, 3])[:nshot], ["force", "moment", "force"][:nshot]
    wav = (O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9).astype(np.float32)
    S = Solver(C.NZ, C.NX, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, len(rx), nshot, fd_order=8, free_surface=True,
               want_gradient=want_gradient)
    S.set_model(vs, vp, rho)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    ref = O.forward_batch(vs, vp, rho, sx, sz, types, rx, rz, C.NX, C.NZ, C.DX, C.DZ, C.DT, nt, C.FC, C.PAD, wav,
                          fd_order=8, free_surface=True, d0_f32=True)
    return S, (vs, vp, rho), ref


def test_wait_timeout_is_reported_and_the_handle_recovers():
    from stfwi_b200 import _native as N
    S, _, ref = _small_solver()
    S.set_adjoint_sources(np.ones((3, 4, S.nt, S.nrec), dtype=np.float32))
    # the forward kernels give up at their first wait
    S.set_wait_limit(0)
    S.forward()
    with pytest.raises(N.StfwiError) as e:
        S.check()
    assert e.value.status == N.STFWI_ERR_TIMEOUT
    # a forward with the default limit clears the status; then the adjoint
    # kernels give up the same way
    S.set_wait_limit(-1)
    S.forward()
    S.check()
    S.set_wait_limit(0)
    with pytest.raises(N.StfwiError) as e:
        S.gradient(exact=False, src=True)
    assert e.value.status == N.STFWI_ERR_TIMEOUT
    S.set_wait_limit(-1)
    S.forward()
    rec = S.records()   # checks the status: fine again
    assert max(_rel(rec[k, c], ref[k, c]) for k in range(3) for c in range(4)) < 1e-5
    S.close()


def test_nan_in_the_model_is_reported():
    from stfwi_b200 import _native as N
    S, (vs, vp, rho), ref = _small_solver()
    bad = vs.copy()
    bad[C.NZ // 2, C.NX // 2] = np.nan
    S.set_model(bad, vp, rho)
    S.forward()
    with pytest.raises(N.StfwiError) as e:
        S.records()
    assert e.value.status == N.STFWI_ERR_NONFINITE
    S.set_model(vs, vp, rho)
    S.forward()
    rec = S.records()
    assert max(_rel(rec[k, c], ref[k, c]) for k in range(3) for c in range(4)) < 1e-5
    S.close()


def _case():
    vs, vp, rho = C.model()
    nt = 80
    rx = np.arange(1, C.NX - 1, 3, dtype=np.int32)
    rz = np.ones_like(rx)
    sx = np.array([4, 10, 16, 22, 28])
    sz = np.array([2, 3, 2, 4, 2])
    types = ["force", "moment", "force", "force", "moment"]
    wav = O.ricker(np.arange(nt) * C.DT, C.FC, 1.5 / C.FC) * 1e9
    geo = dict(rec_x=rx, rec_z=rz, nx_dom=C.NX, nz_dom=C.NZ, dx=C.DX, dz=C.DZ, dt=C.DT, nt=nt, fc=C.FC,
               pad=C.PAD, fd_order=4, free_surface=True)
    obs = O.forward_batch(vs * 1.02, vp, rho, sx, sz, types, src_wavelet=wav, d0_f32=True, **geo)[:, 1]
    kw = dict(Vs=vs, Vp=vp, rho=rho, src_wavelet=wav, component=1, scale=2.0, invert="vs_vp", **geo)
    return sx, sz, types, obs, kw


def _worker(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        from stfwi_b200.parallel import sharded_compute_gradient
        sx, sz, types, obs, kw = _case()
        (g_vs, g_vp, _), loss = sharded_compute_gradient("cuda", src_x=sx, src_z=sz, observed=obs,
                                                         src_types=types, grad_smooth_sigma=1.0, **kw)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), g_vs=g_vs, g_vp=g_vp, loss=loss)
    except Exception as e:
        with open(os.path.join(out_dir, f"r{rank}.err"), "w") as fh:
            fh.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_cuda_path_two_gloo_ranks_equal_one_process(tmp_path):
    from stfwi_b200 import fwi
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    for rank in (0, 1):
        assert not (tmp_path / f"r{rank}.err").exists(), (tmp_path / f"r{rank}.err").read_text()
    sx, sz, types, obs, kw = _case()
    (r_vs, r_vp, _), r_loss = fwi.compute_gradient("cuda", src_x=sx, src_z=sz, observed=obs, src_types=types,
                                                   grad_smooth_sigma=1.0, **kw)
    for rank in (0, 1):
        d = np.load(tmp_path / f"r{rank}.npz")
        # shot groups differ between one handle of 5 shots and handles of 3
        # and 2: FP32 sums over a block's shots round differently
        assert abs(float(d["loss"]) / r_loss - 1) < 1e-6
        assert _rel(d["g_vs"], r_vs) < 1e-5 and _rel(d["g_vp"], r_vp) < 1e-5
