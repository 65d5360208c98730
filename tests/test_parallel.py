"""Shot sharding over two gloo ranks on CPU (the oracle computes each rank's
shots): the reduced gradient and misfit equal the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests import dot_case as C


def _case():
    from oracle import oracle as O
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
    obs = O.forward_batch(vs * 1.02, vp, rho, sx, sz, types, src_wavelet=wav, **geo)[:, 1]
    kw = dict(Vs=vs, Vp=vp, rho=rho, src_wavelet=wav, component=1, scale=2.0, invert="vs_vp", **geo)
    return sx, sz, types, obs, kw


def _oracle_local(backend, idx, n_total, *, src_x, src_z, observed, src_types=None, **kw):
    from oracle import oracle as O
    ref = {"cuda": "ad", "cuda_imaging": "adjoint"}[backend]
    if idx.size == 0:
        z = np.zeros((kw["nz_dom"], kw["nx_dom"]))
        return (z, z, z), 0.0
    grads, loss = O.compute_gradient(ref, src_x=src_x[idx], src_z=src_z[idx], observed=observed[idx],
                                     src_types=[src_types[i] for i in idx], **kw)
    f = idx.size / n_total  # the oracle normalises by its own shot count
    return tuple(g * f for g in grads), loss * f


def _worker(rank, world, port, out_dir, fail_rank):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    from stfwi_b200.parallel import sharded_compute_gradient
    sx, sz, types, obs, kw = _case()
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before the collective")
        (g_vs, g_vp, _), loss = sharded_compute_gradient("cuda", src_x=sx, src_z=sz, observed=obs,
                                                         src_types=types, local_fn=_oracle_local,
                                                         grad_smooth_sigma=1.0, **kw)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), g_vs=g_vs, g_vp=g_vp, loss=loss)
    except Exception as e:  # the failure is reported on the host, never on a device
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


def test_two_gloo_ranks_equal_one_process(tmp_path):
    from oracle import oracle as O
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), -1), nprocs=2, start_method="spawn")
    sx, sz, types, obs, kw = _case()
    (r_vs, r_vp, _), r_loss = O.compute_gradient("ad", src_x=sx, src_z=sz, observed=obs, src_types=types,
                                                 grad_smooth_sigma=1.0, **kw)
    for rank in (0, 1):
        d = np.load(tmp_path / f"r{rank}.npz")
        assert abs(float(d["loss"]) / r_loss - 1) < 1e-12
        assert np.linalg.norm(d["g_vs"] - r_vs) / np.linalg.norm(r_vs) < 1e-12
        assert np.linalg.norm(d["g_vp"] - r_vp) / np.linalg.norm(r_vp) < 1e-12


def test_a_failed_rank_surfaces_as_an_error_on_the_others(tmp_path):
    """Rank 1 raises before the all-reduce; rank 0's collective ends with an
    error (gloo reports the lost peer or the timeout) instead of hanging."""
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), 1), nprocs=2, start_method="spawn")
    assert (tmp_path / "r1.err").exists()
    assert (tmp_path / "r0.err").exists(), "rank 0 should see the failure"
    assert not (tmp_path / "r0.npz").exists()


def test_shard_indices_cover_every_shot_once():
    from stfwi_b200.parallel import shard_indices
    for n, w in ((50, 8), (5, 2), (3, 4)):
        idx = np.concatenate([shard_indices(n, r, w) for r in range(w)])
        assert np.array_equal(np.sort(idx), np.arange(n))
    with pytest.raises(ValueError):
        shard_indices(5, 3, 2)
