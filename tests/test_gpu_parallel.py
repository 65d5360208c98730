"""Shot sharding over two gloo ranks with the CUDA path (``parallel._cuda_local``)
on one GPU: each rank runs its own shots through its own handle, the only
exchange is the FP64 all-reduce on the host, and the reduced gradient and
misfit equal one process running all shots.  The ranks' kernels never wait
on one another (the collective is gloo, between launches)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.test_parallel import _case

pytestmark = pytest.mark.gpu


def _worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from stfwi_b200.parallel import sharded_compute_gradient
        sx, sz, types, obs, kw = _case()
        (g_vs, g_vp, _), loss = sharded_compute_gradient("cuda", src_x=sx, src_z=sz, observed=obs,
                                                         src_types=types, grad_smooth_sigma=1.0, **kw)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), g_vs=g_vs, g_vp=g_vp, loss=loss)
    except Exception as e:
        with open(os.path.join(out_dir, f"r{rank}.err"), "w") as fh:
            fh.write(type(e).__name__ + ": " + str(e))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_cuda_path_equal_one_process(tmp_path):
    from oracle import oracle as O
    from stfwi_b200.fwi import compute_gradient
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    for rank in (0, 1):
        assert not (tmp_path / f"r{rank}.err").exists(), (tmp_path / f"r{rank}.err").read_text()
    sx, sz, types, obs, kw = _case()
    (c_vs, c_vp, _), c_loss = compute_gradient("cuda", src_x=sx, src_z=sz, observed=obs, src_types=types,
                                               grad_smooth_sigma=1.0, **kw)
    (r_vs, r_vp, _), r_loss = O.compute_gradient("ad", src_x=sx, src_z=sz, observed=obs, src_types=types,
                                                 grad_smooth_sigma=1.0, **kw)
    errs = {}
    for rank in (0, 1):
        d = np.load(tmp_path / f"r{rank}.npz")
        # one process vs two ranks: the same FP32 kernels per shot; the shots a
        # block holds are summed in FP32 before the FP64 sums, and the blocks
        # hold different shots
        errs[f"r{rank}_vs_one_process"] = max(
            abs(float(d["loss"]) / c_loss - 1),
            np.linalg.norm(d["g_vs"] - c_vs) / np.linalg.norm(c_vs),
            np.linalg.norm(d["g_vp"] - c_vp) / np.linalg.norm(c_vp))
        errs[f"r{rank}_vs_oracle"] = max(
            abs(float(d["loss"]) / r_loss - 1),
            np.linalg.norm(d["g_vs"] - r_vs) / np.linalg.norm(r_vs),
            np.linalg.norm(d["g_vp"] - r_vp) / np.linalg.norm(r_vp))
    print("sharded CUDA path rel errors:", errs)
    for k, v in errs.items():
        assert v < (2e-6 if k.endswith("one_process") else 1e-5), (k, v)
