"""Shot sharding across ranks (one process per GPU).

Shots are independent: each rank takes every world-th shot, computes the raw
gradient and misfit of its shots with the misfit normalised by the *total*
shot count, and one all-reduce (sum, FP64) of [g_Vs, g_Vp, g_rho, loss]
forms the batch result, the only exchange step.  The post-processing
(smoothing, source taper, illumination) is linear and runs after the
reduction, identically on every rank.  NCCL for CUDA tensors, gloo for CPU.
"""
from __future__ import annotations

import numpy as np


def shard_indices(n_shots, rank, world):
    """Round-robin: rank r takes shots r, r + world, ...  (equal cost per shot)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside [0, {world})")
    return np.arange(rank, n_shots, world)


def allreduce_gradient(grads, loss, group=None, device=None):
    """Sum (g_Vs, g_Vp, g_rho) and the loss over the group with one FP64 all-reduce."""
    import torch
    import torch.distributed as dist
    shape = np.asarray(grads[0]).shape
    flat = [torch.as_tensor(np.asarray(g, dtype=np.float64)).reshape(-1) for g in grads]
    buf = torch.cat(flat + [torch.tensor([float(loss)], dtype=torch.float64)])
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    buf = buf.cpu().numpy()
    n = int(np.prod(shape))
    out = tuple(buf[k * n:(k + 1) * n].reshape(shape) for k in range(len(grads)))
    return out, float(buf[-1])


def sharded_compute_gradient(backend, *, src_x, src_z, observed, src_types=None, group=None, device=None,
                             local_fn=None, grad_smooth_sigma=None, source_taper=None, illumination=None,
                             **kw):
    """compute_gradient over all ranks' shots.  Every rank passes the full
    shot list; ``local_fn(backend, idx, n_total, **kw)`` computes the raw
    (gradients, loss) of shots ``idx`` with the loss normalised by
    ``n_total`` (default: the CUDA path on this rank's GPU)."""
    import torch.distributed as dist
    from .fwi.gradient import _postprocess
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    src_x = np.atleast_1d(np.asarray(src_x))
    src_z = np.broadcast_to(np.atleast_1d(np.asarray(src_z)), src_x.shape)
    idx = shard_indices(src_x.size, rank, world)
    if local_fn is None:
        local_fn = _cuda_local
    grads, loss = local_fn(backend, idx, src_x.size, src_x=src_x, src_z=src_z, observed=observed,
                           src_types=src_types, **kw)
    grads, loss = allreduce_gradient(grads, loss, group=group, device=device)
    return _postprocess(grads, grad_smooth_sigma, source_taper, illumination), loss


def _cuda_local(backend, idx, n_total, *, src_x, src_z, observed, src_types=None, **kw):
    from .fwi.gradient import compute_gradient
    types = None if src_types is None else [src_types[i] for i in idx]
    if idx.size == 0:
        z = np.zeros((kw["nz_dom"], kw["nx_dom"]))
        return (z, z.copy(), z.copy()), 0.0
    return compute_gradient(backend, src_x=src_x[idx], src_z=src_z[idx], observed=np.asarray(observed)[idx],
                            src_types=types, n_shots_total=n_total, **kw)
