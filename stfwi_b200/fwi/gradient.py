"""compute_gradient with the reference's signature (fwi/gradient.py:48-99).

Backends: ``'cuda'`` (alias ``'ad'``) returns the exact gradient of the
discrete forward, what the reference's ``'ad'`` backend gets from JAX AD;
``'cuda_imaging'`` (alias ``'adjoint'``) returns the reference's imaging
condition (fwi/imaging.py), fused into the adjoint sweep.  The forward, the
residual preparation (filter, taper, FP64 misfit), the adjoint and the
post-processing (smoothing, source taper, illumination) all run on the GPU.  Unlike the reference's ``'adjoint'`` backend,
whose forward always injects a force (fwi/gradient.py:176-180), the forward
and the adjoint here use the same ``src_type``.
"""
from __future__ import annotations

import numpy as np

from ..solver import Solver
from .loss import gaussian_smooth_2d

_BACKENDS = {"cuda": "exact", "ad": "exact", "cuda_imaging": "imaging", "adjoint": "imaging"}
_CACHE = {}


def clear_cache():
    """Release the GPU handles kept between calls."""
    for S in _CACHE.values():
        S.close()
    _CACHE.clear()


def _solver(nz_dom, nx_dom, dx, dz, dt, nt, fc, pad, nrec, nshot, fd_order, free_surface, density=False):
    key = (nz_dom, nx_dom, float(dx), float(dz), float(dt), nt, float(fc), pad, nrec, nshot, fd_order,
           bool(free_surface), bool(density))
    S = _CACHE.get(key)
    if S is None:
        if len(_CACHE) >= 4:
            clear_cache()
        S = Solver(nz_dom, nx_dom, dx, dz, dt, nt, fc, pad, nrec, nshot, fd_order=fd_order,
                   free_surface=free_surface, want_gradient=True, density=density)
        _CACHE[key] = S
    return S


def _postprocess(grads, grad_smooth_sigma, source_taper, illumination):
    """fwi/gradient.py:266-277 on the host (build_loss_fn, whose Tikhonov
    term is added to the gradient before this step)."""
    out = list(grads)
    if grad_smooth_sigma is not None:
        out = [gaussian_smooth_2d(g, grad_smooth_sigma) for g in out]
    if source_taper is not None:
        st = np.asarray(source_taper)
        out = [g * st for g in out]
    if illumination is not None:
        il = np.asarray(illumination)
        out = [g * il for g in out]
    return tuple(out)


def compute_gradient(backend, *, Vs, Vp, rho, src_x, src_z, src_wavelet, observed, rec_x, rec_z, nx_dom,
                     nz_dom, dx, dz, dt, nt, fc, pad, component=2, invert="vs", scale=1.0, sos=None,
                     n_taper=0, fd_order=2, free_surface=False, src_type="force", block_size=None,
                     grad_smooth_sigma=None, source_taper=None, illumination=None, src_types=None,
                     n_shots_total=None):
    """(g_Vs, g_Vp, g_rho) on the physical grid and the loss
    scale * mean_shots mean_{t,r}(F T (pred - obs))^2 (FP64).  With
    ``n_shots_total`` the mean over shots divides by that count (these shots
    are one shard of a larger batch)."""
    if backend not in _BACKENDS:
        raise ValueError(f"unknown backend {backend!r}; use 'cuda' or 'cuda_imaging'")
    if invert not in ("vs", "vs_vp", "all"):
        raise ValueError(f"invert={invert!r}; use 'vs', 'vs_vp', or 'all'")
    if fd_order not in (2, 4, 8):
        raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
    mode = _BACKENDS[backend]
    sx = np.atleast_1d(np.asarray(src_x)).astype(np.int64)
    sz = np.broadcast_to(np.atleast_1d(np.asarray(src_z)), sx.shape).astype(np.int64)
    types = list(src_types) if src_types is not None else [src_type] * sx.size
    for t in types:
        if t not in ("force", "moment"):
            raise NotImplementedError(f"src_type={t!r} not supported (use 'force' or 'moment').")
    rx = np.asarray(rec_x, dtype=np.int32).reshape(-1)
    rz = np.asarray(rec_z, dtype=np.int32).reshape(-1)
    # invert='all' keeps the forward velocities for the density gradient
    S = _solver(int(nz_dom), int(nx_dom), dx, dz, dt, int(nt), fc, int(pad), rx.size, sx.size, int(fd_order),
                free_surface, density=(invert == "all"))
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, np.asarray(src_wavelet, dtype=np.float32))
    S.set_model(Vs, Vp, rho)
    S.forward(store=True)
    loss = float(S.misfit(observed, component, scale, sos, n_taper, nshot_norm=n_shots_total or 0).sum())
    # fwi/gradient.py:266-277 on the device, after the adjoint sweep
    S.set_postprocess(grad_smooth_sigma, source_taper, illumination)
    g = S.gradient(exact=(mode == "exact"), imaging=(mode == "imaging"))[mode]
    g_vs, g_vp, g_rho = (np.array(a) for a in g)
    # fwi/gradient.py:250-257: frozen parameters get zero gradients
    if invert == "vs":
        g_vp = np.zeros_like(g_vp)
    if invert != "all":
        g_rho = np.zeros_like(g_rho)
    return (g_vs, g_vp, g_rho), loss
