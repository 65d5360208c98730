"""Multistage SciPy L-BFGS-B FWI driver with the reference's signature
(fwi/optim_lbfgsb.py:137-473 run_multiscale_fwi), on the CUDA path.

The host keeps what SciPy needs (the scaled FP64 parameter vector, bounds,
the L-BFGS-B iteration); every gradient evaluation runs on the device: the
feasibility projection (fwi/projections.py:67-117) in place on FP64 device
tensors, the forward, residual preparation and adjoint of all shots, the
gradient post-processing (smoothing, source taper, preconditioner) and the
stage preconditioner itself.  Stages, block scaling, per-cell bounds in
scaled space, the plateau stop and the checkpoint files follow the
reference.
"""
from __future__ import annotations

import os
import time
from typing import Optional, Sequence

import numpy as np

from .forward import ricker_jax
from .gradient import compute_gradient
from .illumination import compute_illumination_for_stage
from .projections import cfl_vp_cap, project_velocity_device

_KEY_TO_IDX = {"Vs": 0, "Vp": 1, "rho": 2}


class _PlateauStop(Exception):
    """Aborts scipy.optimize.minimize when the plateau detector fires."""


class _Plateau:
    """Stop a stage when mean(last N losses) >= (1 - tol) mean(previous N)
    (fwi/optim_lbfgsb.py:117-134); disabled when the window is None or 0."""

    def __init__(self, window: Optional[int], rel_tol: float):
        self.window = window or 0
        self.rel_tol = float(rel_tol)
        self.history: list = []

    def push(self, loss: float) -> bool:
        self.history.append(float(loss))
        if self.window <= 0 or len(self.history) < 2 * self.window:
            return False
        last = np.mean(self.history[-self.window:])
        prev = np.mean(self.history[-2 * self.window:-self.window])
        return last >= prev * (1.0 - self.rel_tol)


def _block_scales(params):
    return [max(float(np.abs(p).max()), 1e-12) for p in params]


def _active_keys(invert):
    if invert == "vs":
        return ["Vs"]
    if invert == "vs_vp":
        return ["Vs", "Vp"]
    if invert == "all":
        return ["Vs", "Vp", "rho"]
    raise ValueError(f"invert={invert!r}; use 'vs', 'vs_vp', or 'all'")


def _project(params, K_margin, vp_cap):
    """Project (Vs, Vp, rho) on the device; returns CUDA FP64 tensors."""
    import torch
    t = [torch.as_tensor(np.ascontiguousarray(p, dtype=np.float64), device="cuda") for p in params]
    project_velocity_device(t[0], t[1], t[2], K_margin=K_margin, vp_cap=vp_cap)
    return t


def _eprecond3(*, nz_dom, nx_dom, dx, dz, dt, nt, f_c, pad, rec_x, rec_z, fd_order, component, params, src_x,
               src_z, src_wavelet, free_surface, eps):
    """fwi/optim_lbfgsb.py:51-100: the Plessix-Mulder multiplier from the
    forward energy of force sources, built on the device."""
    from ..solver import Solver
    sx = np.atleast_1d(np.asarray(src_x)).astype(np.int64)
    sz = np.broadcast_to(np.atleast_1d(np.asarray(src_z)), sx.shape).astype(np.int64)
    rx = np.asarray(rec_x, dtype=np.int32).reshape(-1)
    rz = np.asarray(rec_z, dtype=np.int32).reshape(-1)
    S = Solver(nz_dom, nx_dom, dx, dz, dt, nt, f_c, pad, rx.size, sx.size, fd_order=fd_order,
               free_surface=free_surface, want_gradient=False)
    try:
        S.set_model(*params)
        S.set_receivers(rx, rz)
        S.set_shots(sx, sz, "force", np.asarray(src_wavelet, dtype=np.float32))
        return S.preconditioner("eprecond3", component, eps)
    finally:
        S.close()


def run_multiscale_fwi(*, Vs_init, Vp_init, rho_init, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt,
                       pad, observed, stages: Sequence[dict], component: int = 2, backend: str = "ad",
                       fd_order: int = 8, free_surface: bool = True, src_type: str = "force",
                       block_size: int = 200, auto_scale: Optional[float] = None, K_margin: float = 0.04,
                       cfl_coeff: Optional[float] = None, vs_bounds: Optional[tuple] = None,
                       vp_bounds: Optional[tuple] = None, rho_bounds: Optional[tuple] = None,
                       plateau_window: Optional[int] = None, plateau_rel_tol: float = 1e-3,
                       save_dir: Optional[str] = None, save_every: Optional[int] = None, verbose: bool = True):
    """Multistage L-BFGS-B FWI.  Each stage dict holds f_c (required),
    cutoff, n_iters (50), invert ('vs'), n_taper_pct (0), illumination_eps,
    precon ('illum' | 'eprecond3' | 'none'), grad_smooth_sigma and
    source_taper, as in the reference.  Returns ((Vs, Vp, rho), history)."""
    from scipy.optimize import minimize
    from scipy.signal import butter

    if not stages:
        raise ValueError("`stages` must be a non-empty list")
    observed = np.asarray(observed)
    if auto_scale is None:
        auto_scale = float(1.0 / (np.mean(observed.astype(np.float64) ** 2) + 1e-45))
    if verbose:
        print(f"auto_scale = {auto_scale:.4e}")
    vp_cap = None
    if cfl_coeff is not None:
        vp_cap = cfl_vp_cap(dx=dx, dz=dz, dt=dt, cfl_coeff=cfl_coeff)
    if vp_bounds is not None and vp_bounds[1] is not None:
        vp_cap = vp_bounds[1] if vp_cap is None else min(vp_cap, vp_bounds[1])

    params = tuple(np.asarray(p, dtype=np.float64).copy() for p in (Vs_init, Vp_init, rho_init))
    history = []
    n_cells = nz_dom * nx_dom

    for istage, stage in enumerate(stages):
        f_c = float(stage["f_c"])
        cutoff = stage.get("cutoff", None)
        n_iters = int(stage.get("n_iters", 50))
        invert = stage.get("invert", "vs")
        n_taper = int(float(stage.get("n_taper_pct", 0.0)) * nt)
        illumination_eps = stage.get("illumination_eps", None)
        grad_smooth_sigma = stage.get("grad_smooth_sigma", None)
        source_taper = stage.get("source_taper", None)
        precon = stage.get("precon", "illum")
        if verbose:
            print(f"\nStage {istage + 1}/{len(stages)}  f_c={f_c} Hz  cutoff={cutoff}  invert={invert}  "
                  f"n_iters={n_iters}  backend={backend}")

        src_wavelet = np.asarray(ricker_jax(np.arange(nt) * dt, f_c, 1.5 / f_c), dtype=np.float64)
        sos = butter(6, cutoff, fs=1.0 / dt, output="sos") if cutoff is not None else None

        illumination = None
        if illumination_eps is not None and precon != "none":
            if precon == "illum":
                illumination = compute_illumination_for_stage(
                    nz_dom, nx_dom, dx, dz, dt, nt, f_c, pad, block_size, rec_x, rec_z, fd_order, component,
                    params[0], params[1], params[2], src_x, src_z, src_wavelet, eps=illumination_eps)
            elif precon == "eprecond3":
                illumination = _eprecond3(nz_dom=nz_dom, nx_dom=nx_dom, dx=dx, dz=dz, dt=dt, nt=nt, f_c=f_c,
                                          pad=pad, rec_x=rec_x, rec_z=rec_z, fd_order=fd_order,
                                          component=component, params=params, src_x=src_x, src_z=src_z,
                                          src_wavelet=src_wavelet, free_surface=free_surface,
                                          eps=illumination_eps)
            else:
                raise ValueError(f"unknown precon={precon!r}; use 'illum', 'eprecond3', or 'none'")

        active = _active_keys(invert)
        scales = _block_scales(params)

        def pack(p):
            return np.concatenate([(p[_KEY_TO_IDX[k]] / scales[_KEY_TO_IDX[k]]).ravel() for k in active])

        def unpack(x, base=params):
            full = list(base)
            off = 0
            for k in active:
                i = _KEY_TO_IDX[k]
                full[i] = (x[off:off + n_cells] * scales[i]).reshape(nz_dom, nx_dom)
                off += n_cells
            return tuple(full)

        bounds = []
        for k in active:
            lohi = {"Vs": vs_bounds, "Vp": vp_bounds, "rho": rho_bounds}[k]
            sc = scales[_KEY_TO_IDX[k]]
            lo, hi = (None, None) if lohi is None else lohi
            bounds.extend([(None if lo is None else float(lo) / sc, None if hi is None else float(hi) / sc)]
                          * n_cells)

        x0 = pack(params)
        plateau = _Plateau(plateau_window, plateau_rel_tol)
        stage_dir = os.path.join(save_dir, f"stage{istage + 1}") if save_dir is not None else None
        if stage_dir is not None and save_every is not None:
            os.makedirs(stage_dir, exist_ok=True)
            np.savez_compressed(os.path.join(stage_dir, "epoch_0000.npz"), Vs=params[0], Vp=params[1],
                                rho=params[2], iter=0, loss=float("nan"))
        eval_count, iter_count = [0], [0]
        loss_history: list = []
        last_x = [x0.copy()]

        def projected_host(x):
            return tuple(t.cpu().numpy() for t in _project(unpack(np.asarray(x)), K_margin, vp_cap))

        def f_and_g(x):
            eval_count[0] += 1
            last_x[0] = x.copy()
            t = _project(unpack(x), K_margin, vp_cap)
            (g_vs, g_vp, g_rho), loss = compute_gradient(
                backend, Vs=t[0], Vp=t[1], rho=t[2], src_x=src_x, src_z=src_z, src_wavelet=src_wavelet,
                observed=observed, rec_x=rec_x, rec_z=rec_z, nx_dom=nx_dom, nz_dom=nz_dom, dx=dx, dz=dz, dt=dt,
                nt=nt, fc=f_c, pad=pad, component=component, invert=invert, scale=auto_scale, sos=sos,
                n_taper=n_taper, fd_order=fd_order, free_surface=free_surface, src_type=src_type,
                block_size=block_size, grad_smooth_sigma=grad_smooth_sigma, source_taper=source_taper,
                illumination=illumination)
            full = (g_vs, g_vp, g_rho)
            g_scaled = np.concatenate([(full[_KEY_TO_IDX[k]] * scales[_KEY_TO_IDX[k]]).ravel()
                                       for k in active]).astype(np.float64)
            loss_history.append(float(loss))
            if verbose:
                print(f"  iter {eval_count[0]:4d}  loss={float(loss):.4e}  |g|_inf={np.max(np.abs(g_scaled)):.3e}")
            if stage_dir is not None and save_every is not None and eval_count[0] % save_every == 0:
                p = projected_host(x)
                np.savez_compressed(os.path.join(stage_dir, f"eval_{eval_count[0]:04d}.npz"), Vs=p[0], Vp=p[1],
                                    rho=p[2], eval=eval_count[0], loss=float(loss))
            if plateau.push(float(loss)):
                if verbose:
                    print("  plateau detected: stage stops")
                raise _PlateauStop()
            return float(loss), g_scaled

        def iter_callback(xk):
            iter_count[0] += 1
            if stage_dir is None or save_every is None or iter_count[0] % save_every != 0:
                return
            p = projected_host(xk)
            np.savez_compressed(os.path.join(stage_dir, f"epoch_{iter_count[0]:04d}.npz"), Vs=p[0], Vp=p[1],
                                rho=p[2], iter=iter_count[0],
                                loss=float(loss_history[-1]) if loss_history else float("nan"))

        t0 = time.time()
        try:
            res = minimize(f_and_g, x0, method="L-BFGS-B", jac=True, bounds=bounds, callback=iter_callback,
                           options=dict(maxiter=n_iters, gtol=0.0, ftol=1e-30))
            res_x, res_fun, ok = res.x, float(res.fun), bool(res.success)
        except _PlateauStop:
            res_x = last_x[0]
            res_fun = loss_history[-1] if loss_history else float("nan")
            ok = False
        t_stage = time.time() - t0
        params = projected_host(res_x)
        history.append(dict(stage=istage, f_c=f_c, cutoff=cutoff, invert=invert, n_iters_max=n_iters,
                            n_evals=eval_count[0], loss_history=np.array(loss_history), final_loss=res_fun,
                            success=ok, time_s=t_stage, Vs=params[0].copy(), Vp=params[1].copy(),
                            rho=params[2].copy()))
        if verbose:
            print(f"  Stage {istage + 1} done in {t_stage:.1f}s  final_loss={res_fun:.4e}  success={ok}")
        if save_dir is not None:
            os.makedirs(stage_dir, exist_ok=True)
            np.savez_compressed(os.path.join(stage_dir, "params.npz"), Vs=params[0], Vp=params[1], rho=params[2],
                                loss_history=np.array(loss_history), f_c=f_c, cutoff=cutoff, invert=invert,
                                backend=backend)
    return params, history
