"""Multistage L-BFGS-B FWI with the reference's entry point
``run_multiscale_fwi`` (fwi/optim_lbfgsb.py:137-473), on the CUDA path.

The work is organised around one object, :class:`MultiscaleDriver`, which
owns the model as a single device tensor ``[3, nz, nx]`` (Vs, Vp, rho; FP64)
and runs every stage of the schedule against it:

* the optimiser (SciPy's L-BFGS-B) sees a host vector holding the planes
  being inverted, each divided by its own largest magnitude at the start of
  the stage; the driver moves that vector into the device model, projects
  the model onto the feasible set in place (fwi/projections.py:67-117, a
  device kernel), and asks the GPU for the misfit and the gradient, which
  it returns scaled the same way;
* bounds are per cell, expressed in the scaled space (``Bounds`` arrays);
* a stage stops early when the mean of the last ``w`` misfits is not at
  least ``rel_tol`` below the mean of the ``w`` before them (the
  reference's plateau rule, fwi/optim_lbfgsb.py:117-134);
* the stage preconditioner (illumination or eprecond3) is built once per
  stage on the device from the current model.

Stage dictionaries, the returned history and the checkpoint file names are
the reference's, so scripts written for it run unchanged.
"""
from __future__ import annotations

import dataclasses
import os
import time
from collections import deque
from typing import Optional, Sequence

import numpy as np

from .forward import ricker_jax
from .gradient import compute_gradient
from .illumination import compute_illumination_for_stage
from .projections import cfl_vp_cap, project_velocity_device

PLANE_NAMES = ("Vs", "Vp", "rho")
# planes the optimiser moves for each `invert` mode (fwi/gradient.py:250-257)
INVERT_PLANES = {"vs": (0,), "vs_vp": (0, 1), "all": (0, 1, 2)}


def planes_of(invert):
    """Indices into (Vs, Vp, rho) of the planes that `invert` optimises."""
    try:
        return INVERT_PLANES[invert]
    except KeyError:
        raise ValueError(f"invert must be one of {sorted(INVERT_PLANES)}, got {invert!r}") from None


def plane_scales(model):
    """Largest magnitude of each plane of a [3, nz, nx] array, floored at
    1e-12 so that an all-zero plane still scales."""
    m = np.abs(np.asarray(model, dtype=np.float64)).reshape(len(model), -1).max(axis=1)
    return np.maximum(m, 1e-12)


class LossWindow:
    """Plateau detector over the misfits of one stage.

    Keeps the last ``2 w`` values; once it holds that many, ``push`` reports
    a plateau when sum(newest w) >= (1 - rel_tol) * sum(older w).  With
    ``w`` None or 0 it never fires."""

    def __init__(self, w: Optional[int], rel_tol: float):
        self.w = int(w or 0)
        self.rel_tol = float(rel_tol)
        self.values = deque(maxlen=max(2 * self.w, 1))

    def push(self, loss: float) -> bool:
        self.values.append(float(loss))
        if self.w <= 0 or len(self.values) < 2 * self.w:
            return False
        v = np.fromiter(self.values, dtype=np.float64)
        return bool(v[self.w:].sum() >= (1.0 - self.rel_tol) * v[:self.w].sum())


class _StageStopped(Exception):
    """Raised from the objective to end a stage on a plateau."""


@dataclasses.dataclass(frozen=True)
class StageSpec:
    """One entry of the stage schedule (the reference's stage-dict keys)."""
    f_c: float
    cutoff: Optional[float] = None
    n_iters: int = 50
    invert: str = "vs"
    n_taper_pct: float = 0.0
    illumination_eps: Optional[float] = None
    precon: str = "illum"
    grad_smooth_sigma: Optional[float] = None
    source_taper: Optional[np.ndarray] = None

    @staticmethod
    def from_dict(d):
        known = {f.name for f in dataclasses.fields(StageSpec)}
        kw = {k: d[k] for k in known if k in d}
        if "f_c" not in kw:
            raise KeyError("every stage needs 'f_c'")
        spec = StageSpec(**kw)
        planes_of(spec.invert)   # validates
        if spec.precon not in ("illum", "eprecond3", "none"):
            raise ValueError(f"precon must be 'illum', 'eprecond3' or 'none', got {spec.precon!r}")
        return spec


class _Checkpoints:
    """Model snapshots of one stage: epoch_NNNN.npz (per optimiser
    iteration), eval_NNNN.npz (per misfit evaluation) and params.npz (the
    stage result), the reference's file names."""

    def __init__(self, save_dir, stage_no, every):
        self.dir = os.path.join(save_dir, f"stage{stage_no}") if save_dir is not None else None
        self.every = every

    @property
    def periodic(self):
        return self.dir is not None and self.every is not None

    def _write(self, name, **arrays):
        os.makedirs(self.dir, exist_ok=True)
        np.savez_compressed(os.path.join(self.dir, name), **arrays)

    def model(self, name, model, **extra):
        self._write(name, Vs=model[0], Vp=model[1], rho=model[2], **extra)

    def result(self, model, **extra):
        if self.dir is not None:
            self.model("params.npz", model, **extra)


class MultiscaleDriver:
    """Runs a stage schedule of L-BFGS-B on a device-resident model.

    Geometry, acquisition and the inversion options are fixed at
    construction; :meth:`run` takes the list of stage dictionaries."""

    def __init__(self, *, model, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt, pad, observed,
                 component, backend, fd_order, free_surface, src_type, block_size, auto_scale, K_margin, vp_cap,
                 bounds, plateau_window, plateau_rel_tol, save_dir, save_every, verbose):
        import torch
        self.torch = torch
        self.model = torch.as_tensor(np.stack([np.asarray(p, dtype=np.float64) for p in model]),
                                     device="cuda").contiguous()
        self.acq = dict(src_x=src_x, src_z=src_z, rec_x=rec_x, rec_z=rec_z, nx_dom=nx_dom, nz_dom=nz_dom,
                        dx=dx, dz=dz, dt=dt, nt=nt, pad=pad)
        self.shape = (int(nz_dom), int(nx_dom))
        self.observed = observed
        self.component, self.backend, self.fd_order = component, backend, fd_order
        self.free_surface, self.src_type, self.block_size = free_surface, src_type, block_size
        self.auto_scale, self.K_margin, self.vp_cap = auto_scale, K_margin, vp_cap
        self.value_bounds = bounds                       # per plane: (lo, hi) or None
        self.plateau = (plateau_window, plateau_rel_tol)
        self.save_dir, self.save_every, self.verbose = save_dir, save_every, verbose

    # ----------------------------------------------------------------- model
    def _project(self, model):
        """Feasibility projection of a [3, nz, nx] device tensor, in place."""
        project_velocity_device(model[0], model[1], model[2], K_margin=self.K_margin, vp_cap=self.vp_cap)
        return model

    def _trial_model(self, x, planes, scales):
        """The stage's model with the optimiser's vector written into the
        active planes, projected (a new device tensor)."""
        m = self.model.clone()
        xs = self.torch.as_tensor(np.asarray(x, dtype=np.float64).reshape(len(planes), *self.shape),
                                  device=m.device)
        for k, p in enumerate(planes):
            m[p] = xs[k] * float(scales[p])
        return self._project(m)

    def host_model(self, model=None):
        m = self.model if model is None else model
        return tuple(a.cpu().numpy() for a in m)

    # ----------------------------------------------------------------- stage pieces
    def _preconditioner(self, spec, wavelet):
        if spec.illumination_eps is None or spec.precon == "none":
            return None
        a = self.acq
        if spec.precon == "illum":
            Vs, Vp, rho = self.host_model()
            return np.asarray(compute_illumination_for_stage(
                a["nz_dom"], a["nx_dom"], a["dx"], a["dz"], a["dt"], a["nt"], spec.f_c, a["pad"],
                self.block_size, a["rec_x"], a["rec_z"], self.fd_order, self.component, Vs, Vp, rho,
                a["src_x"], a["src_z"], wavelet, eps=spec.illumination_eps))
        return self._eprecond3(spec, wavelet)

    def _eprecond3(self, spec, wavelet):
        """Plessix-Mulder multiplier (fwi/optim_lbfgsb.py:51-100) from the
        forward energy of force shots, built on the device."""
        from ..solver import Solver
        a = self.acq
        sx = np.atleast_1d(np.asarray(a["src_x"])).astype(np.int64)
        sz = np.broadcast_to(np.atleast_1d(np.asarray(a["src_z"])), sx.shape).astype(np.int64)
        rx = np.asarray(a["rec_x"], dtype=np.int32).reshape(-1)
        rz = np.asarray(a["rec_z"], dtype=np.int32).reshape(-1)
        S = Solver(a["nz_dom"], a["nx_dom"], a["dx"], a["dz"], a["dt"], a["nt"], spec.f_c, a["pad"], rx.size,
                   sx.size, fd_order=self.fd_order, free_surface=self.free_surface, want_gradient=False)
        try:
            S.set_model(self.model[0], self.model[1], self.model[2])
            S.set_receivers(rx, rz)
            S.set_shots(sx, sz, "force", np.asarray(wavelet, dtype=np.float32))
            return S.preconditioner("eprecond3", self.component, spec.illumination_eps)
        finally:
            S.close()

    def _scaled_bounds(self, planes, scales):
        from scipy.optimize import Bounds
        n = self.shape[0] * self.shape[1]
        lo = np.full(len(planes) * n, -np.inf)
        hi = np.full(len(planes) * n, np.inf)
        for k, p in enumerate(planes):
            b = self.value_bounds[p]
            if b is None:
                continue
            if b[0] is not None:
                lo[k * n:(k + 1) * n] = float(b[0]) / scales[p]
            if b[1] is not None:
                hi[k * n:(k + 1) * n] = float(b[1]) / scales[p]
        return Bounds(lo, hi)

    # ----------------------------------------------------------------- one stage
    def run_stage(self, no, spec: StageSpec):
        from scipy.optimize import minimize
        from scipy.signal import butter
        a = self.acq
        nt, dt = a["nt"], a["dt"]
        if self.verbose:
            print(f"\nStage {no + 1}: f_c={spec.f_c} Hz cutoff={spec.cutoff} invert={spec.invert} "
                  f"n_iters={spec.n_iters} backend={self.backend}")
        wavelet = np.asarray(ricker_jax(np.arange(nt) * dt, spec.f_c, 1.5 / spec.f_c), dtype=np.float64)
        sos = None if spec.cutoff is None else butter(6, spec.cutoff, fs=1.0 / dt, output="sos")
        n_taper = int(float(spec.n_taper_pct) * nt)
        illumination = self._preconditioner(spec, wavelet)

        planes = planes_of(spec.invert)
        scales = plane_scales(self.host_model())
        host = self.model.cpu().numpy()
        x0 = np.concatenate([(host[p] / scales[p]).ravel() for p in planes])
        window = LossWindow(*self.plateau)
        ck = _Checkpoints(self.save_dir, no + 1, self.save_every)
        if ck.periodic:
            ck.model("epoch_0000.npz", host, iter=0, loss=float("nan"))
        losses, last = [], [x0]
        counters = {"evals": 0, "iters": 0}

        def objective(x):
            counters["evals"] += 1
            last[0] = np.array(x, copy=True)
            m = self._trial_model(x, planes, scales)
            grads, loss = compute_gradient(
                self.backend, Vs=m[0], Vp=m[1], rho=m[2], src_wavelet=wavelet, observed=self.observed,
                fc=spec.f_c, component=self.component, invert=spec.invert, scale=self.auto_scale, sos=sos,
                n_taper=n_taper, fd_order=self.fd_order, free_surface=self.free_surface,
                src_type=self.src_type, block_size=self.block_size, grad_smooth_sigma=spec.grad_smooth_sigma,
                source_taper=spec.source_taper, illumination=illumination, **a)
            g = np.concatenate([np.asarray(grads[p], dtype=np.float64).ravel() * scales[p] for p in planes])
            loss = float(loss)
            losses.append(loss)
            if self.verbose:
                print(f"  eval {counters['evals']:4d}  loss={loss:.4e}  |g|_inf={np.abs(g).max():.3e}")
            if ck.periodic and counters["evals"] % ck.every == 0:
                ck.model(f"eval_{counters['evals']:04d}.npz", self.host_model(m), eval=counters["evals"],
                         loss=loss)
            if window.push(loss):
                if self.verbose:
                    print("  plateau: stage ends")
                raise _StageStopped
            return loss, g

        def on_iteration(xk):
            counters["iters"] += 1
            if ck.periodic and counters["iters"] % ck.every == 0:
                ck.model(f"epoch_{counters['iters']:04d}.npz", self.host_model(self._trial_model(xk, planes, scales)),
                         iter=counters["iters"], loss=losses[-1] if losses else float("nan"))

        t0 = time.time()
        try:
            r = minimize(objective, x0, jac=True, method="L-BFGS-B", bounds=self._scaled_bounds(planes, scales),
                         callback=on_iteration, options=dict(maxiter=spec.n_iters, gtol=0.0, ftol=1e-30))
            x_end, final, success = r.x, float(r.fun), bool(r.success)
        except _StageStopped:
            x_end, final, success = last[0], (losses[-1] if losses else float("nan")), False
        elapsed = time.time() - t0
        self.model = self._trial_model(x_end, planes, scales)
        model = self.host_model()
        rec = dict(stage=no, f_c=spec.f_c, cutoff=spec.cutoff, invert=spec.invert, n_iters_max=spec.n_iters,
                   n_evals=counters["evals"], loss_history=np.array(losses), final_loss=final, success=success,
                   time_s=elapsed, Vs=model[0].copy(), Vp=model[1].copy(), rho=model[2].copy())
        ck.result(model, loss_history=np.array(losses), f_c=spec.f_c, cutoff=spec.cutoff, invert=spec.invert,
                  backend=self.backend)
        if self.verbose:
            print(f"  stage {no + 1}: {elapsed:.1f} s, final loss {final:.4e}, success {success}")
        return rec

    def run(self, stages):
        specs = [StageSpec.from_dict(s) for s in stages]
        history = [self.run_stage(k, s) for k, s in enumerate(specs)]
        return self.host_model(), history


def run_multiscale_fwi(*, Vs_init, Vp_init, rho_init, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt,
                       pad, observed, stages: Sequence[dict], component: int = 2, backend: str = "ad",
                       fd_order: int = 8, free_surface: bool = True, src_type: str = "force",
                       block_size: int = 200, auto_scale: Optional[float] = None, K_margin: float = 0.04,
                       cfl_coeff: Optional[float] = None, vs_bounds: Optional[tuple] = None,
                       vp_bounds: Optional[tuple] = None, rho_bounds: Optional[tuple] = None,
                       plateau_window: Optional[int] = None, plateau_rel_tol: float = 1e-3,
                       save_dir: Optional[str] = None, save_every: Optional[int] = None, verbose: bool = True):
    """Multistage L-BFGS-B FWI; returns ((Vs, Vp, rho), history).

    Stage keys: f_c (required), cutoff, n_iters (50), invert ('vs'),
    n_taper_pct (0), illumination_eps, precon ('illum' | 'eprecond3' |
    'none'), grad_smooth_sigma, source_taper.  ``auto_scale`` defaults to
    1 / mean(observed^2); the Vp cap is the tighter of the CFL cap and the
    upper Vp bound."""
    if not stages:
        raise ValueError("`stages` must be a non-empty list")
    observed = np.asarray(observed)
    if auto_scale is None:
        auto_scale = float(1.0 / (np.mean(np.square(observed, dtype=np.float64)) + 1e-45))
    if verbose:
        print(f"auto_scale = {auto_scale:.4e}")
    caps = []
    if cfl_coeff is not None:
        caps.append(cfl_vp_cap(dx=dx, dz=dz, dt=dt, cfl_coeff=cfl_coeff))
    if vp_bounds is not None and vp_bounds[1] is not None:
        caps.append(vp_bounds[1])
    drv = MultiscaleDriver(
        model=(Vs_init, Vp_init, rho_init), src_x=src_x, src_z=src_z, rec_x=rec_x, rec_z=rec_z, nx_dom=nx_dom,
        nz_dom=nz_dom, dx=dx, dz=dz, dt=dt, nt=nt, pad=pad, observed=observed, component=component,
        backend=backend, fd_order=fd_order, free_surface=free_surface, src_type=src_type, block_size=block_size,
        auto_scale=auto_scale, K_margin=K_margin, vp_cap=min(caps) if caps else None,
        bounds=(vs_bounds, vp_bounds, rho_bounds), plateau_window=plateau_window, plateau_rel_tol=plateau_rel_tol,
        save_dir=save_dir, save_every=save_every, verbose=verbose)
    return drv.run(stages)
