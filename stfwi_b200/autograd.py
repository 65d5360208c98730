"""torch.autograd bindings of the CUDA path.

``elastic_forward(vs, vp, rho, solver)`` returns the receiver traces
[nshot, 4, nt, nrec] (vx, vz, exx, ezz) as a differentiable function of Vs and
Vp: its backward feeds the incoming trace gradients to the adjoint as
receiver sources and returns the exact gradient (the transpose of the FP32
forward, checkpointed if the solver was planned that way).
``elastic_misfit(...)`` fuses the residual preparation (filter, taper, FP64
misfit) into the forward and returns the scalar loss.

A solver keeps the history of its last storing forward only: a backward
must follow its own forward before the solver runs another one (checked).
The density gradient needs a solver made with density=True (it keeps the
velocities in the history); otherwise rho.requires_grad raises.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Solver


def _check(solver, rho):
    if not isinstance(solver, Solver):
        raise TypeError("solver must be a stfwi_b200.Solver")
    if rho.requires_grad and not getattr(solver, "density", False):
        raise NotImplementedError("the density gradient needs a Solver created with density=True")


class _Forward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vs, vp, rho, solver):
        _check(solver, rho)
        solver.set_model(vs, vp, rho)
        solver.forward(store=True)
        solver._version = getattr(solver, "_version", 0) + 1
        ctx.solver, ctx.version, ctx.dtypes = solver, solver._version, (vs.dtype, vp.dtype, rho.dtype)
        out = torch.empty((solver.nshot, 4, solver.nt, solver.nrec), dtype=torch.float32, device=vs.device)
        solver.records(out=out)
        return out

    @staticmethod
    def backward(ctx, grad_rec):
        S = ctx.solver
        if S._version != ctx.version:
            raise RuntimeError("the solver ran another forward before this backward")
        S.set_adjoint_sources(grad_rec.detach().to(torch.float32).contiguous())
        g = torch.empty((1, 3, S.nz_dom, S.nx_dom), dtype=torch.float64, device=grad_rec.device)
        S.gradient(exact=True, out=g)
        grho = g[0, 2].to(ctx.dtypes[2]) if S.density else None
        return g[0, 0].to(ctx.dtypes[0]), g[0, 1].to(ctx.dtypes[1]), grho, None


class _Misfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vs, vp, rho, solver, observed, component, scale, sos, n_taper, nshot_norm):
        _check(solver, rho)
        solver.set_model(vs, vp, rho)
        solver.forward(store=True)
        solver._version = getattr(solver, "_version", 0) + 1
        mis = torch.zeros(solver.nshot, dtype=torch.float64, device=vs.device)
        solver.misfit(observed, component, scale, sos, n_taper, nshot_norm=nshot_norm, out=mis)
        ctx.solver, ctx.version, ctx.dtypes = solver, solver._version, (vs.dtype, vp.dtype, rho.dtype)
        return mis.sum()

    @staticmethod
    def backward(ctx, gout):
        S = ctx.solver
        if S._version != ctx.version:
            raise RuntimeError("the solver ran another forward before this backward")
        g = torch.empty((1, 3, S.nz_dom, S.nx_dom), dtype=torch.float64, device=gout.device)
        S.gradient(exact=True, out=g)
        grho = (gout * g[0, 2]).to(ctx.dtypes[2]) if S.density else None
        return ((gout * g[0, 0]).to(ctx.dtypes[0]), (gout * g[0, 1]).to(ctx.dtypes[1]), grho,
                None, None, None, None, None, None, None)


def elastic_forward(vs, vp, rho, solver):
    """Receiver traces [nshot, 4, nt, nrec], differentiable in vs and vp."""
    return _Forward.apply(vs, vp, rho, solver)


def elastic_misfit(vs, vp, rho, solver, observed, component=1, scale=1.0, sos=None, n_taper=0,
                   nshot_norm=0):
    """scale/nshot * sum_shots mean_{t,r}(F T (pred - obs))^2 (FP64 scalar),
    differentiable in vs and vp."""
    sos = None if sos is None else np.asarray(sos, dtype=np.float64)
    return _Misfit.apply(vs, vp, rho, solver, observed, int(component), float(scale), sos, int(n_taper),
                         int(nshot_norm))
