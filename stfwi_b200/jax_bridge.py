"""jax.custom_vjp over the same C ABI (optional: needs JAX).

``make_jax_misfit(solver, observed, ...)`` returns a JAX function of
(Vs, Vp, rho) whose value is the FP64 misfit and whose VJP is the exact
gradient from the CUDA adjoint (dJ/drho too when the solver keeps the
velocity history, ``Solver(..., density=True)``; zero otherwise).  The
calls cross into the C ABI through ``jax.pure_callback`` with host arrays.
The outputs are FP64: enable JAX's 64-bit mode
(``jax.config.update("jax_enable_x64", True)``) before calling.
The wiring is tested against a stand-in for ``jax.custom_vjp`` and
``jax.pure_callback`` (tests/test_jax_bridge.py); JAX itself is not
installed in the build environment.
"""
from __future__ import annotations

import numpy as np


def make_jax_misfit(solver, observed, component=1, scale=1.0, sos=None, n_taper=0):
    try:
        import jax
        import jax.numpy as jnp
    except ImportError as e:  # pragma: no cover
        raise ImportError("make_jax_misfit needs jax") from e
    obs = np.asarray(observed, dtype=np.float32)
    shape = (solver.nz_dom, solver.nx_dom)

    def _value_and_grad_host(vs, vp, rho):
        solver.set_model(np.asarray(vs, np.float32), np.asarray(vp, np.float32), np.asarray(rho, np.float32))
        solver.forward(store=True)
        loss = solver.misfit(obs, component, scale, sos, n_taper).sum()
        g = solver.gradient(exact=True)["exact"]
        grho = np.asarray(g[2], np.float64) if density else np.zeros(shape)
        return np.float64(loss), np.asarray(g[0], np.float64), np.asarray(g[1], np.float64), grho

    density = bool(getattr(solver, "density", False))

    def _call(vs, vp, rho):
        out = (jax.ShapeDtypeStruct((), jnp.float64), jax.ShapeDtypeStruct(shape, jnp.float64),
               jax.ShapeDtypeStruct(shape, jnp.float64), jax.ShapeDtypeStruct(shape, jnp.float64))
        return jax.pure_callback(_value_and_grad_host, out, vs, vp, rho)

    @jax.custom_vjp
    def misfit(vs, vp, rho):
        return _call(vs, vp, rho)[0]

    def fwd(vs, vp, rho):
        loss, gvs, gvp, grho = _call(vs, vp, rho)
        return loss, (gvs, gvp, grho)

    def bwd(res, g):
        gvs, gvp, grho = res
        return (g * gvs).astype(gvs.dtype), (g * gvp).astype(gvp.dtype), (g * grho).astype(grho.dtype)

    misfit.defvjp(fwd, bwd)
    return misfit
