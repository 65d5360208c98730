"""The wiring of stfwi_b200.jax_bridge (jax.custom_vjp over the C ABI)
against a stand-in for the three JAX names it uses (custom_vjp,
pure_callback, ShapeDtypeStruct) and a solver stand-in with a known
quadratic misfit, on the CPU: the value is the solver's summed misfit, the
forward rule's residuals are its gradients, the backward rule scales them
by the cotangent, and dJ/drho is passed through only when the solver keeps
the velocity history.  JAX itself is not installed here."""
import sys
import types

import numpy as np
import pytest


def _fake_jax():
    jax = types.ModuleType("jax")
    jnp = types.ModuleType("jax.numpy")
    jnp.float64 = np.float64
    jnp.zeros_like = np.zeros_like

    class ShapeDtypeStruct:
        def __init__(self, shape, dtype):
            self.shape, self.dtype = tuple(shape), dtype

    def pure_callback(f, out, *args):
        res = f(*[np.asarray(a) for a in args])
        assert len(res) == len(out)
        for r, o in zip(res, out):   # the callback must return what it declared
            assert np.shape(r) == o.shape and np.asarray(r).dtype == o.dtype, (np.shape(r), o.shape)
        return tuple(np.asarray(r) for r in res)

    class custom_vjp:
        def __init__(self, f):
            self.f = f

        def defvjp(self, fwd, bwd):
            self.fwd, self.bwd = fwd, bwd

        def __call__(self, *a):
            return self.f(*a)

    jax.custom_vjp, jax.pure_callback, jax.ShapeDtypeStruct, jax.numpy = custom_vjp, pure_callback, ShapeDtypeStruct, jnp
    return jax, jnp


class _QuadSolver:
    """J = 0.5 |vs - a|^2 + 0.25 |vp - b|^2 + 0.125 |rho - c|^2 split over two
    shots; its gradient is exact in closed form."""

    def __init__(self, density):
        self.nz_dom, self.nx_dom, self.density = 3, 4, density
        rng = np.random.default_rng(0)
        self.a, self.b, self.c = (rng.standard_normal((3, 4)) for _ in range(3))
        self.calls = []

    def set_model(self, vs, vp, rho):
        assert vs.dtype == np.float32 and vs.shape == (3, 4)
        self.m = (vs.astype(np.float64), vp.astype(np.float64), rho.astype(np.float64))
        self.calls.append("set_model")

    def forward(self, store=False):
        assert store
        self.calls.append("forward")

    def misfit(self, obs, component, scale, sos, n_taper):
        vs, vp, rho = self.m
        j = 0.5 * np.sum((vs - self.a) ** 2) + 0.25 * np.sum((vp - self.b) ** 2) + 0.125 * np.sum((rho - self.c) ** 2)
        return np.array([0.25 * j, 0.75 * j]) * scale

    def gradient(self, exact=True):
        vs, vp, rho = self.m
        g = (vs - self.a, 0.5 * (vp - self.b), 0.25 * (rho - self.c) if self.density else np.zeros((3, 4)))
        return {"exact": g}


@pytest.mark.parametrize("density", [False, True])
def test_custom_vjp_wiring(monkeypatch, density):
    jax, jnp = _fake_jax()
    monkeypatch.setitem(sys.modules, "jax", jax)
    monkeypatch.setitem(sys.modules, "jax.numpy", jnp)
    from stfwi_b200.jax_bridge import make_jax_misfit
    S = _QuadSolver(density)
    f = make_jax_misfit(S, np.zeros((2, 5, 6)), component=1, scale=2.0)
    rng = np.random.default_rng(1)
    vs, vp, rho = (rng.standard_normal((3, 4)).astype(np.float32) for _ in range(3))
    m64 = [x.astype(np.float64) for x in (vs, vp, rho)]
    j = 2.0 * (0.5 * np.sum((m64[0] - S.a) ** 2) + 0.25 * np.sum((m64[1] - S.b) ** 2)
               + 0.125 * np.sum((m64[2] - S.c) ** 2))
    assert abs(float(f(vs, vp, rho)) - j) < 1e-12 * abs(j)
    loss, res = f.fwd(vs, vp, rho)
    assert abs(float(loss) - j) < 1e-12 * abs(j)
    gvs, gvp, grho = f.bwd(res, 3.0)
    assert np.allclose(gvs, 3.0 * (m64[0] - S.a)) and np.allclose(gvp, 3.0 * 0.5 * (m64[1] - S.b))
    assert np.allclose(grho, 3.0 * 0.25 * (m64[2] - S.c)) if density else not np.any(grho)
    assert S.calls[:2] == ["set_model", "forward"]
