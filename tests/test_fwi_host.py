"""Host-side pieces of the reference-signature API (CPU)."""
import numpy as np
import pytest

from oracle import oracle as O


def test_filters_and_smoothing_match_the_oracle():
    from scipy.signal import butter
    from stfwi_b200 import fwi
    rng = np.random.default_rng(1)
    x = rng.standard_normal((400, 7))
    sos = butter(6, 3.0, fs=1 / 0.002, output="sos")
    np.testing.assert_allclose(fwi.sosfilt(x, sos), O.sosfilt(x, sos), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(fwi.cosine_taper_end(x, 40), O.cosine_taper_end(x, 40), rtol=1e-12)
    assert np.array_equal(fwi.cosine_taper_end(x, 0), x)
    f = rng.standard_normal((30, 41))
    np.testing.assert_allclose(fwi.gaussian_smooth_2d(f, 1.5), O.gaussian_smooth_2d(f, 1.5), rtol=1e-12)


def test_ricker_matches_the_reference_formula():
    from stfwi_b200 import fwi
    from stfwi_b200 import models as Mo
    t = np.arange(500) * 0.002
    w = fwi.ricker_jax(t, 6.0, 0.25)
    np.testing.assert_allclose(w, O.ricker(t, 6.0, 0.25), rtol=1e-14)
    np.testing.assert_allclose(w, Mo.ricker(t, 6.0, 0.25), rtol=1e-14)
    assert abs(w.max() - 1.0) < 1e-3


def test_layered_fault_model_ranges():
    from stfwi_b200 import models as Mo
    vs, vp, rho = Mo.layered_fault_model(152, 500, seed=3)
    assert vs.shape == (152, 500) and vs.dtype == np.float32
    assert 1500 <= vp.min() and vp.max() <= 4700
    assert 800 <= vs.min() and vs.max() <= 2750
    assert 1700 <= rho.min() and rho.max() <= 2600
    assert np.all(vp / vs >= 1.2 - 1e-6)
    vs0, vp0, rho0 = Mo.smooth_initial(vs, vp, rho, 10.0)
    assert np.abs(np.diff(vs0, axis=0)).max() < np.abs(np.diff(vs, axis=0)).max()
    # config 1 / 2 are stable: CFL number below 1
    for cfg in (Mo.CONFIG1, Mo.CONFIG2):
        assert Mo.cfl_number(4700, cfg["dt"], cfg["dx"], cfg["dz"], cfg["fd_order"]) < 0.7


def test_host_projection_matches_oracle_and_reference_rules():
    """fwi/projections.py:67-117: Vp capped first, then Vs <= Vp / r, floors."""
    from oracle import oracle as O
    from stfwi_b200 import fwi
    rng = np.random.default_rng(4)
    vs = rng.uniform(-10.0, 3000.0, (20, 30))
    vp = rng.uniform(100.0, 5000.0, (20, 30))
    rho = rng.uniform(-1.0, 2500.0, (20, 30))
    for cap in (None, 4000.0):
        got = fwi.project_velocity(vs, vp, rho, K_margin=0.04, vp_cap=cap)
        ref = O.project_velocity(vs, vp, rho, K_margin=0.04, vp_cap=cap)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        r = fwi.k_safe_ratio(0.04)
        above_floor = got[0] > 1e-3
        assert np.all(got[0][above_floor] <= got[1][above_floor] / r)
        assert np.all(got[0] >= 1e-3) and np.all(got[2] >= 1e-3)
        if cap is not None:
            assert np.all(got[1] <= cap)
    assert abs(fwi.k_safe_ratio(0.0) - 2 / np.sqrt(3)) < 1e-15
    assert fwi.cfl_vp_cap(20.0, 10.0, 1e-3, 0.5) == 0.5 * 10.0 / 1e-3


def test_driver_plateau_and_block_helpers():
    """The multiscale driver's stage helpers: the plateau window (the
    reference's rule of fwi/optim_lbfgsb.py:117-134), the planes each
    `invert` mode moves, per-plane scales and stage parsing."""
    from stfwi_b200.fwi import optim_lbfgsb as D
    p = D.LossWindow(3, 1e-3)
    stops = [p.push(v) for v in (10, 9, 8, 7, 6, 5)]   # still dropping: no stop
    assert stops == [False] * 6
    q = D.LossWindow(3, 1e-3)
    stops = [q.push(v) for v in (5.0, 5.0, 5.0, 5.0, 5.0, 4.999)]   # last 3 vs previous 3 within 0.1 %
    assert stops == [False] * 5 + [True]
    assert D.LossWindow(None, 1e-3).push(1.0) is False
    assert D.planes_of("vs") == (0,) and D.planes_of("all") == (0, 1, 2)
    with pytest.raises(ValueError):
        D.planes_of("rho")
    s = D.plane_scales(np.stack([np.array([[-3.0, 2.0]]), np.zeros((1, 2)), np.array([[1.0, 5.0]])]))
    assert s.tolist() == [3.0, 1e-12, 5.0]
    spec = D.StageSpec.from_dict(dict(f_c=3.0, cutoff=2.0, n_iters=4))
    assert (spec.invert, spec.precon, spec.n_taper_pct) == ("vs", "illum", 0.0)
    with pytest.raises(ValueError):
        D.StageSpec.from_dict(dict(f_c=3.0, precon="hessian"))
    with pytest.raises(KeyError):
        D.StageSpec.from_dict(dict(cutoff=3.0))
