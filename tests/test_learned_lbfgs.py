"""The lockstep L-BFGS of the learned-preconditioner experiments on the
CPU: a batch whose 'gradient evaluation' is a seeded quadratic stands in
for the solver handles."""
import numpy as np


class _QuadBatch:
    """f = 1/2 sum a (x - x*)^2 per slot, gradient a (x - x*)."""

    def __init__(self, targets, curv):
        self.targets, self.curv, self.evals = targets, curv, 0

    def evaluate(self, xs):
        out = []
        for k, x in enumerate(xs):
            if x is None:
                out.append(None)
                continue
            r = x - self.targets[k]
            self.evals += 1
            out.append((0.5 * float(np.sum(self.curv[k] * r * r)), self.curv[k] * r))
        return out


def test_lbfgs_converges_in_lockstep_and_respects_bounds():
    from stfwi_b200.learned.inversion import lbfgs, project_vs, run_lockstep
    rng = np.random.default_rng(0)
    shape = (12, 20)
    vp = np.full(shape, 3000.0)
    targets = [rng.uniform(1000, 2000, shape) for _ in range(3)]
    targets[2][0, 0] = 5000.0                           # outside the bound Vp / 1.2 = 2500
    curv = [rng.uniform(0.5, 2.0, shape) for _ in range(3)]
    batch = _QuadBatch(targets, curv)
    hist = [[] for _ in range(3)]
    gens = [lbfgs(np.full(shape, 1500.0), vp, np.ones(shape), n_iter=40, step0=200.0,
                  record=lambda x, f, g, k=k: hist[k].append(f)) for k in range(3)]
    gens.append(None)                                   # an idle slot
    clock = {"t": 0.0}
    xs, rounds = run_lockstep(batch, gens, clock)
    assert xs[3] is None and len(rounds) >= 2 and clock["t"] > 0
    for k in range(2):
        assert np.abs(xs[k] - targets[k]).max() < 1.0, k
        assert all(b <= a for a, b in zip(hist[k], hist[k][1:]))   # monotone accepted misfits
    assert xs[2][0, 0] == 2500.0                        # projected onto the bound
    assert np.allclose(xs[2], project_vs(xs[2], vp))


def test_lbfgs_stops_when_asked():
    from stfwi_b200.learned.inversion import lbfgs, run_lockstep
    shape = (4, 4)
    batch = _QuadBatch([np.full(shape, 1800.0)], [np.ones(shape)])
    seen = []
    gen = lbfgs(np.full(shape, 1500.0), np.full(shape, 3000.0), np.ones(shape), n_iter=50, step0=100.0,
                record=lambda x, f, g: seen.append(f), stop=lambda x, f: f < 1e4)
    run_lockstep(batch, [gen])
    assert seen[-1] < 1e4 and all(f >= 1e4 for f in seen[:-1])


def test_lbfgs_restarts_after_a_failed_line_search():
    """A pseudo-Huber misfit is almost linear far from its minimum, so the
    curvature pairs gathered there make the two-loop step overshoot far
    beyond what the halvings repair; the iteration then restarts from the
    scaled steepest descent instead of stopping."""
    from stfwi_b200.learned.inversion import lbfgs

    shape = (3, 3)

    def ev(x):
        r = x - 1800.0
        return float(np.sum(np.sqrt(1.0 + r * r) - 1.0)), r / np.sqrt(1.0 + r * r)

    n_eval = [0]
    accepted = []
    gen = lbfgs(np.full(shape, 1500.0), np.full(shape, 3000.0), np.ones(shape), n_iter=30, step0=10.0,
                max_ls=3, record=lambda x, f, g: accepted.append((n_eval[0], f)))
    x = next(gen)
    run = longest = 0
    restarted_then_accepted = False
    try:
        while True:
            before = len(accepted)
            n_eval[0] += 1
            x = gen.send(ev(x))
            if len(accepted) > before:
                restarted_then_accepted |= run >= 3
                run = 0
            else:
                run += 1
                longest = max(longest, run)
    except StopIteration:
        pass
    assert longest >= 3 and restarted_then_accepted
    fs = [f for _, f in accepted]
    assert fs[-1] < 0.5 * fs[0] and all(b <= a for a, b in zip(fs, fs[1:]))


def test_experiment_features_and_summary():
    """Network input normalisation, the time-to-target rule and the summary."""
    from stfwi_b200.learned import experiment as E
    rng = np.random.default_rng(4)
    g = rng.standard_normal((6, 9))
    P = rng.uniform(0, 1, (6, 9))
    vp = np.full((6, 9), 4000.0)
    vs = np.full((6, 9), 2200.0)
    f = E.features(g, P, vp, vs)
    assert f.shape == (4, 6, 9) and f.dtype == np.float32
    assert abs(float(np.abs(f[0]).max()) - 1.0) < 1e-6               # preconditioned gradient over its max
    assert np.allclose(f[0], (g * P) / np.abs(g * P).max(), atol=1e-6)
    assert np.allclose(f[1], P) and np.allclose(f[2], 1.0) and np.allclose(f[3], 1.0)
    hist = [(0.5, 0.060, 9.0), (1.0, 0.055, 8.0), (1.5, 0.050, 7.0), (2.0, 0.052, 6.9)]
    assert E._first_time(hist, 0.055) == 1.0 and E._first_time(hist, 0.049) is None
    recs = [dict(ratio=0.2, learned_time_s=1.0, learned_step_accepted=True, err_start=0.06, target=0.05,
                 err_after_learned_step=0.052),
            dict(ratio=None, learned_time_s=None, learned_step_accepted=False, err_start=0.07, target=0.06,
                 err_after_learned_step=None),
            dict(ratio=0.6, learned_time_s=3.0, learned_step_accepted=True, err_start=0.05, target=0.049,
                 err_after_learned_step=0.0495)]
    s = E.summarize(recs)
    assert s["models"] == 3 and s["reached_target"] == 2 and s["learned_step_accepted"] == 2
    assert abs(s["median_time_ratio"] - 0.4) < 1e-12 and abs(s["median_err_after_learned_step"] - 0.05075) < 1e-12
    # the miss counts as an infinite ratio: median of (0.2, inf, 0.6) is 0.6
    assert s["plain_no_progress"] == 0 and abs(s["median_time_ratio_counting_misses"] - 0.6) < 1e-12
    # a model on which the plain run never improved on its start (target =
    # start error, "reached" at once) stays out of the strict median
    recs.append(dict(ratio=0.0, learned_time_s=0.0, learned_step_accepted=False, err_start=0.06, target=0.06,
                     err_after_learned_step=None))
    s = E.summarize(recs)
    assert s["plain_no_progress"] == 1 and abs(s["median_time_ratio_counting_misses"] - 0.6) < 1e-12
    recs.append(dict(ratio=None, learned_time_s=None, learned_step_accepted=True, err_start=0.07, target=0.06,
                     err_after_learned_step=0.065))
    assert E.summarize(recs)["median_time_ratio_counting_misses"] is None   # the median is a miss


def test_acquisition_and_model_pair():
    from stfwi_b200.learned import inversion as I
    sx, sz, types, rx, rz = I.acquisition()
    assert sx.size == 10 and sx.min() >= 0 and sx.max() < 500 and np.all(np.diff(sx) == 50)
    assert types[:2] == ["force", "moment"] and rx.size == 250 and np.all(rz == 1)
    (vs, vp, rho), (vs0, vp0, rho0) = I.true_and_initial(5000)
    assert vs.shape == (152, 500) and np.all(vs <= vp / 1.2 + 1e-3)
    assert I.vs_rel_rms(vs, vs) == 0.0 and 0.0 < I.vs_rel_rms(vs0, vs) < 0.2


def _drive(gen, fg):
    x = next(gen)
    n = 1
    try:
        while True:
            x = gen.send(fg(x))
            n += 1
    except StopIteration as e:
        return e.value, n


def test_reference_lbfgs_converges_and_caps_the_step():
    """The restated reference optimizer (fwi/optimizer.py run_lbfgs: history
    100, step cap step_pct * max|x| / max|g|, strong Wolfe line search of at
    most 40 evaluations) on an ill-conditioned quadratic: it converges, every
    accepted step meets sufficient decrease, and the first step moves no cell
    by more than the cap."""
    from stfwi_b200.learned import inversion as I
    rng = np.random.default_rng(0)
    shape = (8, 10)
    diag = np.exp(rng.uniform(0, 4, shape))
    b = rng.standard_normal(shape) * 5
    x_star = b / diag

    def fg(x):
        return 0.5 * np.sum(diag * x * x) - np.sum(b * x), diag * x - b

    x0 = np.full(shape, 1.5)
    hist = []
    gen = I.lbfgs_reference(x0, np.ones(shape), 60, smooth_sigma=0, step_pct=100.0,
                            record=lambda x, f, g: hist.append((x.copy(), f)))
    x, n = _drive(gen, fg)
    assert np.abs(x - x_star).max() < 1e-5
    assert all(hist[i + 1][1] < hist[i][1] for i in range(len(hist) - 1) if hist[i][1] - fg(x_star)[0] > 1e-9)
    assert n < 2 * 60
    # a 5 % cap: the first accepted step changes no cell by more than 5 % of max|x0|
    hist = []
    gen = I.lbfgs_reference(x0, np.ones(shape), 1, smooth_sigma=0, step_pct=0.05,
                            record=lambda x, f, g: hist.append(x.copy()))
    _drive(gen, fg)
    assert len(hist) == 2
    assert np.abs(hist[1] - hist[0]).max() <= 0.05 * 1.5 * (1 + 1e-12)


def test_strong_wolfe_search_on_a_parabola():
    """phi(a) = (a - 2)^2 from a = 0.5, capped at 10: the search returns a
    step meeting both strong Wolfe conditions."""
    from stfwi_b200.learned import inversion as I
    phi = lambda a: ((a - 2.0) ** 2, 2.0 * (a - 2.0))
    f0, s0 = phi(0.0)
    ls = I.strong_wolfe_search(f0, s0, 0.5, 10.0)
    a = next(ls)
    try:
        while True:
            a = ls.send(phi(a))
    except StopIteration as e:
        step, ok = e.value
    assert ok
    f, s = phi(step)
    assert f <= f0 + 1e-4 * step * s0 and abs(s) <= 0.9 * abs(s0)
