"""Plain illumination-preconditioned L-BFGS over a batch of independent
models, and the learned step that may replace its first iterations.

Each model of a batch has its own solver handle (its own workspace and
strain history) and its own CUDA stream; one "round" evaluates the misfit
and exact Vs gradient of every model that asked for one, the launches of the
models interleaved on their streams, then synchronises once.  The L-BFGS of
each model is a generator that yields the next Vs to evaluate and receives
(misfit, raw gradient); the driver runs all of them in lockstep.

The plain method follows the reference's inversion (fwi/optim_lbfgsb.py:
L-BFGS on Vs with the gradient multiplied by the illumination
preconditioner of fwi/illumination.py:18-48, velocity bounds as in
fwi/projections.py); the L-BFGS itself is the two-loop recursion with a
backtracking Armijo line search (Nocedal and Wright, Algorithms 7.4 and
3.1), written here because SciPy's L-BFGS-B cannot run several models in
lockstep.
"""
from __future__ import annotations

import time

import numpy as np

from .. import models as Mo

# acquisition of the learned-preconditioner experiments: the 152 x 500 grid at
# 20 m (fd8, 20-cell C-PML, free surface), 2000 steps of 1.5 ms, a 5 Hz Ricker,
# 10 shots every 1000 m alternating vertical force and moment source at 40 m
# depth, 250 receivers at 20 m depth every 40 m recording vz; the misfit
# compares traces low-passed by an order-6 Butterworth filter at `cutoff` Hz
# (the first band of the reference's multiscale inversion; None: unfiltered)
GEOMETRY = dict(nz=152, nx=500, dx=20.0, dz=20.0, dt=1.5e-3, nt=2000, fc=5.0, pad=20, fd_order=8,
                free_surface=True, n_shots=10, component=1, cutoff=3.0)


def acquisition(geom=GEOMETRY):
    ns, nx = geom["n_shots"], geom["nx"]
    src_x = (np.arange(ns) * (nx // ns) + nx // (2 * ns)).astype(np.int64)
    src_z = np.full(ns, 2, dtype=np.int64)
    types = ["force" if k % 2 == 0 else "moment" for k in range(ns)]
    rec_x = np.arange(0, nx, 2, dtype=np.int32)
    rec_z = np.ones_like(rec_x)
    return src_x, src_z, types, rec_x, rec_z


def true_and_initial(seed, geom=GEOMETRY):
    """Seeded layered-fault model and its sigma = 10 cells smoothed start."""
    vs, vp, rho = Mo.layered_fault_model(geom["nz"], geom["nx"], seed=seed)
    vs0, vp0, rho0 = Mo.smooth_initial(vs, vp, rho, 10.0)
    return (vs, vp, rho), (vs0, vp0, rho0)


def vs_rel_rms(vs, vs_true):
    """Relative RMS error of Vs, sqrt(mean((vs - true)^2)) / sqrt(mean(true^2))."""
    vs = np.asarray(vs, np.float64); t = np.asarray(vs_true, np.float64)
    return float(np.sqrt(np.mean((vs - t) ** 2)) / np.sqrt(np.mean(t ** 2)))


def project_vs(vs, vp, vs_min=300.0, ratio=1.2):
    """Vs bounds of the inversion: vs_min <= Vs <= Vp / ratio (Vp fixed)."""
    return np.clip(vs, vs_min, np.asarray(vp, np.float64) / ratio)


def lbfgs(vs0, vp, precond, n_iter, mem=10, step0=50.0, c1=1e-4, max_ls=6, record=None, stop=None):
    """L-BFGS on Vs (m/s) with the illumination-preconditioned gradient, as a
    generator: yields the next Vs to evaluate and receives (misfit, raw
    g_Vs).  The first direction is the preconditioned steepest descent scaled
    to a largest change of ``step0`` m/s; later ones come from the two-loop
    recursion over the last ``mem`` pairs; each step backtracks (halving)
    until the Armijo condition holds; when ``max_ls`` halvings find no
    decrease the memory is cleared and the next iteration restarts from the
    scaled steepest descent (the iteration stops only when that fails too).  ``record(vs, f, g_raw)`` is called on
    every accepted iterate (and the start); the iteration ends early when
    ``stop(vs, f)`` is true there.  Returns the final Vs."""
    vp = np.asarray(vp, np.float64)
    P = np.asarray(precond, np.float64)
    x = project_vs(np.asarray(vs0, np.float64), vp)
    f, graw = yield x
    g = graw * P
    if record:
        record(x, f, graw)
    if stop and stop(x, f):
        return x
    S, Y = [], []
    for _ in range(n_iter):
        q = g.copy()
        hist = []
        for s, y in zip(reversed(S), reversed(Y)):
            r = 1.0 / float(np.vdot(y, s))
            a = r * float(np.vdot(s, q))
            q -= a * y
            hist.append((r, a, s, y))
        if S:
            q *= float(np.vdot(S[-1], Y[-1])) / float(np.vdot(Y[-1], Y[-1]))
        else:
            q *= step0 / max(float(np.abs(q).max()), 1e-300)
        for r, a, s, y in reversed(hist):
            b = r * float(np.vdot(y, q))
            q += s * (a - b)
        d = -q
        if float(np.vdot(g, d)) >= 0.0:          # not a descent direction: restart
            S, Y = [], []
            d = -g * (step0 / max(float(np.abs(g).max()), 1e-300))
        alpha, accepted = 1.0, False
        for _ls in range(max_ls):
            xn = project_vs(x + alpha * d, vp)
            fn, graw = yield xn
            if fn <= f + c1 * float(np.vdot(g, xn - x)):
                accepted = True
                break
            alpha *= 0.5
        if not accepted:
            if S:                                # stale curvature pairs: restart
                S, Y = [], []
                continue
            return x
        gn = graw * P
        s, y = xn - x, gn - g
        if float(np.vdot(s, y)) > 1e-12 * float(np.vdot(y, y)):
            S.append(s)
            Y.append(y)
            if len(S) > mem:
                S.pop(0)
                Y.pop(0)
        x, f, g = xn, fn, gn
        if record:
            record(x, f, graw)
        if stop and stop(x, f):
            return x
    return x


def _cubic_min(a, fa, da, b, fb, db):
    """Minimiser of the cubic through (a, fa, fa') and (b, fb, fb'), or None
    (Nocedal and Wright, eq. 3.59)."""
    d1 = da + db - 3.0 * (fa - fb) / (a - b)
    disc = d1 * d1 - da * db
    if disc < 0.0:
        return None
    d2 = np.copysign(np.sqrt(disc), b - a)
    den = db - da + 2.0 * d2
    if den == 0.0:
        return None
    return b - (b - a) * (db + d2 - d1) / den


def strong_wolfe_search(f0, slope0, init_step, max_step, maxls=40, c1=1e-4, c2=0.9):
    """Line search for the strong Wolfe conditions (Nocedal and Wright,
    Algorithms 3.5 and 3.6: bracketing, then zoom with safeguarded cubic
    interpolation), as a generator: yields a step length, receives
    (f, slope) there; at most ``maxls`` evaluations.  Returns (step, ok):
    the first step meeting both conditions, else the best step meeting
    sufficient decrease (0.0 when none did)."""
    a_prev, f_prev, s_prev = 0.0, f0, slope0
    a = min(init_step, max_step)
    best = (0.0, f0)
    n = 0

    def decrease(a_, f_):
        return f_ <= f0 + c1 * a_ * slope0

    def zoom(lo, flo, slo, hi, fhi, shi):
        nonlocal n, best
        while n < maxls:
            t = _cubic_min(lo, flo, slo, hi, fhi, shi)
            lo_b, hi_b = min(lo, hi), max(lo, hi)
            w = hi_b - lo_b
            if t is None or not (lo_b + 0.1 * w <= t <= hi_b - 0.1 * w):
                t = 0.5 * (lo + hi)
            ft, st = yield t
            n += 1
            if decrease(t, ft) and ft < best[1]:
                best = (t, ft)
            if not decrease(t, ft) or ft >= flo:
                hi, fhi, shi = t, ft, st
            else:
                if abs(st) <= -c2 * slope0:
                    return t, True
                if st * (hi - lo) >= 0.0:
                    hi, fhi, shi = lo, flo, slo
                lo, flo, slo = t, ft, st
        return best[0], False

    while n < maxls:
        fa, sa = yield a
        n += 1
        if decrease(a, fa) and fa < best[1]:
            best = (a, fa)
        if not decrease(a, fa) or (n > 1 and fa >= f_prev):
            return (yield from zoom(a_prev, f_prev, s_prev, a, fa, sa))
        if abs(sa) <= -c2 * slope0:
            return a, True
        if sa >= 0.0:
            return (yield from zoom(a, fa, sa, a_prev, f_prev, s_prev))
        if a >= max_step:
            return a, False          # the largest step still descends: take it
        a_prev, f_prev, s_prev = a, fa, sa
        a = min(2.0 * a, max_step)
    return best[0], False


def lbfgs_reference(vs0, precond, n_iter, history_size=100, step_pct=0.05, maxls=40, smooth_sigma=1.0,
                    increase=1.5, record=None, stop=None):
    """The reference's plain inversion loop on Vs (fwi/optimizer.py:20-168
    run_lbfgs with a Vs-only loss from fwi/loss.py build_loss_fn, as
    Main_ex_Vs.py drives it), restated as a generator: yields the next Vs
    to evaluate and receives (misfit, raw g_Vs).

    * the gradient L-BFGS sees is the raw one Gaussian-smoothed (sigma
      ``smooth_sigma``) and multiplied by the illumination preconditioner
      (fwi/loss.py, ``_postprocess`` of fwi/gradient.py:266-277);
    * every iteration caps the step length at step_pct * max|Vs| / max|g|
      (fwi/optimizer.py:96-106, recomputed each epoch at :124-131);
    * the direction comes from the two-loop recursion over the last
      ``history_size`` pairs with the initial matrix s'y / y'y (the jaxopt
      LBFGS the reference uses, history 100); the first is -g;
    * the step is found by a strong Wolfe line search of at most ``maxls``
      evaluations (maxls=40, :110-111), starting from ``increase`` times
      the previous step (jaxopt's "increase" initialisation), the first from
      the cap; if it fails, the best sufficient-decrease step is taken (none:
      the iterate stays).
    No bounds, as in the reference.  ``record(vs, f, g_raw)`` sees every
    accepted iterate (and the start); ``stop(vs, f)`` ends early."""
    from ..fwi.loss import gaussian_smooth_2d
    P = np.asarray(precond, np.float64)

    def direction(graw):
        g = graw if not smooth_sigma else gaussian_smooth_2d(graw, smooth_sigma)
        return np.asarray(g, np.float64) * P

    x = np.asarray(vs0, np.float64).copy()
    f, graw = yield x
    g = direction(graw)
    if record:
        record(x, f, graw)
    if stop and stop(x, f):
        return x
    S, Y, RHO = [], [], []
    gamma = 1.0
    step = None
    for _ in range(n_iter):
        max_step = step_pct * float(np.abs(x).max()) / (float(np.abs(g).max()) + 1e-30)
        q = g.copy()
        alphas = []
        for s, y, r in zip(reversed(S), reversed(Y), reversed(RHO)):
            a = r * float(np.vdot(s, q))
            q -= a * y
            alphas.append(a)
        q *= gamma
        for (s, y, r), a in zip(zip(S, Y, RHO), reversed(alphas)):
            b = r * float(np.vdot(y, q))
            q += s * (a - b)
        d = -q
        slope0 = float(np.vdot(g, d))
        if slope0 >= 0.0:          # not a descent direction: steepest descent
            d = -g
            slope0 = float(np.vdot(g, d))
        init = max_step if step is None else increase * step
        ls = strong_wolfe_search(f, slope0, init, max_step, maxls=maxls)
        trial = {}
        try:
            a = next(ls)
            while True:
                xa = x + a * d
                fa, graw_a = yield xa
                ga = direction(graw_a)
                trial[a] = (xa, fa, graw_a, ga)
                a = ls.send((fa, float(np.vdot(ga, d))))
        except StopIteration as e:
            a_ok, _ok = e.value
        if a_ok <= 0.0 or a_ok not in trial:
            step = step if step is not None else max_step
            continue                   # no decrease found: the iterate stays
        xn, fn, graw_n, gn = trial[a_ok]
        s, y = xn - x, gn - g
        sy = float(np.vdot(s, y))
        if sy > 0.0:
            S.append(s); Y.append(y); RHO.append(1.0 / sy)
            if len(S) > history_size:
                S.pop(0); Y.pop(0); RHO.pop(0)
            gamma = sy / float(np.vdot(y, y))
        x, f, g, step = xn, fn, gn, a_ok
        if record:
            record(x, f, graw_n)
        if stop and stop(x, f):
            return x
    return x


def run_lockstep(batch, gens, clock=None):
    """Drive one generator per slot (None for idle slots) until all finish;
    every round evaluates the Vs each live generator yielded.  ``clock['t']``
    (if given) accumulates the rounds' wall time before the results go back
    to the generators.  Returns the generators' return values and the wall
    time of every round."""
    pending = [None] * len(gens)
    result = [None] * len(gens)
    live = [g is not None for g in gens]
    for k, g in enumerate(gens):
        if g is not None:
            pending[k] = next(g)
    rounds = []
    while any(live):
        t0 = time.perf_counter()
        res = batch.evaluate([pending[k] if live[k] else None for k in range(len(gens))])
        rounds.append(time.perf_counter() - t0)
        if clock is not None:
            clock["t"] += rounds[-1]
        for k, g in enumerate(gens):
            if not live[k]:
                continue
            try:
                pending[k] = g.send(res[k])
            except StopIteration as e:
                result[k] = e.value
                live[k] = False
    return result, rounds


class ModelBatch:
    """K solver handles (one per model slot) on K CUDA streams, same
    acquisition.  ``load(k, true, init)`` models the observed data of slot
    k from its true model, fixes its Vp and rho (the true ones: the
    experiments invert Vs with a known P-velocity and density background,
    so that the Vs error measures the Vs update alone) and computes the
    illumination preconditioner at the initial Vs; ``evaluate`` runs one
    round of misfit + exact gradient evaluations."""

    def __init__(self, K, geom=GEOMETRY, mem_budget_gb=28.0):
        import torch
        from ..solver import Solver
        self.torch = torch
        self.geom = dict(geom)
        self.K = int(K)
        g = self.geom
        self.src_x, self.src_z, self.types, self.rec_x, self.rec_z = acquisition(g)
        self.wavelet = Mo.ricker(np.arange(g["nt"]) * g["dt"], g["fc"], 1.5 / g["fc"]).astype(np.float32)
        self.solvers, self.streams = [], []
        for _ in range(self.K):
            S = Solver(g["nz"], g["nx"], g["dx"], g["dz"], g["dt"], g["nt"], g["fc"], g["pad"], self.rec_x.size,
                       self.src_x.size, fd_order=g["fd_order"], free_surface=g["free_surface"],
                       want_gradient=True, mem_budget_gb=mem_budget_gb)
            S.set_receivers(self.rec_x, self.rec_z)
            S.set_shots(self.src_x, self.src_z, self.types, self.wavelet)
            self.solvers.append(S)
            self.streams.append(torch.cuda.Stream())
        ns, nt, nr = self.src_x.size, g["nt"], self.rec_x.size
        self.obs = [torch.empty((ns, nt, nr), dtype=torch.float32, device="cuda") for _ in range(self.K)]
        self.mis = [torch.zeros(ns, dtype=torch.float64, device="cuda") for _ in range(self.K)]
        self.grad = [torch.zeros((1, 3, g["nz"], g["nx"]), dtype=torch.float64, device="cuda")
                     for _ in range(self.K)]
        self.scale = [1.0] * self.K
        self.vp = [None] * self.K
        self.rho = [None] * self.K
        self.precond = [None] * self.K
        self.evals = 0
        self.sos = None
        if g.get("cutoff"):
            from scipy.signal import butter
            self.sos = butter(6, g["cutoff"], fs=1.0 / g["dt"], output="sos")

    def load(self, k, true, init, known_background=True):
        """Observed data of slot k (component ``geom['component']``) from the
        true model; the background Vp and rho are the true ones (or the
        initial ones with ``known_background=False``); the preconditioner
        comes from the initial Vs on that background."""
        torch = self.torch
        S, st = self.solvers[k], self.streams[k]
        comp = self.geom["component"]
        with torch.cuda.stream(st):
            S.set_model(*true)
            S.forward()
            rec = torch.empty((S.nshot, 4, S.nt, S.nrec), dtype=torch.float32, device="cuda")
            S.records(out=rec)
            self.obs[k].copy_(rec[:, comp])
            self.scale[k] = float(1.0 / (float(self.obs[k].double().pow(2).mean()) + 1e-45))
            bg = true if known_background else init
            self.vp[k] = np.asarray(bg[1], np.float64)
            self.rho[k] = np.asarray(bg[2], np.float64)
            S.set_model(init[0], bg[1], bg[2])
            self.precond[k] = S.preconditioner("illum", comp, 1e-3)
        st.synchronize()

    def set_cutoff(self, cutoff):
        """Low-pass cutoff (Hz) of the misfit filter for the following
        evaluations (an order-6 Butterworth; None: unfiltered)."""
        from scipy.signal import butter
        self.geom["cutoff"] = cutoff
        self.sos = butter(6, cutoff, fs=1.0 / self.geom["dt"], output="sos") if cutoff else None

    def refresh_precond(self, vs_list, eps=1e-3):
        """Illumination preconditioner of each slot at its current Vs (the
        reference recomputes it at the start of every stage,
        Main_ex_Vs.py:237-247); None entries keep theirs."""
        torch = self.torch
        for k, vs in enumerate(vs_list):
            if vs is None:
                continue
            S = self.solvers[k]
            with torch.cuda.stream(self.streams[k]):
                S.set_model(np.asarray(vs, np.float32), self.vp[k].astype(np.float32),
                            self.rho[k].astype(np.float32))
                self.precond[k] = S.preconditioner("illum", self.geom["component"], eps)
        torch.cuda.synchronize()

    def _launch(self, k, vs, gradient):
        S = self.solvers[k]
        S.set_model(np.asarray(vs, np.float32), self.vp[k].astype(np.float32), self.rho[k].astype(np.float32))
        S.forward(store=gradient)
        self.mis[k].zero_()
        S.misfit(self.obs[k], self.geom["component"], self.scale[k], sos=self.sos, out=self.mis[k], sync=False)
        if gradient:
            self.grad[k].zero_()
            S.gradient(exact=True, out=self.grad[k], sync=False)

    def evaluate(self, vs_list):
        """vs_list[k]: Vs (float64 [nz, nx]) to evaluate in slot k, or None.
        Returns [(misfit, raw exact g_Vs)] (None for idle slots)."""
        torch = self.torch
        active = [k for k, v in enumerate(vs_list) if v is not None]
        for k in active:
            with torch.cuda.stream(self.streams[k]):
                self._launch(k, vs_list[k], True)
        torch.cuda.synchronize()
        out = [None] * len(vs_list)
        for k in active:
            try:
                self.solvers[k].check()
                out[k] = (float(self.mis[k].sum()), self.grad[k][0, 0].cpu().numpy())
            except Exception as e:   # an unstable trial model: an infinite misfit for the line search
                if getattr(e, "status", None) != 5:
                    raise
                out[k] = (float("inf"), np.zeros((self.geom["nz"], self.geom["nx"])))
        self.evals += len(active)
        return out

    def misfits(self, vs_list):
        """Misfit only (forward without history) for each non-None Vs."""
        torch = self.torch
        active = [k for k, v in enumerate(vs_list) if v is not None]
        for k in active:
            with torch.cuda.stream(self.streams[k]):
                self._launch(k, vs_list[k], False)
        torch.cuda.synchronize()
        out = [None] * len(vs_list)
        for k in active:
            try:
                self.solvers[k].check()
                out[k] = float(self.mis[k].sum())
            except Exception as e:
                if getattr(e, "status", None) != 5:
                    raise
                out[k] = float("inf")
        return out

    def close(self):
        for S in self.solvers:
            S.close()
        self.solvers = []
