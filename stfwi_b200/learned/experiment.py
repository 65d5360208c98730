"""Training data, training and evaluation of the learned preconditioner.

* pairs: for each seeded layered-fault model, the plain method (lockstep
  L-BFGS, ``inversion.lbfgs``) runs ``n_iter`` iterations from the smoothed
  start; the input is [preconditioned first gradient, illumination
  preconditioner, Vp, Vs] at the start and the target is the Vs update
  the iterations made.
* training: Adam on the masked mean-square error of the U-Net
  (``unet.UNet``, tcgen05 kernels), left-right mirror images as
  augmentation.
* evaluation on held-out models: the plain method for ``n_plain``
  iterations sets each model's target Vs error (the lowest relative RMS
  error it reached); the learned method evaluates the gradient at the
  start, takes the network's direction with a misfit line search (the step
  is accepted only if it lowers the misfit, otherwise the model falls back
  to the plain method from the start) and continues with plain L-BFGS until
  it reaches the same error.  Reported: wall time to the target for both.

``python -m stfwi_b200.learned.experiment --train 192 --test 16 --out DIR``
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import inversion as I
from .unet import UNet, load_weights, padded_shape, save_weights

TARGET_SCALE = 100.0      # m/s per unit of the network's output


def features(g_raw, precond, vp, vs):
    """[4, nz, nx] FP32 network input: the preconditioned gradient over its
    largest magnitude, the preconditioner (in [0, 1]), (Vp - 3000) / 1000 and
    (Vs - 1700) / 500."""
    g = np.asarray(g_raw, np.float64) * np.asarray(precond, np.float64)
    g = g / max(float(np.abs(g).max()), 1e-300)
    return np.stack([g, np.asarray(precond, np.float64), (np.asarray(vp, np.float64) - 3000.0) / 1000.0,
                     (np.asarray(vs, np.float64) - 1700.0) / 500.0]).astype(np.float32)


def generate_pairs(seeds, K=4, n_iter=10, geom=I.GEOMETRY, log=print, method="reference"):
    """Training pairs of the given model seeds: (inputs [n, 4, nz, nx],
    targets [n, nz, nx] in units of TARGET_SCALE, seconds spent).  The
    update is what ``n_iter`` iterations of the plain method make:
    ``method='reference'`` the reference's L-BFGS (``I.lbfgs_reference``),
    ``'armijo'`` the backtracking variant (``I.lbfgs``)."""
    X, Y = [], []
    t0 = time.perf_counter()
    batch = I.ModelBatch(K, geom)
    try:
        for g0 in range(0, len(seeds), K):
            group = list(seeds[g0:g0 + K])
            models = [I.true_and_initial(s, geom) for s in group]
            first = {}
            gens = []
            for k in range(K):
                if k >= len(group):
                    gens.append(None)
                    continue
                batch.load(k, *models[k])

                def rec(x, f, graw, k=k):
                    first.setdefault(k, graw.copy())
                if method == "reference":
                    gens.append(I.lbfgs_reference(models[k][1][0], batch.precond[k], n_iter, record=rec))
                else:
                    gens.append(I.lbfgs(models[k][1][0], batch.vp[k], batch.precond[k], n_iter, record=rec))
            finals, _ = I.run_lockstep(batch, gens)
            for k in range(len(group)):
                init = models[k][1]
                X.append(features(first[k], batch.precond[k], batch.vp[k], init[0]))
                Y.append(((finals[k] - init[0]) / TARGET_SCALE).astype(np.float32))
            log(f"pairs {len(X)}/{len(seeds)}  {time.perf_counter() - t0:.1f} s")
    finally:
        batch.close()
    return np.stack(X), np.stack(Y), time.perf_counter() - t0


def train(X, Y, epochs=60, batch=8, lr=1e-3, seed=0, n_val=0, log=print, device="cuda"):
    """Adam with a cosine learning-rate decay on the pairs (and their
    mirror images); the last ``n_val`` pairs are held out as validation and
    the weights of the epoch with the lowest validation loss are kept.
    Returns (network, per-epoch (train loss, validation loss), best epoch)."""
    import torch
    n_all, _, nz, nx = X.shape
    n = n_all - n_val
    h, w = padded_shape(nz, nx)
    net = UNet(h, w, seed=seed, device=device)
    dev = net.device
    Xd = torch.from_numpy(np.ascontiguousarray(X[:n])).to(dev)
    Yd = torch.from_numpy(np.ascontiguousarray(Y[:n])).to(dev)
    tgt = torch.zeros((batch, h, w), device=dev)
    wgt = torch.zeros((batch, h, w), device=dev)
    wgt[:, :nz, :nx] = 1.0
    inv = 1.0 / (batch * nz * nx)
    rng = np.random.default_rng(seed)
    per_epoch = (2 * n) // batch
    total = max(epochs * per_epoch, 1)
    hist = []
    step = 0
    best = (float("inf"), -1, None)
    for ep in range(epochs):
        perm = rng.permutation(2 * n)
        acc = torch.zeros(1, dtype=torch.float64, device=dev)
        for b0 in range(0, per_epoch * batch, batch):
            idx = torch.from_numpy(perm[b0:b0 + batch]).to(dev)
            src, flip = idx % n, (idx >= n)
            xb, yb = Xd[src], Yd[src]
            xb = torch.where(flip[:, None, None, None], xb.flip(-1), xb)
            yb = torch.where(flip[:, None, None], yb.flip(-1), yb)
            tgt[:, :nz, :nx] = yb
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / total))
            acc += net.train_step(net.pack(xb), tgt, wgt, lr_t, inv_norm=inv)
            step += 1
        tr = float(acc) / max(per_epoch, 1)
        va = validation_loss(net, X[n:], Y[n:], batch) if n_val else float("nan")
        hist.append((tr, va))
        log(f"epoch {ep + 1}/{epochs}  train {tr:.5f}  val {va:.5f}")
        if n_val and va < best[0]:
            best = (va, ep, net.params.detach().clone())
    if best[2] is not None:
        net.params.copy_(best[2])
        net.pack_weights()
    net.check()
    return net, hist, best[1] + 1


def predict(net, X, batch=8):
    """Network output on inputs [n, 4, nz, nx] -> [n, nz, nx] (units of TARGET_SCALE)."""
    import torch
    n, _, nz, nx = X.shape
    out = []
    for b0 in range(0, n, batch):
        xb = torch.from_numpy(np.ascontiguousarray(X[b0:b0 + batch])).to(net.device)
        o = net.forward(net.pack(xb))
        out.append(o[:, :nz, :nx].cpu().numpy())
    return np.concatenate(out)


def validation_loss(net, X, Y, batch=8):
    """Mean-square error of the prediction over the validation pairs."""
    P = predict(net, X, batch)
    return float(np.mean((P.astype(np.float64) - Y) ** 2))


def _first_time(hist, target):
    """Clock time of the first recorded iterate whose Vs error is <= target."""
    for t, err, _f in hist:
        if err <= target * (1.0 + 1e-12):
            return t
    return None


def evaluate(net, seeds, K=4, n_plain=20, geom=I.GEOMETRY, alphas=(1.0, 0.5, 0.25), log=print):
    """Learned vs plain on held-out models; one record per model."""
    import torch
    out = []
    batch = I.ModelBatch(K, geom)
    try:
        for g0 in range(0, len(seeds), K):
            group = list(seeds[g0:g0 + K])
            models = [I.true_and_initial(s, geom) for s in group]
            slots = list(range(len(group)))
            for k in slots:
                batch.load(k, *models[k])
            true_vs = {k: models[k][0][0] for k in slots}
            vs0 = {k: models[k][1][0].astype(np.float64) for k in slots}
            vp0 = {k: batch.vp[k] for k in slots}          # the known background
            # plain: n_plain iterations set the target error of every model
            clock = {"t": 0.0}
            plain = {k: [] for k in slots}
            gens = [I.lbfgs(vs0[k], vp0[k], batch.precond[k], n_plain,
                            record=lambda x, f, g, k=k: plain[k].append((clock["t"], I.vs_rel_rms(x, true_vs[k]), f)))
                    for k in slots] + [None] * (K - len(group))
            I.run_lockstep(batch, gens, clock)
            target = {k: min(e for _, e, _ in plain[k]) for k in slots}
            # learned: gradient at the start, the network's direction, a misfit line search
            clock = {"t": 0.0}
            learned = {k: [] for k in slots}
            t0 = time.perf_counter()
            res = batch.evaluate([vs0[k] if k in slots else None for k in range(K)])
            clock["t"] += time.perf_counter() - t0
            f0 = {k: res[k][0] for k in slots}
            for k in slots:
                learned[k].append((clock["t"], I.vs_rel_rms(vs0[k], true_vs[k]), f0[k]))
            t0 = time.perf_counter()
            X = np.stack([features(res[k][1], batch.precond[k], vp0[k], vs0[k]) for k in slots])
            d = predict(net, X) * TARGET_SCALE
            torch.cuda.synchronize()
            t_net = time.perf_counter() - t0
            clock["t"] += t_net
            accepted, step = {}, {}
            for a in alphas:
                cand = [None] * K
                for k in slots:
                    if k not in accepted:
                        cand[k] = I.project_vs(vs0[k] + a * d[k], vp0[k])
                if all(c is None for c in cand):
                    break
                t0 = time.perf_counter()
                fs = batch.misfits(cand)
                clock["t"] += time.perf_counter() - t0
                for k in slots:
                    if cand[k] is not None and fs[k] < f0[k]:
                        accepted[k], step[k] = cand[k], a
                        learned[k].append((clock["t"], I.vs_rel_rms(cand[k], true_vs[k]), fs[k]))
            gens = []
            for k in range(K):
                if k not in slots:
                    gens.append(None)
                    continue
                x1 = accepted.get(k, vs0[k])            # rejected: the plain method from the start
                gens.append(I.lbfgs(x1, vp0[k], batch.precond[k], n_plain,
                                    record=lambda x, f, g, k=k: learned[k].append(
                                        (clock["t"], I.vs_rel_rms(x, true_vs[k]), f)),
                                    stop=lambda x, f, k=k: I.vs_rel_rms(x, true_vs[k]) <= target[k]))
            I.run_lockstep(batch, gens, clock)
            for k in slots:
                tp = _first_time(plain[k], target[k])
                tl = _first_time(learned[k], target[k])
                rec = dict(seed=int(group[k]), err_start=plain[k][0][1], target=target[k],
                           plain_time_s=tp, learned_time_s=tl,
                           ratio=(tl / tp) if (tl is not None and tp) else None,
                           learned_step_accepted=k in accepted, step=step.get(k),
                           err_after_learned_step=I.vs_rel_rms(accepted[k], true_vs[k]) if k in accepted else None,
                           err_plain_final=plain[k][-1][1], err_learned_final=learned[k][-1][1],
                           plain_iterates=len(plain[k]), learned_iterates=len(learned[k]),
                           network_s=t_net / len(group))
                out.append(rec)
                log(json.dumps(rec))
    finally:
        batch.close()
    return out


BANDS = (3.0, 5.0, 8.0)   # the multiscale schedule's low-pass cutoffs (Hz), 20 iterations each


def evaluate_multiband(net, seeds, K=4, bands=BANDS, iters=20, geom=I.GEOMETRY, alphas=(1.0, 0.5, 0.25),
                       log=print):
    """Learned vs plain on held-out models over the multiscale schedule.

    Plain (the fallback and the yardstick): for each band in turn, the misfit
    filter is set to its cutoff, the illumination preconditioner is
    recomputed at the current Vs, and the reference's L-BFGS
    (``I.lbfgs_reference``: history 100, 5 % step cap, strong Wolfe line
    search of at most 40 evaluations) runs ``iters`` iterations.  Its lowest
    Vs relative-RMS error over the whole schedule is the model's target.
    Learned: the same schedule, except that the first band starts with the
    network's direction (accepted only if a misfit line search over
    ``alphas`` lowers the misfit, otherwise the plain method starts from the
    initial model); it stops as soon as the Vs error reaches the target.
    Both clocks count the GPU rounds, the preconditioners and the network.
    Vp and rho are the true ones, as in the reference's Vs-only driver
    (Main_ex_Vs.py:203-205 keeps the true Vp and rho when no stage inverts
    them)."""
    import torch
    out = []
    batch = I.ModelBatch(K, dict(geom, cutoff=bands[0]))
    try:
        for g0 in range(0, len(seeds), K):
            group = list(seeds[g0:g0 + K])
            models = [I.true_and_initial(s, geom) for s in group]
            slots = list(range(len(group)))
            for k in slots:
                batch.load(k, *models[k])
            true_vs = {k: models[k][0][0] for k in slots}
            vs0 = {k: models[k][1][0].astype(np.float64) for k in slots}

            def band_runs(start, hist, clock, stop_at=None, first_band_start=None):
                """Run the bands from Vs `start`; returns the final Vs per slot."""
                cur = dict(start)
                for b, cut in enumerate(bands):
                    live = [k for k in slots if not (stop_at and hist[k] and hist[k][-1][1] <= stop_at[k])]
                    if not live:
                        break
                    batch.set_cutoff(cut)
                    t0 = time.perf_counter()
                    batch.refresh_precond([cur[k] if k in live else None for k in range(K)])
                    clock["t"] += time.perf_counter() - t0
                    if b == 0 and first_band_start is not None:
                        cur.update(first_band_start(live, clock))
                    gens = []
                    for k in range(K):
                        if k not in live:
                            gens.append(None)
                            continue
                        st = (lambda x, f, k=k: I.vs_rel_rms(x, true_vs[k]) <= stop_at[k]) if stop_at else None
                        gens.append(I.lbfgs_reference(cur[k], batch.precond[k], iters, stop=st,
                                                      record=lambda x, f, g, k=k: hist[k].append(
                                                          (clock["t"], I.vs_rel_rms(x, true_vs[k]), f))))
                    finals, _ = I.run_lockstep(batch, gens, clock)
                    for k in live:
                        cur[k] = finals[k]
                return cur

            clock = {"t": 0.0}
            plain = {k: [] for k in slots}
            band_runs(vs0, plain, clock)
            target = {k: min(e for _, e, _ in plain[k]) for k in slots}

            learned = {k: [] for k in slots}
            accepted, step = {}, {}
            t_net = [0.0]

            def learned_start(live, clock):
                t0 = time.perf_counter()
                res = batch.evaluate([vs0[k] if k in live else None for k in range(K)])
                clock["t"] += time.perf_counter() - t0
                f0 = {k: res[k][0] for k in live}
                t0 = time.perf_counter()
                X = np.stack([features(res[k][1], batch.precond[k], batch.vp[k], vs0[k]) for k in live])
                d = predict(net, X) * TARGET_SCALE
                torch.cuda.synchronize()
                t_net[0] = time.perf_counter() - t0
                clock["t"] += t_net[0]
                dk = {k: d[i] for i, k in enumerate(live)}
                for a in alphas:
                    cand = [I.project_vs(vs0[k] + a * dk[k], batch.vp[k]) if (k in live and k not in accepted)
                            else None for k in range(K)]
                    if all(c is None for c in cand):
                        break
                    t0 = time.perf_counter()
                    fs = batch.misfits(cand)
                    clock["t"] += time.perf_counter() - t0
                    for k in live:
                        if cand[k] is not None and fs[k] < f0[k]:
                            accepted[k], step[k] = cand[k], a
                            learned[k].append((clock["t"], I.vs_rel_rms(cand[k], true_vs[k]), fs[k]))
                return {k: accepted[k] for k in live if k in accepted}

            clock = {"t": 0.0}
            for k in slots:
                learned[k].append((0.0, I.vs_rel_rms(vs0[k], true_vs[k]), float("nan")))
            band_runs(vs0, learned, clock, stop_at=target, first_band_start=learned_start)
            for k in slots:
                tp = _first_time(plain[k], target[k])
                tl = _first_time(learned[k], target[k])
                rec = dict(seed=int(group[k]), err_start=plain[k][0][1], target=target[k],
                           plain_time_s=tp, learned_time_s=tl,
                           ratio=(tl / tp) if (tl is not None and tp) else None,
                           learned_step_accepted=k in accepted, step=step.get(k),
                           err_after_learned_step=I.vs_rel_rms(accepted[k], true_vs[k]) if k in accepted else None,
                           err_plain_final=plain[k][-1][1], err_learned_final=learned[k][-1][1],
                           plain_iterates=len(plain[k]), learned_iterates=len(learned[k]),
                           network_s=t_net[0] / len(group), bands=list(bands), iters_per_band=iters)
                out.append(rec)
                log(json.dumps(rec))
    finally:
        batch.close()
    return out


def summarize(records):
    """Ratios of the models whose learned run reached the target
    (``median_time_ratio``), and the stricter median over the models on
    which the plain method improved on its start at all, a model the learned
    run did not bring to the target counting as an infinite ratio
    (``median_time_ratio_counting_misses``; None when that median is a miss).
    A model whose plain run never improved on the start has its start error
    as the target, which any run "reaches" at time zero: such models are
    counted in ``plain_no_progress`` and left out of the strict median."""
    ratios = [r["ratio"] for r in records if r["ratio"] is not None]
    after = [r["err_after_learned_step"] for r in records if r["err_after_learned_step"] is not None]
    progress = [r for r in records if r["target"] < r["err_start"]]
    strict = [r["ratio"] if r["ratio"] is not None else np.inf for r in progress]
    med_strict = float(np.median(strict)) if strict else None
    return dict(models=len(records), reached_target=sum(r["learned_time_s"] is not None for r in records),
                learned_step_accepted=sum(bool(r["learned_step_accepted"]) for r in records),
                plain_no_progress=len(records) - len(progress),
                median_time_ratio_counting_misses=med_strict if med_strict is not None and np.isfinite(med_strict)
                else None,
                median_time_ratio=float(np.median(ratios)) if ratios else None,
                mean_time_ratio=float(np.mean(ratios)) if ratios else None,
                median_err_start=float(np.median([r["err_start"] for r in records])),
                median_target=float(np.median([r["target"] for r in records])),
                median_err_after_learned_step=float(np.median(after)) if after else None)


def main(argv=None):
    ap = argparse.ArgumentParser(description="learned preconditioner: data, training, evaluation")
    ap.add_argument("--train", type=int, default=192, help="training models (seeds 1000, 1001, ...)")
    ap.add_argument("--test", type=int, default=16, help="held-out models (seeds 5000, 5001, ...)")
    ap.add_argument("--iters", type=int, default=10, help="L-BFGS iterations of a training pair")
    ap.add_argument("--plain", type=int, default=20, help="L-BFGS iterations of the plain arm")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--val", type=int, default=16, help="training pairs held out for validation")
    ap.add_argument("--K", type=int, default=4, help="models evaluated concurrently")
    ap.add_argument("--out", default="learned_out")
    ap.add_argument("--method", default="reference", choices=["reference", "armijo"],
                    help="plain optimizer of the training pairs")
    ap.add_argument("--multiband", action="store_true",
                    help="evaluate over the 3/5/8 Hz schedule (reference L-BFGS as the plain arm)")
    ap.add_argument("--weights", default=None,
                    help="evaluate these trained weights (save_weights format) instead of generating data and training")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, "log.txt"), "a") as logf:
        _run(a, logf)


def _run(a, logf):
    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    if a.weights:
        h, w = padded_shape(I.GEOMETRY["nz"], I.GEOMETRY["nx"])
        net = UNet(h, w)
        net.load_state_dict({"params": load_weights(a.weights), "h": h, "w": w})
        t_data = t_train = 0.0
        hist, best_epoch, zero_val = [], None, None
    else:
        X, Y, t_data = generate_pairs(list(range(1000, 1000 + a.train)), K=a.K, n_iter=a.iters, log=log,
                                      method=a.method)
        n_val = min(a.val, X.shape[0] // 4)
        t0 = time.perf_counter()
        net, hist, best_epoch = train(X, Y, epochs=a.epochs, n_val=n_val, log=log)
        t_train = time.perf_counter() - t0
        zero_val = float(np.mean(Y[X.shape[0] - n_val:].astype(np.float64) ** 2)) if n_val else None
        save_weights(os.path.join(a.out, "unet_weights.npz"), net.params.detach().cpu().numpy())
    if a.multiband:
        recs = evaluate_multiband(net, list(range(5000, 5000 + a.test)), K=a.K, iters=a.plain, log=log)
    else:
        recs = evaluate(net, list(range(5000, 5000 + a.test)), K=a.K, n_plain=a.plain, log=log)
    summary = dict(config=dict(vars(a), geometry=I.GEOMETRY), data_seconds=t_data, train_seconds=t_train,
                   train_history=hist, best_epoch=best_epoch, val_loss_of_zero_prediction=zero_val,
                   evaluation=summarize(recs), records=recs)
    with open(os.path.join(a.out, "results.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    log(json.dumps(summary["evaluation"]))


if __name__ == "__main__":
    main()
