"""The uneven batch of three grids (152x500 at 20 m / 2000 steps, 304x1000 at
10 m / 4000 steps, 608x2000 at 5 m / 8000 steps; 8, 16 and 32 shots; Ricker
5, 10 and 15 Hz; fd 4, 8, 8), each from the seeded layered-fault recipe: one
exact gradient per model, first one model at a time, then all models with
their launches interleaved on separate streams.

    python -m benchmarks.uneven_case [--scale 1.0]

``--scale`` shrinks the step counts (a quick run); the printed JSON line
holds per-model and whole-batch fwd+adj Gcell-updates/s.
"""
import argparse
import json
import time

import numpy as np


def specs(scale=1.0):
    from stfwi_b200 import models as Mo
    out = []
    # memory budgets (GB): store-all history for the small grid, checkpoint
    # segments chosen by the handle for the two larger ones (180 GB in all)
    for (nz, nx, dx, nt, ns, fc, fd, budget) in ((152, 500, 20.0, 2000, 8, 5.0, 4, 16.0),
                                                 (304, 1000, 10.0, 4000, 16, 10.0, 8, 14.0),
                                                 (608, 2000, 5.0, 8000, 32, 15.0, 8, 128.0)):
        nt = max(50, int(nt * scale))
        dt = 1.5e-3 * dx / 20.0
        vs, vp, rho = Mo.layered_fault_model(nz, nx, seed=11)
        sx = np.linspace(nx // 20, nx - nx // 20 - 1, ns).astype(np.int64)
        out.append(dict(nz_dom=nz, nx_dom=nx, dx=dx, dz=dx, dt=dt, nt=nt, fc=fc, pad=20, fd_order=fd,
                        free_surface=True, src_x=sx, src_z=np.full(ns, 2), src_types=["force", "moment"] * (ns // 2),
                        wavelet=Mo.ricker(np.arange(nt) * dt, fc, 1.5 / fc), rec_x=np.arange(0, nx, 4),
                        rec_z=np.ones(nx // 4, dtype=np.int64), mem_budget_gb=budget,
                        true=(vs, vp, rho), init=Mo.smooth_initial(vs, vp, rho, 10.0)))
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--scale", type=float, default=1.0)
    a = p.parse_args()
    import torch
    from stfwi_b200.batch import UnevenBatch
    sp = specs(a.scale)
    torch.cuda.init()
    B = UnevenBatch(sp)
    obs = [r[:, 1].contiguous() for r in B.records([s["true"] for s in sp])]
    inits = [s["init"] for s in sp]
    cells = [S.nshot * S.nz * S.nx * S.nt for S in B.solvers]
    B.gradient(inits, obs)   # warm-up: graph capture
    alone = []
    for k in range(len(sp)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S, st = B.solvers[k], B.streams[k]
        with torch.cuda.stream(st):
            S.set_model(*inits[k])
            S.forward(store=True)
            S.misfit(obs[k], 1, 1.0, sync=False, out=torch.zeros(S.nshot, dtype=torch.float64, device="cuda"))
            S.gradient(exact=True, sync=False, out=torch.zeros((1, 3, S.nz_dom, S.nx_dom), dtype=torch.float64,
                                                               device="cuda"))
        torch.cuda.synchronize()
        alone.append(time.perf_counter() - t0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B.gradient(inits, obs)
    t_batch = time.perf_counter() - t0
    line = {"workload": "uneven batch: 152x500/2000 steps x8 shots fd4, 304x1000/4000 x16 fd8, "
                        "608x2000/8000 x32 fd8 (step counts x%.3g)" % a.scale,
            "unit": "Gcell/s fwd+adj",
            "per_model_alone": [round(c / t / 1e9, 2) for c, t in zip(cells, alone)],
            "per_model_seconds_alone": [round(t, 3) for t in alone],
            "sequential": round(sum(cells) / sum(alone) / 1e9, 2),
            "interleaved": round(sum(cells) / t_batch / 1e9, 2), "batch_seconds": round(t_batch, 3)}
    print(json.dumps(line), flush=True)
    B.close()


if __name__ == "__main__":
    main()
