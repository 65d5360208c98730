"""A small, self-contained run of the batched gradient for profiling.

    python -m benchmarks.profile_case --shots 50 --nt 40

Runs the batched-shot workload (152 x 500 layered-fault model, fd 8, free
surface) with `shots` shots for `nt` steps: forward with history, misfit,
exact adjoint gradient, `reps` times.  Sized to hold a few GB on the device,
with fields larger than L2 when shots >= 50.
"""
import argparse
import time

import numpy as np


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--shots", type=int, default=50)
    p.add_argument("--nt", type=int, default=40)
    p.add_argument("--reps", type=int, default=1)
    p.add_argument("--fd", type=int, default=8)
    p.add_argument("--shot-group", type=int, default=0, help="shots per block (0: automatic)")
    p.add_argument("--tile-rows", type=int, nargs=2, default=(16, 16), metavar=("A", "B"),
                   help="tile heights of fwd_vel/fwd_str/adj_a and of adj_b (8 or 16)")
    a = p.parse_args()
    import torch
    from stfwi_b200 import Solver
    from stfwi_b200 import models as Mo
    cfg = dict(Mo.CONFIG2, nt=a.nt, n_shots=a.shots, fd_order=a.fd)
    vs, vp, rho = Mo.layered_fault_model(cfg["nz"], cfg["nx"], seed=1)
    sx, sz, types, rx, rz = Mo.acquisition(cfg)
    wav = Mo.ricker(np.arange(a.nt) * cfg["dt"], cfg["fc"], 1.5 / cfg["fc"]).astype(np.float32)
    torch.cuda.init()
    S = Solver(cfg["nz"], cfg["nx"], cfg["dx"], cfg["dz"], cfg["dt"], a.nt, cfg["fc"], cfg["pad"],
               len(rx), a.shots, fd_order=a.fd, free_surface=True, want_gradient=True,
               shot_group=a.shot_group)
    S.set_receivers(rx, rz)
    S.set_shots(sx, sz, types, wav)
    S.set_model(vs, vp, rho)
    S.set_tile_rows(*a.tile_rows)
    obs = np.zeros((a.shots, a.nt, len(rx)), np.float32)
    for _ in range(a.reps):
        t0 = time.perf_counter()
        S.forward(store=True)
        mis = S.misfit(obs, 1, 1.0)
        g = S.gradient(exact=True)["exact"][0]
        print(f"gradient {time.perf_counter() - t0:.4f} s  misfit {mis.sum():.4e}  |g|max {np.abs(g).max():.3e}")
    S.close()


if __name__ == "__main__":
    main()
