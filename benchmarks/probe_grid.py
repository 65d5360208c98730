"""The batched gradient (forward with history, misfit, exact adjoint) on a
custom grid: fd 8, free surface, 20-cell C-PML, seeded layered-fault model,
shots every 7 cells alternating force and moment, receivers every 2 cells.

    python benchmarks/probe_grid.py --nz 152 --nx 500 --shots 10
"""
import argparse, os, sys, time
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import numpy as np

p = argparse.ArgumentParser()
p.add_argument("--nz", type=int, default=152)
p.add_argument("--nx", type=int, default=500)
p.add_argument("--shots", type=int, default=10)
p.add_argument("--nt", type=int, default=12)
p.add_argument("--fd", type=int, default=8)
p.add_argument("--reps", type=int, default=1)
p.add_argument("--tile-rows", type=int, nargs=2, default=None, metavar=("A", "B"),
               help="tile heights (8 or 16) of fwd_vel/fwd_str/adj_a and of adj_b; default: autotune")
a = p.parse_args()
import torch
from stfwi_b200 import Solver
from stfwi_b200 import models as Mo
vs, vp, rho = Mo.layered_fault_model(a.nz, a.nx, seed=1)
sx = (np.arange(a.shots) * 7) % a.nx
sz = np.full(a.shots, 2)
types = ["force" if k % 2 == 0 else "moment" for k in range(a.shots)]
rx = np.arange(0, a.nx, 2, dtype=np.int32); rz = np.ones_like(rx)
wav = Mo.ricker(np.arange(a.nt) * 1.5e-3, 5.0, 0.3).astype(np.float32)
torch.cuda.init()
S = Solver(a.nz, a.nx, 20.0, 20.0, 1.5e-3, a.nt, 5.0, 20, len(rx), a.shots, fd_order=a.fd, free_surface=True,
           want_gradient=True)
S.set_receivers(rx, rz); S.set_shots(sx, sz, types, wav); S.set_model(vs, vp, rho)
if a.tile_rows:
    S.set_tile_rows(*a.tile_rows)
    print("tile rows", S.tile_rows())
else:
    print("autotuned: shots per block", S.autotune(steps=20), "tile rows", S.tile_rows())
obs = np.zeros((a.shots, a.nt, len(rx)), np.float32)
for _ in range(a.reps):
    t0 = time.perf_counter()
    S.forward(store=True); S.misfit(obs, 1, 1.0); g = S.gradient(exact=True)["exact"][0]
    torch.cuda.synchronize()
    print(f"{a.nz}x{a.nx} shots {a.shots}: {time.perf_counter()-t0:.4f}s |g| {np.abs(g).max():.3e}")
S.close()
