"""Uneven batches: several grids of different size and step count advanced
together on one GPU.

Each model keeps its own handle (its own workspace, captured graphs and
stream) and its launches go to its own CUDA stream, so the small grids'
kernels fill the SMs the large grid's kernels leave idle; the host only
orders the calls and synchronises once per gradient evaluation.
"""
from __future__ import annotations

import numpy as np

from .solver import Solver


class UnevenBatch:
    """``specs``: one dict per model with the Solver arguments (nz_dom, nx_dom,
    dx, dz, dt, nt, fc, pad, fd_order, free_surface; optional mem_budget_gb,
    ckpt_interval) and its acquisition (src_x, src_z, src_types, wavelet,
    rec_x, rec_z).  Give each model a memory budget: a handle otherwise
    plans with 85 % of the free device memory."""

    def __init__(self, specs, want_gradient=True):
        import torch
        self.specs = [dict(s) for s in specs]
        self.solvers = []
        self.streams = []
        for s in self.specs:
            rx = np.asarray(s["rec_x"], dtype=np.int32).reshape(-1)
            rz = np.asarray(s["rec_z"], dtype=np.int32).reshape(-1)
            sx = np.asarray(s["src_x"]).reshape(-1)
            S = Solver(s["nz_dom"], s["nx_dom"], s["dx"], s["dz"], s["dt"], s["nt"], s["fc"], s["pad"], rx.size,
                       sx.size, fd_order=s.get("fd_order", 8), free_surface=s.get("free_surface", True),
                       want_gradient=want_gradient, ckpt_interval=s.get("ckpt_interval", 0),
                       mem_budget_gb=s.get("mem_budget_gb", 0.0))
            S.set_receivers(rx, rz)
            S.set_shots(sx, s["src_z"], s.get("src_types", "force"), np.asarray(s["wavelet"], dtype=np.float32))
            self.solvers.append(S)
            self.streams.append(torch.cuda.Stream())

    def cells(self):
        """Shot x padded-cell x step updates of one forward over the batch."""
        return sum(S.nshot * S.nz * S.nx * S.nt for S in self.solvers)

    def records(self, models):
        """Forward every model (its traces [nshot, 4, nt, nrec] on the device)."""
        import torch
        out = []
        for S, st, m in zip(self.solvers, self.streams, models):
            with torch.cuda.stream(st):
                S.set_model(*m)
                S.forward()
                r = torch.empty((S.nshot, 4, S.nt, S.nrec), dtype=torch.float32, device="cuda")
                S.records(out=r)
                out.append(r)
        torch.cuda.synchronize()
        return out

    def gradient(self, models, observed, component=1, scales=None, sos=None, n_taper=None):
        """Exact gradient of every model, the models' launches interleaved on
        their streams; returns [(misfit per shot FP64, (g_Vs, g_Vp, g_rho))]
        as device tensors."""
        import torch
        res = []
        for k, (S, st, m, obs) in enumerate(zip(self.solvers, self.streams, models, observed)):
            with torch.cuda.stream(st):
                S.set_model(*m)
                S.forward(store=True)
                mis = torch.zeros(S.nshot, dtype=torch.float64, device="cuda")
                S.misfit(obs, component, 1.0 if scales is None else scales[k], None if sos is None else sos[k],
                         0 if n_taper is None else n_taper[k], out=mis, sync=False)
                g = torch.zeros((1, 3, S.nz_dom, S.nx_dom), dtype=torch.float64, device="cuda")
                S.gradient(exact=True, out=g, sync=False)
                res.append((mis, g[0]))
        torch.cuda.synchronize()
        for S in self.solvers:
            S.check()
        return res

    def close(self):
        for S in self.solvers:
            S.close()
        self.solvers = []
