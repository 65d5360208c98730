"""compute_illumination_for_stage with the reference's signature
(fwi/illumination.py:18-48): Ws = Sum_shots Sum_t field^2, the crop and the
normalised inverse run on the GPU."""
from __future__ import annotations

import numpy as np

from ..solver import Solver


def compute_illumination_for_stage(nz, nx, dx, dz, dt, nt, f_c, pad, block_size, rec_x, rec_z, fd_order,
                                   component, Vs, Vp, rho, src_x, src_z, src_wavelet, eps=0.001,
                                   return_ws=False):
    """H_inv = 1 / (Ws + eps max Ws), normalised to [0, 1], on the physical
    grid.  As in the reference, the forward runs with a free surface and Ws
    is cropped to ``Ws[:nz, pad:pad + nx]``."""
    if component not in (0, 1, 2, 3):
        raise KeyError(component)
    sx = np.atleast_1d(np.asarray(src_x)).astype(np.int64)
    sz = np.broadcast_to(np.atleast_1d(np.asarray(src_z)), sx.shape).astype(np.int64)
    rx = np.asarray(rec_x, dtype=np.int32).reshape(-1)
    rz = np.asarray(rec_z, dtype=np.int32).reshape(-1)
    S = Solver(nz, nx, dx, dz, dt, nt, f_c, pad, rx.size, sx.size, fd_order=fd_order, free_surface=True,
               want_gradient=False)
    try:
        S.set_model(Vs, Vp, rho)
        S.set_receivers(rx, rz)
        S.set_shots(sx, sz, "force", np.asarray(src_wavelet, dtype=np.float32))
        if not return_ws:
            return S.preconditioner("illum", component, eps)
        Ws = S.illumination(component)
    finally:
        S.close()
    Ws = Ws[:nz, pad:pad + nx]
    lamda = eps * np.max(Ws)
    H_inv = 1.0 / (Ws + lamda)
    H_inv = H_inv / np.max(H_inv)
    return (H_inv, Ws) if return_ws else H_inv
