"""imaging_condition with the reference's signature (fwi/imaging.py:83-169).

The reference sums the imaging terms over time from full histories of the
forward strains and the adjoint velocities (and, for the density term, the
forward velocities).  Here the sums run on the GPU
(stfwi_imaging_condition: one thread per physical cell, FP64 sums over
chunks of frames, the periodic centred differences of the reference), on
histories given as NumPy or torch arrays on the host or the device.  The
gradient backend 'cuda_imaging' computes the same quantity without any
history: fused into the adjoint sweep.
"""
from __future__ import annotations

from ..solver import imaging_condition_device


def imaging_condition(Vs, Vp, rho, ex_hist, ez_hist, es_hist, U_a_hist, V_a_hist, dx, dz, dt, pad, free_surface,
                      nz_dom, nx_dom, vx_hist=None, vz_hist=None, time_chunk: int = 64):
    """(g_Vs, g_Vp, g_rho, g_lam, g_mu, g_rho_lame) on the physical grid,
    FP64 NumPy arrays.  Histories are (nt, nz_t, nx_t) on the padded grid."""
    return imaging_condition_device(Vs, Vp, rho, ex_hist, ez_hist, es_hist, U_a_hist, V_a_hist, dx, dz, dt, pad,
                                    free_surface, nz_dom, nx_dom, vx_hist=vx_hist, vz_hist=vz_hist,
                                    time_chunk=time_chunk)
