"""adjoint_jax with the reference's signature (fwi/adjoint_jax_kernel.py:61-69)."""
from __future__ import annotations

import numpy as np

from ..solver import Solver


def adjoint_jax(Vs, Vp, rho, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt, fc, pad,
                rec_vx_a, rec_vz_a, rec_ex_a, rec_ez_a, fd_order=2, free_surface=False,
                src_type="force", return_wavefields=False):
    """Discrete transpose of the forward w.r.t. the source wavelet: receiver
    adjoints (4 x (nt, nrec)) -> src_wavelet_a (nt,); with
    ``return_wavefields`` also the adjoint frames (nt, nz_t, nx_t) of U_a,
    V_a (and, unless it is 'velocity', ex_a, ez_a, es_a)."""
    if fd_order not in (2, 4, 8):
        raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
    if src_type not in ("force", "moment"):
        raise NotImplementedError(f"src_type={src_type!r} not supported (use 'force' or 'moment').")
    rec_x = np.asarray(rec_x, dtype=np.int32).reshape(-1)
    rec_z = np.asarray(rec_z, dtype=np.int32).reshape(-1)
    S = Solver(nz_dom, nx_dom, dx, dz, dt, nt, fc, pad, rec_x.size, 1, fd_order=fd_order,
               free_surface=free_surface, want_gradient=False)
    try:
        S.set_model(Vs, Vp, rho)
        S.set_receivers(rec_x, rec_z)
        S.set_shots([int(src_x)], [int(src_z)], [src_type], np.zeros(nt, dtype=np.float32))
        ra = np.stack([np.asarray(a, dtype=np.float32) for a in (rec_vx_a, rec_vz_a, rec_ex_a, rec_ez_a)])
        S.set_adjoint_sources(ra[None])
        if not return_wavefields:
            return S.gradient(exact=False, src=True)["src"][0].astype(np.float64)
        # fwi/adjoint_jax_kernel.py:91-93, 470-483: 'velocity' -> (src_a, U_a, V_a);
        # True -> (src_a, U_a, V_a, ex_a, ez_a, es_a); frames in forward-time order
        fields = ("vx", "vz") if return_wavefields == "velocity" else ("vx", "vz", "ex", "ez", "es")
        sa, frames, _ = S.adjoint_frames(fields)
        return (sa[0].astype(np.float64),) + tuple(frames[f][0] for f in fields)
    finally:
        S.close()
