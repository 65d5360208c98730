"""Velocity feasibility projections with the reference's signatures
(fwi/projections.py): K > 0 with a margin (Vp/Vs >= (1 + K_margin) 2/sqrt(3)),
a CFL ceiling on Vp, floors on Vs and rho.

``project_velocity`` works on host arrays (NumPy, FP64) like the reference;
``project_velocity_device`` (re-exported from the solver module) does the
same arithmetic in place on CUDA FP64 tensors, which is what the multiscale
driver uses before every gradient evaluation.
"""
from __future__ import annotations

import numpy as np

from ..solver import project_velocity_device  # noqa: F401

R_CONTINUUM = 2.0 / np.sqrt(3.0)   # Vp/Vs where the bulk modulus is zero


def k_safe_ratio(K_margin: float = 0.04) -> float:
    """Vp/Vs lower bound r = (1 + K_margin) 2/sqrt(3) (fwi/projections.py:37-48)."""
    return (1.0 + float(K_margin)) * R_CONTINUUM


def cfl_vp_cap(dx: float, dz: float, dt: float, cfl_coeff: float) -> float:
    """Largest Vp the explicit scheme tolerates: cfl_coeff min(dx, dz) / dt
    (fwi/projections.py:51-62)."""
    return float(cfl_coeff) * float(min(dx, dz)) / float(dt)


def project_velocity(Vs, Vp, rho, K_margin: float = 0.04, vp_cap=None, vs_floor: float = 1e-3,
                     rho_floor: float = 1e-3):
    """Projected FP64 copies (Vs, Vp, rho): Vp <= vp_cap first, then Vs <=
    Vp / r, then the floors (fwi/projections.py:67-117)."""
    vp_p = np.asarray(Vp, dtype=np.float64).copy()
    vs_p = np.asarray(Vs, dtype=np.float64).copy()
    rho_p = np.asarray(rho, dtype=np.float64).copy()
    r = k_safe_ratio(K_margin)
    if vp_cap is not None:
        np.minimum(vp_p, float(vp_cap), out=vp_p)
    np.minimum(vs_p, vp_p / r, out=vs_p)
    np.maximum(vs_p, float(vs_floor), out=vs_p)
    np.maximum(rho_p, float(rho_floor), out=rho_p)
    return vs_p, vp_p, rho_p
