"""Forward modelling with the reference's signatures (fwi/forward.py).

Full wavefields ('vx_full' .. 'es_full', ``return_wavefields``) come from
stfwi_forward_frames: the state of every step copied out of the GPU into a
page-locked host array (nt x nz_t x nx_t float32 per field and shot).

``build_forward_fn(...)`` returns ``run_shot(Vs, Vp, rho, src_x, src_z,
src_wavelet)`` as the reference does (fwi/forward.py:508-544), backed by one
GPU handle per geometry; ``run_shot.batch`` runs many shots in one launch
per phase (the reference's ``jax.vmap(run_shot)``).
"""
from __future__ import annotations

import numpy as np

from ..solver import Solver

_REC = {"vx": 0, "vz": 1, "ex": 2, "ez": 3}
_FULL = ("vx_full", "vz_full", "ex_full", "ez_full", "es_full")


def ricker_jax(t, fc, t0, scaling_factor=1):
    """(1 - 2a) e^(-a), a = (pi fc (t - t0))^2 (fwi/forward.py:25-28)."""
    arg = (np.pi * fc * (np.asarray(t, dtype=np.float64) - t0)) ** 2
    return scaling_factor * (1.0 - 2.0 * arg) * np.exp(-arg)


def _check_vars(return_vars):
    if return_vars is None:
        return ("vx", "vz", "ex", "ez")
    for k in return_vars:
        if k not in _REC and k not in _FULL:
            raise ValueError(f"unknown return var {k!r}")
    return tuple(return_vars)


class _ShotRunner:
    """Holds one Solver per shot-batch size for a fixed geometry."""

    def __init__(self, nz, nx, dx, dz, dt, nt, freq, pad, rec_x, rec_z, fd_order, free_surface,
                 return_vars, src_type="force"):
        self.geo = dict(nz_dom=int(nz), nx_dom=int(nx), dx=float(dx), dz=float(dz), dt=float(dt),
                        nt=int(nt), fc=float(freq), pad=int(pad), fd_order=int(fd_order),
                        free_surface=bool(free_surface))
        self.rec_x = np.asarray(rec_x, dtype=np.int32).reshape(-1)
        self.rec_z = np.asarray(rec_z, dtype=np.int32).reshape(-1)
        self.vars = _check_vars(return_vars)
        self.src_type = src_type
        self._solvers = {}

    def solver(self, nshot, want_gradient=False):
        key = (nshot, want_gradient)
        S = self._solvers.get(key)
        if S is None:
            g = self.geo
            S = Solver(g["nz_dom"], g["nx_dom"], g["dx"], g["dz"], g["dt"], g["nt"], g["fc"], g["pad"],
                       self.rec_x.size, nshot, fd_order=g["fd_order"], free_surface=g["free_surface"],
                       want_gradient=want_gradient)
            S.set_receivers(self.rec_x, self.rec_z)
            self._solvers[key] = S
        return S

    def batch(self, Vs, Vp, rho, src_x, src_z, src_wavelet, src_type=None):
        """All shots at once: a tuple of (nshot, nt, nrec) arrays."""
        sx = np.atleast_1d(np.asarray(src_x)).astype(np.int64)
        sz = np.broadcast_to(np.atleast_1d(np.asarray(src_z)), sx.shape).astype(np.int64)
        S = self.solver(sx.size)
        S.set_model(Vs, Vp, rho)
        S.set_shots(sx, sz, src_type or self.src_type, np.asarray(src_wavelet, dtype=np.float32))
        full = [k[:-5] for k in self.vars if k in _FULL]
        if full:
            # full wavefields (fwi/forward.py:449-463): frames after every step
            frames, _ = S.forward_frames(full)
        else:
            S.forward()
        rec = S.records()
        return tuple(frames[k[:-5]] if k in _FULL else rec[:, _REC[k]] for k in self.vars)

    def __call__(self, Vs, Vp, rho, src_x, src_z, src_wavelet):
        out = self.batch(Vs, Vp, rho, [int(src_x)], [int(src_z)], src_wavelet)
        return tuple(o[0] for o in out)


def build_forward_fn(nz, nx, dx, dz, dt, nt, freq, pad, block_size, rec_x, rec_z, fd_order=2,
                     return_vars=None, free_surface=True):
    """run_shot(Vs, Vp, rho, src_x, src_z, src_wavelet) -> tuple of (nt, nrec)
    arrays (fwi/forward.py:508-544).  Like the reference, the source is a
    vertical force (its build_forward_fn does not pass src_type);
    ``block_size`` (the reference's AD checkpoint interval) has no effect."""
    return _ShotRunner(nz, nx, dx, dz, dt, nt, freq, pad, rec_x, rec_z, fd_order, free_surface,
                       return_vars)


def forward_jax(Vs, Vp, rho, src_x, src_z, rec_x, rec_z, nx_dom, nz_dom, dx, dz, dt, nt, fc, pad,
                src_wavelet, return_wavefields=False, block_size=100, return_vars=None, fd_order=2,
                free_surface=True, src_type="force"):
    """One shot of fwi/forward.py:119-501 on the GPU; returns
    (rec_vx, rec_vz, rec_exx, rec_ezz), with ``return_wavefields`` followed
    by the (nt, nz_t, nx_t) frames of U, V, exx, ezz, or the requested
    ``return_vars`` (receiver names and '*_full' frames)."""
    if fd_order not in (2, 4, 8):
        raise NotImplementedError(f"fd_order={fd_order} not supported (use 2, 4, or 8).")
    if src_type not in ("force", "moment"):
        raise NotImplementedError(f"src_type={src_type!r} not supported (use 'force' or 'moment').")
    if return_wavefields and return_vars is None:
        # fwi/forward.py:460-461: the receiver tuple, then the U, V, ex, ez frames
        return_vars = ["vx", "vz", "ex", "ez", "vx_full", "vz_full", "ex_full", "ez_full"]
    run = _ShotRunner(nz_dom, nx_dom, dx, dz, dt, nt, fc, pad, rec_x, rec_z, fd_order, free_surface,
                      return_vars, src_type)
    try:
        out = run.batch(Vs, Vp, rho, [int(src_x)], [int(src_z)], src_wavelet)
        return tuple(o[0] for o in out)
    finally:
        for S in run._solvers.values():
            S.close()
