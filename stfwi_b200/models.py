"""Seeded synthetic elastic models and the acquisition of the benchmark
configurations.

The layered-fault recipe stands in for the reference's Marmousi-II model
(152 x 500 cells at 20 m): dipping layers whose P velocity grows with depth,
cut by a few faults that shift the layering on one side, with Vp in
[1500, 4700] m/s, Vs in [800, 2750] m/s (Vp/Vs >= 1.2) and rho in
[1700, 2600] kg/m^3.  The initial model is the true one smoothed with a
Gaussian of sigma = 10 cells, applied to slowness for the velocities and
directly to density, as the reference's drivers build theirs
(Main_strain_fwi.py:397-399 smooths 1/V).
"""
from __future__ import annotations

import numpy as np


def layered_fault_model(nz=152, nx=500, seed=0, n_layers=10, n_faults=3):
    """(Vs, Vp, rho) float32 arrays of shape (nz, nx)."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz, dtype=np.float64)[:, None]
    x = np.arange(nx, dtype=np.float64)[None, :]
    # interface depths (fraction of nz) and dips (cells per cell)
    base = np.sort(rng.uniform(0.04, 0.96, n_layers))
    dips = rng.uniform(-0.08, 0.08, n_layers)
    depth = np.broadcast_to(z, (nz, nx)).copy()
    # faults: a line x = x0 + (z - z_mid) * slope; cells right of it are
    # shifted vertically by `throw` (layer index computed at depth - throw)
    for _ in range(n_faults):
        x0 = rng.uniform(0.15, 0.85) * nx
        slope = rng.uniform(-0.4, 0.4)
        throw = rng.uniform(-0.08, 0.08) * nz
        right = x > x0 + (z - nz / 2) * slope
        depth = np.where(right, depth - throw, depth)
    layer = np.zeros((nz, nx), dtype=np.int64)
    for k in range(n_layers):
        iface = base[k] * nz + dips[k] * (x - nx / 2)
        layer += (depth >= iface).astype(np.int64)
    # P velocity per layer: increasing with depth, jittered
    vp_layers = np.linspace(1500.0, 4700.0, n_layers + 1)
    vp_layers[1:-1] += rng.uniform(-120.0, 120.0, n_layers - 1)
    vp_layers = np.clip(vp_layers, 1500.0, 4700.0)
    ratio = rng.uniform(1.55, 2.0, n_layers + 1)
    vp = vp_layers[layer]
    # smooth intra-layer gradient
    vp = vp + 60.0 * (depth / nz - 0.5)
    vp = np.clip(vp, 1500.0, 4700.0)
    vs = np.clip(vp / ratio[layer], 800.0, 2750.0)
    vs = np.minimum(vs, vp / 1.2)
    rho = np.clip(310.0 * vp ** 0.25, 1700.0, 2600.0)
    return vs.astype(np.float32), vp.astype(np.float32), rho.astype(np.float32)


def smooth_initial(vs, vp, rho, sigma=10.0):
    """Gaussian-smoothed starting model (slowness for the velocities)."""
    from scipy.ndimage import gaussian_filter
    vs0 = 1.0 / gaussian_filter(1.0 / vs.astype(np.float64), sigma)
    vp0 = 1.0 / gaussian_filter(1.0 / vp.astype(np.float64), sigma)
    rho0 = gaussian_filter(rho.astype(np.float64), sigma)
    return vs0.astype(np.float32), vp0.astype(np.float32), rho0.astype(np.float32)


def ricker(t, fc, t0, scaling_factor=1.0):
    """(1 - 2a) exp(-a), a = (pi fc (t - t0))^2 (fwi/forward.py:25-28)."""
    arg = (np.pi * fc * (np.asarray(t, dtype=np.float64) - t0)) ** 2
    return scaling_factor * (1.0 - 2.0 * arg) * np.exp(-arg)


def fd_stability_sum(fd_order):
    """Sum of |c_k| of the staggered stencil (the CFL factor S)."""
    if fd_order == 8:
        return 1225 / 1024 + 245 / 3072 + 49 / 5120 + 5 / 7168
    if fd_order >= 4:
        return 9 / 8 + 1 / 24
    return 1.0


def cfl_number(vp_max, dt, dx, dz, fd_order):
    """Vp_max dt S sqrt(1/dx^2 + 1/dz^2); the scheme needs it below 1
    (Main_ex_Vs.py:129-136)."""
    return float(vp_max * dt * fd_stability_sum(fd_order) * np.sqrt(1 / dx ** 2 + 1 / dz ** 2))


# the benchmark configurations (synthetic stand-ins of the reference's setups)
CONFIG1 = dict(name="single-shot gradient 152x500 fd4", nz=152, nx=500, dx=20.0, dz=20.0, pad=20,
               fd_order=4, free_surface=True, nt=2000, dt=1.5e-3, fc=5.0, n_shots=1)
CONFIG2 = dict(name="batched 50 shots 152x500 fd8", nz=152, nx=500, dx=20.0, dz=20.0, pad=20,
               fd_order=8, free_surface=True, nt=2000, dt=1.5e-3, fc=5.0, n_shots=50)


def acquisition(cfg):
    """Shots and receivers of a configuration (physical-domain indices).

    Sources at 40 m depth (z = 2 cells); config 1 has one vertical force at
    x = 5000 m, config 2 has 50 shots every 200 m alternating force and
    moment.  250 receivers at 20 m depth every 40 m."""
    nx = cfg["nx"]
    ns = cfg["n_shots"]
    if ns == 1:
        src_x = np.array([nx // 2])
        types = ["force"]
    else:
        step = max(1, int(round(200.0 / cfg["dx"])))
        src_x = (np.arange(ns) * step) % nx
        types = ["force" if k % 2 == 0 else "moment" for k in range(ns)]
    src_z = np.full(ns, 2)
    rec_x = np.arange(0, nx, 2, dtype=np.int32)
    rec_z = np.ones_like(rec_x)
    return src_x, src_z, types, rec_x, rec_z
