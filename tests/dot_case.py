"""The reference's dot-product test case (test_adjoint_kernel.py:33-74),
restated as data: the 24x32 sinusoidal model, acquisition and the seeded
random wavelet / receiver adjoints (rng seed 2026, same draw order)."""
import numpy as np

NZ, NX = 24, 32
DZ = DX = 10.0
NT = 60
DT = 1.0e-3
FC = 15.0
PAD = 8
CONFIGS = [(fd, fs, st) for fd in (2, 4, 8) for fs in (False, True) for st in ("force", "moment")]


def model(dtype=np.float64):
    zz, xx = np.meshgrid(np.arange(NZ), np.arange(NX), indexing="ij")
    vp = 2500.0 + 150.0 * np.sin(2 * np.pi * zz / NZ) * np.cos(2 * np.pi * xx / NX)
    vs = 1400.0 + 80.0 * np.cos(2 * np.pi * zz / NZ) * np.sin(2 * np.pi * xx / NX)
    rho = 2000.0 + 100.0 * np.sin(np.pi * zz / NZ) * np.cos(np.pi * xx / NX)
    return vs.astype(dtype), vp.astype(dtype), rho.astype(dtype)


def acquisition(free_surface, src_type):
    src_x = NX // 3
    rec_x = np.arange(2, NX - 2, 4, dtype=np.int32)
    if src_type == "moment":
        src_z = NZ // 4
    elif free_surface:
        src_z = 0
    else:
        src_z = NZ // 4
    rec_z = np.zeros_like(rec_x) if free_surface else np.full_like(rec_x, NZ // 5)
    return src_x, src_z, rec_x, rec_z


def random_vectors():
    rng = np.random.default_rng(2026)
    nrec = len(np.arange(2, NX - 2, 4))
    s_in = rng.standard_normal(NT)
    ys = [rng.standard_normal((NT, nrec)) for _ in range(4)]
    return s_in, ys
