"""build_loss_fn with the reference's signature (fwi/loss.py:33-152)."""
from __future__ import annotations

import numpy as np


def gaussian_smooth_2d(field, sigma, truncate=3.0):
    """Normalised 2-D Gaussian, 'same'-size zero-padded convolution
    (fwi/loss.py:17-30)."""
    from scipy.signal import convolve2d
    radius = int(truncate * sigma + 0.5)
    x = np.arange(2 * radius + 1) - radius
    g1 = np.exp(-0.5 * (x / sigma) ** 2)
    k = np.outer(g1, g1)
    k = k / k.sum()
    return convolve2d(np.asarray(field, dtype=np.float64), k, mode="same")


def _diff_reg(a):
    """sum(diff(a, 0)^2) + sum(diff(a, 1)^2) and its gradient."""
    a = np.asarray(a, dtype=np.float64)
    d0, d1 = np.diff(a, axis=0), np.diff(a, axis=1)
    g = np.zeros_like(a)
    g[1:, :] += 2 * d0
    g[:-1, :] -= 2 * d0
    g[:, 1:] += 2 * d1
    g[:, :-1] -= 2 * d1
    return float(np.sum(d0 ** 2) + np.sum(d1 ** 2)), g


def build_loss_fn(run_shot, observed, src_x_list, src_z, src_wavelet, component=1, scale=1e20, invert="vs",
                  sos=None, n_taper=0, source_taper=None, grad_smooth_sigma=None, tikhonov_alpha=None,
                  illumination=None):
    """value_and_grad-style loss: ``loss_fn((Vs, Vp, rho)) -> (loss, (g_Vs,
    g_Vp, g_rho))``.  ``run_shot`` comes from this package's
    build_forward_fn.  As in the reference, every shot uses ``src_z[0]``
    (fwi/loss.py:90) and the sources are forces."""
    from .gradient import _postprocess, _solver
    if invert not in ("vs", "vs_vp", "all"):
        raise ValueError(f"invert={invert!r}; use 'vs', 'vs_vp', or 'all'")
    geo = run_shot.geo
    sx = np.asarray(src_x_list).astype(np.int64).reshape(-1)
    sz = np.full(sx.shape, int(np.asarray(src_z).reshape(-1)[0]))
    obs = np.asarray(observed, dtype=np.float32)

    def loss_fn(params):
        Vs, Vp, rho = params
        S = _solver(geo["nz_dom"], geo["nx_dom"], geo["dx"], geo["dz"], geo["dt"], geo["nt"], geo["fc"],
                    geo["pad"], run_shot.rec_x.size, sx.size, geo["fd_order"], geo["free_surface"],
                    density=(invert == "all"))
        S.set_receivers(run_shot.rec_x, run_shot.rec_z)
        S.set_shots(sx, sz, "force", np.asarray(src_wavelet, dtype=np.float32))
        S.set_model(Vs, Vp, rho)
        S.forward(store=True)
        total = float(S.misfit(obs, component, scale, sos, n_taper).sum())
        S.set_postprocess(None, None, None)   # post-processing below, after the Tikhonov term
        g_vs, g_vp, g_rho = (np.array(a) for a in S.gradient(exact=True)["exact"])
        # fwi/loss.py:73-78: frozen parameters are stop-gradient
        if invert == "vs":
            g_vp = np.zeros_like(g_vp)
        if invert != "all":
            g_rho = np.zeros_like(g_rho)
        if tikhonov_alpha is not None:
            # fwi/loss.py:91-98: first-difference penalty on the inverted
            # parameters, weighted as a fraction of the misfit (the weight
            # itself is stop-gradient)
            reg, dreg_vs = _diff_reg(Vs)
            dregs = [dreg_vs, None, None]
            if invert in ("vs_vp", "all"):
                r2, dregs[1] = _diff_reg(Vp)
                reg += r2
            if invert == "all":
                r3, dregs[2] = _diff_reg(rho)
                reg += r3
            reg_scale = total / (reg + 1e-30)
            total = total + tikhonov_alpha * reg_scale * reg
            g_vs = g_vs + tikhonov_alpha * reg_scale * dregs[0]
            if dregs[1] is not None:
                g_vp = g_vp + tikhonov_alpha * reg_scale * dregs[1]
            if dregs[2] is not None:
                g_rho = g_rho + tikhonov_alpha * reg_scale * dregs[2]
        grads = _postprocess((g_vs, g_vp, g_rho), grad_smooth_sigma, source_taper, illumination)
        return total, grads

    return loss_fn
