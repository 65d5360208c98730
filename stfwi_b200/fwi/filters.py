"""Host-side trace filters (fwi/filters.py): the residual filtering itself
runs on the GPU inside the misfit kernel; these NumPy versions serve callers
that filter observed data on the host."""
from __future__ import annotations

import numpy as np


def cosine_taper_end(x, n_taper):
    """Taper the last ``n_taper`` samples of axis 0 with (cos + 1)/2, 1 -> 0
    (fwi/filters.py:26-32)."""
    x = np.array(x, dtype=np.result_type(x, np.float32), copy=True)
    n_taper = min(int(n_taper), x.shape[0])
    if n_taper <= 0:
        return x
    taper = (np.cos(np.arange(1, n_taper + 1) / n_taper * np.pi) + 1) / 2
    x[-n_taper:] *= taper.reshape((-1,) + (1,) * (x.ndim - 1)).astype(x.dtype)
    return x


def sosfilt(x, sos):
    """Cascade of direct-form-I biquads along axis 0, each normalised by a0
    (fwi/filters.py:14-40)."""
    from scipy.signal import sosfilt as _sosfilt
    return _sosfilt(np.asarray(sos, dtype=np.float64), np.asarray(x), axis=0)


jax_sosfilt = sosfilt
