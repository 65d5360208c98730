"""Drop-in mirror of the reference's ``fwi`` hot-path API on the CUDA path.

Same function names, argument order and meaning, and exceptions as the
reference's ``fwi.forward``, ``fwi.adjoint_jax_kernel``, ``fwi.gradient``,
``fwi.illumination``, ``fwi.imaging``, ``fwi.loss``, ``fwi.filters``, ``fwi.projections``
and ``fwi.optim_lbfgsb``; arrays come back as NumPy arrays instead of JAX
arrays.
"""
from .filters import cosine_taper_end, jax_sosfilt, sosfilt  # noqa: F401
from .forward import build_forward_fn, forward_jax, ricker_jax  # noqa: F401
from .adjoint import adjoint_jax  # noqa: F401
from .gradient import compute_gradient  # noqa: F401
from .illumination import compute_illumination_for_stage  # noqa: F401
from .imaging import imaging_condition  # noqa: F401
from .loss import build_loss_fn, gaussian_smooth_2d  # noqa: F401
from .optim_lbfgsb import run_multiscale_fwi  # noqa: F401
from .projections import cfl_vp_cap, k_safe_ratio, project_velocity, project_velocity_device  # noqa: F401
