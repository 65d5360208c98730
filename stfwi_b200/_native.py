"""ctypes binding of include/stfwi.h (libstfwi.so, built in-tree for sm_100a).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# STFWI_LIB selects another build of the same C ABI (e.g. a tuning variant)
LIB_PATH = os.environ.get("STFWI_LIB") or os.path.join(HERE, "libstfwi.so")

STFWI_OK, STFWI_ERR_INVALID, STFWI_ERR_UNSUPPORTED, STFWI_ERR_CUDA = 0, 1, 2, 3
STFWI_ERR_OOM, STFWI_ERR_NONFINITE, STFWI_ERR_STATE, STFWI_ERR_TIMEOUT = 4, 5, 6, 7
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "UNSUPPORTED", 3: "CUDA", 4: "OOM", 5: "NONFINITE", 6: "STATE",
                7: "TIMEOUT"}

SRC_FORCE, SRC_MOMENT = 0, 1
FWD_STORE = 1
GRAD_EXACT, GRAD_IMAGING, GRAD_SRC = 1, 2, 4

# every symbol include/stfwi.h declares
EXPORTS = (
    "stfwi_workspace_bytes", "stfwi_create", "stfwi_destroy", "stfwi_last_error", "stfwi_set_model",
    "stfwi_set_receivers", "stfwi_set_shots", "stfwi_forward", "stfwi_get_records", "stfwi_misfit",
    "stfwi_set_adjoint_sources", "stfwi_gradient", "stfwi_illumination", "stfwi_check",
    "stfwi_grid_shape", "stfwi_profile", "stfwi_kernel_times", "stfwi_misfit_noalloc",
    "stfwi_set_postprocess", "stfwi_preconditioner", "stfwi_project_velocity", "stfwi_autotune",
    "stfwi_forward_frames", "stfwi_adjoint_frames", "stfwi_imaging_condition", "stfwi_set_wait_limit",
    "stfwi_set_tile_rows", "stfwi_tile_rows", "stfwi_set_chains",
)

# full wavefield frames (bit set, in this order)
FRAME_BITS = {"vx": 1, "vz": 2, "ex": 4, "ez": 8, "es": 16}

# every symbol include/stfwi_nn.h declares (the learned preconditioner's network kernels)
NN_EXPORTS = (
    "stfwi_nn_last_error", "stfwi_nn_check", "stfwi_nn_conv3x3", "stfwi_nn_conv3x3_dgrad",
    "stfwi_nn_conv3x3_wgrad", "stfwi_nn_pack_input", "stfwi_nn_avgpool2", "stfwi_nn_skip_grad",
    "stfwi_nn_upsample2", "stfwi_nn_upsample2_grad", "stfwi_nn_head", "stfwi_nn_head_loss_grad",
    "stfwi_nn_bias_grad", "stfwi_nn_pack_weights", "stfwi_nn_adam",
)

PRECOND_ILLUM, PRECOND_EPRECOND3 = 0, 1

NOALLOC_MAX_TRACES = 1 << 18


class StfwiDesc(ct.Structure):
    _fields_ = [
        ("nz_dom", ct.c_int32), ("nx_dom", ct.c_int32), ("pad", ct.c_int32),
        ("fd_order", ct.c_int32), ("free_surface", ct.c_int32), ("nt", ct.c_int32),
        ("nrec", ct.c_int32), ("max_shots", ct.c_int32),
        ("dx", ct.c_double), ("dz", ct.c_double), ("dt", ct.c_double), ("fc", ct.c_double),
        ("want_gradient", ct.c_int32), ("shot_group", ct.c_int32), ("mem_budget_gb", ct.c_double),
        ("kernel_variant", ct.c_int32), ("ckpt_interval", ct.c_int32),
    ]


class StfwiMisfitDesc(ct.Structure):
    _fields_ = [
        ("component", ct.c_int32), ("n_taper", ct.c_int32), ("nsos", ct.c_int32),
        ("nshot_norm", ct.c_int32), ("scale", ct.c_double), ("sos", ct.POINTER(ct.c_double)),
    ]


class StfwiImagingDesc(ct.Structure):
    _fields_ = [
        ("nz_dom", ct.c_int32), ("nx_dom", ct.c_int32), ("pad", ct.c_int32), ("free_surface", ct.c_int32),
        ("nt", ct.c_int32), ("time_chunk", ct.c_int32),
        ("dx", ct.c_double), ("dz", ct.c_double), ("dt", ct.c_double),
    ]


class StfwiError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"stfwi {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load():
    """Load libstfwi.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m stfwi_b200.build`")
        L = ct.CDLL(LIB_PATH)
        vp, i32, u32 = ct.c_void_p, ct.c_int32, ct.c_uint32
        H = ct.c_void_p
        L.stfwi_workspace_bytes.argtypes = [ct.POINTER(StfwiDesc)]
        L.stfwi_workspace_bytes.restype = ct.c_size_t
        L.stfwi_create.argtypes = [ct.POINTER(StfwiDesc), ct.POINTER(H)]
        L.stfwi_destroy.argtypes = [H]
        L.stfwi_destroy.restype = None
        L.stfwi_last_error.argtypes = [H]
        L.stfwi_last_error.restype = ct.c_char_p
        L.stfwi_set_model.argtypes = [H, vp, vp, vp, vp]
        L.stfwi_set_receivers.argtypes = [H, i32, vp, vp]
        L.stfwi_set_shots.argtypes = [H, i32, vp, vp, vp]
        L.stfwi_forward.argtypes = [H, u32, vp]
        L.stfwi_get_records.argtypes = [H, vp, vp]
        L.stfwi_misfit.argtypes = [H, vp, ct.POINTER(StfwiMisfitDesc), vp, vp]
        L.stfwi_set_adjoint_sources.argtypes = [H, vp, vp]
        L.stfwi_gradient.argtypes = [H, u32, vp, vp, vp]
        L.stfwi_illumination.argtypes = [H, i32, vp, vp]
        L.stfwi_check.argtypes = [H, vp]
        L.stfwi_grid_shape.argtypes = [ct.POINTER(StfwiDesc), ct.POINTER(i32), ct.POINTER(i32)]
        L.stfwi_grid_shape.restype = None
        L.stfwi_profile.argtypes = [H, i32]
        L.stfwi_kernel_times.argtypes = [H, vp]
        L.stfwi_misfit_noalloc.argtypes = [i32, i32, i32, vp, vp, ct.POINTER(StfwiMisfitDesc), vp, vp, vp]
        f64 = ct.c_double
        L.stfwi_set_postprocess.argtypes = [H, f64, vp, vp, vp]
        L.stfwi_preconditioner.argtypes = [H, i32, i32, f64, vp, vp]
        L.stfwi_project_velocity.argtypes = [ct.c_int64, vp, vp, vp, f64, f64, f64, f64, vp]
        L.stfwi_autotune.argtypes = [H, i32, vp, vp]
        L.stfwi_forward_frames.argtypes = [H, u32, vp, vp]
        L.stfwi_set_wait_limit.argtypes = [H, ct.c_int64]
        L.stfwi_set_tile_rows.argtypes = [H, i32, i32]
        L.stfwi_tile_rows.argtypes = [H, vp]
        L.stfwi_set_chains.argtypes = [H, i32]
        L.stfwi_adjoint_frames.argtypes = [H, u32, vp, vp, vp]
        L.stfwi_imaging_condition.argtypes = [ct.POINTER(StfwiImagingDesc)] + [vp] * 10 + [vp, vp]
        sz, f32 = ct.c_size_t, ct.c_float
        L.stfwi_nn_last_error.argtypes = []
        L.stfwi_nn_last_error.restype = ct.c_char_p
        L.stfwi_nn_check.argtypes = [vp]
        L.stfwi_nn_conv3x3.argtypes = [vp, i32, i32, i32, i32, vp, i32, vp, i32, vp, i32, i32, vp]
        L.stfwi_nn_conv3x3_dgrad.argtypes = [vp, i32, i32, i32, i32, vp, i32, vp, i32, i32, vp, vp]
        L.stfwi_nn_conv3x3_wgrad.argtypes = [vp, vp, i32, i32, i32, i32, i32, vp, vp]
        L.stfwi_nn_pack_input.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp, vp]
        L.stfwi_nn_avgpool2.argtypes = [vp, i32, i32, i32, i32, i32, i32, vp, vp]
        L.stfwi_nn_skip_grad.argtypes = [vp, vp, i32, i32, vp, i32, i32, i32, i32, vp, vp]
        L.stfwi_nn_upsample2.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp]
        L.stfwi_nn_upsample2_grad.argtypes = [vp, i32, vp, i32, i32, i32, i32, vp, vp]
        L.stfwi_nn_head.argtypes = [vp, sz, i32, vp, vp, vp, vp]
        L.stfwi_nn_head_loss_grad.argtypes = [vp, sz, i32, vp, vp, vp, vp, f32, vp, vp, vp, vp, vp]
        L.stfwi_nn_bias_grad.argtypes = [vp, sz, i32, vp, vp]
        L.stfwi_nn_pack_weights.argtypes = [vp, i32, i32, vp, vp, vp]
        L.stfwi_nn_adam.argtypes = [vp, vp, vp, vp, sz, f32, f32, f32, f32, f32, vp]
        _lib = L
    return _lib
