"""The C ABI without a GPU: the library loads, exports every function that
include/stfwi.h declares, and its host-only paths behave."""
import ctypes as ct
import os
import re

import pytest

from tests.conftest import ROOT


def _declared(header="stfwi.h"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(stfwi_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from stfwi_b200 import _native as N
    lib = N.load()
    names = _declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(N.EXPORTS), set(names) ^ set(N.EXPORTS)


def test_library_exports_every_network_symbol():
    """include/stfwi_nn.h (the learned preconditioner's kernels)."""
    from stfwi_b200 import _native as N
    lib = N.load()
    names = _declared("stfwi_nn.h")
    assert len(names) >= 14
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(N.NN_EXPORTS), set(names) ^ set(N.NN_EXPORTS)


def test_network_calls_reject_bad_shapes_on_the_host():
    """Shape checks run before any launch, so they answer without a GPU."""
    from stfwi_b200 import _native as N
    lib = N.load()
    x = ct.c_void_p(16)
    # channel count not a multiple of 16
    assert lib.stfwi_nn_conv3x3(x, 1, 128, 128, 24, x, 32, None, 1, x, 32, 0, None) == N.STFWI_ERR_INVALID
    assert b"multiples of 16" in lib.stfwi_nn_last_error()
    # 100 pixels wide does not tile into 128-pixel boxes
    assert lib.stfwi_nn_conv3x3(x, 1, 128, 100, 32, x, 32, None, 1, x, 32, 0, None) == N.STFWI_ERR_INVALID
    # output slice past the channel stride
    assert lib.stfwi_nn_conv3x3(x, 1, 128, 128, 32, x, 32, None, 1, x, 48, 24, None) == N.STFWI_ERR_INVALID
    # weight gradient width not a multiple of 64
    assert lib.stfwi_nn_conv3x3_wgrad(x, x, 1, 64, 96, 32, 32, x, None) == N.STFWI_ERR_INVALID
    # unaligned pointer
    assert lib.stfwi_nn_conv3x3(ct.c_void_p(8), 1, 128, 128, 32, x, 32, None, 1, x, 32, 0, None) == N.STFWI_ERR_INVALID


def test_workspace_and_grid_shape_are_host_only():
    from stfwi_b200 import _native as N
    lib = N.load()
    d = N.StfwiDesc(152, 500, 20, 8, 1, 2000, 250, 50, 20.0, 20.0, 1.5e-3, 5.0, 1, 0, 0.0, 0, 0)
    nz, nx = ct.c_int32(), ct.c_int32()
    lib.stfwi_grid_shape(ct.byref(d), ct.byref(nz), ct.byref(nx))
    assert (nz.value, nx.value) == (172, 540)
    ws = lib.stfwi_workspace_bytes(ct.byref(d))
    # the strain history dominates: 50 shots x 2000 steps x 3 x 76000 cells x 4 B
    assert 91e9 < ws < 95e9
    d.ckpt_interval = 200  # checkpoints every 200 steps: 10 x state + a 201-step history
    ws_ck = lib.stfwi_workspace_bytes(ct.byref(d))
    assert 9e9 < ws_ck < 14e9, ws_ck
    d.ckpt_interval = 0
    d.want_gradient = 0
    assert lib.stfwi_workspace_bytes(ct.byref(d)) < 2e9


def test_create_rejects_bad_descriptors_before_touching_a_device():
    from stfwi_b200 import _native as N
    lib = N.load()
    h = ct.c_void_p()
    d = N.StfwiDesc(24, 32, 8, 6, 1, 10, 3, 1, 10.0, 10.0, 1e-3, 15.0, 0, 0, 0.0, 0, 0)
    assert lib.stfwi_create(ct.byref(d), ct.byref(h)) == N.STFWI_ERR_UNSUPPORTED
    d.fd_order = 8
    d.pad = 2  # thinner than the stencil half-width
    assert lib.stfwi_create(ct.byref(d), ct.byref(h)) == N.STFWI_ERR_INVALID
    d.pad, d.dt = 8, -1.0
    assert lib.stfwi_create(ct.byref(d), ct.byref(h)) == N.STFWI_ERR_INVALID
    d.dt = 1e-3
    d.want_gradient, d.kernel_variant = 2, 5   # an unknown kernel_variant is refused
    assert lib.stfwi_create(ct.byref(d), ct.byref(h)) == N.STFWI_ERR_UNSUPPORTED
    d.want_gradient, d.kernel_variant = 3, 0
    assert lib.stfwi_create(ct.byref(d), ct.byref(h)) == N.STFWI_ERR_INVALID


def test_density_history_holds_five_fields_per_step():
    """want_gradient = 2 (density gradient) keeps U and V beside the three
    stresses: 5/3 of the history bytes, plus one extra slot with checkpoints."""
    from stfwi_b200 import _native as N
    lib = N.load()
    d = N.StfwiDesc(152, 500, 20, 8, 1, 2000, 250, 50, 20.0, 20.0, 1.5e-3, 5.0, 1, 0, 0.0, 0, 0)
    w1 = lib.stfwi_workspace_bytes(ct.byref(d))
    d.want_gradient = 2
    w2 = lib.stfwi_workspace_bytes(ct.byref(d))
    hist = 50 * 2001 * 3 * 152 * 500 * 4
    assert abs((w2 - w1) - 2 * hist / 3) < 0.01 * hist, (w1, w2)


def test_noalloc_size_check_runs_on_the_host():
    from stfwi_b200 import _native as N
    lib = N.load()
    m = N.StfwiMisfitDesc(1, 0, 0, 0, 1.0, None)
    dummy = ct.c_void_p(16)
    st = lib.stfwi_misfit_noalloc(2, 10, N.NOALLOC_MAX_TRACES, dummy, dummy, ct.byref(m), dummy, dummy, None)
    assert st == N.STFWI_ERR_INVALID


def test_solver_rejects_unsupported_options_on_the_host():
    from stfwi_b200 import Solver
    with pytest.raises(NotImplementedError):
        Solver(24, 32, 10.0, 10.0, 1e-3, 10, 15.0, 8, 3, 1, fd_order=6)
