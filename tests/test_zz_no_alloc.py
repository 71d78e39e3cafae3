"""sw2d_get_array_noalloc: reading a result array without any device allocation.

Some callers must not allocate device memory once their run has started (a forecasting
service that reserves its memory at start-up so that it cannot fail with out-of-memory in the
middle of an event, an application whose memory pool forbids allocations from library code).
The entry point stages the array in a fixed buffer compiled into the library instead of a
buffer allocated per call.  These tests call it through the C ABI and compare it with
sw2d_get_array, bit for bit (the tolerance of the parity tests for these arrays), on two calls
in a row, check the size limit, serve the DDP model's map outputs too, and check the property
the entry point exists for: free device memory is the same before and after a call.  This file
is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu

NAMES = ["slope_x", "slope_y", "F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd",
         "lambda_max_int", "lambda_max_bnd"]
LIMIT = 1 << 20


def _get(model, fn, name, n):
    out = np.full(n, np.nan)
    k = fn(model.handle, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size)
    return k, out


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


def test_noalloc_matches_get_array_on_two_calls(pkg):
    case = pkg.workloads.channel_features(n_cells=2500, scheme="muscl_evr", topo="blending", friction="strickler")
    model = pkg.SpModel(case)
    model.set_option("record_wave_speeds", 1)
    model.set_option("record_fluxes", 1)
    n = max(model.n, model.ni, model.nb)
    lib = model.lib
    for call, steps in enumerate((5, 7)):
        assert model.step(steps) == steps
        for name in NAMES:
            k_ref, ref = _get(model, lib.sw2d_get_array, name, n)
            k_new, new = _get(model, lib.sw2d_get_array_noalloc, name, n)
            assert k_ref == k_new > 0, name
            assert np.array_equal(ref[:k_ref].view(np.int64), new[:k_new].view(np.int64)), f"{name}, call {call + 1}"
    # two calls in a row on the same state give the same bits
    a = _get(model, lib.sw2d_get_array_noalloc, "F2_int", n)[1]
    b = _get(model, lib.sw2d_get_array_noalloc, "F2_int", n)[1]
    assert np.array_equal(a.view(np.int64), b.view(np.int64))


def test_noalloc_rejects_arrays_beyond_its_fixed_size(pkg):
    case = pkg.workloads.gaussian_bumps(n_cells=1_150_000)
    model = pkg.SpModel(case)
    assert model.n > LIMIT
    model.set_option("record_fluxes", 1)   # the fused step keeps the slopes only while recording
    model.step(1)
    out = np.empty(model.n)
    k = model.lib.sw2d_get_array_noalloc(model.handle, b"slope_x", out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         out.size)
    assert k == -1
    msg = model.lib.sw2d_last_error(model.handle).decode()
    assert str(LIMIT) in msg and "sw2d_get_array" in msg
    # the allocating entry point still serves it
    k2 = model.lib.sw2d_get_array(model.handle, b"slope_x", out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  out.size)
    assert k2 == model.n


DDP_NAMES = ["water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation", "thetaG_int_hmin"]


def test_noalloc_serves_the_ddp_map_outputs(pkg):
    case = pkg.workloads.ddp_channel(n_cells=2500, laws="linear", friction="manning", outflow="fr", t_max=1.0e9,
                                     seed=61)
    model = pkg.SpModel(case)
    n = max(model.n, model.ni, model.nb)
    lib = model.lib
    for call, steps in enumerate((4, 9)):
        assert model.step(steps) == steps
        for name in DDP_NAMES:
            k_ref, ref = _get(model, lib.sw2d_get_array, name, n)
            k_new, new = _get(model, lib.sw2d_get_array_noalloc, name, n)
            assert k_ref == k_new > 0, name
            assert np.array_equal(ref[:k_ref].view(np.int64), new[:k_new].view(np.int64)), f"{name}, call {call + 1}"


def test_noalloc_leaves_free_device_memory_unchanged(pkg):
    """A call on an array of ~0.9M doubles (7 MB; the allocating entry point would take and give
    back a buffer of that size) leaves cudaMemGetInfo's free bytes exactly where they were."""
    import torch

    case = pkg.workloads.gaussian_bumps(n_cells=900_000)
    model = pkg.SpModel(case)
    model.set_option("record_fluxes", 1)
    assert model.step(2) == 2
    out = np.empty(model.n)
    ptr = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    lib = model.lib
    assert lib.sw2d_get_array_noalloc(model.handle, b"slope_x", ptr, out.size) == model.n   # warm (module loads)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for name in (b"slope_x", b"slope_y"):
        assert lib.sw2d_get_array_noalloc(model.handle, name, ptr, out.size) == model.n
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"
    ref = np.empty(model.n)
    assert lib.sw2d_get_array(model.handle, b"slope_y", ref.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              ref.size) == model.n
    assert np.array_equal(ref.view(np.int64), out.view(np.int64))
