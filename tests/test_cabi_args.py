"""Argument checks of the C ABI that return before any device work, so they run without a
GPU: every entry point rejects null or inconsistent arguments with PXL_ERR_ARG (-1) or
PXL_ERR_CAPACITY (-4) instead of faulting."""
import ctypes

from pixeltrack import _native


def test_fit_entry_points_reject_bad_arguments():
    L = _native.lib()
    assert L.pxl_bl_fit(None, None, None, 4, 0.01, 0, None, None, None, None, None, None, None, 0, None) == -1
    assert L.pxl_bl_fit(1, 1, 1, -1, 0.01, 0, 1, 1, 1, 1, 1, 1, 1, 1 << 20, None) == -1
    assert L.pxl_bl_fit(1, 1, 1, 4, 0.01, 7, 1, 1, 1, 1, 1, 1, 1, 1 << 20, None) == -1  # precision
    assert L.pxl_bl_fit(1, 1, 1, 1 << 20, 0.01, 0, 1, 1, 1, 1, 1, 1, 1, 64, None) == -4  # workspace too small
    assert L.pxl_riemann_fit(None, None, None, 4, 0.01, 0, None, None, None, None, None, 0, None) == -1
    assert L.pxl_riemann_fit(1, 1, 1, 1 << 20, 0.01, 1, 1, 1, 1, 1, 1, 64, None) == -4
    # alignment gradients need module ids and centres
    assert L.pxl_bl_fit_adjoint(1, 1, 1, 4, 0.01, None, None, None, 0, None, 1, 1, None, 1, 1 << 20, None) == -1
    assert L.pxl_fit_workspace_bytes(1000) >= 4 * 1000
    assert L.pxl_adjoint_workspace_bytes(1000, 1856) >= L.pxl_fit_workspace_bytes(1000) + 6 * 1856 * 8


def test_context_entry_points_reject_null():
    L = _native.lib()
    h = ctypes.c_void_p()
    assert L.pxl_ctx_create(None, None, ctypes.byref(h)) == -1
    assert L.pxl_ctx_destroy(None) == -1
    assert L.pxl_event_run(None, None, 0, 63, None) == -1
    assert L.pxl_batch_run(None, None, None, 0, 0, 63, None) == -1
    assert L.pxl_autotune(None, None, 0, 1, None) == -1
    assert L.pxl_clusterize_digis_noalloc(1, 1, 1, 1, (1 << 20) + 1, 1, 1, 1, 1, 1, 1, None) == -4


def test_context_rejects_capacities_out_of_range():
    """Event-local hit ids take 21 bits in the device's hit records, so hits_per_event above
    2^21 is refused before any device work, as are non-positive per-event capacities."""
    L = _native.lib()
    h = ctypes.c_void_p()
    for field, bad in (("hits_per_event", (1 << 21) + 1), ("hits_per_event", 0), ("doublets_per_event", 0),
                       ("tuples_per_event", -1), ("fits_per_multiplicity", 0), ("columns_per_event", 0)):
        p = _native.PxlParams()
        assert L.pxl_params_extended(ctypes.byref(p)) == 0
        setattr(p, field, bad)
        assert L.pxl_ctx_create(ctypes.byref(_native.PxlConditions()), ctypes.byref(p), ctypes.byref(h)) == -1, field


def test_input_slot_entry_points_reject_bad_arguments():
    L = _native.lib()
    assert L.pxl_slot_stage(None, 0, 1, 1, 1, None) == -1
    assert L.pxl_slot_launch(None, 0, None) == -1
