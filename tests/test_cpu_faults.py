"""Failure injection on the host, no GPU needed: the library's device
allocations can be made to fail (ds_debug_fail_allocations_after), and every
create call must then return DS_ERR_OOM with no handle, before any device
work.  The GPU tests drive the same hook through every allocation of each
create call (tests/test_gpu_edge.py)."""
import ctypes as C

import pytest

from diffsplat_b200 import _lib as L


@pytest.fixture
def no_allocations():
    L.lib().ds_debug_fail_allocations_after(0)
    yield
    L.lib().ds_debug_fail_allocations_after(-1)


def test_fitter_create_reports_oom(no_allocations):
    cfg = L.FitterConfig()
    assert L.lib().ds_fitter_default_config(C.byref(cfg)) == L.DS_OK
    cfg.width, cfg.height, cfg.count = 64, 48, 100
    h = C.c_void_p(1)
    assert L.lib().ds_fitter_create(C.byref(cfg), C.byref(h)) == L.DS_ERR_OOM
    assert h.value is None


def test_raster_and_renderer_create_report_oom(no_allocations):
    h = C.c_void_p(1)
    assert L.lib().ds_raster_create(64, 48, 100, 1 << 12, C.byref(h)) == L.DS_ERR_OOM
    assert h.value is None
    h = C.c_void_p(1)
    assert L.lib().ds_renderer_create(64, 48, 100, 0, 1 << 12, L.DS_STORAGE_FP32,
                                      C.byref(h)) == L.DS_ERR_OOM
    assert h.value is None


def test_batch_create_reports_oom(no_allocations):
    cfg = L.BatchConfig()
    assert L.lib().ds_batch_default_config(C.byref(cfg)) == L.DS_OK
    cfg.instances = 2
    inst = (L.BatchInstance * 2)(L.BatchInstance(32, 32, 50, 0), L.BatchInstance(48, 16, 70, 0))
    h = C.c_void_p(1)
    assert L.lib().ds_batch_create(C.byref(cfg), inst, C.byref(h)) == L.DS_ERR_OOM
    assert h.value is None


def test_hook_off_by_default_and_resettable():
    assert L.lib().ds_debug_fail_allocations_after(-1) == L.DS_OK
    assert L.lib().ds_debug_fail_allocations_after(-5) == L.DS_OK
