"""CPU-only checks of the native boundary: the C ABI library loads, exports
every entry point include/fcb200.h declares, rejects bad arguments with the
reference's status codes before touching a device, and the drop-in pybind11
modules import with the reference's names and dtype gates."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT, PKG

HEADER = ROOT / "include" / "fcb200.h"


@pytest.fixture(scope="module")
def native():
    import fcb_build
    fcb_build.build()
    from fcb200 import _native
    return _native


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fcb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("fcb_cs_rank_f32", "fcb_parameter_scan_f32", "fcb_rolling_ic", "fcb_factor_corr",
              "fcb_stock_corr", "fcb_rank_ic_panel", "fcb_workspace_create"):
        assert s in syms


def test_library_exports_every_declared_symbol(native):
    lib = native.lib()
    for s in declared_symbols():
        assert hasattr(lib, s), f"{s} declared in include/fcb200.h but not exported"
    # and the ctypes prototype table covers the header
    assert set(declared_symbols()) <= set(native.PROTOTYPES)


def test_contract_errors_without_device(native):
    lib = native.lib()
    out = np.zeros(4, np.float32)
    x = np.zeros(4, np.float32)
    P = native.ptr
    assert lib.fcb_cs_rank_f32(None, None, 2, 2, 0, P(out), None) == -1
    assert lib.fcb_cs_rank_f32(P(x), None, 0, 2, 0, P(out), None) == -1
    assert lib.fcb_cs_rank_f32(P(x), None, 1, (1 << 24) + 1, 0, P(out), None) == -2
    assert lib.fcb_cs_rank_f32(P(x), None, 1 << 16, 1 << 16, 0, P(out), None) == -3
    ic = np.zeros(2)
    assert lib.fcb_rolling_ic(P(x), 0, P(x), 0, None, None, 2, 2, 1, P(ic), None, None, None) == -4
    assert lib.fcb_rolling_ic(P(x), 0, P(x), 0, None, None, 1 << 16, 1 << 16, 30, P(ic), None, None, None) == -3
    o = np.zeros(4)
    assert lib.fcb_factor_corr(P(x), 0, None, 1, 1, 129, P(o), None) == -3
    assert lib.fcb_factor_corr(P(x), 0, None, 1 << 16, 1 << 16, 2, P(o), None) == -2
    assert lib.fcb_dev_factor_corr(P(x), 0, None, 1, 1, 129, 0, P(o), None, None) == -3
    # the BF16x3 precision form: same caps, F <= 16 on the tensor-core path
    assert lib.fcb_factor_corr_bf16x3(None, None, 2, 2, 2, P(o), None) == -1
    assert lib.fcb_factor_corr_bf16x3(P(x), None, 1, 1, 129, P(o), None) == -3
    assert lib.fcb_factor_corr_bf16x3(P(x), None, 1 << 16, 1 << 16, 2, P(o), None) == -2
    assert lib.fcb_factor_corr_bf16x3(P(x), None, 1, 1, 17, P(o), None) == -5   # F > 16: unsupported
    assert lib.fcb_dev_factor_corr_bf16x3(P(x), None, 1, 1, 2, 2, P(o), None, None) == -1   # planes 0/1
    assert lib.fcb_dev_factor_corr_bf16x3(P(x), None, 1, 1, 2, 1, P(o), None, None) == -1   # workspace required
    assert lib.fcb_dev_factor_corr(P(x), 0, None, 2, 2, 2, 0, P(o), None, None) == -1   # workspace required
    assert lib.fcb_dev_factor_corr(P(x), 0, None, 2, 2, 2, 2, P(o), None, None) == -1   # layout flag
    assert lib.fcb_stock_corr(P(x), 0, None, 1, 46341, P(o), None, None) == -3
    assert lib.fcb_stock_corr(None, 0, None, 1, 2, P(o), None, None) == -1
    st = (C.c_int * 4)()
    outs = (C.c_void_p * 4)(P(out), P(out), P(out), P(out))
    assert lib.fcb_parameter_scan_f32(P(x), None, 1, (1 << 24) + 1, outs, st, None, None, None, None) == -2
    assert list(st) == [-100] * 4
    assert lib.fcb_status_string(-4).decode()


def test_device_entry_contract_errors_without_device(native):
    """The fcb_dev_* variants of the fc.* calls reject bad arguments with the
    host entry points' codes before they touch a device."""
    lib = native.lib()
    P = native.ptr
    x = np.zeros(4, np.float32)
    o = np.zeros(4)
    st = (C.c_int * 4)()
    outs = (C.c_void_p * 4)(P(x), P(x), P(x), P(x))
    assert lib.fcb_dev_parameter_scan_f32(P(x), None, 1, (1 << 24) + 1, outs, st, None, None) == -2
    assert list(st) == [-100] * 4
    assert lib.fcb_dev_parameter_scan_f32(P(x), None, 1 << 16, 1 << 16, outs, st, None, None) == -3
    assert lib.fcb_dev_parameter_scan_f32(None, None, 2, 2, outs, st, None, None) == -1
    nulls = (C.c_void_p * 4)(P(x), None, P(x), P(x))
    assert lib.fcb_dev_parameter_scan_f32(P(x), None, 2, 2, nulls, st, None, None) == -1   # active group, no output
    only0 = (C.c_int * 4)(1, 0, 0, 0)
    assert lib.fcb_dev_parameter_scan_f32(P(x), None, 1, (1 << 24) + 1, nulls, st, only0, None) == -2
    assert lib.fcb_dev_rolling_ic(P(x), 0, P(x), 0, None, None, 2, 2, 1, P(o), None, None, None) == -4
    assert lib.fcb_dev_rolling_ic(P(x), 0, P(x), 0, None, None, 1 << 16, 1 << 16, 30, P(o), None, None, None) == -3
    assert lib.fcb_dev_rolling_ic(P(x), 2, P(x), 0, None, None, 2, 2, 30, P(o), None, None, None) == -1
    assert lib.fcb_dev_rolling_ic(P(x), 0, P(x), 0, None, None, 2, 2, 30, P(o), P(o), None, None) == -1
    assert lib.fcb_dev_stock_corr(P(x), 0, None, 1, 46341, P(o), None, None, None, None) == -3
    assert lib.fcb_dev_stock_corr(P(x), 0, None, 1 << 16, 1 << 16, P(o), None, None, None, None) == -2
    assert lib.fcb_dev_stock_corr(P(x), 0, None, 2, 2, P(o), None, None, None, None) == -1  # workspace required
    assert lib.fcb_selftest_bounded_wait(0, 0) == -1   # poll limit must be positive
    ok = C.c_int(7)
    assert lib.fcb_dev_corr_domain(P(x), 0, None, 2, 2, 2, 2, C.byref(ok), None) == -1      # layout flag
    assert lib.fcb_dev_corr_domain(P(x), 3, None, 2, 2, 2, 0, C.byref(ok), None) == -1      # dtype
    assert lib.fcb_dev_corr_domain(P(x), 1, None, 1 << 16, 1 << 16, 2, 0, C.byref(ok), None) == -2
    assert lib.fcb_dev_corr_domain(P(x), 1, None, 2, 2, 2, 0, None, None) == -1
    assert ok.value == 7


def test_batch_contract_errors_without_device(native):
    """fcb_batch_create rejects bad panels with the single-panel codes before
    it touches a device; the default configuration is the documented one."""
    lib = native.lib()
    cfg = native.FcbBatchConfig()
    lib.fcb_batch_default_config(C.byref(cfg))
    assert cfg.as_dict() == {"nt_small_max": 4096, "nt_mid_max": 8192, "ctas_per_sm": 0, "concurrent": 0,
                             "order": 1, "learn_cap": 256}
    h = C.c_void_p()
    arr = (native.FcbPanel * 2)()
    arr[0] = native.FcbPanel(10, 500, 2, 16, 16, None, None, None, 16, None, None)
    arr[1] = native.FcbPanel(10, 500, 2, 16, 16, None, None, None, 16, None, None)
    assert lib.fcb_batch_create(None, 0, 0, 0, 30, None, C.byref(h)) == -1
    assert lib.fcb_batch_create(arr, 2, 0, 0, 30, None, None) == -1
    assert lib.fcb_batch_create(arr, 2, 0, 0, 1, None, C.byref(h)) == -4          # min_valid < 2
    assert lib.fcb_batch_create(arr, 2, 0, 1, 30, None, C.byref(h)) == -5         # mixed dtypes
    arr[1].N = 20000
    assert lib.fcb_batch_create(arr, 2, 0, 0, 30, None, C.byref(h)) == -5         # N above the SMEM cap
    arr[1].N = 500
    arr[1].ic_out = None
    assert lib.fcb_batch_create(arr, 2, 0, 0, 30, None, C.byref(h)) == -1
    arr[1].ic_out = 16
    arr[1].F, arr[1].corr_out = 129, 16
    assert lib.fcb_batch_create(arr, 2, 0, 0, 30, None, C.byref(h)) == -3         # factor_corr F cap
    arr[1].F, arr[1].corr_out = 2, None
    bad = native.FcbBatchConfig()
    lib.fcb_batch_default_config(C.byref(bad))
    bad.nt_mid_max = 100                                                           # below nt_small_max
    assert lib.fcb_batch_create(arr, 2, 0, 0, 30, C.byref(bad), C.byref(h)) == -1
    assert not h.value


def test_workspace_lifecycle_without_device(native):
    lib = native.lib()
    ws = lib.fcb_workspace_create()
    assert ws
    live, peak, n = C.c_uint64(), C.c_uint64(), C.c_uint64()
    assert lib.fcb_workspace_stats(ws, C.byref(live), C.byref(peak), C.byref(n)) == 0
    assert live.value == 0 and peak.value == 0
    lib.fcb_workspace_clear(ws)
    lib.fcb_workspace_destroy(ws)


def test_dropin_modules_import_and_gate_dtypes(native):
    fcb = native.fcb()
    fcp = native.fcp()
    for name in ("cs_rank_f32", "rolling_ic_f64", "stock_corr_f64", "parameter_scan_f32",
                 "CsRankWorkspace", "RollingIcWorkspace"):
        assert hasattr(fcb, name)
    assert hasattr(fcp, "factor_corr_f64")
    x64 = np.zeros((2, 3))
    with pytest.raises(TypeError):
        fcb.cs_rank_f32(x64)          # strict f32 (src/factor_cuda_pybind.cpp:67-74)
    with pytest.raises(TypeError):
        fcb.cs_rank_f32([[1.0]])      # non-ndarray
    x32 = np.zeros((2, 3), np.float32)
    with pytest.raises(ValueError):
        fcb.cs_rank_f32(x32, np.zeros((2, 3)))          # float mask
    with pytest.raises(ValueError):
        fcb.cs_rank_f32(x32, np.zeros((3, 3), bool))    # mask shape
    with pytest.raises(ValueError):
        fcb.rolling_ic_f64(x32, x32, None, None, 30.5)  # min_valid not an int
    with pytest.raises(ValueError):
        fcb.rolling_ic_f64(x32, x32, None, None, 1)     # min_valid < 2
    with pytest.raises(TypeError):
        fcb.rolling_ic_f64(x32.astype(np.int32), x32)
    with pytest.raises(ValueError):
        fcb.parameter_scan_f32(x32, None)               # masked groups need a mask
    with pytest.raises(ValueError):
        fcb.parameter_scan_f32(x32, np.ones((2, 3), bool), active_groups=[1, 1])
    with pytest.raises(ValueError):
        fcp.factor_corr_f64(np.zeros((2, 2, 129)))      # F > 128
    ws = fcb.CsRankWorkspace()
    ws.clear()
    ws.clear()
    fcb.RollingIcWorkspace().clear()
    # each function takes only the workspace class it is bound to
    # (src/factor_cuda_pybind.cpp:135,179,293 bind the typed handles)
    with pytest.raises(TypeError):
        fcb.cs_rank_f32(x32, None, False, fcb.RollingIcWorkspace())
    with pytest.raises(TypeError):
        fcb.parameter_scan_f32(x32, np.ones((2, 3), bool), workspace=fcb.RollingIcWorkspace())
    with pytest.raises(TypeError):
        fcb.rolling_ic_f64(x32, x32, None, None, 30, workspace=ws)
    with pytest.raises(TypeError):
        fcb.cs_rank_f32(x32, None, False, object())


def test_package_layout():
    assert (PKG / "csrc").is_dir()
    assert (PKG / "fcb200" / "__init__.py").exists()
    for bad in ("models", "ops", "parallel"):
        assert not (PKG / bad).exists()
