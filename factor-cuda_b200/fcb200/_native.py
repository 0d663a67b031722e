"""Loader for the native library and the drop-in binding modules.

``lib()`` returns the ctypes handle of ``build/libfcb200.so`` with every C ABI
prototype declared (include/fcb200.h).  ``fcb()`` / ``fcp()`` import the
drop-in pybind11 modules ``factor_cuda_pybind`` / ``factor_corr_pybind`` from
the same build directory (the reference adapter's ``fc/_util.py:200-219``
loads modules of these names from its own ``build/``).

There is no fallback: a missing build raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import functools
import importlib
import pathlib
import sys

PKG = pathlib.Path(__file__).resolve().parent.parent
BUILD = PKG / "build"
LIB = BUILD / "libfcb200.so"

FCB_DTYPE_F32 = 0
FCB_DTYPE_F64 = 1
FCB_GROUP_NOT_EXECUTED = -100
FCB_ERR_DEVICE_WAIT = 100000

_p = C.c_void_p
_i = C.c_int
_d = C.POINTER(C.c_double)



class FcbPanel(C.Structure):
    """struct fcb_panel (include/fcb200.h)."""
    _fields_ = [("T", C.c_int), ("N", C.c_int), ("F", C.c_int), ("X", _p), ("R", _p), ("fmask", _p),
                ("rmask", _p), ("ranks_out", _p), ("ic_out", _p), ("corr_out", _p), ("model", _p)]


class FcbBatchConfig(C.Structure):
    """struct fcb_batch_config (include/fcb200.h)."""
    _fields_ = [("nt_small_max", C.c_int), ("nt_mid_max", C.c_int), ("ctas_per_sm", C.c_int),
                ("concurrent", C.c_int), ("order", C.c_int), ("learn_cap", C.c_int)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_cfgp = C.POINTER(FcbBatchConfig)

# name -> (restype, argtypes); the symbol table of include/fcb200.h
PROTOTYPES = {
    "fcb_workspace_create": (_p, []),
    "fcb_workspace_clear": (None, [_p]),
    "fcb_workspace_destroy": (None, [_p]),
    "fcb_workspace_stats": (_i, [_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "fcb_memory_budget": (_i, [_i, _i, _i, _i, _i, _i, C.POINTER(C.c_uint64)]),
    "fcb_workspace_learned_state": (_i, [_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "fcb_version": (_i, []),
    "fcb_device_count": (_i, []),
    "fcb_status_string": (C.c_char_p, [_i]),
    "fcb_host_alloc": (_p, [C.c_size_t]),
    "fcb_host_free": (None, [_p]),
    "fcb_cs_rank_f32": (_i, [_p, _p, _i, _i, _i, _p, _p]),
    "fcb_parameter_scan_f32": (_i, [_p, _p, _i, _i, C.POINTER(_p), C.POINTER(_i), _d, C.POINTER(C.c_float),
                                    C.POINTER(_i), _p]),
    "fcb_rolling_ic": (_i, [_p, _i, _p, _i, _p, _p, _i, _i, _i, _p, _p, _p, _p]),
    "fcb_factor_corr": (_i, [_p, _i, _p, _i, _i, _i, _p, _p]),
    "fcb_dev_factor_corr": (_i, [_p, _i, _p, _i, _i, _i, _i, _p, _p, _p]),
    "fcb_stock_corr": (_i, [_p, _i, _p, _i, _i, _p, C.POINTER(_i), C.POINTER(_i)]),
    "fcb_rank_ic_panel": (_i, [_p, _p, _p, _p, _i, _i, _i, _i, _p, _p, _i, _p]),
    "fcb_dev_rank_ic_panel": (_i, [_p, _p, _p, _p, _i, _i, _i, _i, _p, _p, _i, _p]),
    "fcb_dev_status": (_i, []),
    "fcb_selftest_bounded_wait": (_i, [_i, _i]),
    "fcb_dev_cs_rank_f32": (_i, [_p, _p, _i, _i, _i, _p, _p]),
    "fcb_dev_parameter_scan_f32": (_i, [_p, _p, _i, _i, C.POINTER(_p), C.POINTER(_i), C.POINTER(_i), _p]),
    "fcb_dev_rolling_ic": (_i, [_p, _i, _p, _i, _p, _p, _i, _i, _i, _p, _p, _p, _p]),
    "fcb_dev_stock_corr": (_i, [_p, _i, _p, _i, _i, _p, C.POINTER(_i), C.POINTER(_i), _p, _p]),
    "fcb_dev_corr_domain": (_i, [_p, _i, _p, _i, _i, _i, _i, C.POINTER(_i), _p]),
    "fcb_dev_factor_corr_noalloc": (_i, [_p, _i, _p, _i, _i, _i, _p, _p]),
    "fcb_stock_corr_prec": (_i, [_p, _p, _i, _i, _i, _p, _p]),
    "fcb_dev_stock_corr_prec": (_i, [_p, _p, _i, _i, _i, _p, _p, _p]),
    "fcb_factor_corr_bf16x3": (_i, [_p, _p, _i, _i, _i, _p, _p]),
    "fcb_dev_factor_corr_bf16x3": (_i, [_p, _p, _i, _i, _i, _i, _p, _p, _p]),
    "fcb_cdf_model_create": (_p, [_i, C.c_uint64]),
    "fcb_cdf_model_destroy": (None, [_p]),
    "fcb_cdf_model_set_linear": (_i, [_p, _i]),
    "fcb_cdf_model_fit": (_i, [_p, _p, _p, _i, _i, _i, _i, _i, C.c_float, _p]),
    "fcb_cdf_model_sample": (_i, [_p, _p, _p, _i, _i, _i, _i, _p]),
    "fcb_cdf_model_train": (_i, [_p, _i, C.c_float, _i, _p]),
    "fcb_cdf_model_swap": (_i, [_p]),
    "fcb_cdf_model_state": (_i, [_p, _p, _p, _p, _p]),
    "fcb_cdf_model_load": (_i, [_p, _p, _p, _p]),
    "fcb_cdf_grad": (_i, [_p, _p, _p, _i, _p, _p]),
    "fcb_dev_rank_ic_panel_learned": (_i, [_p, _p, _p, _p, _i, _i, _i, _i, _p, _p, _p, _i, _p, _p]),
    "fcb_batch_default_config": (None, [_cfgp]),
    "fcb_batch_create": (_i, [C.POINTER(FcbPanel), _i, _i, _i, _i, _cfgp, C.POINTER(_p)]),
    "fcb_batch_destroy": (None, [_p]),
    "fcb_batch_get_config": (_i, [_p, _cfgp]),
    "fcb_batch_set_config": (_i, [_p, _cfgp]),
    "fcb_batch_run": (_i, [_p, _p]),
    "fcb_batch_run_per_panel": (_i, [_p, _p]),
    "fcb_batch_status": (_i, [_p]),
    "fcb_batch_autotune": (_i, [_p, _i, C.c_char_p, _cfgp, C.POINTER(C.c_float)]),
}


@functools.lru_cache(maxsize=1)
def lib():
    if not LIB.exists():
        raise RuntimeError(f"libfcb200.so not built ({LIB}); run python factor-cuda_b200/fcb_build.py")
    h = C.CDLL(str(LIB))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(h, name)
        fn.restype = res
        fn.argtypes = args
    return h


def _load_module(name: str):
    b = str(BUILD)
    if b not in sys.path:
        sys.path.insert(0, b)
    try:
        return importlib.import_module(name)
    except ImportError as e:
        raise RuntimeError(f"binding {name} not found in {BUILD}; run python factor-cuda_b200/fcb_build.py") from e


@functools.lru_cache(maxsize=1)
def fcb():
    return _load_module("factor_cuda_pybind")


@functools.lru_cache(maxsize=1)
def fcp():
    return _load_module("factor_corr_pybind")


def device_count() -> int:
    return int(lib().fcb_device_count())


def status_string(rc: int) -> str:
    return lib().fcb_status_string(int(rc)).decode()


def check(rc: int, what: str) -> None:
    """Map a C ABI status to the reference's exception classes."""
    if rc == 0:
        return
    if rc < 0:
        raise ValueError(f"{what}: contract error {rc} ({status_string(rc)})")
    raise RuntimeError(f"{what}: error {rc} ({status_string(rc)})")


def ptr(a) -> int | None:
    """Raw data pointer of a numpy array or a torch tensor (None passes through)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    return int(a.ctypes.data)
