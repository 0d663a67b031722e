"""fcb200 -- B200-native cross-sectional analysis path with factor-cuda's ``fc.*`` API.

Public functions mirror the reference adapter (``fc/__init__.py:5-29``):
``cross_sectional_rank``, ``factor_plane``, ``parameter_scan``, ``rolling_ic``,
``factor_corr``, ``stock_corr`` and ``clear_workspaces``, with the same
argument names, validation (dtype whitelist, strict-bool masks, f64->f32
downcast for the rank ops, ``min_valid`` int >= 2), error classes and output
containers (numpy in -> numpy out, torch in -> torch out on the input device).

Every compute call goes to the CUDA path through the drop-in pybind11 modules
``factor_cuda_pybind`` / ``factor_corr_pybind`` over ``libfcb200.so``.  There is
no CPU backend: ``backend='cpu'`` / ``device='cpu'`` raise, and a missing GPU or
build raises ``RuntimeError``.  (The reference's own adapter keeps its CPU
oracle; use it unchanged with these modules for a CPU fallback.)

Extensions beyond the reference API: ``rank_ic_panel`` (F factors against one
forward-return panel in one call), ``workspace_stats``.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from contextlib import contextmanager

import numpy as np

from . import _native as nat

try:  # optional, only to accept / return torch tensors
    import torch as _torch
except Exception:  # pragma: no cover
    _torch = None

__version__ = "1.0.0"
__all__ = ["cross_sectional_rank", "factor_plane", "factor_corr", "stock_corr", "rolling_ic",
           "parameter_scan", "rank_ic_panel", "Workspace", "CdfModel", "Batch", "clear_workspaces",
           "check_device", "__version__"]

_WHITELIST = (np.float32, np.float64)
DOMAIN_MSG = ("correlation domain violation: max|x| > 1e150 or a nonzero |x| < 1e-150 "
              "on a valid cell")


# ---------------------------------------------------------------------------
# container / validation helpers (reference fc/_util.py:79-197)
# ---------------------------------------------------------------------------
def _dtype_ok(dt, dtypes):
    if _torch is not None and isinstance(dt, _torch.dtype):
        allowed = {"f32": (_torch.float32,), "f64": (_torch.float64,)}.get(
            dtypes, (_torch.float32, _torch.float64))
        return dt in allowed
    allowed = {"f32": (np.float32,), "f64": (np.float64,)}.get(dtypes, _WHITELIST)
    return dt in allowed


def _dtype_error(name, dt):
    return ValueError(f"{name}: dtype {dt} is not accepted (float32 or float64 only)")


def _to_numpy(x, *, name, ndim, dtypes="f32f64", downcast_to=None):
    """Host copy of a numpy array, torch tensor or DLPack capsule, with the
    container kind and device it came from.  The input rules are the fc
    adapter's (fc/_util.py:79-136): float32/float64 only (ValueError), a
    DLPack capsule is single-use (ValueError on re-use), anything else is a
    TypeError; f64 is rounded to f32 (nearest-even) when downcast_to asks."""
    kind, device = "numpy", "cpu"
    if isinstance(x, np.ndarray):
        if not _dtype_ok(x.dtype, dtypes):
            raise _dtype_error(name, x.dtype)
        arr = np.ascontiguousarray(x)
    elif _torch is not None and isinstance(x, _torch.Tensor):
        kind = "torch"
        device = "cpu" if not x.is_cuda else f"cuda:{x.device.index}"
        x = x.detach()
        if not _dtype_ok(x.dtype, dtypes):
            raise _dtype_error(name, x.dtype)
        arr = x.contiguous().cpu().numpy()
    else:
        if _torch is None:
            raise TypeError(f"{name}: pass a numpy array or a torch tensor")
        try:
            t = _torch.utils.dlpack.from_dlpack(x)
        except (RuntimeError, TypeError, AttributeError):
            if type(x).__name__ == "PyCapsule":
                raise ValueError(f"{name}: this DLPack capsule was consumed by an earlier call") from None
            raise TypeError(f"{name}: pass a numpy array, a torch tensor or a DLPack capsule") from None
        kind = "dlpack"
        device = "cpu" if not t.is_cuda else f"cuda:{t.device.index}"
        if not _dtype_ok(t.dtype, dtypes):
            raise _dtype_error(name, t.dtype)
        arr = t.detach().contiguous().cpu().numpy()
    ok = arr.ndim == ndim if isinstance(ndim, int) else arr.ndim in ndim
    if not ok:
        raise ValueError(f"{name}: expected a {ndim}-D array, got {arr.ndim}-D")
    if downcast_to == "float32" and arr.dtype == np.float64:
        arr = arr.astype(np.float32)  # IEEE round-to-nearest-even
    return kind, device, np.ascontiguousarray(arr)


def _check_mask(mask, *, name, T, N, allow_none=True):
    """A (T,N) boolean mask as a host array (None passes through when
    allowed).  Masks are strictly bool (the mask alone decides validity)."""
    if mask is None:
        if allow_none:
            return None
        raise ValueError(f"{name}: a mask is needed here")
    if isinstance(mask, np.ndarray):
        if mask.dtype != np.bool_:
            raise ValueError(f"{name}: masks are bool arrays, this one is {mask.dtype}")
        arr = np.ascontiguousarray(mask)
    elif _torch is not None and isinstance(mask, _torch.Tensor):
        if mask.dtype != _torch.bool:
            raise ValueError(f"{name}: masks are bool tensors, this one is {mask.dtype}")
        arr = mask.detach().cpu().numpy()
    else:
        raise TypeError(f"{name}: pass a bool numpy array or torch tensor")
    if arr.shape != (T, N):
        raise ValueError(f"{name}: shape {arr.shape} does not match the input's (T,N) = {(T, N)}")
    return arr


def _mask_device(mask, device, name):
    if mask is None:
        return
    md = "cpu"
    if _torch is not None and isinstance(mask, _torch.Tensor) and mask.is_cuda:
        md = f"cuda:{mask.device.index}"
    if md != device:
        raise ValueError(f"{name} must be on the same device as values ({device}), got {md}")


def _require_cuda(context):
    if nat.device_count() < 1:
        raise RuntimeError(f"CUDA unavailable: {context} runs on the GPU only in fcb200")


def _sync_entry(device):
    if _torch is not None and device.startswith("cuda") and _torch.cuda.is_available():
        _torch.cuda.current_stream(int(device.split(":")[1])).synchronize()


def _make_output(res, kind, device):
    if kind == "numpy":
        return res
    return _torch.as_tensor(res, device=_torch.device(device if device != "cpu" else "cpu"))


def _domain_check(arr, mask):
    """max|x| <= 1e150 and min nonzero |x| >= 1e-150 over valid cells; f32
    panels always satisfy it (fc/correlation.py:16-49)."""
    if arr.dtype == np.float32:
        return
    if arr.ndim == 3:
        T, N, F = arr.shape
        flat = arr.reshape(T * N, F)
        valid = np.isfinite(flat)
        if mask is not None:
            valid &= mask.reshape(T * N, 1)
    else:
        flat = arr
        valid = np.isfinite(flat)
        if mask is not None:
            valid &= mask
    xv = np.abs(flat[valid])
    if xv.size == 0:
        return
    if xv.max() > 1e150:
        raise ValueError(DOMAIN_MSG)
    nz = xv[xv != 0.0]
    if nz.size and nz.min() < 1e-150:
        raise ValueError(DOMAIN_MSG)


# ---------------------------------------------------------------------------
# CUDA-resident inputs: the device entry points of libfcb200 take the tensor's
# memory directly, so a torch CUDA tensor is never copied to the host and back
# (the reference adapter does that round trip, fc/_util.py:121-131).
# ---------------------------------------------------------------------------
def _is_cuda(x):
    return _torch is not None and isinstance(x, _torch.Tensor) and x.is_cuda


def _dev_input(x, *, name, ndim, dtypes="f32f64", downcast_to=None):
    x = x.detach()
    if not _dtype_ok(x.dtype, dtypes):
        raise ValueError(f"{name} dtype {x.dtype} not in whitelist {{float32,float64}}")
    ok = x.dim() == ndim if isinstance(ndim, int) else x.dim() in ndim
    if not ok:
        raise ValueError(f"{name} must be {ndim}-D, got ndim={x.dim()}")
    if downcast_to == "float32" and x.dtype == _torch.float64:
        x = x.to(_torch.float32)  # IEEE round-to-nearest-even, as the host path's astype
    return f"cuda:{x.device.index}", x.contiguous()


def _dev_mask(mask, *, name, T, N, device, allow_none=True):
    """Strict-bool (T,N) mask as a uint8 view on `device` (None passes through)."""
    if mask is None:
        if allow_none:
            return None
        raise ValueError(f"{name} is required")
    if isinstance(mask, np.ndarray):
        if mask.dtype != np.bool_:
            raise ValueError(f"{name} must be bool, got {mask.dtype}")
        mask = _torch.from_numpy(np.ascontiguousarray(mask))
    elif isinstance(mask, _torch.Tensor):
        if mask.dtype != _torch.bool:
            raise ValueError(f"{name} must be bool, got {mask.dtype}")
    else:
        raise TypeError(f"{name} must be a bool numpy array or torch.Tensor")
    if tuple(mask.shape) != (T, N):
        raise ValueError(f"{name} shape must be (T,N) matching input, got {tuple(mask.shape)}")
    return mask.detach().to(device).contiguous().view(_torch.uint8)


def check_device():
    """Synchronise the current CUDA device and raise ``RuntimeError`` if a
    bounded device-side wait in an asynchronous call (the CUDA-tensor route)
    gave up since the last check; the condition is cleared by the check."""
    nat.check(nat.lib().fcb_dev_status(), "device status")


def _stream_of(t):
    return _torch.cuda.current_stream(t.device).cuda_stream


_DT = {"torch.float32": nat.FCB_DTYPE_F32, "torch.float64": nat.FCB_DTYPE_F64}


def _dtype_code(t):
    return _DT[str(t.dtype)]


# ---------------------------------------------------------------------------
# per-shape workspace cache (reference fc/_workspace.py:42-133)
# ---------------------------------------------------------------------------
class _WorkspaceCache:
    _all: list = []

    def __init__(self, factory):
        self._factory = factory
        self._items = {}
        self._guard = threading.Lock()
        _WorkspaceCache._all.append(self)

    @contextmanager
    def use(self, key):
        with self._guard:
            item = self._items.get(key)
            if item is None:
                item = (self._factory(), threading.Lock())
                self._items[key] = item
            ws, lock = item
            lock.acquire()
        try:
            yield ws
        finally:
            lock.release()

    def clear(self):
        with self._guard:
            items = list(self._items.values())
            self._items = {}
        for ws, lock in items:
            with lock:
                ws.clear()


_RANK_CACHE = _WorkspaceCache(lambda: nat.fcb().CsRankWorkspace())
_SCAN_CACHE = _WorkspaceCache(lambda: nat.fcb().CsRankWorkspace())
_ROLL_CACHE = _WorkspaceCache(lambda: nat.fcb().RollingIcWorkspace())
_DEV_CACHE = _WorkspaceCache(lambda: Workspace())  # keyed by device index


def clear_workspaces():
    """Release every cached device workspace (idempotent)."""
    for c in _WorkspaceCache._all:
        c.clear()


# ---------------------------------------------------------------------------
# operators
# ---------------------------------------------------------------------------
def cross_sectional_rank(values, mask=None, descending=False):
    """Stable ordinal rank 1..K per date; invalid cells NaN (0x7fc00000).
    Reference: fc/cross_sectional_rank.py:19-35."""
    if type(descending) is not bool:
        raise ValueError("descending must be a bool (type(x) is bool), got "
                         f"{type(descending).__name__}")
    if _is_cuda(values):
        device, x = _dev_input(values, name="values", ndim=2, downcast_to="float32")
        T, N = x.shape
        _require_cuda("cross_sectional_rank")
        _mask_device(mask, device, "mask")
        m = _dev_mask(mask, name="mask", T=T, N=N, device=x.device)
        out = _torch.empty((T, N), dtype=_torch.float32, device=x.device)
        with _torch.cuda.device(x.device):
            nat.check(nat.lib().fcb_dev_cs_rank_f32(nat.ptr(x), nat.ptr(m), T, N, int(descending), nat.ptr(out),
                                                    _stream_of(x)), "cross_sectional_rank")
        return out
    kind, device, x = _to_numpy(values, name="values", ndim=2, downcast_to="float32")
    T, N = x.shape
    _require_cuda("cross_sectional_rank")
    _mask_device(mask, device, "mask")
    m = _check_mask(mask, name="mask", T=T, N=N)
    _sync_entry(device)
    with _RANK_CACHE.use((T, N)) as ws:
        res = nat.fcb().cs_rank_f32(x, m, descending, workspace=ws)
    return _make_output(res, kind, device)


def factor_plane(factors, f):
    """Factor f of a (T,N,F) panel as a fresh (T,N) array
    (fc/cross_sectional_rank.py:38-54)."""
    if not isinstance(f, int) or isinstance(f, bool):
        raise ValueError(f"f must be an integer, got {type(f).__name__}")
    kind, device, arr = _to_numpy(factors, name="factors", ndim=(2, 3))
    if arr.ndim == 2:
        if f != 0:
            raise ValueError("ndim=2 input requires f == 0")
        plane = np.array(arr, copy=True)
    else:
        if not (0 <= f < arr.shape[2]):
            raise ValueError(f"f={f} out of range [0,F={arr.shape[2]})")
        plane = np.ascontiguousarray(arr[..., f])
    return _make_output(plane, kind, device)


# parameter_scan axes: the values each accepts and the one used when the
# caller leaves the axis out, in the canonical order of the effective spec
# (the rules of fc/parameter_scan.py:26-58).
_SCAN_AXES = {"direction": (("ascending", "descending"), "ascending"),
              "mask_mode": (("masked", "unmasked"), "masked")}
# position of each (direction, mask_mode) group in the binding's four outputs
_BINDING_INDEX = {("ascending", "masked"): 0, ("ascending", "unmasked"): 1,
                  ("descending", "masked"): 2, ("descending", "unmasked"): 3}


def _normalize_axes(axes):
    """Validate a parameter_scan axis list and expand it into the effective
    spec (every axis, canonical order, defaults filled in) and the groups
    (direction-major product of the values).  Any malformed, unknown,
    repeated or empty axis, or an unknown or repeated value, is a ValueError."""
    pairs = list(axes) if isinstance(axes, (list, tuple)) else None
    if pairs is None or any(not isinstance(p, (list, tuple)) or len(p) != 2 for p in pairs):
        raise ValueError("parameter_scan: axes must be a sequence of (name, values) pairs")
    given = {}
    for name, vals in pairs:
        if name not in _SCAN_AXES:
            raise ValueError(f"parameter_scan: {name!r} is not a scan axis (known: {', '.join(_SCAN_AXES)})")
        if name in given:
            raise ValueError(f"parameter_scan: axis {name!r} is given more than once")
        if not isinstance(vals, (list, tuple)) or len(vals) == 0:
            raise ValueError(f"parameter_scan: axis {name!r} needs at least one value")
        if len(set(vals)) < len(vals):
            raise ValueError(f"parameter_scan: axis {name!r} repeats a value in {list(vals)}")
        allowed = _SCAN_AXES[name][0]
        unknown = [v for v in vals if v not in allowed]
        if unknown:
            raise ValueError(f"parameter_scan: {unknown} not allowed for axis {name!r} (allowed: {allowed})")
        given[name] = list(vals)
    eff = {name: given.get(name, [default]) for name, (_, default) in _SCAN_AXES.items()}
    return eff, [(d, m) for d in eff["direction"] for m in eff["mask_mode"]]


def parameter_scan(axes, X, mask=None):
    """direction x mask_mode rank scan; results always host numpy
    (fc/parameter_scan.py:62-132).  The active groups come from one fused pass."""
    effective, combos = _normalize_axes(axes)
    if _is_cuda(X):
        return _parameter_scan_dev(effective, combos, X, mask)
    _, device, x = _to_numpy(X, name="X", ndim=2, downcast_to="float32")
    T, N = x.shape
    _require_cuda("parameter_scan")
    if N > (1 << 24):
        raise ValueError("N > 2^24 (rank precision cap)")
    any_masked = any(mm == "masked" for _, mm in combos)
    m = (_check_mask(mask, name="mask", T=T, N=N, allow_none=False) if any_masked
         else np.ones((T, N), dtype=np.bool_))
    active = [0, 0, 0, 0]
    for combo in combos:
        active[_BINDING_INDEX[combo]] = 1
    _sync_entry(device)
    t0 = time.perf_counter()
    with _SCAN_CACHE.use((T, N)) as ws:
        r = nat.fcb().parameter_scan_f32(x, m, return_timing=True, active_groups=active, workspace=ws)
    elapsed_ms = (time.perf_counter() - t0) * 1e3
    return _scan_result(effective, combos, r, elapsed_ms)


def _parameter_scan_dev(effective, combos, X, mask):
    """parameter_scan of a CUDA tensor through fcb_dev_parameter_scan_f32: the
    panel stays on the device; the group results come back as host numpy."""
    device, x = _dev_input(X, name="X", ndim=2, downcast_to="float32")
    T, N = x.shape
    _require_cuda("parameter_scan")
    if N > (1 << 24):
        raise ValueError("N > 2^24 (rank precision cap)")
    any_masked = any(mm == "masked" for _, mm in combos)
    m = _dev_mask(mask, name="mask", T=T, N=N, device=x.device, allow_none=False) if any_masked else None
    active = [0, 0, 0, 0]
    for combo in combos:
        active[_BINDING_INDEX[combo]] = 1
    nact = sum(active)
    outs = [_torch.empty((T, N), dtype=_torch.float32, device=x.device) if a else None for a in active]
    optrs = (C.c_void_p * 4)(*[nat.ptr(o) for o in outs])
    act = (C.c_int * 4)(*active)
    gst = (C.c_int * 4)()
    stream = _torch.cuda.current_stream(x.device)
    with _torch.cuda.device(x.device):
        e0 = _torch.cuda.Event(enable_timing=True)
        e1 = _torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        nat.check(nat.lib().fcb_dev_parameter_scan_f32(nat.ptr(x), nat.ptr(m), T, N, optrs, gst, act,
                                                       stream.cuda_stream), "parameter_scan")
        e1.record(stream)
        stream.synchronize()
        host_ms = (time.perf_counter() - t0) * 1e3
        gpu_ms = e0.elapsed_time(e1)
    st = [int(v) for v in gst]
    r = {"groups": [o.cpu().numpy() if (o is not None and st[g] == 0) else None for g, o in enumerate(outs)],
         "group_status": st,
         "time_ms": [host_ms / nact if st[g] == 0 else 0.0 for g in range(4)],
         "time_gpu_ms": [gpu_ms / nact if st[g] == 0 else 0.0 for g in range(4)]}
    return _scan_result(effective, combos, r, host_ms)


def _scan_result(effective, combos, r, elapsed_ms):
    """The parameter_scan record (schema of fc/parameter_scan.py:101-132) from
    the binding's four group outputs: one entry per requested group, in
    request order.  Status 0 is a finished group; 9 and 701 (launch
    failures the contract confines to one group) mark that group failed with
    zero time; any other status fails the whole scan with RuntimeError."""
    groups = []
    for gi, (d, mm) in enumerate(combos):
        g = _BINDING_INDEX[(d, mm)]
        st = r["group_status"][g]
        entry = {"group_index": gi, "axis_values": {"direction": d, "mask_mode": mm}}
        if st == 0:
            entry.update(result=r["groups"][g], status="ok", error=None, error_stage=None,
                         time_ms=r["time_ms"][g], time_gpu_ms=r["time_gpu_ms"][g])
        elif st in (9, 701):
            entry.update(result=None, status="failed", error=f"launch of this group failed: CUDA status {st}",
                         error_stage="launch", time_ms=0.0, time_gpu_ms=0.0)
        else:
            raise RuntimeError(f"parameter_scan: CUDA status {st} (group {g}) is not a per-group failure")
        groups.append(entry)
    done = [g for g in groups if g["status"] == "ok"]
    return {"spec": effective, "groups": groups,
            "summary": {"total_groups": len(combos),
                        "n_failed": len(groups) - len(done),
                        "total_time_ms": sum(g["time_ms"] for g in done),
                        "total_time_gpu_ms": sum(g["time_gpu_ms"] for g in done),
                        "elapsed_ms": elapsed_ms}}


def rolling_ic(factor, forward_returns, factor_mask=None, fwd_mask=None, min_valid=30, device=None):
    """Daily Spearman IC (T,) f64 (fc/rolling_ic.py:16-57); GPU only."""
    if device not in (None, "cpu", "cuda"):
        raise ValueError(f"device must be None, 'cpu', or 'cuda', got {device!r}")
    if not isinstance(min_valid, int) or isinstance(min_valid, bool):
        raise ValueError("min_valid must be an integer (bool rejected)")
    if min_valid < 2:
        raise ValueError("min_valid must be >= 2")
    if _is_cuda(factor) and _is_cuda(forward_returns) and factor.device == forward_returns.device:
        return _rolling_ic_dev(factor, forward_returns, factor_mask, fwd_mask, min_valid, device)
    kf, df, f = _to_numpy(factor, name="factor", ndim=2)
    kr, dr, r = _to_numpy(forward_returns, name="forward_returns", ndim=2)
    T, N = f.shape
    if r.shape != (T, N):
        raise ValueError(f"factor and forward_returns shapes must match (T,N), got {f.shape} vs {r.shape}")
    _mask_device(factor_mask, df, "factor_mask")
    _mask_device(fwd_mask, df, "fwd_mask")
    fm = _check_mask(factor_mask, name="factor_mask", T=T, N=N)
    rm = _check_mask(fwd_mask, name="fwd_mask", T=T, N=N)
    if device == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for device='cpu'")
    _require_cuda("rolling_ic")
    _sync_entry(df)
    with _ROLL_CACHE.use((T, N)) as ws:
        res = nat.fcb().rolling_ic_f64(f, r, fm, rm, min_valid, workspace=ws)
    kind = "torch" if (kf == "torch" or kr == "torch") else "numpy"
    if kind == "numpy":
        return res
    return _torch.as_tensor(res, device=_torch.device(df))


def _rolling_ic_dev(factor, forward_returns, factor_mask, fwd_mask, min_valid, device):
    """rolling_ic of two CUDA tensors through fcb_dev_rolling_ic; (T,) f64 on their device."""
    df, f = _dev_input(factor, name="factor", ndim=2)
    _, r = _dev_input(forward_returns, name="forward_returns", ndim=2)
    T, N = f.shape
    if tuple(r.shape) != (T, N):
        raise ValueError(f"factor and forward_returns shapes must match (T,N), got {tuple(f.shape)} vs "
                         f"{tuple(r.shape)}")
    _mask_device(factor_mask, df, "factor_mask")
    _mask_device(fwd_mask, df, "fwd_mask")
    fm = _dev_mask(factor_mask, name="factor_mask", T=T, N=N, device=f.device)
    rm = _dev_mask(fwd_mask, name="fwd_mask", T=T, N=N, device=f.device)
    if device == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for device='cpu'")
    _require_cuda("rolling_ic")
    ic = _torch.empty((T,), dtype=_torch.float64, device=f.device)
    with _torch.cuda.device(f.device):
        nat.check(nat.lib().fcb_dev_rolling_ic(nat.ptr(f), _dtype_code(f), nat.ptr(r), _dtype_code(r), nat.ptr(fm),
                                               nat.ptr(rm), T, N, min_valid, nat.ptr(ic), None, None,
                                               _stream_of(f)), "rolling_ic")
    return ic


def factor_corr(data, mask=None, names=None, backend="cuda"):
    """(F,F) pooled pairwise-complete correlation (fc/correlation.py:52-72)."""
    if backend not in ("cpu", "cuda"):
        raise ValueError(f"backend must be 'cpu' or 'cuda', got {backend!r}")
    if _is_cuda(data):
        return _factor_corr_dev(data, mask, names, backend)
    kind, device, arr = _to_numpy(data, name="data", ndim=3)
    T, N, F = arr.shape
    if names is not None and len(names) != F:
        raise ValueError(f"names length {len(names)} must equal F={F}")
    if backend == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for backend='cpu'")
    _require_cuda("factor_corr backend='cuda'")
    _mask_device(mask, device, "mask")
    m = _check_mask(mask, name="mask", T=T, N=N)
    if F > 128:
        raise ValueError("F > 128 (factor pair grid cap)")
    _domain_check(arr, m)
    _sync_entry(device)
    res = nat.fcp().factor_corr_f64(arr, m)
    return res if kind == "numpy" else _make_output(res, kind, device)


def _factor_corr_dev(data, mask, names, backend):
    """factor_corr of a CUDA (T,N,F) tensor through fcb_dev_factor_corr; (F,F) f64 on its device."""
    device, x = _dev_input(data, name="data", ndim=3)
    T, N, F = x.shape
    if names is not None and len(names) != F:
        raise ValueError(f"names length {len(names)} must equal F={F}")
    if backend == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for backend='cpu'")
    _require_cuda("factor_corr backend='cuda'")
    _mask_device(mask, device, "mask")
    m = _dev_mask(mask, name="mask", T=T, N=N, device=x.device)
    if F > 128:
        raise ValueError("F > 128 (factor pair grid cap)")
    out = _torch.empty((F, F), dtype=_torch.float64, device=x.device)
    stream = _torch.cuda.current_stream(x.device)
    with _torch.cuda.device(x.device):
        if x.dtype == _torch.float64:  # f32 panels always lie inside the domain
            ok = C.c_int(0)
            nat.check(nat.lib().fcb_dev_corr_domain(nat.ptr(x), nat.FCB_DTYPE_F64, nat.ptr(m), T, N, F, 0,
                                                    C.byref(ok), stream.cuda_stream), "factor_corr domain")
            if not ok.value:
                raise ValueError(DOMAIN_MSG)
        with _DEV_CACHE.use(x.device.index) as ws:
            rc = nat.lib().fcb_dev_factor_corr(nat.ptr(x), _dtype_code(x), nat.ptr(m), T, N, F, 0, nat.ptr(out),
                                               ws.handle, stream.cuda_stream)
            stream.synchronize()  # the workspace's scratch is free again once this returns
    if rc != 0:  # the reference binding maps every failure to RuntimeError
        raise RuntimeError(f"factor_corr: error {rc} ({nat.status_string(rc)})")
    return out


def _stock_corr_dev(data, mask, backend):
    """stock_corr of a CUDA (T,N) tensor through fcb_dev_stock_corr; (N,N) f64 on its device."""
    device, x = _dev_input(data, name="data", ndim=2)
    T, N = x.shape
    if backend == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for backend='cpu'")
    _require_cuda("stock_corr backend='cuda'")
    _mask_device(mask, device, "mask")
    m = _dev_mask(mask, name="mask", T=T, N=N, device=x.device)
    if int(N) * N > (1 << 31) - 1:
        raise ValueError("N*N exceeds INT32_MAX (output grid cap, N <= 46340)")
    out = _torch.empty((N, N), dtype=_torch.float64, device=x.device)
    stream = _torch.cuda.current_stream(x.device)
    with _torch.cuda.device(x.device), _DEV_CACHE.use(x.device.index) as ws:
        rc = nat.lib().fcb_dev_stock_corr(nat.ptr(x), _dtype_code(x), nat.ptr(m), T, N, nat.ptr(out), None, None,
                                          ws.handle, stream.cuda_stream)
        stream.synchronize()
    if rc == -4:
        raise ValueError(DOMAIN_MSG)
    nat.check(rc, "stock_corr")
    return out


def stock_corr(data, mask=None, backend="cuda"):
    """(N,N) pairwise-complete correlation over t (fc/correlation.py:75-93)."""
    if backend not in ("cpu", "cuda"):
        raise ValueError(f"backend must be 'cpu' or 'cuda', got {backend!r}")
    if _is_cuda(data):
        return _stock_corr_dev(data, mask, backend)
    kind, device, arr = _to_numpy(data, name="data", ndim=2)
    T, N = arr.shape
    if backend == "cpu":
        raise NotImplementedError("fcb200 has no CPU backend; use the reference adapter for backend='cpu'")
    _require_cuda("stock_corr backend='cuda'")
    _mask_device(mask, device, "mask")
    m = _check_mask(mask, name="mask", T=T, N=N)
    if int(N) * N > (1 << 31) - 1:
        raise ValueError("N*N exceeds INT32_MAX (output grid cap, N <= 46340)")
    _domain_check(arr, m)
    _sync_entry(device)
    res = nat.fcb().stock_corr_f64(arr, m)
    return res if kind == "numpy" else _make_output(res, kind, device)


# ---------------------------------------------------------------------------
# extensions
# ---------------------------------------------------------------------------
class Workspace:
    """Cached device buffers (and, for the learned method, the CDF model)
    reused across ``rank_ic_panel`` calls.  Not thread-safe."""

    def __init__(self):
        self._h = nat.lib().fcb_workspace_create()
        if not self._h:
            raise MemoryError("fcb_workspace_create failed")

    @property
    def handle(self):
        return self._h

    def learned_state(self):
        import ctypes as C
        r, f, lc = C.c_int(), C.c_int(), C.c_int()
        nat.check(nat.lib().fcb_workspace_learned_state(self._h, C.byref(r), C.byref(f), C.byref(lc)),
                  "fcb_workspace_learned_state")
        return {"ready": bool(r.value), "fits": f.value, "learned_chunks": lc.value}

    def clear(self):
        nat.lib().fcb_workspace_clear(self._h)

    def close(self):
        if self._h:
            nat.lib().fcb_workspace_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rank_ic_panel(X, forward_returns, factor_mask=None, fwd_mask=None, min_valid=30,
                  method="radix", return_ranks=True, workspace=None):
    """cs_rank + rolling_ic of F factor panels X (F,T,N) f32 against one
    forward-return panel (T,N) f32, in one streamed call.  Returns
    ``(ranks (F,T,N) f32 | None, ic (F,T) f64)``; ranks follow
    cross_sectional_rank(X[f], factor_mask), ic follows
    rolling_ic(X[f], forward_returns, factor_mask, fwd_mask, min_valid)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    R = np.ascontiguousarray(forward_returns, dtype=np.float32)
    if X.ndim != 3 or R.shape != X.shape[1:]:
        raise ValueError("X must be (F,T,N) and forward_returns (T,N)")
    F, T, N = X.shape
    if not isinstance(min_valid, int) or isinstance(min_valid, bool) or min_valid < 2:
        raise ValueError("min_valid must be an integer >= 2")
    meth = {"radix": 0, "learned": 1}[method]
    fm = None if factor_mask is None else np.ascontiguousarray(factor_mask, dtype=np.uint8)
    rm = None if fwd_mask is None else np.ascontiguousarray(fwd_mask, dtype=np.uint8)
    _require_cuda("rank_ic_panel")
    ranks = np.empty((F, T, N), np.float32) if return_ranks else None
    ic = np.empty((F, T), np.float64)
    rc = nat.lib().fcb_rank_ic_panel(nat.ptr(X), nat.ptr(R), nat.ptr(fm), nat.ptr(rm), F, T, N, min_valid,
                                     nat.ptr(ranks), nat.ptr(ic), meth,
                                     workspace.handle if workspace is not None else None)
    nat.check(rc, "rank_ic_panel")
    return ranks, ic


class CdfModel:
    """Learned-splitter CDF networks (one per factor) on the current device.

    ``fit(d_x, d_ranks, t0, tcount)`` trains on dates [t0, t0+tcount) of
    device-resident (F,T,N) f32 panels and their exact cs ranks (torch CUDA
    tensors or raw device pointers); ``state()`` / ``load()`` save and restore
    parameters, grid range and table (host numpy) for checkpoint / resume."""

    def __init__(self, F, seed=20261203, linear=False):
        self.F = int(F)
        self._h = nat.lib().fcb_cdf_model_create(self.F, int(seed))
        if not self._h:
            raise RuntimeError("fcb_cdf_model_create failed (no CUDA device or out of memory)")
        if linear:
            nat.check(nat.lib().fcb_cdf_model_set_linear(self._h, 1), "fcb_cdf_model_set_linear")

    @property
    def handle(self):
        return self._h

    def fit(self, d_x, d_ranks, T, N, t0, tcount, steps=1500, lr=3e-3, stream=None):
        rc = nat.lib().fcb_cdf_model_fit(self._h, nat.ptr(d_x), nat.ptr(d_ranks), int(T), int(N), int(t0),
                                         int(tcount), int(steps), float(lr), stream)
        nat.check(rc, "fcb_cdf_model_fit")

    def sample(self, d_x, d_ranks, T, N, t0, tcount, stream=None):
        """Draw training samples from dates [t0, t0+tcount) (first half of a fit)."""
        rc = nat.lib().fcb_cdf_model_sample(self._h, nat.ptr(d_x), nat.ptr(d_ranks), int(T), int(N), int(t0),
                                            int(tcount), stream)
        nat.check(rc, "fcb_cdf_model_sample")

    def train(self, steps, lr, into_idle=True, stream=None):
        """Adam steps on the drawn samples, tabulated into the idle table slot
        (rank calls keep reading the current one) or the current slot."""
        nat.check(nat.lib().fcb_cdf_model_train(self._h, int(steps), float(lr), 1 if into_idle else 0, stream),
                  "fcb_cdf_model_train")

    def swap(self):
        """Make the slot the last train(into_idle=True) wrote the current one."""
        nat.check(nat.lib().fcb_cdf_model_swap(self._h), "fcb_cdf_model_swap")

    def state(self):
        P, K = 1153, 1024
        params = np.empty((self.F, P), np.float32)
        zr = np.empty((self.F, 2), np.float32)
        tab = np.empty((self.F, K), np.float32)
        loss = np.empty(self.F, np.float32)
        nat.check(nat.lib().fcb_cdf_model_state(self._h, nat.ptr(params), nat.ptr(zr), nat.ptr(tab), nat.ptr(loss)),
                  "fcb_cdf_model_state")
        return {"params": params, "zrange": zr, "table": tab, "loss": loss}

    def load(self, st):
        p = np.ascontiguousarray(st["params"], np.float32)
        z = np.ascontiguousarray(st["zrange"], np.float32)
        t = np.ascontiguousarray(st["table"], np.float32)
        nat.check(nat.lib().fcb_cdf_model_load(self._h, nat.ptr(p), nat.ptr(z), nat.ptr(t)), "fcb_cdf_model_load")

    def close(self):
        if self._h:
            nat.lib().fcb_cdf_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cdf_grad(params, z, u):
    """Loss and gradient of the CDF network on one batch (<= 256 samples),
    computed by the GPU training kernel's forward/backward code."""
    p = np.ascontiguousarray(params, np.float32)
    z = np.ascontiguousarray(z, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    g = np.empty(1153, np.float32)
    loss = np.empty(1, np.float32)
    nat.check(nat.lib().fcb_cdf_grad(nat.ptr(p), nat.ptr(z), nat.ptr(u), int(z.size), nat.ptr(g), nat.ptr(loss)),
              "fcb_cdf_grad")
    return float(loss[0]), g


class Batch:
    """Many panels of uneven T x N per launch (fcb_batch_* in include/fcb200.h).

    ``panels`` is a list of dicts of device-resident torch tensors on the
    current CUDA device: ``X`` (F,T,N) factor planes, ``R`` (T,N) forward
    returns, optional ``fmask`` / ``rmask`` (T,N) uint8, outputs ``ic`` (F,T)
    f64 (required), ``ranks`` (F,T,N) f32 and ``corr`` (F,F) f64 (optional),
    and optional ``model`` (a fitted :class:`CdfModel`, f32 panels).  All
    panels share one dtype pair, (f32, f32) or (f64, f64).  The tensors are
    kept referenced for the batch's lifetime.  ``run()`` replays the batch's
    CUDA graph on the current stream; ``run_per_panel()`` issues the same work
    one panel at a time (the comparison arm); results agree bit for bit."""

    def __init__(self, panels, min_valid=30, config=None):
        _require_cuda("Batch")
        if not panels:
            raise ValueError("Batch needs at least one panel")
        self._keep = []
        arr = (nat.FcbPanel * len(panels))()
        dts = set()
        for k, p in enumerate(panels):
            X, R = p["X"], p["R"]
            F, T, N = (int(v) for v in X.shape)
            if tuple(R.shape) != (T, N):
                raise ValueError(f"panel {k}: R must be (T,N) = {(T, N)}")
            dts.add((str(X.dtype), str(R.dtype)))
            model = p.get("model")
            arr[k] = nat.FcbPanel(T, N, F, nat.ptr(X), nat.ptr(R), nat.ptr(p.get("fmask")), nat.ptr(p.get("rmask")),
                                  nat.ptr(p.get("ranks")), nat.ptr(p["ic"]), nat.ptr(p.get("corr")),
                                  model.handle if model is not None else None)
            self._keep.append(p)
        if len(dts) != 1:
            raise ValueError("all panels of a batch share one dtype pair")
        (dx, dr), = dts
        code = {"torch.float32": nat.FCB_DTYPE_F32, "torch.float64": nat.FCB_DTYPE_F64}
        if dx not in code or dr not in code:
            raise TypeError(f"unsupported panel dtypes {dx}, {dr}")
        cfgp = None
        if config is not None:
            cfg = nat.FcbBatchConfig()
            nat.lib().fcb_batch_default_config(C.byref(cfg))
            for k2, v in dict(config).items():
                setattr(cfg, k2, int(v))
            cfgp = C.byref(cfg)
        h = C.c_void_p()
        nat.check(nat.lib().fcb_batch_create(arr, len(panels), code[dx], code[dr], int(min_valid), cfgp, C.byref(h)),
                  "fcb_batch_create")
        self._h = h
        self._arr = arr

    def _stream(self):
        return C.c_void_p(_torch.cuda.current_stream().cuda_stream)

    def run(self):
        nat.check(nat.lib().fcb_batch_run(self._h, self._stream()), "fcb_batch_run")

    def run_per_panel(self):
        nat.check(nat.lib().fcb_batch_run_per_panel(self._h, self._stream()), "fcb_batch_run_per_panel")

    def status(self):
        nat.check(nat.lib().fcb_batch_status(self._h), "fcb_batch_status")

    @property
    def config(self):
        cfg = nat.FcbBatchConfig()
        nat.check(nat.lib().fcb_batch_get_config(self._h, C.byref(cfg)), "fcb_batch_get_config")
        return cfg.as_dict()

    @config.setter
    def config(self, value):
        cfg = nat.FcbBatchConfig()
        nat.check(nat.lib().fcb_batch_get_config(self._h, C.byref(cfg)), "fcb_batch_get_config")
        for k, v in dict(value).items():
            setattr(cfg, k, int(v))
        nat.check(nat.lib().fcb_batch_set_config(self._h, C.byref(cfg)), "fcb_batch_set_config")

    def autotune(self, reps=3, cache_path=None):
        """Measure alternative configurations and keep the fastest; returns
        (config dict, mean ms per replay, from_cache)."""
        cfg = nat.FcbBatchConfig()
        ms = C.c_float()
        path = None if cache_path is None else str(cache_path).encode()
        rc = nat.lib().fcb_batch_autotune(self._h, int(reps), path, C.byref(cfg), C.byref(ms))
        if rc not in (0, 1):
            nat.check(rc, "fcb_batch_autotune")
        return cfg.as_dict(), float(ms.value), rc == 1

    def close(self):
        if getattr(self, "_h", None):
            nat.lib().fcb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
