"""The no-allocation factor_corr entry point (fcb_dev_factor_corr_noalloc).

It serves callers that cannot let a library allocate device memory -- code
whose device memory belongs to a framework pool or a hard budget, and
latency-sensitive loops that cannot take the device-wide synchronisation of
cudaMalloc/cudaFree.  Its scratch lives in one fixed device array inside the
library, so this test checks, through the C ABI, that two calls in a row on
caller-owned device buffers give the same (F,F) matrix as the regular entry
points (within the 1e-12 tolerance the correlation tests use: the fixed array
fixes the row partition, so sums are added in another order), including a
column whose large bias sends pairs through the two-pass fallback and a pool
large enough for the fallback's multi-block split; that a call after the
first allocates no device memory; and that an F above the array's limit is
refused.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import corr_match

pytestmark = pytest.mark.gpu


def _cases(rng):
    # (T, N, F, dtype, bias column): small pools, a pool above the multi-block
    # fallback threshold (R >= 4096 rows, several row blocks per pair) and a
    # bias near the cancellation gate
    yield 120, 900, 12, np.float32, 1e9
    yield 33, 71, 5, np.float64, 1e9
    yield 400, 1000, 6, np.float64, 1e7
    yield 25, 40, 4, np.float32, 3e3


def test_noalloc_factor_corr_matches_regular_entry_points():
    torch = pytest.importorskip("torch")
    from fcb200 import _native as nat

    if nat.device_count() < 1:
        pytest.skip("no CUDA device")
    lib = nat.lib()
    rng = np.random.default_rng(2024)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    for (T, N, F, dt, bias) in _cases(rng):
        X = rng.standard_normal((T, N, F)).astype(dt)
        X[..., 1] += 0.7 * X[..., 0]
        X[rng.random((T, N, F)) < 0.04] = np.nan
        X[..., F - 1] += bias  # large bias: exercises the two-pass fallback
        mask = (rng.random((T, N)) < 0.9).astype(np.uint8)
        dtype = nat.FCB_DTYPE_F32 if dt == np.float32 else nat.FCB_DTYPE_F64

        ref = np.empty((F, F))
        rc = lib.fcb_factor_corr(nat.ptr(X), dtype, nat.ptr(mask), T, N, F, nat.ptr(ref), None)
        assert rc == 0, nat.status_string(rc)

        dX = torch.from_numpy(X).to(dev)
        dM = torch.from_numpy(mask).to(dev)
        # the regular device entry point on the same device buffers
        dReg = torch.empty((F, F), dtype=torch.float64, device=dev)
        ws = lib.fcb_workspace_create()
        try:
            rc = lib.fcb_dev_factor_corr(dX.data_ptr(), dtype, dM.data_ptr(), T, N, F, 0, dReg.data_ptr(), ws,
                                         stream.cuda_stream)
            assert rc == 0, nat.status_string(rc)
            torch.cuda.synchronize(dev)
        finally:
            lib.fcb_workspace_destroy(ws)
        reg = dReg.cpu().numpy()
        outs = []
        for _ in range(2):  # two calls in a row share the scratch array
            dOut = torch.full((F, F), -7.0, dtype=torch.float64, device=dev)
            rc = lib.fcb_dev_factor_corr_noalloc(dX.data_ptr(), dtype, dM.data_ptr(), T, N, F,
                                                 dOut.data_ptr(), stream.cuda_stream)
            assert rc == 0, nat.status_string(rc)
            torch.cuda.synchronize(dev)
            outs.append(dOut.cpu().numpy())
        for got in outs:
            assert corr_match(got, ref, tol=1e-12), np.nanmax(np.abs(got - ref))
            assert corr_match(got, reg, tol=1e-12), np.nanmax(np.abs(got - reg))
            assert np.array_equal(got, got.T, equal_nan=True)


def test_noalloc_second_call_allocates_nothing():
    torch = pytest.importorskip("torch")
    from fcb200 import _native as nat

    if nat.device_count() < 1:
        pytest.skip("no CUDA device")
    lib = nat.lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    T, N, F = 300, 2000, 8
    X = torch.from_numpy(rng.standard_normal((T, N, F)).astype(np.float32)).to(dev)
    M = torch.from_numpy((rng.random((T, N)) < 0.95).astype(np.uint8)).to(dev)
    out = torch.empty((F, F), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def call():
        rc = lib.fcb_dev_factor_corr_noalloc(X.data_ptr(), 0, M.data_ptr(), T, N, F, out.data_ptr(),
                                             stream.cuda_stream)
        assert rc == 0, nat.status_string(rc)
        torch.cuda.synchronize(dev)

    call()  # the first call on the device may load the library's device image
    first = out.cpu().numpy()
    free0, _ = torch.cuda.mem_get_info(dev)
    torch_bytes = torch.cuda.memory_allocated(dev)
    call()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.memory_allocated(dev) == torch_bytes
    assert np.array_equal(out.cpu().numpy(), first, equal_nan=True)


def test_noalloc_rejects_f_above_limit():
    from fcb200 import _native as nat

    lib = nat.lib()
    limit = 32  # FCB_NOALLOC_MAX_F in include/fcb200.h
    rc = lib.fcb_dev_factor_corr_noalloc(C.c_void_p(16), 0, None, 2, 2, limit + 1, C.c_void_p(16), None)
    assert rc == -6
    assert "FCB_NOALLOC_MAX_F" in nat.status_string(rc)
