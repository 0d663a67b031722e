"""GPU checks of the precision forms (BF16x3 tensor cores, FP32).

stock_corr: error is measured against the f64 path (itself within 1e-12 of
the oracle): BF16x3 must stay within max |err| <= 1e-6 (the stated bound of
the precision form); FP32 within 5e-5.  factor_corr BF16x3: within 1e-6 of
the oracle per output.  NaN pattern and the diagonal follow the f64 results
on degenerate columns."""
import numpy as np
import pytest

from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat():
    from fcb200 import _native
    if _native.device_count() < 1:
        pytest.skip("no CUDA device")
    return _native


def run(nat, X, mask, mode):
    N = X.shape[1]
    out = np.empty((N, N))
    ws = nat.lib().fcb_workspace_create()
    try:
        rc = nat.lib().fcb_stock_corr_prec(nat.ptr(X), nat.ptr(mask), X.shape[0], N, mode, nat.ptr(out), ws)
        nat.check(rc, "fcb_stock_corr_prec")
    finally:
        nat.lib().fcb_workspace_destroy(ws)
    return out


@pytest.mark.parametrize("N", [37, 300, 1000])
def test_precision_forms_against_f64(nat, N):
    import bench
    X, mask = bench.make_stock_panel(T=1218, N=N, seed=N)
    m8 = mask.astype(np.uint8)
    ref = nat.fcb().stock_corr_f64(X, mask)
    for mode, tol in ((0, 1e-6), (1, 5e-5)):
        got = run(nat, X, m8, mode)
        assert np.array_equal(np.isnan(got), np.isnan(ref)), mode
        err = np.nanmax(np.abs(got - ref))
        assert err <= tol, (mode, err)
        assert np.array_equal(got, got.T, equal_nan=True)


def test_precision_degenerate_columns(nat):
    rng = np.random.default_rng(1)
    T, N = 200, 70
    X = (0.01 * rng.standard_normal((T, N))).astype(np.float32)
    X[:, 3] = 0.5          # constant column
    X[:, 4] = np.nan       # empty column
    X[:150, 5] = np.nan    # short column
    mask = np.ones((T, N), bool)
    mask[:, 6] = False
    mask[0, 6] = True      # one valid date -> n < 2
    ref = O.stock_corr(X, mask)
    for mode in (0, 1):
        got = run(nat, X, mask.astype(np.uint8), mode)
        assert np.array_equal(np.isnan(got), np.isnan(ref)), mode
        assert np.nanmax(np.abs(got - ref)) <= 5e-5


# ------------------------------------------------ factor_corr BF16x3 form
def fc_bf16x3(nat, X3, mask):
    T, N, F = X3.shape
    out = np.empty((F, F))
    m8 = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    rc = nat.lib().fcb_factor_corr_bf16x3(nat.ptr(np.ascontiguousarray(X3, np.float32)),
                                          None if m8 is None else nat.ptr(m8), T, N, F, nat.ptr(out), None)
    nat.check(rc, "fcb_factor_corr_bf16x3")
    return out


@pytest.mark.parametrize("F", [1, 4, 12, 16])
def test_factor_corr_bf16x3_against_oracle(nat, F):
    rng = np.random.default_rng(F)
    T, N = 60, 700
    X = rng.standard_normal((T, N, F)).astype(np.float32)
    if F > 2:
        X[..., 1] = np.exp(X[..., 1])                       # lognormal column
        X[..., 2] = 0.6 * X[..., 0] + 0.4 * X[..., 2] + 50  # correlated, biased column
    X[rng.random((T, N, F)) < 0.05] = np.nan
    mask = rng.random((T, N)) < 0.9
    exp = O.factor_corr(X, mask)
    got = fc_bf16x3(nat, X, mask)
    assert np.array_equal(np.isnan(got), np.isnan(exp))
    assert np.nanmax(np.abs(got - exp)) <= 1e-6, np.nanmax(np.abs(got - exp))
    assert np.array_equal(got, got.T, equal_nan=True)
    got_nm = fc_bf16x3(nat, X, None)
    assert np.nanmax(np.abs(got_nm - O.factor_corr(X, None))) <= 1e-6


def test_factor_corr_bf16x3_degenerate_and_planes(nat):
    import torch
    rng = np.random.default_rng(11)
    T, N, F = 30, 401, 6
    X = rng.standard_normal((T, N, F)).astype(np.float32)
    X[..., 1] = 0.25            # constant factor -> NaN row, NaN diagonal
    X[..., 2] = np.nan          # empty factor
    X[:, 1:, 3] = np.nan        # one valid row per date
    X[1:, :, 4] = np.nan        # valid on the first date only
    X[0, 0, 4] = np.nan
    mask = np.ones((T, N), bool)
    exp = O.factor_corr(X, mask)
    got = fc_bf16x3(nat, X, mask)
    assert np.array_equal(np.isnan(got), np.isnan(exp))
    assert np.nanmax(np.abs(got - exp)) <= 1e-6
    # the device entry point on factor planes gives the same result
    dev = torch.device("cuda", 0)
    planes = torch.from_numpy(np.ascontiguousarray(np.moveaxis(X, -1, 0))).to(dev)
    dm = torch.from_numpy(mask.astype(np.uint8)).to(dev)
    out = torch.empty((F, F), dtype=torch.float64, device=dev)
    lib = nat.lib()
    ws = lib.fcb_workspace_create()
    try:
        nat.check(lib.fcb_dev_factor_corr_bf16x3(planes.data_ptr(), dm.data_ptr(), T, N, F, 1, out.data_ptr(), ws,
                                                 torch.cuda.current_stream(dev).cuda_stream),
                  "fcb_dev_factor_corr_bf16x3")
        torch.cuda.synchronize(dev)
    finally:
        lib.fcb_workspace_destroy(ws)
    assert np.array_equal(out.cpu().numpy(), got, equal_nan=True)
    nat.check(lib.fcb_dev_status(), "fcb_dev_status")
