"""GPU checks of the stock_corr precision forms (BF16x3 tensor cores, FP32).

Error is measured against the f64 path (itself within 1e-12 of the oracle):
BF16x3 must stay within max |err| <= 1e-6 (the stated bound of the
precision form); FP32 within 5e-5.  NaN pattern and the diagonal follow the
f64 path on degenerate columns."""
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
