"""GPU parity: every golden case and seeded random panels, through the drop-in
modules (which call the C ABI) and through the fc-compatible adapter, against
the oracle.  Ranks and IC bit-exact; correlations within 1e-12 (the
reference suite's tolerance, tests/test_adapter_v1.py:67-82)."""
import numpy as np
import pytest

from conftest import bitwise_f32, corr_match
from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fcb():
    from fcb200 import _native
    if _native.device_count() < 1:
        pytest.skip("no CUDA device")
    return _native.fcb()


@pytest.fixture(scope="module")
def fcp():
    from fcb200 import _native
    return _native.fcp()


def _ic_cap(fdt, rdt):
    """Largest N the fused shared-memory rank+IC kernel takes for these dtypes."""
    return 8192 if (np.dtype(fdt) == np.float64 or np.dtype(rdt) == np.float64) else 11000


def _ic_equal(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and \
        np.array_equal(a[~np.isnan(a)].view(np.uint64), b[~np.isnan(b)].view(np.uint64))


# ------------------------------------------------------------------ golden
def test_golden_cs_rank(golden, fcb):
    cases, A = golden
    n = 0
    for c in cases:
        if c["op"] != "cs_rank":
            continue
        x = A[c["inputs"][0]]
        x = x[None, :] if x.ndim == 1 else x
        m = A[c["masks"]["mask"]] if "mask" in c["masks"] else None
        if m is not None and m.ndim == 1:
            m = m[None, :]
        if x.shape[1] > 16384:
            continue  # the global-memory path covers N > 16384 (test_large_n)
        got = fcb.cs_rank_f32(np.ascontiguousarray(x, np.float32), m, c["params"]["descending"])
        assert bitwise_f32(got, A[c["ref_out"]]), c["id"]
        n += 1
    assert n >= 40


def test_golden_parameter_scan(golden, fcb):
    cases, A = golden
    for c in cases:
        if c["op"] != "parameter_scan" or "ref_out" not in c:
            continue
        r = fcb.parameter_scan_f32(A[c["inputs"][0]], A[c["masks"]["mask"]], return_timing=True)
        assert r["group_status"] == [0, 0, 0, 0]
        for g in range(4):
            assert bitwise_f32(r["groups"][g], A[c["ref_out"]][g]), (c["id"], g)


def test_golden_rolling_ic(golden, fcb):
    cases, A = golden
    n = 0
    for c in cases:
        if c["op"] != "rolling_ic":
            continue
        f = A[c["inputs"][0]]
        r = A[c["inputs"][1]]
        if f.ndim == 1:
            f, r = f[None, :], r[None, :]
        fm = A[c["masks"]["factor_mask"]] if "factor_mask" in c["masks"] else None
        rm = A[c["masks"]["fwd_mask"]] if "fwd_mask" in c["masks"] else None
        got = fcb.rolling_ic_f64(f, r, fm, rm, c["params"]["min_valid"])
        assert _ic_equal(got, A[c["ref_out"]]), c["id"]
        n += 1
    assert n >= 20


def test_golden_stock_corr(golden, fcb):
    cases, A = golden
    for c in cases:
        if c["op"] != "stock_corr":
            continue
        X = A[c["inputs"][0]]
        m = A[c["masks"]["mask"]] if "mask" in c["masks"] else None
        if c.get("ref_error"):
            with pytest.raises(ValueError):
                fcb.stock_corr_f64(X, m)
            continue
        got = fcb.stock_corr_f64(X, m)
        if c["id"] == "corpus_pearson_overflow":
            # The reference CPU path's product-form denominator sqrt(vx*vy)
            # overflows to inf here and returns 0.0; the manifest, the
            # contract and the reference's GPU kernel (sequential
            # (sxy/sqrt(sxx))/sqrt(syy)) give 1.0, which is what this path returns.
            assert A[c["ref_out"]][0, 1] == 0.0 and c["expected"] == 1.0
            assert got[0, 1] == 1.0 and got[1, 0] == 1.0
            continue
        assert corr_match(got, A[c["ref_out"]]), (c["id"], np.nanmax(np.abs(got - A[c["ref_out"]])))
        assert np.array_equal(got, got.T, equal_nan=True)


def test_golden_factor_corr(golden, fcp):
    cases, A = golden
    for c in cases:
        if c["op"] != "factor_corr" or "ref_out" not in c:
            continue
        x = A[c["inputs"][0]]
        if len(c["inputs"]) >= 2 or x.ndim == 1:
            cols = [A[k].astype(np.float64) for k in c["inputs"]]
            if len(cols) == 1:
                cols = [cols[0], cols[0]]
            x = np.stack(cols, axis=1)[:, None, :]
            m = A[c["masks"]["mask"]][:, None] if "mask" in c["masks"] else None
        else:
            m = A[c["masks"]["mask"]] if "mask" in c["masks"] else None
        got = fcp.factor_corr_f64(x, m)
        assert corr_match(got, A[c["ref_out"]]), (c["id"], got, A[c["ref_out"]])


# ------------------------------------------------------------ random panels
@pytest.mark.parametrize("N", [1, 2, 31, 33, 255, 256, 1000, 4096, 4097, 5000, 8192, 8193, 16384])
def test_random_rank_and_ic(fcb, N):
    rng = np.random.default_rng(N)
    T = 5
    x = rng.standard_normal((T, N)).astype(np.float32)
    x[rng.random((T, N)) < 0.05] = 0.0
    k = rng.random((T, N)) < 0.3
    x[k] = np.round(x[k], 1)
    x[rng.random((T, N)) < 0.05] = np.nan
    x[rng.random((T, N)) < 0.01] = -0.0
    m = rng.random((T, N)) < 0.9
    for desc in (False, True):
        assert bitwise_f32(fcb.cs_rank_f32(x, m, desc), O.cs_rank(x, m, desc))
        assert bitwise_f32(fcb.cs_rank_f32(x, None, desc), O.cs_rank(x, None, desc))
    r = (0.2 * np.nan_to_num(x) + rng.standard_normal((T, N))).astype(np.float64)
    r[rng.random((T, N)) < 0.05] = np.inf
    rm = rng.random((T, N)) < 0.95
    if N <= _ic_cap(x.dtype, r.dtype):
        ic, rf, rr = fcb.rolling_ic_f64(x, r, m, rm, 2, return_ranks=True)
        ic_e, rf_e, rr_e = O.rolling_ic(x, r, m, rm, 2, return_ranks=True)
        assert _ic_equal(ic, ic_e)
        assert np.array_equal(rf, rf_e) and np.array_equal(rr, rr_e)
    res = fcb.parameter_scan_f32(x, m)
    exp = O.parameter_scan(x, m)
    for g in range(4):
        assert bitwise_f32(res["groups"][g], exp[g]), g


def test_workspace_reuse_bitwise(fcb):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((20, 3000)).astype(np.float32)
    ws = fcb.CsRankWorkspace()
    a = fcb.cs_rank_f32(x, None, False, workspace=ws)
    b = fcb.cs_rank_f32(x, None, False, workspace=ws)
    c = fcb.cs_rank_f32(x, None, False)
    assert bitwise_f32(a, b) and bitwise_f32(a, c)
    x2 = rng.standard_normal((7, 1234)).astype(np.float32)
    d = fcb.cs_rank_f32(x2, None, True, workspace=ws)  # shape switch re-allocates
    assert bitwise_f32(d, O.cs_rank(x2, None, True))
    ws.clear()


def test_rank_ic_panel_matches_per_factor_ops():
    import fcb200
    rng = np.random.default_rng(11)
    F, T, N = 3, 9, 2500
    X = rng.standard_normal((F, T, N)).astype(np.float32)
    X[rng.random((F, T, N)) < 0.05] = np.nan
    R = (0.05 * np.nan_to_num(X[0]) + rng.standard_normal((T, N))).astype(np.float32)
    R[rng.random((T, N)) < 0.02] = np.nan
    fm = rng.random((T, N)) < 0.9
    rm = rng.random((T, N)) < 0.97
    ranks, ic = fcb200.rank_ic_panel(X, R, fm, rm, min_valid=30)
    for f in range(F):
        assert bitwise_f32(ranks[f], O.cs_rank(X[f], fm, False))
        assert _ic_equal(ic[f], O.rolling_ic(X[f], R, fm, rm, 30))


def test_rank_ic_panel_returns_pass_edge_dates():
    """The per-date returns pass ranks by sampled splitters and falls back to
    the radix sort inside the same CTA.  Dates that take each branch: ordinary
    heavy-tailed returns; returns with three distinct values (buckets far
    above the cap); constant returns (no usable sample range); a single valid
    return; a date where every sampled column is invalid but others are
    valid; ±0 and a value spread of 1e30.  Ranks and IC bitwise vs the
    oracle, N on both sides of the 2048 / 5120 kernel widths."""
    import fcb200
    rng = np.random.default_rng(23)
    for N in (300, 2500, 5000, 7000):
        F, T = 2, 8
        X = rng.standard_normal((F, T, N)).astype(np.float32)
        R = rng.standard_t(3, (T, N)).astype(np.float32)
        R[1] = rng.integers(0, 3, N).astype(np.float32)
        R[2] = 0.25
        R[3] = np.nan
        R[3, N // 3] = 1.0
        S = min(N, 256)
        sampled = (np.arange(S) * N) // 256 if N >= 256 else np.arange(S)
        R[4, sampled] = np.nan
        R[5, ::2] = -0.0
        R[5, 1::2] = 0.0
        R[6, : N // 2] *= 1e30
        fm = rng.random((T, N)) < 0.95
        ranks, ic = fcb200.rank_ic_panel(X, R, fm, None, min_valid=3)
        for f in range(F):
            assert bitwise_f32(ranks[f], O.cs_rank(X[f], fm, False)), N
            assert _ic_equal(ic[f], O.rolling_ic(X[f], R, fm, None, 3)), (N, f)


def test_stock_corr_random(fcb):
    rng = np.random.default_rng(5)
    T, N = 200, 300
    X = rng.standard_normal((T, N)) + rng.standard_normal((1, N)) * 3
    X[:, 5] += 1e9
    m = rng.random((T, N)) < 0.9
    got = fcb.stock_corr_f64(X, m)
    assert corr_match(got, O.stock_corr(X, m))
    gf, st = fcb.stock_corr_f64(X, None, return_stats=True)
    assert st["selected_path"] == 0
    assert corr_match(gf, O.stock_corr(X, None))
    X32 = X.astype(np.float32)
    assert np.array_equal(fcb.stock_corr_f64(X32, m), fcb.stock_corr_f64(X32.astype(np.float64), m),
                          equal_nan=True)


def test_factor_corr_random(fcp):
    rng = np.random.default_rng(9)
    T, N, F = 60, 500, 12
    F3 = rng.standard_normal((T, N, F)).astype(np.float32)
    F3[..., 1] += 0.5 * F3[..., 0]
    F3[rng.random((T, N, F)) < 0.05] = np.nan
    m = rng.random((T, N)) < 0.9
    got = fcp.factor_corr_f64(F3, m)
    assert corr_match(got, O.factor_corr(F3, m))
    assert np.array_equal(got, fcp.factor_corr_f64(F3.astype(np.float64), m), equal_nan=True)


@pytest.mark.parametrize("F", [33, 64, 65, 128])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_factor_corr_wide_panels(fcp, F, dtype):
    """Wide panels up to the F <= 128 cap: the Gram pass stages fewer rows
    per step above F = 64 and splits its tiles over several block rows."""
    rng = np.random.default_rng(F)
    T, N = 12, 700
    F3 = rng.standard_normal((T, N, F))
    F3[..., 1] += 0.5 * F3[..., 0]
    F3[..., 2] = np.exp(F3[..., 2]) + 50.0          # far-from-zero mean: the cancellation fallback
    F3[..., F - 1] = 3.0                            # constant factor
    F3[rng.random((T, N, F)) < 0.03] = np.nan
    F3 = F3.astype(dtype)
    m = rng.random((T, N)) < 0.93
    got = fcp.factor_corr_f64(F3, m)
    assert corr_match(got, O.factor_corr(F3, m))


def test_factor_corr_large_pool_fallback():
    """Pairs the cancellation gate flags on a large pool (200k rows) take the
    multi-block two-pass fallback: same results as the oracle (<= 1e-12) and
    as the single-block fallback of the no-allocation entry point."""
    import torch
    from fcb200 import _native as nat
    rng = np.random.default_rng(21)
    T, N, F = 200, 1000, 5
    F3 = rng.standard_normal((T, N, F))
    F3[..., 0] = 1e3 + F3[..., 0]                          # |mean| >> std: gate fires against 1, 2
    F3[..., 1] = 5e2 + 0.3 * F3[..., 0] + F3[..., 1]
    F3[..., 2] = np.exp(F3[..., 2])                        # lognormal
    F3[..., 3] = 3.0                                       # constant -> NaN row / column
    F3[rng.random((T, N, F)) < 0.02] = np.nan
    m = rng.random((T, N)) < 0.95
    for dt in (np.float64, np.float32):
        X = np.ascontiguousarray(F3.astype(dt))
        m8 = m.astype(np.uint8)
        out = np.empty((F, F))
        flags = np.zeros((F, F), np.uint8)
        nat.check(nat.lib().fcb_factor_corr(nat.ptr(X), 0 if dt == np.float32 else 1, nat.ptr(m8), T, N, F,
                                            nat.ptr(out), nat.ptr(flags)), "fcb_factor_corr")
        assert flags.sum() >= 2, "the gate should flag the biased pairs"
        assert corr_match(out, O.factor_corr(X, m))
        dX = torch.from_numpy(X).cuda()
        dM = torch.from_numpy(m8).cuda()
        dO = torch.empty((F, F), dtype=torch.float64, device="cuda")
        nat.check(nat.lib().fcb_dev_factor_corr_noalloc(dX.data_ptr(), 0 if dt == np.float32 else 1, dM.data_ptr(),
                                                        T, N, F, dO.data_ptr(), None), "noalloc")
        torch.cuda.synchronize()
        assert corr_match(out, dO.cpu().numpy())


def test_dev_factor_corr_layouts():
    """The device entry point, in both layouts, equals the host entry point."""
    import torch
    from fcb200 import _native as nat
    rng = np.random.default_rng(33)
    T, N, F = 40, 900, 6
    F3 = rng.standard_normal((T, N, F)).astype(np.float32)
    F3[..., 2] = np.exp(F3[..., 2]) + 3.0
    F3[rng.random((T, N, F)) < 0.03] = np.nan
    m8 = (rng.random((T, N)) < 0.9).astype(np.uint8)
    ref = np.empty((F, F))
    nat.check(nat.lib().fcb_factor_corr(nat.ptr(F3), 0, nat.ptr(m8), T, N, F, nat.ptr(ref), None), "host")
    ws = nat.lib().fcb_workspace_create()
    try:
        for planes, arr in ((0, F3), (1, np.ascontiguousarray(np.moveaxis(F3, -1, 0)))):
            dX = torch.from_numpy(arr).cuda()
            dM = torch.from_numpy(m8).cuda()
            dO = torch.empty((F, F), dtype=torch.float64, device="cuda")
            nat.check(nat.lib().fcb_dev_factor_corr(dX.data_ptr(), 0, dM.data_ptr(), T, N, F, planes, dO.data_ptr(), ws,
                                                    None), "dev")
            torch.cuda.synchronize()
            got = dO.cpu().numpy()
            assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), planes
    finally:
        nat.lib().fcb_workspace_destroy(ws)


def test_adapter_end_to_end():
    import fcb200
    rng = np.random.default_rng(1)
    x = rng.standard_normal((4, 300))
    m = rng.random((4, 300)) < 0.8
    got = fcb200.cross_sectional_rank(x, m)          # f64 -> f32 RNE downcast
    assert bitwise_f32(got, O.cs_rank(x.astype(np.float32), m, False))
    res = fcb200.parameter_scan([("direction", ["ascending", "descending"]),
                                 ("mask_mode", ["masked", "unmasked"])], x, m)
    assert [g["status"] for g in res["groups"]] == ["ok"] * 4
    assert res["summary"]["total_groups"] == 4
    big = np.full((5, 3), 1e151)
    with pytest.raises(ValueError, match="1e150"):
        fcb200.stock_corr(big)
    with pytest.raises(ValueError, match="1e150"):
        fcb200.factor_corr(big[:, :, None].repeat(2, axis=2))
