"""Pin the oracle (oracle/fc_oracle.py) against the reference's own outputs.

Every golden case was computed by the reference's CPU path or taken from its
frozen fixtures (tests/golden/make_golden.py).  Ranks must agree bitwise,
IC bitwise (the ordinal-rank Pearson is exact before its final divide/sqrt),
correlations within 1e-12 with the same NaN pattern.
"""
import numpy as np
import pytest

from conftest import bitwise_f32, corr_match
from oracle import fc_oracle as O


def _cases(golden, op):
    cases, arrays = golden
    return [c for c in cases if c["op"] == op], arrays


def test_golden_has_every_op(golden):
    ops = {c["op"] for c in golden[0]}
    assert {"cs_rank", "parameter_scan", "rolling_ic", "factor_corr", "stock_corr"} <= ops


def test_cs_rank_pins(golden):
    cases, A = _cases(golden, "cs_rank")
    assert len(cases) >= 50
    for c in cases:
        x = A[c["inputs"][0]]
        if x.ndim == 1:
            x = x[None, :]
        m = A[c["masks"]["mask"]] if "mask" in c["masks"] else None
        if m is not None and m.ndim == 1:
            m = m[None, :]
        out = O.cs_rank(x, m, c["params"]["descending"])
        assert bitwise_f32(out, A[c["ref_out"]]), c["id"]
        if isinstance(c.get("expected"), list):
            exp = np.array([np.nan if e == "nan" else e for e in c["expected"]], np.float32)
            assert np.array_equal(out[0], exp, equal_nan=True), c["id"]


def test_parameter_scan_pins(golden):
    cases, A = _cases(golden, "parameter_scan")
    for c in cases:
        if "ref_out" not in c:
            continue
        outs = O.parameter_scan(A[c["inputs"][0]], A[c["masks"]["mask"]])
        for g in range(4):
            assert bitwise_f32(outs[g], A[c["ref_out"]][g]), (c["id"], g)


def test_rolling_ic_pins(golden):
    cases, A = _cases(golden, "rolling_ic")
    assert len(cases) >= 20
    for c in cases:
        f = A[c["inputs"][0]]
        r = A[c["inputs"][1]]
        if f.ndim == 1:
            f, r = f[None, :], r[None, :]
        fm = A[c["masks"]["factor_mask"]] if "factor_mask" in c["masks"] else None
        rm = A[c["masks"]["fwd_mask"]] if "fwd_mask" in c["masks"] else None
        out = O.rolling_ic(f, r, fm, rm, c["params"]["min_valid"])
        ref = A[c["ref_out"]]
        # bit-exact, NaN pattern included
        assert np.array_equal(out.view(np.uint64)[~np.isnan(out)],
                              ref.view(np.uint64)[~np.isnan(ref)]), c["id"]
        assert np.array_equal(np.isnan(out), np.isnan(ref)), c["id"]
        if c.get("expected") not in (None,) and not isinstance(c.get("expected"), dict):
            e = c["expected"]
            if e == "nan":
                assert np.isnan(out).all(), c["id"]
            elif isinstance(e, float):
                assert abs(out[0] - e) <= 1e-12, c["id"]


def test_factor_corr_pins(golden):
    cases, A = _cases(golden, "factor_corr")
    for c in cases:
        if c.get("ref_error"):
            cols = [A[k].astype(np.float64) for k in c["inputs"]]
            if len(cols) == 1:
                with pytest.raises(ValueError):
                    O.factor_corr(cols[0][:, None, None][..., 0])
                continue
            with pytest.raises(ValueError):
                O.factor_corr(np.stack(cols, axis=1)[:, None, :])
            continue
        if "ref_out" not in c:
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
        out = O.factor_corr(x, m)
        assert corr_match(out, A[c["ref_out"]]), c["id"]
        e = c.get("expected")
        if isinstance(e, float):
            assert abs(out[0, 1] - e) <= 1e-12, c["id"]
        elif e == "nan":
            assert np.isnan(out[0, 1]), c["id"]


def test_stock_corr_pins(golden):
    cases, A = _cases(golden, "stock_corr")
    for c in cases:
        X = A[c["inputs"][0]]
        m = A[c["masks"]["mask"]] if "mask" in c["masks"] else None
        if c.get("ref_error"):
            with pytest.raises(ValueError):
                O.stock_corr(X, m)
            continue
        out = O.stock_corr(X, m)
        assert corr_match(out, A[c["ref_out"]]), c["id"]
        if c["source"] == "corr_corpus_v1":
            ref01 = float(A[c["ref_out"]][0, 1])
            if c["expected_is_nan"]:
                assert np.isnan(out[0, 1]), c["id"]
            elif abs(ref01 - c["expected"]) <= 1e-12:
                # The manifest's exact-arithmetic value for bias_1e15 is not
                # what the reference's two-pass/Kahan-mean path returns (its
                # own suite checks against serial Kahan instead), so the
                # manifest value is asserted only where the reference meets it.
                assert abs(out[0, 1] - c["expected"]) <= 1e-12, c["id"]


def test_canonical_keys_order_and_zero_fold():
    v = np.array([-np.inf, -3.5, -1e-45, -0.0, 0.0, 1e-45, 2.0, np.inf, np.nan], np.float32)
    k = O.canonical_key_f32(v)
    fin = k[1:7]
    assert list(fin) == sorted(fin)
    assert k[3] == k[4] == 0x80000000
    assert k[0] == k[7] == k[8] == 0xFFFFFFFF
    k64 = O.canonical_key_f64(v.astype(np.float64))
    assert list(k64[1:7]) == sorted(k64[1:7])
    assert k64[3] == k64[4]
