"""numpy restatement of factor-cuda's CPU path (TEST INFRASTRUCTURE ONLY).

This module is the oracle the CUDA path is checked against.  It restates, in
this project's own code, the algorithms of the reference's CPU core
``fc/_cpu_core.py`` and the key transforms of its kernels; every function cites
the reference lines it follows.  It is pinned against the reference's own
outputs by ``tests/test_oracle_pins.py`` (golden vectors in ``tests/golden``).

Never imported by the product.  The CUDA extension fails loudly instead of
falling back here.
"""
from __future__ import annotations

import numpy as np

INVALID_KEY32 = np.uint32(0xFFFFFFFF)
INVALID_KEY64 = np.uint64(0xFFFFFFFFFFFFFFFF)
QNAN_BITS = np.uint32(0x7FC00000)

DOMAIN_MAX_ABS = 1e150   # src/stock_corr_impl.cuh:41 ; fc/_cpu_core.py:37-40
DOMAIN_MIN_ABS = 1e-150  # src/stock_corr_impl.cuh:42
CANCEL_RATIO = 3.0       # fc/_cpu_core.py:171 (_CANCEL_RATIO_THRESHOLD)


# --------------------------------------------------------------------------
# canonical ordinal keys
# --------------------------------------------------------------------------

def canonical_key_f32(x):
    """Order-preserving u32 key of f32 values.

    Follows src/cross_sectional_rank.cu:35-39 (canonical_ordinal_key_f32):
    +0/-0 fold to one key, negatives map to ~bits, non-negatives to
    bits|0x80000000, non-finite to 0xFFFFFFFF.
    """
    x = np.ascontiguousarray(x, dtype=np.float32)
    bits = x.view(np.uint32).copy()
    bits[x == 0.0] = 0
    neg = (bits & np.uint32(0x80000000)) != 0
    key = np.where(neg, ~bits, bits | np.uint32(0x80000000)).astype(np.uint32)
    key[~np.isfinite(x)] = INVALID_KEY32
    return key


def canonical_key_f64(x):
    """Order-preserving u64 key of f64 values (src/rolling_ic.cu:34-38)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    bits = x.view(np.uint64).copy()
    bits[x == 0.0] = 0
    neg = (bits & np.uint64(0x8000000000000000)) != 0
    key = np.where(neg, ~bits, bits | np.uint64(0x8000000000000000)).astype(np.uint64)
    key[~np.isfinite(x)] = INVALID_KEY64
    return key


def _rank_rows(keys, valid):
    """Stable ordinal rank 1..K of each row over ``valid`` cells (0 elsewhere).

    Restates the per-row ``argsort(kind='stable')`` of fc/_cpu_core.py:43-55
    and :57-78 on order-preserving keys (stable sort by key, ties by column).
    """
    T, N = keys.shape
    sentinel = np.iinfo(keys.dtype).max
    k = np.where(valid, keys, sentinel)
    order = np.argsort(k, axis=1, kind="stable")
    ranks = np.empty((T, N), dtype=np.int64)
    rows = np.arange(T)[:, None]
    ranks[rows, order] = np.arange(1, N + 1, dtype=np.int64)[None, :]
    ranks[~valid] = 0
    return ranks


# --------------------------------------------------------------------------
# cross_sectional_rank / parameter_scan
# --------------------------------------------------------------------------

def cs_rank(X, mask=None, descending=False):
    """(T,N) f32 stable ordinal rank; invalid cells are NaN (0x7fc00000).

    Follows fc/_cpu_core.py:57-78 (np_cs_rank): values are f32, descending
    ranks -X ascending, valid = isfinite & mask, ties by column index.
    """
    X = np.asarray(X, dtype=np.float32)
    if X.ndim != 2:
        raise ValueError("cs_rank input must be 2-D (T,N)")
    if X.shape[1] > 2 ** 24:
        raise ValueError("N > 2^24")
    Xw = -X if descending else X
    valid = np.isfinite(Xw)
    if mask is not None:
        valid &= np.asarray(mask, dtype=bool)
    ranks = _rank_rows(canonical_key_f32(Xw), valid)
    out = ranks.astype(np.float32)
    out.view(np.uint32)[~valid] = QNAN_BITS
    return out


def parameter_scan(X, mask):
    """Four groups in binding order asc-masked, asc-unmasked, desc-masked,
    desc-unmasked (fc/_cpu_core.py:295-301; fc/parameter_scan.py:26-30)."""
    res = []
    for desc in (False, True):
        for use_mask in (True, False):
            res.append(cs_rank(X, mask if use_mask else None, desc))
    return res


# --------------------------------------------------------------------------
# rolling_ic
# --------------------------------------------------------------------------

def rolling_ic(f, r, factor_mask=None, fwd_mask=None, min_valid=30,
               return_ranks=False):
    """Daily Spearman IC, (T,) f64.

    Follows fc/_cpu_core.py:271-293 (np_rolling_ic): joint valid set
    isfinite(f) & isfinite(r) & masks; fewer than min_valid cells -> NaN;
    ptp==0 of either side on the joint set -> NaN; ordinal ranks at the
    received dtype; two-pass Pearson (fc/_cpu_core.py:111-137) with the
    sequential (sxy/sqrt(sxx))/sqrt(syy) finalize.

    The rank panels returned with ``return_ranks`` follow the binding's
    diagnostics convention (src/factor_cuda_pybind.cpp:171-176): 0 for cells
    outside the joint set.
    """
    f = np.asarray(f)
    r = np.asarray(r)
    T, N = f.shape
    ok = np.isfinite(f) & np.isfinite(r)
    if factor_mask is not None:
        ok &= np.asarray(factor_mask, dtype=bool)
    if fwd_mask is not None:
        ok &= np.asarray(fwd_mask, dtype=bool)
    kf = canonical_key_f32(f) if f.dtype == np.float32 else canonical_key_f64(f)
    kr = canonical_key_f32(r) if r.dtype == np.float32 else canonical_key_f64(r)
    rf = _rank_rows(kf, ok)
    rr = _rank_rows(kr, ok)
    m = ok.sum(axis=1)
    out = np.full(T, np.nan)
    for t in range(T):
        if m[t] < min_valid or m[t] < 2:
            continue
        o = ok[t]
        if kf[t][o].min() == kf[t][o].max() or kr[t][o].min() == kr[t][o].max():
            continue
        a = rf[t][o].astype(np.float64)
        b = rr[t][o].astype(np.float64)
        a -= a.mean()
        b -= b.mean()
        sxx = float((a * a).sum())
        syy = float((b * b).sum())
        sxy = float((a * b).sum())
        out[t] = (sxy / np.sqrt(sxx)) / np.sqrt(syy)
    if return_ranks:
        return out, rf.astype(np.float64), rr.astype(np.float64)
    return out


# --------------------------------------------------------------------------
# correlations
# --------------------------------------------------------------------------

def in_corr_domain(x, valid):
    """max|x| <= 1e150 and min nonzero |x| >= 1e-150 over valid cells
    (fc/_cpu_core.py:15-41)."""
    xv = np.asarray(x, dtype=np.float64)[valid]
    if xv.size == 0:
        return True
    ax = np.abs(xv)
    if ax.max() > DOMAIN_MAX_ABS:
        return False
    nz = ax[ax != 0.0]
    if nz.size and nz.min() < DOMAIN_MIN_ABS:
        return False
    return True


def _kahan_mean(x):
    """Serial compensated mean (fc/_cpu_core.py:80-96)."""
    s = 0.0
    c = 0.0
    for v in np.asarray(x, dtype=np.float64):
        y = v - c
        t = s + y
        c = (t - s) - y
        s = t
    return s / x.size


def _bias_sensitive(x):
    """|mean| > 1e3 * std (fc/_cpu_core.py:99-108)."""
    return float(abs(x.mean())) > 1e3 * float(x.std())


def two_pass_corr(a, b):
    """Two-pass centred Pearson on an already-joint subset
    (fc/_cpu_core.py:111-137): Kahan mean when bias-sensitive, NaN when a
    centred sum of squares is not positive and finite."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size < 2:
        return float("nan")
    if _bias_sensitive(a) or _bias_sensitive(b):
        am, bm = _kahan_mean(a), _kahan_mean(b)
    else:
        am, bm = a.mean(), b.mean()
    ac = a - am
    bc = b - bm
    sxx = float((ac * ac).sum())
    syy = float((bc * bc).sum())
    sxy = float((ac * bc).sum())
    if not (sxx > 0.0 and syy > 0.0) or not (np.isfinite(sxx) and np.isfinite(syy)):
        return float("nan")
    return float((sxy / np.sqrt(sxx)) / np.sqrt(syy))


def _gram_corr(X64, valid):
    """Masked-GEMM moment sums and uncentred-Gram correlation
    (fc/_cpu_core.py:139-169) plus the cancellation mask
    (fc/_cpu_core.py:171-192) and the |r|>1 sanity flag."""
    M = valid.astype(np.float64)
    Xm = np.where(valid, X64, 0.0)
    n = M.T @ M
    sx = Xm.T @ M
    sy = M.T @ Xm
    sxy = Xm.T @ Xm
    Xsq = Xm * Xm
    sx2 = Xsq.T @ M
    sy2 = M.T @ Xsq
    ns = np.maximum(n, 1.0)
    den = ns - 1.0
    with np.errstate(all="ignore"):
        cov = (sxy - sx * sy / ns) / den
        vx = (sx2 - sx * sx / ns) / den
        vy = (sy2 - sy * sy / ns) / den
        corr = cov / np.sqrt(vx * vy)
        cov_u = sxy - sx * sy / ns
        vx_u = sx2 - sx * sx / ns
        vy_u = sy2 - sy * sy / ns
        fix = ((np.abs(sx * sy / ns) > CANCEL_RATIO * np.abs(cov_u))
               | (np.abs(sx * sx / ns) > CANCEL_RATIO * np.abs(vx_u))
               | (np.abs(sy * sy / ns) > CANCEL_RATIO * np.abs(vy_u)))
        fix |= np.abs(corr) > 1.0
    corr[n < 2] = np.nan
    fix = fix | fix.T
    return corr, fix


def _finish_corr(X64, valid, corr, fix):
    """Fallback of flagged pairs, diagonal rule and bitwise mirror
    (fc/_cpu_core.py:211-230 and :254-269)."""
    P = X64.shape[1]
    for i, j in zip(*np.where(fix)):
        if i >= j:
            continue
        o = valid[:, i] & valid[:, j]
        v = float("nan") if o.sum() < 2 else two_pass_corr(X64[o, i], X64[o, j])
        corr[i, j] = corr[j, i] = v
    for i in range(P):
        o = valid[:, i]
        v = two_pass_corr(X64[o, i], X64[o, i])
        corr[i, i] = 1.0 if np.isfinite(v) else np.nan
    return np.triu(corr) + np.triu(corr, 1).T


def stock_corr(X, mask=None):
    """(N,N) pairwise-complete Pearson over t (fc/_cpu_core.py:194-230)."""
    X64 = np.asarray(X, dtype=np.float64)
    valid = np.isfinite(X64)
    if mask is not None:
        valid &= np.asarray(mask, dtype=bool)
    if not in_corr_domain(X64, valid):
        raise ValueError("corr domain violation: max|x|>1e150 or min nonzero |x|<1e-150")
    corr, fix = _gram_corr(X64, valid)
    return _finish_corr(X64, valid, corr, fix)


def factor_corr(F3, mask=None):
    """(F,F) pooled pairwise-complete Pearson over (t,i) rows
    (fc/_cpu_core.py:232-269)."""
    F3 = np.asarray(F3)
    if F3.ndim != 3:
        raise ValueError("factor_corr input must be 3-D (T,N,F)")
    T, N, F = F3.shape
    X64 = F3.astype(np.float64).reshape(T * N, F)
    valid = np.isfinite(X64)
    if mask is not None:
        valid &= np.asarray(mask, dtype=bool).reshape(-1, 1)
    if not in_corr_domain(X64, valid):
        raise ValueError("corr domain violation: max|x|>1e150 or min nonzero |x|<1e-150")
    corr, fix = _gram_corr(X64, valid)
    return _finish_corr(X64, valid, corr, fix)


def corr_pair(a, b, mask_a=None, mask_b=None):
    """np.corrcoef on the joint finite/mask subset, NaN for n<2
    (tests/fixtures/corr_oracle_v1.py:55-88)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    v = np.isfinite(a) & np.isfinite(b)
    if mask_a is not None:
        v &= np.asarray(mask_a, dtype=bool)
    if mask_b is not None:
        v &= np.asarray(mask_b, dtype=bool)
    a, b = a[v], b[v]
    if a.size < 2:
        return float("nan")
    with np.errstate(all="ignore"):
        return float(np.corrcoef(np.stack([a, b]))[0, 1])
