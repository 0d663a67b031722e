"""GPU parity at the workload sizes the benchmarks are quoted on, against the
oracle (itself pinned to the reference CPU path by test_oracle_pins.py).

* C1 -- f64, T=250, N=500, F=4: X ~ N(0,1), Y = 0.05 X[...,0] + N(0,1),
  Bernoulli(0.95) mask with NaN on the masked cells; rolling_ic(min_valid=30)
  bitwise and factor_corr (4x4) within 1e-12, through the drop-in modules and
  through the fc-compatible adapter.
* C2 -- f32, 1218 x 5000 x 12 (the bench's panel): cs_rank of all 12 planes
  bitwise; the bench's fused rank + IC step (radix, and learned after a fit on
  dates [0, 250)) bitwise on every (factor, date); all four parameter_scan
  groups of three planes bitwise; factor_corr (12x12) within 1e-12 of the
  oracle's np_factor_corr restatement, on the reference's (T,N,F) layout and
  on the device-resident factor planes, and its BF16x3 tensor-core form
  within 1e-6 of the oracle per output.
* C3 -- stock_corr at N=2000, T=1218: the FP64 drop-in within 1e-12 of the
  oracle's np_stock_corr restatement; the BF16x3 tensor-core form within
  1e-6 and the FP32 form within 5e-5 of the oracle (absolute, per output).
"""
import numpy as np
import pytest

from conftest import bitwise_f32, corr_match
from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def nat():
    from fcb200 import _native
    if _native.device_count() < 1:
        pytest.skip("no CUDA device")
    return _native


def _ic_equal(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and \
        np.array_equal(a[~np.isnan(a)].view(np.uint64), b[~np.isnan(b)].view(np.uint64))


# ------------------------------------------------------------------ C1
def c1_panel(seed=20261201):
    rng = np.random.default_rng(seed)
    T, N, F = 250, 500, 4
    X = rng.standard_normal((T, N, F))
    Y = 0.05 * X[..., 0] + rng.standard_normal((T, N))
    mask = rng.random((T, N)) < 0.95
    X[~mask] = np.nan
    Y[~mask] = np.nan
    return X, Y, mask


def test_c1_rolling_ic_and_factor_corr(nat):
    import fcb200
    X, Y, mask = c1_panel()
    f0 = np.ascontiguousarray(X[..., 0])
    exp_ic = O.rolling_ic(f0, Y, mask, mask, 30)
    assert np.isfinite(exp_ic).sum() > 200
    got = nat.fcb().rolling_ic_f64(f0, Y, mask, mask, 30)
    assert _ic_equal(got, exp_ic)
    assert _ic_equal(fcb200.rolling_ic(f0, Y, mask, mask, min_valid=30), exp_ic)
    exp_c = O.factor_corr(X, mask)
    assert corr_match(nat.fcp().factor_corr_f64(X, mask), exp_c)
    assert corr_match(fcb200.factor_corr(X, mask), exp_c)


# ------------------------------------------------------------------ C2
@pytest.fixture(scope="module")
def c2():
    import bench
    X, R, fm, rm = bench.make_panel()
    return X, R, fm, rm


@pytest.fixture(scope="module")
def c2_oracle(c2):
    X, R, fm, rm = c2
    F = X.shape[0]
    fmb, rmb = fm.astype(bool), rm.astype(bool)
    ranks = [O.cs_rank(X[f], fmb, False) for f in range(F)]
    ics = [O.rolling_ic(X[f], R, fmb, rmb, 30) for f in range(F)]
    return ranks, ics


def _panel_call(nat, dX, dR, dfm, drm, F, T, N, model=None):
    lib = nat.lib()
    dev = dX.device
    ranks = torch.empty((F, T, N), dtype=torch.float32, device=dev)
    ic = torch.empty((F, T), dtype=torch.float64, device=dev)
    st = torch.zeros((F, T, 4), dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    if model is None:
        rc = lib.fcb_dev_rank_ic_panel(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T, N, 30,
                                       ranks.data_ptr(), ic.data_ptr(), 0, s)
    else:
        rc = lib.fcb_dev_rank_ic_panel_learned(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T,
                                               N, 30, ranks.data_ptr(), ic.data_ptr(), model.handle, 64,
                                               st.data_ptr(), s)
    nat.check(rc, "rank_ic_panel")
    torch.cuda.synchronize(dev)
    return ranks, ic, st


def test_c2_cs_rank_all_planes(nat, c2, c2_oracle):
    X, R, fm, rm = c2
    fmb = fm.astype(bool)
    for f in range(X.shape[0]):
        got = nat.fcb().cs_rank_f32(X[f], fmb, False)
        assert bitwise_f32(got, c2_oracle[0][f]), f


def test_c2_rank_ic_step_radix_and_learned(nat, c2, c2_oracle):
    import fcb200
    X, R, fm, rm = c2
    F, T, N = X.shape
    dev = torch.device("cuda", 0)
    dX, dR = torch.from_numpy(X).to(dev), torch.from_numpy(R).to(dev)
    dfm, drm = torch.from_numpy(fm).to(dev), torch.from_numpy(rm).to(dev)
    rk0, ic0, _ = _panel_call(nat, dX, dR, dfm, drm, F, T, N)
    rk0h, ic0h = rk0.cpu().numpy(), ic0.cpu().numpy()
    for f in range(F):
        assert bitwise_f32(rk0h[f], c2_oracle[0][f]), ("radix ranks", f)
        assert _ic_equal(ic0h[f], c2_oracle[1][f]), ("radix IC", f)
    model = fcb200.CdfModel(F, seed=20261203)
    model.fit(dX, rk0, T, N, 0, 250, steps=1500, lr=3e-3)
    rk1, ic1, st = _panel_call(nat, dX, dR, dfm, drm, F, T, N, model=model)
    rk1h, ic1h = rk1.cpu().numpy(), ic1.cpu().numpy()
    for f in range(F):
        assert bitwise_f32(rk1h[f], c2_oracle[0][f]), ("learned ranks", f)
        assert _ic_equal(ic1h[f], c2_oracle[1][f]), ("learned IC", f)
    # the learned buckets served (nearly) every section of the panel
    assert float((st[..., 0] == 1).float().mean()) >= 0.99


def test_c2_parameter_scan_planes(nat, c2):
    X, R, fm, rm = c2
    fmb = fm.astype(bool)
    for f in (0, 6, 9):   # Gaussian, lognormal, Student-t planes
        r = nat.fcb().parameter_scan_f32(X[f], fmb, return_timing=True)
        assert r["group_status"] == [0, 0, 0, 0]
        exp = O.parameter_scan(X[f], fmb)
        for g in range(4):
            assert bitwise_f32(r["groups"][g], exp[g]), (f, g)


def test_c2_factor_corr(nat, c2):
    X, R, fm, rm = c2
    F, T, N = X.shape
    x3 = np.ascontiguousarray(np.moveaxis(X, 0, -1))          # the reference's (T, N, F) layout
    exp = O.factor_corr(x3, fm.astype(bool))
    assert corr_match(nat.fcp().factor_corr_f64(x3, fm.astype(bool)), exp)
    # device-resident factor planes (the bench's factor_corr leg)
    lib = nat.lib()
    dev = torch.device("cuda", 0)
    dX, dfm = torch.from_numpy(X).to(dev), torch.from_numpy(fm).to(dev)
    out = torch.empty((F, F), dtype=torch.float64, device=dev)
    ws = lib.fcb_workspace_create()
    try:
        nat.check(lib.fcb_dev_factor_corr(dX.data_ptr(), 0, dfm.data_ptr(), T, N, F, 1, out.data_ptr(), ws,
                                          torch.cuda.current_stream(dev).cuda_stream), "fcb_dev_factor_corr")
        torch.cuda.synchronize(dev)
        assert corr_match(out.cpu().numpy(), exp)
        # the BF16x3 tensor-core form on the same planes: within 1e-6 per output
        nat.check(lib.fcb_dev_factor_corr_bf16x3(dX.data_ptr(), dfm.data_ptr(), T, N, F, 1, out.data_ptr(), ws,
                                                 torch.cuda.current_stream(dev).cuda_stream),
                  "fcb_dev_factor_corr_bf16x3")
        torch.cuda.synchronize(dev)
        nat.check(lib.fcb_dev_status(), "fcb_dev_status")
    finally:
        lib.fcb_workspace_destroy(ws)
    got = out.cpu().numpy()
    assert np.array_equal(np.isnan(got), np.isnan(exp))
    assert np.nanmax(np.abs(got - exp)) <= 1e-6, np.nanmax(np.abs(got - exp))


# ------------------------------------------------------------------ C3
def test_c3_stock_corr_n2000(nat):
    import bench
    X, mask = bench.make_stock_panel(T=1218, N=2000)
    exp = O.stock_corr(X, mask)
    got = nat.fcb().stock_corr_f64(X, mask)
    assert corr_match(got, exp)
    m8 = mask.astype(np.uint8)
    N = X.shape[1]
    ws = nat.lib().fcb_workspace_create()
    try:
        for mode, tol in ((0, 1e-6), (1, 5e-5)):
            out = np.empty((N, N))
            nat.check(nat.lib().fcb_stock_corr_prec(nat.ptr(X), nat.ptr(m8), X.shape[0], N, mode, nat.ptr(out), ws),
                      "fcb_stock_corr_prec")
            assert np.array_equal(np.isnan(out), np.isnan(exp)), mode
            assert np.nanmax(np.abs(out - exp)) <= tol, (mode, np.nanmax(np.abs(out - exp)))
    finally:
        nat.lib().fcb_workspace_destroy(ws)
