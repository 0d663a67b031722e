"""Cross-sections wider than one CTA's shared memory (the global-memory rank
path): cs_rank, parameter_scan, rolling_ic and the device rank+IC panel at N
above the shared-memory capacity give the oracle's results bit for bit --
ties, +-0, NaN/inf, masks, empty and constant sections included."""
import numpy as np
import pytest

from conftest import bitwise_f32
from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fcb():
    from fcb200 import _native
    if _native.device_count() < 1:
        pytest.skip("no CUDA device")
    return _native.fcb()


def _panel(rng, T, N, dtype=np.float32):
    x = rng.standard_normal((T, N)).astype(dtype)
    k = rng.random((T, N)) < 0.3
    x[k] = np.round(x[k], 1)                 # many ties
    x[rng.random((T, N)) < 0.03] = np.nan
    x[rng.random((T, N)) < 0.01] = -0.0
    x[rng.random((T, N)) < 0.005] = np.inf
    x[0] = np.nan                            # empty section
    x[1] = 2.5                               # constant section
    m = rng.random((T, N)) < 0.9
    return x, m


def _ic_equal(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and \
        np.array_equal(a[~np.isnan(a)].view(np.uint64), b[~np.isnan(b)].view(np.uint64))


@pytest.mark.parametrize("N", [16385, 40000])
def test_cs_rank_and_scan_wide(fcb, N):
    rng = np.random.default_rng(N)
    x, m = _panel(rng, 5, N)
    for desc in (False, True):
        assert bitwise_f32(fcb.cs_rank_f32(x, m, desc), O.cs_rank(x, m, desc))
        assert bitwise_f32(fcb.cs_rank_f32(x, None, desc), O.cs_rank(x, None, desc))
    res = fcb.parameter_scan_f32(x, m)
    exp = O.parameter_scan(x, m)
    for g in range(4):
        assert bitwise_f32(res["groups"][g], exp[g]), g


@pytest.mark.parametrize("N,fdt,rdt", [(11500, np.float32, np.float32), (9000, np.float64, np.float64),
                                       (20000, np.float32, np.float64), (20000, np.float64, np.float32)])
def test_rolling_ic_wide(fcb, N, fdt, rdt):
    rng = np.random.default_rng(N + 7)
    f, fm = _panel(rng, 6, N, fdt)
    r = (0.2 * np.nan_to_num(f, posinf=0.0) + rng.standard_normal((6, N))).astype(rdt)
    r[rng.random((6, N)) < 0.05] = np.nan
    r[2] = 1.0                               # constant returns section -> NaN IC
    rm = rng.random((6, N)) < 0.95
    ic, rf, rr = fcb.rolling_ic_f64(f, r, fm, rm, 30, return_ranks=True)
    ic_e, rf_e, rr_e = O.rolling_ic(f, r, fm, rm, 30, return_ranks=True)
    assert _ic_equal(ic, ic_e)
    assert np.array_equal(rf, rf_e) and np.array_equal(rr, rr_e)
    assert np.isnan(ic[2]) and np.isnan(ic[0]) and np.isnan(ic[1])


def test_dev_rank_ic_panel_wide():
    import torch
    from fcb200 import _native as nat
    if nat.device_count() < 1:
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(3)
    F, T, N = 3, 4, 18000
    X = rng.standard_normal((F, T, N)).astype(np.float32)
    X[rng.random((F, T, N)) < 0.02] = np.nan
    R = (0.1 * np.nan_to_num(X[0]) + rng.standard_normal((T, N))).astype(np.float32)
    fm = (rng.random((T, N)) < 0.93).astype(np.uint8)
    rm = np.isfinite(R).astype(np.uint8)
    dev = torch.device("cuda")
    dX, dR = torch.from_numpy(X).to(dev), torch.from_numpy(R).to(dev)
    dfm, drm = torch.from_numpy(fm).to(dev), torch.from_numpy(rm).to(dev)
    dranks = torch.empty((F, T, N), dtype=torch.float32, device=dev)
    dic = torch.empty((F, T), dtype=torch.float64, device=dev)
    nat.check(nat.lib().fcb_dev_rank_ic_panel(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T, N,
                                              30, dranks.data_ptr(), dic.data_ptr(), 0,
                                              torch.cuda.current_stream().cuda_stream), "fcb_dev_rank_ic_panel")
    torch.cuda.synchronize()
    ranks, ic = dranks.cpu().numpy(), dic.cpu().numpy()
    for f in range(F):
        assert bitwise_f32(ranks[f], O.cs_rank(X[f], fm.astype(bool)))
        assert _ic_equal(ic[f], O.rolling_ic(X[f], R, fm.astype(bool), rm.astype(bool), 30))
    # the host streaming entry point (workspace scratch) agrees
    hr = np.empty((F, T, N), np.float32)
    hic = np.empty((F, T))
    nat.check(nat.lib().fcb_rank_ic_panel(nat.ptr(X), nat.ptr(R), nat.ptr(fm), nat.ptr(rm), F, T, N, 30,
                                          nat.ptr(hr), nat.ptr(hic), 0, None), "fcb_rank_ic_panel")
    assert bitwise_f32(hr, ranks) and _ic_equal(hic, ic)
