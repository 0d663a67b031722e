"""CUDA-resident inputs: the fc-compatible operators given torch CUDA tensors
run on the tensor's memory through the fcb_dev_* entry points (no host round
trip) and return the same bits as the host route and the oracle.  Ranks and IC
bit-exact; correlations identical to the host route (same kernels) and within
1e-12 of the oracle."""
import numpy as np
import pytest

from conftest import bitwise_f32, corr_match
from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def fc():
    import fcb200
    from fcb200 import _native
    if _native.device_count() < 1 or not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return fcb200


DEV = "cuda:0"


def _panel(T, N, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((T, N)).astype(dtype)
    x[rng.random((T, N)) < 0.05] = 0.0
    k = rng.random((T, N)) < 0.2
    x[k] = np.round(x[k], 1)                      # ties
    x[rng.random((T, N)) < 0.04] = np.nan
    x[rng.random((T, N)) < 0.01] = -0.0
    m = rng.random((T, N)) < 0.9
    return x, m


def _same_bits(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    it = {4: np.uint32, 8: np.uint64}[a.dtype.itemsize]
    return a.shape == b.shape and a.dtype == b.dtype and bool(np.array_equal(a.view(it), b.view(it)))


@pytest.mark.parametrize("T,N", [(37, 1000), (5, 20000)])
@pytest.mark.parametrize("desc", [False, True])
def test_cs_rank_device(fc, T, N, desc):
    x, m = _panel(T, N, N + desc)
    got = fc.cross_sectional_rank(torch.from_numpy(x).to(DEV), torch.from_numpy(m).to(DEV), descending=desc)
    assert isinstance(got, torch.Tensor) and got.device.type == "cuda" and got.dtype == torch.float32
    got = got.cpu().numpy()
    assert bitwise_f32(got, fc.cross_sectional_rank(x, m, descending=desc))
    assert bitwise_f32(got, O.cs_rank(x, m, descending=desc))


def test_cs_rank_device_f64_downcast_and_no_mask(fc):
    x, _ = _panel(9, 777, 5, np.float64)
    got = fc.cross_sectional_rank(torch.from_numpy(x).to(DEV)).cpu().numpy()
    assert bitwise_f32(got, O.cs_rank(x.astype(np.float32)))


@pytest.mark.parametrize("N", [1500, 17000])
def test_parameter_scan_device(fc, N):
    x, m = _panel(11, N, N)
    axes = [("direction", ["ascending", "descending"]), ("mask_mode", ["masked", "unmasked"])]
    got = fc.parameter_scan(axes, torch.from_numpy(x).to(DEV), torch.from_numpy(m).to(DEV))
    ref = fc.parameter_scan(axes, x, m)
    orc = O.parameter_scan(x, m)
    assert got["spec"] == ref["spec"]
    assert got["summary"]["total_groups"] == 4 and got["summary"]["n_failed"] == 0
    order = {("ascending", "masked"): 0, ("ascending", "unmasked"): 1,
             ("descending", "masked"): 2, ("descending", "unmasked"): 3}
    for g, r in zip(got["groups"], ref["groups"]):
        assert g["axis_values"] == r["axis_values"] and g["status"] == "ok"
        assert isinstance(g["result"], np.ndarray)           # results are host numpy
        assert bitwise_f32(g["result"], r["result"])
        k = order[(g["axis_values"]["direction"], g["axis_values"]["mask_mode"])]
        assert bitwise_f32(g["result"], orc[k])
        assert g["time_gpu_ms"] > 0.0


def test_parameter_scan_device_unmasked_only_ignores_mask(fc):
    x, m = _panel(6, 900, 4)
    axes = [("mask_mode", ["unmasked"])]
    got = fc.parameter_scan(axes, torch.from_numpy(x).to(DEV), None)
    assert len(got["groups"]) == 1
    assert bitwise_f32(got["groups"][0]["result"], O.cs_rank(x))


@pytest.mark.parametrize("fdt,rdt,N", [(np.float32, np.float32, 3000), (np.float32, np.float64, 2500),
                                       (np.float64, np.float32, 2000), (np.float64, np.float64, 1800),
                                       (np.float32, np.float32, 14000), (np.float64, np.float64, 9000)])
def test_rolling_ic_device(fc, fdt, rdt, N):
    f, fm = _panel(13, N, N, fdt)
    rng = np.random.default_rng(N + 1)
    r = (0.2 * np.nan_to_num(f.astype(np.float64)) + rng.standard_normal(f.shape)).astype(rdt)
    r[rng.random(f.shape) < 0.03] = np.inf
    rm = rng.random(f.shape) < 0.95
    fm[3, :] = False                                         # an empty date
    got = fc.rolling_ic(torch.from_numpy(f).to(DEV), torch.from_numpy(r).to(DEV),
                        torch.from_numpy(fm).to(DEV), torch.from_numpy(rm).to(DEV), min_valid=30)
    assert isinstance(got, torch.Tensor) and got.device.type == "cuda" and got.dtype == torch.float64
    got = got.cpu().numpy()
    ref = fc.rolling_ic(f, r, fm, rm, min_valid=30)
    assert _same_bits(got, ref)
    orc = O.rolling_ic(f, r, fm, rm, min_valid=30)
    assert np.array_equal(np.isnan(got), np.isnan(orc))
    assert np.isnan(got[3])
    fin = ~np.isnan(orc)
    assert np.allclose(got[fin], orc[fin], rtol=0, atol=1e-12)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_factor_corr_device(fc, dtype):
    rng = np.random.default_rng(21)
    T, N, F = 40, 700, 6
    X = rng.standard_normal((T, N, F)).astype(dtype)
    X[..., 2] = np.exp(X[..., 2]) + 1e3                      # far-from-zero means: the fallback path
    X[rng.random((T, N, F)) < 0.05] = np.nan
    X[..., 5] = 0.25                                         # constant factor -> NaN row / column
    m = rng.random((T, N)) < 0.93
    got = fc.factor_corr(torch.from_numpy(X).to(DEV), torch.from_numpy(m).to(DEV))
    assert isinstance(got, torch.Tensor) and got.device.type == "cuda" and got.dtype == torch.float64
    got = got.cpu().numpy()
    assert _same_bits(got, fc.factor_corr(X, m))
    assert corr_match(got, O.factor_corr(X, m))


def test_factor_corr_device_domain(fc):
    X = np.random.default_rng(2).standard_normal((10, 50, 3))
    X[4, 7, 1] = 1e151
    with pytest.raises(ValueError):
        fc.factor_corr(torch.from_numpy(X).to(DEV))
    m = np.ones((10, 50), bool)
    m[4, 7] = False                                          # the out-of-domain cell is masked out
    got = fc.factor_corr(torch.from_numpy(X).to(DEV), torch.from_numpy(m).to(DEV)).cpu().numpy()
    assert corr_match(got, O.factor_corr(X, m))
    X2 = np.random.default_rng(3).standard_normal((10, 50, 3))
    X2[1, 1, 0] = 1e-151
    with pytest.raises(ValueError):
        fc.factor_corr(torch.from_numpy(X2).to(DEV))
    X2[1, 1, 0] = np.nan                                     # invalid cells are outside the check
    fc.factor_corr(torch.from_numpy(X2).to(DEV))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stock_corr_device(fc, dtype):
    rng = np.random.default_rng(31)
    T, N = 120, 300
    X = (0.02 * rng.standard_t(4, (T, N)) + rng.standard_normal((T, 1)) * 0.01).astype(dtype)
    X[rng.random((T, N)) < 0.03] = np.nan
    X[:, 7] = 1.0                                            # constant column
    m = rng.random((T, N)) < 0.97
    got = fc.stock_corr(torch.from_numpy(X).to(DEV), torch.from_numpy(m).to(DEV))
    assert isinstance(got, torch.Tensor) and got.device.type == "cuda" and got.dtype == torch.float64
    got = got.cpu().numpy()
    assert _same_bits(got, fc.stock_corr(X, m))
    assert corr_match(got, O.stock_corr(X, m))


def test_stock_corr_device_domain(fc):
    X = np.random.default_rng(4).standard_normal((30, 20))
    X[3, 3] = 2e150
    with pytest.raises(ValueError):
        fc.stock_corr(torch.from_numpy(X).to(DEV))


def test_device_inputs_validation(fc):
    x, m = _panel(4, 100, 1)
    dx = torch.from_numpy(x).to(DEV)
    with pytest.raises(ValueError):                          # mask on another device
        fc.cross_sectional_rank(dx, torch.from_numpy(m))
    with pytest.raises(ValueError):                          # non-bool mask
        fc.cross_sectional_rank(dx, torch.from_numpy(m).to(DEV).to(torch.uint8))
    with pytest.raises(ValueError):                          # mask shape
        fc.cross_sectional_rank(dx, torch.from_numpy(m[:2]).to(DEV))
    with pytest.raises(ValueError):                          # dtype whitelist
        fc.cross_sectional_rank(dx.to(torch.float16))
    with pytest.raises(ValueError):                          # ndim
        fc.cross_sectional_rank(dx[0])
    with pytest.raises(ValueError):                          # masked scan needs a mask
        fc.parameter_scan([("mask_mode", ["masked"])], dx, None)
    with pytest.raises(ValueError):
        fc.rolling_ic(dx, dx, min_valid=1)
    with pytest.raises(NotImplementedError):
        fc.rolling_ic(dx, dx, device="cpu")


def test_device_status_after_async_calls(fc):
    """The asynchronous route reports bounded-wait failures through a
    per-device status word; after ordinary calls it reads clear."""
    x, m = _panel(20, 3000, 12)
    dx, dm = torch.from_numpy(x).to(DEV), torch.from_numpy(m).to(DEV)
    fc.cross_sectional_rank(dx, dm)
    fc.rolling_ic(dx, dx * 0.5 + 1.0, dm, None)
    fc.check_device()
    fc.check_device()


def test_bounded_wait_runs_out_and_reports(fc):
    """A wait on a barrier that nothing completes ends after its poll limit
    with FCB_ERR_DEVICE_WAIT (no hang, no fault); the context stays usable:
    a completed wait and an ordinary call succeed right after."""
    from fcb200 import _native as nat
    lib = nat.lib()
    assert lib.fcb_selftest_bounded_wait(0, 2000) == nat.FCB_ERR_DEVICE_WAIT
    assert lib.fcb_selftest_bounded_wait(1, 2000) == 0
    assert lib.fcb_selftest_bounded_wait(0, 0) == -1
    x, m = _panel(5, 700, 3)
    got = fc.cross_sectional_rank(torch.from_numpy(x).to(DEV), torch.from_numpy(m).to(DEV)).cpu().numpy()
    assert bitwise_f32(got, O.cs_rank(x, m))
    fc.check_device()


def test_device_inputs_follow_the_stream(fc):
    """Work is issued on the caller's current stream: a result read on that
    stream after the call sees the finished ranks without a device sync."""
    x, m = _panel(50, 4000, 9)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        dx = torch.from_numpy(x).to(DEV, non_blocking=False)
        dm = torch.from_numpy(m).to(DEV)
        out = fc.cross_sectional_rank(dx * 1.0, dm)      # producer kernel on s, then the rank kernel on s
        host = out.to("cpu", non_blocking=False)
    s.synchronize()
    assert bitwise_f32(host.numpy(), O.cs_rank(x, m))
