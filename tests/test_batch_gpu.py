"""Batched panels (fcb_batch_*): the persistent, graph-captured rank+IC over
(panel, date) items and the per-panel factor_corr give, for every panel of an
uneven batch, exactly what the single-panel entry points give for it alone --
and the oracle agrees.  Scheduling knobs (and the autotuner that picks them)
change no result."""
import numpy as np
import pytest

from conftest import bitwise_f32, corr_match
from oracle import fc_oracle as O

pytestmark = pytest.mark.gpu

# (T, N, F, pre-listing gap fraction): every block-size class, uneven sizes
SPECS = [(40, 300, 3, 0.1), (25, 3000, 2, 0.2), (60, 5000, 3, 0.0), (30, 9000, 2, 0.1), (20, 10000, 2, 0.05),
         (50, 1200, 4, 0.15), (35, 4096, 2, 0.0), (45, 4097, 2, 0.1)]


@pytest.fixture(scope="module")
def env():
    import torch
    from fcb200 import _native
    if _native.device_count() < 1:
        pytest.skip("no CUDA device")
    return torch, _native


def make_host(rng, T, N, F, gap, dtype):
    X = rng.standard_normal((F, T, N)).astype(dtype)
    start = rng.integers(0, max(1, int(gap * T)), N)
    listed = np.arange(T)[:, None] >= start[None, :]
    X[rng.random((F, T, N)) < 0.01] = np.nan
    X[:, ~listed] = np.nan
    tie = rng.random((F, T, N)) < 0.05
    X[tie] = np.round(X[tie], 2)
    R = (0.05 * np.nan_to_num(X[0]) + rng.standard_normal((T, N))).astype(dtype)
    R[~listed] = np.nan
    return X, R, listed.astype(np.uint8), np.isfinite(R).astype(np.uint8)


def to_panels(torch, host, with_ranks=True):
    dev = torch.device("cuda")
    out = []
    for X, R, fm, rm in host:
        F, T, N = X.shape
        out.append({"X": torch.from_numpy(X).to(dev), "R": torch.from_numpy(R).to(dev),
                    "fmask": torch.from_numpy(fm).to(dev), "rmask": torch.from_numpy(rm).to(dev),
                    "ranks": torch.full((F, T, N), -1.0, dtype=torch.float32, device=dev) if with_ranks else None,
                    "ic": torch.full((F, T), -1.0, dtype=torch.float64, device=dev),
                    "corr": torch.full((F, F), -1.0, dtype=torch.float64, device=dev)})
    return out


def snapshot(panels):
    return [(p["ranks"].cpu().numpy().copy() if p["ranks"] is not None else None, p["ic"].cpu().numpy().copy(),
             p["corr"].cpu().numpy().copy() if p["corr"] is not None else None) for p in panels]


def same_f64(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def single_panel(env, X, R, fm, rm):
    """ranks + IC from fcb_dev_rank_ic_panel, corr from fcb_factor_corr."""
    torch, nat = env
    F, T, N = X.shape
    dev = torch.device("cuda")
    dX, dR = torch.from_numpy(X).to(dev), torch.from_numpy(R).to(dev)
    dfm, drm = torch.from_numpy(fm).to(dev), torch.from_numpy(rm).to(dev)
    dranks = torch.empty((F, T, N), dtype=torch.float32, device=dev)
    dic = torch.empty((F, T), dtype=torch.float64, device=dev)
    nat.check(nat.lib().fcb_dev_rank_ic_panel(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T, N,
                                              30, dranks.data_ptr(), dic.data_ptr(), 0,
                                              torch.cuda.current_stream().cuda_stream), "fcb_dev_rank_ic_panel")
    x3 = np.ascontiguousarray(np.moveaxis(X, 0, -1))
    corr = np.empty((F, F))
    nat.check(nat.lib().fcb_factor_corr(nat.ptr(x3), 0 if X.dtype == np.float32 else 1, nat.ptr(fm), T, N, F,
                                        nat.ptr(corr), None), "fcb_factor_corr")
    torch.cuda.synchronize()
    return dranks.cpu().numpy(), dic.cpu().numpy(), corr


def test_batch_matches_single_panel_paths_and_oracle(env):
    torch, nat = env
    import fcb200
    rng = np.random.default_rng(7)
    host = [make_host(rng, T, N, F, g, np.float32) for T, N, F, g in SPECS]
    panels = to_panels(torch, host)
    b = fcb200.Batch(panels, min_valid=30)
    b.run()
    b.status()
    got = snapshot(panels)
    for k, (X, R, fm, rm) in enumerate(host):
        rk, ic, corr = single_panel(env, X, R, fm, rm)
        assert bitwise_f32(got[k][0], rk), f"panel {k} ranks"
        assert same_f64(got[k][1], ic), f"panel {k} IC"
        assert same_f64(got[k][2], corr), f"panel {k} factor_corr"
    # the oracle on the smallest panels (ranks bit-exact, IC bit-exact, corr <= 1e-12)
    for k in (0, 5):
        X, R, fm, rm = host[k]
        F = X.shape[0]
        for f in range(F):
            assert bitwise_f32(got[k][0][f], O.cs_rank(X[f], fm.astype(bool)))
            ic = O.rolling_ic(X[f], R, fm.astype(bool), rm.astype(bool), min_valid=30)
            assert same_f64(np.nan_to_num(got[k][1][f], nan=7.0), np.nan_to_num(ic, nan=7.0))
        assert corr_match(got[k][2], O.factor_corr(np.moveaxis(X, 0, -1), fm.astype(bool)))


def test_per_panel_arm_and_every_config_agree(env, tmp_path):
    torch, nat = env
    import fcb200
    rng = np.random.default_rng(11)
    host = [make_host(rng, T, N, F, g, np.float32) for T, N, F, g in SPECS[:6]]
    panels = to_panels(torch, host)
    b = fcb200.Batch(panels)
    b.run()
    ref = snapshot(panels)
    configs = [{"concurrent": 1}, {"order": 0}, {"nt_small_max": 1024}, {"ctas_per_sm": 1},
               {"nt_small_max": 2048, "nt_mid_max": 6000, "concurrent": 1}]
    for cfg in configs:
        for p in panels:
            p["ranks"].fill_(-1.0)
            p["ic"].fill_(-1.0)
            p["corr"].fill_(-1.0)
        b.config = cfg
        b.run()
        b.run()   # replay the same graph
        b.status()
        got = snapshot(panels)
        for k in range(len(panels)):
            assert bitwise_f32(got[k][0], ref[k][0]) and same_f64(got[k][1], ref[k][1]) and \
                same_f64(got[k][2], ref[k][2]), (cfg, k)
    for p in panels:
        p["ic"].fill_(-1.0)
    b.run_per_panel()
    b.status()
    got = snapshot(panels)
    for k in range(len(panels)):
        assert bitwise_f32(got[k][0], ref[k][0]) and same_f64(got[k][1], ref[k][1]) and same_f64(got[k][2], ref[k][2])
    # autotune: measures, keeps a valid configuration, changes no result; the
    # cache returns the same choice without measuring
    cache = tmp_path / "tune.txt"
    cfg, ms, cached = b.autotune(reps=2, cache_path=cache)
    assert not cached and ms > 0 and cfg == b.config
    b.run()
    b.status()
    got = snapshot(panels)
    for k in range(len(panels)):
        assert bitwise_f32(got[k][0], ref[k][0]) and same_f64(got[k][1], ref[k][1])
    b2 = fcb200.Batch(panels)
    cfg2, ms2, cached2 = b2.autotune(reps=2, cache_path=cache)
    assert cached2 and cfg2 == cfg
    b2.close()
    b.close()


def test_batch_f64_and_no_rank_output(env):
    torch, nat = env
    import fcb200
    rng = np.random.default_rng(5)
    host = [make_host(rng, T, N, F, g, np.float64) for T, N, F, g in [(30, 700, 2, 0.1), (40, 2500, 3, 0.0),
                                                                      (20, 6000, 2, 0.2)]]
    panels = to_panels(torch, host, with_ranks=False)
    b = fcb200.Batch(panels)
    b.run()
    b.status()
    got = snapshot(panels)
    for k, (X, R, fm, rm) in enumerate(host):
        F = X.shape[0]
        for f in range(F):
            ic = O.rolling_ic(X[f], R, fm.astype(bool), rm.astype(bool), min_valid=30)
            assert same_f64(np.nan_to_num(got[k][1][f], nan=7.0), np.nan_to_num(ic, nan=7.0)), (k, f)
        assert corr_match(got[k][2], O.factor_corr(np.moveaxis(X, 0, -1), fm.astype(bool)))


def test_batch_learned_panels_bit_exact(env):
    """Panels carrying a fitted CDF model take the learned-splitter sort inside
    the persistent kernel; results equal the radix batch bit for bit."""
    torch, nat = env
    import fcb200
    rng = np.random.default_rng(3)
    host = [make_host(rng, T, N, F, g, np.float32) for T, N, F, g in [(300, 5000, 2, 0.0), (280, 2000, 3, 0.1)]]
    panels = to_panels(torch, host)
    plain = fcb200.Batch(panels)
    plain.run()
    plain.status()
    ref = snapshot(panels)
    models = []
    for p in panels:
        F, T, N = p["X"].shape
        m = fcb200.CdfModel(F, seed=1)
        m.fit(p["X"], p["ranks"], T, N, 0, 250, steps=300, lr=3e-3)
        p["model"] = m
        models.append(m)
        p["ranks"].fill_(-1.0)
        p["ic"].fill_(-1.0)
    torch.cuda.synchronize()
    lb = fcb200.Batch(panels)
    lb.run()
    lb.status()
    got = snapshot(panels)
    for k in range(len(panels)):
        assert bitwise_f32(got[k][0], ref[k][0]) and same_f64(got[k][1], ref[k][1])


def test_batched_factor_corr_small_and_large_pools_with_fallback(env):
    """factor_corr of the whole batch runs as one launch per kernel kind.
    Mixed pools -- below 4096 rows (one block per flagged pair), above (the
    row-split fallback), a panel without a corr output -- and a column with a
    large bias that the cancellation gate sends to the fallback: every panel
    equals the single-panel entry point bit for bit and the oracle to 1e-12,
    f32 and f64."""
    torch, nat = env
    import fcb200
    for dt, seed in ((np.float32, 17), (np.float64, 19)):
        rng = np.random.default_rng(seed)
        specs = [(10, 300, 3, 0.1), (40, 2000, 4, 0.0), (12, 200, 5, 0.0), (30, 3000, 3, 0.2), (25, 150, 2, 0.0)]
        host = []
        for T, N, F, g in specs:
            X, R, fm, rm = make_host(rng, T, N, F, g, dt)
            X[F - 1] += dt(1e9)  # large bias: the pair's uncentred sums cancel -> fallback
            host.append((X, R, fm, rm))
        panels = to_panels(torch, host)
        panels[2]["corr"] = None
        b = fcb200.Batch(panels)
        b.run()
        b.status()
        got = snapshot(panels)
        for k, (X, R, fm, rm) in enumerate(host):
            if k == 2:
                continue
            _, _, corr = single_panel(env, X, R, fm, rm)
            assert same_f64(got[k][2], corr), (dt, k)
            assert corr_match(got[k][2], O.factor_corr(np.moveaxis(X, 0, -1), fm.astype(bool))), (dt, k)
        b.close()
