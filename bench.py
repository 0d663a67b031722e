"""Benchmark of the rank + IC hot path (cs_rank + rolling_ic over F factors).

Workload: T=1218 dates x N=5000 stocks x F=12 factors, f32 -- the corpus shape
the reference publishes its numbers on.  Synthetic, seeded: 6 Gaussian, 3
lognormal(sigma=1), 3 Student-t(3) factors; per-stock pre-listing gaps plus 1%
random NaN (~8% missing); 5% of values rounded to 1e-3 (ties); forward returns
0.03*factor0 + t(4) noise.  One step = cs_rank of every factor (ranks written)
plus the daily Spearman IC of every factor against the forward returns.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--method radix|learned]

Prints one JSON line (rank 0).  ``value`` is device-resident throughput
(inputs in HBM, CUDA events on the launching stream, inputs larger than L2
so no flush is needed); ``e2e`` is the same metric through the C ABI host
entry point with pinned host buffers (copies inside the timed region).
With --gpus N (torchrun) every rank runs an independent replica of the
workload on its own GPU ("replicas only": the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG = ROOT / "factor-cuda_b200"
for _p in (str(ROOT), str(PKG)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

T_DEF, N_DEF, F_DEF = 1218, 5000, 12
MIN_VALID = 30
METRIC = "rank+IC Gelem/s @1218x5000x12"


# ---------------------------------------------------------------- workload
def make_panel(T=T_DEF, N=N_DEF, F=F_DEF, seed=20261203):
    """Seeded synthetic stand-in for the 1218x5000x12 corpus panel."""
    rng = np.random.default_rng(seed)
    X = np.empty((F, T, N), np.float32)
    for f in range(F):
        if f < 6:
            X[f] = rng.standard_normal((T, N), dtype=np.float32)
        elif f < 9:
            X[f] = rng.lognormal(0.0, 1.0, (T, N)).astype(np.float32)
        else:
            X[f] = rng.standard_t(3, (T, N)).astype(np.float32)
    start = rng.integers(0, max(1, int(0.14 * T)), N)       # pre-listing gaps (~7%)
    listed = np.arange(T)[:, None] >= start[None, :]
    nan_cells = rng.random((F, T, N)) < 0.01                 # 1% random NaN
    X[nan_cells] = np.nan
    X[:, ~listed] = np.nan
    tie = rng.random((F, T, N)) < 0.05                       # ties
    X[tie] = np.round(X[tie], 3)
    R = (0.03 * np.nan_to_num(X[0]) + rng.standard_t(4, (T, N))).astype(np.float32)
    R[~listed] = np.nan
    fmask = listed.astype(np.uint8)
    rmask = np.isfinite(R).astype(np.uint8)
    return X, R, fmask, rmask


def make_stock_panel(T=1218, N=5000, seed=20261204):
    """Stock returns for the stock_corr precision forms: 0.02 * t(4) noise
    plus a 3-factor Gaussian common component (loadings ~ N(0, 0.5), factor
    returns ~ N(0, 0.01^2)); mask = pre-listing gaps & Bernoulli(0.98)."""
    rng = np.random.default_rng(seed)
    B = rng.normal(0.0, 0.5, (N, 3))
    f = rng.normal(0.0, 0.01, (T, 3))
    X = (0.02 * rng.standard_t(4, (T, N)) + f @ B.T).astype(np.float32)
    start = rng.integers(0, max(1, int(0.1 * T)), N)
    mask = (np.arange(T)[:, None] >= start[None, :]) & (rng.random((T, N)) < 0.98)
    return X, mask


def algorithmic_bytes(F, T, N):
    """Bytes one launch must move: factor read + rank write (4+4 B/cell),
    returns + two masks per (t,i) (4+1+1 B), IC out (8 B per (f,t))."""
    return F * T * N * 8 + T * N * 6 + F * T * 8


# ---------------------------------------------------------------- helpers
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.idx)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU legs
def _cpu_work(args):
    import sys as _s
    _s.path.insert(0, str(ROOT))
    from oracle import fc_oracle as O
    X, R, fm, rm = args
    t0 = time.perf_counter()
    for f in range(X.shape[0]):
        O.cs_rank(X[f], fm.astype(bool), False)
        O.rolling_ic(X[f], R, fm.astype(bool), rm.astype(bool), MIN_VALID)
    return time.perf_counter() - t0


def cpu_baseline(X, R, fm, rm, budget_s=12.0, procs=1):
    """Oracle port timed on a bounded sample of dates (all factors)."""
    F, T, N = X.shape
    per = 16
    chunks = []
    for t0 in range(0, T, per):
        chunks.append((X[:, t0:t0 + per], R[t0:t0 + per], fm[t0:t0 + per], rm[t0:t0 + per]))
    done_cells = 0
    t_start = time.perf_counter()
    if procs <= 1:
        for c in chunks:
            _cpu_work(c)
            done_cells += c[0].size
            if time.perf_counter() - t_start > budget_s:
                break
        el = time.perf_counter() - t_start
    else:
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        n = 0
        with ctx.Pool(procs) as pool:
            t_start = time.perf_counter()
            while time.perf_counter() - t_start < budget_s and n < len(chunks):
                batch = chunks[n:n + procs]
                pool.map(_cpu_work, batch)
                done_cells += sum(c[0].size for c in batch)
                n += len(batch)
            el = time.perf_counter() - t_start
    dates = done_cells // (F * N)
    return done_cells / el / 1e9, el, dates


# ---------------------------------------------------------------- GPU legs
def run_b200(args, rank, world):
    import torch
    from fcb200 import _native as nat

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = nat.lib()
    X, R, fm, rm = make_panel(T=args.T, N=args.N, F=args.F, seed=20261203 + rank)
    F, T, N = X.shape
    method = {"radix": 0, "learned": 1}[args.method]
    dX = torch.from_numpy(X).to(dev)
    dR = torch.from_numpy(R).to(dev)
    dfm = torch.from_numpy(fm).to(dev)
    drm = torch.from_numpy(rm).to(dev)
    dranks = torch.empty((F, T, N), dtype=torch.float32, device=dev)
    dic = torch.empty((F, T), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def radix_step():
        rc = lib.fcb_dev_rank_ic_panel(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T, N,
                                       MIN_VALID, dranks.data_ptr(), dic.data_ptr(), 0, stream.cuda_stream)
        nat.check(rc, "fcb_dev_rank_ic_panel")

    learn = None
    if method == 1:
        import fcb200
        # exact radix ranks of the earlier dates are the training labels
        radix_step()
        torch.cuda.synchronize(dev)
        model = fcb200.CdfModel(F, seed=20261203)
        tfit = min(T, 250)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        model.fit(dX, dranks, T, N, 0, tfit, steps=1500, lr=3e-3, stream=stream.cuda_stream)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        dstats = torch.zeros((F, T, 4), dtype=torch.int32, device=dev)
        learn = {"model": model, "fit_ms": f0.elapsed_time(f1), "train_dates": tfit, "stats": dstats}

    def step():
        if learn is None:
            radix_step()
            return
        rc = lib.fcb_dev_rank_ic_panel_learned(dX.data_ptr(), dR.data_ptr(), dfm.data_ptr(), drm.data_ptr(), F, T,
                                               N, MIN_VALID, dranks.data_ptr(), dic.data_ptr(),
                                               learn["model"].handle, 64, learn["stats"].data_ptr(),
                                               stream.cuda_stream)
        nat.check(rc, "fcb_dev_rank_ic_panel_learned")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        # keep the GPU loaded for ~1 s before the timed region so that the
        # 200 ms clock samples bracket it (extra untimed warm-up steps)
        t_pre = time.perf_counter()
        while time.perf_counter() - t_pre < 1.0:
            for _ in range(5):
                step()
            torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    # parity spot check of the timed outputs against the oracle (a few dates)
    spot = check_spot(X, R, fm, rm, dranks, dic)
    learned_info = None
    if learn is not None:
        st = learn["stats"].cpu().numpy()
        codes = st[..., 0]
        # bit-exactness of the whole learned output against the radix path
        lr_ranks = dranks.clone()
        lr_ic = dic.clone()
        radix_step()
        torch.cuda.synchronize(dev)
        exact = bool(torch.equal(lr_ranks.view(torch.int32), dranks.view(torch.int32))) and \
            bool(torch.equal(torch.nan_to_num(lr_ic, nan=7.0), torch.nan_to_num(dic, nan=7.0)))
        # learned vs radix under the same conditions: alternating windows of
        # max(K, 20) steps each, three rounds, medians (the headline `value`
        # above is the contract's K-step measurement)
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        n_cmp = max(args.steps, 20)

        def window(fn):
            torch.cuda.synchronize(dev)
            e2.record(stream)
            for _ in range(n_cmp):
                fn()
            e3.record(stream)
            torch.cuda.synchronize(dev)
            return e2.elapsed_time(e3) / n_cmp

        rounds = [(window(step), window(radix_step)) for _ in range(3)]
        learned_ms_cmp = sorted(r[0] for r in rounds)[1]
        radix_ms = sorted(r[1] for r in rounds)[1]
        learned_info = {"fit_ms": learn["fit_ms"], "train_dates": learn["train_dates"],
                        "learned_fraction": float((codes == 1).mean()),
                        "fallback_overflow": float((codes == 2).mean()),
                        "fallback_judge": float((codes == 3).mean()),
                        "fallback_scale": float((codes == 4).mean()),
                        "mean_max_bucket": float(st[..., 1][codes == 1].mean()) if (codes == 1).any() else None,
                        "bit_exact_vs_radix": exact, "radix_ms_per_step": radix_ms,
                        "learned_ms_per_step_paired": learned_ms_cmp,
                        "comparison": f"median of 3 alternating windows of {n_cmp} steps each",
                        "speedup_vs_radix": radix_ms / learned_ms_cmp}

    # e2e: host entry point, pinned buffers, copies in the timed region
    if args.no_e2e:
        res = finish(args, world, X, R, fm, rm, ms, None, None, clk, spot, dev, learned_info)
        res["factor_corr"] = bench_factor_corr(dX, dfm, X, fm, dev, steps=max(3, args.steps // 2))
        res["c2_stages"] = bench_c2_stages(dX, X, fm, dev, ms, res["factor_corr"]["ms"])
        return res
    hX = torch.from_numpy(X).pin_memory()
    hR = torch.from_numpy(R).pin_memory()
    hfm = torch.from_numpy(fm).pin_memory()
    hrm = torch.from_numpy(rm).pin_memory()
    hranks = torch.empty((F, T, N), dtype=torch.float32).pin_memory()
    hic = torch.empty((F, T), dtype=torch.float64).pin_memory()
    ws = lib.fcb_workspace_create()

    def host_step():
        rc = lib.fcb_rank_ic_panel(hX.data_ptr(), hR.data_ptr(), hfm.data_ptr(), hrm.data_ptr(), F, T, N,
                                   MIN_VALID, hranks.data_ptr(), hic.data_ptr(), method, ws)
        nat.check(rc, "fcb_rank_ic_panel")

    for _ in range(max(1, args.warmup)):
        host_step()
    if method == 1:
        # let the workspace's background fit land before timing (bounded)
        import ctypes as C
        rdy, fits, lch = C.c_int(), C.c_int(), C.c_int()
        for _ in range(5):
            lib.fcb_workspace_learned_state(ws, C.byref(rdy), C.byref(fits), C.byref(lch))
            if rdy.value:
                break
            host_step()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    lib.fcb_workspace_destroy(ws)
    e2e_ok = bool(np.array_equal(hranks.numpy().view(np.uint32), dranks.cpu().numpy().view(np.uint32)))
    res = finish(args, world, X, R, fm, rm, ms, e2e_s, e2e_ok, clk, spot, dev, learned_info)
    res["factor_corr"] = bench_factor_corr(dX, dfm, X, fm, dev, steps=max(3, args.steps // 2))
    res["c2_stages"] = bench_c2_stages(dX, X, fm, dev, ms, res["factor_corr"]["ms"])
    return res


# DRAM bytes of one rank + IC step per date at N=5000, F=12 (k_ric_returns +
# k_rank_ic_item), from one ncu capture each at T=600
# (profiles/k_rank_ic_item_T600_N5000_F12.md): dram__bytes_read.sum +
# dram__bytes_write.sum.  Traffic grows with the number of dates at fixed N
# and F, so the bench's step is that times T.
TRAFFIC_PER_DATE = {"learned": (153.391360e6 + 103.361792e6 + 18.050048e6) / 600,
                    "radix": (153.914368e6 + 102.658048e6 + 18.050048e6) / 600}


def max_over_ranks(values, device):
    """Element-wise maximum of a list of floats over every rank of the process
    group: a replica job is as slow as its slowest rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_throughput(world, cells_per_rank, ms_max):
    """Whole-job Gelem/s of `world` replicas, each ranking `cells_per_rank`
    cells, timed by the slowest rank."""
    return world * cells_per_rank / (ms_max / 1e3) / 1e9


def finish(args, world, X, R, fm, rm, ms, e2e_s, e2e_ok, clk, spot, dev, learned_info=None):
    F, T, N = X.shape
    ms_all, e2e_all = ms, (e2e_s if e2e_s is not None else 0.0)
    if world > 1:
        ms_all, e2e_all = max_over_ranks([ms, e2e_all], dev)
    cells = F * T * N
    peak, peak_kind = measured_peaks()
    bytes_launch = algorithmic_bytes(F, T, N)
    achieved = bytes_launch / (ms / 1e3) / 1e9
    traffic = TRAFFIC_PER_DATE[args.method] * T if (N, F) == (5000, 12) else None
    res = {
        "metric": METRIC, "value": job_throughput(world, cells, ms_all), "unit": "Gelem/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_all,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded stand-in for the 1218x5000x12 corpus panel)",
        "config": {"workload": "cs_rank + rolling_ic(min_valid=30), F=12 factor panels vs one "
                               "forward-return panel", "T": T, "N": N, "F": F, "method": args.method,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs (292 MB factors) larger than the 126 MB L2; no flush"},
        "e2e": None if e2e_s is None else {"value": world * cells / e2e_all / 1e9, "unit": "Gelem/s",
                "h2d_bytes_per_step": int(X.nbytes + R.nbytes + fm.nbytes + rm.nbytes),
                "d2h_bytes_per_step": int(F * T * N * 4 + F * T * 8),
                "api": "fcb_rank_ic_panel (C ABI, pinned host buffers, date-chunked streaming)",
                "matches_device_path": e2e_ok},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "traffic_source": "ncu dram bytes at T=600 scaled by T/600" if traffic else None,
                     "kernel": "k_ric_returns + k_rank_ic_item", "algorithmic_bytes_per_launch": bytes_launch},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "parity_spot_check": spot,
    }
    if learned_info is not None:
        res["learned"] = learned_info
    return res


def bench_factor_corr(dX, dfm, X, fm, dev, steps=5, warmup=2):
    """factor_corr of the C2 panel (F factors pooled over the T*N (t, i) rows,
    factor mask broadcast per column), device-resident factor planes, through
    fcb_dev_factor_corr; spot-checked against the host entry point on the
    reference's (T,N,F) layout."""
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    F, T, N = X.shape
    ws = lib.fcb_workspace_create()
    out = torch.empty((F, F), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def run():
        nat.check(lib.fcb_dev_factor_corr(dX.data_ptr(), 0, dfm.data_ptr(), T, N, F, 1, out.data_ptr(), ws,
                                          stream.cuda_stream), "fcb_dev_factor_corr")

    for _ in range(warmup):
        run()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        run()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    got = out.cpu().numpy()
    ref = np.empty((F, F))
    x3 = np.ascontiguousarray(np.moveaxis(X, 0, -1))
    nat.check(lib.fcb_factor_corr(nat.ptr(x3), 0, nat.ptr(fm), T, N, F, nat.ptr(ref), None), "fcb_factor_corr")
    lib.fcb_workspace_destroy(ws)
    rows = T * N
    alg_bytes = rows * (4 * F + 1)
    peak, _ = measured_peaks()
    same = bool(np.array_equal(np.isnan(got), np.isnan(ref)) and
                np.nanmax(np.abs(np.nan_to_num(got) - np.nan_to_num(ref))) <= 1e-12)
    return {"workload": f"factor_corr {F}x{F} over {rows} (t,i) rows, f32 factor planes, factor mask",
            "ms": ms, "rows_per_s": rows / (ms / 1e3), "algorithmic_gb_s": alg_bytes / (ms / 1e3) / 1e9,
            "hbm_frac": alg_bytes / (ms / 1e3) / 1e9 / peak, "matches_host_entry_point": same}


def bench_c2_stages(dX, X, fm, dev, rank_ic_ms, factor_corr_ms, steps=3):
    """The C2 pipeline stage by stage on the same panel: cs_rank of every factor
    plane (device entry point, CUDA events), parameter_scan (4 groups) of every
    plane (its own device timing, host buffers), and the fused rank + IC and
    factor_corr legs measured above -- the counterpart of the reference's
    parameter_scan -> rolling_ic -> factor_corr pipeline figure."""
    import ctypes as C
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    F, T, N = X.shape
    dfm = torch.from_numpy(fm).to(dev)
    out = torch.empty((T, N), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def cs_all():
        for f in range(F):
            nat.check(lib.fcb_dev_cs_rank_f32(dX[f].data_ptr(), dfm.data_ptr(), T, N, 0, out.data_ptr(),
                                              stream.cuda_stream), "fcb_dev_cs_rank_f32")

    cs_all()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        cs_all()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    cs_ms = e0.elapsed_time(e1) / steps
    # parameter_scan: device time of the fused four-group pass per plane
    outs = [np.empty((T, N), np.float32) for _ in range(4)]
    optr = (C.c_void_p * 4)(*[nat.ptr(o) for o in outs])
    st = (C.c_int * 4)()
    tg = (C.c_float * 4)()
    ws = lib.fcb_workspace_create()
    scan_ms = []
    for _ in range(2):
        tot = 0.0
        for f in range(F):
            xf = np.ascontiguousarray(X[f])
            nat.check(lib.fcb_parameter_scan_f32(nat.ptr(xf), nat.ptr(fm), T, N, optr, st, None, tg, None, ws),
                      "fcb_parameter_scan_f32")
            tot += sum(float(v) for v in tg)
        scan_ms.append(tot)
    lib.fcb_workspace_destroy(ws)
    scan = min(scan_ms)
    return {"workload": f"C2 stages on {F} factor planes of {T}x{N}",
            "cs_rank_ms_all_planes": cs_ms, "parameter_scan_ms_all_planes": scan,
            "rank_ic_ms_all_planes": rank_ic_ms, "factor_corr_ms": factor_corr_ms,
            "pipeline_ms": scan + rank_ic_ms + factor_corr_ms,
            "pipeline": "parameter_scan (4 groups) + cs_rank/rolling_ic (fused, learned) + factor_corr, "
                        "device-resident kernels"}


def make_batch_panels(dev, n=64, F=8, seed=20261205):
    """Seeded uneven panels for the batched path, generated on the device:
    N ~ U[300, 6000], T ~ U[250, 2500]; half the factors Gaussian, half
    lognormal(sigma=1); per-panel missing rate q ~ U[0, 0.2] as per-stock
    pre-listing gaps (start date ~ U[0, 2qT)); returns = 0.03 * factor 0 +
    N(0, 1) noise."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    nan = float("nan")
    panels = []
    for _ in range(n):
        N = int(rng.integers(300, 6001))
        T = int(rng.integers(250, 2501))
        q = float(rng.uniform(0.0, 0.2))
        X = torch.randn((F, T, N), generator=g, device=dev, dtype=torch.float32)
        X[F // 2:].exp_()
        start = torch.from_numpy(rng.integers(0, max(1, int(2 * q * T)), N)).to(dev)
        listed = torch.arange(T, device=dev)[:, None] >= start[None, :]
        X.masked_fill_(~listed[None], nan)
        R = 0.03 * torch.nan_to_num(X[0]) + torch.randn((T, N), generator=g, device=dev, dtype=torch.float32)
        R.masked_fill_(~listed, nan)
        panels.append({"X": X, "R": R, "fmask": listed.to(torch.uint8), "rmask": torch.isfinite(R).to(torch.uint8),
                       "ranks": torch.empty((F, T, N), dtype=torch.float32, device=dev),
                       "ic": torch.empty((F, T), dtype=torch.float64, device=dev),
                       "corr": torch.empty((F, F), dtype=torch.float64, device=dev)})
    return panels


def bench_batch(dev, steps=5, warmup=2, tune_cache=None):
    """Batched uneven panels: one autotuned CUDA-graph replay of the
    persistent rank+IC kernels + per-panel factor_corr, against the same work
    issued one panel at a time.  Device-resident inputs (8.8 GB of factors,
    far above L2)."""
    import torch
    import fcb200
    panels = make_batch_panels(dev)
    cells = sum(int(p["X"].numel()) for p in panels)
    torch.cuda.synchronize(dev)
    b = fcb200.Batch(panels, min_valid=MIN_VALID)
    t0 = time.perf_counter()
    # with a cache file, a second run takes the tuned configuration without
    # measuring alternatives (so a profiler sees only the timed launches)
    cfg, tuned_ms, cached = b.autotune(reps=2, cache_path=tune_cache)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    ms_graph = timed(b.run)
    b.status()
    ic_g = [p["ic"].clone() for p in panels]
    corr_g = [p["corr"].clone() for p in panels]
    rk_g = [p["ranks"][:, :3].clone() for p in panels]
    ms_pp = timed(b.run_per_panel)
    b.status()
    same = all(torch.equal(torch.nan_to_num(a, nan=7.0), torch.nan_to_num(p["ic"], nan=7.0)) and
               torch.equal(torch.nan_to_num(c, nan=7.0), torch.nan_to_num(p["corr"], nan=7.0)) and
               torch.equal(r.view(torch.int32), p["ranks"][:, :3].view(torch.int32))
               for a, c, r, p in zip(ic_g, corr_g, rk_g, panels))
    classes = sorted({0 if p["X"].shape[2] <= cfg["nt_small_max"] else (1 if p["X"].shape[2] <= cfg["nt_mid_max"]
                                                                           else 2) for p in panels})
    res = {"workload": "64 uneven panels (N ~ U[300,6000], T ~ U[250,2500], F=8, gaps ~ U[0,0.2]): "
                       "cs_rank + rolling_ic(30) + factor_corr per panel",
           "cells": cells, "unit": "Gelem/s",
           # kernels: one persistent rank + IC kernel per size class; per panel, factor_corr's
           # column pass + merge, Gram + finalize and the four fallback kernels (launched for
           # every pool of 4096 rows or more; they exit at once when no pair is flagged); the
           # per-panel arm ranks through the returns kernel + per-(date, factor) kernel (F >= 2)
           "graph": {"ms": ms_graph, "value": cells / (ms_graph / 1e3) / 1e9,
                     "kernels_per_replay": len(classes) + 8 * len(panels)},
           "per_panel": {"ms": ms_pp, "value": cells / (ms_pp / 1e3) / 1e9,
                         "kernels_per_step": sum((2 if p["X"].shape[0] >= 2 else 1) + 8 for p in panels)},
           "speedup_graph_vs_per_panel": ms_pp / ms_graph,
           "bit_exact_graph_vs_per_panel": bool(same),
           "autotune": {"config": cfg, "tuned_ms": tuned_ms, "tuning_s": tune_s, "from_cache": cached}}
    b.close()
    del panels
    torch.cuda.empty_cache()
    return res


def make_c5_block(dev, g, rng, state, F, Tb, N, start):
    """One block of Tb dates of the learned-splitter streaming panel, on the
    device.  Per factor: AR(1) (phi = 0.98) drift of the mean and of the log
    scale; 70 % of the factors Gaussian, 30 % lognormal(sigma = 0.8); 0.5 %
    exact duplicates (a cell copies another cell of the same date); stocks
    missing before a per-stock listing date (10 % of cells on average).
    `state` carries the drifts from block to block."""
    import torch
    nan = float("nan")
    t_idx = torch.arange(start, start + Tb, device=dev)
    mu = torch.empty((F, Tb), device=dev)
    ls = torch.empty((F, Tb), device=dev)
    m, l = state[0], state[1]
    for t in range(Tb):
        m = 0.98 * m + 0.05 * torch.randn(F, generator=g, device=dev)
        l = 0.98 * l + 0.05 * torch.randn(F, generator=g, device=dev)
        mu[:, t] = m
        ls[:, t] = l
    state[0], state[1] = m, l
    base = torch.randn((F, Tb, N), generator=g, device=dev)
    nlog = int(round(0.3 * F))
    base[F - nlog:] = torch.exp(0.8 * base[F - nlog:])
    X = (mu[:, :, None] + torch.exp(ls)[:, :, None] * base).float()
    dup = torch.rand((F, Tb, N), generator=g, device=dev) < 0.005
    src = torch.randint(0, N, (F, Tb, N), generator=g, device=dev)
    X = torch.where(dup, torch.gather(X, 2, src), X)
    listed = t_idx[:, None] >= state[2][None, :]
    X.masked_fill_(~listed[None], nan)
    R = 0.03 * torch.nan_to_num(X[0]) + torch.randn((Tb, N), generator=g, device=dev)
    R.masked_fill_(~listed, nan)
    return X.contiguous(), R.float().contiguous(), listed.to(torch.uint8), torch.isfinite(R).to(torch.uint8)


def bench_c5(dev, T=5000, N=8000, F=128, Tb=250, seed=20261206):
    """Learned splitters on the streaming configuration (T=5000, N=8000,
    F=128: 5.12 G cells, 20.5 GB of f32 factors, device-resident in blocks of
    250 dates).  The CDF networks are fitted on the exact ranks of dates
    [0, 500) and refitted on every later block's ranks before the next block;
    every block is ranked by the learned path and by the plain radix path, and
    the two outputs are compared bit for bit."""
    import torch
    import fcb200
    from fcb200 import _native as nat
    lib = nat.lib()
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    state = [torch.zeros(F, device=dev), torch.zeros(F, device=dev),
             torch.from_numpy(rng.integers(0, int(0.2 * T), N)).to(dev)]
    blocks = [make_c5_block(dev, g, rng, state, F, Tb, N, b * Tb) for b in range(T // Tb)]
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    ranks_r = torch.empty((F, Tb, N), dtype=torch.float32, device=dev)
    ranks_l = torch.empty_like(ranks_r)
    ic_r = torch.empty((F, Tb), dtype=torch.float64, device=dev)
    ic_l = torch.empty_like(ic_r)
    stats = torch.zeros((F, Tb, 4), dtype=torch.int32, device=dev)
    model = fcb200.CdfModel(F, seed=seed)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    t_radix = t_radix_lb = t_learn = t_fit = 0.0
    exact = True
    codes = []
    learned_cells = 0
    for b, (X, R, fm, rm) in enumerate(blocks):
        ev[0].record(stream)
        nat.check(lib.fcb_dev_rank_ic_panel(X.data_ptr(), R.data_ptr(), fm.data_ptr(), rm.data_ptr(), F, Tb, N,
                                            MIN_VALID, ranks_r.data_ptr(), ic_r.data_ptr(), 0, s), "radix")
        ev[1].record(stream)
        if b >= 2:
            nat.check(lib.fcb_dev_rank_ic_panel_learned(X.data_ptr(), R.data_ptr(), fm.data_ptr(), rm.data_ptr(), F,
                                                        Tb, N, MIN_VALID, ranks_l.data_ptr(), ic_l.data_ptr(),
                                                        model.handle, 64, stats.data_ptr(), s), "learned")
        ev[2].record(stream)
        # fit on the exact ranks of this block: dates [0, 500) first, then a refit per block
        if b == 0:
            model.fit(X, ranks_r, Tb, N, 0, Tb, steps=1500, lr=3e-3, stream=s)
        else:
            model.fit(X, ranks_r, Tb, N, 0, Tb, steps=300 if b == 1 else 100, lr=1e-3, stream=s)
        ev[3].record(stream)
        torch.cuda.synchronize(dev)
        t_radix += ev[0].elapsed_time(ev[1])
        t_fit += ev[2].elapsed_time(ev[3])
        if b >= 2:
            t_learn += ev[1].elapsed_time(ev[2])
            t_radix_lb += ev[0].elapsed_time(ev[1])
            learned_cells += F * Tb * N
            exact = exact and bool(torch.equal(ranks_l.view(torch.int32), ranks_r.view(torch.int32))) and \
                bool(torch.equal(torch.nan_to_num(ic_l, nan=7.0), torch.nan_to_num(ic_r, nan=7.0)))
            codes.append(stats[..., 0].flatten().cpu().numpy())
    codes = np.concatenate(codes)
    res = {"workload": f"learned splitters, streaming: T={T}, N={N}, F={F} ({F * T * N / 1e9:.2f} G cells, "
                       f"{F * T * N * 4 / 1e9:.1f} GB f32), blocks of {Tb} dates; fit on dates [0, {2 * Tb}), "
                       f"refit after every block",
           "learned_gelem_s": learned_cells / (t_learn / 1e3) / 1e9,
           "radix_gelem_s": F * T * N / (t_radix / 1e3) / 1e9,
           "speedup_vs_radix": (t_radix_lb / t_learn) if t_learn > 0 else None,
           "learned_fraction": float((codes == 1).mean()),
           "fallback_overflow": float((codes == 2).mean()), "fallback_judge": float((codes == 3).mean()),
           "fallback_scale": float((codes == 4).mean()),
           "bit_exact_vs_radix": exact, "fit_ms_total": t_fit,
           "cells_ranked_learned": learned_cells}
    del blocks
    torch.cuda.empty_cache()
    return res


def bench_stock_corr(dev, N, T=1218, steps=5, warmup=2):
    """stock_corr precision forms on one (T,N) panel, device-resident:
    BF16x3 tensor-core path vs plain FP32, error against the f64 path."""
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    X, mask = make_stock_panel(T=T, N=N)
    m8 = mask.astype(np.uint8)
    ref = np.empty((N, N))
    nat.check(lib.fcb_stock_corr(nat.ptr(X), 0, nat.ptr(m8), T, N, nat.ptr(ref), None, None), "fcb_stock_corr")
    dX = torch.from_numpy(X).to(dev)
    dM = torch.from_numpy(m8).to(dev)
    dO = torch.empty((N, N), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ws = lib.fcb_workspace_create()
    alg_flops = 4 * 2.0 * N * N * T           # X.X^T, X.M^T, X^2.M^T, M.M^T (dense-equivalent)
    Tp = (T + 31) // 32 * 32
    n_i = (N + 127) // 128
    tiles = sum(1 for ti in range(n_i) for tj in range((N + 31) // 32) if tj * 32 + 31 >= ti * 128)
    exec_flops = tiles * (Tp // 16) * 2.0 * 128 * 704 * 16   # issued MMA work (N-total 704 per 16 dates)
    res = {"N": N, "T": T, "algorithmic_gflop": alg_flops / 1e9}
    out = {}
    for name, mode in (("bf16x3", 0), ("fp32", 1)):
        def call():
            nat.check(lib.fcb_dev_stock_corr_prec(dX.data_ptr(), dM.data_ptr(), T, N, mode, dO.data_ptr(), ws,
                                                  stream.cuda_stream), "fcb_dev_stock_corr_prec")
        for _ in range(warmup):
            call()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        got = dO.cpu().numpy()
        err = np.abs(got - ref)
        same_nan = bool(np.array_equal(np.isnan(got), np.isnan(ref)))
        d = {"ms": ms, "tflops_algorithmic": alg_flops / (ms / 1e3) / 1e12,
             "max_abs_err_vs_f64": float(np.nanmax(err)), "mean_abs_err_vs_f64": float(np.nanmean(err)),
             "nan_pattern_matches": same_nan}
        if mode == 0:
            d["tflops_mma_issued"] = exec_flops / (ms / 1e3) / 1e12
        out[name] = d
    lib.fcb_workspace_destroy(ws)
    res.update(out)
    res["bf16x3_speedup_vs_fp32"] = out["fp32"]["ms"] / out["bf16x3"]["ms"]
    return res


def check_spot(X, R, fm, rm, dranks, dic):
    from oracle import fc_oracle as O
    F, T, N = X.shape
    ts = [0, T // 2, T - 1]
    ok = True
    for f in (0, F - 1):
        sl = slice(ts[1], ts[1] + 2)
        exp_r = O.cs_rank(X[f, sl], fm[sl].astype(bool), False)
        got_r = dranks[f, sl].cpu().numpy()
        ok &= bool(np.array_equal(exp_r.view(np.uint32), got_r.view(np.uint32)))
        exp_ic = O.rolling_ic(X[f, sl], R[sl], fm[sl].astype(bool), rm[sl].astype(bool), MIN_VALID)
        got_ic = dic[f, sl].cpu().numpy()
        ok &= bool(np.array_equal(np.nan_to_num(exp_ic, nan=7.0), np.nan_to_num(got_ic, nan=7.0)))
    return "bit-exact" if ok else "MISMATCH"


def run_reference(args):
    """The reference arm: the oracle port of the reference CPU path
    (fc/_cpu_core.py np_cs_rank + np_rolling_ic) on the host cores."""
    X, R, fm, rm = make_panel()
    F, T, N = X.shape
    procs = max(1, min(os.cpu_count() or 1, 32))
    for _ in range(args.warmup):
        cpu_baseline(X, R, fm, rm, budget_s=1.0, procs=1)
    vals = []
    els = []
    for _ in range(args.steps):
        v, el, dates = cpu_baseline(X, R, fm, rm, budget_s=6.0, procs=procs)
        vals.append(v)
        els.append(el)
    v = statistics.median(vals)
    return {
        "metric": METRIC, "value": v, "unit": "Gelem/s", "impl": "reference", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(els) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded stand-in for the 1218x5000x12 corpus panel)",
        "config": {"workload": "cs_rank + rolling_ic(min_valid=30), F=12 factor panels vs one "
                               "forward-return panel", "T": T, "N": N, "F": F},
        "cpu_baseline": {"value": v, "unit": "Gelem/s", "cores": procs, "kind": "port",
                         "sample": "16-date chunks of all 12 factors, ~6 s per step, spawn pool"},
        "e2e": {"value": v, "unit": "Gelem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--method", choices=["radix", "learned"], default="learned")
    ap.add_argument("--no-stock-corr", action="store_true", help="skip the stock_corr precision-form leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--only-stock-corr", type=int, default=0, metavar="N",
                    help="run only the stock_corr precision leg at this N (profiling)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven-panel leg")
    ap.add_argument("--only-batch", action="store_true", help="run only the batched uneven-panel leg")
    ap.add_argument("--batch-tune-cache", default=None, metavar="PATH",
                    help="autotuner cache file for the batch leg (a hit skips the tuning replays)")
    ap.add_argument("--no-c5", action="store_true", help="skip the learned-splitter streaming leg")
    ap.add_argument("--only-c5", action="store_true",
                    help="run only the learned-splitter streaming leg (T=5000, N=8000, F=128)")
    ap.add_argument("--T", type=int, default=T_DEF)
    ap.add_argument("--N", type=int, default=N_DEF)
    ap.add_argument("--F", type=int, default=F_DEF)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.only_stock_corr:
        import torch
        print(json.dumps(bench_stock_corr(torch.device("cuda", 0), args.only_stock_corr, steps=args.steps,
                                          warmup=args.warmup)))
        return
    if args.only_c5:
        import torch
        print(json.dumps(bench_c5(torch.device("cuda", 0))))
        return
    if args.only_batch:
        import torch
        print(json.dumps(bench_batch(torch.device("cuda", 0), steps=args.steps, warmup=args.warmup,
                                     tune_cache=args.batch_tune_cache)))
        return
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_b200(args, rank, world)
    if not args.no_stock_corr:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        peak_bf16 = None
        p = ROOT / "MEASURED_PEAKS.json"
        if p.exists():
            peak_bf16 = float(json.loads(p.read_text())["bf16_tflops"])
        sc = [bench_stock_corr(dev, N) for N in (2000, 5000)]
        for r in sc:
            if peak_bf16:
                r["bf16x3"]["tensor_frac_of_measured_bf16_peak"] = r["bf16x3"]["tflops_mma_issued"] / peak_bf16
        res["stock_corr"] = {"workload": "pairwise-complete (N,N) Pearson, T=1218, f32 returns "
                                         "(0.02*t4 + 3-factor component), pre-listing gaps + Bernoulli(0.98) mask",
                             "bf16_peak_tflops_measured": peak_bf16, "results": sc}
    if not args.no_batch:
        import torch
        res["batch"] = bench_batch(torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0))))
    if not args.no_c5:
        import torch
        res["c5_learned_streaming"] = bench_c5(torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0))))
    if rank == 0:
        if not args.no_cpu_baseline:
            X, R, fm, rm = make_panel()
            v, el, dates = cpu_baseline(X, R, fm, rm, budget_s=12.0, procs=1)
            res["cpu_baseline"] = {"value": v, "unit": "Gelem/s", "cores": 1, "kind": "port",
                                   "sample": f"{dates} dates x 12 factors x 5000 stocks "
                                             f"({el:.1f} s, single thread, oracle port of "
                                             "np_cs_rank + np_rolling_ic)"}
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
