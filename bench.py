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
import hashlib
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
                                               learn["model"].handle, args.learn_cap, learn["stats"].data_ptr(),
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
    timed_ranks = dranks.cpu().numpy()
    timed_ic = dic.cpu().numpy()
    learned_info = None
    if learn is not None:
        st = learn["stats"].cpu().numpy()
        codes = st[..., 0]
        # bit-exactness of the whole learned output against the radix path
        radix_step()
        torch.cuda.synchronize(dev)
        exact = bool(np.array_equal(timed_ranks.view(np.uint32), dranks.cpu().numpy().view(np.uint32))) and \
            ic_bitwise(timed_ic, dic.cpu().numpy())
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
        saved = radix_ms - learned_ms_cmp
        learned_info = {"fit_ms": learn["fit_ms"], "train_dates": learn["train_dates"],
                        "fit": "1500 Adam steps on 64 samples per (factor, date) of dates [0, 250), once, "
                               "before the timed steps (not in ms_per_step)",
                        "break_even_steps": (learn["fit_ms"] / saved) if saved > 0 else None,
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
    e2e_s = e2e_ok = e2e_floor = None
    if not args.no_e2e:
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
        e2e_ok = bool(np.array_equal(hranks.numpy().view(np.uint32), timed_ranks.view(np.uint32)))
        h2d = hX.numel() * 4 + hR.numel() * 4 + hfm.numel() + hrm.numel()
        d2h = hranks.numel() * 4 + hic.numel() * 8
        del hX, hR, hfm, hrm, hranks, hic
        e2e_floor = transfer_floor(h2d, d2h, dev)
    res = finish(args, world, X, R, fm, rm, ms, e2e_s, e2e_ok, clk, dev, learned_info)
    if e2e_floor is not None and res.get("e2e"):
        e = res["e2e"]
        floor_v = world * X.size / e2e_floor["both_s"] / 1e9
        e["transfer_floor"] = {
            "what": "this machine's copy floor: the step's input and output bytes as one plain pinned copy each way, "
                    "both directions at once, no compute (best of 3)",
            "value": floor_v, "unit": "Gelem/s", "ms": e2e_floor["both_s"] * 1e3,
            "h2d_gb_s": e2e_floor["h2d_gb_s"], "d2h_gb_s": e2e_floor["d2h_gb_s"],
            "both_gb_s": e2e_floor["both_gb_s"], "e2e_frac_of_floor": e["value"] / floor_v}
    fcl = bench_factor_corr(dX, dfm, X, fm, dev, steps=max(3, args.steps // 2))
    res["factor_corr"] = fcl
    res["c2_stages"] = bench_c2_stages(dX, X, fm, dev, ms, fcl["f64"]["ms"])
    # parity of the timed outputs (and of the stage legs) against the oracle on
    # the whole panel
    if not args.no_parity and rank == 0:
        orc = oracle_c2(X, R, fm, rm)
        rank_ok = all(_sha(timed_ranks[f]) == orc["rank_sha"][f] for f in range(F))
        ic_ok = ic_bitwise(timed_ic, orc["ic"])
        fmb = fm.astype(bool)
        scan_ok = True
        for f, shas in orc["scan_sha"].items():
            r = nat.fcb().parameter_scan_f32(np.ascontiguousarray(X[f]), fmb, return_timing=False)
            scan_ok &= [_sha(g) for g in r["groups"]] == shas
        ex = orc["factor_corr"]
        f64 = np.asarray(fcl.pop("_f64_out"))
        bf = np.asarray(fcl.pop("_bf16x3_out"))
        same_nan = bool(np.array_equal(np.isnan(f64), np.isnan(ex)))
        e64 = float(np.nanmax(np.abs(f64 - ex)))
        ebf = np.abs(bf - ex)
        res["parity"] = {
            "oracle": "numpy restatement of the reference CPU path (fc/_cpu_core.py), pinned to its outputs",
            "rank_ic": {"compared": f"cs ranks of all {F}x{T}x{N} cells (bit patterns) and the IC of all "
                                    f"{F}x{T} (factor, date) sections of the timed step",
                        "bit_exact": bool(rank_ok and ic_ok)},
            "parameter_scan": {"compared": f"all four groups of planes {sorted(orc['scan_sha'])} "
                                           f"({T}x{N}), drop-in binding parameter_scan_f32",
                               "bit_exact": bool(scan_ok)},
            "factor_corr_f64": {"compared": f"{F}x{F} over {T * N} rows, fcb_dev_factor_corr on factor planes",
                                "max_abs_err": e64, "tol": 1e-12, "ok": bool(same_nan and e64 <= 1e-12)},
            "factor_corr_bf16x3": {"max_abs_err": float(np.nanmax(ebf)), "mean_abs_err": float(np.nanmean(ebf)),
                                   "tol": 1e-6, "nan_pattern_matches": bool(np.array_equal(np.isnan(bf),
                                                                                           np.isnan(ex)))},
            "oracle_seconds": orc["seconds"]}
        fcl["f64"]["max_abs_err_vs_oracle"] = e64
        fcl["bf16x3"]["max_abs_err_vs_oracle"] = float(np.nanmax(ebf))
        fcl["bf16x3"]["mean_abs_err_vs_oracle"] = float(np.nanmean(ebf))
    else:
        fcl.pop("_f64_out", None)
        fcl.pop("_bf16x3_out", None)
    return res


# DRAM bytes of one rank + IC step per date at N=5000, F=12 (the returns
# preparation plus the per-(date, factor) rank kernel), from one ncu capture
# of each kernel at T=600: dram__bytes_read.sum + dram__bytes_write.sum.
# Traffic grows with the number of dates at fixed N and F, so the bench's step
# is that times T.
TRAFFIC_PER_DATE = {"learned": (156.591104e6 + 88.684544e6 + 18.057728e6) / 600,
                    "radix": (156.073472e6 + 86.176000e6 + 18.057728e6) / 600}


def transfer_floor(h2d_bytes, d2h_bytes, dev, reps=3):
    """The host<->device copy floor of the e2e leg on this machine: the same bytes
    as one pinned copy per direction, alone and both at once (best of reps)."""
    import torch
    hin = torch.empty(h2d_bytes, dtype=torch.uint8).pin_memory()
    hout = torch.empty(d2h_bytes, dtype=torch.uint8).pin_memory()
    din = torch.empty(h2d_bytes, dtype=torch.uint8, device=dev)
    dout = torch.zeros(d2h_bytes, dtype=torch.uint8, device=dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    best = {}
    for mode in ("h2d", "d2h", "both"):
        t = []
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            if mode in ("h2d", "both"):
                with torch.cuda.stream(s_in):
                    din.copy_(hin, non_blocking=True)
            if mode in ("d2h", "both"):
                with torch.cuda.stream(s_out):
                    hout.copy_(dout, non_blocking=True)
            torch.cuda.synchronize(dev)
            t.append(time.perf_counter() - t0)
        best[mode] = min(t)
    del hin, hout, din, dout
    return {"h2d_gb_s": h2d_bytes / best["h2d"] / 1e9, "d2h_gb_s": d2h_bytes / best["d2h"] / 1e9,
            "both_gb_s": (h2d_bytes + d2h_bytes) / best["both"] / 1e9, "both_s": best["both"]}


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


def finish(args, world, X, R, fm, rm, ms, e2e_s, e2e_ok, clk, dev, learned_info=None):
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
                     "kernel": "k_ric_prep + k_ric_learned" if args.method == "learned" else
                               "k_ric_prep + k_ric_radix",
                     "algorithmic_bytes_per_launch": bytes_launch},
        "gpu_launches": args.steps * (3 if args.method == "learned" else 2),
        "clocks": clk.summary(),
    }
    if learned_info is not None:
        res["learned"] = learned_info
    return res


def bench_factor_corr(dX, dfm, X, fm, dev, steps=5, warmup=2):
    """factor_corr of the C2 panel (F factors pooled over the T*N (t, i) rows,
    factor mask broadcast per column) on the device-resident factor planes:
    the FP64 drop-in (fcb_dev_factor_corr) and the BF16x3 tensor-core form
    (fcb_dev_factor_corr_bf16x3).  Both outputs are handed back for the
    oracle comparison."""
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    F, T, N = X.shape
    ws = lib.fcb_workspace_create()
    out = torch.empty((F, F), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rows = T * N
    peak, _ = measured_peaks()
    res = {"workload": f"factor_corr {F}x{F} over {rows} (t,i) rows, f32 factor planes, factor mask"}
    for name, fn in (("f64", lib.fcb_dev_factor_corr), ("bf16x3", lib.fcb_dev_factor_corr_bf16x3)):
        def run():
            if name == "f64":
                nat.check(fn(dX.data_ptr(), 0, dfm.data_ptr(), T, N, F, 1, out.data_ptr(), ws, stream.cuda_stream),
                          "fcb_dev_factor_corr")
            else:
                nat.check(fn(dX.data_ptr(), dfm.data_ptr(), T, N, F, 1, out.data_ptr(), ws, stream.cuda_stream),
                          "fcb_dev_factor_corr_bf16x3")

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
        nat.check(lib.fcb_dev_status(), "fcb_dev_status")
        alg_bytes = rows * (4 * F + 1)
        res[name] = {"ms": ms, "rows_per_s": rows / (ms / 1e3), "algorithmic_gb_s": alg_bytes / (ms / 1e3) / 1e9,
                     "hbm_frac": alg_bytes / (ms / 1e3) / 1e9 / peak}
        res["_" + name + "_out"] = out.cpu().numpy()
    lib.fcb_workspace_destroy(ws)
    res["bf16x3"]["algorithmic_tflops"] = 4 * 2.0 * F * F * rows / (res["bf16x3"]["ms"] / 1e3) / 1e12
    res["bf16x3_speedup_vs_f64"] = res["f64"]["ms"] / res["bf16x3"]["ms"]
    return res


def bench_c2_stages(dX, X, fm, dev, rank_ic_ms, factor_corr_ms, steps=3):
    """The C2 pipeline stage by stage on the same panel: cs_rank of every factor
    plane (device entry point, CUDA events), parameter_scan (4 groups) of every
    plane (device entry point, CUDA events), and the fused rank + IC and
    factor_corr legs measured above -- the counterpart of the reference's
    parameter_scan -> rolling_ic -> factor_corr pipeline figure."""
    import ctypes as C
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    F, T, N = X.shape
    dfm = torch.from_numpy(fm).to(dev)
    out = torch.empty((T, N), dtype=torch.float32, device=dev)
    souts = [torch.empty((T, N), dtype=torch.float32, device=dev) for _ in range(4)]
    optr = (C.c_void_p * 4)(*[o.data_ptr() for o in souts])
    st = (C.c_int * 4)()
    stream = torch.cuda.current_stream(dev)

    def cs_all():
        for f in range(F):
            nat.check(lib.fcb_dev_cs_rank_f32(dX[f].data_ptr(), dfm.data_ptr(), T, N, 0, out.data_ptr(),
                                              stream.cuda_stream), "fcb_dev_cs_rank_f32")

    def scan_all():
        for f in range(F):
            nat.check(lib.fcb_dev_parameter_scan_f32(dX[f].data_ptr(), dfm.data_ptr(), T, N, optr, st, None,
                                                     stream.cuda_stream), "fcb_dev_parameter_scan_f32")

    def timed(fn):
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

    cs_ms = timed(cs_all)
    scan = timed(scan_all)
    return {"workload": f"C2 stages on {F} factor planes of {T}x{N}",
            "cs_rank_ms_all_planes": cs_ms, "parameter_scan_ms_all_planes": scan,
            "rank_ic_ms_all_planes": rank_ic_ms, "factor_corr_ms": factor_corr_ms,
            "pipeline_ms": scan + rank_ic_ms + factor_corr_ms,
            "pipeline": "parameter_scan (4 groups) + cs_rank/rolling_ic (fused, learned) + factor_corr (f64), "
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


def bench_batch(dev, steps=5, warmup=2, tune_cache=None, cpu_sample=True):
    """Batched uneven panels: one autotuned CUDA-graph replay of the batched
    rank+IC kernels + per-panel factor_corr, against the same work issued one
    panel at a time.  Device-resident inputs (8.8 GB of factors, far above
    L2).  Rank + IC use learned splitters: one CdfModel for the 8 factors,
    fitted once (timed, outside the replays) on the exact radix ranks of
    panel 0's first 250 dates and shared by every panel (the model works on
    per-date standardised values, so it does not depend on a panel's T or N);
    the same batch without the model is timed as the radix replay."""
    import torch
    import fcb200
    from fcb200 import _native as nat
    panels = make_batch_panels(dev)
    cells = sum(int(p["X"].numel()) for p in panels)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    # the radix batch first (its replay is the comparison), then the model
    # fitted on panel 0's exact ranks
    b_rx = fcb200.Batch(panels, min_valid=MIN_VALID)
    p0 = panels[0]
    F0, T0, N0 = (int(v) for v in p0["X"].shape)
    nat.check(nat.lib().fcb_dev_rank_ic_panel(p0["X"].data_ptr(), p0["R"].data_ptr(), p0["fmask"].data_ptr(),
                                              p0["rmask"].data_ptr(), F0, T0, N0, MIN_VALID,
                                              p0["ranks"].data_ptr(), p0["ic"].data_ptr(), 0, stream.cuda_stream),
              "fcb_dev_rank_ic_panel")
    model = fcb200.CdfModel(F0, seed=20261205)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    model.fit(p0["X"], p0["ranks"], T0, N0, 0, min(T0, 250), steps=1500, lr=3e-3, stream=stream.cuda_stream)
    f1.record(stream)
    torch.cuda.synchronize(dev)
    fit_ms = f0.elapsed_time(f1)
    for p in panels:
        p["model"] = model
    b = fcb200.Batch(panels, min_valid=MIN_VALID)
    t0 = time.perf_counter()
    # with a cache file, a second run takes the tuned configuration without
    # measuring alternatives (so a profiler sees only the timed launches)
    cfg, tuned_ms, cached = b.autotune(reps=2, cache_path=tune_cache)
    tune_s = time.perf_counter() - t0

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

    b_rx.config = cfg
    ms_graph_rx = timed(b_rx.run)
    b_rx.status()
    b_rx.close()
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
    def variant(n):  # the f32 kernel variant a panel of width n runs in (fcb200.h, batched panels)
        if n <= min(cfg["nt_small_max"], 2048):
            return 0
        if n <= min(cfg["nt_mid_max"], 5120):
            return 1
        return 2 if n <= 8192 else 3
    variants = sorted({variant(p["X"].shape[2]) for p in panels})
    res = {"workload": "64 uneven panels (N ~ U[300,6000], T ~ U[250,2500], F=8, gaps ~ U[0,0.2]): "
                       "cs_rank + rolling_ic(30) + factor_corr per panel",
           "cells": cells, "unit": "Gelem/s",
           # kernels: per kernel variant, the returns pass, the rank pass over all its
           # panels and the pass over the sections the learned buckets handed back; for all
           # panels together, factor_corr's column pass + merge, Gram pass + finalize and the
           # four fallback kernels (every pool here has 4096 rows or more; they exit at once
           # when no pair is flagged); the per-panel arm runs, for each panel, those three
           # rank kernels and the eight factor_corr kernels
           "method": "learned splitters, one CdfModel (F=8) fitted on panel 0 and shared by every panel",
           "fit_ms": fit_ms,
           "graph": {"ms": ms_graph, "value": cells / (ms_graph / 1e3) / 1e9,
                     "kernels_per_replay": 3 * len(variants) + 8},
           "graph_radix": {"ms": ms_graph_rx, "value": cells / (ms_graph_rx / 1e3) / 1e9},
           "learned_speedup_vs_radix_graph": ms_graph_rx / ms_graph,
           "per_panel": {"ms": ms_pp, "value": cells / (ms_pp / 1e3) / 1e9,
                         "kernels_per_step": sum((3 if p["X"].shape[0] >= 2 else 1) + 8 for p in panels)},
           "speedup_graph_vs_per_panel": ms_pp / ms_graph,
           "bit_exact_graph_vs_per_panel": bool(same),
           "autotune": {"config": cfg, "tuned_ms": tuned_ms, "tuning_s": tune_s, "from_cache": cached}}
    b.close()
    if cpu_sample:
        # CPU baseline: the oracle port of the reference CPU path on one whole
        # panel (cs_rank + rolling_ic of every factor, factor_corr), scaled to
        # the batch by cells
        from oracle import fc_oracle as O
        p0 = panels[0]
        Xh, Rh = p0["X"].cpu().numpy(), p0["R"].cpu().numpy()
        fmh, rmh = p0["fmask"].cpu().numpy().astype(bool), p0["rmask"].cpu().numpy().astype(bool)
        t0 = time.perf_counter()
        for f in range(Xh.shape[0]):
            O.cs_rank(Xh[f], fmh, False)
            O.rolling_ic(Xh[f], Rh, fmh, rmh, MIN_VALID)
        O.factor_corr(np.ascontiguousarray(np.moveaxis(Xh, 0, -1)), fmh)
        el = time.perf_counter() - t0
        v = Xh.size / el / 1e9
        res["cpu_baseline"] = {"value": v, "unit": "Gelem/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"panel 0 ({Xh.shape[1]}x{Xh.shape[2]}x{Xh.shape[0]}, {el:.1f} s): "
                                         "np_cs_rank + np_rolling_ic per factor + np_factor_corr; the 64-panel "
                                         f"batch extrapolates to {cells / v / 1e9:.0f} s"}
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


def bench_c5(dev, T=5000, N=8000, F=128, Tb=250, seed=20261206, cpu_sample=True, head=1, fit_steps=300,
             refit_every=4, overlap_fit=False):
    """Learned splitters on the streaming configuration (T=5000, N=8000,
    F=128: 5.12 G cells, 20.5 GB of f32 factors, device-resident in blocks of
    250 dates), two end-to-end runs timed by CUDA events around the whole
    block loop:
      radix    every block ranked by the plain radix path;
      learned  the first `head` blocks are ranked by radix; the training
               samples are drawn from block 0's exact ranks and the networks
               are fitted (`fit_steps` Adam steps) on a second stream while
               blocks 1 .. head-1 are ranked (overlap_fit; otherwise in line
               on the ranking stream); block `head` waits for that fit on the
               device, and every later block is ranked by the learned path.  After every `refit_every`-th learned block b, samples
               of its (exact) ranks feed a 100-step refit on the second stream
               into the idle table slot while block b + 1 is ranked; block
               b + 2 waits for it on the device and ranks with the new table.
    Every fit is inside the learned figure.  An untimed pass then compares
    the learned output of every learned block with the radix output bit for
    bit."""
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
    nb = len(blocks)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    side = torch.cuda.Stream(dev)
    s = stream.cuda_stream
    ranks = torch.empty((F, Tb, N), dtype=torch.float32, device=dev)
    ranks2 = torch.empty_like(ranks)
    ic = torch.empty((F, Tb), dtype=torch.float64, device=dev)
    stats = torch.zeros((nb, F, Tb, 4), dtype=torch.int32, device=dev)

    def radix(X, R, fm, rm, out):
        nat.check(lib.fcb_dev_rank_ic_panel(X.data_ptr(), R.data_ptr(), fm.data_ptr(), rm.data_ptr(), F, Tb, N,
                                            MIN_VALID, out.data_ptr(), ic.data_ptr(), 0, s), "radix")

    def learned(model, b, X, R, fm, rm, out):
        nat.check(lib.fcb_dev_rank_ic_panel_learned(X.data_ptr(), R.data_ptr(), fm.data_ptr(), rm.data_ptr(), F,
                                                    Tb, N, MIN_VALID, out.data_ptr(), ic.data_ptr(), model.handle,
                                                    256, stats[b].data_ptr(), s), "learned")

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # ---- radix run (per-block events for the same-blocks comparison)
    bev = [torch.cuda.Event(enable_timing=True) for _ in range(nb + 1)]
    bev[0].record(stream)
    for b, (X, R, fm, rm) in enumerate(blocks):
        radix(X, R, fm, rm, ranks)
        bev[b + 1].record(stream)
    torch.cuda.synchronize(dev)
    t_radix = bev[0].elapsed_time(bev[nb])
    t_radix_lb = bev[head].elapsed_time(bev[nb])
    # ---- learned run, every fit included
    model = fcb200.CdfModel(F, seed=seed)
    # a model allocates its sample buffer on its first sample call: make one
    # (on the last radix block's ranks, overwritten by the timed call) before
    # the timing, so that no host-side allocation sits inside it
    model.sample(blocks[-1][0], ranks, Tb, N, 0, Tb, stream=s)
    torch.cuda.synchronize(dev)
    fit_done = torch.cuda.Event()
    swap_at = -1
    refits = swaps = 0
    ev[0].record(stream)
    for b, (X, R, fm, rm) in enumerate(blocks):
        if b < head:
            radix(X, R, fm, rm, ranks)
            if b == 0:
                model.sample(X, ranks, Tb, N, 0, Tb, stream=s)
                fit_stream = side if overlap_fit else stream
                fit_stream.wait_stream(stream)
                model.train(fit_steps, 3e-3, into_idle=False, stream=fit_stream.cuda_stream)
                fit_done.record(fit_stream)
            if b == head - 1:
                ev[1].record(stream)
            continue
        if b == head:
            stream.wait_event(fit_done)  # on the device: the first fit has landed
        if b == swap_at:
            stream.wait_event(fit_done)  # on the device: the refit has landed
            model.swap()
            swaps += 1
            swap_at = -1
        learned(model, b, X, R, fm, rm, ranks)
        if swap_at < 0 and (b - head) % refit_every == refit_every - 1 and b + 2 < nb:
            model.sample(X, ranks, Tb, N, 0, Tb, stream=s)
            side.wait_stream(stream)
            model.train(100, 1e-3, into_idle=True, stream=side.cuda_stream)
            fit_done.record(side)
            swap_at = b + 2
            refits += 1
    stream.wait_stream(side)
    ev[2].record(stream)
    torch.cuda.synchronize(dev)
    t_learn_all = ev[0].elapsed_time(ev[2])
    t_learn_lb = ev[1].elapsed_time(ev[2])
    t_fit0 = ev[0].elapsed_time(ev[1])
    codes = stats[head:, ..., 0].flatten().cpu().numpy()
    # ---- untimed exactness pass: learned (final model) vs radix, every block
    exact = True
    for b, (X, R, fm, rm) in enumerate(blocks):
        if b < head:
            continue
        radix(X, R, fm, rm, ranks)
        ic_r = ic.clone()
        learned(model, b, X, R, fm, rm, ranks2)
        exact = exact and bool(torch.equal(ranks.view(torch.int32), ranks2.view(torch.int32))) and \
            bool(torch.equal(torch.nan_to_num(ic_r, nan=7.0), torch.nan_to_num(ic, nan=7.0)))
    torch.cuda.synchronize(dev)
    lb_cells = F * (T - head * Tb) * N
    res = {"workload": f"learned splitters, streaming: T={T}, N={N}, F={F} ({F * T * N / 1e9:.2f} G cells, "
                       f"{F * T * N * 4 / 1e9:.1f} GB f32), blocks of {Tb} dates; a {fit_steps}-step fit on "
                       f"block 0's exact ranks " + (f"overlapped with radix blocks 1-{head - 1}" if overlap_fit
                                                    else "in line") +
                       f", learned from block {head}; a 100-step refit after every {refit_every}th learned "
                       f"block, overlapped with the next block",
           "radix_gelem_s": F * T * N / (t_radix / 1e3) / 1e9,
           "learned_incl_fit_gelem_s": F * T * N / (t_learn_all / 1e3) / 1e9,
           "learned_blocks_gelem_s": lb_cells / (t_learn_lb / 1e3) / 1e9,
           "radix_same_blocks_gelem_s": lb_cells / (t_radix_lb / 1e3) / 1e9,
           "speedup_vs_radix_same_blocks_incl_refits": t_radix_lb / t_learn_lb,
           "speedup_vs_radix_whole_run_incl_all_fits": t_radix / t_learn_all,
           "initial_fit_and_radix_blocks_ms": t_fit0, "refits_overlapped": refits, "table_swaps": swaps,
           "learned_fraction": float((codes == 1).mean()),
           "fallback_overflow": float((codes == 2).mean()), "fallback_judge": float((codes == 3).mean()),
           "fallback_scale": float((codes == 4).mean()),
           "bit_exact_vs_radix": exact}
    if cpu_sample:
        from oracle import fc_oracle as O
        X, R, fm, rm = blocks[2]
        nd = 16
        Xh, Rh = X[:, :nd].cpu().numpy(), R[:nd].cpu().numpy()
        fmh, rmh = fm[:nd].cpu().numpy().astype(bool), rm[:nd].cpu().numpy().astype(bool)
        t0 = time.perf_counter()
        for f in range(F):
            O.cs_rank(Xh[f], fmh, False)
            O.rolling_ic(Xh[f], Rh, fmh, rmh, MIN_VALID)
        el = time.perf_counter() - t0
        v = Xh.size / el / 1e9
        res["cpu_baseline"] = {"value": v, "unit": "Gelem/s", "cores": 1, "kind": "port",
                               "sample": f"{nd} dates x {F} factors x {N} stocks of block 2 ({el:.1f} s, "
                                         "np_cs_rank + np_rolling_ic); the whole panel extrapolates to "
                                         f"{F * T * N / v / 1e9 / 60:.0f} min"}
    del blocks
    torch.cuda.empty_cache()
    return res


def bench_stock_corr(dev, N, T=1218, steps=5, warmup=2, oracle=True):
    """stock_corr precision forms on one (T,N) panel, device-resident:
    BF16x3 tensor-core path vs plain FP32, each against the oracle's
    np_stock_corr restatement (FP64), which is also timed on the host as the
    CPU baseline; the FP64 drop-in's distance to the oracle is reported too."""
    import torch
    from fcb200 import _native as nat
    lib = nat.lib()
    X, mask = make_stock_panel(T=T, N=N)
    m8 = mask.astype(np.uint8)
    f64 = np.empty((N, N))
    nat.check(lib.fcb_stock_corr(nat.ptr(X), 0, nat.ptr(m8), T, N, nat.ptr(f64), None, None), "fcb_stock_corr")
    alg_flops = 4 * 2.0 * N * N * T           # X.X^T, X.M^T, X^2.M^T, M.M^T (dense-equivalent)
    res = {"N": N, "T": T, "algorithmic_gflop": alg_flops / 1e9}
    if oracle:
        from oracle import fc_oracle as O
        t0 = time.perf_counter()
        ref = O.stock_corr(X, mask)
        cpu_s = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": alg_flops / cpu_s / 1e12, "unit": "TFLOP/s", "ms": cpu_s * 1e3,
                               "cores": os.cpu_count(), "kind": "port",
                               "sample": f"the whole (T={T}, N={N}) panel, oracle np_stock_corr (numpy, "
                                         "OpenBLAS GEMMs on every core)"}
        res["error_reference"] = "oracle (numpy FP64 restatement of np_stock_corr)"
        res["f64_dropin_max_abs_err_vs_oracle"] = float(np.nanmax(np.abs(f64 - ref)))
    else:
        ref = f64
        res["error_reference"] = "FP64 drop-in path (fcb_stock_corr)"
    dX = torch.from_numpy(X).to(dev)
    dM = torch.from_numpy(m8).to(dev)
    dO = torch.empty((N, N), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ws = lib.fcb_workspace_create()
    Tp = (T + 31) // 32 * 32
    n_i, n_j = (N + 127) // 128, (N + 63) // 64
    tiles = n_i * n_j - n_i * (n_i - 1)   # 128 x 64 tiles with tj >= 2 ti
    # issued MMA work: per tile and 16 dates, M=128 MMAs of N-total 1216
    # (D1 256 + 192 + 128, n|sy 128 + 64 + 64, sy2 3 x 64, sx2 3 x 64)
    exec_flops = tiles * (Tp // 16) * 2.0 * 128 * 1216 * 16
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
             "max_abs_err": float(np.nanmax(err)), "mean_abs_err": float(np.nanmean(err)),
             "nan_pattern_matches": same_nan}
        if mode == 0:
            d["tflops_mma_issued"] = exec_flops / (ms / 1e3) / 1e12
        out[name] = d
    lib.fcb_workspace_destroy(ws)
    res.update(out)
    res["bf16x3_speedup_vs_fp32"] = out["fp32"]["ms"] / out["bf16x3"]["ms"]
    return res


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8)).hexdigest()


def oracle_c2(X, R, fm, rm, scan_planes=(0, 6), threads=None):
    """The oracle's results on the whole panel: cs ranks (as digests of their
    bit patterns) and IC of every factor, all four parameter_scan groups of
    `scan_planes`, and factor_corr.  Computed in a thread pool (numpy releases
    the GIL inside its sorts and GEMMs)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import fc_oracle as O
    F = X.shape[0]
    fmb, rmb = fm.astype(bool), rm.astype(bool)
    threads = threads or max(1, min(16, os.cpu_count() or 1))

    def rank_ic(f):
        return _sha(O.cs_rank(X[f], fmb, False)), O.rolling_ic(X[f], R, fmb, rmb, MIN_VALID)

    def scan(f):
        return [_sha(g) for g in O.parameter_scan(X[f], fmb)]

    def fcorr():
        return O.factor_corr(np.ascontiguousarray(np.moveaxis(X, 0, -1)), fmb)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        fc_fut = ex.submit(fcorr)
        sc_fut = {f: ex.submit(scan, f) for f in scan_planes}
        ri = list(ex.map(rank_ic, range(F)))
        res = {"rank_sha": [a for a, _ in ri], "ic": np.stack([b for _, b in ri]),
               "scan_sha": {f: v.result() for f, v in sc_fut.items()}, "factor_corr": fc_fut.result()}
    res["seconds"] = time.perf_counter() - t0
    return res


def ic_bitwise(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and bool(np.array_equal(np.isnan(a), np.isnan(b))) and \
        bool(np.array_equal(a[~np.isnan(a)].view(np.uint64), b[~np.isnan(b)].view(np.uint64)))


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
    ap.add_argument("--learn-cap", type=int, default=256,
                    help="largest bucket the learned rank kernel ranks itself (larger ones go to radix)")
    ap.add_argument("--no-stock-corr", action="store_true", help="skip the stock_corr precision-form leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-parity", action="store_true", help="skip the whole-panel oracle comparison")
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
                                          warmup=args.warmup, oracle=not args.no_cpu_baseline)))
        return
    if args.only_c5:
        import torch
        print(json.dumps(bench_c5(torch.device("cuda", 0), cpu_sample=not args.no_cpu_baseline)))
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
        sc = [bench_stock_corr(dev, N, oracle=not args.no_cpu_baseline) for N in (2000, 5000)]
        for r in sc:
            if peak_bf16:
                r["bf16x3"]["tensor_frac_of_measured_bf16_peak"] = r["bf16x3"]["tflops_mma_issued"] / peak_bf16
        res["stock_corr"] = {"workload": "pairwise-complete (N,N) Pearson, T=1218, f32 returns "
                                         "(0.02*t4 + 3-factor component), pre-listing gaps + Bernoulli(0.98) mask",
                             "bf16_peak_tflops_measured": peak_bf16, "results": sc}
    if not args.no_batch:
        import torch
        res["batch"] = bench_batch(torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0))),
                                   cpu_sample=not args.no_cpu_baseline)
    if not args.no_c5:
        import torch
        res["c5_learned_streaming"] = bench_c5(torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0))),
                                               cpu_sample=not args.no_cpu_baseline)
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
