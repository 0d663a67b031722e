"""Generate the golden vectors that pin the oracle and the CUDA path.

Run where a checkout of the reference is available (it is only read; nothing
is copied from it except the outputs its own CPU path computes here and the
frozen anchor arrays/expected values of its fixtures):

    python tests/golden/make_golden.py <path to the reference checkout>

Writes ``tests/golden/golden_v1.npz`` (arrays) and ``tests/golden/golden_v1.json``
(case list).  Sources of truth, all from the reference:

* ``fc/_cpu_core.py`` -- np_cs_rank / np_parameter_scan / np_rolling_ic /
  np_factor_corr / np_stock_corr, evaluated here on seeded inputs;
* ``benchmark_corpus/parity_anchors_v1.{npz,manifest.json}`` -- frozen anchors
  with their manifest ``expected`` values;
* ``tests/fixtures/corr_corpus_v1.{npz,manifest.json}`` -- adversarial
  correlation pairs with manifest ``expected`` values;
* ``CLAUDE.md`` contract counter-examples (desc ties, constant IC section).
"""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    ref = pathlib.Path(ref_root)
    sys.path.insert(0, str(ref))
    from fc import _cpu_core as cc  # the reference CPU path

    arrays: dict[str, np.ndarray] = {}
    cases: list[dict] = []

    def put(name, arr):
        assert name not in arrays, name
        arrays[name] = np.ascontiguousarray(arr)
        return name

    def add(case):
        cases.append(case)

    # ---------------------------------------------------------------- anchors
    anc = np.load(ref / "benchmark_corpus" / "parity_anchors_v1.npz")
    man = json.loads((ref / "benchmark_corpus" / "parity_anchors_v1.manifest.json")
                     .read_text(encoding="utf-8"))
    for c in man["case_schema"]:
        cid = "anchor_" + c["id"]
        op = c["operation"]
        ins = [put(f"{cid}_in{k}", anc[nm]) for k, nm in enumerate(c["inputs"])]
        msk = {k: put(f"{cid}_{k}", anc[v]) for k, v in c.get("masks", {}).items()}
        exp = c["expected"]
        rec = {"id": cid, "source": "parity_anchors_v1", "op": op,
               "inputs": ins, "masks": msk, "params": c.get("params", {}),
               "expected": exp, "tolerance": c.get("tolerance")}
        try:
            if op == "cs_rank":
                x = anc[c["inputs"][0]].astype(np.float32)[None, :]
                m = anc[c["masks"]["mask"]][None, :] if "mask" in c.get("masks", {}) else None
                out = cc.np_cs_rank(x, m, bool(c["params"]["descending"]))
                rec["ref_out"] = put(cid + "_ref", out)
            elif op == "rolling_ic":
                f = anc[c["inputs"][0]][None, :]
                r = anc[c["inputs"][1]][None, :]
                out = cc.np_rolling_ic(f, r, None, None, int(c["params"]["min_valid"]))
                rec["ref_out"] = put(cid + "_ref", out)
            elif op == "factor_corr" and exp not in ("ValueError",):
                cols = [anc[nm].astype(np.float64) for nm in c["inputs"]]
                if len(cols) == 1:
                    cols = [cols[0], cols[0]]
                F3 = np.stack(cols, axis=1)[:, None, :]
                m = anc[c["masks"]["mask"]][:, None] if "mask" in c.get("masks", {}) else None
                out = cc.np_factor_corr(F3, m)
                rec["ref_out"] = put(cid + "_ref", out)
        except ValueError as e:  # domain / shape errors are expected results
            rec["ref_error"] = "ValueError"
            rec["ref_error_msg"] = str(e)
        add(rec)

    # ------------------------------------------------------ correlation corpus
    cz = np.load(ref / "tests" / "fixtures" / "corr_corpus_v1.npz")
    cm = json.loads((ref / "tests" / "fixtures" / "corr_corpus_v1.manifest.json")
                    .read_text(encoding="utf-8"))
    for c in cm["cases"]:
        cid = "corpus_" + c["id"]
        a = cz[c["id"] + "_a"]
        b = cz[c["id"] + "_b"]
        ma = cz[c["id"] + "_mask_a"] if (c["id"] + "_mask_a") in cz.files else None
        mb = cz[c["id"] + "_mask_b"] if (c["id"] + "_mask_b") in cz.files else None
        X = np.stack([a, b], axis=1)
        mask = None
        if ma is not None or mb is not None:
            mask = np.ones(X.shape, dtype=bool)
            if ma is not None:
                mask[:, 0] = ma
            if mb is not None:
                mask[:, 1] = mb
        rec = {"id": cid, "source": "corr_corpus_v1", "op": "stock_corr",
               "inputs": [put(cid + "_x", X)],
               "masks": ({"mask": put(cid + "_mask", mask)} if mask is not None else {}),
               "expected": (None if c["expected_is_nan"] else c["expected"]),
               "expected_is_nan": bool(c["expected_is_nan"]), "tolerance": 1e-12}
        try:
            rec["ref_out"] = put(cid + "_ref", cc.np_stock_corr(X, mask))
        except ValueError as e:
            rec["ref_error"] = "ValueError"
            rec["ref_error_msg"] = str(e)
        add(rec)

    # ------------------------------------------------ contract counter-examples
    y = np.array([[3.0, 3.0, 1.0]], dtype=np.float32)
    add({"id": "contract_desc_ties", "source": "CLAUDE.md:63", "op": "cs_rank",
         "inputs": [put("contract_desc_ties_x", y)], "masks": {},
         "params": {"descending": True}, "expected": [1.0, 2.0, 3.0],
         "ref_out": put("contract_desc_ties_ref", cc.np_cs_rank(y, None, True))})
    f = np.full((2, 100), 0.5)
    r = np.full((2, 100), 0.1)
    add({"id": "contract_const_ic", "source": "CLAUDE.md:143", "op": "rolling_ic",
         "inputs": [put("contract_const_ic_f", f), put("contract_const_ic_r", r)],
         "masks": {}, "params": {"min_valid": 30}, "expected": "nan",
         "ref_out": put("contract_const_ic_ref", cc.np_rolling_ic(f, r, None, None, 30))})

    # ---------------------------------------------------------- random panels
    rng = np.random.default_rng(20261203)

    def rank_panel(T, N, tie_frac=0.2, nan_frac=0.05, zero_frac=0.02):
        x = rng.standard_normal((T, N)).astype(np.float32)
        k = rng.random((T, N)) < tie_frac
        x[k] = np.round(x[k], 1)
        z = rng.random((T, N)) < zero_frac
        x[z] = np.where(rng.random(z.sum()) < 0.5, 0.0, -0.0).astype(np.float32)
        bad = rng.random((T, N)) < nan_frac
        x[bad] = rng.choice(np.array([np.nan, np.inf, -np.inf], dtype=np.float32), bad.sum())
        if T > 2:
            x[1, :] = np.nan          # empty section
            x[2, :] = np.float32(1.25)  # constant section
        return x

    for (T, N) in [(3, 1), (4, 2), (5, 31), (5, 32), (5, 33), (4, 257), (3, 1000),
                   (2, 5000), (2, 8191), (2, 8192), (2, 8193), (1, 16384), (1, 20000)]:
        x = rank_panel(T, N)
        m = rng.random((T, N)) < 0.85
        for desc in (False, True):
            for use_m in (False, True):
                cid = f"rank_T{T}_N{N}_d{int(desc)}_m{int(use_m)}"
                if f"rank_T{T}_N{N}_x" not in arrays:
                    put(f"rank_T{T}_N{N}_x", x)
                    put(f"rank_T{T}_N{N}_mask", m)
                out = cc.np_cs_rank(x, m if use_m else None, desc)
                add({"id": cid, "source": "fc/_cpu_core.py:np_cs_rank", "op": "cs_rank",
                     "inputs": [f"rank_T{T}_N{N}_x"],
                     "masks": ({"mask": f"rank_T{T}_N{N}_mask"} if use_m else {}),
                     "params": {"descending": desc}, "ref_out": put(cid + "_ref", out)})
    # parameter_scan on one panel
    x = rank_panel(6, 777)
    m = rng.random(x.shape) < 0.8
    outs = cc.np_parameter_scan(x, m)
    add({"id": "scan_T6_N777", "source": "fc/_cpu_core.py:np_parameter_scan",
         "op": "parameter_scan", "inputs": [put("scan_T6_N777_x", x)],
         "masks": {"mask": put("scan_T6_N777_mask", m)}, "params": {},
         "ref_out": put("scan_T6_N777_ref", np.stack(outs))})

    # rolling_ic: dtype mixes, masks, min_valid edges, constant sections, ties
    for (T, N, fdt, rdt) in [(6, 40, np.float32, np.float64), (5, 500, np.float64, np.float64),
                             (4, 3000, np.float32, np.float32), (3, 8192, np.float32, np.float32),
                             (3, 9000, np.float64, np.float32), (2, 20000, np.float32, np.float32)]:
        f = rng.standard_normal((T, N))
        r = 0.1 * f + rng.standard_normal((T, N))
        f[rng.random((T, N)) < 0.1] = np.nan
        r[rng.random((T, N)) < 0.05] = np.inf
        k = rng.random((T, N)) < 0.3
        f[k] = np.round(f[k], 1)
        f = f.astype(fdt)
        r = r.astype(rdt)
        if T > 3:
            f[1, :] = 2.0                     # constant factor section
            r[2, : N - 3] = np.nan            # below min_valid
        fm = rng.random((T, N)) < 0.9
        rm = rng.random((T, N)) < 0.95
        base = f"ic_T{T}_N{N}"
        put(base + "_f", f)
        put(base + "_r", r)
        put(base + "_fm", fm)
        put(base + "_rm", rm)
        for mv in (2, 30):
            for use_m in (False, True):
                cid = f"{base}_mv{mv}_m{int(use_m)}"
                out = cc.np_rolling_ic(f, r, fm if use_m else None, rm if use_m else None, mv)
                add({"id": cid, "source": "fc/_cpu_core.py:np_rolling_ic", "op": "rolling_ic",
                     "inputs": [base + "_f", base + "_r"],
                     "masks": ({"factor_mask": base + "_fm", "fwd_mask": base + "_rm"}
                               if use_m else {}),
                     "params": {"min_valid": mv}, "ref_out": put(cid + "_ref", out)})

    # factor_corr: small panels with masks, NaN, a large-bias column, constants
    for (T, N, F, dt) in [(20, 15, 4, np.float64), (30, 40, 12, np.float32),
                          (8, 9, 3, np.float64)]:
        F3 = rng.standard_normal((T, N, F))
        F3[..., 1] = 0.6 * F3[..., 0] + 0.8 * F3[..., 1]
        F3[rng.random((T, N, F)) < 0.05] = np.nan
        if F >= 3:
            F3[..., 2] = F3[..., 2] + 1e9        # large bias -> fallback branch
        if F >= 4:
            F3[..., 3] = 0.25                    # constant column -> NaN
        F3 = F3.astype(dt)
        m = rng.random((T, N)) < 0.9
        cid = f"fcorr_T{T}_N{N}_F{F}"
        add({"id": cid, "source": "fc/_cpu_core.py:np_factor_corr", "op": "factor_corr",
             "inputs": [put(cid + "_x", F3)], "masks": {"mask": put(cid + "_mask", m)},
             "ref_out": put(cid + "_ref", cc.np_factor_corr(F3, m))})

    # stock_corr: masked / fully valid / large bias / constant column
    for (T, N, kind) in [(50, 30, "masked"), (64, 20, "full"), (40, 12, "bias"),
                         (300, 64, "masked")]:
        X = rng.standard_normal((T, N))
        X[:, 1] = 0.5 * X[:, 0] + X[:, 1]
        m = None
        if kind == "masked":
            m = rng.random((T, N)) < 0.85
            X[rng.random((T, N)) < 0.03] = np.nan
            X[:, 2] = 7.0
        if kind == "bias":
            X[:, :4] += 1e12
        cid = f"scorr_T{T}_N{N}_{kind}"
        add({"id": cid, "source": "fc/_cpu_core.py:np_stock_corr", "op": "stock_corr",
             "inputs": [put(cid + "_x", X)],
             "masks": ({"mask": put(cid + "_mask", m)} if m is not None else {}),
             "ref_out": put(cid + "_ref", cc.np_stock_corr(X, m))})

    np.savez_compressed(HERE / "golden_v1.npz", **arrays)
    (HERE / "golden_v1.json").write_text(json.dumps(
        {"version": 1, "generator": "tests/golden/make_golden.py",
         "reference_numpy": np.__version__, "cases": cases}, indent=1))
    print(f"wrote {len(cases)} cases, {len(arrays)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
