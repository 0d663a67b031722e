"""Run the reference's own adapter acceptance suite against this build.

    python tests/adapter_acceptance/run_suite.py <reference checkout> [--out summary.json]
                                                 [--tests tests/test_adapter_v1.py]

The reference's Python adapter ``fc/`` loads its two native modules,
``factor_cuda_pybind`` and ``factor_corr_pybind``, from ``<fc root>/build``
(fc/_util.py:200-219).  This script assembles, in a temporary directory
outside this repository, an unmodified copy of the reference's ``fc/``,
``tests/`` and ``benchmark_corpus/`` (the suite's fixtures and frozen
anchors) plus its ``pytest.ini``, puts this build's three shared libraries in
``build/`` -- the whole drop-in integration -- and runs the suite there with
pytest.  It prints the pytest summary and, with --out, writes
the pass / skip / fail counts and the failing test ids as JSON.  Nothing of
the reference is written into this repository.
"""
from __future__ import annotations

import argparse
import json
import pathlib
import re
import shutil
import subprocess
import sys
import tempfile

HERE = pathlib.Path(__file__).resolve().parent
BUILD = HERE.parent.parent / "factor-cuda_b200" / "build"


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("reference", help="path of a checkout of the reference project")
    ap.add_argument("--out", default=None, help="write the counts here (JSON)")
    ap.add_argument("--tests", default="tests/test_adapter_v1.py", help="suite file(s) inside the reference tree")
    a = ap.parse_args()
    ref = pathlib.Path(a.reference).resolve()
    libs = [BUILD / "libfcb200.so"] + sorted(BUILD.glob("factor_cuda_pybind*.so")) + \
        sorted(BUILD.glob("factor_corr_pybind*.so"))
    if len(libs) != 3 or not all(p.exists() for p in libs):
        sys.exit(f"build the library first (python factor-cuda_b200/fcb_build.py); found {libs}")
    with tempfile.TemporaryDirectory(prefix="fc_accept_") as tmp:
        root = pathlib.Path(tmp)
        for d in ("fc", "tests", "benchmark_corpus"):
            shutil.copytree(ref / d, root / d)
        shutil.copy2(ref / "pytest.ini", root / "pytest.ini")
        (root / "build").mkdir()
        for p in libs:
            shutil.copy2(p, root / "build" / p.name)
        cmd = [sys.executable, "-m", "pytest", *a.tests.split(), "-q", "-rfEs", "-p", "no:cacheprovider"]
        r = subprocess.run(cmd, cwd=root, capture_output=True, text=True)
        out = r.stdout + r.stderr
    print(out[-6000:])
    counts = {k: int(v) for v, k in re.findall(r"(\d+) (passed|failed|skipped|error|errors|xfailed|xpassed)", out)}
    failed = sorted(set(re.findall(r"^(?:FAILED|ERROR) (\S+)", out, flags=re.M)))
    summary = {"suite": a.tests, "returncode": r.returncode, "counts": counts, "failed": failed}
    print(json.dumps(summary))
    if a.out:
        pathlib.Path(a.out).write_text(json.dumps(summary, indent=1))
    return r.returncode


if __name__ == "__main__":
    sys.exit(main())
