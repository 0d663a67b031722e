"""Build libfcb200.so and the drop-in pybind11 modules in-tree.

    python factor-cuda_b200/fcb_build.py [--force] [-j N]

Outputs go to ``factor-cuda_b200/build/``:
  * ``libfcb200.so``                 -- every CUDA kernel + the C ABI (include/fcb200.h),
                                        compiled for sm_100a only;
  * ``factor_cuda_pybind<ext>``      -- drop-in for the reference module of that name;
  * ``factor_corr_pybind<ext>``      -- drop-in for the reference module of that name.
Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import subprocess
import sys
import sysconfig

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "build"
OBJ = BUILD / "obj"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I", str(CSRC)]

CU_SOURCES = sorted(p.name for p in CSRC.glob("*.cu"))
PYBIND_MODULES = {"factor_cuda_pybind": "pybind_factor_cuda.cpp",
                  "factor_corr_pybind": "pybind_factor_corr.cpp"}


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def lib_path() -> pathlib.Path:
    return BUILD / "libfcb200.so"


def ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> pathlib.Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    hdrs = _headers()
    jobs = jobs or min(8, os.cpu_count() or 4)

    def compile_one(src: str) -> pathlib.Path:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([NVCC, *NVCC_FLAGS, "-c", str(s), "-o", str(o)])
            if verbose:
                print(f"  nvcc {src}")
        return o

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, CU_SOURCES))
    lib = lib_path()
    if force or _stale(lib, objs):
        # link to a temporary name and rename: a process that loads the
        # library meanwhile sees the old file or the new one, never a partial one
        tmp = lib.with_name(lib.name + ".tmp")
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(tmp), *map(str, objs),
              "-cudart", "static"])
        os.replace(tmp, lib)
        if verbose:
            print(f"  link {lib.name}")

    import pybind11
    py_inc = sysconfig.get_paths()["include"]
    for mod, src in PYBIND_MODULES.items():
        out = BUILD / (mod + ext_suffix())
        s = CSRC / src
        if force or _stale(out, [s, lib] + hdrs):
            tmp = out.with_name(out.name + ".tmp")
            _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
                  "-I", py_inc, "-I", pybind11.get_include(), "-I", str(INCLUDE),
                  str(s), "-o", str(tmp), "-L", str(BUILD), "-lfcb200", "-Wl,-rpath,$ORIGIN"])
            os.replace(tmp, out)
            if verbose:
                print(f"  g++ {out.name}")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    p = build(force=a.force, jobs=a.j, verbose=True)
    print(p)
    sys.exit(0)
