"""Builds rbps_b200/librbps_b200.so from rbps_b200/csrc for sm_100a.

    python -m rbps_b200.build [--force]

Each translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; the FP64 step
kernels and the GJK kernels (double arithmetic in every precision) are
compiled with ``-fmad=false`` so double arithmetic rounds like the
reference's x86-64 build (no FMA contraction).  Objects are rebuilt only
when a source or header is newer than the library.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librbps_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
          "-I" + INCLUDE, "-I" + CSRC]

UNITS = {
    "engine_f64.cu": ["-fmad=false"],
    "engine_f32.cu": [],
    "gjk_f64.cu": ["-fmad=false"],
    "gjk_f32.cu": ["-fmad=false"],
    "batch.cu": [],
    "bp_api.cu": [],
    "selftest.cu": [],
    "sap_static.cu": [],
    "quickhull.cpp": [],
}


def _deps():
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _compile(unit, extra, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if unit.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False, verbose=False):
    """Compiles and links the library if it is missing or stale; returns its path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True))
    sys.exit(0)
