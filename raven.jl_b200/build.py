"""Builds libravenb200.so (sm_100a) in-tree from raven.jl_b200/csrc.

The stage kernel is instantiated once per (dim, nq) pair in separate translation units
(stage_inst.cu compiled with -DRB_DIM/-DRB_NQ) so that nvcc runs in parallel.

Usage: python raven.jl_b200/build.py [--force] [--jobs N] [--verbose-ptxas]
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libravenb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", CSRC,
              "-I", INCLUDE]
DIMS_NQS = [(d, q) for d in (1, 2, 3) for q in range(2, 9)]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    units = []
    for d, q in DIMS_NQS:
        units.append((os.path.join(CSRC, "stage_inst.cu"), os.path.join(BUILD, f"stage_d{d}_q{q}.o"),
                      [f"-DRB_DIM={d}", f"-DRB_NQ={q}"]))
    for d in (2, 3):
        units.append((os.path.join(CSRC, "serve_inst.cu"), os.path.join(BUILD, f"serve_d{d}.o"),
                      [f"-DRB_SERVE_DIM={d}"]))
    for name in ("dispatch", "reduce", "pipelined_inst", "serve", "utilities", "mortar", "relaxation", "diagnostics",
                 "halo", "api"):
        units.append((os.path.join(CSRC, f"{name}.cu"), os.path.join(BUILD, f"{name}.o"), []))
    return units


def _deps_mtime():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "raven_b200.h")]
    return max(os.path.getmtime(f) for f in files)


def _compile(unit, extra, verbose):
    src, obj, defs = unit
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + defs + extra + ["-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{r.stderr}")
    return obj, r.stderr


def build(force=False, jobs=None, verbose=False, extra=()):
    """Compiles every CUDA translation unit for sm_100a and links the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    units = _sources()
    jobs = jobs or max(2, min(len(units), os.cpu_count() or 4))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, log in ex.map(lambda u: _compile(u, list(extra), verbose), units):
            logs.append((obj, log))
    objs = [u[1] for u in units]
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    if verbose:
        for obj, log in logs:
            if log.strip():
                print(f"== {os.path.basename(obj)}\n{log}")
    return LIB


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--force", action="store_true")
    p.add_argument("--jobs", type=int, default=None)
    p.add_argument("--verbose-ptxas", action="store_true")
    a = p.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose_ptxas))


if __name__ == "__main__":
    sys.exit(main())
