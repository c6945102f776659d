"""Build libklft_b200.so (sm_100a) and the C++ host binaries in-tree.

    python -m klft_b200.build [--force] [--jobs N]

Each CUDA translation unit under csrc/ is compiled separately with nvcc for
sm_100a, in parallel, then linked into klft_b200/libklft_b200.so.  The host
binaries (metropolis, hmc) go to klft_b200/bin/.  Objects live in
klft_b200/_build/.  Rebuilds only what changed (source or any header newer than
the object).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libklft_b200.so")
BIN = os.path.join(PKG, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                  "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    hs += glob.glob(os.path.join(HOST, "*.hpp")) + glob.glob(os.path.join(ROOT, "include", "klft", "*.hpp"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    headers = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(HOST, "lib_*.cpp")))
    objs, todo = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            todo.append((s, o))
    log = []
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_run, [NVCC] + NVFLAGS + (["-x", "cu"] if s.endswith(".cpp") else []) + ["-c", s, "-o", o])
                for s, o in todo]
        for f in futs:
            log.append(f.result())
    if force or todo or _stale(LIB, objs):
        log.append(_run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]))
    for prog in sorted(glob.glob(os.path.join(HOST, "main_*.cpp"))):
        name = os.path.basename(prog)[len("main_"):-len(".cpp")]
        exe = os.path.join(BIN, name)
        if force or _stale(exe, [prog, LIB] + headers):
            log.append(_run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), prog, "-o", exe,
                             "-L" + PKG, "-lklft_b200", "-Wl,-rpath,$ORIGIN/..",
                             "-L/usr/local/cuda/lib64", "-lcudart"]))
    out = "".join(log)
    if verbose:
        print(out)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(a.force, a.jobs, a.verbose)
    print(LIB)


if __name__ == "__main__":
    sys.exit(main())
