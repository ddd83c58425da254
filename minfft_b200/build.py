"""Builds the engine's shared libraries in-tree with nvcc for sm_100a.

    python -m minfft_b200.build            # both precisions
    python -m minfft_b200.build --jobs 8

Outputs ``minfft_b200/lib/libminfft_b200.so`` (double; reference default
precision) and ``minfft_b200/lib/libminfft_b200_single.so`` (float; the
reference's MINFFT_SINGLE build).  Objects go to ``minfft_b200/_build/``.
Every object is rebuilt when its source or any header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB_NAMES = {False: "libminfft_b200.so", True: "libminfft_b200_single.so"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def flags(single: bool):
    return ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden",
            "-I", CSRC, "-I", INCLUDE, f"-DMINFFT_SINGLE={1 if single else 0}", "--expt-relaxed-constexpr"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, single: bool, verbose: bool):
    tag = "single" if single else "double"
    obj = os.path.join(BUILD, tag, os.path.basename(src)[:-3] + ".o")
    if not _stale(obj, [src, *headers()]):
        return obj, None
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    cmd = [nvcc(), *flags(single), "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} ({tag}):\n{r.stdout}{r.stderr}")
    return obj, (r.stderr if verbose else None)


def build(jobs: int = 0, verbose: bool = False, precisions=(False, True)) -> list:
    jobs = jobs or max(1, os.cpu_count() or 1)
    os.makedirs(LIBDIR, exist_ok=True)
    libs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {single: [ex.submit(_compile, s, single, verbose) for s in sources()] for single in precisions}
        for single in precisions:
            objs = []
            for f in futs[single]:
                obj, log = f.result()
                objs.append(obj)
                if log:
                    sys.stderr.write(log)
            lib = os.path.join(LIBDIR, LIB_NAMES[single])
            if _stale(lib, objs):
                cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-Xlinker", "-Bsymbolic", "-cudart", "static"]
                r = subprocess.run(cmd, capture_output=True, text=True)
                if r.returncode != 0:
                    raise RuntimeError(f"link failed for {lib}:\n{r.stdout}{r.stderr}")
            libs.append(lib)
    return libs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    ap.add_argument("--precision", choices=["both", "double", "single"], default="both")
    a = ap.parse_args()
    prec = {"both": (False, True), "double": (False,), "single": (True,)}[a.precision]
    for lib in build(a.jobs, a.verbose, prec):
        print(lib)


if __name__ == "__main__":
    main()
