"""Build liborq_cuda.so (sm_100a) in-tree.

Each translation unit under csrc/ is compiled separately and in parallel
(the AES kernels are large after unrolling), then linked into one shared
library next to this file. Usage: python -m orq_b200.build [-j N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liborq_cuda.so")
UNITS = ["runtime.cu", "prims.cu", "perm.cu", "radix.cu", "scan.cu", "cmp.cu", "agg.cu", "tsort.cu", "qsort.cu", "conv.cu", "proto24.cu", "party.cu", "capi.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
]


STAMP = LIB + ".sha256"


def _sources_hash() -> str:
    """Content hash of the sources and flags (copies do not keep mtimes)."""
    import hashlib

    h = hashlib.sha256(" ".join(FLAGS).encode())
    files = sorted(os.listdir(CSRC))
    hdr = os.path.join(os.path.dirname(HERE), "include", "orq_cuda.h")
    for f in [os.path.join(CSRC, x) for x in files] + [hdr]:
        if os.path.isfile(f):
            h.update(os.path.basename(f).encode())
            with open(f, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()


def is_current() -> bool:
    if not (os.path.exists(LIB) and os.path.exists(STAMP)):
        return False
    with open(STAMP) as f:
        return f.read().strip() == _sources_hash()


def _compile(unit: str, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
    cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr[-6000:]}")
    return r.stderr if verbose else obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if not force and is_current():
        return LIB
    jobs = jobs or min(len(UNITS), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        outs = list(ex.map(lambda u: _compile(u, verbose), UNITS))
    if verbose:
        for u, o in zip(UNITS, outs):
            sys.stderr.write(f"== {u}\n{o}")
    objs = [os.path.join(BUILD, u.replace(".cu", ".o")) for u in UNITS]
    tmp = LIB + ".tmp"
    r = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
                        "-o", tmp], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    os.replace(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write(_sources_hash())
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true", help="print -Xptxas -v")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))
