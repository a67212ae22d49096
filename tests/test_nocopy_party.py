"""A GPU party among CPU parties: tests/cpp/gpu_party.cpp plays one party of
replicated 3PC (include/orq_b200/party.hpp over the orqcu_party_* entries),
the other two are the reference itself (oracle/_ref/ref_driver), and they talk
over ORQ's NoCopy wire (include/orq_b200/nocopy.hpp).

CPU: the program compiles; the key exchange of setup_random_generation runs
against two reference parties and the GPU party ends up with the keys they
drew (`setup` op; no GPU needed).
GPU: with the GPU party at each rank in turn, every party's shares of the
reference driver's prims sequence equal the all-CPU run's (the golden
digests), and the replicated copies held by a CPU and the GPU party agree.
"""
import ctypes
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
SRC = os.path.join(ROOT, "tests", "cpp", "gpu_party.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build")
LIBDIR = os.path.join(ROOT, "orq_b200")


def build() -> str:
    from orq_b200 import build as b

    b.build()
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "gpu_party")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-pthread", "-I",
           os.path.join(ROOT, "include", "orq_b200"), SRC, "-L", LIBDIR, "-lorq_cuda", f"-Wl,-rpath,{LIBDIR}",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def _ref_driver():
    from oracle import run_ref

    if not os.path.exists(run_ref.DRIVER):
        pytest.skip("reference driver not built (make -C oracle ref)")
    return run_ref


def _keygen(seed, party, call):
    lib = ctypes.CDLL(os.path.join(LIBDIR, "liborq_cuda.so"))
    buf = (ctypes.c_uint8 * 32)()
    assert lib.orqcu_keygen(ctypes.c_uint64(seed), party, call, buf) == 0
    return bytes(buf).hex()


def test_gpu_party_compiles():
    assert os.path.exists(build())


@pytest.mark.parametrize("rank", [0, 1, 2])
def test_key_exchange_with_reference_parties(rank):
    """setup_random_generation's exchange against two reference parties: the
    GPU party's received keys are the ones the reference parties drew."""
    run_ref = _ref_driver()
    exe = build()
    seed = 5
    tmp, _ = run_ref.run("setup", 0, 1, shim_seed=seed, timeout=120, exe={rank: exe}, parser=None)
    keys = dict(line.split() for line in open(os.path.join(tmp, f"p{rank}.keys")))
    own_call = {0: 5, 1: 2, 2: 1}  # the pairwise key's keygen call of each party
    want = {"local": _keygen(seed, rank, 0), "own": _keygen(seed, rank, own_call[rank]),
            "prev": _keygen(seed, (rank + 2) % 3, own_call[(rank + 2) % 3])}
    groups = {"g01": ({0, 1}, (0, 1)), "g02": ({0, 2}, (0, 2)), "g12": ({1, 2}, (1, 1)), "g012": ({0, 1, 2}, (0, 3))}
    for name, (members, (who, call)) in groups.items():
        if rank in members:
            want[name] = _keygen(seed, who, call)
    assert keys == want


@pytest.mark.gpu
@pytest.mark.parametrize("rank", [0, 1, 2])
@pytest.mark.parametrize("tag", ["prims_n1000", "prims_n300000"])
def test_gpu_party_prims_match_reference_shares(digests, rank, tag):
    """Two reference parties and one GPU party run the prims sequence; all
    three parties' shares equal the all-CPU run's digest for digest, and the
    copies of each distinct share held by two parties agree."""
    run_ref = _ref_driver()
    exe = build()
    m = digests[tag]["meta"]
    dumps, _ = run_ref.run(m["op"], m["n"], m["data_seed"], shim_seed=m["shim_seed"], timeout=900,
                           exe={rank: exe}, parser=run_ref.parse_dump)
    want = digests[tag]["arrays"]
    assert set(dumps[rank]) == set(want)
    for name, arrs in want.items():
        if name.split("_", 1)[1].startswith("open"):
            for p in range(3):
                got = hashlib.sha256(np.ascontiguousarray(dumps[p][name][0]).tobytes()).hexdigest()
                assert got == arrs[0], (name, p)
            continue
        S = run_ref.distinct_shares(dumps, name)
        assert [hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() for a in S] == arrs, name
