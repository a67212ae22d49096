"""The C++ drop-in boundary: a program written against ORQ's C++ API
(tests/cpp/test_loopback.cpp) compiled against the loopback orq.h
(include/orq_b200/) and linked with liborq_cuda.so.

CPU: the C header compiles as C, the C++ program compiles and links (every
entry point it uses is exported), and it fails cleanly without a GPU.
GPU: the reference tests' opened-value checks pass, and the reference
driver's prims / radix / join_agg sequences, run from C++, produce the
reference's own shares (the golden digests).
"""
import hashlib
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_loopback.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build")
LIBDIR = os.path.join(ROOT, "orq_b200")


def build(variant: str = "default") -> str:
    """Compile the C++ program; the "radix" variant sets the sort protocol of
    EncodedTable sorts to RADIXSORT, as the reference driver is built; "p2" /
    "p4" build it for Beaver 2PC / Fantastic-4PC (PROTOCOL_NUM)."""
    from orq_b200 import build as b

    b.build()
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, f"test_loopback_{variant}")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include", "orq_b200"),
           SRC, "-L", LIBDIR, "-lorq_cuda", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    if variant == "radix":
        cmd.insert(1, "-DORQ_B200_DEFAULT_SORT_PROTO=RADIXSORT")
    elif variant in ("p2", "p4"):
        cmd.insert(1, f"-DPROTOCOL_NUM={variant[1]}")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_c_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "orq_cuda.h"\nint main(void) { return orqcu_version() < 0; }\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-L", LIBDIR, "-lorq_cuda", f"-Wl,-rpath,{LIBDIR}", "-o", str(tmp_path / "t")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("variant", ["default", "radix", "p2", "p4"])
def test_cpp_program_compiles_and_links(variant):
    exe = build(variant)
    assert os.path.exists(exe)


def test_cpp_program_fails_cleanly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("host-only check")
    exe = build()
    r = subprocess.run([exe, "check"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "error:" in r.stderr


def read_dump(path):
    """Records of test_loopback's Dumper: name, width, n, count, arrays."""
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (nl,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off:off + nl].decode()
        off += nl
        w, n, k = struct.unpack_from("<IQI", data, off)
        off += 16
        arrs = []
        for _ in range(k):
            arrs.append(np.frombuffer(data, dtype=dt[w], count=n, offset=off))
            off += n * w
        out[name] = arrs
    return out


@pytest.mark.gpu
def test_cpp_program_reference_checks_pass():
    exe = build()
    r = subprocess.run([exe, "check"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    lines = r.stdout.splitlines()
    assert not [ln for ln in lines if ln.startswith("FAIL")]
    assert sum(ln.startswith("OK ") for ln in lines) >= 40


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["prims_n1000", "prims_n300000", "radix_n20000_b40", "join_agg_n16",
                                 "join_agg_n300"])
def test_cpp_program_matches_reference_shares(digests, tmp_path, tag):
    """The reference driver's sequence, written against ORQ's C++ API and run
    through the C ABI, gives the reference's shares digest for digest."""
    exe = build("radix")
    m = digests[tag]["meta"]
    out = tmp_path / "d.bin"
    env = dict(os.environ, ORQ_SEED=str(m["shim_seed"]))
    r = subprocess.run([exe, "dump", m["op"], str(m["n"]), str(m["data_seed"]), str(out), str(m["bits"])],
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    got = read_dump(out)
    want = digests[tag]["arrays"]
    assert set(got) == set(want)
    for name, arrs in got.items():
        assert [hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() for a in arrs] == want[name], name


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["p2_prims_n1000", "p2_prims_n300000", "p4_prims_n1000", "p4_prims_n300000"])
def test_cpp_program_np_matches_reference_shares(digests, tmp_path, tag):
    """The 2PC / 4PC prims sequence of the reference's PROTOCOL_NUM=2|4 build,
    written against ORQ's C++ API compiled with the same PROTOCOL_NUM, gives
    the reference's distinct shares (S0, S1 or X0..X3) digest for digest."""
    m = digests[tag]["meta"]
    exe = build(f"p{m['parties']}")
    out = tmp_path / "d.bin"
    env = dict(os.environ, ORQ_SEED=str(m["shim_seed"]))
    r = subprocess.run([exe, "dump", m["op"], str(m["n"]), str(m["data_seed"]), str(out)],
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    got = read_dump(out)
    want = digests[tag]["arrays"]
    assert set(got) == set(want)
    for name, arrs in got.items():
        assert [hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() for a in arrs] == want[name], name
