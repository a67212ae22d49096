"""Beaver 2PC (dummy triples) and Fantastic-4PC on the GPU: the primitive
sequence of the reference driver (secret sharing by two owners, and_b, xor_b,
multiply_a, add_a, b2a_bit, opens at 1-, 4- and 8-byte widths) gives the
reference's own shares, and equals the restatement on sizes that exercise
ragged tails, the unaligned second half of a dummy-triple draw and several
1 MiB keystream chunks."""
import hashlib

import numpy as np
import pytest

from replay import GpuNPBackend, OracleNPBackend, replay_prims_np, same

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def orq(cuda_lib):
    import orq_b200

    return orq_b200


@pytest.mark.parametrize("tag", ["p2_prims_n1000", "p2_prims_n1", "p4_prims_n1000", "p4_prims_n1"])
def test_np_prims_match_reference_shares(orq, golden, digests, tag):
    m = digests[tag]["meta"]
    out = replay_prims_np(GpuNPBackend(m["shim_seed"], m["parties"]), m["n"], m["data_seed"])
    assert set(out) == set(digests[tag]["arrays"])
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


@pytest.mark.parametrize("tag", ["p2_prims_n300000", "p4_prims_n300000"])
def test_np_prims_large_match_reference_digests(orq, digests, tag):
    d = digests[tag]
    m = d["meta"]
    out = replay_prims_np(GpuNPBackend(m["shim_seed"], m["parties"]), m["n"], m["data_seed"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("nparties", [2, 4])
@pytest.mark.parametrize("n", [3, 17, 4097, (1 << 18) + 5, (1 << 20) + 3])
def test_np_prims_match_restatement(orq, nparties, n):
    gpu = replay_prims_np(GpuNPBackend(29, nparties), n, 41)
    cpu = replay_prims_np(OracleNPBackend(29, nparties), n, 41)
    for k in gpu:
        assert same(gpu[k], cpu[k]), (nparties, n, k)


@pytest.mark.parametrize("nparties", [2, 4])
def test_np_opened_values(orq, nparties):
    """Opened results against plaintext (the reference tests' checks)."""
    n = 1 << 16
    rng = np.random.default_rng(5)
    x = rng.integers(0, 2**63, n, dtype=np.uint64)
    y = rng.integers(0, 2**63, n, dtype=np.uint64)
    be = GpuNPBackend(3, nparties)
    xb, yb = be.share(x, False, 0), be.share(y, False, 1)
    xa, ya = be.share(x, True, 1), be.share(y, True, 0)
    with np.errstate(over="ignore"):
        assert np.array_equal(be.open(be.and_b(xb, yb), False).view(np.uint64), x & y)
        assert np.array_equal(be.open(be.mul_a(xa, ya), True).view(np.uint64), x * y)
        assert np.array_equal(be.open(be.b2a_bit(xb), True).view(np.uint64), x & np.uint64(1))


def test_np_runtime_refuses_3pc_entry_points(orq, cuda_lib):
    import ctypes

    rt = orq.NPRuntime(4, seed=1)
    t = rt.secret_share(np.arange(8, dtype=np.int64), False, 0)
    p = (ctypes.c_void_p * 3)(*[t[j].data_ptr() for j in range(3)])
    assert cuda_lib.orqcu_and_b(rt.h, 8, ctypes.c_size_t(8), p, p, p) == -1
    assert b"2PC/4PC" in cuda_lib.orqcu_last_error()
