"""The C restatement (oracle/) against the reference's own outputs.

Golden vectors come from ORQ's code run as three party processes
(tests/golden/make_golden.py); the AES keystream against Python
`cryptography` known answers.
"""
import hashlib

import numpy as np
import pytest

from replay import (OracleBackend, replay_agg, replay_bitonic, replay_cmprows, replay_compare,
                    replay_prims, replay_qsort, replay_radix, replay_relops, replay_rows, replay_tsort, same)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_aes_gcm_keystream_kat(oracle_lib, aes_kat):
    from oracle.oracle import Oracle

    o = Oracle(0)
    lib = o.lib
    import ctypes

    for case in aes_kat:
        key = bytes.fromhex(case["key"])
        rk = (ctypes.c_uint32 * 60)()
        lib.oro_aes256_expand(key, rk)
        buf = np.zeros(case["nbytes"], dtype=np.uint8)
        lib.oro_keystream(rk, ctypes.c_uint64(case["nonce0"]), buf.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_size_t(case["nbytes"]))
        assert buf[:64].tobytes().hex() == case["head"]
        assert hashlib.sha256(buf.tobytes()).hexdigest() == case["sha256"]


def test_fips197_aes256_vector(oracle_lib):
    import ctypes

    from oracle.oracle import Oracle

    lib = Oracle(0).lib
    rk = (ctypes.c_uint32 * 60)()
    lib.oro_aes256_expand(bytes(range(32)), rk)
    out = ctypes.create_string_buffer(16)
    lib.oro_aes256_encrypt(rk, bytes.fromhex("00112233445566778899aabbccddeeff"), out)
    assert out.raw.hex() == "8ea2b7ca516745bfeafc49904b496089"  # FIPS-197 C.3


@pytest.mark.parametrize("tag,n,seed,shim", [("prims_n1000", 1000, 7, 1), ("prims_n1", 1, 11, 2)])
def test_prims_match_reference_shares(oracle_lib, golden, tag, n, seed, shim):
    out = replay_prims(OracleBackend(shim), n, seed)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


def test_prims_large_match_reference_digests(oracle_lib, digests):
    d = digests["prims_n300000"]
    m = d["meta"]
    out = replay_prims(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag", ["radix_n1000_b40", "radix_n513_b8", "radix_n64_b64"])
def test_radix_matches_reference_shares(oracle_lib, golden, digests, tag):
    m = digests[tag]["meta"]
    out, (key, p1, p2) = replay_radix(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"])
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    # and the plaintext semantics: stable sort on the signed key
    order = np.argsort(key.view(np.int64), kind="stable")
    assert same(out["open_key"][0], key[order])
    assert same(out["open_pay1"][0], p1[order])


def test_radix_large_matches_reference_digests(oracle_lib, digests):
    d = digests["radix_n20000_b40"]
    m = d["meta"]
    out, _ = replay_radix(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


def test_gen_perm_is_a_permutation(oracle_lib):
    from oracle.oracle import G01, Oracle

    o = Oracle(5)
    for n in (0, 1, 2, 3, 100, 1024, 4097):
        p, draws = o.gen_perm(G01, n)
        assert sorted(p.tolist()) == list(range(n))
        assert draws >= n


@pytest.mark.parametrize("tag,w", [("compare32_n1000", 4), ("compare64_n333", 8)])
def test_compare_matches_reference_shares(oracle_lib, golden, digests, tag, w):
    m = digests[tag]["meta"]
    out, (x, y) = replay_compare(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    assert np.array_equal(out["open_eq"][0], (x == y).astype(x.dtype))
    assert np.array_equal(out["open_gt"][0], (x.view(sd) > y.view(sd)).astype(x.dtype))


def test_compare_large_matches_reference_digests(oracle_lib, digests):
    d = digests["compare32_n100000"]
    m = d["meta"]
    out, _ = replay_compare(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], 4)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,w,desc", [("bitonic32_n256", 4, False), ("bitonic64_n64", 8, False),
                                        ("bitonic32_desc_n128", 4, True)])
def test_bitonic_matches_reference_shares(oracle_lib, golden, digests, tag, w, desc):
    m = digests[tag]["meta"]
    out, key = replay_bitonic(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w, desc)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    want = np.sort(key.view(sd))
    assert same(out["open_key"][0].view(sd), want[::-1] if desc else want)


def test_bitonic_large_matches_reference_digests(oracle_lib, digests):
    d = digests["bitonic32_n4096"]
    m = d["meta"]
    out, _ = replay_bitonic(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], 4)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,op", [("agg_fwd_n256", "agg_fwd"), ("agg_rev_n128", "agg_rev"),
                                    ("agg_nokey_n64", "agg_nokey")])
def test_aggregate_matches_reference_shares(oracle_lib, golden, digests, tag, op):
    m = digests[tag]["meta"]
    out, x = replay_agg(OracleBackend(m["shim_seed"]), op, m["n"], m["data_seed"])
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


@pytest.mark.parametrize("tag,op", [("agg_fwd_n4096", "agg_fwd"), ("agg_rev_n4096", "agg_rev")])
def test_aggregate_large_matches_reference_digests(oracle_lib, digests, tag, op):
    d = digests[tag]
    m = d["meta"]
    out, _ = replay_agg(OracleBackend(m["shim_seed"]), op, m["n"], m["data_seed"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


def test_aggregate_forward_sum_is_group_total(oracle_lib):
    """plaintext meaning: after the forward network the first row of every
    key group holds the group's sum"""
    n = 512
    out, x = replay_agg(OracleBackend(3), "agg_fwd", n, 5)
    k0, v = x["k0"], x["va1"]
    o1 = out["open_o1"][0]
    heads = np.nonzero(np.r_[True, k0[1:] != k0[:-1]])[0]
    for h in heads:
        assert int(o1[h]) == int(v[k0 == k0[h]].sum())


@pytest.mark.parametrize("tag,desc", [("radix_desc_n100_b40", True), ("radix_desc_n64_b64", True),
                                      ("radix_n33_b1", False)])
def test_radix_desc_and_single_bit_match_reference_shares(oracle_lib, golden, digests, tag, desc):
    m = digests[tag]["meta"]
    out, (key, _, _) = replay_radix(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"], desc)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


def test_radix_desc_large_matches_reference_digests(oracle_lib, digests):
    d = digests["radix_desc_n3000_b16"]
    m = d["meta"]
    out, _ = replay_radix(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"], True)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,op", [("tsort_n64", "tsort"), ("tsort_qs_n64", "tsort_qs"),
                                    ("distinct_n64", "distinct")])
def test_table_sort_and_distinct_match_reference_shares(oracle_lib, golden, digests, tag, op):
    m = digests[tag]["meta"]
    out, _ = replay_tsort(OracleBackend(m["shim_seed"]), op, m["n"], m["data_seed"])
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


@pytest.mark.parametrize("tag,op", [("tsort_n200", "tsort"), ("tsort_qs_n3000", "tsort_qs"),
                                    ("distinct_n5000", "distinct")])
def test_table_sort_and_distinct_large_match_reference_digests(oracle_lib, digests, tag, op):
    d = digests[tag]
    m = d["meta"]
    out, _ = replay_tsort(OracleBackend(m["shim_seed"]), op, m["n"], m["data_seed"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


def test_table_sort_plaintext_order(oracle_lib):
    """rows ordered by (c0 asc, c1 desc, c2 asc), stable, data carried"""
    n = 128
    out, (v0, v1, v2, va, vb) = replay_tsort(OracleBackend(9), "tsort", n, 4)
    order = sorted(range(n), key=lambda i: (int(v0[i]), -int(v1[i]), int(v2[i])))
    assert out["open_c1"][0].tolist() == [int(v1[i]) for i in order]
    assert sorted(out["open_da"][0].tolist()) == sorted(int(x) for x in va)


@pytest.mark.parametrize("tag,w", [("relops32_n500", 4), ("relops64_n333", 8)])
def test_relational_operators_match_reference_shares(oracle_lib, golden, digests, tag, w):
    """operator== != >= <= (b_shared_vector.h:493-580), share for share"""
    m = digests[tag]["meta"]
    out, (x, y) = replay_relops(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    xs, ys = x.view(sd), y.view(sd)
    for nm, want in (("eq", xs == ys), ("ne", xs != ys), ("ge", xs >= ys), ("le", xs <= ys)):
        assert np.array_equal(out["open_" + nm][0], want.astype(x.dtype)), nm


@pytest.mark.parametrize("tag,w", [("rows32_n256", 4), ("rows64_n128", 8)])
def test_bitonic_rows_match_reference_shares(oracle_lib, golden, digests, tag, w):
    """bitonic_sort over two keys with A and B data (sorting.h:266-353)"""
    m = digests[tag]["meta"]
    out, ins = replay_rows(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    k0, k1 = ins[0].view(sd), ins[1].view(sd)
    rows = sorted(zip(k0.tolist(), (-k1.astype(object)).tolist(), ins[2].tolist(), ins[3].tolist(),
                      ins[4].tolist()))
    got_k0 = out["open_k0"][0].view(sd).tolist()
    got_k1 = out["open_k1"][0].view(sd).tolist()
    assert got_k0 == [r[0] for r in rows]
    assert got_k1 == [-r[1] for r in rows]
    got = sorted(zip(got_k0, got_k1, out["open_b0"][0].tolist(), out["open_a0"][0].tolist(),
                     out["open_a1"][0].tolist()))
    assert got == sorted(zip(k0.tolist(), k1.tolist(), ins[2].tolist(), ins[3].tolist(), ins[4].tolist()))


def test_bitonic_rows_large_matches_reference_digests(oracle_lib, digests):
    d = digests["rows32_n2048"]
    m = d["meta"]
    out, _ = replay_rows(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], 4)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


def test_bitonic_rows_one_key_equals_bitonic(oracle_lib, golden):
    """the multi-column network on one key and no data is the one-column sort"""
    from oracle.oracle import splitmix64_fast

    o = OracleBackend(2).o
    key = splitmix64_fast(7, 256).astype(np.uint32)
    kb = o.secret_share(key, False, 0)
    o.bitonic_sort_rows([kb], [False])
    assert same(np.stack(kb), golden["bitonic32_n256/key"])


@pytest.mark.parametrize("tag,w", [("cmprows32_n500", 4), ("cmprows64_n333", 8)])
def test_compare_rows_swap_multiplex_match_reference_shares(oracle_lib, golden, digests, tag, w):
    """compare_rows, extend_lsb, multiplex (B, A) and swap (B, A), share for share"""
    m = digests[tag]["meta"]
    out, (x0, y0, x1, y1, u, v) = replay_cmprows(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    a0, b0, a1, b1 = x0.view(sd), y0.view(sd), x1.view(sd), y1.view(sd)
    want = (a0 > b0) | ((a0 == b0) & (b1 > a1))  # key 0 ASC, key 1 DESC
    assert np.array_equal(out["open_gt"][0], want.astype(x0.dtype))
    assert np.array_equal(out["open_x1"][0], np.where(want, y1, x1))
    assert np.array_equal(out["open_y1"][0], np.where(want, x1, y1))
    assert np.array_equal(out["open_u"][0], np.where(want, v, u))
    assert np.array_equal(out["open_v"][0], np.where(want, u, v))


def test_compare_rows_large_matches_reference_digests(oracle_lib, digests):
    d = digests["cmprows64_n20000"]
    m = d["meta"]
    out, _ = replay_cmprows(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], 8)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,w,desc", [("qsort_n1000_b40", 8, False), ("qsort_desc_n333_b64", 8, True),
                                        ("qsort32_n500", 4, False), ("qsort_n2_b40", 8, False)])
def test_quicksort_matches_reference_shares(oracle_lib, golden, digests, tag, w, desc):
    """quicksort (quicksort.h:61-246): shuffle, opened pivot comparisons,
    Lomuto partitions, remove_padding and invert, share for share"""
    m = digests[tag]["meta"]
    out, (key, p1, p2) = replay_qsort(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"], w, desc)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    sd = {4: np.int32, 8: np.int64}[w]
    k = key.view(sd)
    o = np.argsort(-k if desc else k, kind="stable")
    assert np.array_equal(out["open_key"][0].view(sd), k[o])
    assert np.array_equal(out["open_pay1"][0].view(p1.dtype), p1[o])


@pytest.mark.parametrize("tag,w", [("qsort_n20000_b40", 8), ("qsort32_n30000", 4)])
def test_quicksort_large_matches_reference_digests(oracle_lib, digests, tag, w):
    d = digests[tag]
    m = d["meta"]
    out, _ = replay_qsort(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], m["bits"], w)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,w", [("a2b32_n500", 4), ("a2b64_n333", 8)])
def test_a2b_matches_reference_shares(oracle_lib, golden, digests, tag, w):
    """ASharedVector::a2b: redistribute_shares_b + ripple-carry adder, share for share"""
    from replay import replay_a2b

    m = digests[tag]["meta"]
    out, x = replay_a2b(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    assert np.array_equal(out["open_xb"][0].view(x.dtype), x)


def test_a2b_large_matches_reference_digests(oracle_lib, digests):
    from replay import replay_a2b

    d = digests["a2b64_n20000"]
    m = d["meta"]
    out, _ = replay_a2b(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], 8)
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


@pytest.mark.parametrize("tag,w", [("badd32_n500", 4), ("badd64_n333", 8)])
def test_boolean_add_sub_match_reference_shares(oracle_lib, golden, digests, tag, w):
    """BSharedVector + and - (the ripple-carry adder), share for share"""
    from replay import replay_badd

    m = digests[tag]["meta"]
    out, (x, y) = replay_badd(OracleBackend(m["shim_seed"]), m["n"], m["data_seed"], w)
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name
    assert np.array_equal(out["open_sum"][0].view(x.dtype), x + y)
    assert np.array_equal(out["open_diff"][0].view(x.dtype), x - y)


@pytest.mark.parametrize("tag", ["p2_prims_n1000", "p2_prims_n1", "p4_prims_n1000", "p4_prims_n1"])
def test_np_prims_match_reference_shares(oracle_lib, golden, digests, tag):
    """Beaver 2PC (dummy triples) and Fantastic-4PC: the restatement's shares
    of every vector of the primitive sequence equal the reference's."""
    from replay import OracleNPBackend, replay_prims_np

    m = digests[tag]["meta"]
    out = replay_prims_np(OracleNPBackend(m["shim_seed"], m["parties"]), m["n"], m["data_seed"])
    assert set(out) == set(digests[tag]["arrays"])
    for name, arr in out.items():
        assert same(arr, golden[f"{tag}/{name}"]), name


@pytest.mark.parametrize("tag", ["p2_prims_n300000", "p4_prims_n300000"])
def test_np_prims_large_match_reference_digests(oracle_lib, digests, tag):
    from replay import OracleNPBackend, replay_prims_np

    d = digests[tag]
    m = d["meta"]
    out = replay_prims_np(OracleNPBackend(m["shim_seed"], m["parties"]), m["n"], m["data_seed"])
    for name, arr in out.items():
        assert [sha(a) for a in arr] == d["arrays"][name], name


def test_serving_admission_keeps_one_large_request_in_flight():
    """The dispatcher's pick: FIFO, except that a large request waits while
    another large one runs and smaller ones within the lookahead go first."""
    from types import SimpleNamespace as NS

    from orq_b200.serve import LARGE_ROWS, LOOKAHEAD, pick_next

    big, small = NS(rows=LARGE_ROWS), NS(rows=LARGE_ROWS // 2)
    idle, runs_big, runs_small = NS(busy=False, large=False), NS(busy=True, large=True), NS(busy=True, large=False)
    assert pick_next([big, small], [idle, idle]) == 0
    assert pick_next([big, small], [runs_small, idle]) == 0
    assert pick_next([big, big, small], [runs_big, idle]) == 2
    assert pick_next([big, big], [runs_big, idle]) is None
    assert pick_next([big] * LOOKAHEAD + [small], [runs_big, idle]) is None
    assert pick_next([], [idle]) is None
