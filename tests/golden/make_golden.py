"""Generate the golden fixtures from the reference itself.

Runs ORQ's own code (oracle/_ref/ref_driver, built by `make -C oracle ref`
from the reference headers with the deterministic libsodium shim) as three
local party processes and stores each dumped share array as the three
distinct shares S0, S1, S2:

  ref_golden.npz    small cases, full arrays
  ref_digests.json  large cases, SHA-256 of every share array
  aes_gcm_kat.json  AES-256-GCM keystream known answers from Python
                    `cryptography` (FIPS-197 / SP 800-38D)

Usage: python tests/golden/make_golden.py [--only tag1,tag2]   (needs the
reference tree; run in the build container, not at test time)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import run_ref  # noqa: E402

# (tag, op, n, data_seed, shim_seed, bits, full arrays?)
CASES = [
    ("prims_n1000", "prims", 1000, 7, 1, 40, True),
    ("prims_n1", "prims", 1, 11, 2, 40, True),
    ("prims_n300000", "prims", 300000, 7, 1, 40, False),
    ("radix_n1000_b40", "radix", 1000, 7, 3, 40, True),
    ("radix_n513_b8", "radix", 513, 7, 3, 8, True),
    ("radix_n64_b64", "radix", 64, 5, 4, 64, True),
    ("radix_n20000_b40", "radix", 20000, 9, 5, 40, False),
    ("shuffle_n1000", "shuffle", 1000, 7, 6, 40, True),
    ("compare32_n1000", "compare32", 1000, 7, 2, 32, True),
    ("compare64_n333", "compare64", 333, 8, 3, 64, True),
    ("compare32_n100000", "compare32", 100000, 9, 4, 32, False),
    ("bitonic32_n256", "bitonic32", 256, 7, 2, 32, True),
    ("bitonic64_n64", "bitonic64", 64, 5, 3, 64, True),
    ("bitonic32_desc_n128", "bitonic32_desc", 128, 6, 4, 32, True),
    ("bitonic32_n4096", "bitonic32", 4096, 10, 5, 32, False),
    ("agg_fwd_n256", "agg_fwd", 256, 7, 2, 64, True),
    ("agg_rev_n128", "agg_rev", 128, 8, 3, 64, True),
    ("agg_nokey_n64", "agg_nokey", 64, 9, 4, 64, True),
    ("agg_fwd_n4096", "agg_fwd", 4096, 11, 5, 64, False),
    ("agg_rev_n4096", "agg_rev", 4096, 12, 6, 64, False),
    ("radix_desc_n100_b40", "radix_desc", 100, 7, 3, 40, True),
    ("radix_desc_n64_b64", "radix_desc", 64, 7, 3, 64, True),
    ("radix_n33_b1", "radix", 33, 7, 3, 1, True),
    ("radix_desc_n3000_b16", "radix_desc", 3000, 8, 4, 16, False),
    ("tsort_n64", "tsort", 64, 5, 4, 64, True),
    ("tsort_n200", "tsort", 200, 6, 5, 64, False),
    ("distinct_n64", "distinct", 64, 5, 4, 64, True),
    ("distinct_n5000", "distinct", 5000, 6, 5, 64, False),
    ("join_agg_n16", "join_agg", 16, 7, 2, 64, True),
    ("join_agg_n300", "join_agg", 300, 8, 3, 64, False),
    ("relops32_n500", "relops32", 500, 7, 2, 32, True),
    ("relops64_n333", "relops64", 333, 8, 3, 64, True),
    ("rows32_n256", "rows32", 256, 7, 2, 32, True),
    ("rows64_n128", "rows64", 128, 8, 3, 64, True),
    ("rows32_n2048", "rows32", 2048, 9, 4, 32, False),
    ("cmprows32_n500", "cmprows32", 500, 7, 2, 32, True),
    ("cmprows64_n333", "cmprows64", 333, 8, 3, 64, True),
    ("cmprows64_n20000", "cmprows64", 20000, 9, 4, 64, False),
    ("qsort_n1000_b40", "qsort", 1000, 7, 3, 40, True),
    ("qsort_desc_n333_b64", "qsort_desc", 333, 8, 4, 64, True),
    ("qsort32_n500", "qsort32", 500, 9, 5, 32, True),
    ("qsort_n2_b40", "qsort", 2, 5, 2, 40, True),
    ("qsort_n20000_b40", "qsort", 20000, 10, 6, 40, False),
    ("qsort32_n30000", "qsort32", 30000, 11, 7, 32, False),
    ("tsort_qs_n64", "tsort_qs", 64, 5, 4, 64, True),
    ("tsort_qs_n3000", "tsort_qs", 3000, 6, 5, 64, False),
    ("tshuffle_n64", "tshuffle", 64, 7, 2, 64, True),
    ("tshuffle_n1000", "tshuffle", 1000, 8, 3, 64, False),
    ("a2b32_n500", "a2b32", 500, 7, 2, 32, True),
    ("a2b64_n333", "a2b64", 333, 8, 3, 64, True),
    ("a2b64_n20000", "a2b64", 20000, 9, 4, 64, False),
    ("badd32_n500", "badd32", 500, 7, 2, 32, True),
    ("badd64_n333", "badd64", 333, 8, 3, 64, True),
    # the 2^22-row headline workload and 2^20: every Fisher-Yates permutation
    # spans many 2^20-draw getNext buffers (about 127 at 2^22)
    ("radix_n1048576_b40", "radix", 1 << 20, 7, 7, 40, False),
    ("radix_n4194304_b40", "radix", 1 << 22, 7, 7, 40, False),
    ("qsort_n1048576_b40", "qsort", 1 << 20, 7, 7, 40, False),
]

# Beaver 2PC (dummy triples) and Fantastic-4PC primitive sequences
# (oracle/ref_driver_np.cpp): (tag, parties, n, data_seed, shim_seed, full?)
NP_CASES = [
    ("p2_prims_n1000", 2, 1000, 7, 3, True),
    ("p2_prims_n1", 2, 1, 11, 4, True),
    ("p2_prims_n300000", 2, 300000, 9, 5, False),
    ("p4_prims_n1000", 4, 1000, 7, 3, True),
    ("p4_prims_n1", 4, 1, 11, 4, True),
    ("p4_prims_n300000", 4, 300000, 9, 5, False),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def aes_kat():
    from cryptography.hazmat.primitives.ciphers.aead import AESGCM

    out = []
    rng = np.random.default_rng(2024)
    for nonce0, nbytes in ((0, 48), (5, (1 << 20) + 37), (2**33 + 7, 4096)):
        key = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        ks = b""
        off, nonce = 0, nonce0
        while off < nbytes:
            ln = min(1 << 20, nbytes - off)
            iv = nonce.to_bytes(8, "little") + b"\0\0\0\0"
            ks += AESGCM(key).encrypt(iv, b"\0" * ln, None)[:ln]
            off += ln
            nonce += 1
        out.append({"key": key.hex(), "nonce0": nonce0, "nbytes": nbytes,
                    "head": ks[:64].hex(), "sha256": hashlib.sha256(ks).hexdigest()})
    return out


def main():
    # --only tag1,tag2 regenerates those cases and keeps every other fixture
    only = None
    if "--only" in sys.argv:
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    arrays = {}
    digests = {}
    if only:
        with np.load(os.path.join(HERE, "ref_golden.npz")) as z:
            arrays = {k: z[k] for k in z.files}
        with open(os.path.join(HERE, "ref_digests.json")) as f:
            digests = json.load(f)
    for tag, op, n, dseed, sseed, bits, full in CASES:
        if only and tag not in only:
            continue
        dumps, _ = run_ref.run(op, n, dseed, shim_seed=sseed, bits=bits)
        meta = {"op": op, "n": n, "data_seed": dseed, "shim_seed": sseed, "bits": bits}
        digests[tag] = {"meta": meta, "arrays": {}}
        for name in dumps[0]:
            if name.startswith("open_") or "open" in name:
                S = [dumps[0][name][0]]
            else:
                S = run_ref.distinct_shares(dumps, name)
            stacked = np.stack(S)
            digests[tag]["arrays"][name] = [digest(s) for s in S]
            if full:
                arrays[f"{tag}/{name}"] = stacked
        print(tag, "ok", flush=True)
    for tag, npar, n, dseed, sseed, full in NP_CASES:
        if only and tag not in only:
            continue
        dumps, _ = run_ref.run_np(npar, "prims", n, dseed, shim_seed=sseed)
        meta = {"op": "prims", "parties": npar, "n": n, "data_seed": dseed, "shim_seed": sseed}
        digests[tag] = {"meta": meta, "arrays": {}}
        for name in dumps[0]:
            if "open" in name:
                S = [dumps[0][name][0]]
            else:
                S = run_ref.distinct_shares_np(dumps, name, npar)
            digests[tag]["arrays"][name] = [digest(s) for s in S]
            if full:
                arrays[f"{tag}/{name}"] = np.stack(S)
        print(tag, "ok", flush=True)
    np.savez_compressed(os.path.join(HERE, "ref_golden.npz"), **arrays)
    with open(os.path.join(HERE, "ref_digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "aes_gcm_kat.json"), "w") as f:
        json.dump(aes_kat(), f, indent=1)


if __name__ == "__main__":
    main()
