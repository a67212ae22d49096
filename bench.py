#!/usr/bin/env python
"""bench.py — ORQ's 3PC oblivious operators on B200.

Default workload (the headline, per GPU): 2^22 rows, uint64 key uniform in
[0, 2^40) boolean-shared, two uint32 payload columns arithmetic-shared mod
2^64, seed 7; one step = radix_sort(key, ASC, 40) followed by
oblivious_apply_elementwise_perm of both payloads, including the
Fisher–Yates generation of the 44 sharded permutations it consumes (ORQ
reserves them inside radix_sort).

Other workloads (--workload): bitonic (2^16 int32 keys, seed 1), join (A
2^22 rows inner-join B 2^24 rows, product, group-by sum/count), batch (512
ragged sorts through the batched path) and serve (continuous batching loop
with p50/p99 latency).

  value  device-resident rows/s: shares already in HBM, CUDA events on the
         runtime's stream around each of K steps (each step re-copies the
         input shares), max over ranks.
  e2e    the same through the public API with host buffers: pinned plaintext
         H2D, secret sharing, the operators, open, D2H.
  --impl reference   ORQ's own CPU code (oracle/_ref/ref_driver: three party
         processes over its socket communicator) on a bounded sample.

Multi-GPU: independent replicas (each rank runs its own workload; weak
scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "oblivious-sort rows/s (3PC, 1 B200) vs host CPU; batched p50/p99 latency"
WORKLOAD = ("3PC oblivious shuffle-based radix sort, 2^22 rows, uint64 key uniform [0,2^40) "
            "B-shared + 2 uint32 payloads A-shared mod 2^64, seed 7, per-call operators")
# T-table AES-256: 16 shared-memory lookups per round x 14 rounds (+4 in the
# last) = 228 LDS per block at one warp-wide LDS per clock per SM.
AES_LDS_PER_BLOCK = 228
DEFAULT_N = 1 << 22
# DRAM traffic of the dominant k_apply instance (padded 16-byte key + int32
# permutation, one group): dram__bytes_read.sum + dram__bytes_write.sum of one
# ncu capture of that kernel at 2^21 rows, scaled per row to the benchmarked
# size. A constant taken from that capture, not measured by this run (a bench
# run is never under ncu).
APPLY_TRAFFIC_BYTES_PER_ROW = 690.5e6 / (1 << 21)


def cpu_model():
    """The host CPU's model name and logical core count (reported beside every
    CPU figure)."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": name, "logical_cores": os.cpu_count() or 1}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("sm_max_mhz", 1965.0), "measured"
    return 6650.0, 1965.0, "fallback"


def gen_inputs(n, seed, bits):
    import numpy as np

    with np.errstate(over="ignore"):
        s = np.uint64(seed) + np.arange(1, 3 * n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z = s
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    km = np.uint64((1 << bits) - 1)
    return z[:n] & km, z[n:2 * n] & np.uint64(0xFFFFFFFF), z[2 * n:] & np.uint64(0xFFFFFFFF)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.device), "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def parse_profile(text):
    out = {}
    for line in text.strip().splitlines():
        name, launches, ms, by, bl = line.split()
        out[name] = {"launches": int(launches), "ms": float(ms), "bytes": float(by), "aes_blocks": float(bl)}
    return out


class RadixWorkload:
    """Config 2 (the headline): radix_sort(key, ASC, 40) of 2^22 rows plus two
    payload applies."""

    name = "radix"

    def __init__(self, args, seed):
        self.n, self.bits, self.seed = args.n, args.bits, seed
        self.units = self.n
        self.flush_l2 = False  # 302 MB of shares per step, larger than L2
        self.config = {"workload": WORKLOAD, "rows_per_gpu": self.n, "key_bits": self.bits, "payloads": 2,
                       "l2": "inputs larger than L2 (302 MB of shares per GPU)", "seed": 7}

    def setup(self, rt, orq):
        import numpy as np

        self.orq, self.rt, self.np = orq, rt, np
        self.key, self.p1, self.p2 = gen_inputs(self.n, self.seed, self.bits)
        self.kb = rt.secret_share_b(self.key, 0)
        self.a1 = rt.secret_share_a(self.p1, 0)
        self.a2 = rt.secret_share_a(self.p2, 0)
        self.orig = [self.kb.shares.clone(), self.a1.shares.clone(), self.a2.shares.clone()]

    def step(self):
        orq = self.orq
        self.kb.shares.copy_(self.orig[0])
        self.a1.shares.copy_(self.orig[1])
        self.a2.shares.copy_(self.orig[2])
        perm = self.sort(self.kb)
        orq.oblivious_apply_elementwise_perm(self.a1, perm)
        orq.oblivious_apply_elementwise_perm(self.a2, perm)

    def sort(self, kb):
        return self.orq.radix_sort(kb, self.orq.ASC, self.bits)

    def check(self):
        np = self.np
        ko = self.kb.open().cpu().numpy().view(np.uint64)
        return bool(np.all(ko[1:] >= ko[:-1])) and np.array_equal(np.sort(self.key), ko)

    def e2e_setup(self, dev):
        import torch

        np, n = self.np, self.n
        self.pin = [torch.from_numpy(a.view(np.int64)).pin_memory() for a in (self.key, self.p1, self.p2)]
        self.outs = [torch.empty(n, dtype=torch.int64).pin_memory() for _ in range(3)]
        self.dbuf = [torch.empty(n, dtype=torch.int64, device=dev) for _ in range(3)]
        self.h2d = self.d2h = 3 * n * 8

    def e2e_step(self):
        orq, rt = self.orq, self.rt
        for h, d in zip(self.pin, self.dbuf):
            d.copy_(h, non_blocking=True)
        k = rt.secret_share_b(self.dbuf[0], 0)
        x1 = rt.secret_share_a(self.dbuf[1], 0)
        x2 = rt.secret_share_a(self.dbuf[2], 0)
        perm = self.sort(k)
        orq.oblivious_apply_elementwise_perm(x1, perm)
        orq.oblivious_apply_elementwise_perm(x2, perm)
        for v, o in zip((k, x1, x2), self.outs):
            o.copy_(v.open(), non_blocking=True)

    def e2e_check(self):
        return bool(self.np.array_equal(self.outs[0].numpy().view(self.np.uint64), self.np.sort(self.key)))

    def cpu_reference(self, sample, threads):
        sec = run_ref_seconds("radix_time", sample, 7, self.bits, threads)
        return sample / sec, sec, (f"n={sample} rows of the same distributions (bounded sample of the 2^22 "
                              f"workload), ORQ's own radix_sort + 2 payload applies, 3 party processes x "
                              f"{threads} worker threads, batch -1, NoCopy sockets over 127.0.0.1")


class QuicksortWorkload(RadixWorkload):
    """The headline's rows (2^22 int64 keys uniform in [0, 2^40) + two payload
    applies) sorted by quicksort, the reference's default sort protocol."""

    name = "qsort"

    def __init__(self, args, seed):
        super().__init__(args, seed)
        self.config["workload"] = WORKLOAD.replace("shuffle-based radix sort", "quicksort (shuffle + opened "
                                                   "pivot compares)")

    def sort(self, kb):
        return self.orq.quicksort(kb, self.orq.ASC)

    def cpu_reference(self, sample, threads):
        sec = run_ref_seconds("qsort_time", sample, 7, self.bits, threads)
        return sample / sec, sec, (f"n={sample} rows of the same distributions (bounded sample of the 2^22 "
                              f"workload), ORQ's own quicksort + 2 payload applies, 3 party processes x "
                              f"{threads} worker threads, batch -1, NoCopy sockets over 127.0.0.1")


class BitonicWorkload:
    """Config 1: bitonic_sort of 2^16 int32 keys drawn over all 32 bits from
    seed 1, ascending (the reference's CPU configuration, on the GPU here)."""

    name = "bitonic"

    def __init__(self, args, seed):
        self.n = args.n if args.n != DEFAULT_N else 1 << 16
        self.seed = 1 + (seed - 7)
        self.units = self.n
        self.flush_l2 = True  # 786 KB of shares: L2 is flushed between steps
        self.config = {"workload": f"3PC bitonic sort, {self.n} int32 keys B-shared, uniform over 32 bits, "
                                   "seed 1, ascending", "rows_per_gpu": self.n,
                       "l2": "L2 flushed (256 MB write) between timed steps", "seed": 1}

    def setup(self, rt, orq):
        import numpy as np

        self.orq, self.rt, self.np = orq, rt, np
        self.key = splitmix(self.seed, self.n).astype(np.uint32)
        self.kb = rt.secret_share_b(self.key.view(np.int32), 0)
        self.orig = self.kb.shares.clone()

    def step(self):
        self.kb.shares.copy_(self.orig)
        self.orq.bitonic_sort(self.kb, self.orq.ASC)

    def check(self):
        np = self.np
        ko = self.kb.open().cpu().numpy().view(np.int32)
        return bool(np.array_equal(np.sort(self.key.view(np.int32)), ko))

    def e2e_setup(self, dev):
        import torch

        np, n = self.np, self.n
        self.pin = torch.from_numpy(self.key.view(np.int32).copy()).pin_memory()
        self.out = torch.empty(n, dtype=torch.int32).pin_memory()
        self.dbuf = torch.empty(n, dtype=torch.int32, device=dev)
        self.h2d = self.d2h = n * 4

    def e2e_step(self):
        self.dbuf.copy_(self.pin, non_blocking=True)
        k = self.rt.secret_share_b(self.dbuf, 0)
        self.orq.bitonic_sort(k, self.orq.ASC)
        self.out.copy_(k.open(), non_blocking=True)

    def e2e_check(self):
        np = self.np
        return bool(np.array_equal(self.out.numpy(), np.sort(self.key.view(np.int32))))

    def cpu_reference(self, sample, threads):
        n = self.n
        sec = run_ref_seconds("bitonic_time", n, self.seed, 32, threads)
        return n / sec, sec, (f"the full workload (n={n}), ORQ's own bitonic_sort, 3 party processes x "
                         f"{threads} worker threads, batch -1, NoCopy sockets over 127.0.0.1")


def zipf_keys(u, s=1.1, m=10000):
    """Zipf(s) over m values by inverse CDF of u in [0, 1)."""
    import numpy as np

    w = 1.0 / np.arange(1, m + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, u, side="right"), m - 1).astype(np.int64)


def gen_join(seed, na, nb):
    """Config 3 tables: A (pk = seeded Fisher-Yates permutation of 0..na-1,
    group Zipf s=1.1 over 10^4 values, value uniform [0, 10^6)); B (fk uniform
    over A.pk, quantity uniform [1, 50])."""
    import numpy as np

    st = splitmix(seed, 2 * na + 2 * nb)
    pk = np.random.Generator(np.random.PCG64(seed)).permutation(na).astype(np.int64)
    u = (st[:na] >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    g = zipf_keys(u)
    v = (st[na:2 * na] % np.uint64(1000000)).astype(np.int64)
    fk = (st[2 * na:2 * na + nb] % np.uint64(na)).astype(np.int64)
    q = (1 + st[2 * na + nb:] % np.uint64(50)).astype(np.int64)
    return pk, g, v, fk, q


def join_expected(pk, g, v, fk, q):
    """SELECT g, SUM(value*qty), COUNT(*) FROM A JOIN B ON pk = fk GROUP BY g."""
    import numpy as np

    gv = np.empty(len(pk), dtype=np.int64)
    vv = np.empty(len(pk), dtype=np.int64)
    gv[pk] = g
    vv[pk] = v
    gb, vb = gv[fk], vv[fk] * q
    keys = np.unique(gb)
    sums = np.bincount(np.searchsorted(keys, gb), weights=None, minlength=len(keys))
    tot = np.zeros(len(keys), dtype=np.int64)
    np.add.at(tot, np.searchsorted(keys, gb), vb)
    return keys, tot, sums.astype(np.int64)


# The reference's published micro_primitives figures (README.md:213-236), 3PC,
# one worker, 32-bit elements, seconds per call on the authors' 8-core machine.
PUBLISHED_PRIMS = {1 << 20: {"AND": 0.01723, "MULT": 0.01167, "EQ": 0.04605, "GR": 0.07226, "RCA": 0.1298},
                   1 << 24: {"AND": 0.1686, "MULT": 0.1992, "EQ": 1.14, "GR": 1.499, "RCA": 1.913}}


class PrimsWorkload:
    """ORQ's micro_primitives sequence (bench/micro/micro_primitives.cpp) on
    n 32-bit elements, 3PC: AND (and_b), MULT (multiply_a), EQ (==), GR (>)
    and RCA (binary +): the protocols' local AND / MUL steps fused with their
    correlated randomness, and the compare circuits built on them. One step =
    the five calls; a row is one element of one call."""

    name = "prims"
    PRIMS = ("AND", "MULT", "EQ", "GR", "RCA")

    def __init__(self, args, seed):
        self.n = args.n if args.n != DEFAULT_N else 1 << 24
        self.seed = seed
        self.units = 5 * self.n
        self.flush_l2 = False  # 5 x 3 x 64 MB of input shares per step
        self.config = {"workload": f"3PC primitives AND, MULT, EQ, GR, RCA on 2^{self.n.bit_length() - 1} "
                                   "int32 elements (ORQ's micro_primitives), one element of one call = one row",
                       "rows_per_gpu": self.units, "elements": self.n,
                       "l2": "inputs larger than L2 (192 MB of shares per operand)", "seed": seed}

    def setup(self, rt, orq):
        import numpy as np

        self.orq, self.rt, self.np = orq, rt, np
        st = splitmix(self.seed, 2 * self.n)
        self.x = st[:self.n].astype(np.uint32)
        self.y = st[self.n:].astype(np.uint32)
        self.xb, self.yb = rt.secret_share_b(self.x, 0), rt.secret_share_b(self.y, 1)
        self.xa, self.ya = rt.secret_share_a(self.x, 0), rt.secret_share_a(self.y, 1)

    def ops(self):
        xb, yb, xa, ya = self.xb, self.yb, self.xa, self.ya
        return {"AND": lambda: xb & yb, "MULT": lambda: xa * ya, "EQ": lambda: xb == yb,
                "GR": lambda: xb > yb, "RCA": lambda: xb + yb}

    def step(self):
        self.out = {k: f() for k, f in self.ops().items()}

    def check(self):
        np = self.np
        x, y = self.x, self.y
        o = {k: v.open().cpu().numpy().view(np.uint32) for k, v in self.out.items()}
        xs, ys = x.view(np.int32), y.view(np.int32)
        with np.errstate(over="ignore"):
            return (np.array_equal(o["AND"], x & y) and np.array_equal(o["MULT"], x * y)
                    and np.array_equal(o["EQ"], (x == y).astype(np.uint32))
                    and np.array_equal(o["GR"], (xs > ys).astype(np.uint32))
                    and np.array_equal(o["RCA"], x + y))

    def breakdown(self):
        """Seconds per primitive call (CUDA events, median of 5), beside the
        reference's published figure at the same size."""
        import torch

        out = {}
        pub = PUBLISHED_PRIMS.get(self.n, {})
        for k, f in self.ops().items():
            ts = []
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                f()
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1) / 1e3)
            sec = statistics.median(ts)
            out[k] = {"seconds": sec, "elements_per_s": self.n / sec}
            if k in pub:
                out[k]["published_s"] = pub[k]
                out[k]["speedup_vs_published"] = pub[k] / sec
        return out

    def e2e_setup(self, dev):
        import torch

        np, n = self.np, self.n
        self.pin = [torch.from_numpy(a.view(np.int32)).pin_memory() for a in (self.x, self.y)]
        self.dbuf = [torch.empty(n, dtype=torch.int32, device=dev) for _ in range(2)]
        self.outs = {k: torch.empty(n, dtype=torch.int32).pin_memory() for k in self.PRIMS}
        self.h2d = 2 * n * 4
        self.d2h = 5 * n * 4

    def e2e_step(self):
        rt = self.rt
        for h, d in zip(self.pin, self.dbuf):
            d.copy_(h, non_blocking=True)
        xb, yb = rt.secret_share_b(self.dbuf[0], 0), rt.secret_share_b(self.dbuf[1], 1)
        xa, ya = rt.secret_share_a(self.dbuf[0], 0), rt.secret_share_a(self.dbuf[1], 1)
        res = {"AND": xb & yb, "MULT": xa * ya, "EQ": xb == yb, "GR": xb > yb, "RCA": xb + yb}
        for k, v in res.items():
            self.outs[k].copy_(v.open(), non_blocking=True)

    def e2e_check(self):
        np = self.np
        return bool(np.array_equal(self.outs["AND"].numpy().view(np.uint32), self.x & self.y))

    def cpu_reference(self, sample, threads):
        from oracle import run_ref

        n = max(1024, min(sample, 1 << 22))
        t0 = time.time()
        _, out = run_ref.run("prims_time", n, self.seed, shim_seed=7, bits=32, threads=threads, timeout=1800)
        prims = None
        for line in out.splitlines():
            if line.startswith('{"prims"'):
                prims = json.loads(line)["prims"]
        sec = sum(prims.values()) if prims else time.time() - t0
        self.ref_prims = prims
        return 5 * n / sec, sec, (f"n={n} int32 elements, ORQ's own AND, MULT, EQ, GR, RCA (5 calls), 3 party "
                                  f"processes x {threads} worker threads, batch -1, NoCopy sockets over 127.0.0.1")


class JoinWorkload:
    """Config 3: A (2^22 rows) inner-join B (2^24 rows) on pk = fk, copying
    the group key and value; VQ = value * quantity; group-by SUM(VQ), COUNT."""

    name = "join"

    def __init__(self, args, seed):
        self.na = args.na
        self.nb = 4 * self.na
        self.seed = seed
        self.units = self.na + self.nb
        self.flush_l2 = False
        self.quick = args.sort_protocol == "quick"
        self.config = {"workload": f"3PC PK-FK join + group-by: A {self.na} rows (pk perm, Zipf(1.1, 10^4) "
                                   f"group, value U[0,10^6)), B {self.nb} rows (fk U over pk, qty U[1,50]); "
                                   "inner_join copy g, value; vq = value*qty; aggregate by g: sum(vq), count",
                       "rows_per_gpu": self.units, "l2": "inputs larger than L2", "seed": seed,
                       "sort_protocol": args.sort_protocol}

    def setup(self, rt, orq):
        import numpy as np

        from orq_b200.table import EncodedTable

        self.orq, self.rt, self.np, self.ET = orq, rt, np, EncodedTable
        self.proto = orq.SortingProtocol.QUICKSORT if self.quick else orq.SortingProtocol.RADIXSORT
        self.data = gen_join(self.seed, self.na, self.nb)
        pk, g, v, fk, q = self.data
        self.A0 = EncodedTable.secret_share(rt, [pk, g, v], ["[K]", "[G]", "V"], protocol=self.proto)
        self.B0 = EncodedTable.secret_share(rt, [fk, q], ["[K]", "Q"], protocol=self.proto)

    def _copy(self, t):
        cols = {k: type(t[k])(self.rt, t[k].shares.clone()) for k in t.getColumnNames()}
        return self.ET(self.rt, cols, t.rows, protocol=self.proto)

    def _pipeline(self, A, B):
        ag = self.orq.aggregators
        J = A.inner_join(B, ["[K]"], [("[G]", "[G]", ag.copy), ("V", "V", ag.copy)])
        J.addColumns(["VQ", "CNT"])
        J["VQ"] = J["V"] * J["Q"]
        J.aggregate(["[G]"], [("VQ", "VQ", ag.sum), ("CNT", "CNT", ag.count)])
        return J

    def step(self):
        self.J = self._pipeline(self._copy(self.A0), self._copy(self.B0))

    def _check_table(self, cols, names):
        np = self.np
        keys, tot, cnt = join_expected(*self.data)
        d = dict(zip(names, cols))
        order = np.argsort(d["[G]"], kind="stable")
        return (np.array_equal(d["[G]"][order], keys) and np.array_equal(d["VQ"][order], tot)
                and np.array_equal(d["CNT"][order], cnt))

    def check(self):
        cols, names = self.J.open_with_schema()
        return bool(self._check_table([c.view(self.np.int64) for c in cols], names))

    def e2e_setup(self, dev):
        import torch

        np = self.np
        self.pin = [torch.from_numpy(a).pin_memory() for a in self.data]
        self.dbuf = [torch.empty(len(a), dtype=torch.int64, device=dev) for a in self.data]
        self.h2d = 8 * (3 * self.na + 2 * self.nb)

    def e2e_step(self):
        import torch

        for h, d in zip(self.pin, self.dbuf):
            d.copy_(h, non_blocking=True)
        rt, ET = self.rt, self.ET
        A = ET(rt, {"[K]": rt.secret_share_b(self.dbuf[0], 0), "[G]": rt.secret_share_b(self.dbuf[1], 0),
                    "V": rt.secret_share_a(self.dbuf[2], 0)}, self.na, protocol=self.proto)
        B = ET(rt, {"[K]": rt.secret_share_b(self.dbuf[3], 0), "Q": rt.secret_share_a(self.dbuf[4], 0)}, self.nb,
               protocol=self.proto)
        J = self._pipeline(A, B)
        # open every column (the result table) and copy it to pinned host memory
        names = J.getColumnNames()
        opened = [J[k].open() for k in names]
        self.e2e_out = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in opened]
        for h, o in zip(self.e2e_out, opened):
            h.copy_(o, non_blocking=True)
        self.e2e_names = names
        self.d2h = sum(o.numel() * o.element_size() for o in opened)

    def e2e_check(self):
        np = self.np
        d = dict(zip(self.e2e_names, [o.numpy().view(np.int64) for o in self.e2e_out]))
        keep = d.pop("[##V]") != 0
        names = list(d)
        return bool(self._check_table([d[k][keep] for k in names], names))

    def cpu_reference(self, sample, threads):
        na = max(64, sample)
        sec = run_ref_seconds("join_time", na, self.seed, 64, threads, quick_tables=self.quick)
        kind = "quicksort" if self.quick else "radix sort"
        return 5 * na / sec, sec, (f"A={na}, B={4 * na} rows of the same distributions (bounded sample), ORQ's "
                              f"own inner_join + product + aggregate ({kind} protocol), 3 party processes "
                              f"x {threads} worker threads, batch -1, NoCopy sockets over 127.0.0.1")


def run_batch(args, rank, world, local_rank):
    """Config 4: 512 independent sorts (256 bitonic with sizes padded to 2^k,
    256 radix), lengths log-uniform over 2^10..2^20, int32 keys uniform over
    32 bits. Batched path: one bitonic_sort_batch (persistent work-list kernel
    per network round, autotuned CTA size, CUDA graph) then one
    radix_sort_batch (the radix items back to back, one synchronisation);
    plain path: 512 per-call operators in the same order (bitonic items, then
    radix items), which yields the same shares. Timed with CUDA events on the
    runtime's stream; both paths' opened outputs are checked."""
    import numpy as np
    import torch

    import orq_b200 as orq

    torch.cuda.set_device(local_rank)
    rng = np.random.Generator(np.random.PCG64(args.seed_batch + rank))
    count = args.batch_items
    kinds = ["bitonic"] * (count // 2) + ["radix"] * (count - count // 2)
    rng.shuffle(kinds)
    sizes = [int(round(2 ** rng.uniform(10, 20))) for _ in range(count)]
    keys = [splitmix(1000 + 7 * i + rank, n).astype(np.uint32).view(np.int32) for i, n in enumerate(sizes)]
    padded = []
    for kind, k in zip(kinds, keys):
        if kind == "bitonic":
            m = 1 << max(0, (len(k) - 1).bit_length())
            k = np.concatenate([k, np.full(m - len(k), np.iinfo(np.int32).max, dtype=np.int32)])
        padded.append(k)
    rows = sum(sizes)
    rt = orq.Runtime(seed=7 + rank, device=local_rank)
    vecs = [rt.secret_share_b(k, 0) for k in padded]
    orig = [v.shares.clone() for v in vecs]
    bit_idx = [i for i, kd in enumerate(kinds) if kd == "bitonic"]
    rad_idx = [i for i, kd in enumerate(kinds) if kd == "radix"]

    def restore():
        for v, o in zip(vecs, orig):
            v.shares.copy_(o)

    def batched():
        orq.bitonic_sort_batch([vecs[i] for i in bit_idx], orq.ASC, use_graph=True)
        orq.radix_sort_batch([vecs[i] for i in rad_idx], orq.ASC, 32)

    def plain():
        for i in bit_idx:
            orq.bitonic_sort(vecs[i], orq.ASC)
        for i in rad_idx:
            orq.radix_sort(vecs[i], orq.ASC, 32)

    def check():
        ok = True
        for i, (k, n) in enumerate(zip(keys, sizes)):
            o = vecs[i].open().cpu().numpy().view(np.int32)[:n]
            ok = ok and np.array_equal(o, np.sort(k))
        return bool(ok)

    def timed(fn, steps):
        ms = 0.0
        for _ in range(steps):
            restore()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / steps

    for _ in range(args.warmup):
        restore()
        batched()
    torch.cuda.synchronize()
    ok = check()
    k0 = rt.kernels_launched()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ms_b = timed(batched, args.steps)
    clk = clocks.stop()
    launches = (rt.kernels_launched() - k0) // max(1, args.steps)
    restore()
    plain()
    torch.cuda.synchronize()
    ok = ok and check()
    ms_p = timed(plain, max(1, min(args.steps, 2)))
    rt.close()
    return {"rows": rows, "ms_batched": ms_b, "ms_plain": ms_p, "ok": ok, "clocks": clk,
            "launches_per_step": launches, "items": count,
            "padded_rows": int(sum(len(p) for p in padded))}


def run_serve(args, rank, world, local_rank):
    """Config 5: Poisson arrivals of mixed requests (60% sort, 30% group-by
    over 2^10 groups, 10% PK-FK join with a 4x foreign-key side), sizes
    log-uniform over 2^12..2^22 rows, int64 keys. Capacity is measured first
    on the plain per-request path (one slot, all requests queued at once) and
    on the continuous-batching server (the same requests, all at once): the
    saturated rows/s of both. The trace then arrives at 80% of the plain
    capacity and is served (a) by the continuous-batching server and (b) by
    the plain path (latency at load). Every result is checked against its
    plaintext answer after the timed runs."""
    import torch

    from orq_b200.serve import Server, check_result, make_trace

    torch.cuda.set_device(local_rank)
    # warm-up: a small trace through both paths (tables, pools, kernels)
    for _ in range(max(1, args.warmup)):
        for slots in (1, args.slots):
            srv = Server(slots=slots, device=local_rank, protocol=args.sort_protocol,
                         share_sms=bool(args.share_sms))
            srv.run(make_trace(6, 0.0, seed=99, min_log=10, max_log=12))
            srv.close()
    out = {"repeats": []}
    # each repeat draws a fresh trace (its own sizes and arrivals), measures
    # the plain path's capacity on it (every request queued at once), and
    # serves it at 80 % of that capacity both ways; the spread over repeats
    # is the run-to-run noise of the comparison
    for r in range(max(1, args.serve_repeats)):
        seed = 5 + rank + 1000 * r
        sat = {}
        for name, slots in (("plain", 1), ("serving", args.slots)):
            calib = make_trace(args.serve_requests, 0.0, seed=seed, max_log=args.serve_max_log)
            srv = Server(slots=slots, device=local_rank, protocol=args.sort_protocol,
                         share_sms=bool(args.share_sms) and slots > 1)
            st = srv.run(calib)
            srv.close()
            st["ok"] = all(check_result(r_, r_.result) for r_ in calib)
            sat[name] = st
        cap_stats = sat["plain"]
        capacity = cap_stats["requests"] / cap_stats["makespan_s"]
        rate = 0.8 * capacity
        if r == 0:
            out["capacity_req_per_s"], out["rate_req_per_s"] = capacity, rate
        rep = {"capacity_req_per_s": capacity, "saturated": sat}
        for name, slots in (("serving", args.slots), ("plain", 1)):
            trace = make_trace(args.serve_requests, rate, seed=seed, max_log=args.serve_max_log)
            srv = Server(slots=slots, device=local_rank, protocol=args.sort_protocol,
                         share_sms=bool(args.share_sms))
            clocks = ClockSampler(local_rank)
            clocks.start()
            st = srv.run(trace)
            st["clocks"] = clocks.stop()
            srv.close()
            st["ok"] = all(check_result(r_, r_.result) for r_ in trace)
            rep[name] = st
            if r == 0:
                out[name] = st
        out["repeats"].append(rep)
    return out


class BatchReference:
    """CPU reference arm of the ragged batch: ORQ's own bitonic and radix sorts
    of a bounded sample of items, one call per item."""

    name = "batch"

    def __init__(self, args, seed):
        self.config = {"workload": "ragged batch of independent 3PC sorts (half bitonic, half radix), "
                                   "lengths log-uniform 2^10..2^20, 32-bit keys", "seed": seed}

    def cpu_reference(self, sample, threads):
        n = max(1024, min(sample, 1 << 14))
        sb = run_ref_seconds("bitonic_time", n, 1, 32, threads)
        sr = run_ref_seconds("radix_time", n, 7, 32, threads)
        return 2 * n / (sb + sr), sb + sr, (f"one bitonic sort of {n} int32 keys and one radix sort of {n} "
                                            f"32-bit keys (bounded sample of the 512-item batch), ORQ's own "
                                            f"operators, 3 party processes x {threads} worker threads")


class ServeReference:
    """CPU reference arm of the serving mix: ORQ's own sort, group-by and join
    on bounded request sizes, one request at a time."""

    name = "serve"

    def __init__(self, args, seed):
        self.protocol = args.sort_protocol
        self.config = {"workload": "mixed requests (60% sort, 30% group-by, 10% join) served one at a time",
                       "sort_protocol": self.protocol, "seed": seed}

    def cpu_reference(self, sample, threads):
        n = max(1024, min(sample, 1 << 12))
        quick = self.protocol == "quick"
        ss = run_ref_seconds("qsort_time" if quick else "radix_time", n, 7, 64, threads)
        sj = run_ref_seconds("join_time", n // 4, 7, 64, threads, quick_tables=quick)
        rows = 0.6 * n + 0.1 * (5 * (n // 4))
        sec = 0.6 * ss + 0.1 * sj
        kind = "quicksort" if quick else "radix sort"
        return rows / sec, sec, (f"a {n}-row 64-bit {kind} and a {n // 4} x {n} join with {kind} table "
                                 f"sorts (bounded samples) weighted 0.6 / 0.1 by the request mix (group-by "
                                 f"runs the same table sort as a sort), ORQ's own operators, 3 party "
                                 f"processes x {threads} worker threads")


WORKLOADS = {"radix": RadixWorkload, "qsort": QuicksortWorkload, "bitonic": BitonicWorkload,
             "join": JoinWorkload, "prims": PrimsWorkload}


def max_over_ranks(x):
    """The maximum of a float over the ranks of the default process group (x
    itself when there is none): every multi-GPU time is the slowest rank's."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = f"cuda:{torch.cuda.current_device()}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def init_replicas(world):
    """One process group for the replicas (NCCL, short timeout) when world > 1."""
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist


def run_orq(args, rank, world, local_rank):
    import ctypes

    import torch

    import orq_b200 as orq

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    dist = init_replicas(world)

    def barrier():
        if dist is not None:
            dist.barrier()

    wl = WORKLOADS[args.workload](args, 7 + rank)
    rt = orq.Runtime(seed=7 + rank, device=local_rank)
    wl.setup(rt, orq)
    flush = torch.empty(1 << 26, dtype=torch.float32, device=dev) if wl.flush_l2 else None

    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()
    ok = wl.check()

    clocks = ClockSampler(local_rank)
    _lib = rt.lib

    def timed(steps):
        evs = []
        for _ in range(steps):
            if flush is not None:
                flush.fill_(1.0)  # write 256 MB: evicts L2 between timed steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            wl.step()
            e1.record()
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs)

    # the timed region runs without per-launch events
    k0 = rt.kernels_launched()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms = timed(args.steps)
    clk = clocks.stop()
    barrier()
    launches = rt.kernels_launched() - k0
    ms = max_over_ranks(ms)
    # a separate profiled pass (CUDA events around every launch, on the stream
    # each kernel runs on) gives the per-kernel times of the roofline
    prof_steps = max(1, min(args.steps, 3))
    orq._check(_lib.orqcu_profile_enable(rt.h, 1))
    prof_ms = timed(prof_steps)
    buf = ctypes.create_string_buffer(1 << 16)
    orq._check(_lib.orqcu_profile_report(rt.h, buf, ctypes.c_size_t(len(buf))))
    orq._check(_lib.orqcu_profile_enable(rt.h, 0))
    prof = parse_profile(buf.value.decode())
    prof["_pass"] = {"steps": prof_steps, "ms_per_step": prof_ms / prof_steps}

    # ---- e2e through the public API with host buffers ----------------------
    e2e = None
    if not args.no_e2e:
        wl.e2e_setup(dev)
        wl.e2e_step()
        torch.cuda.synchronize()
        ke = max(1, min(args.steps, 3))
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(ke):
            wl.e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        ems = max_over_ranks(ems)
        ok = ok and wl.e2e_check()
        e2e = {"value": world * wl.units * ke / (ems / 1e3), "unit": "rows/s",
               "h2d_bytes_per_step": wl.h2d, "d2h_bytes_per_step": wl.d2h, "ms_per_step": ems / ke}
    ok = max_over_ranks(0.0 if ok else 1.0) == 0.0  # every replica's output checked
    if hasattr(wl, "breakdown"):
        wl.extra = {"primitives": wl.breakdown()}
    if dist is not None:
        dist.destroy_process_group()
    return wl, ms, launches, prof, clk, e2e, ok


def roofline(prof, steps, n):
    hbm, sm_mhz, src = load_peaks()
    pas = prof.pop("_pass", None)
    if pas:
        steps = pas["steps"]
    # dominant kernel by device time among the ones accounted in bytes
    mem = {k: v for k, v in prof.items() if v["bytes"] > 0}
    top = max(mem.items(), key=lambda kv: kv[1]["ms"]) if mem else None
    out = {}
    if top:
        name, v = top
        per_launch_ms = v["ms"] / v["launches"]
        ach = (v["bytes"] / v["launches"]) / (per_launch_ms / 1e3) / 1e9
        out["roofline"] = {"bound": "hbm", "kernel": name, "achieved": round(ach, 1), "peak": hbm,
                           "unit": "GB/s", "frac": round(ach / hbm, 4),
                           "traffic": (round(APPLY_TRAFFIC_BYTES_PER_ROW * n)
                                       if name == "apply_group" and n else None),
                           "traffic_note": ("fixed constant, not measured by this run: bytes per launch of the "
                                            "key-apply instance from one ncu capture at 2^21 rows, scaled by rows"),
                           "peak_source": src, "launches_per_step": v["launches"] / steps,
                           "avg_launch_ms": round(per_launch_ms, 4)}
    aes = {k: v for k, v in prof.items() if v["aes_blocks"] > 0}
    if aes:
        tot_bl = sum(v["aes_blocks"] for v in aes.values())
        tot_ms = sum(v["ms"] for v in aes.values())
        ceil = 148 * sm_mhz * 1e6 * 32 / AES_LDS_PER_BLOCK
        topa = max(aes.items(), key=lambda kv: kv[1]["ms"])
        ta = topa[1]
        out["aes"] = {"blocks_per_s": round(tot_bl / (tot_ms / 1e3), 1), "ceiling_blocks_per_s": round(ceil, 1),
                      "frac": round(tot_bl / (tot_ms / 1e3) / ceil, 4), "top_kernel": topa[0],
                      "top_kernel_blocks_per_s": round(ta["aes_blocks"] / (ta["ms"] / 1e3), 1),
                      "ceiling": "148 SMs x max SM clock x 32 lanes / 228 shared-memory lookups per AES-256 block"}
    total = sum(v["ms"] for v in prof.values())
    out["kernel_time_share"] = {k: round(v["ms"] / total, 4) for k, v in
                                sorted(prof.items(), key=lambda kv: -kv[1]["ms"])} if total else {}
    # summed launch time per kernel class and step (streams overlap, so the
    # sum can exceed the step)
    out["kernel_ms_per_step"] = {k: round(v["ms"] / steps, 3) for k, v in
                                 sorted(prof.items(), key=lambda kv: -kv[1]["ms"])}
    if pas:
        out["profile_pass"] = {"steps": pas["steps"], "ms_per_step": round(pas["ms_per_step"], 3),
                               "note": ("per-kernel times come from this separate pass with CUDA events "
                                        "around every launch; value is timed without them")}
    return out


def run_ref_seconds(op, n, seed, bits, threads, timeout=1800, quick_tables=False):
    """ORQ's own CPU code for one op (oracle/_ref/ref_driver, three party
    processes; with quick_tables the build whose EncodedTable sorts default to
    quicksort); returns the seconds it reports for the timed region."""
    from oracle import run_ref

    t0 = time.time()
    _, out = run_ref.run(op, n, seed, shim_seed=7, bits=bits, threads=threads, timeout=timeout,
                         driver=run_ref.DRIVER_QS if quick_tables else None)
    wall = time.time() - t0
    sec = None
    for line in out.splitlines():
        if line.startswith("{"):
            sec = json.loads(line)["seconds"]
    return sec if sec else wall


def splitmix(seed, n):
    """SplitMix64 outputs for state seed (Steele, Lea, Flood, OOPSLA 2014)."""
    import numpy as np

    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="orq", choices=["orq", "reference"])
    ap.add_argument("--workload", default="radix", choices=sorted(WORKLOADS) + ["batch", "serve"])
    ap.add_argument("--n", type=int, default=DEFAULT_N)
    ap.add_argument("--na", type=int, default=1 << 22, help="join: rows of A (B has 4x)")
    ap.add_argument("--bits", type=int, default=40)
    ap.add_argument("--cpu-sample", type=int, default=1 << 20,
                    help="rows of the bounded CPU sample (radix/qsort; join uses 2^11 rows of A)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-items", type=int, default=512)
    ap.add_argument("--seed-batch", type=int, default=4)
    ap.add_argument("--slots", type=int, default=2)
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-max-log", type=int, default=22)
    ap.add_argument("--serve-repeats", type=int, default=3,
                    help="serve: fresh traces served both ways, for the run-to-run spread")
    ap.add_argument("--share-sms", type=int, default=0,
                    help="serve: partition the SMs between slots (1) or let every slot use all of them (0)")
    ap.add_argument("--sort-protocol", default="quick", choices=["quick", "radix"],
                    help="serve and join: sort protocol of sort requests and table sorts (the reference's "
                         "default is quicksort)")
    args = ap.parse_args()
    if args.workload == "join" and args.cpu_sample == 1 << 20:
        args.cpu_sample = 1 << 11
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    nproc = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        refs = dict(WORKLOADS, batch=BatchReference, serve=ServeReference)
        wl = refs[args.workload](args, 7)
        config = dict(wl.config, parallelism=f"replicas x{args.gpus}")
        # the reference's best configuration on this host: one worker per party
        # (shares identical to the GPU's) or every core (nproc/3 per party),
        # whichever is faster on a 1/16 sample; the reference splits each call
        # over its workers, which does not always pay
        calib_sample = max(args.cpu_sample // 16, min(args.cpu_sample, 1 << 10))
        cands = sorted({1, max(1, nproc // 3)})
        calib = {t: wl.cpu_reference(calib_sample, t)[0] for t in cands} if len(cands) > 1 else {1: None}
        threads = max(calib, key=lambda t: calib[t] or 0.0)
        # warm-up runs are whole fresh party processes: a small sample suffices
        warm_sample = min(args.cpu_sample, max(calib_sample // 4, 1 << 10))
        for _ in range(args.warmup):
            wl.cpu_reference(warm_sample, threads)
        runs = [wl.cpu_reference(args.cpu_sample, threads) for _ in range(args.steps)]
        v = statistics.mean(r[0] for r in runs)
        sample = runs[0][2]
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "rows/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(r[1] for r in runs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": v, "unit": "rows/s", "cores": 3 * threads, "kind": "reference",
                             "sample": sample, "cpu": cpu_model(), "threads_per_party": threads,
                             "calibration": {"sample_rows": calib_sample,
                                             "rows_per_s_by_threads_per_party": calib},
                             "warmup_sample_rows": warm_sample},
            "e2e": {"value": v, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    if args.workload in ("batch", "serve") and args.impl == "orq":
        fn = run_batch if args.workload == "batch" else run_serve
        import torch

        torch.cuda.set_device(local_rank)
        dist = init_replicas(world)
        res = fn(args, rank, world, local_rank)
        # whole-job figures from the slowest replica
        if args.workload == "batch":
            for k in ("ms_batched", "ms_plain"):
                res[k] = max_over_ranks(res[k])
        else:
            for rp in res.get("repeats", []):  # every rank takes the same steps
                for part in ("serving", "plain"):
                    for k in ("makespan_s", "p50_ms", "p99_ms"):
                        rp[part][k] = max_over_ranks(rp[part][k])
                    rp["saturated"][part]["makespan_s"] = max_over_ranks(rp["saturated"][part]["makespan_s"])
            for part in ("serving", "plain"):
                res[part]["rows_per_s"] = res[part]["rows"] / res[part]["makespan_s"]
        if dist is not None:
            dist.destroy_process_group()
        if rank != 0:
            return
        if args.workload == "batch":
            value = world * res["rows"] / (res["ms_batched"] / 1e3)
            line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": res["ms_batched"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                    "config": {"workload": f"ragged batch: {res['items']} independent 3PC sorts (half bitonic "
                                           "padded to 2^k, half radix), lengths log-uniform 2^10..2^20, int32 "
                                           "keys uniform; batched bitonic work-list kernels + CUDA graph",
                               "rows_per_gpu": res["rows"], "padded_rows": res["padded_rows"],
                               "parallelism": f"replicas x{world}", "l2": "inputs larger than L2"},
                    "correct": res["ok"], "gpu_launches": res["launches_per_step"] * args.steps,
                    "clocks": res["clocks"],
                    "plain": {"value": world * res["rows"] / (res["ms_plain"] / 1e3), "unit": "rows/s",
                              "ms_per_step": res["ms_plain"]},
                    "batched_over_plain": res["ms_plain"] / res["ms_batched"]}
        else:
            sv, pl = res["serving"], res["plain"]
            line = {"metric": METRIC, "value": world * sv["rows_per_s"], "unit": "rows/s", "n_gpus": world,
                    "steps": 1, "warmup": args.warmup, "ms_per_step": 1e3 * sv["makespan_s"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                    "data": "synthetic",
                    "config": {"workload": f"serving loop: {args.serve_requests} Poisson arrivals at 80% of the "
                                           "plain path's capacity, 60% sort / 30% group-by (2^10 groups) / 10% "
                                           f"PK-FK join (4x fk side), rows log-uniform 2^12..2^{args.serve_max_log}, "
                                           f"int64 keys; continuous batching over {args.slots} slots",
                               "parallelism": f"replicas x{world}", "slots": args.slots,
                               "sort_protocol": args.sort_protocol, "share_sms": bool(args.share_sms)},
                    "correct": sv["ok"] and pl["ok"], "p50_ms": sv["p50_ms"], "p99_ms": sv["p99_ms"],
                    "clocks": sv["clocks"], "capacity_req_per_s": res["capacity_req_per_s"],
                    "rate_req_per_s": res["rate_req_per_s"],
                    "plain": {"value": pl["rows_per_s"], "unit": "rows/s", "p50_ms": pl["p50_ms"],
                              "p99_ms": pl["p99_ms"], "makespan_s": pl["makespan_s"]},
                    "timing": "host wall clock from each request's arrival to its opened result on the host"}
            reps = res.get("repeats", [])
            if reps:
                rows_s = [rp["serving"]["rows"] / rp["serving"]["makespan_s"] for rp in reps]
                rows_p = [rp["plain"]["rows"] / rp["plain"]["makespan_s"] for rp in reps]
                ratio = [a / b for a, b in zip(rows_s, rows_p)]
                line["repeats"] = [{"capacity_req_per_s": rp["capacity_req_per_s"],
                                    "serving_rows_per_s": a, "plain_rows_per_s": b, "serving_over_plain": c,
                                    "serving_p50_ms": rp["serving"]["p50_ms"], "serving_p99_ms": rp["serving"]["p99_ms"],
                                    "plain_p50_ms": rp["plain"]["p50_ms"], "plain_p99_ms": rp["plain"]["p99_ms"]}
                                   for a, b, c, rp in zip(rows_s, rows_p, ratio, reps)]
                line["serving_over_plain"] = {"mean": statistics.mean(ratio), "min": min(ratio), "max": max(ratio)}
                # throughput: every request queued at once, both ways
                sat_s = [world * rp["saturated"]["serving"]["rows"] / rp["saturated"]["serving"]["makespan_s"]
                         for rp in reps]
                sat_p = [world * rp["saturated"]["plain"]["rows"] / rp["saturated"]["plain"]["makespan_s"]
                         for rp in reps]
                sat_r = [a / b for a, b in zip(sat_s, sat_p)]
                line["saturated"] = {"serving_rows_per_s": sat_s, "plain_rows_per_s": sat_p,
                                     "serving_over_plain": {"mean": statistics.mean(sat_r), "min": min(sat_r),
                                                            "max": max(sat_r)},
                                     "note": "the same requests all queued at time 0: served by the slots "
                                             "vs one after another on the plain path"}
                line["correct"] = line["correct"] and all(
                    rp["serving"]["ok"] and rp["plain"]["ok"] and rp["saturated"]["serving"]["ok"]
                    and rp["saturated"]["plain"]["ok"] for rp in reps)
        print(json.dumps(line))
        return

    wl, ms, launches, prof, clk, e2e, ok = run_orq(args, rank, world, local_rank)
    if rank != 0:
        return
    config = dict(wl.config, parallelism=f"replicas x{world}")
    value = world * wl.units * args.steps / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic", "config": config,
        "correct": ok, "gpu_launches": launches, "clocks": clk,
    }
    line.update(roofline(prof, args.steps, wl.units if wl.name == "radix" else None))
    if wl.name == "prims":
        line["dtype"] = "int32"
    line.update(getattr(wl, "extra", {}))
    if e2e:
        line["e2e"] = e2e
    if not args.no_cpu_baseline and world == 1:
        v, _, sample = wl.cpu_reference(args.cpu_sample, 1)
        line["cpu_baseline"] = {"value": v, "unit": "rows/s", "cores": 3, "kind": "reference",
                                "sample": sample, "cpu": cpu_model(), "threads_per_party": 1}
        if getattr(wl, "ref_prims", None):
            line["cpu_baseline"]["seconds_per_primitive"] = wl.ref_prims
    print(json.dumps(line))


if __name__ == "__main__":
    main()
