"""Serving loop with continuous batching for oblivious sort, group-by
aggregate and PK-FK join requests.

A server owns S slots. Each slot is a worker thread with its own runtime
(keys, nonces, device memory pool) on its own CUDA stream. Requests wait in
one queue; the oldest request is admitted as soon as a slot is free and its
estimated device memory fits in the part of the HBM budget that running
requests have not reserved, so requests that arrive while others run start
as soon as a slot and memory free up, and their kernels overlap on the
device. One exception: at most one large request (LARGE_ROWS rows or more,
which fills the GPU by itself) runs at a time, and smaller requests behind a
waiting large one (within LOOKAHEAD) take the free slots meanwhile. A slot re-keys its runtime with the request's own seed before
running it (orqcu_runtime_reseed): a request's shares and opened result are
the same whether it runs alone or in a mix. A slot keeps its device memory
pool warm between requests (re-allocating and re-mapping gigabytes per
request costs more than the request); optionally each slot's grids are sized
for its share of the SMs.

Sort requests and the table sorts of group-by and join requests use the
server's sort protocol: quicksort (the reference's default) or radix sort.

Latency is measured from a request's arrival to the host having its opened
result; the server reports throughput (rows/s over the whole trace) and the
latency percentiles. `plain` mode runs the same trace through one slot
without overlap: the plain per-request path.
"""
from __future__ import annotations

import collections
import math
import threading
import time

import numpy as np

from . import ASC, Runtime, SortingProtocol, _torch, aggregators, quicksort, radix_sort
from .table import EncodedTable

KINDS = ("sort", "groupby", "join")
# device bytes per row (rows = all input rows of the request), measured
# upper bounds of the pool's peak use: the sharded permutations reserved by
# 64-bit radix sorts dominate (66 permutations x 3 groups x 8 bytes per row)
_BYTES_PER_ROW = {"sort": 2200, "groupby": 2600, "join": 2600}
_FIXED_BYTES = 64 << 20


def _splitmix(seed, n):
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


class Request:
    """One request: kind, size, its own seed, its host inputs and, when done,
    its opened result and timings (seconds on the server's clock)."""

    def __init__(self, rid, kind, n, seed, arrival=0.0):
        assert kind in KINDS
        self.id, self.kind, self.n, self.seed, self.arrival = rid, kind, n, seed, arrival
        st = _splitmix(seed, 6 * n)
        if kind == "sort":
            self.inputs = (st[:n].view(np.int64).copy(),)
            self.rows = n
        elif kind == "groupby":
            self.inputs = ((st[:n] % np.uint64(1 << 10)).astype(np.int64),
                           (st[n:2 * n] % np.uint64(1000000)).astype(np.int64))
            self.rows = n
        else:
            pk = np.random.Generator(np.random.PCG64(seed)).permutation(n).astype(np.int64)
            v = (st[:n] % np.uint64(1000000)).astype(np.int64)
            fk = (st[n:5 * n] % np.uint64(n)).astype(np.int64)
            q = (1 + _splitmix(seed + 1, 4 * n) % np.uint64(50)).astype(np.int64)
            self.inputs = (pk, v, fk, q)
            self.rows = 5 * n
        self.est_bytes = _FIXED_BYTES + _BYTES_PER_ROW[kind] * self.rows
        self.result = None
        self.t_admit = self.t_done = None
        self.slot = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


def run_request(rt, req, protocol="quick"):
    """Runs one request on a runtime (on the caller's current CUDA stream) and
    returns its opened result as host arrays. `protocol` ("quick" or "radix")
    sorts sort requests and every table sort of group-by and join requests."""
    torch = _torch()
    tp = SortingProtocol.QUICKSORT if protocol == "quick" else SortingProtocol.RADIXSORT
    if req.kind == "sort":
        kb = rt.secret_share_b(req.inputs[0], 0)
        if protocol == "quick":
            quicksort(kb, ASC)
        else:
            radix_sort(kb, ASC, 64)
        out = {"key": kb.open().cpu().numpy()}
    elif req.kind == "groupby":
        g, v = req.inputs
        T = EncodedTable.secret_share(rt, [g, v], ["[G]", "V"], protocol=tp)
        T.addColumns(["CNT"])
        T.aggregate(["[G]"], [("V", "V", aggregators.sum), ("CNT", "CNT", aggregators.count)])
        cols, names = T.open_with_schema()
        out = dict(zip(names, cols))
    else:
        pk, v, fk, q = req.inputs
        A = EncodedTable.secret_share(rt, [pk, v], ["[K]", "V"], protocol=tp)
        B = EncodedTable.secret_share(rt, [fk, q], ["[K]", "Q"], protocol=tp)
        J = A.inner_join(B, ["[K]"], [("V", "V", aggregators.copy)])
        cols, names = J.open_with_schema()
        out = dict(zip(names, cols))
    torch.cuda.current_stream().synchronize()
    return out


def expected_result(req):
    """The plaintext answer of a request (for checking)."""
    if req.kind == "sort":
        return {"key": np.sort(req.inputs[0])}
    if req.kind == "groupby":
        g, v = req.inputs
        keys, inv = np.unique(g, return_inverse=True)
        s = np.zeros(len(keys), dtype=np.int64)
        np.add.at(s, inv, v)
        return {"[G]": keys, "V": s, "CNT": np.bincount(inv).astype(np.int64)}
    pk, v, fk, q = req.inputs
    vv = np.empty(len(pk), dtype=np.int64)
    vv[pk] = v
    return {"[K]": fk, "V": vv[fk], "Q": q}


def check_result(req, out):
    """Opened result equals the plaintext answer (row order as sorted keys)."""
    want = expected_result(req)
    if req.kind == "sort":
        return bool(np.array_equal(out["key"].view(np.int64), want["key"]))
    if req.kind == "groupby":
        o = np.argsort(out["[G]"].view(np.int64), kind="stable")
        return all(np.array_equal(out[k].view(np.int64)[o], want[k]) for k in want)
    k = out["[K]"].view(np.int64)
    rows_got = sorted(zip(k.tolist(), out["V"].view(np.int64).tolist(), out["Q"].view(np.int64).tolist()))
    rows_want = sorted(zip(want["[K]"].tolist(), want["V"].tolist(), want["Q"].tolist()))
    return rows_got == rows_want


class _Slot:
    def __init__(self, idx, device, sm_limit=0):
        torch = _torch()
        self.idx = idx
        self.stream = torch.cuda.Stream(device=device)
        with torch.cuda.stream(self.stream):
            self.rt = Runtime(seed=1, device=device)
        if sm_limit:
            self.rt.set_sm_limit(sm_limit)
        self.busy = False
        self.large = False  # running a request of at least LARGE_ROWS rows


# Requests of at least this many rows fill the GPU on their own (their
# Fisher-Yates chains and sorts use every SM): two of them side by side only
# contend, while a small request (latency-bound, a few SMs) overlaps a large
# one well. The dispatcher therefore keeps at most one large request in
# flight and lets small ones behind it in the queue take the other slots.
LARGE_ROWS = 1 << 19
LOOKAHEAD = 16


def pick_next(queue, slots):
    """Index in `queue` of the request to admit next, or None: the oldest one,
    unless a large request is running and it is large too, in which case the
    oldest small one within LOOKAHEAD."""
    large_running = any(s.busy and s.large for s in slots)
    for k, cand in enumerate(queue):
        if k >= LOOKAHEAD:
            break
        if large_running and cand.rows >= LARGE_ROWS:
            continue
        return k
    return None


class Server:
    """Continuous-batching server over `slots` concurrent runtimes."""

    def __init__(self, slots=4, device=0, budget_fraction=0.8, budget_bytes=None, share_sms=False,
                 protocol="quick"):
        torch = _torch()
        self.protocol = protocol
        torch.cuda.set_device(device)
        free, _ = torch.cuda.mem_get_info(device)
        self.budget = int(budget_bytes if budget_bytes is not None else free * budget_fraction)
        self.device = device
        # share_sms: with several slots, each slot's grids are sized for its
        # share of the SMs so concurrent requests' kernels stay resident side by
        # side. That pays for long requests (radix sorts); with quicksort the
        # requests are short and a slot running at a fraction of the GPU
        # costs more latency than the overlap saves, so it is off by default.
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        limit = sms // slots if (share_sms and slots > 1) else 0
        self.slots = [_Slot(i, device, limit) for i in range(slots)]

    def close(self):
        for s in self.slots:
            s.rt.close()

    def run(self, requests, check=False):
        """Serves `requests` (their .arrival are offsets in seconds from the
        start); returns summary statistics. Requests keep their results."""
        torch = _torch()
        reqs = sorted(requests, key=lambda r: r.arrival)
        lock = threading.Condition()
        queue = collections.deque()
        state = {"reserved": 0, "done": 0, "error": None}
        t0 = time.perf_counter()
        work = {s.idx: collections.deque() for s in self.slots}

        def worker(slot):
            torch.cuda.set_device(self.device)
            while True:
                with lock:
                    while not work[slot.idx]:
                        lock.wait()
                    req = work[slot.idx].popleft()
                if req is None:
                    return
                try:
                    with torch.cuda.stream(slot.stream):
                        slot.rt.reseed(req.seed)
                        req.result = run_request(slot.rt, req, self.protocol)
                        slot.stream.synchronize()
                    req.t_done = time.perf_counter() - t0
                    if check:
                        req.ok = check_result(req, req.result)
                except Exception as e:  # surfaces on the dispatcher
                    state["error"] = e
                with lock:
                    slot.busy = False
                    slot.large = False
                    state["reserved"] -= req.est_bytes
                    state["done"] += 1
                    lock.notify_all()

        threads = [threading.Thread(target=worker, args=(s,), daemon=True) for s in self.slots]
        for t in threads:
            t.start()
        i = 0
        with lock:
            while state["done"] < len(reqs):
                now = time.perf_counter() - t0
                while i < len(reqs) and reqs[i].arrival <= now:
                    queue.append(reqs[i])
                    i += 1
                # admit while a slot and memory are free: the oldest request
                # that fits, except that a large one waits while another large
                # one runs (smaller ones within LOOKAHEAD go ahead of it)
                while queue:
                    free_slot = next((s for s in self.slots if not s.busy), None)
                    if free_slot is None:
                        break
                    pick = pick_next(queue, self.slots)
                    if pick is None:
                        break
                    head = queue[pick]
                    fits = state["reserved"] + head.est_bytes <= self.budget or state["reserved"] == 0
                    if not fits:
                        break
                    del queue[pick]
                    free_slot.busy = True
                    free_slot.large = head.rows >= LARGE_ROWS
                    state["reserved"] += head.est_bytes
                    head.t_admit = time.perf_counter() - t0
                    head.slot = free_slot.idx
                    work[free_slot.idx].append(head)
                    lock.notify_all()
                if state["error"] is not None:
                    break
                wait = (reqs[i].arrival - now) if i < len(reqs) else None
                lock.wait(timeout=max(1e-4, wait) if wait is not None else 0.05)
            for s in self.slots:
                work[s.idx].append(None)
            lock.notify_all()
        for t in threads:
            t.join()
        if state["error"] is not None:
            raise state["error"]
        makespan = max(r.t_done for r in reqs)
        lat = np.array([r.latency for r in reqs])
        return {
            "requests": len(reqs),
            "rows": int(sum(r.rows for r in reqs)),
            "makespan_s": makespan,
            "rows_per_s": sum(r.rows for r in reqs) / makespan,
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "slots": len(self.slots),
        }


def make_trace(count, rate, seed=1, min_log=12, max_log=22, mix=(0.6, 0.3, 0.1)):
    """Poisson arrivals at `rate` requests/s of mixed requests (sort, groupby,
    join with probabilities `mix`), sizes log-uniform over 2^min_log..2^max_log
    rows (a join's n is its primary-key side; its foreign-key side is 4n)."""
    # requests and arrivals come from separate generators: the same seed gives
    # the same requests at any rate (capacity is measured on them at rate 0)
    rng = np.random.Generator(np.random.PCG64(seed))
    arr = np.random.Generator(np.random.PCG64(seed + 7919))
    t = 0.0
    out = []
    for k in range(count):
        t += arr.exponential(1.0 / rate) if rate > 0 else 0.0
        kind = KINDS[int(rng.choice(3, p=list(mix)))]
        n = int(round(2 ** rng.uniform(min_log, max_log)))
        out.append(Request(k, kind, n, seed * 1000003 + k, t))
    return out
