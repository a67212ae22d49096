#!/usr/bin/env python
"""bench.py — 3PC oblivious radix sort on B200 (ORQ's shuffle-based radix sort).

Workload (per GPU): 2^22 rows, uint64 key uniform in [0, 2^40) boolean-shared,
two uint32 payload columns arithmetic-shared mod 2^64, seed 7; one step =
radix_sort(key, ASC, 40) followed by oblivious_apply_elementwise_perm of both
payloads, including the Fisher–Yates generation of the 44 sharded
permutations it consumes (ORQ reserves them inside radix_sort).

  value  device-resident rows/s: shares already in HBM, CUDA events on the
         runtime's stream around K steps (each step re-copies the unsorted
         shares), max over ranks.
  e2e    the same through the C ABI with host buffers: pinned plaintext
         H2D, secret sharing, sort + payload applies, open, D2H.
  --impl reference   ORQ's own CPU code (oracle/_ref/ref_driver: three party
         processes over its socket communicator) on a bounded sample.

Multi-GPU: independent replicas (each rank sorts its own 2^22 rows; weak
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
# DRAM traffic of the dominant k_apply instance (padded 16-byte key + int32
# permutation, one group), dram__bytes_read.sum + dram__bytes_write.sum from
# one ncu capture at 2^21 rows (profiles/radix_sort_2p22.md): 729 MB, scaled
# per row to the benchmarked size.
APPLY_TRAFFIC_BYTES_PER_ROW = 729.0e6 / (1 << 21)


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


def run_orq(args, rank, world, local_rank):
    import ctypes

    import numpy as np
    import torch

    import orq_b200 as orq

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    n, bits = args.n, args.bits
    rt = orq.Runtime(seed=7 + rank, device=local_rank)
    key, p1, p2 = gen_inputs(n, 7 + rank, bits)
    kb = rt.secret_share_b(key, 0)
    a1 = rt.secret_share_a(p1, 0)
    a2 = rt.secret_share_a(p2, 0)
    orig = [kb.shares.clone(), a1.shares.clone(), a2.shares.clone()]

    def step():
        kb.shares.copy_(orig[0])
        a1.shares.copy_(orig[1])
        a2.shares.copy_(orig[2])
        perm = orq.radix_sort(kb, orq.ASC, bits)
        orq.oblivious_apply_elementwise_perm(a1, perm)
        orq.oblivious_apply_elementwise_perm(a2, perm)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # correctness of the last warm-up step (opened, size-independent checks)
    ko = kb.open().cpu().numpy().view(np.uint64)
    ok = bool(np.all(ko[1:] >= ko[:-1])) and np.array_equal(np.sort(key), ko)

    clocks = ClockSampler(local_rank)
    _lib = rt.lib
    orq._check(_lib.orqcu_profile_enable(rt.h, 1))
    k0 = rt.kernels_launched()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    launches = rt.kernels_launched() - k0
    buf = ctypes.create_string_buffer(1 << 16)
    orq._check(_lib.orqcu_profile_report(rt.h, buf, ctypes.c_size_t(len(buf))))
    orq._check(_lib.orqcu_profile_enable(rt.h, 0))
    prof = parse_profile(buf.value.decode())
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # ---- e2e through the C ABI with host buffers --------------------------
    e2e = None
    if not args.no_e2e:
        pin = [torch.from_numpy(a.view(np.int64)).pin_memory() for a in (key, p1, p2)]
        outs = [torch.empty(n, dtype=torch.int64).pin_memory() for _ in range(3)]
        dbuf = [torch.empty(n, dtype=torch.int64, device=dev) for _ in range(3)]

        def e2e_step():
            for h, d in zip(pin, dbuf):
                d.copy_(h, non_blocking=True)
            k = rt.secret_share_b(dbuf[0], 0)
            x1 = rt.secret_share_a(dbuf[1], 0)
            x2 = rt.secret_share_a(dbuf[2], 0)
            perm = orq.radix_sort(k, orq.ASC, bits)
            orq.oblivious_apply_elementwise_perm(x1, perm)
            orq.oblivious_apply_elementwise_perm(x2, perm)
            for v, o in zip((k, x1, x2), outs):
                o.copy_(v.open(), non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        ke = max(1, min(args.steps, 3))
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(ke):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        ok = ok and bool(np.array_equal(outs[0].numpy().view(np.uint64), np.sort(key)))
        e2e = {"value": world * n * ke / (ems / 1e3), "unit": "rows/s",
               "h2d_bytes_per_step": 3 * n * 8, "d2h_bytes_per_step": 3 * n * 8,
               "ms_per_step": ems / ke}
    if dist is not None:
        dist.destroy_process_group()
    return ms, launches, prof, clk, e2e, ok


def roofline(prof, steps, n):
    hbm, sm_mhz, src = load_peaks()
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
                           "traffic": (round(APPLY_TRAFFIC_BYTES_PER_ROW * n) if name == "apply_group" else None),
                           "traffic_note": "bytes per launch of the key-apply instance, ncu at 2^21 rows scaled by rows",
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
    return out


def cpu_reference(n_sample, bits, threads, timeout=900):
    """ORQ's own CPU radix sort on the host (three party processes)."""
    from oracle import run_ref

    t0 = time.time()
    _, out = run_ref.run("radix_time", n_sample, 7, shim_seed=7, bits=bits, threads=threads,
                         timeout=timeout)
    wall = time.time() - t0
    sec = None
    for line in out.splitlines():
        if line.startswith("{"):
            sec = json.loads(line)["seconds"]
    return sec if sec else wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="orq", choices=["orq", "reference"])
    ap.add_argument("--n", type=int, default=1 << 22)
    ap.add_argument("--bits", type=int, default=40)
    ap.add_argument("--cpu-sample", type=int, default=1 << 17)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    nproc = os.cpu_count() or 1
    config = {"workload": WORKLOAD, "rows_per_gpu": args.n, "key_bits": args.bits, "payloads": 2,
              "parallelism": f"replicas x{args.gpus}", "l2": "inputs larger than L2 (302 MB of shares per GPU)",
              "seed": 7}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = max(1, nproc // 3)
        for _ in range(args.warmup):
            cpu_reference(args.cpu_sample, args.bits, threads)
        secs = [cpu_reference(args.cpu_sample, args.bits, threads) for _ in range(args.steps)]
        v = args.cpu_sample / statistics.mean(secs)
        sample = (f"n={args.cpu_sample} rows of the same distributions per step (bounded sample of the "
                  f"2^22 workload), 3 party processes x {threads} worker threads, batch -1, NoCopy sockets")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "rows/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": v, "unit": "rows/s", "cores": 3 * threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    ms, launches, prof, clk, e2e, ok = run_orq(args, rank, world, local_rank)
    if rank != 0:
        return
    value = world * args.n * args.steps / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic", "config": config,
        "correct": ok, "gpu_launches": launches, "clocks": clk,
    }
    line.update(roofline(prof, args.steps, args.n))
    if e2e:
        line["e2e"] = e2e
    if not args.no_cpu_baseline and world == 1:
        sec = cpu_reference(args.cpu_sample, args.bits, 1)
        line["cpu_baseline"] = {"value": args.cpu_sample / sec, "unit": "rows/s", "cores": 3,
                                "kind": "reference",
                                "sample": f"n={args.cpu_sample} rows, same distributions, ORQ's own "
                                          "radix_sort + 2 payload applies, 3 party processes x 1 thread, "
                                          "batch -1, NoCopy sockets over 127.0.0.1"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
