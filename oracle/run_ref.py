"""Launch the reference driver (oracle/_ref/ref_driver) as three local party
processes and read back every party's share dump.

TEST INFRASTRUCTURE ONLY. The parties talk over ORQ's NoCopy socket
communicator on 127.0.0.1; the environment mirrors what ORQ's `startmpc`
launcher sets (include/backend/nocopy_communicator/startmpc/startmpc.h:77-147:
STARTMPC_EXEC_MODE=0, STARTMPC_HOST_COUNT, STARTMPC_HOST_RANK,
STARTMPC_BASE_PORT). Processes are started in their own session and stopped by
PID on timeout. ORQ_SHIM_SEED selects the deterministic AES keys of the shim.
"""
from __future__ import annotations

import os
import random
import socket
import struct
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "ref_driver")
_DT = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}


def _free_base_port(span: int = 16) -> int:
    for _ in range(200):
        base = random.randint(20000, 60000)
        ok = True
        for p in range(base, base + span):
            s = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
            try:
                s.bind(("127.0.0.1", p))
            except OSError:
                ok = False
            finally:
                s.close()
            if not ok:
                break
        if ok:
            return base
    raise RuntimeError("no free port range")


def parse_dump(path: str) -> dict:
    """Records written by Dumper in ref_driver.cpp: name, element width, n,
    then share column 0 and share column 1 (raw little-endian)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (nl,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off : off + nl].decode()
        off += nl
        w, n = struct.unpack_from("<IQ", data, off)
        off += 12
        dt = _DT[w]
        a = np.frombuffer(data, dtype=dt, count=n, offset=off).copy()
        off += n * w
        b = np.frombuffer(data, dtype=dt, count=n, offset=off).copy()
        off += n * w
        out[name] = (a, b)
    return out


DRIVER_QS = os.path.join(HERE, "_ref", "ref_driver_qs")  # EncodedTable sorts by quicksort


DRIVER_2PC = os.path.join(HERE, "_ref", "ref_driver_2pc")  # Beaver 2PC, dummy triples
DRIVER_4PC = os.path.join(HERE, "_ref", "ref_driver_4pc")  # Fantastic-4PC


def parse_dump_k(path: str) -> dict:
    """Records written by ref_driver_np.cpp: name, element width, n, k, then
    the k local share columns of the party (raw little-endian)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (nl,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off : off + nl].decode()
        off += nl
        w, n, k = struct.unpack_from("<IQI", data, off)
        off += 16
        cols = []
        for _ in range(k):
            cols.append(np.frombuffer(data, dtype=_DT[w], count=n, offset=off).copy())
            off += n * w
        out[name] = cols
    return out


def run_np(nparties: int, op: str, n: int, data_seed: int, shim_seed: int = 1, timeout: float = 600.0):
    """Run ref_driver_np (Beaver 2PC or Fantastic-4PC) on 2 or 4 parties.
    Returns (list of per-party dicts of local share columns, stdout of P0)."""
    driver = {2: DRIVER_2PC, 4: DRIVER_4PC}[nparties]
    return run(op, n, data_seed, shim_seed=shim_seed, timeout=timeout, driver=driver, nparties=nparties,
               parser=parse_dump_k)


def run(op: str, n: int, data_seed: int, shim_seed: int = 1, bits: int = 40,
        threads: int = 1, batch: int = -1, timeout: float = 600.0, outdir: str | None = None,
        driver: str | None = None, nparties: int = 3, parser=None, exe: dict | None = None):
    """Run one op on 3 parties (or `nparties` with another driver). Returns
    (list of per-party dicts, stdout of P0). `exe` maps a rank to another
    program that plays that party with the driver's arguments and
    environment (ORQ_SEED carries the key seed to it); parser None with exe
    given skips reading the dumps."""
    driver = driver or DRIVER
    if not os.path.exists(driver):
        raise FileNotFoundError(driver + " (run `make -C oracle ref`)")
    tmp = outdir or tempfile.mkdtemp(prefix="orqref_")
    base = _free_base_port()
    procs = []
    for rank in range(nparties):
        env = dict(os.environ)
        env.update({
            "STARTMPC_EXEC_MODE": "0",
            "STARTMPC_HOST_COUNT": str(nparties),
            "STARTMPC_HOST_RANK": str(rank),
            "STARTMPC_BASE_PORT": str(base),
            "ORQ_SHIM_SEED": str(shim_seed),
            "ORQ_SEED": str(shim_seed),
        })
        prog = (exe or {}).get(rank, driver)
        cmd = [prog, str(threads), "1", str(batch), op, str(n), str(data_seed), tmp, str(bits)]
        procs.append(subprocess.Popen(cmd, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, start_new_session=True))
    deadline = time.time() + timeout
    outs = [None] * nparties
    try:
        for i, p in enumerate(procs):
            left = max(1.0, deadline - time.time())
            outs[i] = p.communicate(timeout=left)
    except subprocess.TimeoutExpired:
        for p in procs:
            if p.poll() is None:
                p.kill()
        raise
    for i, p in enumerate(procs):
        if p.returncode != 0:
            raise RuntimeError(f"party {i} exited {p.returncode}: {outs[i][1].decode()[-2000:]}")
    if exe and parser is None:
        return tmp, outs[0][0].decode()
    parser = parser or parse_dump
    dumps = [parser(os.path.join(tmp, f"p{r}.bin")) for r in range(nparties)]
    return dumps, outs[0][0].decode()


def distinct_shares(dumps: list, name: str):
    """Party p holds (S[p], S[p+1]); return (S0, S1, S2) after checking that
    the replicated copies agree."""
    S = [dumps[p][name][0] for p in range(3)]
    for p in range(3):
        if not np.array_equal(dumps[p][name][1], S[(p + 1) % 3]):
            raise AssertionError(f"{name}: party {p} second share differs from S[{(p + 1) % 3}]")
    return S


if __name__ == "__main__":
    op = sys.argv[1] if len(sys.argv) > 1 else "prims"
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 100
    d, o = run(op, n, 7)
    print(o)
    for k in d[0]:
        print(k, d[0][k][0][:4])


def distinct_shares_np(dumps: list, name: str, nparties: int):
    """The distinct shares of a 2PC or 4PC vector from the parties' dumps.
    2PC: party p holds S[p]. 4PC: party p's local share k is X[(p + k + 1) % 4]
    (X[j] is the share party j lacks); the three holders of each X[j] must
    agree."""
    if nparties == 2:
        return [dumps[0][name][0], dumps[1][name][0]]
    X = [None] * 4
    for p in range(4):
        for k in range(3):
            j = (p + k + 1) % 4
            col = dumps[p][name][k]
            if X[j] is None:
                X[j] = col
            elif not np.array_equal(X[j], col):
                raise AssertionError(f"{name}: holders of X[{j}] disagree (party {p})")
    return X
