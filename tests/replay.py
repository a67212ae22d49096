"""Replays of the call sequences in oracle/ref_driver.cpp on a backend.

Both the C restatement (OracleBackend) and the GPU runtime (GpuBackend)
expose the same small interface; every function returns the three distinct
share arrays as a (3, n) numpy array so results can be compared with the
reference's golden dumps and with each other.
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import Oracle, splitmix64_fast

_U = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


class OracleBackend:
    def __init__(self, seed):
        self.o = Oracle(seed)

    def share(self, data, arith, party):
        return self.o.secret_share(data, arith, party)

    def and_b(self, x, y):
        return self.o.and_b(x, y)

    def xor_b(self, x, y):
        return self.o.xor_b(x, y)

    def mul_a(self, x, y):
        return self.o.mul_a(x, y)

    def add_a(self, x, y):
        return self.o.add_a(x, y)

    def b2a_bit(self, x):
        return self.o.b2a_bit(x)

    def open(self, x, arith):
        return self.o.open(x, arith)

    def np(self, x):
        return np.stack(x)

    def radix(self, key, bits, payloads, desc=False):
        perm = self.o.radix_sort(key, bits, payloads, desc=desc)
        return perm

    def table_sort(self, cols, desc, single_bit, data_a, data_b, quick=False):
        self.o.table_sort(cols, desc, single_bit, data_a, data_b, quick)

    def distinct(self, keys):
        return self.o.distinct(keys)

    def compare(self, x, y):
        return self.o.compare(x, y)

    def relops(self, x, y):
        o = self.o
        eq = o.equal(x, y)
        ne = o.not_b1(o.equal(x, y))
        ge = o.not_b1(o.compare(y, x)[1])
        le = o.not_b1(o.compare(x, y)[1])
        return eq, ne, ge, le

    def aggregate(self, keys, bs, as_, reverse, sel):
        return self.o.aggregate(keys, bs, as_, reverse, sel)

    def bitonic(self, key, desc):
        self.o.bitonic_sort(key, desc)

    def qsort(self, key, payloads, desc=False):
        return self.o.quicksort(key, payloads, desc)

    def a2b(self, x):
        return self.o.a2b(x)

    def add_b(self, x, y):
        return self.o.add_b(x, y)

    def sub_b(self, x, y):
        return self.o.sub_b(x, y)

    def bitonic_rows(self, keys, desc, data_a, data_b):
        self.o.bitonic_sort_rows(keys, desc, data_a, data_b)

    def compare_rows(self, xs, ys, desc):
        return self.o.compare_rows(xs, ys, desc)

    def extend_lsb(self, x):
        return self.o.extend_lsb(x)

    def mux_b(self, sel, a, b):
        """multiplex (operators/common.h:20-28) as the reference composes it."""
        o = self.o
        return o.xor_b(a, o.and_b(o.extend_lsb(sel), o.xor_b(b, a)))

    def mux_a(self, sel, a, b):
        """multiplex (operators/common.h:43-49): a + sel * (b - a)."""
        o = self.o
        return o.add_a(a, o.mul_a(sel, o.sub_a(b, a)))

    def swap(self, xs, ys, bits, arith):
        self.o.swap(xs, ys, bits, arith)


class GpuBackend:
    def __init__(self, seed, device=0):
        import orq_b200 as orq

        self.orq = orq
        self.rt = orq.Runtime(seed=seed, device=device)

    def share(self, data, arith, party):
        return (self.rt.secret_share_a if arith else self.rt.secret_share_b)(data, party)

    def and_b(self, x, y):
        return x & y

    def xor_b(self, x, y):
        return x ^ y

    def mul_a(self, x, y):
        return x * y

    def add_a(self, x, y):
        return x + y

    def b2a_bit(self, x):
        return x.b2a_bit()

    def open(self, x, arith):
        return x.open().cpu().numpy()

    def np(self, x):
        a = x.shares.cpu().numpy()
        return a.view(_U[a.dtype.itemsize]) if a.ndim == 2 else a

    def radix(self, key, bits, payloads, desc=False):
        perm = self.orq.radix_sort(key, self.orq.DESC if desc else self.orq.ASC, bits)
        for p in payloads:
            self.orq.oblivious_apply_elementwise_perm(p, perm)
        return perm

    def table_sort(self, cols, desc, single_bit, data_a, data_b, quick=False):
        o = self.orq
        o.table_sort(cols, data_a, data_b, [o.DESC if d else o.ASC for d in desc], single_bit,
                     o.SortingProtocol.QUICKSORT if quick else o.SortingProtocol.RADIXSORT)

    def distinct(self, keys):
        return self.orq.distinct(keys)

    def compare(self, x, y):
        return x._compare(y)

    def relops(self, x, y):
        return x == y, x != y, x >= y, x <= y

    def aggregate(self, keys, bs, as_, reverse, sel):
        orq, rt = self.orq, self.rt
        n = len((keys[0] if keys else (bs or as_)[0][0]))
        bo = [orq.BSharedVector(rt, rt._alloc(n, x.width)) for x, _ in bs]
        ao = [orq.ASharedVector(rt, rt._alloc(n, x.width)) for x, _ in as_]
        orq.aggregate(keys, [(x, o, f) for (x, f), o in zip(bs, bo)],
                      [(x, o, f) for (x, f), o in zip(as_, ao)],
                      orq.Direction.Reverse if reverse else orq.Direction.Forward, sel)
        return bo, ao

    def bitonic(self, key, desc):
        self.orq.bitonic_sort(key, self.orq.DESC if desc else self.orq.ASC)

    def a2b(self, x):
        return x.a2b()

    def add_b(self, x, y):
        return x + y

    def sub_b(self, x, y):
        return x - y

    def qsort(self, key, payloads, desc=False):
        perm = self.orq.quicksort(key, self.orq.DESC if desc else self.orq.ASC)
        for p in payloads:
            self.orq.oblivious_apply_elementwise_perm(p, perm)
        return perm

    def bitonic_rows(self, keys, desc, data_a, data_b):
        o = self.orq
        o.bitonic_sort(keys, data_a, data_b, [o.DESC if d else o.ASC for d in desc])

    def compare_rows(self, xs, ys, desc):
        o = self.orq
        return o.compare_rows(xs, ys, [o.DESC if d else o.ASC for d in desc])

    def extend_lsb(self, x):
        y = self.orq.BSharedVector(self.rt, self.rt._alloc(x.size(), x.width))
        y.extend_lsb(x)
        return y

    def mux_b(self, sel, a, b):
        return self.orq.multiplex(sel, a, b)

    def mux_a(self, sel, a, b):
        return self.orq.multiplex(sel, a, b)

    def swap(self, xs, ys, bits, arith):
        self.orq.swap(xs, ys, bits)


def prim_inputs(n, seed, dt):
    st = splitmix64_fast(seed, 2 * n)
    return st[:n].astype(dt), st[n:].astype(dt)


def replay_prims(be, n, seed):
    """run_prims<int32>, <int64>, <int8> of ref_driver.cpp, in order."""
    out = {}
    for tag, dt, s in (("w4_", np.uint32, seed), ("w8_", np.uint64, seed + 1), ("w1_", np.uint8, seed + 2)):
        x, y = prim_inputs(n, s, dt)
        xb = be.share(x, False, 0)
        yb = be.share(y, False, 1)
        out[tag + "xb"] = be.np(xb)
        out[tag + "yb"] = be.np(yb)
        zb = be.and_b(xb, yb)
        out[tag + "and"] = be.np(zb)
        out[tag + "xor"] = be.np(be.xor_b(xb, yb))
        xa = be.share(x, True, 2)
        ya = be.share(y, True, 0)
        out[tag + "xa"] = be.np(xa)
        out[tag + "ya"] = be.np(ya)
        za = be.mul_a(xa, ya)
        out[tag + "mul"] = be.np(za)
        out[tag + "add"] = be.np(be.add_a(xa, ya))
        ba = be.b2a_bit(xb)
        out[tag + "b2a"] = be.np(ba)
        out[tag + "open_and"] = be.open(zb, False)[None]
        out[tag + "open_mul"] = be.open(za, True)[None]
        out[tag + "open_b2a"] = be.open(ba, True)[None]
    return out


def radix_inputs(n, seed, bits):
    st = splitmix64_fast(seed, 3 * n)
    km = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(2**64 - 1)
    return st[:n] & km, st[n:2 * n] & np.uint64(0xFFFFFFFF), st[2 * n:] & np.uint64(0xFFFFFFFF)


def replay_radix(be, n, seed, bits, desc=False):
    """The "radix" ("radix_desc") op of ref_driver.cpp: radix_sort(key, ASC
    (DESC), bits) then the permutation applied to two A-shared int64 payloads."""
    key, p1, p2 = radix_inputs(n, seed, bits)
    kb = be.share(key, False, 0)
    a1 = be.share(p1, True, 0)
    a2 = be.share(p2, True, 0)
    perm = be.radix(kb, bits, [a1, a2], desc)
    out = {"key": be.np(kb), "pay1": be.np(a1), "pay2": be.np(a2), "perm": be.np(perm)}
    out["open_key"] = be.open(kb, False)[None]
    out["open_pay1"] = be.open(a1, True)[None]
    out["open_pay2"] = be.open(a2, True)[None]
    return out, (key, p1, p2)


def qsort_inputs(n, seed, bits, w):
    """Inputs of the "qsort"/"qsort_desc" (int64) and "qsort32" ops."""
    st = splitmix64_fast(seed, 3 * n)
    if w == 4:
        m32 = np.uint64(0xFFFFFFFF)
        return st[:n].astype(np.uint32), (st[n:2 * n] & m32).astype(np.uint32), (st[2 * n:] & m32).astype(np.uint32)
    return radix_inputs(n, seed, bits)


def replay_qsort(be, n, seed, bits, w=8, desc=False):
    """The quicksort ops of ref_driver.cpp: quicksort(key, order) then the
    permutation applied to two A-shared payloads of the key's width."""
    key, p1, p2 = qsort_inputs(n, seed, bits, w)
    kb = be.share(key, False, 0)
    a1 = be.share(p1, True, 0)
    a2 = be.share(p2, True, 0)
    perm = be.qsort(kb, [a1, a2], desc)
    out = {"key": be.np(kb), "pay1": be.np(a1), "pay2": be.np(a2), "perm": be.np(perm)}
    out["open_key"] = be.open(kb, False)[None]
    out["open_pay1"] = be.open(a1, True)[None]
    out["open_pay2"] = be.open(a2, True)[None]
    return out, (key, p1, p2)


def compare_inputs(n, seed, dt):
    """x, y uniform over all bits; every fourth pair equal."""
    x, y = prim_inputs(n, seed, dt)
    y[::4] = x[::4]
    return x, y


def replay_compare(be, n, seed, w):
    """The "compare32"/"compare64" op of ref_driver.cpp: x._compare(y)."""
    x, y = compare_inputs(n, seed, _U[w])
    xb = be.share(x, False, 0)
    yb = be.share(y, False, 1)
    eq, gt = be.compare(xb, yb)
    out = {"xb": be.np(xb), "yb": be.np(yb), "eq": be.np(eq), "gt": be.np(gt)}
    out["open_eq"] = be.open(eq, False)[None]
    out["open_gt"] = be.open(gt, False)[None]
    return out, (x, y)


def replay_relops(be, n, seed, w):
    """The "relops32"/"relops64" ops of ref_driver.cpp: == != >= <= in order."""
    x, y = compare_inputs(n, seed, _U[w])
    xb = be.share(x, False, 0)
    yb = be.share(y, False, 1)
    outs = be.relops(xb, yb)
    out = {}
    for nm, v in zip(("eq", "ne", "ge", "le"), outs):
        out[nm] = be.np(v)
        out["open_" + nm] = be.open(v, False)[None]
    return out, (x, y)


def replay_bitonic(be, n, seed, w, desc=False):
    """The "bitonic32"/"bitonic64"/"bitonic32_desc" ops of ref_driver.cpp."""
    key = splitmix64_fast(seed, n).astype(_U[w])
    kb = be.share(key, False, 0)
    be.bitonic(kb, desc)
    out = {"key": be.np(kb), "open_key": be.open(kb, False)[None]}
    return out, key


def rows_inputs(n, seed, w):
    """Inputs of the "rows32"/"rows64" ops of ref_driver.cpp."""
    dt = _U[w]
    st = splitmix64_fast(seed, 5 * n)
    k0 = ((st[:n] & np.uint64(7)) - np.uint64(4)).astype(dt)
    k1 = st[n:2 * n].astype(dt)
    b0 = st[2 * n:3 * n].astype(dt)
    a0 = (st[3 * n:4 * n] & np.uint64(0xFFFFFFFF)).astype(dt)
    a1 = (st[4 * n:5 * n] & np.uint64(0xFFFF)).astype(dt)
    return k0, k1, b0, a0, a1


def replay_rows(be, n, seed, w):
    """The "rows32"/"rows64" ops: bitonic_sort over (k0 ASC, k1 DESC) with
    data columns a0, a1 (A-shared) and b0 (B-shared)."""
    k0, k1, b0, a0, a1 = rows_inputs(n, seed, w)
    K0, K1, B0 = be.share(k0, False, 0), be.share(k1, False, 1), be.share(b0, False, 2)
    A0, A1 = be.share(a0, True, 0), be.share(a1, True, 1)
    be.bitonic_rows([K0, K1], [False, True], [A0, A1], [B0])
    out = {}
    for nm, v, ar in (("k0", K0, False), ("k1", K1, False), ("b0", B0, False), ("a0", A0, True),
                      ("a1", A1, True)):
        out[nm] = be.np(v)
        out["open_" + nm] = be.open(v, ar)[None]
    return out, (k0, k1, b0, a0, a1)


def cmprows_inputs(n, seed, w):
    """Inputs of the "cmprows32"/"cmprows64" ops of ref_driver.cpp."""
    dt = _U[w]
    st = splitmix64_fast(seed, 6 * n)
    x0 = (st[:n] & np.uint64(3)).astype(dt)
    y0 = (st[n:2 * n] & np.uint64(3)).astype(dt)
    x1 = st[2 * n:3 * n].astype(dt)
    y1 = st[3 * n:4 * n].astype(dt)
    y1[::4] = x1[::4]
    u = (st[4 * n:5 * n] & np.uint64(0xFFFFFFFF)).astype(dt)
    v = (st[5 * n:6 * n] & np.uint64(0xFFFFFFFF)).astype(dt)
    return x0, y0, x1, y1, u, v


def replay_cmprows(be, n, seed, w):
    """The "cmprows32"/"cmprows64" ops: compare_rows((x0, x1), (y0, y1),
    {ASC, DESC}), b2a_bit of it, extend_lsb, multiplex B and A, then swap of
    the key columns and of (u, v) with the A-shared bits."""
    x0, y0, x1, y1, u, v = cmprows_inputs(n, seed, w)
    X0, X1 = be.share(x0, False, 0), be.share(x1, False, 0)
    Y0, Y1 = be.share(y0, False, 1), be.share(y1, False, 1)
    U, V = be.share(u, True, 2), be.share(v, True, 2)
    gt = be.compare_rows([X0, X1], [Y0, Y1], [False, True])
    out = {"gt": be.np(gt)}
    gta = be.b2a_bit(gt)
    out["gta"] = be.np(gta)
    out["ext"] = be.np(be.extend_lsb(gt))
    out["mux_b"] = be.np(be.mux_b(gt, X1, Y1))
    out["mux_a"] = be.np(be.mux_a(gta, U, V))
    be.swap([X0, X1], [Y0, Y1], gt, False)
    be.swap([U], [V], gta, True)
    for nm, x in (("x0", X0), ("x1", X1), ("y0", Y0), ("y1", Y1), ("u", U), ("v", V)):
        out[nm] = be.np(x)
    out["open_gt"] = be.open(gt, False)[None]
    out["open_x1"] = be.open(X1, False)[None]
    out["open_y1"] = be.open(Y1, False)[None]
    out["open_u"] = be.open(U, True)[None]
    out["open_v"] = be.open(V, True)[None]
    return out, (x0, y0, x1, y1, u, v)


# aggregation function codes (the reference's aggregators, in this order)
SUM, COUNT, COPY, VALID, BIT_OR, MIN, MAX = range(7)


def agg_inputs(n, seed):
    """Inputs of the "agg_*" ops of ref_driver.cpp: key0 sorted in [0, n/4],
    key1 sorted within key0 runs, then A and B value columns and sel bits."""
    st = splitmix64_fast(seed, 10 * n)
    f = st[0:2 * n:2] % np.uint64(n // 4 + 1)
    s2 = st[1:2 * n:2] & np.uint64(1)
    order = np.lexsort((s2, f))
    r = st[2 * n:]
    cols = [r[i * n:(i + 1) * n] for i in range(8)]
    m32 = np.uint64(0xFFFFFFFF)
    return {"k0": f[order], "k1": s2[order], "va1": cols[0] & m32, "va3": cols[1] & m32,
            "vb1": cols[2], "vb2": cols[3] & np.uint64(1), "vb3": cols[4], "vb4": cols[5],
            "vb5": cols[6], "sel": cols[7] & np.uint64(1)}


def replay_agg(be, op, n, seed):
    """The "agg_fwd" / "agg_rev" / "agg_nokey" ops of ref_driver.cpp."""
    x = agg_inputs(n, seed)
    keys = []
    if op != "agg_nokey":
        keys.append(be.share(x["k0"], False, 0))
    if op == "agg_rev":
        keys.append(be.share(x["k1"], False, 0))
    a1 = be.share(x["va1"], True, 0)
    a3 = be.share(x["va3"], True, 0)
    b = [be.share(x[k], False, 0) for k in ("vb1", "vb2", "vb3", "vb4", "vb5")]
    sel = be.share(x["sel"], False, 0)
    bs = [(b[0], COPY), (b[1], VALID), (b[2], BIT_OR), (b[3], MAX), (b[4], MIN)]
    as_ = [(a1, SUM), (a1, COUNT), (a3, COPY)]
    if op == "agg_nokey":
        bs, as_ = bs[:1], as_[:1]
    bo, ao = be.aggregate(keys, bs, as_, op == "agg_rev", sel if op == "agg_rev" else None)
    out = {"o1": be.np(ao[0]), "q1": be.np(bo[0])}
    if op != "agg_nokey":
        out.update({"o2": be.np(ao[1]), "o3": be.np(ao[2]), "q2": be.np(bo[1]), "q3": be.np(bo[2]),
                    "q4": be.np(bo[3]), "q5": be.np(bo[4])})
    out["open_o1"] = be.open(ao[0], True)[None]
    return out, x


def tsort_inputs(n, seed):
    """Inputs of the "tsort"/"distinct" ops: bit, 3-bit, bit key columns, then
    a u32 A column and a full-width B column."""
    st = splitmix64_fast(seed, 5 * n)
    one = np.uint64(1)
    return (st[:n] & one, st[n:2 * n] & np.uint64(7), st[2 * n:3 * n] & one,
            st[3 * n:4 * n] & np.uint64(0xFFFFFFFF), st[4 * n:])


def replay_tsort(be, op, n, seed):
    """The "tsort" ("tsort_qs") op (table_sort with the radix (quicksort)
    protocol on [bit ASC, 3-bit DESC, bit ASC] with one A and one B data
    column) or the "distinct" op (distinct on the first two
    key columns) of ref_driver.cpp."""
    v0, v1, v2, va, vb = tsort_inputs(n, seed)
    b0, b1, b2 = (be.share(v, False, 0) for v in (v0, v1, v2))
    a0 = be.share(va, True, 0)
    b3 = be.share(vb, False, 0)
    if op in ("tsort", "tsort_qs"):
        be.table_sort([b0, b1, b2], [False, True, False], [True, False, True], [a0], [b3], op == "tsort_qs")
        out = {"c0": be.np(b0), "c1": be.np(b1), "c2": be.np(b2), "da": be.np(a0), "db": be.np(b3)}
        for k, v in (("c0", b0), ("c1", b1), ("c2", b2)):
            out["open_" + k] = be.open(v, False)[None]
        out["open_da"] = be.open(a0, True)[None]
    else:
        r = be.distinct([b0, b1])
        out = {"res": be.np(r), "open_res": be.open(r, False)[None]}
    return out, (v0, v1, v2, va, vb)


def join_inputs(n, seed):
    """Inputs of the "join_agg" op of ref_driver.cpp: A has n rows (pk a
    Fisher-Yates permutation, group 0..4, value < 10^6), B has 2n rows (fk
    uniform over pk, quantity 1..50)."""
    na, nb = n, 2 * n
    st = splitmix64_fast(seed, (na - 1) + 2 * na + 2 * nb)
    pk = np.arange(na, dtype=np.int64)
    k = 0
    for i in range(na - 1, 0, -1):
        j = int(st[k] % np.uint64(i + 1))
        k += 1
        pk[i], pk[j] = pk[j], pk[i]
    g = (st[k:k + na] % np.uint64(5)).astype(np.int64)
    k += na
    v = (st[k:k + na] % np.uint64(1000000)).astype(np.int64)
    k += na
    fk = (st[k:k + nb] % np.uint64(na)).astype(np.int64)
    k += nb
    q = (1 + st[k:k + nb] % np.uint64(50)).astype(np.int64)
    return pk, g, v, fk, q


def run_join_agg(rt, pk, g, v, fk, q):
    """The relational pipeline of the "join_agg" op on the device:
    A.inner_join(B, [K], copy [G], V); VQ = V*Q; aggregate by [G] (sum, count)."""
    from orq_b200 import aggregators as ag
    from orq_b200.table import EncodedTable

    A = EncodedTable.secret_share(rt, [pk, g, v], ["[K]", "[G]", "V"])
    B = EncodedTable.secret_share(rt, [fk, q], ["[K]", "Q"])
    J = A.inner_join(B, ["[K]"], [("[G]", "[G]", ag.copy), ("V", "V", ag.copy)])
    J.addColumns(["VQ", "CNT"])
    J["VQ"] = J["V"] * J["Q"]
    J.aggregate(["[G]"], [("VQ", "VQ", ag.sum), ("CNT", "CNT", ag.count)])
    return J


def replay_join(n, seed, shim_seed):
    be = GpuBackend(shim_seed)
    J = run_join_agg(be.rt, *join_inputs(n, seed))
    out = {k: be.np(J[k]) for k in J.getColumnNames()}
    data, names = J.open_with_schema()
    for d, nm in zip(data, names):
        out["open_" + nm] = d.view(np.uint64)[None]
    return out


def same(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def tshuffle_inputs(n, seed):
    """Inputs of the "tshuffle" op of ref_driver.cpp."""
    st = splitmix64_fast(seed, 4 * n)
    return (st[:n], st[n:2 * n] & np.uint64(0xFF), st[2 * n:3 * n] & np.uint64(0xFFFFFFFF),
            st[3 * n:] & np.uint64(1))


def replay_tshuffle(rt_seed, n, seed):
    """The "tshuffle" op on the device runtime: an EncodedTable {[A], [B], V,
    [F]} filtered on [F], then finalize() (shuffle and mask)."""
    import orq_b200 as orq
    from orq_b200.table import EncodedTable

    rt = orq.Runtime(seed=rt_seed)
    cols = tshuffle_inputs(n, seed)
    T = EncodedTable.secret_share(rt, [c.view(np.int64) for c in cols], ["[A]", "[B]", "V", "[F]"])
    T.filter(T["[F]"])
    T.finalize()
    out = {k: T[k].shares.cpu().numpy().view(np.uint64) for k in T.getColumnNames()}
    data, names = T.open_with_schema(remove_invalid=False)
    for k, d in zip(names, data):
        out["open_" + k] = d.view(np.uint64)[None]
    return out, cols


def replay_a2b(be, n, seed, w):
    """The "a2b32"/"a2b64" ops of ref_driver.cpp."""
    x = splitmix64_fast(seed, n).astype(_U[w])
    xa = be.share(x, True, 1)
    xb = be.a2b(xa)
    return {"xa": be.np(xa), "xb": be.np(xb), "open_xb": be.open(xb, False)[None]}, x


def replay_badd(be, n, seed, w):
    """The "badd32"/"badd64" ops: BSharedVector + and -."""
    x, y = prim_inputs(n, seed, _U[w])
    xb, yb = be.share(x, False, 0), be.share(y, False, 1)
    s, d = be.add_b(xb, yb), be.sub_b(xb, yb)
    out = {"sum": be.np(s), "diff": be.np(d), "open_sum": be.open(s, False)[None],
           "open_diff": be.open(d, False)[None]}
    return out, (x, y)


def replay_prims_np(be, n, seed):
    """The "prims" op of ref_driver_np.cpp (Beaver 2PC / Fantastic-4PC) on a
    backend with share / and_b / xor_b / mul_a / add_a / b2a_bit / open:
    widths 4, 8, 1 with data seeds seed, seed+1, seed+2."""
    out = {}
    for w, tag, sd in ((4, "w4_", seed), (8, "w8_", seed + 1), (1, "w1_", seed + 2)):
        st = splitmix64_fast(sd, 2 * n)
        x, y = st[:n].astype(_U[w]), st[n:].astype(_U[w])
        xb = be.share(x, False, 0)
        yb = be.share(y, False, 1)
        out[tag + "xb"], out[tag + "yb"] = be.np(xb), be.np(yb)
        zb = be.and_b(xb, yb)
        out[tag + "and"] = be.np(zb)
        out[tag + "xor"] = be.np(be.xor_b(xb, yb))
        xa = be.share(x, True, 1)
        ya = be.share(y, True, 0)
        out[tag + "xa"], out[tag + "ya"] = be.np(xa), be.np(ya)
        za = be.mul_a(xa, ya)
        out[tag + "mul"] = be.np(za)
        out[tag + "add"] = be.np(be.add_a(xa, ya))
        ba = be.b2a_bit(xb)
        out[tag + "b2a"] = be.np(ba)
        out[tag + "open_and"] = be.open(zb, False)[None]
        out[tag + "open_mul"] = be.open(za, True)[None]
        out[tag + "open_b2a"] = be.open(ba, True)[None]
    return out


class OracleNPBackend:
    """The 2PC / 4PC restatement (oracle.oracle.OracleNP) behind the replay
    interface; shares are lists of numpy arrays."""

    def __init__(self, seed, nparties):
        from oracle.oracle import OracleNP

        self.o = OracleNP(seed, nparties)

    def share(self, data, arith, party):
        return self.o.secret_share(data, arith, party)

    def and_b(self, x, y):
        return self.o.and_b(x, y)

    def xor_b(self, x, y):
        return self.o.xor_b(x, y)

    def mul_a(self, x, y):
        return self.o.mul_a(x, y)

    def add_a(self, x, y):
        return self.o.add_a(x, y)

    def b2a_bit(self, x):
        return self.o.b2a_bit(x)

    def open(self, x, arith):
        return self.o.open(x, arith)

    def np(self, x):
        return np.stack(x)


class GpuNPBackend:
    """The device 2PC / 4PC runtime (orq_b200.NPRuntime) behind the replay
    interface."""

    def __init__(self, seed, nparties, device=0):
        import orq_b200 as orq

        self.rt = orq.NPRuntime(nparties, seed=seed, device=device)

    def share(self, data, arith, party):
        return self.rt.secret_share(data, arith, party)

    def and_b(self, x, y):
        return self.rt.and_b(x, y)

    def xor_b(self, x, y):
        return self.rt.xor_b(x, y)

    def mul_a(self, x, y):
        return self.rt.multiply_a(x, y)

    def add_a(self, x, y):
        return self.rt.add_a(x, y)

    def b2a_bit(self, x):
        return self.rt.b2a_bit(x)

    def open(self, x, arith):
        return self.rt.open(x, arith).cpu().numpy()

    def np(self, x):
        a = x.cpu().numpy()
        return a.view(_U[a.dtype.itemsize])
