"""ctypes wrapper for the C restatement (oracle/_ref/liborq_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker; the product never imports it.
Shares are numpy arrays; a shared vector is a list [S0, S1, S2].
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liborq_oracle.so")

_DT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
PAIR0, PAIR1, PAIR2, G01, G02, G12, G012, LOCAL0, LOCAL1, LOCAL2 = range(10)


def splitmix64_stream(seed: int, n: int) -> np.ndarray:
    """SplitMix64 outputs (Steele, Lea, Flood, OOPSLA 2014) as uint64, matching
    the sm64() input generator of ref_driver.cpp."""
    M = (1 << 64) - 1
    out = np.empty(n, dtype=np.uint64)
    s = seed & M
    for i in range(n):
        s = (s + 0x9E3779B97F4A7C15) & M
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        out[i] = z ^ (z >> 31)
    return out


def splitmix64_fast(seed: int, n: int) -> np.ndarray:
    """Vectorised SplitMix64: state_i = seed + (i+1)*golden, then the mix."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        z = s
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


# aggregation function codes (orq_oracle.h)
AGG_SUM, AGG_COUNT, AGG_COPY, AGG_VALID, AGG_BIT_OR, AGG_MIN, AGG_MAX = range(7)


class _Ctx(ctypes.Structure):
    _fields_ = [("rk", (ctypes.c_uint32 * 60) * 10), ("nonce", ctypes.c_uint64 * 10)]


def _lib():
    lib = ctypes.CDLL(LIB_PATH)
    lib.oro_keystream.restype = ctypes.c_uint64
    lib.oro_gen_perm.restype = ctypes.c_uint64
    return lib


class Oracle:
    def __init__(self, seed: int):
        self.lib = _lib()
        self.ctx = _Ctx()
        self.lib.oro_ctx_init(ctypes.byref(self.ctx), ctypes.c_uint64(seed))

    # -- helpers -----------------------------------------------------------
    @staticmethod
    def _ptrs(arrs):
        return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])

    @staticmethod
    def new(n, w):
        return [np.zeros(n, dtype=_DT[w]) for _ in range(3)]

    def nonce(self, stream):
        return int(self.ctx.nonce[stream])

    # -- primitives --------------------------------------------------------
    def secret_share(self, data, arith, party=0):
        w = data.dtype.itemsize
        d = np.ascontiguousarray(data).view(_DT[w])
        s = self.new(len(d), w)
        self.lib.oro_secret_share(ctypes.byref(self.ctx), int(arith), w, ctypes.c_size_t(len(d)),
                                  d.ctypes.data_as(ctypes.c_void_p), party, self._ptrs(s))
        return s

    def open(self, s, arith):
        w = s[0].dtype.itemsize
        out = np.zeros(len(s[0]), dtype=_DT[w])
        self.lib.oro_open(int(arith), w, ctypes.c_size_t(len(out)), self._ptrs(s),
                          out.ctypes.data_as(ctypes.c_void_p))
        return out

    def _bin(self, fn, x, y, ctx=True):
        w = x[0].dtype.itemsize
        z = self.new(len(x[0]), w)
        args = [w, ctypes.c_size_t(len(x[0])), self._ptrs(x), self._ptrs(y), self._ptrs(z)]
        if ctx:
            args = [ctypes.byref(self.ctx)] + args
        fn(*args)
        return z

    def and_b(self, x, y):
        return self._bin(self.lib.oro_and_b, x, y)

    def mul_a(self, x, y):
        return self._bin(self.lib.oro_mul_a, x, y)

    def xor_b(self, x, y):
        return self._bin(self.lib.oro_xor_b, x, y, ctx=False)

    def add_a(self, x, y):
        return self._bin(self.lib.oro_add_a, x, y, ctx=False)

    def sub_a(self, x, y):
        return self._bin(self.lib.oro_sub_a, x, y, ctx=False)

    def b2a_bit(self, x):
        w = x[0].dtype.itemsize
        y = self.new(len(x[0]), w)
        self.lib.oro_b2a_bit(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(x[0])), self._ptrs(x),
                             self._ptrs(y))
        return y

    def reshare(self, s, group, arith):
        w = s[0].dtype.itemsize
        self.lib.oro_reshare(ctypes.byref(self.ctx), int(arith), w, ctypes.c_size_t(len(s[0])),
                             group, self._ptrs(s))

    def zero_share(self, n, w, arith):
        r = self.new(n, w)
        self.lib.oro_zero_share(ctypes.byref(self.ctx), int(arith), w, ctypes.c_size_t(n), self._ptrs(r))
        return r

    def gen_perm(self, stream, n):
        p = np.zeros(n, dtype=np.int32)
        draws = self.lib.oro_gen_perm(ctypes.byref(self.ctx), stream,
                                      p.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(n))
        return p, int(draws)

    def keystream(self, stream, nonce0, nbytes):
        buf = np.zeros(nbytes, dtype=np.uint8)
        self.lib.oro_keystream(self.ctx.rk[stream], ctypes.c_uint64(nonce0),
                               buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(nbytes))
        return buf

    def radix_sort(self, key, bits, payloads=(), desc=False):
        """Sorts key (list of 3 uint64/uint32 share arrays) in place; payloads
        (A-shared 64-bit) are permuted in place. Returns the A-shared perm."""
        kw = key[0].dtype.itemsize
        n = len(key[0])
        pay = []
        for p in payloads:
            pay.extend(p)
        pay_arr = (ctypes.c_void_p * max(1, len(pay)))(*[a.ctypes.data for a in pay])
        perm = self.new(n, 4)
        self.lib.oro_radix_sort(ctypes.byref(self.ctx), kw, ctypes.c_size_t(n), self._ptrs(key),
                                bits, int(desc), len(payloads), pay_arr, self._ptrs(perm))
        return perm

    def shuffle(self, s, arith):
        w = s[0].dtype.itemsize
        self.lib.oro_shuffle(ctypes.byref(self.ctx), int(arith), w, ctypes.c_size_t(len(s[0])),
                             self._ptrs(s))

    def prefix_sum(self, s):
        w = s[0].dtype.itemsize
        self.lib.oro_prefix_sum(w, ctypes.c_size_t(len(s[0])), self._ptrs(s))

    def compare(self, x, y):
        w = x[0].dtype.itemsize
        n = len(x[0])
        eq, gt = self.new(n, w), self.new(n, w)
        self.lib.oro_compare(ctypes.byref(self.ctx), w, ctypes.c_size_t(n), self._ptrs(x), self._ptrs(y),
                             self._ptrs(eq), self._ptrs(gt))
        return eq, gt

    def aggregate(self, keys, b_specs, a_specs, reverse=False, sel=None):
        """orq::aggregators::aggregate; specs are (input shares, function code);
        returns the output shares of the boolean and arithmetic specs."""
        w = (keys[0] if keys else (b_specs or a_specs)[0][0])[0].dtype.itemsize
        n = len((keys[0] if keys else (b_specs or a_specs)[0][0])[0])
        flat = lambda arrs: (ctypes.c_void_p * max(1, 3 * len(arrs)))(
            *[x.ctypes.data for a in arrs for x in a])
        b_out = [self.new(n, w) for _ in b_specs]
        a_out = [self.new(n, w) for _ in a_specs]
        bf = (ctypes.c_int * max(1, len(b_specs)))(*[f for _, f in b_specs])
        af = (ctypes.c_int * max(1, len(a_specs)))(*[f for _, f in a_specs])
        self.lib.oro_aggregate(ctypes.byref(self.ctx), w, ctypes.c_size_t(n), len(keys), flat(keys),
                               len(b_specs), flat([i for i, _ in b_specs]), flat(b_out), bf,
                               len(a_specs), flat([i for i, _ in a_specs]), flat(a_out), af,
                               int(reverse), self._ptrs(sel) if sel is not None else None)
        return b_out, a_out

    def compose_permutations(self, sigma, rho):
        """rho <- compose(sigma, rho); sigma is consumed."""
        self.lib.oro_compose_permutations(ctypes.byref(self.ctx), ctypes.c_size_t(len(rho[0])),
                                          self._ptrs(sigma), self._ptrs(rho))
        return rho

    def table_sort(self, cols, desc, single_bit, data_a=(), data_b=(), quick=False):
        """operators::table_sort (radix or quicksort protocol); every column
        sorted in place."""
        w = cols[0][0].dtype.itemsize
        flat = lambda arrs: (ctypes.c_void_p * max(1, 3 * len(arrs)))(
            *[x.ctypes.data for a in arrs for x in a])
        self.lib.oro_table_sort(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(cols[0][0])), len(cols),
                                flat(cols), (ctypes.c_int * len(cols))(*[int(d) for d in desc]),
                                (ctypes.c_int * len(cols))(*[int(b) for b in single_bit]),
                                len(data_a), flat(data_a), len(data_b), flat(data_b), int(quick))

    def distinct(self, keys):
        w = keys[0][0].dtype.itemsize
        n = len(keys[0][0])
        res = self.new(n, w)
        flat = (ctypes.c_void_p * (3 * len(keys)))(*[x.ctypes.data for a in keys for x in a])
        self.lib.oro_distinct(ctypes.byref(self.ctx), w, ctypes.c_size_t(n), len(keys), flat,
                              self._ptrs(res))
        return res

    def equal(self, x, y):
        w = x[0].dtype.itemsize
        eq = self.new(len(x[0]), w)
        self.lib.oro_equal(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(x[0])), self._ptrs(x),
                           self._ptrs(y), self._ptrs(eq))
        return eq

    def not_b1(self, x):
        w = x[0].dtype.itemsize
        y = self.new(len(x[0]), w)
        self.lib.oro_not_b1(w, ctypes.c_size_t(len(x[0])), self._ptrs(x), self._ptrs(y))
        return y

    def bitonic_sort(self, key, desc=False):
        w = key[0].dtype.itemsize
        self.lib.oro_bitonic_sort(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(key[0])), self._ptrs(key),
                                  int(desc))

    @staticmethod
    def _flat(arrs):
        return (ctypes.c_void_p * max(1, 3 * len(arrs)))(*[x.ctypes.data for a in arrs for x in a])

    def extend_lsb(self, x):
        w = x[0].dtype.itemsize
        y = self.new(len(x[0]), w)
        self.lib.oro_extend_lsb(w, ctypes.c_size_t(len(x[0])), self._ptrs(x), self._ptrs(y))
        return y

    def compare_rows(self, xs, ys, desc):
        """operators::compare_rows over the key columns xs vs ys; returns gt."""
        w = xs[0][0].dtype.itemsize
        n = len(xs[0][0])
        gt = self.new(n, w)
        self.lib.oro_compare_rows(ctypes.byref(self.ctx), w, ctypes.c_size_t(n), len(xs), self._flat(xs),
                                  self._flat(ys), (ctypes.c_int * len(xs))(*[int(d) for d in desc]),
                                  self._ptrs(gt))
        return gt

    def swap(self, xs, ys, bits, arith):
        """operators::swap of column pairs (in place) with B- or A-shared bits."""
        w = bits[0].dtype.itemsize
        self.lib.oro_swap(ctypes.byref(self.ctx), int(arith), w, ctypes.c_size_t(len(bits[0])), len(xs),
                          self._flat(xs), self._flat(ys), self._ptrs(bits))

    def bitonic_sort_rows(self, keys, desc, data_a=(), data_b=()):
        """operators::bitonic_sort over several key columns with data columns."""
        w = keys[0][0].dtype.itemsize
        self.lib.oro_bitonic_sort_rows(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(keys[0][0])),
                                       len(keys), self._flat(keys),
                                       (ctypes.c_int * len(keys))(*[int(d) for d in desc]),
                                       len(data_a), self._flat(data_a), len(data_b), self._flat(data_b))

    def quicksort(self, key, payloads=(), desc=False):
        """operators::quicksort of key (3 share arrays) in place; payloads
        (A-shared, the key's width) are permuted in place. Returns the A-shared
        permutation."""
        kw = key[0].dtype.itemsize
        n = len(key[0])
        pay = [a for p in payloads for a in p]
        pay_arr = (ctypes.c_void_p * max(1, len(pay)))(*[a.ctypes.data for a in pay])
        perm = self.new(n, 4)
        self.lib.oro_quicksort(ctypes.byref(self.ctx), kw, ctypes.c_size_t(n), self._ptrs(key), int(desc),
                               len(payloads), pay_arr, self._ptrs(perm))
        return perm

    def a2b(self, x):
        """ASharedVector::a2b: the boolean sharing of an arithmetic one."""
        w = x[0].dtype.itemsize
        y = self.new(len(x[0]), w)
        self.lib.oro_a2b(ctypes.byref(self.ctx), w, ctypes.c_size_t(len(x[0])), self._ptrs(x), self._ptrs(y))
        return y

    def add_b(self, x, y):
        """BSharedVector::operator+ (ripple-carry adder)."""
        return self._bin(self.lib.oro_add_b, x, y)

    def sub_b(self, x, y):
        """BSharedVector::operator- (x + ~y + 1 by the adder)."""
        return self._bin(self.lib.oro_sub_b, x, y)


class OracleNP:
    """Restatement of the Beaver-2PC (dummy triples) and Fantastic-4PC local
    steps (orq_oracle.c, oro_np_*). A vector is a list of the distinct shares:
    [S0, S1] for 2PC, [X0, X1, X2, X3] for 4PC (X[j] is the share party j
    lacks)."""

    def __init__(self, seed: int, nparties: int):
        assert nparties in (2, 4)
        self.np = nparties
        self.lib = _lib()
        self.ctx = _Ctx()
        self.lib.oro_ctx_init_np(ctypes.byref(self.ctx), ctypes.c_uint64(seed), nparties)

    def _p(self, arrs):
        return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])

    def new(self, n, w):
        return [np.zeros(n, dtype=_DT[w]) for _ in range(self.np)]

    def secret_share(self, data, arith, party=0):
        data = np.ascontiguousarray(data)
        w = data.itemsize
        s = self.new(len(data), w)
        self.lib.oro_np_secret_share(ctypes.byref(self.ctx), self.np, int(arith), w, ctypes.c_size_t(len(data)),
                                     data.ctypes.data_as(ctypes.c_void_p), party, self._p(s))
        return s

    def open(self, s, arith):
        w = s[0].itemsize
        out = np.zeros(len(s[0]), dtype=_DT[w])
        self.lib.oro_np_open(self.np, int(arith), w, ctypes.c_size_t(len(s[0])), self._p(s),
                             out.ctypes.data_as(ctypes.c_void_p))
        return out

    def _mult(self, x, y, arith):
        w = x[0].itemsize
        z = self.new(len(x[0]), w)
        self.lib.oro_np_mult(ctypes.byref(self.ctx), self.np, int(arith), w, ctypes.c_size_t(len(x[0])),
                             self._p(x), self._p(y), self._p(z))
        return z

    def and_b(self, x, y):
        return self._mult(x, y, False)

    def mul_a(self, x, y):
        return self._mult(x, y, True)

    def b2a_bit(self, x):
        w = x[0].itemsize
        y = self.new(len(x[0]), w)
        self.lib.oro_np_b2a_bit(ctypes.byref(self.ctx), self.np, w, ctypes.c_size_t(len(x[0])), self._p(x),
                                self._p(y))
        return y

    def _local(self, op, x, y):
        w = x[0].itemsize
        z = self.new(len(x[0]), w)
        self.lib.oro_np_local(self.np, op, w, ctypes.c_size_t(len(x[0])), self._p(x), self._p(y), self._p(z))
        return z

    def xor_b(self, x, y):
        return self._local(0, x, y)

    def add_a(self, x, y):
        return self._local(1, x, y)
