"""orq_b200 — ORQ's replicated-3PC share computation on one B200.

Python mirror of the reference's user-facing API (include/mpc.h,
core/containers/{b,a}_shared_vector.h, core/operators/{radixsort,shuffle}.h)
over the C ABI of liborq_cuda.so (include/orq_cuda.h). All three parties live
in one process: a shared vector is the three distinct share arrays
S[0], S[1], S[2] (party p holds S[p], S[p+1]) as one (3, n) CUDA tensor.

    rt = Runtime(seed=1)                     # orq_init(argc, argv)
    k = rt.secret_share_b(keys, party=0)     # secret_share_b(Vector, 0)
    perm = radix_sort(k, ASC, bits=40)       # orq::operators::radix_sort
    oblivious_apply_elementwise_perm(payload, perm)
    k.open()                                 # BSharedVector::open()

There is no CPU fallback: creating a Runtime without the compiled library or
a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborq_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "orq_cuda.h")

ASC, DESC = 0, 1
STREAM_PAIR0, STREAM_PAIR1, STREAM_PAIR2 = 0, 1, 2
STREAM_G01, STREAM_G02, STREAM_G12, STREAM_G012 = 3, 4, 5, 6
STREAM_LOCAL0, STREAM_LOCAL1, STREAM_LOCAL2 = 7, 8, 9

_lib = None


class OrqError(RuntimeError):
    pass


def header_symbols() -> list[str]:
    """Entry points declared in include/orq_cuda.h."""
    with open(HEADER) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(orqcu_[a-z0-9_]+)\s*\(", txt)))


def load_library():
    """Load liborq_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m orq_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    lib.orqcu_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(rc: int):
    if rc != 0:
        msg = _lib.orqcu_last_error().decode() if _lib else "?"
        raise OrqError(f"orqcu error {rc}: {msg}")


def _torch():
    import torch  # plumbing only: device memory and streams
    return torch


_TDT = None


def _tdtype(width: int):
    torch = _torch()
    return {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64, 16: torch.int64}[width]


def _p3(t):
    """(3, ...) tensor -> ctypes array of the three share row pointers."""
    return (ctypes.c_void_p * 3)(*[t[j].data_ptr() for j in range(3)])


class Runtime:
    """The loopback runtime for all three parties (stands in for orq_init and
    the per-party RunTime, include/backend/common/setup.h:8-58)."""

    def __init__(self, seed: int = 1, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise OrqError("orq_b200 needs a CUDA device (no CPU fallback)")
        self.lib = load_library()
        self.device = device
        torch.cuda.set_device(device)
        h = ctypes.c_void_p()
        _check(self.lib.orqcu_runtime_create(ctypes.c_uint64(seed), device, ctypes.byref(h)))
        self.h = h
        # run on torch's current stream so tensor ops and ORQ kernels are ordered
        _check(self.lib.orqcu_runtime_set_stream(self.h, ctypes.c_void_p(
            torch.cuda.current_stream(device).cuda_stream)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.orqcu_runtime_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ------------------------------------------------------------
    def nonce(self, stream: int) -> int:
        v = ctypes.c_uint64()
        _check(self.lib.orqcu_get_nonce(self.h, stream, ctypes.byref(v)))
        return v.value

    def kernels_launched(self) -> int:
        v = ctypes.c_uint64()
        _check(self.lib.orqcu_kernels_launched(self.h, ctypes.byref(v)))
        return v.value

    def synchronize(self):
        _check(self.lib.orqcu_synchronize(self.h))

    def reseed(self, seed: int):
        """Fresh keys and nonces for `seed`, keeping stream and cached memory."""
        _check(self.lib.orqcu_runtime_reseed(self.h, ctypes.c_uint64(seed)))

    def set_sm_limit(self, sms: int):
        """Size this runtime's grids for `sms` SMs (0 = the whole device)."""
        _check(self.lib.orqcu_runtime_set_sm_limit(self.h, int(sms)))

    def trim(self) -> int:
        """Return cached device memory (stream-ordered); bytes that were cached."""
        v = ctypes.c_size_t()
        _check(self.lib.orqcu_runtime_trim(self.h, ctypes.byref(v)))
        return v.value

    # -- sharing ----------------------------------------------------------
    def _alloc(self, n: int, width: int):
        torch = _torch()
        if width == 16:
            return torch.empty((3, n, 2), dtype=torch.int64, device=f"cuda:{self.device}")
        return torch.empty((3, n), dtype=_tdtype(width), device=f"cuda:{self.device}")

    def _to_dev(self, data, width: int):
        torch = _torch()
        if isinstance(data, np.ndarray):
            data = torch.from_numpy(np.ascontiguousarray(data))
        if data.element_size() != width:
            raise ValueError("data element size does not match the share width")
        return data.to(f"cuda:{self.device}").contiguous()

    def secret_share_b(self, data, party: int = 0) -> "BSharedVector":
        """secret_share_b (replicated_3pc.h:401-420): owner `party` splits data
        with its local PRG."""
        return BSharedVector(self, self._share(data, party, arith=False))

    def secret_share_a(self, data, party: int = 0) -> "ASharedVector":
        """secret_share_a (replicated_3pc.h:429-448)."""
        return ASharedVector(self, self._share(data, party, arith=True))

    def _share(self, data, party, arith):
        w = data.itemsize if isinstance(data, np.ndarray) else data.element_size()
        d = self._to_dev(data, w)
        n = d.shape[0]
        s = self._alloc(n, w)
        _check(self.lib.orqcu_secret_share(self.h, int(arith), w, ctypes.c_size_t(n),
                                           ctypes.c_void_p(d.data_ptr()), party, _p3(s)))
        return s

    def public_share(self, data, arith=True):
        """public_share (replicated_3pc.h:456-470)."""
        w = data.itemsize if isinstance(data, np.ndarray) else data.element_size()
        d = self._to_dev(data, w)
        s = self._alloc(d.shape[0], w)
        _check(self.lib.orqcu_public_share(self.h, w, ctypes.c_size_t(d.shape[0]),
                                           ctypes.c_void_p(d.data_ptr()), _p3(s)))
        return (ASharedVector if arith else BSharedVector)(self, s)

    def from_shares(self, shares, arith: bool):
        """Wrap existing (3, n) device shares."""
        return (ASharedVector if arith else BSharedVector)(self, shares)

    def input_secret_shares(self, paths, n: int, width: int, arith: bool = False):
        """BSharedVector / ASharedVector(size, file) (e_vector.h:300-348) for
        all three parties: paths[p] is party p's share file (orq_b200.io)."""
        from . import io

        S = io.read_party_shares(paths, n, width)
        return self.from_shares(self._to_dev(S.view({1: np.int8, 2: np.int16, 4: np.int32,
                                                        8: np.int64}[width]), width), arith)

    # -- randomness -------------------------------------------------------
    def keystream(self, stream: int, nonce0: int, nbytes: int):
        torch = _torch()
        out = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{self.device}")
        _check(self.lib.orqcu_keystream(self.h, stream, ctypes.c_uint64(nonce0),
                                        ctypes.c_size_t(nbytes), ctypes.c_void_p(out.data_ptr())))
        return out

    def zero_share(self, n: int, width: int, arith: bool):
        s = self._alloc(n, width)
        _check(self.lib.orqcu_zero_share(self.h, int(arith), width, ctypes.c_size_t(n), _p3(s)))
        return s

    def reserve_permutations(self, n: int, count: int):
        """PermutationManager::reserve (permutation_manager.h:102-181)."""
        _check(self.lib.orqcu_reserve_permutations(self.h, ctypes.c_size_t(n), ctypes.c_size_t(count)))

    def next_permutation(self, n: int):
        """The three group-local permutations of the next sharded permutation."""
        torch = _torch()
        out = torch.empty((3, n), dtype=torch.int32, device=f"cuda:{self.device}")
        ptrs = (ctypes.c_void_p * 3)(*[out[g].data_ptr() for g in range(3)])
        _check(self.lib.orqcu_next_permutation(self.h, ctypes.c_size_t(n), ptrs))
        return out


class SharedVector:
    arith = False

    def __init__(self, rt: Runtime, shares):
        self.rt = rt
        self.shares = shares

    @property
    def width(self) -> int:
        s = self.shares
        return 16 if s.dim() == 3 else s.element_size()

    def size(self) -> int:
        return self.shares.shape[1]

    def __len__(self):
        return self.size()

    def open(self):
        """open_shares_a/b (replicated_3pc.h:310-330); returns a device tensor."""
        rt = self.rt
        n, w = self.size(), self.width
        out = rt._alloc(1, w)[0] if n == 0 else None
        torch = _torch()
        shape = (n, 2) if w == 16 else (n,)
        out = torch.empty(shape, dtype=self.shares.dtype, device=self.shares.device)
        _check(rt.lib.orqcu_open(rt.h, int(self.arith), w, ctypes.c_size_t(n), _p3(self.shares),
                                 ctypes.c_void_p(out.data_ptr())))
        return out

    def _bin(self, other, fn, cls):
        if other.size() != self.size() or other.width != self.width:
            raise ValueError("size/width mismatch")
        z = self.rt._alloc(self.size(), self.width)
        _check(fn(self.rt.h, self.width, ctypes.c_size_t(self.size()), _p3(self.shares),
                  _p3(other.shares), _p3(z)))
        return cls(self.rt, z)

    def _ibin(self, other, fn):
        if other.size() != self.size() or other.width != self.width:
            raise ValueError("size/width mismatch")
        _check(fn(self.rt.h, self.width, ctypes.c_size_t(self.size()), _p3(self.shares),
                  _p3(other.shares), _p3(self.shares)))
        return self

    def clone(self):
        return type(self)(self.rt, self.shares.clone())

    def outputSecretShares(self, paths):
        """EVector::output (e_vector.h:249-266) for all three parties: party p
        writes its replicated shares (S[p], S[p+1]) to paths[p]."""
        from . import io

        io.write_party_shares(self.shares.cpu().numpy(), paths)


class BSharedVector(SharedVector):
    """Boolean (XOR) shares (core/containers/b_shared_vector.h)."""
    arith = False

    def __and__(self, o):
        return self._bin(o, self.rt.lib.orqcu_and_b, BSharedVector)

    def __xor__(self, o):
        return self._bin(o, self.rt.lib.orqcu_xor_b, BSharedVector)

    def __iand__(self, o):
        return self._ibin(o, self.rt.lib.orqcu_and_b)

    def __ixor__(self, o):
        return self._ibin(o, self.rt.lib.orqcu_xor_b)

    def __add__(self, o):
        """operator+ (b_shared_vector.h:588-590): the ripple-carry adder."""
        return self._bin(o, self.rt.lib.orqcu_add_b, BSharedVector)

    def __sub__(self, o):
        """operator- (b_shared_vector.h:620-622): self + ~o + 1 by the adder."""
        return self._bin(o, self.rt.lib.orqcu_sub_b, BSharedVector)

    def __or__(self, o):
        """operator| (b_shared_vector.h:438-441): ~(~a & ~b)."""
        return ~((~self) & (~o))

    def __invert__(self):
        z = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_not_b(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                       _p3(self.shares), _p3(z)))
        return BSharedVector(self.rt, z)

    def extend_lsb(self, inp: "BSharedVector"):
        """BSharedVector::extend_lsb (b_shared_vector.h:145-147): every element
        of self becomes all ones where inp's LSB is set (local)."""
        if inp.size() != self.size() or inp.width != self.width:
            raise ValueError("size/width mismatch")
        _check(self.rt.lib.orqcu_extend_lsb(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                            _p3(inp.shares), _p3(self.shares)))
        return self

    def mask(self, m: int):
        """BSharedVector::mask (b_shared_vector.h:462-464): shares &= m, in place."""
        _check(self.rt.lib.orqcu_mask_b(self.rt.h, self.width, ctypes.c_size_t(self.size()), _p3(self.shares),
                                        ctypes.c_uint64(m & ((1 << (8 * self.width)) - 1))))
        return self

    def b2a_bit(self) -> "ASharedVector":
        """b2a_bit (b_shared_vector.h:279-284, replicated_3pc.h:220-251)."""
        z = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_b2a_bit(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                         _p3(self.shares), _p3(z)))
        return ASharedVector(self.rt, z)

    def _compare(self, other: "BSharedVector"):
        """BSharedVector::_compare (circuits.h:231-295): (eq, gt) as B-shared
        bits, self vs other in the signed order."""
        if other.size() != self.size() or other.width != self.width:
            raise ValueError("size/width mismatch")
        eq = self.rt._alloc(self.size(), self.width)
        gt = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_compare_b(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                           _p3(self.shares), _p3(other.shares), _p3(eq), _p3(gt)))
        return BSharedVector(self.rt, eq), BSharedVector(self.rt, gt)

    def __gt__(self, other: "BSharedVector") -> "BSharedVector":
        """operator> (b_shared_vector.h:538-545)."""
        return self._compare(other)[1]

    def __lt__(self, other: "BSharedVector") -> "BSharedVector":
        """operator< (b_shared_vector.h:556-558): other > self."""
        return other._compare(self)[1]

    def __eq__(self, other: "BSharedVector") -> "BSharedVector":
        """operator== (b_shared_vector.h:493-504): bit_same, then mask(1)."""
        if other.size() != self.size() or other.width != self.width:
            raise ValueError("size/width mismatch")
        eq = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_equal_b(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                         _p3(self.shares), _p3(other.shares), _p3(eq)))
        return BSharedVector(self.rt, eq)

    def lnot(self) -> "BSharedVector":
        """operator! (not_b_1, replicated_3pc.h:207): logical NOT of a bit."""
        y = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_not_b_1(self.rt.h, self.width, ctypes.c_size_t(self.size()),
                                         _p3(self.shares), _p3(y)))
        return BSharedVector(self.rt, y)

    def __ne__(self, other: "BSharedVector") -> "BSharedVector":
        """operator!= (b_shared_vector.h:514-516): !(self == other)."""
        return (self == other).lnot()

    def __ge__(self, other: "BSharedVector") -> "BSharedVector":
        """operator>= (b_shared_vector.h:566-568): !(self < other)."""
        return (self < other).lnot()

    def __le__(self, other: "BSharedVector") -> "BSharedVector":
        """operator<= (b_shared_vector.h:578-580): !(self > other)."""
        return (self > other).lnot()

    __hash__ = object.__hash__


class ASharedVector(SharedVector):
    """Arithmetic shares mod 2^(8w) (core/containers/a_shared_vector.h)."""
    arith = True

    def a2b(self) -> "BSharedVector":
        """ASharedVector::a2b (a_shared_vector.h:138-144): full-width
        arithmetic -> boolean conversion (redistribution + ripple-carry adder)."""
        z = self.rt._alloc(self.size(), self.width)
        _check(self.rt.lib.orqcu_a2b(self.rt.h, self.width, ctypes.c_size_t(self.size()), _p3(self.shares),
                                     _p3(z)))
        return BSharedVector(self.rt, z)

    def __mul__(self, o):
        return self._bin(o, self.rt.lib.orqcu_multiply_a, ASharedVector)

    def __add__(self, o):
        return self._bin(o, self.rt.lib.orqcu_add_a, ASharedVector)

    def __sub__(self, o):
        return self._bin(o, self.rt.lib.orqcu_sub_a, ASharedVector)

    def __imul__(self, o):
        return self._ibin(o, self.rt.lib.orqcu_multiply_a)

    def __iadd__(self, o):
        return self._ibin(o, self.rt.lib.orqcu_add_a)

    def __isub__(self, o):
        return self._ibin(o, self.rt.lib.orqcu_sub_a)


def prefix_sum(v: ASharedVector):
    """SharedVector::prefix_sum (shared_vector.h:249): in-place inclusive scan."""
    rt = v.rt
    _check(rt.lib.orqcu_prefix_sum_a(rt.h, v.width, ctypes.c_size_t(v.size()), _p3(v.shares)))


class ElementwisePermutation(ASharedVector):
    """A-shared int32 destination indices (core/containers/permutation.h)."""


def reshare(v: SharedVector, group: int):
    """Protocol::reshare (protocol.h:500-541) in place."""
    rt = v.rt
    _check(rt.lib.orqcu_reshare(rt.h, int(v.arith), v.width, ctypes.c_size_t(v.size()), group,
                                _p3(v.shares)))


def shuffle(v: SharedVector):
    """orq::operators::shuffle (shuffle.h:752-757), in place."""
    rt = v.rt
    _check(rt.lib.orqcu_shuffle(rt.h, int(v.arith), v.width, ctypes.c_size_t(v.size()),
                                _p3(v.shares)))


def oblivious_apply_elementwise_perm(x: SharedVector, perm: ASharedVector):
    """shuffle.h:687-706, in place on x."""
    rt = x.rt
    _check(rt.lib.orqcu_apply_elementwise_perm(rt.h, int(x.arith), x.width,
                                               ctypes.c_size_t(x.size()), _p3(x.shares),
                                               _p3(perm.shares)))


def bitonic_sort(columns, data_a=(), data_b=(), order=ASC):
    """orq::operators::bitonic_sort (sorting.h:266-353,394-399), in place; the
    size must be a power of two. Either one B-shared key column and one order
    (bitonic_sort(vec, order)), or a list of key columns (most significant
    first) with A- and B-shared data columns moved along and one order per key
    column (bitonic_sort(columns, data_a, data_b, order))."""
    if isinstance(columns, BSharedVector):
        v = columns
        if isinstance(data_a, int):  # bitonic_sort(vec, order)
            order, data_a = data_a, ()
        if data_a or data_b:
            raise ValueError("data columns need the list form")
        if isinstance(order, (list, tuple)):
            order = order[0]
        _check(v.rt.lib.orqcu_bitonic_sort(v.rt.h, v.width, ctypes.c_size_t(v.size()), _p3(v.shares),
                                           int(order == DESC)))
        return
    columns = list(columns)
    rt, n, w = columns[0].rt, columns[0].size(), columns[0].width
    orders = list(order) if isinstance(order, (list, tuple)) else [order] * len(columns)
    if len(orders) != len(columns):
        raise ValueError("one order per key column")
    for v in list(columns) + list(data_a) + list(data_b):
        if v.size() != n or v.width != w:
            raise ValueError("size/width mismatch")
    _check(rt.lib.orqcu_bitonic_sort_rows(rt.h, w, ctypes.c_size_t(n), len(columns), _flat(columns),
                                          (ctypes.c_int * len(columns))(*[int(o == DESC) for o in orders]),
                                          len(data_a), _flat(data_a), len(data_b), _flat(data_b)))


def shuffle_columns(data_a, data_b):
    """orq::operators::shuffle(data_a, data_b, size) (shuffle.h:769-786): the
    rows of every column permuted by one random secret permutation, in place."""
    first = (list(data_a) + list(data_b))[0]
    rt, n, w = first.rt, first.size(), first.width
    _check(rt.lib.orqcu_table_shuffle(rt.h, w, ctypes.c_size_t(n), len(data_a), _flat(data_a), len(data_b),
                                      _flat(data_b)))


def compare_rows(x_vec, y_vec, order) -> BSharedVector:
    """orq::operators::compare_rows (sorting.h:80-108): row i of x is greater
    than row i of y in the lexicographic order of the key columns (each ASC or
    DESC); returns the B-shared result bits."""
    if not x_vec or len(x_vec) != len(y_vec) or len(order) != len(x_vec):
        raise ValueError("compare_rows needs matching key lists and one order per key")
    rt, n, w = x_vec[0].rt, x_vec[0].size(), x_vec[0].width
    for v in list(x_vec) + list(y_vec):
        if v.size() != n or v.width != w:
            raise ValueError("size/width mismatch")
    gt = rt._alloc(n, w)
    _check(rt.lib.orqcu_compare_rows(rt.h, w, ctypes.c_size_t(n), len(x_vec), _flat(x_vec), _flat(y_vec),
                                     (ctypes.c_int * len(x_vec))(*[int(o == DESC) for o in order]),
                                     _p3(gt)))
    return BSharedVector(rt, gt)


def swap(x_vec, y_vec, bits):
    """orq::operators::swap (sorting.h:146-212): rows i of the column pairs
    (x, y) are exchanged in place where bits[i] is 1. B-shared bits swap
    B-shared columns (multiplex on the LSB), A-shared bits A-shared columns.
    Single vectors are accepted for one column pair."""
    if isinstance(x_vec, SharedVector):
        x_vec, y_vec = [x_vec], [y_vec]
    arith = isinstance(bits, ASharedVector)
    rt, n, w = bits.rt, bits.size(), bits.width
    for v in list(x_vec) + list(y_vec):
        if v.size() != n or v.width != w or v.arith != arith:
            raise ValueError("swap columns must match the bits in size, width and sharing")
    _check(rt.lib.orqcu_swap(rt.h, int(arith), w, ctypes.c_size_t(n), len(x_vec), _flat(x_vec),
                             _flat(y_vec), _p3(bits.shares)))


def multiplex(sel, a, b):
    """orq::operators::multiplex (operators/common.h:20-49): b where sel is 1,
    else a. B-shared: a ^ (extend_lsb(sel) & (b ^ a)); A-shared: a + sel*(b - a)."""
    if isinstance(sel, BSharedVector):
        ext = BSharedVector(sel.rt, sel.rt._alloc(sel.size(), sel.width))
        ext.extend_lsb(sel)
        return a ^ (ext & (b ^ a))
    return a + sel * (b - a)


class aggregators:
    """Aggregation functions of orq::aggregators (aggregation.h:27-140), as the
    codes orqcu_aggregate takes."""
    sum, count, copy, valid, bit_or, min, max = range(7)


class Direction:
    Forward, Reverse = 0, 1


class _AggSpec(ctypes.Structure):
    _fields_ = [("inp", ctypes.c_void_p * 3), ("out", ctypes.c_void_p * 3), ("func", ctypes.c_int)]


def aggregate(keys, agg_spec_b, agg_spec_a, direction: int = Direction.Forward, sel=None):
    """orq::aggregators::aggregate (aggregation.h:167-346). keys: list of
    BSharedVector; agg_spec_b / agg_spec_a: lists of (input, output, function)
    with BSharedVector / ASharedVector columns; sel: optional BSharedVector
    (table id) restricting non-copy aggregations to rows of one table. The
    outputs are overwritten in place."""
    first = keys[0] if keys else (agg_spec_b or agg_spec_a)[0][1]
    rt, n, w = first.rt, first.size(), first.width
    kp = (ctypes.c_void_p * max(1, 3 * len(keys)))(*[k.shares[j].data_ptr() for k in keys for j in range(3)])

    def specs(lst):
        arr = (_AggSpec * max(1, len(lst)))()
        for i, (inp, out, f) in enumerate(lst):
            src = inp if inp is not None else out
            for j in range(3):
                arr[i].inp[j] = src.shares[j].data_ptr()
                arr[i].out[j] = out.shares[j].data_ptr()
            arr[i].func = int(f)
        return arr

    sp = _p3(sel.shares) if sel is not None else None
    _check(rt.lib.orqcu_aggregate(rt.h, w, ctypes.c_size_t(n), len(keys), kp, len(agg_spec_b),
                                  specs(agg_spec_b), len(agg_spec_a), specs(agg_spec_a),
                                  int(direction == Direction.Reverse), sp))


def _flat(vecs):
    return (ctypes.c_void_p * max(1, 3 * len(vecs)))(*[v.shares[j].data_ptr() for v in vecs for j in range(3)])


def compose_permutations(sigma: ASharedVector, rho: ASharedVector) -> ASharedVector:
    """orq::operators::compose_permutations (shuffle.h:717-743); sigma is
    consumed, rho is updated in place and returned."""
    rt = rho.rt
    _check(rt.lib.orqcu_compose_permutations(rt.h, ctypes.c_size_t(rho.size()), _p3(sigma.shares),
                                             _p3(rho.shares)))
    return rho


class SortingProtocol:
    """orq::SortingProtocol (sorting.h:15-21). The mirror's DEFAULT is RADIXSORT,
    the protocol of a reference built with DEFAULT_SORT_PROTO=RADIXSORT."""
    BITONICSORT, QUICKSORT, RADIXSORT = 0, 1, 2
    DEFAULT = 2


def table_sort(columns, data_a=(), data_b=(), order=None, single_bit=None,
               protocol: int = SortingProtocol.DEFAULT):
    """orq::operators::table_sort (sorting.h:509-612) with the quicksort or
    radix sort protocol: columns are B-shared key columns (most significant
    first), each sorted ASC/DESC per `order`, on one bit where `single_bit`
    says so; data columns are permuted along. Everything is updated in place."""
    rt, n, w = columns[0].rt, columns[0].size(), columns[0].width
    order = order or [ASC] * len(columns)
    single_bit = single_bit or [False] * len(columns)
    _check(rt.lib.orqcu_table_sort(rt.h, w, ctypes.c_size_t(n), len(columns), _flat(columns),
                                   (ctypes.c_int * len(columns))(*[int(o == DESC) for o in order]),
                                   (ctypes.c_int * len(columns))(*[int(bool(b)) for b in single_bit]),
                                   len(data_a), _flat(data_a), len(data_b), _flat(data_b), int(protocol)))


def distinct(keys) -> BSharedVector:
    """orq::operators::distinct (distinct.h:20-53) over adjacent rows."""
    rt, n, w = keys[0].rt, keys[0].size(), keys[0].width
    res = rt._alloc(n, w)
    _check(rt.lib.orqcu_distinct(rt.h, w, ctypes.c_size_t(n), len(keys), _flat(keys), _p3(res)))
    return BSharedVector(rt, res)


def bitonic_sort_batch(vectors, order=ASC, use_graph: bool = True):
    """Batched bitonic_sort of many independent key columns (power-of-two
    sizes, same width), in place: the shares equal those of calling
    bitonic_sort on each column in list order. `order` is one order or a list."""
    if not vectors:
        return
    rt, w = vectors[0].rt, vectors[0].width
    orders = order if isinstance(order, (list, tuple)) else [order] * len(vectors)
    ns = (ctypes.c_size_t * len(vectors))(*[v.size() for v in vectors])
    _check(rt.lib.orqcu_bitonic_sort_batch(rt.h, w, len(vectors), ns, _flat(vectors),
                                           (ctypes.c_int * len(vectors))(*[int(o == DESC) for o in orders]),
                                           int(bool(use_graph))))


def radix_sort_batch(vectors, order=ASC, bits=None):
    """Radix sorts of many independent B-shared key columns (same width), in
    place; returns their sorting permutations. Shares equal those of calling
    radix_sort on each column in list order; item i's bit passes overlap item
    i+1's permutation generation. `order` and `bits` are one value or a list."""
    if not vectors:
        return []
    rt, w = vectors[0].rt, vectors[0].width
    k = len(vectors)
    orders = order if isinstance(order, (list, tuple)) else [order] * k
    bl = bits if isinstance(bits, (list, tuple)) else [bits if bits is not None else 8 * w] * k
    perms = [ElementwisePermutation(rt, rt._alloc(v.size(), 4)) for v in vectors]
    ns = (ctypes.c_size_t * k)(*[v.size() for v in vectors])
    _check(rt.lib.orqcu_radix_sort_batch(rt.h, w, k, ns, _flat(vectors), (ctypes.c_int * k)(*bl),
                                         (ctypes.c_int * k)(*[int(o == DESC) for o in orders]), _flat(perms)))
    return perms


def quicksort(v: BSharedVector, order: int = ASC) -> ElementwisePermutation:
    """orq::operators::quicksort (quicksort.h:214-246): sorts v in place and
    returns the A-shared sorting permutation."""
    rt = v.rt
    perm = rt._alloc(v.size(), 4)
    _check(rt.lib.orqcu_quicksort(rt.h, v.width, ctypes.c_size_t(v.size()), _p3(v.shares),
                                  int(order == DESC), _p3(perm)))
    return ElementwisePermutation(rt, perm)


def radix_sort(v: BSharedVector, order: int = ASC, bits: int | None = None) -> ElementwisePermutation:
    """orq::operators::radix_sort (radixsort.h:205-229): sorts v in place and
    returns the A-shared sorting permutation."""
    rt = v.rt
    if bits is None:
        bits = 8 * v.width
    perm = rt._alloc(v.size(), 4)
    _check(rt.lib.orqcu_radix_sort(rt.h, v.width, ctypes.c_size_t(v.size()), _p3(v.shares),
                                   bits, int(order == DESC), _p3(perm)))
    return ElementwisePermutation(rt, perm)


# ---------------------------------------------------------------------------
# Beaver 2PC (dummy triples) and Fantastic-4PC: the local steps of ORQ's other
# protocol classes (include/core/protocols/beaver_2pc.h, dalskov_4pc.h), every
# party in this process. A vector is an (nparties, n) tensor of its distinct
# shares: S[0], S[1] for 2PC; X[0..3] for 4PC, X[j] being the share party j
# lacks.
class NPRuntime(Runtime):
    """Runtime of the Beaver-2PC (nparties=2) or Fantastic-4PC (4) protocol."""

    def __init__(self, nparties: int, seed: int = 1, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise OrqError("orq_b200 needs a CUDA device (no CPU fallback)")
        if nparties not in (2, 4):
            raise ValueError("nparties must be 2 or 4")
        self.lib = load_library()
        self.device = device
        self.nparties = nparties
        torch.cuda.set_device(device)
        h = ctypes.c_void_p()
        _check(self.lib.orqcu_runtime_create_np(ctypes.c_uint64(seed), device, nparties, ctypes.byref(h)))
        self.h = h
        _check(self.lib.orqcu_runtime_set_stream(self.h, ctypes.c_void_p(
            torch.cuda.current_stream(device).cuda_stream)))

    def _pn(self, t):
        return (ctypes.c_void_p * self.nparties)(*[t[j].data_ptr() for j in range(self.nparties)])

    def _new(self, n, w):
        torch = _torch()
        dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[w]
        return torch.empty((self.nparties, n), dtype=dt, device=f"cuda:{self.device}")

    def secret_share(self, data, arith: bool, party: int = 0):
        """secret_share_b / secret_share_a from `party`'s local PRG."""
        w = data.itemsize if isinstance(data, np.ndarray) else data.element_size()
        d = self._to_dev(data, w)
        s = self._new(d.shape[0], w)
        _check(self.lib.orqcu_np_secret_share(self.h, int(arith), w, ctypes.c_size_t(d.shape[0]),
                                              ctypes.c_void_p(d.data_ptr()), party, self._pn(s)))
        return s

    def open(self, s, arith: bool):
        torch = _torch()
        out = torch.empty(s.shape[1], dtype=s.dtype, device=s.device)
        _check(self.lib.orqcu_np_open(self.h, int(arith), s.element_size(), ctypes.c_size_t(s.shape[1]),
                                      self._pn(s), ctypes.c_void_p(out.data_ptr())))
        return out

    def _bin(self, fn, x, y):
        z = self._new(x.shape[1], x.element_size())
        _check(fn(self.h, x.element_size(), ctypes.c_size_t(x.shape[1]), self._pn(x), self._pn(y), self._pn(z)))
        return z

    def and_b(self, x, y):
        return self._bin(self.lib.orqcu_np_and_b, x, y)

    def multiply_a(self, x, y):
        return self._bin(self.lib.orqcu_np_multiply_a, x, y)

    def xor_b(self, x, y):
        return self._bin(self.lib.orqcu_np_xor_b, x, y)

    def add_a(self, x, y):
        return self._bin(self.lib.orqcu_np_add_a, x, y)

    def sub_a(self, x, y):
        return self._bin(self.lib.orqcu_np_sub_a, x, y)

    def b2a_bit(self, x):
        y = self._new(x.shape[1], x.element_size())
        _check(self.lib.orqcu_np_b2a_bit(self.h, x.element_size(), ctypes.c_size_t(x.shape[1]), self._pn(x),
                                         self._pn(y)))
        return y
