// party.cu — one party of replicated 3PC on the GPU, beside CPU parties.
//
// The loopback kernels compute every party's local step at once. A runtime
// created with orqcu_party_runtime_create plays ONE party p instead: it holds
// p's two shares (S[p], S[p+1]) and only the PRG keys p holds (its local key,
// its pairwise key, the key received from p-1, the groups it belongs to), and
// each kernel here computes p's local step of a Replicated_3PC primitive
// (include/core/protocols/replicated_3pc.h). The exchange that follows each
// step is the host's: the caller moves the arrays over its communicator
// (include/orq_b200/nocopy.hpp speaks ORQ's NoCopy socket format), so a GPU
// party runs with CPU parties of the reference unchanged.
//
// Nonces: party p's PRG objects advance exactly as the CPU party's do; one
// zero-sharing draw advances PAIR[p-1] and PAIR[p] by the chunk count.
#include "launch.cuh"

namespace orqcu {

namespace {

template <int W>
__device__ __forceinline__ uint4 lsb_one() {
    if constexpr (W == 1) return make_uint4(0x01010101u, 0x01010101u, 0x01010101u, 0x01010101u);
    if constexpr (W == 2) return make_uint4(0x00010001u, 0x00010001u, 0x00010001u, 0x00010001u);
    if constexpr (W == 4) return make_uint4(1u, 1u, 1u, 1u);
    if constexpr (W == 8) return make_uint4(1u, 0u, 1u, 0u);
    return make_uint4(1u, 0u, 0u, 0u);
}

struct PMultArgs {
    const void* x[2];
    const void* y[2];
    void* z;
    StreamArg prev, self;  // PAIR[p-1] (get(-1)) and PAIR[p] (get(+1))
    unsigned long long nbytes;
};

// and_b / multiply_a of party p (replicated_3pc.h:44-67,166-191): the zero
// share prev (-|^) self plus x0·y0 + x0·y1 + x1·y0. With SUB, the inputs are
// the exchanged (s0, s1) of b2a_bit and the product is (s0 - s1)^2
// (replicated_3pc.h:247-250).
template <int W, bool ARITH, bool SUB>
__global__ void __launch_bounds__(kAesThreads) k_pmult(PMultArgs a) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        const uint4 kp = keystream_block(S, a.prev, b);
        const uint4 ks = keystream_block(S, a.self, b);
        uint4 x0 = ld16(a.x[0], b, a.nbytes), x1 = ld16(a.x[1], b, a.nbytes);
        uint4 y0, y1;
        if constexpr (SUB) {
            x0 = Ring<W>::sub(x0, ld16(a.y[0], b, a.nbytes));
            x1 = Ring<W>::sub(x1, ld16(a.y[1], b, a.nbytes));
            y0 = x0;
            y1 = x1;
        } else {
            y0 = ld16(a.y[0], b, a.nbytes);
            y1 = ld16(a.y[1], b, a.nbytes);
        }
        uint4 v = Sh::plus(Sh::minus(kp, ks), Sh::times(x0, y0));
        v = Sh::plus(v, Sh::times(x0, y1));
        v = Sh::plus(v, Sh::times(x1, y0));
        st16(a.z, b, a.nbytes, v);
    }
}

struct PB2AArgs {
    const void* x[2];
    void* s0;
    void* s1;
    StreamArg prev, self;
    unsigned long long chunks;
    int party;
    unsigned long long nbytes;
};

// First half of b2a_bit (replicated_3pc.h:220-245) for party p: two
// arithmetic zero shares; P0 adds the LSB of x0 ^ x1 to the first, P1 the LSB
// of its second share to the second. The caller exchanges both.
template <int W>
__global__ void __launch_bounds__(kAesThreads) k_pb2a_pre(PB2AArgs a) {
    using R = Ring<W>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const uint4 one = lsb_one<W>();
    StreamArg prev2 = a.prev, self2 = a.self;
    prev2.nonce += a.chunks;
    self2.nonce += a.chunks;
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        uint4 z0 = R::sub(keystream_block(S, a.prev, b), keystream_block(S, a.self, b));
        uint4 z1 = R::sub(keystream_block(S, prev2, b), keystream_block(S, self2, b));
        if (a.party == 0) {
            z0 = R::add(z0, (ld16(a.x[0], b, a.nbytes) ^ ld16(a.x[1], b, a.nbytes)) & one);
        } else if (a.party == 1) {
            z1 = R::add(z1, ld16(a.x[1], b, a.nbytes) & one);
        }
        st16(a.s0, b, a.nbytes, z0);
        st16(a.s1, b, a.nbytes, z1);
    }
}

struct PLocalArgs {
    const void* x[2];
    const void* y[2];
    void* z[2];
    unsigned long long nbytes;
};
// xor / add / sub of both local shares (replicated_3pc.h: the share-local ops)
template <int W, int OP>
__global__ void k_plocal(PLocalArgs a) {
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const uint4 x = ld16(a.x[k], b, a.nbytes), y = ld16(a.y[k], b, a.nbytes);
            uint4 v;
            if constexpr (OP == 0) v = x ^ y;
            else if constexpr (OP == 1) v = Ring<W>::add(x, y);
            else v = Ring<W>::sub(x, y);
            st16(a.z[k], b, a.nbytes, v);
        }
    }
}

void need_party(const Ctx& c) {
    if (c.party < 0 || c.party > 2) throw std::invalid_argument("this runtime is not a one-party runtime");
}

}  // namespace

// ---------------------------------------------------------------------------
void op_party_mult(Ctx& c, bool arith, int w, size_t n, const void* const x[2], const void* const y[2], void* z) {
    need_party(c);
    const int p = c.party;
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    PMultArgs a;
    for (int k = 0; k < 2; k++) {
        a.x[k] = x[k];
        a.y[k] = y[k];
    }
    a.z = z;
    a.prev = c.stream_arg(PAIR0 + (p + 2) % 3);
    a.self = c.stream_arg(PAIR0 + p);
    a.nbytes = nb;
    if (nb) {
        ORQ_DISPATCH_W(w, {
            const double by = 5.0 * nb, bl = 2.0 * ceil_div(nb, 16);
            if (arith) launch_aes(c, "party_multiply_a", by, bl, k_pmult<W, true, false>, ceil_div(nb, 16), a);
            else launch_aes(c, "party_and_b", by, bl, k_pmult<W, false, false>, ceil_div(nb, 16), a);
        });
    }
    c.nonce[PAIR0 + (p + 2) % 3] += ch;
    c.nonce[PAIR0 + p] += ch;
}

void op_party_b2a_pre(Ctx& c, int w, size_t n, const void* const x[2], void* s0, void* s1) {
    need_party(c);
    const int p = c.party;
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    PB2AArgs a;
    a.x[0] = x[0];
    a.x[1] = x[1];
    a.s0 = s0;
    a.s1 = s1;
    a.prev = c.stream_arg(PAIR0 + (p + 2) % 3);
    a.self = c.stream_arg(PAIR0 + p);
    a.chunks = ch;
    a.party = p;
    a.nbytes = nb;
    if (nb) {
        ORQ_DISPATCH_W(w, { launch_aes(c, "party_b2a_pre", 4.0 * nb, 4.0 * ceil_div(nb, 16), k_pb2a_pre<W>, ceil_div(nb, 16), a); });
    }
    c.nonce[PAIR0 + (p + 2) % 3] += 2 * ch;
    c.nonce[PAIR0 + p] += 2 * ch;
}

void op_party_b2a_post(Ctx& c, int w, size_t n, const void* const s0[2], const void* const s1[2], void* z) {
    need_party(c);
    const int p = c.party;
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    PMultArgs a;
    for (int k = 0; k < 2; k++) {
        a.x[k] = s0[k];
        a.y[k] = s1[k];
    }
    a.z = z;
    a.prev = c.stream_arg(PAIR0 + (p + 2) % 3);
    a.self = c.stream_arg(PAIR0 + p);
    a.nbytes = nb;
    if (nb) {
        ORQ_DISPATCH_W(w, { launch_aes(c, "party_b2a_post", 5.0 * nb, 2.0 * ceil_div(nb, 16), k_pmult<W, true, true>, ceil_div(nb, 16), a); });
    }
    c.nonce[PAIR0 + (p + 2) % 3] += ch;
    c.nonce[PAIR0 + p] += ch;
}

void op_party_local(Ctx& c, int op, int w, size_t n, const void* const x[2], const void* const y[2], void* const z[2]) {
    need_party(c);
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    PLocalArgs a;
    for (int k = 0; k < 2; k++) {
        a.x[k] = x[k];
        a.y[k] = y[k];
        a.z[k] = z[k];
    }
    a.nbytes = nb;
    const unsigned g = plain_grid(c, ceil_div(nb, 16));
    ProfScope ps(c, "party_local", 6.0 * nb);
    ORQ_DISPATCH_W(w, {
        if (op == 0) k_plocal<W, 0><<<g, 256, 0, c.stream>>>(a);
        else if (op == 1) k_plocal<W, 1><<<g, 256, 0, c.stream>>>(a);
        else if (op == 2) k_plocal<W, 2><<<g, 256, 0, c.stream>>>(a);
        else throw std::invalid_argument("unknown local op");
    });
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

// secret_share_b/a on the data owner (replicated_3pc.h:401-448): the owner's
// local PRG draws S[p] and S[p+1]; S[p+2] completes the sharing. `s` is
// indexed by absolute share number.
void op_party_share(Ctx& c, bool arith, int w, size_t n, const void* data, Sh3 s) {
    need_party(c);
    op_secret_share(c, arith, w, n, data, c.party, s);
}

// open_shares_b/a (replicated_3pc.h:310-330) after the exchange: the party's
// two shares and the one received from p+1.
void op_party_open(Ctx& c, bool arith, int w, size_t n, const void* const x[2], const void* third, void* out) {
    need_party(c);
    op_open(c, arith, w, n, CSh3{{x[0], x[1], third}}, out);
}

}  // namespace orqcu
