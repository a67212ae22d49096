// proto24.cu — the local steps of ORQ's other protocol classes, all parties in
// one process: Beaver 2PC with dummy triples (include/core/protocols/
// beaver_2pc.h, random/correlation/dummy_ole.h, beaver_triple_generator.h)
// and Fantastic-4PC (include/core/protocols/dalskov_4pc.h).
//
// Layout. A 2PC vector is S[0], S[1] (party p holds S[p]). A 4PC vector is
// X[0..3], X[j] being the share party j lacks; party p holds X[p+1], X[p+2],
// X[p+3] as its local shares 0, 1, 2 (get_shares, dalskov_4pc.h:152-168).
//
// Every opening and every jump-send of the CPU protocol is element-local, so
// and_b / multiply_a / b2a_bit are one pass each: a thread owns a 16-byte unit
// of every share array, computes the AES blocks its correlated randomness
// needs, and writes the result shares.
#include "launch.cuh"

namespace orqcu {

namespace {

template <int W>
__device__ __forceinline__ uint4 lsb_one() {
    if constexpr (W == 1) return make_uint4(0x01010101u, 0x01010101u, 0x01010101u, 0x01010101u);
    if constexpr (W == 2) return make_uint4(0x00010001u, 0x00010001u, 0x00010001u, 0x00010001u);
    if constexpr (W == 4) return make_uint4(1u, 1u, 1u, 1u);
    return make_uint4(1u, 0u, 1u, 0u);
}

// bytes [r, r + 16) of the 32 bytes lo | hi (r uniform, 0..15)
__device__ __forceinline__ uint4 extract16(uint4 lo, uint4 hi, int r) {
    const int ws = r >> 2, bs = (r & 3) * 8;
    const uint32_t w0 = ws == 0 ? lo.x : ws == 1 ? lo.y : ws == 2 ? lo.z : lo.w;
    const uint32_t w1 = ws == 0 ? lo.y : ws == 1 ? lo.z : ws == 2 ? lo.w : hi.x;
    const uint32_t w2 = ws == 0 ? lo.z : ws == 1 ? lo.w : ws == 2 ? hi.x : hi.y;
    const uint32_t w3 = ws == 0 ? lo.w : ws == 1 ? hi.x : ws == 2 ? hi.y : hi.z;
    const uint32_t w4 = ws == 0 ? hi.x : ws == 1 ? hi.y : ws == 2 ? hi.z : hi.w;
    return make_uint4(__funnelshift_r(w0, w1, bs), __funnelshift_r(w1, w2, bs), __funnelshift_r(w2, w3, bs),
                      __funnelshift_r(w3, w4, bs));
}

struct P2Args {
    const void* x[2];
    const void* y[2];
    void* z[2];
    StreamArg common;           // the {0,1} PRG at the first of the three draws
    unsigned long long ch2;     // nonces per draw of 2n elements
    unsigned long long nbytes;  // n * W
};

// Beaver-triple multiply_a / and_b (beaver_2pc.h:50-59,108-117) with the
// dummy triple of the same call. DummyOLE::getNext(2n) (dummy_ole.h) draws
// B, C, D of 2n elements from the {0,1} PRG; A = C*D - B (B ^ C&D); party 0
// holds (A, C), party 1 (B, D). The triple (beaver_triple_generator.h:getNext)
// is a0 = C[:n], b0 = C[n:], c0 = a0*b0 + A[:n] + A[n:]; a1 = D[n:],
// b1 = D[:n], c1 = a1*b1 + B[:n] + B[n:]. With A' = open(x + a) and
// B' = open(y + b): z_p = y_p*A' - a_p*B' + c_p. B2A: the operands are
// b2a_bit's (beaver_2pc.h:147-158) x & 1 with party 1's share negated,
// multiplied by themselves.
template <int W, bool ARITH, bool B2A>
__global__ void __launch_bounds__(kAesThreads) k_p2_mult(P2Args a) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    const unsigned long long rb = a.nbytes >> 4;  // first block of the right half
    const int r = (int)(a.nbytes & 15);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        // draws B, C, D (left and right halves), rotated through static slots
        uint4 Bl, Cl, Dl, Br, Cr, Dr;
        Bl = Cl = Dl = Br = Cr = Dr = make_uint4(0, 0, 0, 0);
#pragma unroll 1
        for (int d = 0; d < 3; d++) {
            StreamArg st = a.common;
            st.nonce += (unsigned long long)d * a.ch2;
            const uint4 l = keystream_block(S, st, b);
            uint4 rr = keystream_block(S, st, rb + b);
            if (r) rr = extract16(rr, keystream_block(S, st, rb + b + 1), r);
            Bl = Cl;
            Cl = Dl;
            Dl = l;
            Br = Cr;
            Cr = Dr;
            Dr = rr;
        }
        const uint4 Al = Sh::minus(Sh::times(Cl, Dl), Bl), Ar = Sh::minus(Sh::times(Cr, Dr), Br);
        const uint4 a0 = Cl, b0 = Cr, c0 = Sh::plus(Sh::plus(Sh::times(a0, b0), Al), Ar);
        const uint4 a1 = Dr, b1 = Dl, c1 = Sh::plus(Sh::plus(Sh::times(a1, b1), Bl), Br);
        uint4 x0 = ld16(a.x[0], b, a.nbytes), x1 = ld16(a.x[1], b, a.nbytes);
        uint4 y0, y1;
        if constexpr (B2A) {
            const uint4 one = lsb_one<W>();
            x0 = x0 & one;
            x1 = Ring<W>::sub(make_uint4(0, 0, 0, 0), x1 & one);
            y0 = x0;
            y1 = x1;
        } else {
            y0 = ld16(a.y[0], b, a.nbytes);
            y1 = ld16(a.y[1], b, a.nbytes);
        }
        const uint4 Ao = Sh::plus(Sh::plus(x0, a0), Sh::plus(x1, a1));
        const uint4 Bo = Sh::plus(Sh::plus(y0, b0), Sh::plus(y1, b1));
        st16(a.z[0], b, a.nbytes, Sh::plus(Sh::minus(Sh::times(y0, Ao), Sh::times(a0, Bo)), c0));
        st16(a.z[1], b, a.nbytes, Sh::plus(Sh::minus(Sh::times(y1, Ao), Sh::times(a1, Bo)), c1));
    }
}

struct P4Args {
    const void* x[4];
    const void* y[4];
    void* z[4];
    StreamArg st[8];  // the six pair draws in pair order; for b2a_bit then NOT2, NOT0 of the inputs
    unsigned long long nbytes;
};

// Fantastic-4PC multiply_a / and_b (dalskov_4pc.h:384-420,479-506): for the
// pairs (i,j) = (0,1) (0,2) (0,3) (1,2) (1,3) (2,3), with g = next_party(i,j)
// and h the fourth party, inp (dalskov_4pc.h:300-340) shares
// v = X_h*Y_g + X_g*Y_h as X'_g = R (the PRG of the three parties other than
// g), X'_h = v - R; the result is the sum of the six sharings plus X_k*Y_k in
// every share. (g, h) per pair: (2,3) (1,3) (1,2) (3,0) (2,0) (0,1).
// B2A (dalskov_4pc.h:562-590): the operands are inp(X2^X3 bit, 1, 0) minus
// inp(X0^X1 bit, 3, 2), squared.
template <int W, bool ARITH, bool B2A>
__global__ void __launch_bounds__(kAesThreads) k_p4_mult(P4Args a) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        uint4 k0, k1, k2, k3, k4, k5;
        k0 = k1 = k2 = k3 = k4 = k5 = make_uint4(0, 0, 0, 0);
#pragma unroll 1
        for (int p = 0; p < 6; p++) {
            const uint4 k = keystream_block(S, a.st[p], b);
            k0 = k1;
            k1 = k2;
            k2 = k3;
            k3 = k4;
            k4 = k5;
            k5 = k;
        }
        uint4 X[4], Y[4];
        if constexpr (B2A) {
            const uint4 one = lsb_one<W>(), zero = make_uint4(0, 0, 0, 0);
            uint4 x[4];
#pragma unroll
            for (int j = 0; j < 4; j++) x[j] = ld16(a.x[j], b, a.nbytes);
            const uint4 s0 = (x[2] ^ x[3]) & one, s1 = (x[0] ^ x[1]) & one;
            const uint4 R2 = keystream_block(S, a.st[6], b), R0 = keystream_block(S, a.st[7], b);
            X[0] = Ring<W>::sub(zero, R0);
            X[1] = Ring<W>::sub(R0, s1);
            X[2] = R2;
            X[3] = Ring<W>::sub(s0, R2);
#pragma unroll
            for (int j = 0; j < 4; j++) Y[j] = X[j];
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                X[j] = ld16(a.x[j], b, a.nbytes);
                Y[j] = ld16(a.y[j], b, a.nbytes);
            }
        }
        uint4 acc[4];
#pragma unroll
        for (int j = 0; j < 4; j++) acc[j] = Sh::times(X[j], Y[j]);
        const uint4 R[6] = {k0, k1, k2, k3, k4, k5};
        constexpr int G[6] = {2, 1, 1, 3, 2, 0}, H[6] = {3, 3, 2, 0, 0, 1};
#pragma unroll
        for (int p = 0; p < 6; p++) {
            const int g = G[p], h = H[p];
            const uint4 v = Sh::plus(Sh::times(X[h], Y[g]), Sh::times(X[g], Y[h]));
            acc[g] = Sh::plus(acc[g], R[p]);
            acc[h] = Sh::plus(acc[h], Sh::minus(v, R[p]));
        }
#pragma unroll
        for (int j = 0; j < 4; j++) st16(a.z[j], b, a.nbytes, acc[j]);
    }
}

// secret_share (beaver_2pc.h:214-260; dalskov_4pc.h:152-201): the owner d
// draws `draws` vectors from its local PRG; 2PC: S[d] = r, S[1-d] = data - r;
// 4PC: X[(d+k)%4] = s_k (k < 3), X[(d+3)%4] = data - s0 - s1 - s2.
template <int W, bool ARITH>
__global__ void __launch_bounds__(kAesThreads)
    k_np_share(const uint8_t* data, void* out0, void* out1, void* out2, void* out3, StreamArg st,
               unsigned long long ch, int draws, unsigned long long nbytes) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(nbytes, 16);
    void* outs[3] = {out0, out1, out2};
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        uint4 rest = ld16(data, b, nbytes);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (k < draws) {
                StreamArg s = st;
                s.nonce += (unsigned long long)k * ch;
                const uint4 r = keystream_block(S, s, b);
                st16(outs[k], b, nbytes, r);
                rest = Sh::minus(rest, r);
            }
        }
        st16(draws == 1 ? out1 : out3, b, nbytes, rest);
    }
}

template <int W, bool ARITH>
__global__ void k_np_open(const void* s0, const void* s1, const void* s2, const void* s3, int np, void* out,
                          unsigned long long nbytes) {
    using Sh = Share<W, ARITH>;
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        uint4 v = Sh::plus(ld16(s0, b, nbytes), ld16(s1, b, nbytes));
        if (np == 4) v = Sh::plus(Sh::plus(v, ld16(s2, b, nbytes)), ld16(s3, b, nbytes));
        st16(out, b, nbytes, v);
    }
}

struct NpLocalArgs {
    const void* x[4];
    const void* y[4];
    void* z[4];
    int np;
    unsigned long long nbytes;
};
template <int W, int OP>
__global__ void k_np_local(NpLocalArgs a) {
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (k < a.np) {
                const uint4 x = ld16(a.x[k], b, a.nbytes), y = ld16(a.y[k], b, a.nbytes);
                uint4 v;
                if constexpr (OP == 0) v = x ^ y;
                else if constexpr (OP == 1) v = Ring<W>::add(x, y);
                else v = Ring<W>::sub(x, y);
                st16(a.z[k], b, a.nbytes, v);
            }
        }
    }
}

#define ORQ_DISPATCH_W124(w, ...)                                                    \
    switch (w) {                                                                     \
        case 1: { constexpr int W = 1; __VA_ARGS__; } break;                         \
        case 2: { constexpr int W = 2; __VA_ARGS__; } break;                         \
        case 4: { constexpr int W = 4; __VA_ARGS__; } break;                         \
        case 8: { constexpr int W = 8; __VA_ARGS__; } break;                         \
        default: throw std::invalid_argument("share width must be 1, 2, 4 or 8 bytes"); \
    }

void need_np(const Ctx& c) {
    if (c.nparties != 2 && c.nparties != 4)
        throw std::invalid_argument("this runtime runs replicated 3PC; create one with orqcu_runtime_create_np");
}
void need_w124(int w) {
    if (w != 1 && w != 2 && w != 4 && w != 8) throw std::invalid_argument("share width must be 1, 2, 4 or 8 bytes");
}

// the six pair draws of one 4PC multiplication from the PRGs that exclude g,
// each PRG advancing by one draw per use (the b2a pre-stage has used NOT2 and
// NOT0 once already when pre = true)
void p4_pair_streams(Ctx& c, unsigned long long ch, StreamArg st[6], unsigned long long used[4]) {
    static const int G[6] = {2, 1, 1, 3, 2, 0};
    for (int p = 0; p < 6; p++) {
        const int g = G[p];
        st[p] = c.stream_arg(P4_NOT0 + g, used[g] * ch);
        used[g]++;
    }
}

}  // namespace

void op_np_secret_share(Ctx& c, bool arith, int w, size_t n, const void* data, int party, void* const* s) {
    need_np(c);
    need_w124(w);
    const int np = c.nparties;
    if (party < 0 || party >= np) throw std::invalid_argument("data party out of range");
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    const int draws = np == 2 ? 1 : 3;
    const int local = (np == 2 ? P2_LOCAL0 : P4_LOCAL0) + party;
    StreamArg st = c.stream_arg(local);
    if (nb) {
        void* o[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int k = 0; k < np; k++) o[k] = s[(party + k) % np];
        ORQ_DISPATCH_W124(w, {
            {
                const double by = (1.0 + np) * nb, bl = (double)draws * ceil_div(nb, 16);
                if (arith)
                    launch_aes(c, "np_share", by, bl, k_np_share<W, true>, ceil_div(nb, 16), (const uint8_t*)data, o[0], o[1],
                               o[2], o[3], st, ch, draws, nb);
                else
                    launch_aes(c, "np_share", by, bl, k_np_share<W, false>, ceil_div(nb, 16), (const uint8_t*)data, o[0], o[1],
                               o[2], o[3], st, ch, draws, nb);
            }
        });
    }
    c.nonce[local] += (unsigned long long)draws * ch;
}

void op_np_open(Ctx& c, bool arith, int w, size_t n, const void* const* s, void* out) {
    need_np(c);
    need_w124(w);
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    const int np = c.nparties;
    ProfScope ps(c, "np_open", (1.0 + np) * nb);
    const unsigned g = plain_grid(c, ceil_div(nb, 16));
    const void* s2 = np == 4 ? s[2] : s[0];
    const void* s3 = np == 4 ? s[3] : s[0];
    ORQ_DISPATCH_W124(w, {
        {
            if (arith) k_np_open<W, true><<<g, 256, 0, c.stream>>>(s[0], s[1], s2, s3, np, out, nb);
            else k_np_open<W, false><<<g, 256, 0, c.stream>>>(s[0], s[1], s2, s3, np, out, nb);
        }
    });
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

void op_np_local(Ctx& c, int op, int w, size_t n, const void* const* x, const void* const* y, void* const* z) {
    need_np(c);
    need_w124(w);
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    NpLocalArgs a{};
    a.np = c.nparties;
    for (int k = 0; k < a.np; k++) {
        a.x[k] = x[k];
        a.y[k] = y[k];
        a.z[k] = z[k];
    }
    a.nbytes = nb;
    const unsigned g = plain_grid(c, ceil_div(nb, 16));
    ProfScope ps(c, "np_local", 3.0 * a.np * nb);
    ORQ_DISPATCH_W124(w, {
        {
            if (op == 0) k_np_local<W, 0><<<g, 256, 0, c.stream>>>(a);
            else if (op == 1) k_np_local<W, 1><<<g, 256, 0, c.stream>>>(a);
            else if (op == 2) k_np_local<W, 2><<<g, 256, 0, c.stream>>>(a);
            else throw std::invalid_argument("unknown local op");
        }
    });
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

// mode: 0 and_b, 1 multiply_a, 2 b2a_bit (y unused)
void op_np_mult(Ctx& c, int mode, int w, size_t n, const void* const* x, const void* const* y, void* const* z) {
    need_np(c);
    need_w124(w);
    const unsigned long long nb = (unsigned long long)n * w;
    if (c.nparties == 2) {
        const unsigned long long ch2 = chunks_of(2 * nb);
        if (nb) {
            P2Args a{};
            for (int p = 0; p < 2; p++) {
                a.x[p] = x[p];
                a.y[p] = mode == 2 ? x[p] : y[p];
                a.z[p] = z[p];
            }
            a.common = c.stream_arg(P2_COMMON);
            a.ch2 = ch2;
            a.nbytes = nb;
            const double by = (mode == 2 ? 4.0 : 6.0) * nb, bl = (nb & 15 ? 9.0 : 6.0) * ceil_div(nb, 16);
            ORQ_DISPATCH_W124(w, {
                {
                    if (mode == 0) launch_aes(c, "p2_and_b", by, bl, k_p2_mult<W, false, false>, ceil_div(nb, 16), a);
                    else if (mode == 1) launch_aes(c, "p2_multiply_a", by, bl, k_p2_mult<W, true, false>, ceil_div(nb, 16), a);
                    else launch_aes(c, "p2_b2a_bit", by, bl, k_p2_mult<W, true, true>, ceil_div(nb, 16), a);
                }
            });
        }
        c.nonce[P2_COMMON] += 3 * ch2;
        return;
    }
    const unsigned long long ch = chunks_of(nb);
    unsigned long long used[4] = {0, 0, 0, 0};
    P4Args a{};
    if (mode == 2) {
        // the b2a inputs: inp(s0, 1, 0) draws from NOT2, then inp(s1, 3, 2) from NOT0
        a.st[6] = c.stream_arg(P4_NOT0 + 2, 0);
        a.st[7] = c.stream_arg(P4_NOT0 + 0, 0);
        used[2] = used[0] = 1;
    }
    p4_pair_streams(c, ch, a.st, used);
    for (int j = 0; j < 4; j++) {
        a.x[j] = x[j];
        a.y[j] = mode == 2 ? x[j] : y[j];
        a.z[j] = z[j];
    }
    a.nbytes = nb;
    if (nb) {
        const double by = (mode == 2 ? 8.0 : 12.0) * nb, bl = (mode == 2 ? 8.0 : 6.0) * ceil_div(nb, 16);
        ORQ_DISPATCH_W124(w, {
            {
                if (mode == 0) launch_aes(c, "p4_and_b", by, bl, k_p4_mult<W, false, false>, ceil_div(nb, 16), a);
                else if (mode == 1) launch_aes(c, "p4_multiply_a", by, bl, k_p4_mult<W, true, false>, ceil_div(nb, 16), a);
                else launch_aes(c, "p4_b2a_bit", by, bl, k_p4_mult<W, true, true>, ceil_div(nb, 16), a);
            }
        });
    }
    for (int g = 0; g < 4; g++) c.nonce[P4_NOT0 + g] += used[g] * ch;
}

}  // namespace orqcu
