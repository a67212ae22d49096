// prims.cu — replicated-3PC primitives fused with their correlated randomness.
//
// Each kernel computes, for all three parties at once, the local step of an
// ORQ protocol primitive together with the AES keystream it consumes, and
// writes the post-exchange shares directly (in loopback the ±1 exchange of
// Replicated_3PC is the identity on the distinct-share layout: party p's
// "remote" share is party p+1's "local" one, include/core/protocols/
// replicated_3pc.h:60,183). One thread owns one 16-byte unit of every share
// array and the matching AES block of every stream it needs.
#include "launch.cuh"

namespace orqcu {

namespace {

template <int W>
__device__ __forceinline__ uint4 lsb_mask() {
    if constexpr (W == 1) return make_uint4(0x01010101u, 0x01010101u, 0x01010101u, 0x01010101u);
    if constexpr (W == 2) return make_uint4(0x00010001u, 0x00010001u, 0x00010001u, 0x00010001u);
    if constexpr (W == 4) return make_uint4(1u, 1u, 1u, 1u);
    if constexpr (W == 8) return make_uint4(1u, 0u, 1u, 0u);
    return make_uint4(1u, 0u, 0u, 0u);
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kAesThreads) k_keystream(StreamArg st, uint8_t* out,
                                                           unsigned long long nbytes) {
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride())
        st16(out, b, nbytes, keystream_block(S, st, b));
}

// secret_share_b/a on the owner (replicated_3pc.h:353-448): share_1, share_2
// are two consecutive draws of the owner's local PRG.
template <int W, bool ARITH>
__global__ void __launch_bounds__(kAesThreads)
    k_share(const uint8_t* data, void* s1, void* s2, void* s3, StreamArg st,
            unsigned long long chunks, unsigned long long nbytes) {
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    StreamArg st2 = st;
    st2.nonce += chunks;
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        const uint4 a = keystream_block(S, st, b);
        const uint4 c = keystream_block(S, st2, b);
        const uint4 d = ld16(data, b, nbytes);
        st16(s1, b, nbytes, a);
        st16(s2, b, nbytes, c);
        st16(s3, b, nbytes, Share<W, ARITH>::minus(Share<W, ARITH>::minus(d, a), c));
    }
}

struct MultArgs {
    const void* x[3];
    const void* y[3];
    void* z[3];
    StreamArg pair[3];
    unsigned long long nbytes;
};

// and_b / multiply_a (replicated_3pc.h:44-67,166-191) with the zero-sharing
// of ZeroSharingGenerator::getNextBinary/Arithmetic (zero_sharing_generator.h:
// 101-148): r_p = PAIR[p-1] (-|^) PAIR[p].
template <int W, bool ARITH>
__global__ void __launch_bounds__(kAesThreads) k_mult(MultArgs a) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        const uint4 k0 = keystream_block(S, a.pair[0], b);
        const uint4 k1 = keystream_block(S, a.pair[1], b);
        const uint4 k2 = keystream_block(S, a.pair[2], b);
        uint4 x[3], y[3];
#pragma unroll
        for (int p = 0; p < 3; p++) {
            x[p] = ld16(a.x[p], b, a.nbytes);
            y[p] = ld16(a.y[p], b, a.nbytes);
        }
        const uint4 r[3] = {Sh::minus(k2, k0), Sh::minus(k0, k1), Sh::minus(k1, k2)};
#pragma unroll
        for (int p = 0; p < 3; p++) {
            const int q = (p + 1) % 3;
            uint4 v = Sh::plus(r[p], Sh::times(x[p], y[p]));
            v = Sh::plus(v, Sh::times(x[p], y[q]));
            v = Sh::plus(v, Sh::times(x[q], y[p]));
            st16(a.z[p], b, a.nbytes, v);
        }
    }
}

struct B2AArgs {
    const void* x[3];
    void* y[3];
    StreamArg pair[3];
    unsigned long long chunks;
    unsigned long long nbytes;
};

// b2a_bit (replicated_3pc.h:220-251): three arithmetic zero-sharings (two for
// s0/s1, one inside multiply_a) and the two exchanges are element-local in
// loopback, so the whole conversion is one pass.
template <int W>
__global__ void __launch_bounds__(kAesThreads) k_b2a(B2AArgs a) {
    using R = Ring<W>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const uint4 one = lsb_mask<W>();
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        // z[call][party]; the call loop stays rolled (three AES bodies, not
        // nine, keep the loop inside the instruction cache): each call shifts
        // the rows up and appends its own, so z[c] ends up holding call c
        uint4 z[3][3] = {};
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            uint4 k[3];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                StreamArg st = a.pair[q];
                st.nonce += (unsigned long long)c * a.chunks;
                k[q] = keystream_block(S, st, b);
            }
#pragma unroll
            for (int p = 0; p < 3; p++) {
                z[0][p] = z[1][p];
                z[1][p] = z[2][p];
            }
            z[2][0] = R::sub(k[2], k[0]);
            z[2][1] = R::sub(k[0], k[1]);
            z[2][2] = R::sub(k[1], k[2]);
        }
        const uint4 x0 = ld16(a.x[0], b, a.nbytes), x1 = ld16(a.x[1], b, a.nbytes),
                    x2 = ld16(a.x[2], b, a.nbytes);
        const uint4 abit = (x0 ^ x1) & one;  // P0 folds its two masked shares
        const uint4 bbit = x2 & one;         // P1 adds its second masked share
        uint4 d[3];
        d[0] = R::sub(R::add(z[0][0], abit), z[1][0]);
        d[1] = R::sub(z[0][1], R::add(z[1][1], bbit));
        d[2] = R::sub(z[0][2], z[1][2]);
#pragma unroll
        for (int p = 0; p < 3; p++) {
            const int q = (p + 1) % 3;
            uint4 v = R::add(z[2][p], R::mul(d[p], d[p]));
            v = R::add(v, R::mul(d[p], d[q]));
            v = R::add(v, R::mul(d[q], d[p]));
            st16(a.y[p], b, a.nbytes, v);
        }
    }
}

// Protocol::reshare (protocol.h:500-541) in place: r0, r1 from the group
// stream, r2 = r0^r1 or -r0-r1 (zero_sharing_generator.h:158-183).
template <int W, bool ARITH>
__global__ void __launch_bounds__(kAesThreads)
    k_reshare(void* s0, void* s1, void* s2, StreamArg g, unsigned long long chunks,
              unsigned long long nbytes) {
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    StreamArg g2 = g;
    g2.nonce += chunks;
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        const uint4 r0 = keystream_block(S, g, b);
        const uint4 r1 = keystream_block(S, g2, b);
        uint4 r2;
        if constexpr (ARITH) r2 = Ring<W>::sub(Ring<W>::sub(make_uint4(0, 0, 0, 0), r0), r1);
        else r2 = r0 ^ r1;
        st16(s0, b, nbytes, Share<W, ARITH>::plus(ld16(s0, b, nbytes), r0));
        st16(s1, b, nbytes, Share<W, ARITH>::plus(ld16(s1, b, nbytes), r1));
        st16(s2, b, nbytes, Share<W, ARITH>::plus(ld16(s2, b, nbytes), r2));
    }
}

template <int W, bool ARITH>
__global__ void __launch_bounds__(kAesThreads)
    k_zero(void* r0o, void* r1o, void* r2o, StreamArg p0, StreamArg p1, StreamArg p2,
           unsigned long long nbytes) {
    using Sh = Share<W, ARITH>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
        const uint4 k0 = keystream_block(S, p0, b);
        const uint4 k1 = keystream_block(S, p1, b);
        const uint4 k2 = keystream_block(S, p2, b);
        st16(r0o, b, nbytes, Sh::minus(k2, k0));
        st16(r1o, b, nbytes, Sh::minus(k0, k1));
        st16(r2o, b, nbytes, Sh::minus(k1, k2));
    }
}

// ---- local (communication-free) ops ---------------------------------------
template <int W, bool ARITH>
__global__ void k_open(const void* s0, const void* s1, const void* s2, void* out,
                       unsigned long long nbytes) {
    using Sh = Share<W, ARITH>;
    const unsigned long long nblk = ceil_div(nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride())
        st16(out, b, nbytes,
             Sh::plus(Sh::plus(ld16(s0, b, nbytes), ld16(s1, b, nbytes)), ld16(s2, b, nbytes)));
}

struct LocalArgs {
    const void* x[3];
    const void* y[3];
    void* z[3];
    unsigned long long nbytes;
};
template <int W, int OP>
__global__ void k_local(LocalArgs a) {
    const unsigned long long nblk = ceil_div(a.nbytes, 16);
    for (unsigned long long b = gtid(); b < nblk; b += gstride()) {
#pragma unroll
        for (int p = 0; p < 3; p++) {
            const uint4 x = ld16(a.x[p], b, a.nbytes);
            uint4 v;
            if constexpr (OP == 3) {
                v = make_uint4(~x.x, ~x.y, ~x.z, ~x.w);
            } else {
                const uint4 y = ld16(a.y[p], b, a.nbytes);
                if constexpr (OP == 0) v = x ^ y;
                else if constexpr (OP == 1) v = Ring<W>::add(x, y);
                else v = Ring<W>::sub(x, y);
            }
            st16(a.z[p], b, a.nbytes, v);
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
void launch_keystream(Ctx& c, int stream_id, unsigned long long nonce0, void* out, size_t nbytes) {
    StreamArg st;
    st.rk = c.rk[stream_id];
    st.nonce = nonce0;
    if (!nbytes) return;
    launch_aes(c, "keystream", (double)nbytes, (double)ceil_div(nbytes, 16), k_keystream,
               ceil_div(nbytes, 16), st, (uint8_t*)out, (unsigned long long)nbytes);
}

void op_secret_share(Ctx& c, bool arith, int w, size_t n, const void* data, int party, Sh3 s) {
    if (party < 0 || party > 2) throw std::invalid_argument("data party must be 0, 1 or 2");
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    StreamArg st = c.stream_arg(LOCAL0 + party);
    if (nb) {
        void* a = s.p[party % 3];
        void* b = s.p[(party + 1) % 3];
        void* d = s.p[(party + 2) % 3];
        ORQ_DISPATCH_W(w, {
            const double by = 4.0 * nb, bl = 2.0 * ceil_div(nb, 16);
            if (arith)
                launch_aes(c, "secret_share", by, bl, k_share<W, true>, ceil_div(nb, 16), (const uint8_t*)data, a, b, d, st, ch, nb);
            else
                launch_aes(c, "secret_share", by, bl, k_share<W, false>, ceil_div(nb, 16), (const uint8_t*)data, a, b, d, st, ch, nb);
        });
    }
    c.nonce[LOCAL0 + party] += 2 * ch;
}

void op_public_share(Ctx& c, int w, size_t n, const void* data, Sh3 s) {
    const size_t nb = n * (size_t)w;
    if (!nb) return;
    if (s.p[0] != data)
        ORQ_CUDA_CHECK(cudaMemcpyAsync(s.p[0], data, nb, cudaMemcpyDeviceToDevice, c.stream));
    ORQ_CUDA_CHECK(cudaMemsetAsync(s.p[1], 0, nb, c.stream));
    ORQ_CUDA_CHECK(cudaMemsetAsync(s.p[2], 0, nb, c.stream));
}

void op_open(Ctx& c, bool arith, int w, size_t n, CSh3 s, void* out) {
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    ProfScope ps(c, "open", 4.0 * nb);
    ORQ_DISPATCH_W(w, {
        if (arith)
            k_open<W, true><<<plain_grid(c, ceil_div(nb, 16)), 256, 0, c.stream>>>(s.p[0], s.p[1], s.p[2], out, nb);
        else
            k_open<W, false><<<plain_grid(c, ceil_div(nb, 16)), 256, 0, c.stream>>>(s.p[0], s.p[1], s.p[2], out, nb);
    });
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

void op_mult(Ctx& c, bool arith, int w, size_t n, CSh3 x, CSh3 y, Sh3 z) {
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    MultArgs a;
    for (int p = 0; p < 3; p++) {
        a.x[p] = x.p[p];
        a.y[p] = y.p[p];
        a.z[p] = z.p[p];
        a.pair[p] = c.stream_arg(PAIR0 + p);
    }
    a.nbytes = nb;
    if (nb) {
        ORQ_DISPATCH_W(w, {
            const double by = 9.0 * nb, bl = 3.0 * ceil_div(nb, 16);
            if (arith) launch_aes(c, "multiply_a", by, bl, k_mult<W, true>, ceil_div(nb, 16), a);
            else launch_aes(c, "and_b", by, bl, k_mult<W, false>, ceil_div(nb, 16), a);
        });
    }
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += ch;
}

void op_local(Ctx& c, int op, int w, size_t n, CSh3 x, CSh3 y, Sh3 z) {
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    LocalArgs a;
    for (int p = 0; p < 3; p++) {
        a.x[p] = x.p[p];
        a.y[p] = y.p[p];
        a.z[p] = z.p[p];
    }
    a.nbytes = nb;
    const unsigned g = plain_grid(c, ceil_div(nb, 16));
    ProfScope ps(c, "local", 9.0 * nb);
    ORQ_DISPATCH_W(w, {
        if (op == 0) k_local<W, 0><<<g, 256, 0, c.stream>>>(a);
        else if (op == 1) k_local<W, 1><<<g, 256, 0, c.stream>>>(a);
        else if (op == 2) k_local<W, 2><<<g, 256, 0, c.stream>>>(a);
        else throw std::invalid_argument("unknown local op");
    });
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

// not_b (replicated_3pc.h:199): every party complements both of its shares,
// so each distinct share is complemented once.
void op_not(Ctx& c, int w, size_t n, CSh3 x, Sh3 y) {
    const unsigned long long nb = (unsigned long long)n * w;
    if (!nb) return;
    LocalArgs a;
    for (int p = 0; p < 3; p++) {
        a.x[p] = x.p[p];
        a.y[p] = x.p[p];
        a.z[p] = y.p[p];
    }
    a.nbytes = nb;
    k_local<4, 3><<<plain_grid(c, ceil_div(nb, 16)), 256, 0, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

void op_b2a_bit(Ctx& c, int w, size_t n, CSh3 x, Sh3 y) {
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    B2AArgs a;
    for (int p = 0; p < 3; p++) {
        a.x[p] = x.p[p];
        a.y[p] = y.p[p];
        a.pair[p] = c.stream_arg(PAIR0 + p);
    }
    a.chunks = ch;
    a.nbytes = nb;
    if (nb) {
        ORQ_DISPATCH_W(w, { launch_aes(c, "b2a_bit", 6.0 * nb, 9.0 * ceil_div(nb, 16), k_b2a<W>, ceil_div(nb, 16), a); });
    }
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += 3 * ch;
}

void op_zero_share(Ctx& c, bool arith, int w, size_t n, Sh3 r) {
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    if (nb) {
        StreamArg p0 = c.stream_arg(PAIR0), p1 = c.stream_arg(PAIR1), p2 = c.stream_arg(PAIR2);
        ORQ_DISPATCH_W(w, {
            const double by = 3.0 * nb, bl = 3.0 * ceil_div(nb, 16);
            if (arith) launch_aes(c, "zero_share", by, bl, k_zero<W, true>, ceil_div(nb, 16), r.p[0], r.p[1], r.p[2], p0, p1, p2, nb);
            else launch_aes(c, "zero_share", by, bl, k_zero<W, false>, ceil_div(nb, 16), r.p[0], r.p[1], r.p[2], p0, p1, p2, nb);
        });
    }
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += ch;
}

void op_reshare(Ctx& c, bool arith, int w, size_t n, int group, Sh3 s) {
    if (group < 0 || group > 2) throw std::invalid_argument("reshare group must be 0..2");
    const unsigned long long nb = (unsigned long long)n * w, ch = chunks_of(nb);
    StreamArg g = c.stream_arg(G01 + group);
    if (nb) {
        ORQ_DISPATCH_W(w, {
            const double by = 6.0 * nb, bl = 2.0 * ceil_div(nb, 16);
            if (arith) launch_aes(c, "reshare", by, bl, k_reshare<W, true>, ceil_div(nb, 16), s.p[0], s.p[1], s.p[2], g, ch, nb);
            else launch_aes(c, "reshare", by, bl, k_reshare<W, false>, ceil_div(nb, 16), s.p[0], s.p[1], s.p[2], g, ch, nb);
        });
    }
    c.nonce[G01 + group] += 2 * ch;
}

}  // namespace orqcu
