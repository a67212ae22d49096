// agg.cu — the aggregation network (orq::aggregators::aggregate,
// include/core/operators/aggregation.h:167-346).
//
// Level i of the network compares row k with row k+d (d = N/2^i forward,
// N/2^(log N - i + 1) reverse) for k < N-d: group bits from key equality
// (bit_same + mask, b_shared_vector.h:164-178,493-504), optionally restricted
// to rows of the same table (sel), then every aggregation updates row k
// (forward) or row k+d (reverse) from the other. In loopback every protocol
// call of a level is element-local, so a level is ONE kernel: a thread owns a
// 16-byte unit of the level's range (16/W rows), computes the zero-sharing
// keystream of each call for that unit once (the unit is exactly one AES
// block of every call's draw), and runs the calls in the reference's order in
// registers. Outputs ping-pong between the output column and a scratch copy,
// because row k+d is read by one thread while another writes it.
#include <type_traits>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr int kMaxAggKeys = 4;
// A thread carries the group bits of its unit in four forms (boolean and
// arithmetic, with and without the table restriction) across the level's
// calls, so it needs up to 255 registers: 256 threads per CTA, one CTA per SM
// (the AES tables take 128 KiB of shared memory).
constexpr int kAggThreads = 256;
constexpr int kMaxAggSpecs = 8;

struct AggLevelArgs {
    const void* key[kMaxAggKeys][3];
    const void* sel[3];
    const void* b_src[kMaxAggSpecs][3];
    void* b_dst[kMaxAggSpecs][3];
    const void* a_src[kMaxAggSpecs][3];
    void* a_dst[kMaxAggSpecs][3];
    int b_func[kMaxAggSpecs];
    int a_func[kMaxAggSpecs];
    int nkeys, nb, na, use_sel, b2a_noncopy, b2a_copy, reverse;
    unsigned long long d, dr;  // offset and range of the level
    unsigned long long C;      // nonces per protocol call (dr*W bytes)
    unsigned long long Cp;     // nonces per packed call of a compare (ceil(dr/8W)*W bytes)
    StreamArg pair[3];         // nonces at the start of the level
};

template <typename T>
__device__ __forceinline__ T ashr_t(T v, int s) {
    using S = typename std::make_signed<T>::type;
    return (T)((S)v >> s);
}

// and_b of one element for the three parties (r_p = K[p-1] ^ K[p])
template <typename T>
__device__ __forceinline__ void and3(const T* x, const T* y, const T* k, T* z) {
    const T r0 = k[2] ^ k[0], r1 = k[0] ^ k[1], r2 = k[1] ^ k[2];
    const T z0 = r0 ^ (x[0] & y[0]) ^ (x[0] & y[1]) ^ (x[1] & y[0]);
    const T z1 = r1 ^ (x[1] & y[1]) ^ (x[1] & y[2]) ^ (x[2] & y[1]);
    const T z2 = r2 ^ (x[2] & y[2]) ^ (x[2] & y[0]) ^ (x[0] & y[2]);
    z[0] = z0;
    z[1] = z1;
    z[2] = z2;
}
// multiply_a of one element (r_p = K[p-1] - K[p])
template <typename T>
__device__ __forceinline__ void mul3(const T* x, const T* y, const T* k, T* z) {
    const T r0 = k[2] - k[0], r1 = k[0] - k[1], r2 = k[1] - k[2];
    const T z0 = r0 + x[0] * y[0] + x[0] * y[1] + x[1] * y[0];
    const T z1 = r1 + x[1] * y[1] + x[1] * y[2] + x[2] * y[1];
    const T z2 = r2 + x[2] * y[2] + x[2] * y[0] + x[0] * y[2];
    z[0] = z0;
    z[1] = z1;
    z[2] = z2;
}

// bit i of x to bit 2i (32 -> 64 bits)
__device__ __forceinline__ unsigned long long spread2(uint32_t v) {
    unsigned long long x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
// bit i of an 8-bit x to bit 4i
__device__ __forceinline__ uint32_t spread4(uint32_t x) {
    x = (x | (x << 12)) & 0x000F000Fu;
    x = (x | (x << 6)) & 0x03030303u;
    x = (x | (x << 3)) & 0x11111111u;
    return x;
}

// Packs one bit per row of this thread into the 8W-row word its rows belong
// to (bit r = row r of the word), for every lane of the word's group. The
// group is the whole warp for W = 8 (32 units x 2 rows) and 8 lanes for
// W = 4 (8 units x 4 rows); the grid-stride loop keeps warps unit-aligned.
template <typename T, int E, int W>
__device__ __forceinline__ T pack_word(const bool (&bit)[E]) {
    const int lane = threadIdx.x & 31;
    if constexpr (W == 8) {
        const uint32_t b0 = __ballot_sync(0xffffffffu, bit[0]);
        const uint32_t b1 = __ballot_sync(0xffffffffu, bit[1]);
        return (T)(spread2(b0) | (spread2(b1) << 1));
    } else {
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < E; k++) {
            const uint32_t b = __ballot_sync(0xffffffffu, bit[k]);
            w |= spread4((b >> (lane & ~7)) & 0xffu) << k;
        }
        return (T)w;
    }
}

// BSharedVector::_compare (circuits.h:231-295) of the thread's rows, this =
// X, other = Y: L bit_same ANDs, gt & this, and the packed sign fix-up (its
// AND runs on ceil(dr/8W) words, Cp nonces). Leaves gt (LSB) in Gt.
template <typename T, int E, int W, int L, typename NextCall, typename Args>
__device__ __forceinline__ void compare_rows(const T (&X)[E][3], const T (&Y)[E][3],
                                             const bool (&ok)[E], T (&K)[E][3], NextCall& next_call,
                                             const Args& a, unsigned long long u,
                                             unsigned long long& off, const AesSmem& S,
                                             T (&Gt)[E][3]) {
    constexpr int B = 8 * W;
    T Sm[E][3];
#pragma unroll
    for (int k = 0; k < E; k++)
#pragma unroll
        for (int p = 0; p < 3; p++) Sm[k][p] = ~(X[k][p] ^ Y[k][p]);
#pragma unroll 1
    for (int lev = 0; lev < L; lev++) {
        next_call();
#pragma unroll
        for (int k = 0; k < E; k++) {
            T Tm[3];
#pragma unroll
            for (int p = 0; p < 3; p++) Tm[p] = ashr_t(Sm[k][p], 1 << lev);
            and3(Sm[k], Tm, K[k], Sm[k]);
        }
    }
    next_call();
#pragma unroll
    for (int k = 0; k < E; k++) {
        T Gi[3];
#pragma unroll
        for (int p = 0; p < 3; p++) Gi[p] = ashr_t(Sm[k][p], 1) ^ Sm[k][p];
        and3(Gi, X[k], K[k], Gt[k]);
    }
    // packed words of the sign bits and gt parities
    T s1[3], s2[3], r[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
        bool b1[E], b2[E], br[E];
#pragma unroll
        for (int k = 0; k < E; k++) {
            b1[k] = ok[k] && ((X[k][p] >> (B - 1)) & 1);
            b2[k] = ok[k] && ((Y[k][p] >> (B - 1)) & 1);
            br[k] = ok[k] && (__popcll((unsigned long long)Gt[k][p]) & 1);
        }
        s1[p] = pack_word<T, E, W>(b1);
        s2[p] = pack_word<T, E, W>(b2);
        r[p] = pack_word<T, E, W>(br);
    }
    // the packed AND: word c of the draw sits in keystream block c*W/16
    const unsigned long long c = u * E / B;
    T Kp[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        StreamArg st = a.pair[q];
        st.nonce += off;
        const uint4 b = keystream_block(S, st, c * W / 16);
        if constexpr (W == 4) {
            const uint32_t w4[4] = {b.x, b.y, b.z, b.w};
            Kp[q] = w4[c & 3];
        } else {
            Kp[q] = (c & 1) ? ((T)b.z | ((T)b.w << 32)) : ((T)b.x | ((T)b.y << 32));
        }
    }
    off += a.Cp;
    T ns2[3], nr[3], Z[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
        nr[p] = ~(r[p] ^ s2[p]);
        ns2[p] = ~(s2[p] ^ s1[p]);
    }
    and3(ns2, nr, Kp, Z);
#pragma unroll
    for (int p = 0; p < 3; p++) s1[p] ^= ~Z[p];
    const int rowbase = (int)((u * E) % B);
#pragma unroll
    for (int k = 0; k < E; k++)
#pragma unroll
        for (int p = 0; p < 3; p++) Gt[k][p] = (s1[p] >> (rowbase + k)) & 1;
}

// MINMAX: whether the level has a min or max aggregation; without one the
// compare circuit is compiled out (it holds most of the registers)
template <int W, bool MINMAX>
__global__ void __launch_bounds__(kAggThreads, 1) k_agg_level(AggLevelArgs a) {
    using T = typename std::conditional<W == 4, uint32_t, unsigned long long>::type;
    constexpr int E = 16 / W;               // rows per unit
    constexpr int L = (W == 4) ? 5 : 6;     // bit_same rounds
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long units = ceil_div(a.dr * W, 16);
    const int lane = threadIdx.x & 31;
    // warp-uniform loop: min/max use warp ballots over all 32 lanes
    for (unsigned long long wb = gtid() - lane; wb < units; wb += gstride()) {
        const unsigned long long u = wb + lane;
        unsigned long long off = 0;  // nonces consumed by the level's calls so far
        T K[E][3];
        // keystream of the next protocol call for this unit, split per row
        auto next_call = [&]() {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                StreamArg st = a.pair[q];
                st.nonce += off;
                const uint4 b = keystream_block(S, st, u);
                if constexpr (W == 4) {
                    K[0][q] = b.x;
                    K[1][q] = b.y;
                    K[2][q] = b.z;
                    K[3][q] = b.w;
                } else {
                    K[0][q] = (T)b.x | ((T)b.y << 32);
                    K[1][q] = (T)b.z | ((T)b.w << 32);
                }
            }
            off += a.C;
        };
        unsigned long long lo[E], hi[E];
        bool ok[E];
#pragma unroll
        for (int k = 0; k < E; k++) {
            lo[k] = u * E + k;
            hi[k] = lo[k] + a.d;
            ok[k] = u < units && lo[k] < a.dr;
        }
        auto ld = [&](const void* p, unsigned long long i, bool v) -> T {
            return v ? reinterpret_cast<const T*>(p)[i] : (T)0;
        };
        // ---- group bits
        T G[E][3], JG[E][3];
        if (a.nkeys == 0) {
#pragma unroll
            for (int k = 0; k < E; k++) {
                G[k][0] = 1;
                G[k][1] = 0;
                G[k][2] = 0;
            }
        }
#pragma unroll 1
        for (int j = 0; j < a.nkeys; j++) {
            T Sm[E][3];
#pragma unroll
            for (int k = 0; k < E; k++)
#pragma unroll
                for (int p = 0; p < 3; p++)
                    Sm[k][p] = ~(ld(a.key[j][p], lo[k], ok[k]) ^ ld(a.key[j][p], hi[k], ok[k]));
#pragma unroll 1
            for (int lev = 0; lev < L; lev++) {
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T Tm[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) Tm[p] = ashr_t(Sm[k][p], 1 << lev);
                    and3(Sm[k], Tm, K[k], Sm[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < E; k++)
#pragma unroll
                for (int p = 0; p < 3; p++) Sm[k][p] &= (T)1;
            if (j == 0) {
#pragma unroll
                for (int k = 0; k < E; k++)
#pragma unroll
                    for (int p = 0; p < 3; p++) G[k][p] = Sm[k][p];
            } else {
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) and3(G[k], Sm[k], K[k], G[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < E; k++)
#pragma unroll
            for (int p = 0; p < 3; p++) JG[k][p] = G[k][p];
        if (a.use_sel) {
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                T s[3];
#pragma unroll
                for (int p = 0; p < 3; p++)
                    s[p] = ~(ld(a.sel[p], hi[k], ok[k]) ^ ld(a.sel[p], lo[k], ok[k]));
                and3(G[k], s, K[k], G[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < E; k++)
#pragma unroll
            for (int p = 0; p < 3; p++) G[k][p] &= (T)1;
        // ---- boolean aggregations: func(g, a, b) updates a; reverse swaps roles
#pragma unroll 1
        for (int s = 0; s < a.nb; s++) {
            const int f = a.b_func[s];
            T X[E][3], Y[E][3], R[E][3], Ex[E][3];
#pragma unroll
            for (int k = 0; k < E; k++)
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const T vlo = ld(a.b_src[s][p], lo[k], ok[k]), vhi = ld(a.b_src[s][p], hi[k], ok[k]);
                    X[k][p] = a.reverse ? vhi : vlo;  // the updated side
                    Y[k][p] = a.reverse ? vlo : vhi;
                    const T g = (f == AGG_COPY) ? JG[k][p] : G[k][p];
                    Ex[k][p] = (g & 1) ? ~(T)0 : (T)0;  // extend_lsb
                }
            if (f == AGG_COPY) {  // a ^ (ext(g) & (b ^ a))
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T D[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) D[p] = Y[k][p] ^ X[k][p];
                    and3(Ex[k], D, K[k], R[k]);
#pragma unroll
                    for (int p = 0; p < 3; p++) R[k][p] ^= X[k][p];
                }
            } else if (f == AGG_VALID) {  // agg = a & b ; a ^ (ext(g) & (agg ^ a))
                next_call();
                T Ag[E][3];
#pragma unroll
                for (int k = 0; k < E; k++) and3(X[k], Y[k], K[k], Ag[k]);
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T D[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) D[p] = Ag[k][p] ^ X[k][p];
                    and3(Ex[k], D, K[k], R[k]);
#pragma unroll
                    for (int p = 0; p < 3; p++) R[k][p] ^= X[k][p];
                }
            } else if (MINMAX && (f == AGG_MIN || f == AGG_MAX)) {
                // bg = b > a (_compare with this = b), ! for min; then
                // a = multiplex(g, a, multiplex(bg, a, b))
                T Gt[E][3];
                compare_rows<T, E, W, L>(Y, X, ok, K, next_call, a, u, off, S, Gt);
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T Eb[3], D[3], Tm[3];
                    if (f == AGG_MIN)
#pragma unroll
                        for (int p = 0; p < 3; p++) Gt[k][p] = (Gt[k][p] & 1) ^ 1;
#pragma unroll
                    for (int p = 0; p < 3; p++) Eb[p] = (Gt[k][p] & 1) ? ~(T)0 : (T)0;
                    Gt[k][0] = Eb[0];
                    Gt[k][1] = Eb[1];
                    Gt[k][2] = Eb[2];
                    (void)D;
                    (void)Tm;
                }
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T D[3], Tm[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) D[p] = Y[k][p] ^ X[k][p];
                    and3(Gt[k], D, K[k], Tm);
#pragma unroll
                    for (int p = 0; p < 3; p++) R[k][p] = X[k][p] ^ Tm[p];  // inner multiplex
                }
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T D[3], Tm[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) D[p] = R[k][p] ^ X[k][p];
                    and3(Ex[k], D, K[k], Tm);
#pragma unroll
                    for (int p = 0; p < 3; p++) R[k][p] = X[k][p] ^ Tm[p];
                }
            } else {  // AGG_BIT_OR: x = ext(g) & b ; ~(~a & ~x)
                next_call();
                T Xm[E][3];
#pragma unroll
                for (int k = 0; k < E; k++) and3(Ex[k], Y[k], K[k], Xm[k]);
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T na_[3], nx[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) {
                        na_[p] = ~X[k][p];
                        nx[p] = ~Xm[k][p];
                    }
                    and3(na_, nx, K[k], R[k]);
#pragma unroll
                    for (int p = 0; p < 3; p++) R[k][p] = ~R[k][p];
                }
            }
#pragma unroll
            for (int k = 0; k < E; k++)
                if (ok[k])
#pragma unroll
                    for (int p = 0; p < 3; p++)
                        reinterpret_cast<T*>(a.b_dst[s][p])[a.reverse ? hi[k] : lo[k]] = R[k][p];
        }
        if (a.na == 0) continue;  // uniform across the grid
        // ---- group bits as arithmetic shares (b2a_bit, replicated_3pc.h:220-251)
        T GA[E][3], JGA[E][3];
#pragma unroll
        for (int k = 0; k < E; k++) {
            GA[k][0] = JGA[k][0] = a.nkeys == 0 ? (T)1 : (T)0;
            GA[k][1] = JGA[k][1] = 0;
            GA[k][2] = JGA[k][2] = 0;
        }
        auto b2a = [&](T (*X)[3], T (*Y)[3]) {
            T Za[E][3], Zb[E][3];
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                Za[k][0] = K[k][2] - K[k][0];
                Za[k][1] = K[k][0] - K[k][1];
                Za[k][2] = K[k][1] - K[k][2];
            }
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                Zb[k][0] = K[k][2] - K[k][0];
                Zb[k][1] = K[k][0] - K[k][1];
                Zb[k][2] = K[k][1] - K[k][2];
            }
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                T D[3];
                D[0] = Za[k][0] + ((X[k][0] ^ X[k][1]) & 1) - Zb[k][0];
                D[1] = Za[k][1] - (Zb[k][1] + (X[k][2] & 1));
                D[2] = Za[k][2] - Zb[k][2];
                mul3(D, D, K[k], Y[k]);
            }
        };
        if (a.nkeys > 0) {
            if (a.b2a_noncopy) b2a(G, GA);
            if (a.b2a_copy) b2a(JG, JGA);
        }
        // ---- arithmetic aggregations: sum/count a + g*b, copy a + g*(b - a)
#pragma unroll 1
        for (int s = 0; s < a.na; s++) {
            const int f = a.a_func[s];
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                T X[3], Y[3], Z[3];
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const T vlo = ld(a.a_src[s][p], lo[k], ok[k]), vhi = ld(a.a_src[s][p], hi[k], ok[k]);
                    X[p] = a.reverse ? vhi : vlo;
                    Y[p] = a.reverse ? vlo : vhi;
                }
                if (f == AGG_COPY) {
                    T D[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
                    mul3(JGA[k], D, K[k], Z);
                } else {
                    mul3(GA[k], Y, K[k], Z);
                }
                if (ok[k])
#pragma unroll
                    for (int p = 0; p < 3; p++)
                        reinterpret_cast<T*>(a.a_dst[s][p])[a.reverse ? hi[k] : lo[k]] = X[p] + Z[p];
            }
        }
    }
}

template <int W>
__global__ void k_fill_one(void* s0, void* s1, void* s2, unsigned long long n) {
    using T = typename std::conditional<W == 4, uint32_t, unsigned long long>::type;
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        reinterpret_cast<T*>(s0)[i] = 1;
        reinterpret_cast<T*>(s1)[i] = 0;
        reinterpret_cast<T*>(s2)[i] = 0;
    }
}

void copy3(Ctx& c, void* const dst[3], const void* const src[3], size_t off, size_t n, int w) {
    if (!n) return;
    for (int p = 0; p < 3; p++) {
        if (dst[p] == src[p]) continue;
        ORQ_CUDA_CHECK(cudaMemcpyAsync((char*)dst[p] + off * w, (const char*)src[p] + off * w, n * w,
                                       cudaMemcpyDeviceToDevice, c.stream));
    }
}

}  // namespace

void op_aggregate(Ctx& c, int w, size_t n, int nkeys, const void* const* keys, int nb,
                  const AggSpec* bs, int na, const AggSpec* as, bool reverse,
                  const void* const* sel) {
    if (w != 4 && w != 8) throw std::invalid_argument("aggregate supports 4 and 8-byte shares");
    if (n == 0 || (n & (n - 1))) throw std::invalid_argument("aggregate needs a power-of-two size");
    if (nkeys < 0 || nkeys > kMaxAggKeys) throw std::invalid_argument("aggregate supports at most 4 key columns");
    if (nb < 0 || na < 0 || nb > kMaxAggSpecs || na > kMaxAggSpecs)
        throw std::invalid_argument("aggregate supports at most 8 boolean and 8 arithmetic specs");
    if (nkeys == 0 && nb == 0 && na == 0) throw std::invalid_argument("Empty aggregation!");
    bool a_copy = false, a_noncopy = false, b_noncopy = false;
    for (int s = 0; s < na; s++) {
        const int f = as[s].func;
        if (f != AGG_SUM && f != AGG_COUNT && f != AGG_COPY)
            throw std::invalid_argument("arithmetic aggregations are sum, count and copy");
        (f == AGG_COPY ? a_copy : a_noncopy) = true;
    }
    for (int s = 0; s < nb; s++) {
        const int f = bs[s].func;
        if (f != AGG_COPY && f != AGG_VALID && f != AGG_BIT_OR && f != AGG_MIN && f != AGG_MAX)
            throw std::invalid_argument("boolean aggregations are copy, valid, bit_or, min and max");
        if (f != AGG_COPY) b_noncopy = true;
    }
    // ---- preprocessing: out = in (count: ones, or b2a_bit(sel) inside joins)
    for (int s = 0; s < na; s++) {
        if (as[s].func == AGG_COUNT) {
            if (sel) {
                op_b2a_bit(c, w, n, CSh3{{sel[0], sel[1], sel[2]}}, Sh3{{as[s].out[0], as[s].out[1], as[s].out[2]}});
            } else {
                ProfScope ps(c, "agg_fill", 3.0 * w * n);
                if (w == 4) k_fill_one<4><<<plain_grid(c, n), 256, 0, c.stream>>>(as[s].out[0], as[s].out[1], as[s].out[2], n);
                else k_fill_one<8><<<plain_grid(c, n), 256, 0, c.stream>>>(as[s].out[0], as[s].out[1], as[s].out[2], n);
                ORQ_CUDA_CHECK(cudaGetLastError());
                c.kernels_launched++;
            }
        } else {
            copy3(c, as[s].out, as[s].in, 0, n, w);
        }
    }
    for (int s = 0; s < nb; s++) copy3(c, bs[s].out, bs[s].in, 0, n, w);
    int log_size = 0;
    while (((size_t)2 << log_size) <= n) log_size++;
    if (log_size == 0) return;
    // ---- ping-pong buffers per output column
    const size_t col = n * (size_t)w;
    Scratch scratch(c, (size_t)(na + nb) * 3 * col + 16);
    void* cur_b[kMaxAggSpecs][3];
    void* alt_b[kMaxAggSpecs][3];
    void* cur_a[kMaxAggSpecs][3];
    void* alt_a[kMaxAggSpecs][3];
    char* sp = scratch.as<char>();
    for (int s = 0; s < nb; s++)
        for (int p = 0; p < 3; p++) {
            cur_b[s][p] = bs[s].out[p];
            alt_b[s][p] = sp;
            sp += col;
        }
    for (int s = 0; s < na; s++)
        for (int p = 0; p < 3; p++) {
            cur_a[s][p] = as[s].out[p];
            alt_a[s][p] = sp;
            sp += col;
        }
    const int L = (w == 4) ? 5 : 6;
    const bool use_sel = sel && (a_noncopy || b_noncopy);
    int calls = 0, packed = 0;  // full-size protocol calls and packed compare calls per level
    if (nkeys > 0) calls += nkeys * L + (nkeys - 1);
    if (use_sel) calls += 1;
    for (int s = 0; s < nb; s++) {
        const int f = bs[s].func;
        if (f == AGG_MIN || f == AGG_MAX) {
            calls += L + 1 + 2;
            packed += 1;
        } else {
            calls += f == AGG_COPY ? 1 : 2;
        }
    }
    if (nkeys > 0 && na > 0) calls += (a_noncopy ? 3 : 0) + (a_copy ? 3 : 0);
    calls += na;
    for (int i = 1; i <= log_size; i++) {
        const size_t d = reverse ? n >> (log_size - i + 1) : n >> i;
        const size_t dr = n - d;
        AggLevelArgs a{};
        for (int j = 0; j < nkeys; j++)
            for (int p = 0; p < 3; p++) a.key[j][p] = keys[3 * j + p];
        if (sel)
            for (int p = 0; p < 3; p++) a.sel[p] = sel[p];
        for (int s = 0; s < nb; s++) {
            a.b_func[s] = bs[s].func;
            for (int p = 0; p < 3; p++) {
                a.b_src[s][p] = cur_b[s][p];
                a.b_dst[s][p] = alt_b[s][p];
            }
        }
        for (int s = 0; s < na; s++) {
            a.a_func[s] = as[s].func;
            for (int p = 0; p < 3; p++) {
                a.a_src[s][p] = cur_a[s][p];
                a.a_dst[s][p] = alt_a[s][p];
            }
        }
        a.nkeys = nkeys;
        a.nb = nb;
        a.na = na;
        a.use_sel = use_sel;
        a.b2a_noncopy = a_noncopy;
        a.b2a_copy = a_copy;
        a.reverse = reverse;
        a.d = d;
        a.dr = dr;
        a.C = chunks_of((unsigned long long)dr * w);
        a.Cp = chunks_of(ceil_div(dr, 8ull * w) * w);
        for (int q = 0; q < 3; q++) a.pair[q] = c.stream_arg(PAIR0 + q);
        const unsigned long long units = ceil_div((unsigned long long)dr * w, 16);
        const double bytes = (double)dr * w * 3.0 * (2.0 * nkeys + (sel ? 2.0 : 0.0) + 3.0 * (na + nb));
        {
            bool minmax = false;
            for (int s2 = 0; s2 < nb; s2++) minmax = minmax || bs[s2].func == AGG_MIN || bs[s2].func == AGG_MAX;
            auto kern = w == 4 ? (minmax ? k_agg_level<4, true> : k_agg_level<4, false>)
                               : (minmax ? k_agg_level<8, true> : k_agg_level<8, false>);
            prep_aes_kernel(kern);
            const unsigned grid = (unsigned)std::min<unsigned long long>(ceil_div(units, kAggThreads), (unsigned long long)c.num_sms);
            ProfScope ps(c, "agg_level", bytes, 3.0 * calls * units + 3.0 * packed * units);
            kern<<<grid, kAggThreads, kAesSmemBytes, c.stream>>>(a);
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched++;
        }
        for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (unsigned long long)calls * a.C + packed * a.Cp;
        // rows the level leaves alone: [dr, n) forward, [0, d) reverse
        const size_t keep = reverse ? 0 : dr;
        for (int s = 0; s < nb; s++) {
            copy3(c, alt_b[s], cur_b[s], keep, d, w);
            for (int p = 0; p < 3; p++) std::swap(cur_b[s][p], alt_b[s][p]);
        }
        for (int s = 0; s < na; s++) {
            copy3(c, alt_a[s], cur_a[s], keep, d, w);
            for (int p = 0; p < 3; p++) std::swap(cur_a[s][p], alt_a[s][p]);
        }
    }
    for (int s = 0; s < nb; s++) copy3(c, bs[s].out, cur_b[s], 0, n, w);
    for (int s = 0; s < na; s++) copy3(c, as[s].out, cur_a[s], 0, n, w);
}

}  // namespace orqcu
