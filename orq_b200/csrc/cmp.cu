// cmp.cu — the compare circuit and the bitonic sorting network.
//
// BSharedVector::_compare (include/core/operators/circuits.h:231-295) with
// bit_same (containers/b_shared_vector.h:164-178): log2(8W) AND rounds of a
// prefix-AND over ~(x^y), one AND for ((eq>>1)^eq) & x, a local parity, and a
// sign fix-up on bits packed 8W per word with one more AND (the OR of
// operator|=, b_shared_vector.h:450-455). bitonic_sort
// (operators/sorting.h:266-353) runs one compare per pair and stage followed
// by two multiplexes (operators/common.h:20-28).
//
// In loopback every AND round of a pair is local to the thread that holds the
// pair, so a whole stage is one kernel: each warp first computes the
// zero-sharing keystream of all its rounds into shared memory (every AES block
// once), then each thread runs the circuit in registers. The packed fix-up
// (a bit transpose of 8W consecutive pairs) is a warp ballot.
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "launch.cuh"

namespace orqcu {

namespace {

// Threads (= pairs) per CTA iteration. The AES tables take 128 KiB of shared
// memory, so one CTA runs per SM; the per-warp keystream buffers take the rest
// (3 KiB per warp for int32 stages, 6.75 KiB for int64; 512 threads keep the
// int32 tile within 128 registers a thread).
// 16-byte shares (padded int64 keys) only run compares (MODE 1) and equality:
// 256 threads keep 8 keystream calls of 128 words per warp within shared memory.
template <int W>
constexpr int cmp_threads() { return W == 4 ? 512 : (W == 8 ? 448 : 256); }

// bit_same rounds: log2 of the share's bit width
template <int W>
constexpr int cmp_levels() { return W == 4 ? 5 : (W == 8 ? 6 : 7); }

template <typename T>
struct CmpArgs {
    T* key[3];          // bitonic: the sorted column (in place)
    const T* x[3];      // compare: this
    const T* y[3];      // compare: other
    T* eq[3];
    T* gt[3];
    StreamArg pair[3];  // nonces at the start of the stage / compare
    unsigned long long C, Cp;  // nonces per full-size and per packed AND call
    unsigned long long m;      // pairs
    int hs;                    // bitonic half-box size h = 2^hs
    int first;                 // bitonic stage j == 0 (reversed partner)
    int desc;
};

template <typename T>
__device__ __forceinline__ T ashr(T v, int s) {
    if constexpr (sizeof(T) == 16) return (T)((__int128)v >> s);
    else return (T)((typename std::make_signed<T>::type)v >> s);
}

// parity of the bits of v
template <typename T>
__device__ __forceinline__ int parity(T v) {
    if constexpr (sizeof(T) == 16) return (__popcll((unsigned long long)v) ^ __popcll((unsigned long long)(v >> 64))) & 1;
    else return __popcll((unsigned long long)v) & 1;
}

// binary and_b of one element for all three parties: z_p = r_p ^ x_p&y_p ^
// x_p&y_{p+1} ^ x_{p+1}&y_p, r_p = K[p-1] ^ K[p]
template <typename T>
__device__ __forceinline__ void and3(const T x[3], const T y[3], const T k[3], T z[3]) {
    const T r[3] = {(T)(k[2] ^ k[0]), (T)(k[0] ^ k[1]), (T)(k[1] ^ k[2])};
#pragma unroll
    for (int p = 0; p < 3; p++) {
        const int q = (p + 1) % 3;
        z[p] = r[p] ^ (x[p] & y[p]) ^ (x[p] & y[q]) ^ (x[q] & y[p]);
    }
}

// bit_same (b_shared_vector.h:164-178) of one pair for all parties: the
// prefix-AND of ~(a ^ b) from the MSB down; AND round lev uses keystream call
// lev (kword(call, stream) is this thread's word of that call).
template <typename T, typename KW>
__device__ __forceinline__ void bit_same3(const T (&A)[3], const T (&Bv)[3], const KW& kword, T (&Sm)[3]) {
    constexpr int L = cmp_levels<sizeof(T)>();
#pragma unroll
    for (int j = 0; j < 3; j++) Sm[j] = ~(A[j] ^ Bv[j]);
#pragma unroll
    for (int lev = 0; lev < L; lev++) {
        T Tm[3], K[3], Z[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Tm[j] = ashr(Sm[j], 1 << lev);
            K[j] = kword(lev, j);
        }
        and3(Sm, Tm, K, Z);
#pragma unroll
        for (int j = 0; j < 3; j++) Sm[j] = Z[j];
    }
}

// The rest of _compare (circuits.h:249-292) once bit_same is in Sm: gt =
// parity(((eq >> 1) ^ eq) & this) on keystream call L, then the signed fix-up
// on words of 8W packed pairs with one packed AND whose keystream block is kp
// (this warp's [stream][word]). A warp holds pairs [p0w, p0w + 32); for 8-byte
// shares two warps make one packed word, exchanged through `ballots` (every
// thread of the CTA must call this). Returns the masked gt bit of the pair.
template <typename T, typename KW>
__device__ __forceinline__ void gt_bits3(const T (&A)[3], const T (&Bv)[3], const T (&Sm)[3], bool valid,
                                         unsigned long long p, unsigned long long p0w, int warp,
                                         const KW& kword, const uint32_t (*kp)[4],
                                         uint32_t (*ballots)[3][3], T (&gt)[3]) {
    constexpr int W = sizeof(T);
    constexpr int B = 8 * W;
    constexpr int L = cmp_levels<W>();
    T G[3];
    {
        T Gi[3], K[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Gi[j] = ashr(Sm[j], 1) ^ Sm[j];
            K[j] = kword(L, j);
        }
        and3(Gi, A, K, G);
    }
    uint32_t b1[3], b2[3], br[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        b1[j] = __ballot_sync(0xffffffffu, valid && ((A[j] >> (B - 1)) & 1));
        b2[j] = __ballot_sync(0xffffffffu, valid && ((Bv[j] >> (B - 1)) & 1));
        br[j] = __ballot_sync(0xffffffffu, valid && parity(G[j]));
    }
    T s1[3], s2[3], r[3];
    if constexpr (W == 4) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            s1[j] = b1[j];
            s2[j] = b2[j];
            r[j] = br[j];
        }
    } else {
        // W / 4 warps per packed word of 8W pairs
        constexpr int WPW = W / 4;
        const int lane = threadIdx.x & 31;
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                ballots[warp][0][j] = b1[j];
                ballots[warp][1][j] = b2[j];
                ballots[warp][2][j] = br[j];
            }
        __syncthreads();
        const int w0 = warp & ~(WPW - 1);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            s1[j] = s2[j] = r[j] = 0;
#pragma unroll
            for (int k = 0; k < WPW; k++) {
                s1[j] |= (T)ballots[w0 + k][0][j] << (32 * k);
                s2[j] |= (T)ballots[w0 + k][1][j] << (32 * k);
                r[j] |= (T)ballots[w0 + k][2][j] << (32 * k);
            }
        }
    }
    {
        // r ^= s2 ; s2 ^= s1 ; s2 = ~(~s2 & ~r) ; s1 ^= s2
        T ns2[3], nr[3], K[3], Z[3];
        const unsigned long long c = p0w / B;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const T rr = r[j] ^ s2[j];
            const T ss = s2[j] ^ s1[j];
            ns2[j] = ~ss;
            nr[j] = ~rr;
            if constexpr (W == 4) K[j] = (T)kp[j][c & 3];
            else if constexpr (W == 8) K[j] = (T)kp[j][2 * (c & 1)] | ((T)kp[j][2 * (c & 1) + 1] << 32);
            else K[j] = (T)kp[j][0] | ((T)kp[j][1] << 32) | ((T)kp[j][2] << 64) | ((T)kp[j][3] << 96);
        }
        and3(ns2, nr, K, Z);
#pragma unroll
        for (int j = 0; j < 3; j++) s1[j] ^= ~Z[j];
    }
    const int bitpos = (int)(p % B);
#pragma unroll
    for (int j = 0; j < 3; j++) gt[j] = (s1[j] >> bitpos) & 1;
}

// One CTA tile of a bitonic stage (MODE 0) or of a compare (MODE 1): the
// pairs [base, base + blockDim.x).
template <typename T, int MODE>
__device__ __forceinline__ void cmp_tile(const CmpArgs<T>& a, const StreamArg (&pairs)[3],
                                         const unsigned long long (&nonce)[3], unsigned long long base,
                                         const AesSmem& S, uint32_t* ksw,
                                         uint32_t (*ksp)[3][4], uint32_t (*ballots)[3][3]) {
    constexpr int W = sizeof(T);
    constexpr int B = 8 * W;               // pairs per packed word
    constexpr int L = cmp_levels<W>();     // bit_same rounds
    constexpr int NFULL = MODE == 0 ? L + 3 : (MODE == 1 ? L + 1 : L);
    constexpr int WORDS = 32 * W / 4;      // keystream words per call and stream per warp
    constexpr int NB = 32 * W / 16;        // AES blocks per call and stream per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* myks = ksw + (size_t)warp * NFULL * 3 * WORDS;
    {
        const unsigned long long p0w = base + warp * 32;  // this warp's first pair
        const unsigned long long p = p0w + lane;
        const bool valid = p < a.m;
        // ---- operands, loaded first so their latency hides under the AES work
        unsigned long long xi = p, yi = p;
        if (MODE == 0) {
            const unsigned long long h = 1ull << a.hs, cb = p >> a.hs, k = p & (h - 1);
            xi = (cb << (a.hs + 1)) + k;
            yi = a.first ? (cb << (a.hs + 1)) + 2 * h - 1 - k : (cb << (a.hs + 1)) + h + k;
        }
        T X[3] = {0, 0, 0}, Y[3] = {0, 0, 0};
        if (valid) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
                if (MODE == 0) {
                    X[j] = a.key[j][xi];
                    Y[j] = a.key[j][yi];
                } else {
                    X[j] = a.x[j][p];
                    Y[j] = a.y[j][p];
                }
            }
        }
        // ---- keystream of every round, each AES block once per warp
        for (int idx = lane; idx < NFULL * 3 * NB; idx += 32) {
            const int call = idx / (3 * NB), q = (idx / NB) % 3, b = idx % NB;
            unsigned long long off = (unsigned long long)call * a.C;
            if (call > L) off = (unsigned long long)(L + 1) * a.C + a.Cp + (unsigned long long)(call - L - 1) * a.C;
            const uint4 ks = keystream_block_n(S, pairs[q].rk, nonce[q] + off, p0w * W / 16 + b);
            uint32_t* o = myks + (call * 3 + q) * WORDS + b * 4;
            o[0] = ks.x;
            o[1] = ks.y;
            o[2] = ks.z;
            o[3] = ks.w;
        }
        if (MODE != 2 && lane < 3) {
            // the packed AND: word c = pair / B covers pairs [cB, cB+B)
            const unsigned long long c = p0w / B;
            const unsigned long long nl = lane == 0 ? nonce[0] : (lane == 1 ? nonce[1] : nonce[2]);
            const uint4 ks = keystream_block_n(S, pairs[lane].rk, nl + (unsigned long long)(L + 1) * a.C,
                                               c * W / 16);
            ksp[warp][lane][0] = ks.x;
            ksp[warp][lane][1] = ks.y;
            ksp[warp][lane][2] = ks.z;
            ksp[warp][lane][3] = ks.w;
        }
        __syncwarp();
        // compare_rows: ASC compares x > y, DESC compares y > x
        T A[3], Bv[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            A[j] = (MODE == 0 && a.desc) ? Y[j] : X[j];
            Bv[j] = (MODE == 0 && a.desc) ? X[j] : Y[j];
        }
        auto kword = [&](int call, int q) -> T {
            const uint32_t* w = myks + (call * 3 + q) * WORDS;
            if constexpr (W == 4) return (T)w[lane];
            else if constexpr (W == 8) return (T)w[2 * lane] | ((T)w[2 * lane + 1] << 32);
            else
                return (T)w[4 * lane] | ((T)w[4 * lane + 1] << 32) | ((T)w[4 * lane + 2] << 64) |
                       ((T)w[4 * lane + 3] << 96);
        };
        T Sm[3];
        bit_same3(A, Bv, kword, Sm);
        if constexpr (MODE == 2) {
            // operator== : bit_same then mask(1)
            if (valid)
#pragma unroll
                for (int j = 0; j < 3; j++) a.eq[j][p] = Sm[j] & 1;
            __syncthreads();  // keystream buffers are rewritten by the next tile
            return;
        }
        T gt[3], eq[3];
        gt_bits3(A, Bv, Sm, valid, p, p0w, warp, kword, ksp[warp], ballots, gt);
#pragma unroll
        for (int j = 0; j < 3; j++) eq[j] = Sm[j] & 1;
        if (MODE == 1) {
            if (valid)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    a.eq[j][p] = eq[j];
                    a.gt[j][p] = gt[j];
                }
        } else {
            // swap: x' = x ^ (ext(b) & (y ^ x)), y' = y ^ (ext(b) & (x ^ y))
            T E[3], D[3], K[3], Z[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                E[j] = gt[j] ? ~(T)0 : (T)0;
                D[j] = X[j] ^ Y[j];
                K[j] = kword(L + 1, j);
            }
            and3(E, D, K, Z);
            T Xn[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                Xn[j] = X[j] ^ Z[j];
                K[j] = kword(L + 2, j);
            }
            and3(E, D, K, Z);
            if (valid)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    a.key[j][xi] = Xn[j];
                    a.key[j][yi] = Y[j] ^ Z[j];
                }
        }
        __syncthreads();  // keystream buffers are rewritten by the next tile
    }
}

template <typename T, int MODE>  // MODE 0: bitonic stage, MODE 1: compare
__global__ void __launch_bounds__(cmp_threads<sizeof(T)>(), 1) k_cmp(CmpArgs<T> a) {
    constexpr int kCmpThreads = cmp_threads<sizeof(T)>();
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t ksp[kCmpThreads / 32][3][4];      // packed call block per warp
    __shared__ uint32_t ballots[kCmpThreads / 32][3][3];  // [warp][s1,s2,r][share]
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long nonce[3] = {a.pair[0].nonce, a.pair[1].nonce, a.pair[2].nonce};
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < a.m;
         base += (unsigned long long)gridDim.x * blockDim.x)
        cmp_tile<T, MODE>(a, a.pair, nonce, base, S, sm + kAesSmemBytes / 4, ksp, ballots);
}

// ---- compare_rows and swap over several columns -------------------------------
// compare_rows (operators/sorting.h:80-108) runs _compare on every key column,
// in order, and folds key k >= 1 in with two ANDs: gt ^= new_gt & eq, then
// eq &= new_eq. The calls of key k follow each other on the PAIR streams:
// L + 1 full calls and one packed call for the compare, then (k >= 1) the two
// fold calls. A key's keystream is staged per warp exactly as in a compare.
constexpr int kMaxRowKeys = 8;
constexpr int kMaxRowCols = 40;

template <typename T>
struct RowsCmpArgs {
    const T* x[kMaxRowKeys][3];  // bitonic: the key columns (x and y the same)
    const T* y[kMaxRowKeys][3];
    int desc[kMaxRowKeys];
    int nkeys;
    T* gt[3];            // the masked comparison bit per pair
    StreamArg pair[3];   // nonces at the first call
    unsigned long long C, Cp, m;
    int hs;              // bitonic half-box size 2^hs, or -1: pair p is (x[p], y[p])
    int first;
};

// pair p's two rows in a bitonic stage: the box of 2h rows that holds it, row
// k of the first half against row k (or, at j == 0, row h-1-k) of the second
__device__ __forceinline__ void bitonic_rows(unsigned long long p, int hs, int first,
                                             unsigned long long& xi, unsigned long long& yi) {
    const unsigned long long h = 1ull << hs, cb = p >> hs, k = p & (h - 1);
    xi = (cb << (hs + 1)) + k;
    yi = first ? (cb << (hs + 1)) + 2 * h - 1 - k : (cb << (hs + 1)) + h + k;
}

template <typename T>
__global__ void __launch_bounds__(cmp_threads<sizeof(T)>(), 1) k_rows_cmp(RowsCmpArgs<T> a) {
    constexpr int W = sizeof(T);
    constexpr int B = 8 * W;
    constexpr int L = cmp_levels<W>();
    constexpr int NCALL = L + 3;
    constexpr int WORDS = 32 * W / 4;
    constexpr int NB = 32 * W / 16;
    constexpr int kThreads = cmp_threads<W>();
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t ksp[kThreads / 32][3][4];
    __shared__ uint32_t ballots[kThreads / 32][3][3];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* myks = sm + kAesSmemBytes / 4 + (size_t)warp * NCALL * 3 * WORDS;
    auto kword = [&](int call, int q) -> T {
        const uint32_t* w = myks + (call * 3 + q) * WORDS;
        if constexpr (W == 4) return (T)w[lane];
        else return (T)w[2 * lane] | ((T)w[2 * lane + 1] << 32);
    };
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < a.m;
         base += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long p0w = base + warp * 32, p = p0w + lane;
        const bool valid = p < a.m;
        unsigned long long xi = p, yi = p;
        if (a.hs >= 0) bitonic_rows(p, a.hs, a.first, xi, yi);
        T G[3] = {0, 0, 0}, E[3] = {0, 0, 0};
        unsigned long long koff = 0;  // nonce offset of key k's first call
        for (int k = 0; k < a.nkeys; k++) {
            T X[3] = {0, 0, 0}, Y[3] = {0, 0, 0};
            if (valid)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    X[j] = a.x[k][j][xi];
                    Y[j] = a.y[k][j][yi];
                }
            const int ncall = k ? L + 3 : L + 1;
            __syncwarp();  // the previous key's keystream has been read
            for (int idx = lane; idx < ncall * 3 * NB; idx += 32) {
                const int call = idx / (3 * NB), q = (idx / NB) % 3, b = idx % NB;
                const unsigned long long off =
                    koff + (call <= L ? (unsigned long long)call * a.C
                                      : (unsigned long long)(L + 1) * a.C + a.Cp + (unsigned long long)(call - L - 1) * a.C);
                const uint4 ks = keystream_block_n(S, a.pair[q].rk, a.pair[q].nonce + off, p0w * W / 16 + b);
                uint32_t* o = myks + (call * 3 + q) * WORDS + b * 4;
                o[0] = ks.x;
                o[1] = ks.y;
                o[2] = ks.z;
                o[3] = ks.w;
            }
            if (lane < 3) {
                const uint4 ks = keystream_block_n(S, a.pair[lane].rk,
                                                   a.pair[lane].nonce + koff + (unsigned long long)(L + 1) * a.C,
                                                   (p0w / B) * W / 16);
                ksp[warp][lane][0] = ks.x;
                ksp[warp][lane][1] = ks.y;
                ksp[warp][lane][2] = ks.z;
                ksp[warp][lane][3] = ks.w;
            }
            __syncwarp();
            T A[3], Bv[3], Sm[3], g[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                A[j] = a.desc[k] ? Y[j] : X[j];
                Bv[j] = a.desc[k] ? X[j] : Y[j];
            }
            bit_same3(A, Bv, kword, Sm);
            gt_bits3(A, Bv, Sm, valid, p, p0w, warp, kword, ksp[warp], ballots, g);
            if (k == 0) {
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    G[j] = g[j];
                    E[j] = Sm[j] & 1;
                }
            } else {
                T K[3], Z[3], e[3];
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    K[j] = kword(L + 1, j);
                    e[j] = Sm[j] & 1;
                }
                and3(g, E, K, Z);
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    G[j] ^= Z[j];
                    K[j] = kword(L + 2, j);
                }
                and3(E, e, K, Z);
#pragma unroll
                for (int j = 0; j < 3; j++) E[j] = Z[j];
            }
            koff += (unsigned long long)ncall * a.C + a.Cp;
        }
        if (valid)
#pragma unroll
            for (int j = 0; j < 3; j++) a.gt[j][p] = G[j] & 1;
    }
}

// swap (operators/sorting.h:146-212) of nbool B-shared then narith A-shared
// column pairs with the same bits: per column tmp = multiplex(b, x, y),
// y = multiplex(b, y, x), x = tmp (operators/common.h:20-49), two AND (or
// multiply_a) calls on the PAIR streams, columns in order. With b2a the
// arithmetic columns use b2a_bit(bits) (replicated_3pc.h:220-251, three
// arithmetic calls after the boolean columns), as bitonic_sort does for its
// A-shared data; otherwise `bits` is already A-shared. One thread owns 16/W
// consecutive pairs and one AES block per stream and call.
template <typename T>
struct RowsSwapArgs {
    T* x[kMaxRowCols][3];
    T* y[kMaxRowCols][3];
    int nbool, narith, b2a;
    const T* bits[3];
    StreamArg pair[3];  // nonces at the first swap call
    unsigned long long C, m;
    int hs, first;      // bitonic mapping as in RowsCmpArgs (hs < 0: none)
};

// keystream of one 16-byte unit u of a call that starts `off` nonces past the
// PAIR streams' nonces: K[e][stream] is element e's word of each stream
template <typename T, int E>
__device__ __forceinline__ void unit_keystream(const AesSmem& S, const StreamArg (&pair)[3],
                                               unsigned long long off, unsigned long long u, T (&K)[E][3]) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const uint4 b = keystream_block_n(S, pair[q].rk, pair[q].nonce + off, u);
        if constexpr (sizeof(T) == 4) {
            K[0][q] = b.x;
            K[1][q] = b.y;
            K[2][q] = b.z;
            K[3][q] = b.w;
        } else {
            K[0][q] = (T)b.x | ((T)b.y << 32);
            K[1][q] = (T)b.z | ((T)b.w << 32);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kAesThreads, 1) k_rows_swap(RowsSwapArgs<T> a) {
    constexpr int W = sizeof(T);
    constexpr int E = 16 / W;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long units = ceil_div(a.m, (unsigned long long)E);
    for (unsigned long long u = gtid(); u < units; u += gstride()) {
        auto rows = [&](int e, unsigned long long& xi, unsigned long long& yi) {
            const unsigned long long p = u * E + e;
            xi = yi = p;
            if (a.hs >= 0) bitonic_rows(p, a.hs, a.first, xi, yi);
        };
        auto ok = [&](int e) { return u * E + e < a.m; };
        T bt[E][3];
#pragma unroll
        for (int e = 0; e < E; e++)
#pragma unroll
            for (int j = 0; j < 3; j++) bt[e][j] = ok(e) ? a.bits[j][u * E + e] : (T)0;
        unsigned long long call = 0;
        T K[E][3];
#define ORQ_NEXT_CALL() (unit_keystream(S, a.pair, call++ * a.C, u, K))
#pragma unroll 1
        for (int c = 0; c < a.nbool; c++) {
            T D[E][3];
#pragma unroll
            for (int e = 0; e < E; e++) {
                unsigned long long xi, yi;
                rows(e, xi, yi);
#pragma unroll
                for (int j = 0; j < 3; j++) D[e][j] = ok(e) ? a.x[c][j][xi] ^ a.y[c][j][yi] : (T)0;
            }
            // x' = x ^ (ext(b) & (y ^ x)) on the first call, y' on the second
#pragma unroll 1  // one AES call in flight keeps the tile in registers
            for (int side = 0; side < 2; side++) {
                ORQ_NEXT_CALL();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    if (!ok(e)) continue;
                    unsigned long long xi, yi;
                    rows(e, xi, yi);
                    T Ex[3], Z[3];
#pragma unroll
                    for (int j = 0; j < 3; j++) Ex[j] = (bt[e][j] & 1) ? ~(T)0 : (T)0;  // extend_lsb
                    and3(Ex, D[e], K[e], Z);
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        T* const v = side ? a.y[c][j] + yi : a.x[c][j] + xi;
                        *v ^= Z[j];
                    }
                }
            }
        }
        if (a.narith == 0) continue;
        if (a.b2a) {
            // b2a_bit: d = s0 - s1 from two zero-sharings, then d * d on the third
            T d[E][3];
#pragma unroll 1  // one AES call in flight keeps the tile in registers
            for (int t = 0; t < 3; t++) {
                ORQ_NEXT_CALL();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    T z[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) z[p] = K[e][(p + 2) % 3] - K[e][p];
                    if (t == 0) {
#pragma unroll
                        for (int p = 0; p < 3; p++) d[e][p] = z[p];
                        d[e][0] += (bt[e][0] ^ bt[e][1]) & 1;  // P0 folds its two masked shares
                    } else if (t == 1) {
#pragma unroll
                        for (int p = 0; p < 3; p++) d[e][p] -= z[p];
                        d[e][1] -= bt[e][2] & 1;  // P1 adds its second masked share to s1
                    } else {
#pragma unroll
                        for (int p = 0; p < 3; p++) {
                            const int q = (p + 1) % 3;
                            bt[e][p] = z[p] + d[e][p] * d[e][p] + d[e][p] * d[e][q] + d[e][q] * d[e][p];
                        }
                    }
                }
            }
        }
        // bt now holds A-shared bits
#pragma unroll 1
        for (int c = a.nbool; c < a.nbool + a.narith; c++) {
            T D[E][3];
#pragma unroll
            for (int e = 0; e < E; e++) {
                unsigned long long xi, yi;
                rows(e, xi, yi);
#pragma unroll
                for (int j = 0; j < 3; j++) D[e][j] = ok(e) ? a.y[c][j][yi] - a.x[c][j][xi] : (T)0;
            }
            // multiply_a (replicated_3pc.h:44-67) of the bits with y - x, then
            // with x - y: z_p = r_p + s_p d_p + s_p d_q + s_q d_p
#pragma unroll 1  // one AES call in flight keeps the tile in registers
            for (int side = 0; side < 2; side++) {
                ORQ_NEXT_CALL();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    if (!ok(e)) continue;
                    unsigned long long xi, yi;
                    rows(e, xi, yi);
#pragma unroll
                    for (int p = 0; p < 3; p++) {
                        const int q = (p + 1) % 3;
                        const T prod = bt[e][p] * D[e][p] + bt[e][p] * D[e][q] + bt[e][q] * D[e][p];
                        T* const v = side ? a.y[c][p] + yi : a.x[c][p] + xi;
                        *v += (K[e][(p + 2) % 3] - K[e][p]) + (side ? (T)0 - prod : prod);
                    }
                }
            }
        }
    }
}
#undef ORQ_NEXT_CALL

// BSharedVector::extend_lsb (b_shared_vector.h:145-147): every share becomes
// all ones where its LSB is set (local: repeating a bit is XOR-linear)
template <typename T>
__global__ void k_extend_lsb(CSh3 x, Sh3 y, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride())
#pragma unroll
        for (int j = 0; j < 3; j++)
            reinterpret_cast<T*>(y.p[j])[i] = (T)0 - (reinterpret_cast<const T*>(x.p[j])[i] & 1);
}

// ---- batched bitonic sorting -------------------------------------------------
// Many independent sorts advance one network stage per launch ("round"): a
// round's work list holds (item, first pair) tiles of every item that still
// has a stage; stage r has the same (box size, reversal) for every item, and
// item i's nonces at stage r are its base plus r times its per-stage use, so
// the shares equal those of sequential plain calls in list order.
struct CmpBatchItem {
    void* key[3];
    unsigned long long m;          // pairs (n / 2)
    unsigned long long nonce0[3];  // PAIR nonces at the item's first stage
    unsigned long long C, Cp;      // nonces per full / packed AND call
    int stages;
    int desc;
};

template <typename T>
struct CmpBatchArgs {
    CmpArgs<T> proto;  // keys of the PAIR streams
    const CmpBatchItem* items;
    const uint2* work;  // (item, first pair) per tile
    unsigned nwork;
    int round, hs, first;
};

// at most 512 threads per CTA (the item bookkeeping needs registers)
template <int W>
constexpr int batch_max_threads() { return W == 4 ? 512 : 448; }

template <typename T>
__global__ void __launch_bounds__(batch_max_threads<sizeof(T)>(), 1) k_cmp_batch(CmpBatchArgs<T> ba) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    constexpr int kCmpThreads = batch_max_threads<W>();
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t ksp[kCmpThreads / 32][3][4];
    __shared__ uint32_t ballots[kCmpThreads / 32][3][3];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    for (unsigned w = blockIdx.x; w < ba.nwork; w += gridDim.x) {
        const uint2 wk = ba.work[w];
        const CmpBatchItem& it = ba.items[wk.x];
        CmpArgs<T> a;  // the stream keys stay in the kernel parameters (ba.proto)
        unsigned long long nonce[3];
        for (int j = 0; j < 3; j++) {
            a.key[j] = (T*)it.key[j];
            nonce[j] = it.nonce0[j] + (unsigned long long)ba.round * ((L + 3) * it.C + it.Cp);
        }
        a.m = it.m;
        a.C = it.C;
        a.Cp = it.Cp;
        a.hs = ba.hs;
        a.first = ba.first;
        a.desc = it.desc;
        cmp_tile<T, 0>(a, ba.proto.pair, nonce, wk.y, S, sm + kAesSmemBytes / 4, ksp, ballots);
    }
}

template <typename T, int MODE>
void launch_cmp(Ctx& c, const CmpArgs<T>& a, const char* name) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    constexpr int NFULL = MODE == 0 ? L + 3 : (MODE == 1 ? L + 1 : L);
    constexpr int kCmpThreads = cmp_threads<W>();
    // spread small stages over every SM: threads per CTA a multiple of 64
    // (whole packed words for both widths) up to the maximum
    const unsigned long long per_sm = ceil_div(a.m, (unsigned long long)c.num_sms);
    constexpr unsigned long long G = W == 16 ? 128 : 64;  // threads of whole packed words
    const int nt = (int)std::min<unsigned long long>(kCmpThreads, std::max<unsigned long long>(G, ceil_div(per_sm, G) * G));
    const size_t ks_bytes = (size_t)(nt / 32) * NFULL * 3 * (32 * W / 4) * 4;
    const size_t smem = kAesSmemBytes + ks_bytes;
    const size_t smem_max = kAesSmemBytes + (size_t)(kCmpThreads / 32) * NFULL * 3 * (32 * W / 4) * 4;
    auto kern = k_cmp<T, MODE>;
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    const unsigned long long units = ceil_div(a.m, nt);
    const unsigned grid = (unsigned)std::min<unsigned long long>(units ? units : 1, (unsigned long long)c.num_sms);
    const double calls = NFULL;
    ProfScope ps(c, name, (MODE == 2 ? 9.0 : 12.0) * W * a.m,
                 calls * 3.0 * ceil_div(a.m * W, 16) + (MODE == 2 ? 0.0 : 3.0 * ceil_div(ceil_div(a.m, 8 * W) * W, 16)));
    kern<<<grid, nt, smem, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

template <typename T>
void compare_t(Ctx& c, size_t n, CSh3 x, CSh3 y, Sh3 eq, Sh3 gt) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    CmpArgs<T> a{};
    for (int j = 0; j < 3; j++) {
        a.x[j] = (const T*)x.p[j];
        a.y[j] = (const T*)y.p[j];
        a.eq[j] = (T*)eq.p[j];
        a.gt[j] = (T*)gt.p[j];
        a.pair[j] = c.stream_arg(PAIR0 + j);
    }
    a.C = chunks_of((unsigned long long)n * W);
    a.Cp = chunks_of(ceil_div(n, 8 * W) * W);
    a.m = n;
    if (n) launch_cmp<T, 1>(c, a, "compare");
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (unsigned long long)(L + 1) * a.C + a.Cp;
}

template <typename T>
void equal_t(Ctx& c, size_t n, CSh3 x, CSh3 y, Sh3 eq) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    CmpArgs<T> a{};
    for (int j = 0; j < 3; j++) {
        a.x[j] = (const T*)x.p[j];
        a.y[j] = (const T*)y.p[j];
        a.eq[j] = (T*)eq.p[j];
        a.pair[j] = c.stream_arg(PAIR0 + j);
    }
    a.C = chunks_of((unsigned long long)n * W);
    a.m = n;
    if (n) launch_cmp<T, 2>(c, a, "equal");
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (unsigned long long)L * a.C;
}

// not_b_1 (replicated_3pc.h:207): every share becomes !(s & 1)
template <typename T>
__global__ void k_not1(CSh3 x, Sh3 y, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride())
#pragma unroll
        for (int j = 0; j < 3; j++)
            reinterpret_cast<T*>(y.p[j])[i] = (reinterpret_cast<const T*>(x.p[j])[i] & 1) ^ 1;
}

template <typename T>
void bitonic_t(Ctx& c, size_t n, Sh3 key, bool desc) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    int rounds = 0;
    while (((size_t)1 << rounds) < n) rounds++;
    const size_t m = n / 2;
    CmpArgs<T> a{};
    for (int j = 0; j < 3; j++) a.key[j] = (T*)key.p[j];
    a.C = chunks_of((unsigned long long)m * W);
    a.Cp = chunks_of(ceil_div(m, 8 * W) * W);
    a.m = m;
    a.desc = desc;
    for (int i = 0; i < rounds; i++)
        for (int jj = 0; jj <= i; jj++) {
            a.hs = i - jj;
            a.first = jj == 0;
            for (int q = 0; q < 3; q++) a.pair[q] = c.stream_arg(PAIR0 + q);
            launch_cmp<T, 0>(c, a, "bitonic_stage");
            for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (unsigned long long)(L + 3) * a.C + a.Cp;
        }
}

// stage r of a bitonic network: round i with i(i+1)/2 <= r, substage jj
void stage_of(int r, int& hs, int& first) {
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= r) i++;
    const int jj = r - i * (i + 1) / 2;
    hs = i - jj;
    first = jj == 0;
}

template <typename T>
void build_items(Ctx& c, int count, const size_t* n, const Sh3* keys, const int* desc,
                 std::vector<CmpBatchItem>& items, unsigned long long advance[1], int& rounds) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    items.resize(count);
    unsigned long long off = 0;
    rounds = 0;
    for (int i = 0; i < count; i++) {
        CmpBatchItem& it = items[i];
        int k = 0;
        while (((size_t)1 << k) < n[i]) k++;
        it.m = n[i] / 2;
        it.C = chunks_of(it.m * W);
        it.Cp = chunks_of(ceil_div(it.m, 8ull * W) * W);
        it.stages = n[i] < 2 ? 0 : k * (k + 1) / 2;
        it.desc = desc[i];
        for (int j = 0; j < 3; j++) {
            it.key[j] = keys[i].p[j];
            it.nonce0[j] = c.nonce[PAIR0 + j] + off;
        }
        off += (unsigned long long)it.stages * ((L + 3) * it.C + it.Cp);
        rounds = std::max(rounds, it.stages);
    }
    advance[0] = off;
}

void build_work(const std::vector<CmpBatchItem>& items, int rounds, int nt, std::vector<uint2>& work,
                std::vector<size_t>& round_off) {
    work.clear();
    round_off.assign(rounds + 1, 0);
    for (int r = 0; r < rounds; r++) {
        round_off[r] = work.size();
        for (size_t i = 0; i < items.size(); i++) {
            if (items[i].stages <= r) continue;
            for (unsigned long long p = 0; p < items[i].m; p += nt) work.push_back(make_uint2((unsigned)i, (unsigned)p));
        }
    }
    round_off[rounds] = work.size();
}

template <typename T>
size_t batch_smem(int nt) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    return kAesSmemBytes + (size_t)(nt / 32) * (L + 3) * 3 * (32 * W / 4) * 4;
}

template <typename T>
CmpArgs<T> batch_proto(Ctx& c) {
    CmpArgs<T> p{};
    for (int q = 0; q < 3; q++) p.pair[q] = c.stream_arg(PAIR0 + q);
    return p;
}

template <typename T>
void launch_rounds(Ctx& c, cudaStream_t st, const CmpArgs<T>& proto, const CmpBatchItem* items_dev,
                   const uint2* work_dev, const std::vector<size_t>& round_off, int rounds, int nt,
                   bool profile) {
    auto kern = k_cmp_batch<T>;
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)batch_smem<T>(batch_max_threads<sizeof(T)>())));
    for (int r = 0; r < rounds; r++) {
        CmpBatchArgs<T> ba;
        ba.proto = proto;
        ba.items = items_dev;
        ba.work = work_dev + round_off[r];
        ba.nwork = (unsigned)(round_off[r + 1] - round_off[r]);
        ba.round = r;
        stage_of(r, ba.hs, ba.first);
        if (!ba.nwork) continue;
        const unsigned grid = std::min<unsigned>(ba.nwork, (unsigned)c.num_sms);
        if (profile) {
            ProfScope ps(c, "bitonic_batch_round", 0.0, 0.0, st);
            kern<<<grid, nt, batch_smem<T>(nt), st>>>(ba);
        } else {
            kern<<<grid, nt, batch_smem<T>(nt), st>>>(ba);
        }
        ORQ_CUDA_CHECK(cudaGetLastError());
    }
}

// Autotuner: threads per CTA for a size class, chosen by timing round 0 of
// the batch on scratch copies of (a prefix of) its keys with every candidate.
template <typename T>
int autotune(Ctx& c, const std::vector<CmpBatchItem>& items) {
    constexpr int W = sizeof(T);
    const int cands4[] = {256, 384, 512};
    const int cands8[] = {256, 448};
    const int* cands = W == 4 ? cands4 : cands8;
    const int nc = W == 4 ? 3 : 2;
    // a prefix of items of at most 256 MB of shares
    std::vector<CmpBatchItem> sub;
    size_t bytes = 0;
    for (const auto& it : items) {
        const size_t b = 2 * it.m * W * 3;
        if (!sub.empty() && bytes + b > (256u << 20)) break;
        sub.push_back(it);
        bytes += b;
    }
    Scratch keys(c, bytes + 16), itb(c, sub.size() * sizeof(CmpBatchItem) + 16);
    size_t off = 0;
    for (auto& it : sub) {
        for (int j = 0; j < 3; j++) {
            void* dst = keys.as<uint8_t>() + off;
            ORQ_CUDA_CHECK(cudaMemcpyAsync(dst, it.key[j], 2 * it.m * W, cudaMemcpyDeviceToDevice, c.stream));
            it.key[j] = dst;
            off += 2 * it.m * W;
        }
    }
    ORQ_CUDA_CHECK(cudaMemcpyAsync(itb.p, sub.data(), sub.size() * sizeof(CmpBatchItem),
                                   cudaMemcpyHostToDevice, c.stream));
    const CmpArgs<T> proto = batch_proto<T>(c);
    cudaEvent_t e0, e1;
    ORQ_CUDA_CHECK(cudaEventCreate(&e0));
    ORQ_CUDA_CHECK(cudaEventCreate(&e1));
    int best = cands[0];
    float best_ms = 1e30f;
    for (int k = 0; k < nc; k++) {
        std::vector<uint2> work;
        std::vector<size_t> roff;
        build_work(sub, 1, cands[k], work, roff);
        Scratch wb(c, work.size() * sizeof(uint2) + 16);
        ORQ_CUDA_CHECK(cudaMemcpyAsync(wb.p, work.data(), work.size() * sizeof(uint2),
                                       cudaMemcpyHostToDevice, c.stream));
        float ms = 0;
        for (int rep = 0; rep < 2; rep++) {
            ORQ_CUDA_CHECK(cudaEventRecord(e0, c.stream));
            launch_rounds<T>(c, c.stream, proto, itb.as<CmpBatchItem>(), wb.as<uint2>(), roff, 1, cands[k], false);
            ORQ_CUDA_CHECK(cudaEventRecord(e1, c.stream));
            ORQ_CUDA_CHECK(cudaEventSynchronize(e1));
            ORQ_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        }
        c.kernels_launched += 2;
        if (ms < best_ms) {
            best_ms = ms;
            best = cands[k];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

template <typename T>
void bitonic_batch_t(Ctx& c, int count, const size_t* n, const Sh3* keys, const int* desc, bool use_graph) {
    constexpr int W = sizeof(T);
    std::vector<CmpBatchItem> items;
    unsigned long long advance[1];
    int rounds;
    build_items<T>(c, count, n, keys, desc, items, advance, rounds);
    if (rounds == 0) return;
    // size class: key width and log2 of round 0's pairs
    unsigned long long pairs0 = 0;
    for (const auto& it : items) pairs0 += it.stages ? it.m : 0;
    int lg = 0;
    while ((1ull << lg) < pairs0) lg++;
    const std::string cls = "bitonic:" + std::to_string(W) + ":" + std::to_string(lg);
    int nt;
    if (auto f = c.tuned.find(cls); f != c.tuned.end()) {
        nt = f->second;
    } else {
        nt = autotune<T>(c, items);
        c.tuned[cls] = nt;
    }
    const CmpArgs<T> proto = batch_proto<T>(c);
    const size_t ibytes = items.size() * sizeof(CmpBatchItem);
    if (use_graph) {
        std::string shape = cls + ":" + std::to_string(nt) + ":";
        for (int i = 0; i < count; i++) shape += std::to_string(n[i]) + ",";
        BatchGraph& g = c.graphs[shape];
        if (!g.exec) {
            std::vector<uint2> work;
            std::vector<size_t> roff;
            build_work(items, rounds, nt, work, roff);
            ORQ_CUDA_CHECK(cudaMalloc(&g.work, std::max<size_t>(16, work.size() * sizeof(uint2))));
            ORQ_CUDA_CHECK(cudaMemcpy(g.work, work.data(), work.size() * sizeof(uint2), cudaMemcpyHostToDevice));
            ORQ_CUDA_CHECK(cudaMalloc(&g.items_dev, ibytes));
            ORQ_CUDA_CHECK(cudaHostAlloc(&g.items_host, ibytes, cudaHostAllocDefault));
            ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
            g.items_bytes = ibytes;
            g.nt = nt;
            if (!c.capture_stream)
                ORQ_CUDA_CHECK(cudaStreamCreateWithFlags(&c.capture_stream, cudaStreamNonBlocking));
            // the proto's nonces are overwritten per item, so the graph only
            // depends on the stream keys and the shape
            cudaGraph_t graph;
            ORQ_CUDA_CHECK(cudaStreamBeginCapture(c.capture_stream, cudaStreamCaptureModeThreadLocal));
            ORQ_CUDA_CHECK(cudaMemcpyAsync(g.items_dev, g.items_host, ibytes, cudaMemcpyHostToDevice,
                                           c.capture_stream));
            launch_rounds<T>(c, c.capture_stream, proto, (const CmpBatchItem*)g.items_dev,
                             (const uint2*)g.work, roff, rounds, nt, false);
            ORQ_CUDA_CHECK(cudaStreamEndCapture(c.capture_stream, &graph));
            ORQ_CUDA_CHECK(cudaGraphInstantiate(&g.exec, graph, 0));
            ORQ_CUDA_CHECK(cudaGraphDestroy(graph));
            for (int r = 0; r < rounds; r++) g.launches += roff[r + 1] > roff[r];
        }
        ORQ_CUDA_CHECK(cudaEventSynchronize(g.done));  // the previous replay has read the table
        std::memcpy(g.items_host, items.data(), ibytes);
        {
            ProfScope ps(c, "bitonic_batch_graph", 0.0, 0.0);
            ORQ_CUDA_CHECK(cudaGraphLaunch(g.exec, c.stream));
        }
        ORQ_CUDA_CHECK(cudaEventRecord(g.done, c.stream));
        c.kernels_launched += g.launches;
    } else {
        std::vector<uint2> work;
        std::vector<size_t> roff;
        build_work(items, rounds, nt, work, roff);
        Scratch wb(c, work.size() * sizeof(uint2) + 16), itb(c, ibytes + 16);
        ORQ_CUDA_CHECK(cudaMemcpyAsync(wb.p, work.data(), work.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                                       c.stream));
        ORQ_CUDA_CHECK(cudaMemcpyAsync(itb.p, items.data(), ibytes, cudaMemcpyHostToDevice, c.stream));
        launch_rounds<T>(c, c.stream, proto, itb.as<CmpBatchItem>(), wb.as<uint2>(), roff, rounds, nt,
                         c.profiling);
        for (int r = 0; r < rounds; r++) c.kernels_launched += roff[r + 1] > roff[r];
        // the host vectors are read by the copies above before they return
        // (pageable memory), and the scratch goes back to the pool in stream order
        ORQ_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    }
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += advance[0];
}

// nonces of one compare_rows over nkeys keys (each call of m pairs)
template <int W>
unsigned long long rows_cmp_nonces(int nkeys, unsigned long long C, unsigned long long Cp) {
    constexpr int L = cmp_levels<W>();
    return (unsigned long long)nkeys * ((L + 1) * C + Cp) + 2ull * (nkeys - 1) * C;
}

template <typename T>
void launch_rows_cmp(Ctx& c, const RowsCmpArgs<T>& a) {
    constexpr int W = sizeof(T);
    constexpr int L = cmp_levels<W>();
    constexpr int kThreads = cmp_threads<W>();
    const unsigned long long per_sm = ceil_div(a.m, (unsigned long long)c.num_sms);
    const int nt = (int)std::min<unsigned long long>(kThreads, std::max<unsigned long long>(64, ceil_div(per_sm, 64) * 64));
    const size_t per_warp = (size_t)(L + 3) * 3 * (32 * W / 4) * 4;
    const size_t smem = kAesSmemBytes + (size_t)(nt / 32) * per_warp;
    auto kern = k_rows_cmp<T>;
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(kAesSmemBytes + (size_t)(kThreads / 32) * per_warp)));
    const unsigned long long units = ceil_div(a.m, (unsigned long long)nt);
    const unsigned grid = (unsigned)std::min<unsigned long long>(units ? units : 1, (unsigned long long)c.num_sms);
    const double full_calls = (double)a.nkeys * (L + 1) + 2.0 * (a.nkeys - 1);
    ProfScope ps(c, "compare_rows", (6.0 * a.nkeys + 3.0) * W * a.m,
                 full_calls * 3.0 * ceil_div(a.m * W, 16) + 3.0 * a.nkeys * ceil_div(ceil_div(a.m, 8 * W) * W, 16));
    kern<<<grid, nt, smem, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

// launches one swap and returns the nonces it used: two calls per column and
// three for the b2a of the bits
template <typename T>
unsigned long long launch_rows_swap(Ctx& c, const RowsSwapArgs<T>& a) {
    constexpr int W = sizeof(T);
    const unsigned long long calls = 2ull * (a.nbool + a.narith) + (a.b2a && a.narith ? 3ull : 0ull);
    if (a.m && (a.nbool + a.narith))
        launch_aes(c, "swap", (12.0 * (a.nbool + a.narith) + 3.0) * W * a.m,
                   3.0 * calls * ceil_div(a.m * W, 16), k_rows_swap<T>, ceil_div(a.m, (unsigned long long)(16 / W)), a);
    return calls * a.C;
}

template <typename T>
void compare_rows_t(Ctx& c, size_t n, int nkeys, const CSh3* x, const CSh3* y, const int* desc, Sh3 gt) {
    constexpr int W = sizeof(T);
    RowsCmpArgs<T> a{};
    for (int k = 0; k < nkeys; k++) {
        for (int j = 0; j < 3; j++) {
            a.x[k][j] = (const T*)x[k].p[j];
            a.y[k][j] = (const T*)y[k].p[j];
        }
        a.desc[k] = desc[k] != 0;
    }
    for (int j = 0; j < 3; j++) {
        a.gt[j] = (T*)gt.p[j];
        a.pair[j] = c.stream_arg(PAIR0 + j);
    }
    a.nkeys = nkeys;
    a.m = n;
    a.hs = -1;
    a.C = chunks_of((unsigned long long)n * W);
    a.Cp = chunks_of(ceil_div(n, 8 * W) * W);
    if (n) launch_rows_cmp(c, a);
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += rows_cmp_nonces<W>(nkeys, a.C, a.Cp);
}

template <typename T>
void swap_t(Ctx& c, size_t n, bool arith, int ncols, const Sh3* x, const Sh3* y, CSh3 bits) {
    constexpr int W = sizeof(T);
    RowsSwapArgs<T> a{};
    for (int k = 0; k < ncols; k++)
        for (int j = 0; j < 3; j++) {
            a.x[k][j] = (T*)x[k].p[j];
            a.y[k][j] = (T*)y[k].p[j];
        }
    for (int j = 0; j < 3; j++) {
        a.bits[j] = (const T*)bits.p[j];
        a.pair[j] = c.stream_arg(PAIR0 + j);
    }
    a.nbool = arith ? 0 : ncols;
    a.narith = arith ? ncols : 0;
    a.m = n;
    a.hs = -1;
    a.C = chunks_of((unsigned long long)n * W);
    const unsigned long long used = launch_rows_swap(c, a);
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += used;
}

// bitonic_sort (operators/sorting.h:266-353) over several key columns with
// A- and B-shared data columns: per stage one compare_rows launch writes the
// comparison bits, one swap launch moves keys, B data and (through b2a_bit of
// the bits) A data.
template <typename T>
void bitonic_rows_t(Ctx& c, size_t n, int nkeys, const Sh3* keys, const int* desc, int na,
                    const Sh3* data_a, int nb, const Sh3* data_b) {
    constexpr int W = sizeof(T);
    int rounds = 0;
    while (((size_t)1 << rounds) < n) rounds++;
    const size_t m = n / 2;
    Scratch bits(c, 3 * m * W);
    RowsCmpArgs<T> ca{};
    RowsSwapArgs<T> sa{};
    for (int k = 0; k < nkeys; k++) {
        for (int j = 0; j < 3; j++) {
            ca.x[k][j] = ca.y[k][j] = (const T*)keys[k].p[j];
            sa.x[k][j] = sa.y[k][j] = (T*)keys[k].p[j];
        }
        ca.desc[k] = desc[k] != 0;
    }
    for (int k = 0; k < nb; k++)
        for (int j = 0; j < 3; j++) sa.x[nkeys + k][j] = sa.y[nkeys + k][j] = (T*)data_b[k].p[j];
    for (int k = 0; k < na; k++)
        for (int j = 0; j < 3; j++) sa.x[nkeys + nb + k][j] = sa.y[nkeys + nb + k][j] = (T*)data_a[k].p[j];
    for (int j = 0; j < 3; j++) {
        ca.gt[j] = bits.as<T>() + j * m;
        sa.bits[j] = bits.as<T>() + j * m;
    }
    ca.nkeys = nkeys;
    ca.m = sa.m = m;
    ca.C = sa.C = chunks_of((unsigned long long)m * W);
    ca.Cp = chunks_of(ceil_div(m, 8 * W) * W);
    sa.nbool = nkeys + nb;
    sa.narith = na;
    sa.b2a = 1;
    for (int i = 0; i < rounds; i++)
        for (int jj = 0; jj <= i; jj++) {
            ca.hs = sa.hs = i - jj;
            ca.first = sa.first = jj == 0;
            for (int q = 0; q < 3; q++) ca.pair[q] = c.stream_arg(PAIR0 + q);
            launch_rows_cmp(c, ca);
            for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += rows_cmp_nonces<W>(nkeys, ca.C, ca.Cp);
            for (int q = 0; q < 3; q++) sa.pair[q] = c.stream_arg(PAIR0 + q);
            const unsigned long long used = launch_rows_swap(c, sa);
            for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += used;
        }
}

template <typename T>
void extend_lsb_t(Ctx& c, size_t n, CSh3 x, Sh3 y) {
    if (!n) return;
    ProfScope ps(c, "extend_lsb", 6.0 * sizeof(T) * n);
    k_extend_lsb<T><<<plain_grid(c, n), 256, 0, c.stream>>>(x, y, n);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

}  // namespace

void op_compare_rows(Ctx& c, int w, size_t n, int nkeys, const CSh3* x, const CSh3* y, const int* desc, Sh3 gt) {
    if (nkeys < 1 || nkeys > kMaxRowKeys) throw std::invalid_argument("compare_rows takes 1 to 8 key columns");
    if (w == 4) compare_rows_t<uint32_t>(c, n, nkeys, x, y, desc, gt);
    else if (w == 8) compare_rows_t<unsigned long long>(c, n, nkeys, x, y, desc, gt);
    else throw std::invalid_argument("compare_rows supports int32 and int64 keys");
}

void op_swap(Ctx& c, int w, size_t n, bool arith, int ncols, const Sh3* x, const Sh3* y, CSh3 bits) {
    if (ncols < 0 || ncols > kMaxRowCols) throw std::invalid_argument("swap takes 0 to 40 column pairs");
    if (w == 4) swap_t<uint32_t>(c, n, arith, ncols, x, y, bits);
    else if (w == 8) swap_t<unsigned long long>(c, n, arith, ncols, x, y, bits);
    else throw std::invalid_argument("swap supports 4 and 8-byte shares");
}

void op_extend_lsb(Ctx& c, int w, size_t n, CSh3 x, Sh3 y) {
    if (w == 4) extend_lsb_t<uint32_t>(c, n, x, y);
    else if (w == 8) extend_lsb_t<unsigned long long>(c, n, x, y);
    else throw std::invalid_argument("extend_lsb supports 4 and 8-byte shares");
}

void op_bitonic_sort_rows(Ctx& c, int w, size_t n, int nkeys, const Sh3* keys, const int* desc, int na,
                          const Sh3* data_a, int nb, const Sh3* data_b) {
    if (n & (n - 1)) throw std::invalid_argument("bitonic sort needs a power-of-two size");
    if (nkeys < 1 || nkeys > kMaxRowKeys) throw std::invalid_argument("bitonic sort takes 1 to 8 key columns");
    if (na < 0 || nb < 0 || nkeys + na + nb > kMaxRowCols)
        throw std::invalid_argument("bitonic sort takes at most 40 key and data columns");
    if (w != 4 && w != 8) throw std::invalid_argument("bitonic sort supports int32 and int64 keys");
    if (n < 2) return;
    if (nkeys == 1 && na == 0 && nb == 0) {  // one fused launch per stage
        op_bitonic_sort(c, w, n, keys[0], desc[0] != 0);
        return;
    }
    if (w == 4) bitonic_rows_t<uint32_t>(c, n, nkeys, keys, desc, na, data_a, nb, data_b);
    else bitonic_rows_t<unsigned long long>(c, n, nkeys, keys, desc, na, data_a, nb, data_b);
}

void op_compare(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 eq, Sh3 gt) {
    if (w == 4) compare_t<uint32_t>(c, n, x, y, eq, gt);
    else if (w == 8) compare_t<unsigned long long>(c, n, x, y, eq, gt);
    else if (w == 16) compare_t<unsigned __int128>(c, n, x, y, eq, gt);
    else throw std::invalid_argument("compare supports 4, 8 and 16-byte keys");
}

void op_equal(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 eq) {
    if (w == 4) equal_t<uint32_t>(c, n, x, y, eq);
    else if (w == 8) equal_t<unsigned long long>(c, n, x, y, eq);
    else if (w == 16) equal_t<unsigned __int128>(c, n, x, y, eq);
    else throw std::invalid_argument("equality supports 4, 8 and 16-byte keys");
}

void op_not1(Ctx& c, int w, size_t n, CSh3 x, Sh3 y) {
    if (!n) return;
    const unsigned g = plain_grid(c, n);
    ProfScope ps(c, "not_b_1", 6.0 * w * n);
    if (w == 4) k_not1<uint32_t><<<g, 256, 0, c.stream>>>(x, y, n);
    else if (w == 8) k_not1<unsigned long long><<<g, 256, 0, c.stream>>>(x, y, n);
    else throw std::invalid_argument("not_b_1 supports 4 and 8-byte shares");
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

void op_bitonic_sort(Ctx& c, int w, size_t n, Sh3 key, bool desc) {
    if (n & (n - 1)) throw std::invalid_argument("bitonic sort needs a power-of-two size");
    if (n < 2) return;
    if (w == 4) bitonic_t<uint32_t>(c, n, key, desc);
    else if (w == 8) bitonic_t<unsigned long long>(c, n, key, desc);
    else throw std::invalid_argument("bitonic sort supports int32 and int64 keys");
}

}  // namespace orqcu

namespace orqcu {
void op_bitonic_sort_batch(Ctx& c, int w, int count, const size_t* n, const Sh3* keys, const int* desc,
                           bool use_graph) {
    if (w == 4) bitonic_batch_t<uint32_t>(c, count, n, keys, desc, use_graph);
    else if (w == 8) bitonic_batch_t<unsigned long long>(c, count, n, keys, desc, use_graph);
    else throw std::invalid_argument("bitonic sort supports int32 and int64 keys");
}
}  // namespace orqcu
