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
#include <type_traits>

#include "launch.cuh"

namespace orqcu {

namespace {

// Threads (= pairs) per CTA iteration. The AES tables take 128 KiB of shared
// memory, so one CTA runs per SM; the per-warp keystream buffers take the rest
// (3 KiB per warp for int32 stages, 6.75 KiB for int64).
template <int W>
constexpr int cmp_threads() { return W == 4 ? 768 : 448; }

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
    using S = typename std::make_signed<T>::type;
    return (T)((S)v >> s);
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

template <typename T, int MODE>  // MODE 0: bitonic stage, MODE 1: compare
__global__ void __launch_bounds__(cmp_threads<sizeof(T)>(), 1) k_cmp(CmpArgs<T> a) {
    constexpr int W = sizeof(T);
    constexpr int kCmpThreads = cmp_threads<W>();
    constexpr int B = 8 * W;               // pairs per packed word
    constexpr int L = (W == 4) ? 5 : 6;    // bit_same rounds
    constexpr int NFULL = MODE == 0 ? L + 3 : L + 1;
    constexpr int WORDS = 32 * W / 4;      // keystream words per call and stream per warp
    constexpr int NB = 32 * W / 16;        // AES blocks per call and stream per warp
    extern __shared__ __align__(16) uint32_t sm[];
    uint32_t* ksw = sm + kAesSmemBytes / 4;  // [warp][call][stream][WORDS]
    __shared__ uint32_t ksp[kCmpThreads / 32][3][4];      // packed call block per warp
    __shared__ uint32_t ballots[kCmpThreads / 32][3][3];  // [warp][s1,s2,r][share]
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* myks = ksw + (size_t)warp * NFULL * 3 * WORDS;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < a.m;
         base += (unsigned long long)gridDim.x * blockDim.x) {
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
            StreamArg st = a.pair[q];
            st.nonce += off;
            const uint4 ks = keystream_block(S, st, p0w * W / 16 + b);
            uint32_t* o = myks + (call * 3 + q) * WORDS + b * 4;
            o[0] = ks.x;
            o[1] = ks.y;
            o[2] = ks.z;
            o[3] = ks.w;
        }
        if (lane < 3) {
            // the packed AND: word c = pair / B covers pairs [cB, cB+B)
            const unsigned long long c = p0w / B;
            StreamArg st = a.pair[lane];
            st.nonce += (unsigned long long)(L + 1) * a.C;
            const uint4 ks = keystream_block(S, st, c * W / 16);
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
            else return (T)w[2 * lane] | ((T)w[2 * lane + 1] << 32);
        };
        // ---- bit_same: prefix-AND from the MSB down
        T Sm[3];
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
        // ---- gt = parity(((eq >> 1) ^ eq) & this)
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
        // ---- sign fix-up on words of B packed pairs
        uint32_t b1[3], b2[3], br[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            b1[j] = __ballot_sync(0xffffffffu, valid && ((A[j] >> (B - 1)) & 1));
            b2[j] = __ballot_sync(0xffffffffu, valid && ((Bv[j] >> (B - 1)) & 1));
            br[j] = __ballot_sync(0xffffffffu, valid && (__popcll((unsigned long long)G[j]) & 1));
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
            // two warps per 64-pair word
            __syncthreads();
            if (lane == 0)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    ballots[warp][0][j] = b1[j];
                    ballots[warp][1][j] = b2[j];
                    ballots[warp][2][j] = br[j];
                }
            __syncthreads();
            const int w0 = warp & ~1;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                s1[j] = (T)ballots[w0][0][j] | ((T)ballots[w0 + 1][0][j] << 32);
                s2[j] = (T)ballots[w0][1][j] | ((T)ballots[w0 + 1][1][j] << 32);
                r[j] = (T)ballots[w0][2][j] | ((T)ballots[w0 + 1][2][j] << 32);
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
                if constexpr (W == 4) K[j] = (T)ksp[warp][j][c & 3];
                else K[j] = (T)ksp[warp][j][2 * (c & 1)] | ((T)ksp[warp][j][2 * (c & 1) + 1] << 32);
            }
            and3(ns2, nr, K, Z);
#pragma unroll
            for (int j = 0; j < 3; j++) s1[j] ^= ~Z[j];
        }
        const int bitpos = (int)(p % B);
        T gt[3], eq[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            gt[j] = (s1[j] >> bitpos) & 1;
            eq[j] = Sm[j] & 1;
        }
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
        __syncthreads();  // keystream buffers are rewritten by the next iteration
    }
}

template <typename T, int MODE>
void launch_cmp(Ctx& c, const CmpArgs<T>& a, const char* name) {
    constexpr int W = sizeof(T);
    constexpr int L = (W == 4) ? 5 : 6;
    constexpr int NFULL = MODE == 0 ? L + 3 : L + 1;
    constexpr int kCmpThreads = cmp_threads<W>();
    // spread small stages over every SM: threads per CTA a multiple of 64
    // (whole packed words for both widths) up to the maximum
    const unsigned long long per_sm = ceil_div(a.m, (unsigned long long)c.num_sms);
    const int nt = (int)std::min<unsigned long long>(kCmpThreads, std::max<unsigned long long>(64, ceil_div(per_sm, 64) * 64));
    const size_t ks_bytes = (size_t)(nt / 32) * NFULL * 3 * (32 * W / 4) * 4;
    const size_t smem = kAesSmemBytes + ks_bytes;
    const size_t smem_max = kAesSmemBytes + (size_t)(kCmpThreads / 32) * NFULL * 3 * (32 * W / 4) * 4;
    auto kern = k_cmp<T, MODE>;
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    const unsigned long long units = ceil_div(a.m, nt);
    const unsigned grid = (unsigned)std::min<unsigned long long>(units ? units : 1, (unsigned long long)c.num_sms);
    const double calls = NFULL;
    ProfScope ps(c, name, 12.0 * W * a.m,
                 calls * 3.0 * ceil_div(a.m * W, 16) + 3.0 * ceil_div(ceil_div(a.m, 8 * W) * W, 16));
    kern<<<grid, nt, smem, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

template <typename T>
void compare_t(Ctx& c, size_t n, CSh3 x, CSh3 y, Sh3 eq, Sh3 gt) {
    constexpr int W = sizeof(T);
    constexpr int L = (W == 4) ? 5 : 6;
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
void bitonic_t(Ctx& c, size_t n, Sh3 key, bool desc) {
    constexpr int W = sizeof(T);
    constexpr int L = (W == 4) ? 5 : 6;
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

}  // namespace

void op_compare(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 eq, Sh3 gt) {
    if (w == 4) compare_t<uint32_t>(c, n, x, y, eq, gt);
    else if (w == 8) compare_t<unsigned long long>(c, n, x, y, eq, gt);
    else throw std::invalid_argument("compare supports int32 and int64 keys");
}

void op_bitonic_sort(Ctx& c, int w, size_t n, Sh3 key, bool desc) {
    if (n & (n - 1)) throw std::invalid_argument("bitonic sort needs a power-of-two size");
    if (n < 2) return;
    if (w == 4) bitonic_t<uint32_t>(c, n, key, desc);
    else if (w == 8) bitonic_t<unsigned long long>(c, n, key, desc);
    else throw std::invalid_argument("bitonic sort supports int32 and int64 keys");
}

}  // namespace orqcu
