// tsort.cu — multi-column table sort, permutation composition and distinct.
//
// table_sort (include/core/operators/sorting.h:509-612) with the radix or
// quicksort protocol sorts the last key column first and every earlier column after
// applying the running permutation, composing the permutations
// (compose_permutations, operators/shuffle.h:717-743); all of it is host
// orchestration of the radix sort and apply kernels. distinct
// (operators/distinct.h:20-53) is one fused kernel: per row pair (k, k+1),
// bit_same over every key column, != and the OR into the result, with the
// zero-sharing keystream of each AND call computed once per 16-byte unit.
#include <type_traits>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr int kMaxDistinctKeys = 8;

// local_apply_inverse_perm (shuffle.h:250-270): dst[i] = src[idx[i]]; an
// index outside [0, n) sets error bit 32 and is skipped.
__global__ void k_gather4(CSh3 src, Sh3 dst, const int32_t* idx, unsigned long long n, int* err) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        const long long j = idx[i];
        if (j < 0 || (unsigned long long)j >= n) {
            atomicOr(err, 32);
            continue;
        }
#pragma unroll
        for (int p = 0; p < 3; p++)
            reinterpret_cast<int32_t*>(dst.p[p])[i] = reinterpret_cast<const int32_t*>(src.p[p])[j];
    }
}

struct DistinctArgs {
    const void* key[kMaxDistinctKeys][3];
    void* res[3];
    int nkeys;
    unsigned long long m;  // row pairs (n - 1)
    unsigned long long C;  // nonces per AND call (m*W bytes)
    StreamArg pair[3];
};

template <typename T>
__device__ __forceinline__ void and3d(const T* x, const T* y, const T* k, T* z) {
    const T r0 = k[2] ^ k[0], r1 = k[0] ^ k[1], r2 = k[1] ^ k[2];
    const T z0 = r0 ^ (x[0] & y[0]) ^ (x[0] & y[1]) ^ (x[1] & y[0]);
    const T z1 = r1 ^ (x[1] & y[1]) ^ (x[1] & y[2]) ^ (x[2] & y[1]);
    const T z2 = r2 ^ (x[2] & y[2]) ^ (x[2] & y[0]) ^ (x[0] & y[2]);
    z[0] = z0;
    z[1] = z1;
    z[2] = z2;
}

template <int W>
__global__ void __launch_bounds__(kAesThreads) k_distinct(DistinctArgs a) {
    using T = typename std::conditional<W == 4, uint32_t, unsigned long long>::type;
    using ST = typename std::make_signed<T>::type;
    constexpr int E = 16 / W;
    constexpr int L = (W == 4) ? 5 : 6;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    if (gtid() == 0) {  // the first row is always distinct (public 1)
        reinterpret_cast<T*>(a.res[0])[0] = 1;
        reinterpret_cast<T*>(a.res[1])[0] = 0;
        reinterpret_cast<T*>(a.res[2])[0] = 0;
    }
    const unsigned long long units = ceil_div(a.m * W, 16);
    for (unsigned long long u = gtid(); u < units; u += gstride()) {
        unsigned long long off = 0;
        T K[E][3];
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
        bool ok[E];
#pragma unroll
        for (int k = 0; k < E; k++) ok[k] = u * E + k < a.m;
        T R[E][3];
#pragma unroll
        for (int k = 0; k < E; k++) R[k][0] = R[k][1] = R[k][2] = 0;
#pragma unroll 1
        for (int j = 0; j < a.nkeys; j++) {
            T Sm[E][3];
#pragma unroll
            for (int k = 0; k < E; k++)
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const T* kp = reinterpret_cast<const T*>(a.key[j][p]);
                    const unsigned long long e = u * E + k;
                    Sm[k][p] = ok[k] ? (T)~(kp[e] ^ kp[e + 1]) : (T)0;
                }
#pragma unroll 1
            for (int lev = 0; lev < L; lev++) {
                next_call();
#pragma unroll
                for (int k = 0; k < E; k++) {
                    T Tm[3];
#pragma unroll
                    for (int p = 0; p < 3; p++) Tm[p] = (T)((ST)Sm[k][p] >> (1 << lev));
                    and3d(Sm[k], Tm, K[k], Sm[k]);
                }
            }
            // != is !(== & 1); |= is ~(~rest & ~x)
            next_call();
#pragma unroll
            for (int k = 0; k < E; k++) {
                T nr[3], nx[3], Z[3];
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    nx[p] = ~((Sm[k][p] & 1) ^ 1);
                    nr[p] = ~R[k][p];
                }
                and3d(nr, nx, K[k], Z);
#pragma unroll
                for (int p = 0; p < 3; p++) R[k][p] = ~Z[p];
            }
        }
#pragma unroll
        for (int k = 0; k < E; k++)
            if (ok[k])
#pragma unroll
                for (int p = 0; p < 3; p++) reinterpret_cast<T*>(a.res[p])[u * E + k + 1] = R[k][p];
    }
}

// ElementwisePermutation(size, BShared) (permutation.h:62-69): the identity,
// public-shared (S0 = i, S1 = S2 = 0) at width W
template <typename T>
__global__ void k_identity(Sh3 p, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        reinterpret_cast<T*>(p.p[0])[i] = (T)i;
        reinterpret_cast<T*>(p.p[1])[i] = 0;
        reinterpret_cast<T*>(p.p[2])[i] = 0;
    }
}

// an opened permutation of width W narrowed to int32; a value outside [0, n)
// sets error bit 128 and becomes i (the scatter then keeps every index valid)
template <typename T>
__global__ void k_narrow(const void* src, int32_t* dst, unsigned long long n, int* err) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        const unsigned long long v = (unsigned long long)reinterpret_cast<const T*>(src)[i];
        if (v >= n) {
            atomicOr(err, 128);
            dst[i] = (int32_t)i;
        } else {
            dst[i] = (int32_t)v;
        }
    }
}

// BSharedVector::mask(m) (b_shared_vector.h:462-464): every share &= m
template <typename T>
__global__ void k_mask(Sh3 s, unsigned long long n, T m) {
    for (unsigned long long i = gtid(); i < n; i += gstride())
#pragma unroll
        for (int j = 0; j < 3; j++) reinterpret_cast<T*>(s.p[j])[i] &= m;
}

void copy_sh(Ctx& c, Sh3 dst, CSh3 src, size_t bytes) {
    if (!bytes) return;
    for (int p = 0; p < 3; p++)
        ORQ_CUDA_CHECK(cudaMemcpyAsync(dst.p[p], src.p[p], bytes, cudaMemcpyDeviceToDevice, c.stream));
}

CSh3 cc(Sh3 s) { return CSh3{{s.p[0], s.p[1], s.p[2]}}; }

}  // namespace

// oblivious_apply_elementwise_perm (shuffle.h:687-706) with a B-shared
// permutation of width pw (the table shuffle's): x and a copy of the
// permutation are shuffled by the same sharded permutation (x's reshare
// before the permutation's on every group stream), the permutation is opened
// and x scattered by it. Composed from the sharded apply, open and scatter.
static void apply_elementwise_bperm(Ctx& c, bool x_arith, int xw, size_t n, Sh3 x, CSh3 perm, int pw) {
    ShardedPerm sp = next_perm(c, n);
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch cpb(c, 3 * n1 * pw), opened(c, n1 * pw), sig(c, n1 * 4), tmp(c, 3 * n1 * xw);
    Sh3 P, Xt;
    for (int j = 0; j < 3; j++) {
        P.p[j] = cpb.as<uint8_t>() + j * n1 * pw;
        Xt.p[j] = tmp.as<uint8_t>() + j * n1 * xw;
    }
    copy_sh(c, P, perm, n * pw);
    op_apply_sharded(c, x_arith, xw, n, x, sp, false);
    op_apply_sharded(c, false, pw, n, P, sp, false);
    c.free_perm(sp);
    if (!n) return;
    op_open(c, false, pw, n, cc(P), opened.p);
    if (pw == 4) k_narrow<uint32_t><<<plain_grid(c, n), 256, 0, c.stream>>>(opened.p, sig.as<int32_t>(), n, c.d_err);
    else k_narrow<unsigned long long><<<plain_grid(c, n), 256, 0, c.stream>>>(opened.p, sig.as<int32_t>(), n, c.d_err);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
    op_scatter(c, xw, n, cc(x), Xt, sig.as<int32_t>());
    copy_sh(c, x, cc(Xt), n * xw);
}

void op_table_shuffle(Ctx& c, int w, size_t n, int na, const Sh3* data_a, int nb, const Sh3* data_b) {
    if (w != 4 && w != 8) throw std::invalid_argument("table shuffle supports 4 and 8-byte columns");
    // operators::shuffle(data_a, data_b, size) (shuffle.h:769-786): a random
    // elementwise permutation (the identity under a sharded permutation),
    // applied to every arithmetic column, then every boolean one
    ShardedPerm sp = next_perm(c, n);
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch pb(c, 3 * n1 * w);
    Sh3 P;
    for (int j = 0; j < 3; j++) P.p[j] = pb.as<uint8_t>() + j * n1 * w;
    if (n) {
        if (w == 4) k_identity<uint32_t><<<plain_grid(c, n), 256, 0, c.stream>>>(P, n);
        else k_identity<unsigned long long><<<plain_grid(c, n), 256, 0, c.stream>>>(P, n);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched++;
    }
    op_apply_sharded(c, false, w, n, P, sp, false);
    c.free_perm(sp);
    for (int k = 0; k < na; k++) apply_elementwise_bperm(c, true, w, n, data_a[k], cc(P), w);
    for (int k = 0; k < nb; k++) apply_elementwise_bperm(c, false, w, n, data_b[k], cc(P), w);
}

void op_mask_b(Ctx& c, int w, size_t n, Sh3 s, unsigned long long m) {
    if (!n) return;
    const unsigned g = plain_grid(c, n);
    if (w == 4) k_mask<uint32_t><<<g, 256, 0, c.stream>>>(s, n, (uint32_t)m);
    else if (w == 8) k_mask<unsigned long long><<<g, 256, 0, c.stream>>>(s, n, m);
    else throw std::invalid_argument("mask supports 4 and 8-byte shares");
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

void op_compose(Ctx& c, size_t n, Sh3 sigma, Sh3 rho) {
    ShardedPerm sp = next_perm(c, n);
    op_apply_sharded(c, true, 4, n, sigma, sp, false);
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch opened(c, n1 * 4), tmp(c, 3 * n1 * 4);
    op_open(c, true, 4, n, cc(sigma), opened.p);
    Sh3 T;
    for (int p = 0; p < 3; p++) T.p[p] = tmp.as<uint8_t>() + p * n1 * 4;
    if (n) {
        k_gather4<<<plain_grid(c, n), 256, 0, c.stream>>>(cc(rho), T, opened.as<int32_t>(), n, c.d_err);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched++;
    }
    copy_sh(c, rho, cc(T), n * 4);
    op_apply_sharded(c, true, 4, n, rho, sp, true);
    c.free_perm(sp);
}

void op_table_sort(Ctx& c, int w, size_t n, int ncols, const Sh3* cols, const int* desc,
                   const int* single_bit, int na, const Sh3* data_a, int nb, const Sh3* data_b, bool quick) {
    if (w != 4 && w != 8) throw std::invalid_argument("table sort supports 4 and 8-byte columns");
    if (ncols < 1) throw std::invalid_argument("table sort needs a key column");
    int ns = 0;
    for (int k = 0; k < ncols; k++) ns += single_bit[k] != 0;
    const int nk = ncols - ns, nc = na + nb, L = 8 * w;
    // PermutationManager::reserve(size, perms, pairs): for 3PC pairs are
    // single permutations too. Quicksort needs an extra permutation per
    // multi-bit key (its shuffle), radix sort an extra pair per bit.
    const size_t perms = (size_t)(nk + ns - 1) + (size_t)(nk + ns) + (quick ? (size_t)nk : 0);
    const size_t pairs = (size_t)(4 * ns + 3 * nk + nc - 1) + (quick ? 0 : (size_t)nk * L);
    reserve_perms(c, n, perms + pairs);
    // sort_sub (sorting.h:565-576): single-bit columns by a 1-bit radix sort
    auto sort_sub = [&](int k, Sh3 perm) {
        if (single_bit[k]) op_radix_sort(c, w, n, cols[k], 1, desc[k] != 0, perm);
        else if (quick) op_quicksort(c, w, n, cols[k], desc[k] != 0, perm);
        else op_radix_sort(c, w, n, cols[k], L, desc[k] != 0, perm);
    };
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch origb(c, 3 * n1 * w), spb(c, 3 * n1 * 4), npb(c, 3 * n1 * 4);
    Sh3 orig, sp, np;
    for (int p = 0; p < 3; p++) {
        orig.p[p] = origb.as<uint8_t>() + p * n1 * w;
        sp.p[p] = spb.as<uint8_t>() + p * n1 * 4;
        np.p[p] = npb.as<uint8_t>() + p * n1 * 4;
    }
    int C = ncols - 1;
    copy_sh(c, orig, cc(cols[C]), n * w);
    sort_sub(C, sp);
    copy_sh(c, cols[C], cc(orig), n * w);
    for (C--; C >= 0; C--) {
        copy_sh(c, orig, cc(cols[C]), n * w);
        op_apply_elementwise(c, false, w, n, cols[C], cc(sp));
        sort_sub(C, np);
        copy_sh(c, cols[C], cc(orig), n * w);
        op_compose(c, n, sp, np);
        std::swap(sp, np);
    }
    for (int k = 0; k < ncols; k++) op_apply_elementwise(c, false, w, n, cols[k], cc(sp));
    for (int k = 0; k < na; k++) op_apply_elementwise(c, true, w, n, data_a[k], cc(sp));
    for (int k = 0; k < nb; k++) op_apply_elementwise(c, false, w, n, data_b[k], cc(sp));
}

void op_distinct(Ctx& c, int w, size_t n, int nkeys, const CSh3* keys, Sh3 res) {
    if (w != 4 && w != 8) throw std::invalid_argument("distinct supports 4 and 8-byte keys");
    if (nkeys < 1 || nkeys > kMaxDistinctKeys) throw std::invalid_argument("distinct takes 1 to 8 key columns");
    if (n == 0) return;
    const unsigned long long m = n - 1;
    DistinctArgs a{};
    for (int j = 0; j < nkeys; j++)
        for (int p = 0; p < 3; p++) a.key[j][p] = keys[j].p[p];
    for (int p = 0; p < 3; p++) a.res[p] = res.p[p];
    a.nkeys = nkeys;
    a.m = m;
    a.C = chunks_of(m * w);
    for (int q = 0; q < 3; q++) a.pair[q] = c.stream_arg(PAIR0 + q);
    const int L = (w == 4) ? 5 : 6;
    const unsigned long long units = ceil_div(m * w, 16);
    const double calls = (double)nkeys * (L + 1);
    const double bytes = 3.0 * w * (2.0 * nkeys * m + n);
    if (w == 4) launch_aes(c, "distinct", bytes, 3.0 * calls * units, k_distinct<4>, std::max(units, 1ull), a);
    else launch_aes(c, "distinct", bytes, 3.0 * calls * units, k_distinct<8>, std::max(units, 1ull), a);
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (unsigned long long)nkeys * (L + 1) * a.C;
}

}  // namespace orqcu
