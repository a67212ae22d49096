// radix.cu — ORQ's shuffle-based oblivious radix sort on the loopback runtime.
//
// Restates orq::operators::radix_sort (include/core/operators/radixsort.h:
// 116-229) with pad_input / remove_padding (operators/sorting.h:405-495) and
// ElementwisePermutation::b2a / invert (containers/permutation.h:205-258),
// calling the same protocol steps in the same order so every PRG stream is
// consumed exactly as the reference consumes it. Per sorted bit:
//   1. k_radix_b2a   bit (32+i) of every padded share -> b2a_bit        (1 pass)
//   2. k_scan_*      inclusive scan of s = [1 - f1, f1] with s[0] -= 1  (3 passes)
//   3. k_radix_perm  t = s0 + f1 * (s1 - s0)  (multiply_a + add_a)      (1 pass)
//   4. op_apply_elementwise(padded, t)        (3 passes, one per group)
#include <algorithm>
#include <functional>
#include <numeric>
#include <vector>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr int kScanTile = 4096;  // elements per scan tile (256 threads x 16)

struct RadixB2AArgs {
    const void* P[3];   // padded key shares (PW bytes per element)
    void* f1[3];        // out: A-shared int32
    StreamArg pair[3];
    unsigned long long chunks;  // nonces per getNext of n int32
    unsigned long long n;
    uint32_t shift;
    uint32_t invert;
};

// bit_arithmetic_right_shift(v, 32+i) [+ inplace_invert], copy-cast to int32
// and b2a_bit, fused. b2a_bit only looks at the LSB of every share, which is
// bit (32+i) of the padded share (the shift never reaches the sign fill for
// bits <= 64).
template <int PW>
__global__ void __launch_bounds__(kAesThreads) k_radix_b2a(RadixB2AArgs a) {
    using R = Ring<4>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long units = ceil_div(a.n, 4);
    const uint32_t wsel = a.shift >> 5, bsel = a.shift & 31;
    const unsigned long long nbytes = a.n * 4;
    for (unsigned long long b = gtid(); b < units; b += gstride()) {
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
        uint32_t x[3][4];
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const unsigned long long i = b * 4 + e;
                uint32_t w = 0;
                if (i < a.n)
                    w = __ldg(reinterpret_cast<const uint32_t*>(a.P[j]) + i * (PW / 4) + wsel);
                x[j][e] = ((w >> bsel) ^ a.invert) & 1u;
            }
        const uint4 abit = make_uint4(x[0][0] ^ x[1][0], x[0][1] ^ x[1][1], x[0][2] ^ x[1][2],
                                      x[0][3] ^ x[1][3]);
        const uint4 bbit = make_uint4(x[2][0], x[2][1], x[2][2], x[2][3]);
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
            st16(a.f1[p], b, nbytes, v);
        }
    }
}

// s_j[i] for i in [0, 2n): first half 1 - f1 (the public one sits in S0) with
// s[0] -= 1 on S0, second half f1.
__device__ __forceinline__ uint32_t s_val(const uint32_t* f1, int j, unsigned long long i,
                                          unsigned long long n) {
    if (i < n) {
        uint32_t v = (j == 0 ? 1u : 0u) - __ldg(f1 + i);
        if (j == 0 && i == 0) v -= 1u;
        return v;
    }
    return __ldg(f1 + (i - n));
}

struct ScanArgs {
    const uint32_t* f1[3];
    uint32_t* sc[3];       // out: inclusive scan, 2n per share
    uint32_t* tsum;        // [3][tiles]
    unsigned long long n;  // 2n elements are scanned
    uint32_t tiles;
};

__global__ void __launch_bounds__(256) k_scan_up(ScanArgs a) {
    __shared__ uint32_t red[33];
    const int j = blockIdx.y;
    const unsigned long long m = 2 * a.n;
    for (uint32_t t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        uint32_t s = 0;
        for (int u = 0; u < kScanTile / 256; u++) {
            const unsigned long long i = (unsigned long long)t * kScanTile + u * 256 + threadIdx.x;
            if (i < m) s += s_val(a.f1[j], j, i, a.n);
        }
        uint32_t tot;
        block_excl_sum(s, red, tot);
        if (threadIdx.x == 0) a.tsum[(size_t)j * a.tiles + t] = tot;
    }
}

__global__ void __launch_bounds__(1024) k_scan_mid(ScanArgs a) {
    __shared__ uint32_t red[33];
    const int j = blockIdx.x;
    uint32_t* ts = a.tsum + (size_t)j * a.tiles;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < a.tiles; b0 += 1024) {
        const uint32_t k = b0 + threadIdx.x;
        const uint32_t v = k < a.tiles ? ts[k] : 0;
        uint32_t tot;
        const uint32_t pre = block_excl_sum(v, red, tot);
        if (k < a.tiles) ts[k] = carry + pre;
        carry += tot;
    }
}

__global__ void __launch_bounds__(256) k_scan_down(ScanArgs a) {
    __shared__ uint32_t red[33];
    const int j = blockIdx.y;
    const unsigned long long m = 2 * a.n;
    constexpr int PER = kScanTile / 256;
    for (uint32_t t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        // thread owns PER consecutive elements
        const unsigned long long base = (unsigned long long)t * kScanTile + threadIdx.x * PER;
        uint32_t v[PER], s = 0;
#pragma unroll
        for (int u = 0; u < PER; u++) {
            v[u] = (base + u < m) ? s_val(a.f1[j], j, base + u, a.n) : 0u;
            s += v[u];
        }
        uint32_t tot;
        uint32_t pre = block_excl_sum(s, red, tot) + a.tsum[(size_t)j * a.tiles + t];
#pragma unroll
        for (int u = 0; u < PER; u++) {
            pre += v[u];
            if (base + u < m) a.sc[j][base + u] = pre;
        }
    }
}

struct PermMulArgs {
    const uint32_t* f1[3];
    const uint32_t* sc[3];
    void* t[3];
    StreamArg pair[3];
    unsigned long long n;
};

// s1 -= s0 ; f1 *= s1 (multiply_a) ; s0 += f1  (radixsort.h:183-185)
__global__ void __launch_bounds__(kAesThreads) k_radix_perm(PermMulArgs a) {
    using R = Ring<4>;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long units = ceil_div(a.n, 4), nbytes = a.n * 4;
    for (unsigned long long b = gtid(); b < units; b += gstride()) {
        const uint4 k0 = keystream_block(S, a.pair[0], b);
        const uint4 k1 = keystream_block(S, a.pair[1], b);
        const uint4 k2 = keystream_block(S, a.pair[2], b);
        const uint4 r[3] = {R::sub(k2, k0), R::sub(k0, k1), R::sub(k1, k2)};
        uint4 x[3], y[3], s0[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            x[j] = ld16(a.f1[j], b, nbytes);
            uint32_t lo[4], hi[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const unsigned long long i = b * 4 + e;
                lo[e] = i < a.n ? __ldg(a.sc[j] + i) : 0u;
                hi[e] = i < a.n ? __ldg(a.sc[j] + a.n + i) : 0u;
            }
            s0[j] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            y[j] = R::sub(make_uint4(hi[0], hi[1], hi[2], hi[3]), s0[j]);
        }
#pragma unroll
        for (int p = 0; p < 3; p++) {
            const int q = (p + 1) % 3;
            uint4 v = R::add(r[p], R::mul(x[p], y[p]));
            v = R::add(v, R::mul(x[p], y[q]));
            v = R::add(v, R::mul(x[q], y[p]));
            st16(a.t[p], b, nbytes, R::add(s0[p], v));
        }
    }
}

// pad_input (sorting.h:431-462): (v << 32) | index, index public-shared into
// S0 only (P0 and P2 hold it); v is sign-extended to the padded width.
// Descending (reverse_order): the index is -1-i and the padded vector is
// reversed, so row i lands at position n-1-i.
template <int KW, int PW>
__global__ void k_pad(CSh3 key, Sh3 P, unsigned long long n, int desc) {
    for (unsigned long long i0 = gtid(); i0 < n; i0 += gstride()) {
        const unsigned long long i = desc ? n - 1 - i0 : i0;  // destination
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const uint32_t idx = j == 0 ? (desc ? (uint32_t)(-1ll - (long long)i0) : (uint32_t)i0) : 0u;
            if constexpr (KW == 8) {
                const long long v = reinterpret_cast<const long long*>(key.p[j])[i0];
                const unsigned long long lo = ((unsigned long long)v << 32) | idx;
                const unsigned long long hi = (unsigned long long)(v >> 32);  // sign fill
                reinterpret_cast<uint4*>(P.p[j])[i] = mk4(lo, hi);
            } else {
                const int v = reinterpret_cast<const int*>(key.p[j])[i0];
                const unsigned long long p = ((unsigned long long)(long long)v << 32) | idx;
                reinterpret_cast<unsigned long long*>(P.p[j])[i] = p;
            }
        }
    }
}

// remove_padding (sorting.h:475-495): low 32 bits -> B-shared permutation,
// arithmetic shift by 32 -> the key.
// Descending: the padded vector is reversed back first (row i reads n-1-i).
template <int KW, int PW>
__global__ void k_unpad(CSh3 P, Sh3 key, Sh3 perm, unsigned long long n, int desc) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        const unsigned long long src = desc ? n - 1 - i : i;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if constexpr (PW == 16) {
                const uint4 v = reinterpret_cast<const uint4*>(P.p[j])[src];
                reinterpret_cast<uint32_t*>(perm.p[j])[i] = v.x;
                const unsigned long long k = (unsigned long long)v.y | ((unsigned long long)v.z << 32);
                reinterpret_cast<unsigned long long*>(key.p[j])[i] = k;
            } else {
                const unsigned long long v = reinterpret_cast<const unsigned long long*>(P.p[j])[src];
                reinterpret_cast<uint32_t*>(perm.p[j])[i] = (uint32_t)v;
                reinterpret_cast<uint32_t*>(key.p[j])[i] = (uint32_t)(v >> 32);
            }
        }
    }
}

__global__ void k_iota(int32_t* out, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) out[i] = (int32_t)i;
}

// public_share of the constant -1 (S0 = -1, S1 = S2 = 0)
__global__ void k_minus_one(Sh3 m, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        reinterpret_cast<int32_t*>(m.p[0])[i] = -1;
        reinterpret_cast<int32_t*>(m.p[1])[i] = 0;
        reinterpret_cast<int32_t*>(m.p[2])[i] = 0;
    }
}

}  // namespace

// The frame both sort protocols share (radix_sort, radixsort.h:205-229, and
// quicksort, quicksort.h:214-246): pad_input, the protocol's body on the
// padded rows, remove_padding (permutation b2a, negate for descending order)
// and invert. `reserve` is the number of permutations the body and the frame
// take from the PermutationManager queue, reserved up front.
void sort_padded(Ctx& c, int kw, size_t n, Sh3 key, bool desc, Sh3 perm_out, size_t reserve,
                 const std::function<void(Sh3 P, int PW)>& body) {
    if (kw != 4 && kw != 8) throw std::invalid_argument("sort keys must be int32 or int64");
    if (n >= (1ull << 31)) throw std::invalid_argument("sorts support n < 2^31");
    const int PW = kw == 8 ? 16 : 8;
    reserve_perms(c, n, reserve);

    Scratch Pbuf(c, 3 * std::max<size_t>(n, 1) * PW);
    Sh3 P;
    for (int j = 0; j < 3; j++) P.p[j] = Pbuf.as<uint8_t>() + j * n * (size_t)PW;
    const unsigned pg = plain_grid(c, n);
    if (n) {
        CSh3 k{{key.p[0], key.p[1], key.p[2]}};
        if (kw == 8) k_pad<8, 16><<<pg, 256, 0, c.stream>>>(k, P, n, desc);
        else k_pad<4, 8><<<pg, 256, 0, c.stream>>>(k, P, n, desc);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched++;
    }
    body(P, PW);
    const size_t n1 = std::max<size_t>(n, 1);

    // remove_padding: permutation = low 32 bits (B-shared), key = padded >> 32
    Scratch pm(c, 3 * n1 * 4);
    Sh3 PM;
    for (int j = 0; j < 3; j++) PM.p[j] = pm.as<uint8_t>() + j * n1 * 4;
    if (n) {
        CSh3 Pc{{P.p[0], P.p[1], P.p[2]}};
        if (kw == 8) k_unpad<8, 16><<<pg, 256, 0, c.stream>>>(Pc, key, PM, n, desc);
        else k_unpad<4, 8><<<pg, 256, 0, c.stream>>>(Pc, key, PM, n, desc);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched++;
    }

    // ElementwisePermutation::b2a (permutation.h:222-258): shuffle a copy with
    // pi, open it, public-share it arithmetically, un-apply pi.
    {
        ShardedPerm sp = next_perm(c, n);
        Scratch pcb(c, 3 * n1 * 4), sig(c, n1 * 4);
        Sh3 PC;
        for (int j = 0; j < 3; j++) {
            PC.p[j] = pcb.as<uint8_t>() + j * n1 * 4;
            if (n)
                ORQ_CUDA_CHECK(cudaMemcpyAsync(PC.p[j], PM.p[j], n * 4, cudaMemcpyDeviceToDevice, c.stream));
        }
        op_apply_sharded(c, false, 4, n, PC, sp, false);
        op_open(c, false, 4, n, CSh3{{PC.p[0], PC.p[1], PC.p[2]}}, sig.p);
        op_public_share(c, 4, n, sig.p, PM);
        op_apply_sharded(c, true, 4, n, PM, sp, true);
        c.free_perm(sp);
    }
    // negate (permutation.h:268-280) for descending sorts: v *= -1 (a
    // multiply_a with the public -1), v += -1
    if (desc) {
        Scratch mb(c, 3 * n1 * 4);
        Sh3 M1;
        for (int j = 0; j < 3; j++) M1.p[j] = mb.as<uint8_t>() + j * n1 * 4;
        if (n) {
            k_minus_one<<<pg, 256, 0, c.stream>>>(M1, n);
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched++;
        }
        const CSh3 m1c{{M1.p[0], M1.p[1], M1.p[2]}};
        op_mult(c, true, 4, n, CSh3{{PM.p[0], PM.p[1], PM.p[2]}}, m1c, PM);
        op_local(c, 1, 4, n, CSh3{{PM.p[0], PM.p[1], PM.p[2]}}, m1c, PM);
    }
    // invert (permutation.h:205-213): apply the permutation to a public identity
    {
        Scratch inv(c, 3 * n1 * 4);
        Sh3 I;
        for (int j = 0; j < 3; j++) I.p[j] = inv.as<uint8_t>() + j * n1 * 4;
        if (n) {
            k_iota<<<pg, 256, 0, c.stream>>>((int32_t*)I.p[0], n);
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched++;
        }
        op_public_share(c, 4, n, I.p[0], I);
        op_apply_elementwise(c, true, 4, n, I, CSh3{{PM.p[0], PM.p[1], PM.p[2]}});
        for (int j = 0; j < 3; j++)
            if (n)
                ORQ_CUDA_CHECK(cudaMemcpyAsync(perm_out.p[j], I.p[j], n * 4, cudaMemcpyDeviceToDevice, c.stream));
    }
}

void op_radix_sort(Ctx& c, int kw, size_t n, Sh3 key, int bits, bool desc, Sh3 perm_out) {
    if (kw != 4 && kw != 8) throw std::invalid_argument("radix sort keys must be int32 or int64");
    if (bits < 1 || bits > kw * 8) throw std::invalid_argument("bits out of range");
    const bool full_width = (kw * 8 == bits);
    // radix_sort_body: 1 permutation for remove_padding + (bits + 1) pairs
    sort_padded(c, kw, n, key, desc, perm_out, (size_t)bits + 2, [&](Sh3 P, int PW) {
        const size_t n1 = std::max<size_t>(n, 1);
        Scratch f1b(c, 3 * n1 * 4), scb(c, 3 * 2 * n1 * 4), tb(c, 3 * n1 * 4);
        const uint32_t tiles = (uint32_t)ceil_div(2 * n1, kScanTile);
        Scratch tsb(c, 3 * (size_t)tiles * 4);
        uint32_t* f1[3];
        uint32_t* sc[3];
        uint32_t* t[3];
        for (int j = 0; j < 3; j++) {
            f1[j] = f1b.as<uint32_t>() + j * n1;
            sc[j] = scb.as<uint32_t>() + j * 2 * n1;
            t[j] = tb.as<uint32_t>() + j * n1;
        }
        const unsigned long long ch4 = chunks_of((unsigned long long)n * 4);

        for (int b = 0; b < bits; b++) {
            if (n) {
                RadixB2AArgs ba;
                for (int j = 0; j < 3; j++) {
                    ba.P[j] = P.p[j];
                    ba.f1[j] = f1[j];
                    ba.pair[j] = c.stream_arg(PAIR0 + j);
                }
                ba.chunks = ch4;
                ba.n = n;
                ba.shift = 32 + b;
                ba.invert = (full_width && b == bits - 1) ? 1u : 0u;
                const double by = 24.0 * n, bl = 9.0 * ceil_div(n, 4);
                if (PW == 16) launch_aes(c, "radix_bit_b2a", by, bl, k_radix_b2a<16>, ceil_div(n, 4), ba);
                else launch_aes(c, "radix_bit_b2a", by, bl, k_radix_b2a<8>, ceil_div(n, 4), ba);
            }
            for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += 3 * ch4;

            if (n) {
                ScanArgs sa;
                for (int j = 0; j < 3; j++) {
                    sa.f1[j] = f1[j];
                    sa.sc[j] = sc[j];
                }
                sa.tsum = tsb.as<uint32_t>();
                sa.n = n;
                sa.tiles = tiles;
                const dim3 grid(std::min<uint32_t>(tiles, (uint32_t)c.num_sms * 8), 3);
                {
                    ProfScope ps(c, "radix_scan", 72.0 * n);
                    k_scan_up<<<grid, 256, 0, c.stream>>>(sa);
                    k_scan_mid<<<3, 1024, 0, c.stream>>>(sa);
                    k_scan_down<<<grid, 256, 0, c.stream>>>(sa);
                }
                ORQ_CUDA_CHECK(cudaGetLastError());
                c.kernels_launched += 3;

                PermMulArgs pa;
                for (int j = 0; j < 3; j++) {
                    pa.f1[j] = f1[j];
                    pa.sc[j] = sc[j];
                    pa.t[j] = t[j];
                    pa.pair[j] = c.stream_arg(PAIR0 + j);
                }
                pa.n = n;
                launch_aes(c, "radix_perm_mul", 48.0 * n, 3.0 * ceil_div(n, 4), k_radix_perm, ceil_div(n, 4), pa);
            }
            for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += ch4;

            CSh3 tp{{t[0], t[1], t[2]}};
            op_apply_elementwise(c, false, PW, n, P, tp);
        }
    });
}

// ---------------------------------------------------------------------------
// Batched radix sorts: `count` items in list order, the shares of `count`
// plain calls. Items run back to back on the runtime's stream with no host
// synchronisation between them (a plain call ends with one). Overlapping item
// k's bit passes with item k+1's Fisher-Yates chain is allowed by the PRG
// order (the chain only needs nonces the host knows once item k's chain has
// ended) and was measured: on a second stream, with or without a static SM
// split, it made the ragged batch slower (both halves want every SM for AES,
// and the data side's CTAs delay the scanner launches the chain waits on).
void op_radix_sort_batch(Ctx& c, int kw, int count, const size_t* n, void* const* keys, const int* bits,
                         const int* desc, void* const* perms_out) {
    if (count <= 0) return;
    for (int k = 0; k < count; k++) {
        if (kw != 4 && kw != 8) throw std::invalid_argument("radix sort keys must be int32 or int64");
        if (bits[k] < 1 || bits[k] > kw * 8) throw std::invalid_argument("bits out of range");
        if (n[k] >= (1ull << 31)) throw std::invalid_argument("sorts support n < 2^31");
    }
    for (int k = 0; k < count; k++) {
        Sh3 key{{keys[3 * k], keys[3 * k + 1], keys[3 * k + 2]}};
        Sh3 po{{perms_out[3 * k], perms_out[3 * k + 1], perms_out[3 * k + 2]}};
        op_radix_sort(c, kw, n[k], key, bits[k], desc[k] != 0, po);
    }
    c.check_device_error();
}

}  // namespace orqcu
