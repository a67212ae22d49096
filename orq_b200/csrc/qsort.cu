// qsort.cu — quicksort (include/core/operators/quicksort.h:61-246) on the
// device.
//
// quicksort_body shuffles the padded rows, then repeats rounds: every row that
// is not a pivot is compared with the pivot heading its segment (_compare on
// the padded width, then opened), and every segment is partitioned by the
// Lomuto loop of partition (quicksort.h:28-49), after which the pivot's final
// position and the position right after it (the pivot of the right part) are
// pivots too. Rows' shares are only moved, never recomputed, but the next
// round's segments (and so the sizes of its compares, i.e. the PRG nonces they
// consume) follow from the exact Lomuto arrangement, so it is reproduced
// exactly, in closed form. For a segment [h, h+len] with opened bits c_1..c_len
// at relative positions (c = 0: row <= pivot), Z zeros, and Z_t the zeros
// among 1..t:
//  * relative 0 receives the last zero (the pivot itself when Z = 0),
//    relative 1..Z-1 the zeros in order, relative Z the pivot;
//  * relative t > Z receives W(t): row t when c_t = 1, else W(Z_t) — Lomuto
//    swaps the row at the front of its "greater" run into position t when the
//    zero at t arrives, and no later swap reaches a position beyond Z.
// A round is: a scan for segment heads and the ranks of the non-pivots, a
// gather of the compared rows, the compare and open, a scan of the zero
// flags, and one gather that moves every row to its new position.
#include <algorithm>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr int kQsThreads = 1024;
constexpr int kQsPer = 4;  // consecutive positions per thread in the scans
constexpr uint32_t kQsChunk = kQsThreads * kQsPer;

struct QsRound {
    uint32_t n, chunks;
    int32_t* piv;    // [n] q at pivot positions, -1 elsewhere
    int32_t* head;   // [n] segment head: the largest pivot position <= q
    uint32_t* idx;   // [n] positions of the non-pivots, in order
    uint8_t* cb;     // [n] opened comparison bit at each non-pivot position
    uint32_t* gz;    // [n] zeros (non-pivots with bit 0) at positions <= q
    uint32_t* zseg;  // [n] at a segment head: zeros in the segment
    uint32_t* send;  // [n] at a segment head: last position of the segment
    uint32_t* zpos;  // [n] at h + k: position of segment h's k-th zero
    uint32_t* psum;  // [chunks] chunk sums, then their exclusive scan
    int32_t* pmax;   // [chunks] chunk maxima, then their exclusive prefix max
    uint32_t* npiv;  // pivot count
    int* err;
};

// Block-wide exclusive scans of a sum and a max (-1 as the max identity);
// tot_s / tot_m are the block totals. rs / rm hold at least 32 words.
__device__ __forceinline__ void block_scan2(uint32_t s, int32_t m, uint32_t* rs, int32_t* rm, uint32_t& ex_s,
                                            int32_t& ex_m, uint32_t& tot_s, int32_t& tot_m) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t is = s;
    int32_t im = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t ys = __shfl_up_sync(0xffffffffu, is, o);
        const int32_t ym = __shfl_up_sync(0xffffffffu, im, o);
        if (lane >= o) {
            is += ys;
            im = max(im, ym);
        }
    }
    int32_t xm = __shfl_up_sync(0xffffffffu, im, 1);
    if (lane == 0) xm = -1;
    if (lane == 31) {
        rs[wid] = is;
        rm[wid] = im;
    }
    __syncthreads();
    if (wid == 0) {
        uint32_t ts = lane < nw ? rs[lane] : 0u;
        int32_t tm = lane < nw ? rm[lane] : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ys = __shfl_up_sync(0xffffffffu, ts, o);
            const int32_t ym = __shfl_up_sync(0xffffffffu, tm, o);
            if (lane >= o) {
                ts += ys;
                tm = max(tm, ym);
            }
        }
        rs[lane] = ts;
        rm[lane] = tm;
    }
    __syncthreads();
    ex_s = is - s + (wid ? rs[wid - 1] : 0u);
    ex_m = max(xm, wid ? rm[wid - 1] : -1);
    tot_s = rs[nw - 1];
    tot_m = rm[nw - 1];
    __syncthreads();  // rs / rm are reused by the caller's next scan
}

// MODE 0: (non-pivots, max pivot) per chunk; MODE 1: zeros per chunk
template <int MODE>
__global__ void __launch_bounds__(kQsThreads) k_qs_part(QsRound a) {
    __shared__ uint32_t rs[32];
    __shared__ int32_t rm[32];
    const size_t base = (size_t)blockIdx.x * kQsChunk + (size_t)threadIdx.x * kQsPer;
    uint32_t s = 0;
    int32_t m = -1;
#pragma unroll
    for (int u = 0; u < kQsPer; u++) {
        const size_t q = base + u;
        if (q < a.n) {
            const int32_t p = a.piv[q];
            if (MODE == 0) {
                s += p < 0;
                m = max(m, p);
            } else {
                s += p < 0 && a.cb[q] == 0;
            }
        }
    }
    uint32_t es, ts;
    int32_t em, tm;
    block_scan2(s, m, rs, rm, es, em, ts, tm);
    if (threadIdx.x == 0) {
        a.psum[blockIdx.x] = ts;
        a.pmax[blockIdx.x] = tm;
    }
}

// exclusive scans of the chunk sums and maxima (one CTA)
__global__ void __launch_bounds__(kQsThreads) k_qs_top(QsRound a) {
    __shared__ uint32_t rs[32];
    __shared__ int32_t rm[32];
    uint32_t cs = 0;
    int32_t cm = -1;
    for (uint32_t b0 = 0; b0 < a.chunks; b0 += kQsThreads) {
        const uint32_t k = b0 + threadIdx.x;
        const uint32_t s = k < a.chunks ? a.psum[k] : 0u;
        const int32_t m = k < a.chunks ? a.pmax[k] : -1;
        uint32_t es, ts;
        int32_t em, tm;
        block_scan2(s, m, rs, rm, es, em, ts, tm);
        if (k < a.chunks) {
            a.psum[k] = cs + es;
            a.pmax[k] = max(cm, em);
        }
        cs += ts;
        cm = max(cm, tm);
    }
}

// segment heads (running max of pivot positions) and the non-pivots' positions
__global__ void __launch_bounds__(kQsThreads) k_qs_heads(QsRound a) {
    __shared__ uint32_t rs[32];
    __shared__ int32_t rm[32];
    const size_t base = (size_t)blockIdx.x * kQsChunk + (size_t)threadIdx.x * kQsPer;
    int32_t p[kQsPer];
    uint32_t s = 0;
    int32_t m = -1;
#pragma unroll
    for (int u = 0; u < kQsPer; u++) {
        p[u] = base + u < a.n ? a.piv[base + u] : 0;
        if (base + u < a.n) {
            s += p[u] < 0;
            m = max(m, p[u]);
        }
    }
    uint32_t es, ts;
    int32_t em, tm;
    block_scan2(s, m, rs, rm, es, em, ts, tm);
    uint32_t r = a.psum[blockIdx.x] + es;
    int32_t h = max(a.pmax[blockIdx.x], em);
#pragma unroll
    for (int u = 0; u < kQsPer; u++) {
        const size_t q = base + u;
        if (q >= a.n) break;
        h = max(h, p[u]);
        a.head[q] = h;
        if (p[u] < 0) a.idx[r++] = (uint32_t)q;
    }
}

// zeros up to and including each position
__global__ void __launch_bounds__(kQsThreads) k_qs_zeros(QsRound a) {
    __shared__ uint32_t rs[32];
    __shared__ int32_t rm[32];
    const size_t base = (size_t)blockIdx.x * kQsChunk + (size_t)threadIdx.x * kQsPer;
    uint32_t z[kQsPer], s = 0;
#pragma unroll
    for (int u = 0; u < kQsPer; u++) {
        const size_t q = base + u;
        z[u] = q < a.n && a.piv[q] < 0 && a.cb[q] == 0;
        s += z[u];
    }
    uint32_t es, ts;
    int32_t em, tm;
    block_scan2(s, -1, rs, rm, es, em, ts, tm);
    uint32_t g = a.psum[blockIdx.x] + es;
#pragma unroll
    for (int u = 0; u < kQsPer; u++) {
        const size_t q = base + u;
        if (q >= a.n) break;
        g += z[u];
        a.gz[q] = g;
    }
}

// rows compared this round: row idx[k] and the pivot heading its segment
template <int PW>
__global__ void k_qs_gather(QsRound a, CSh3 P, Sh3 R, Sh3 PV, uint32_t size) {
    using V = typename std::conditional<PW == 16, uint4, unsigned long long>::type;
    for (unsigned long long k = gtid(); k < size; k += gstride()) {
        const uint32_t q = a.idx[k];
        const uint32_t h = (uint32_t)a.head[q];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            reinterpret_cast<V*>(R.p[j])[k] = reinterpret_cast<const V*>(P.p[j])[q];
            reinterpret_cast<V*>(PV.p[j])[k] = reinterpret_cast<const V*>(P.p[j])[h];
        }
    }
}

// the opened comparison bit (LSB of the opened value) at its row's position
template <int PW>
__global__ void k_qs_bits(QsRound a, const uint8_t* opened, uint32_t size) {
    for (unsigned long long k = gtid(); k < size; k += gstride()) a.cb[a.idx[k]] = opened[k * PW] & 1u;
}

// segment totals at the heads, and each zero's position by rank
__global__ void k_qs_seg(QsRound a) {
    for (unsigned long long q = gtid(); q < a.n; q += gstride()) {
        const uint32_t h = (uint32_t)a.head[q];
        if (q + 1 == a.n || a.piv[q + 1] >= 0) {
            a.zseg[h] = a.gz[q] - a.gz[h];
            a.send[h] = (uint32_t)q;
        }
        if (a.piv[q] < 0 && a.cb[q] == 0) a.zpos[h + (a.gz[q] - a.gz[h])] = (uint32_t)q;
    }
}

// every row to its position after the round's partitions; new pivots marked
template <int PW>
__global__ void k_qs_move(QsRound a, CSh3 P, Sh3 NP) {
    using V = typename std::conditional<PW == 16, uint4, unsigned long long>::type;
    for (unsigned long long p = gtid(); p < a.n; p += gstride()) {
        const uint32_t h = (uint32_t)a.head[p];
        const uint32_t t = (uint32_t)p - h;
        const uint32_t len = a.send[h] - h, Z = a.zseg[h];
        uint32_t src = (uint32_t)p;
        if (len > 0) {
            if (t == 0) src = Z ? a.zpos[h + Z] : h;
            else if (t < Z) src = a.zpos[h + t];
            else if (t == Z) src = h;
            else {
                uint32_t f = t;  // W(t): follow zeros back to the run's front
                while (a.cb[h + f] == 0) {
                    const uint32_t r = a.gz[h + f] - a.gz[h];
                    if (r >= f) {  // a zero with only zeros before it: cannot sit past Z
                        atomicOr(a.err, 64);
                        break;
                    }
                    f = r;
                }
                src = h + f;
            }
            if (t == 0) {
                if (Z) a.piv[h + Z] = (int32_t)(h + Z);
                if (Z + 1 <= len) a.piv[h + Z + 1] = (int32_t)(h + Z + 1);
                const uint32_t added = (Z ? 1u : 0u) + (Z + 1 <= len ? 1u : 0u);
                if (added) atomicAdd(a.npiv, added);
            }
        }
#pragma unroll
        for (int j = 0; j < 3; j++)
            reinterpret_cast<V*>(NP.p[j])[p] = reinterpret_cast<const V*>(P.p[j])[src];
    }
}

template <int PW>
void quicksort_rounds(Ctx& c, size_t n, Sh3 P) {
    const uint32_t chunks = (uint32_t)ceil_div(n, (size_t)kQsChunk);
    Scratch pivb(c, n * 4), headb(c, n * 4), idxb(c, n * 4), cbb(c, n), gzb(c, n * 4), zsegb(c, n * 4),
        sendb(c, n * 4), zposb(c, n * 4), psb(c, chunks * 4), pmb(c, chunks * 4), npb(c, 4);
    Scratch npbuf(c, 3 * n * PW), rbuf(c, 3 * n * PW), pvbuf(c, 3 * n * PW), ebuf(c, 3 * n * PW),
        gbuf(c, 3 * n * PW), obuf(c, n * PW);
    QsRound a;
    a.n = (uint32_t)n;
    a.chunks = chunks;
    a.piv = pivb.as<int32_t>();
    a.head = headb.as<int32_t>();
    a.idx = idxb.as<uint32_t>();
    a.cb = cbb.as<uint8_t>();
    a.gz = gzb.as<uint32_t>();
    a.zseg = zsegb.as<uint32_t>();
    a.send = sendb.as<uint32_t>();
    a.zpos = zposb.as<uint32_t>();
    a.psum = psb.as<uint32_t>();
    a.pmax = pmb.as<int32_t>();
    a.npiv = npb.as<uint32_t>();
    a.err = c.d_err;
    auto split = [&](Scratch& b, size_t rows) {
        Sh3 s;
        for (int j = 0; j < 3; j++) s.p[j] = b.as<uint8_t>() + (size_t)j * rows * PW;
        return s;
    };
    auto cc = [](Sh3 s) { return CSh3{{s.p[0], s.p[1], s.p[2]}}; };
    Sh3 cur = P, nxt = split(npbuf, n);
    // pivots: position 0 only
    ORQ_CUDA_CHECK(cudaMemsetAsync(a.piv, 0xff, n * 4, c.stream));
    ORQ_CUDA_CHECK(cudaMemsetAsync(a.piv, 0, 4, c.stream));
    uint32_t num_pivots = 1;
    ORQ_CUDA_CHECK(cudaMemcpyAsync(a.npiv, &num_pivots, 4, cudaMemcpyHostToDevice, c.stream));
    const unsigned gg = plain_grid(c, n);
    for (size_t round = 0; num_pivots < n; round++) {
        if (round > 4 * n + 64) throw std::runtime_error("quicksort did not converge");
        const uint32_t size = (uint32_t)(n - num_pivots);
        Sh3 R = split(rbuf, size), PV = split(pvbuf, size), E = split(ebuf, size), G = split(gbuf, size);
        {
            ProfScope ps(c, "quicksort_round", 0.0);
            k_qs_part<0><<<chunks, kQsThreads, 0, c.stream>>>(a);
            k_qs_top<<<1, kQsThreads, 0, c.stream>>>(a);
            k_qs_heads<<<chunks, kQsThreads, 0, c.stream>>>(a);
            k_qs_gather<PW><<<plain_grid(c, size), 256, 0, c.stream>>>(a, cc(cur), R, PV, size);
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched += 4;
        }
        // reduced._compare(pivot): gt = row > pivot, opened
        op_compare(c, PW, size, cc(R), cc(PV), E, G);
        op_open(c, false, PW, size, cc(G), obuf.p);
        {
            ProfScope ps(c, "quicksort_round", 0.0);
            k_qs_bits<PW><<<plain_grid(c, size), 256, 0, c.stream>>>(a, obuf.as<uint8_t>(), size);
            k_qs_part<1><<<chunks, kQsThreads, 0, c.stream>>>(a);
            k_qs_top<<<1, kQsThreads, 0, c.stream>>>(a);
            k_qs_zeros<<<chunks, kQsThreads, 0, c.stream>>>(a);
            k_qs_seg<<<gg, 256, 0, c.stream>>>(a);
            k_qs_move<PW><<<gg, 256, 0, c.stream>>>(a, cc(cur), nxt);
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched += 6;
        }
        std::swap(cur, nxt);
        ORQ_CUDA_CHECK(cudaMemcpyAsync(&num_pivots, a.npiv, 4, cudaMemcpyDeviceToHost, c.stream));
        ORQ_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    }
    if (cur.p[0] != P.p[0])
        for (int j = 0; j < 3; j++)
            ORQ_CUDA_CHECK(cudaMemcpyAsync(P.p[j], cur.p[j], n * PW, cudaMemcpyDeviceToDevice, c.stream));
    c.check_device_error();
}

}  // namespace

void op_quicksort(Ctx& c, int kw, size_t n, Sh3 key, bool desc, Sh3 perm_out) {
    // 2 permutations (the shuffle, remove_padding's b2a) + 1 pair (invert)
    sort_padded(c, kw, n, key, desc, perm_out, 3, [&](Sh3 P, int PW) {
        op_shuffle(c, false, PW, n, P);  // quicksort_body: v.shuffle()
        if (n < 2) return;
        if (PW == 16) quicksort_rounds<16>(c, n, P);
        else quicksort_rounds<8>(c, n, P);
    });
}

}  // namespace orqcu
