// conv.cu — ASharedVector::a2b (a_shared_vector.h:138-144): the arithmetic
// sharing is redistributed as two boolean sharings (redistribute_shares_b,
// replicated_3pc.h:259-262: party 0 shares S0 + S1, party 2 shares S2) whose
// sum, computed by the boolean ripple-carry adder (operators/circuits.h:35-76),
// is the boolean sharing of the value.
//
// The adder works on bit-packed words: bit i of 8W consecutive elements forms
// one word (pack_from), and each of the 8W-1 carry rounds is one AND over the
// ceil(n / 8W) words, c_i = ((c_{i-1} ^ a_i) & (a ^ b)_i) ^ a_i. Here a warp
// owns the words of one keystream block (k_rca); a ballot packs a bit of 32
// elements, and the sum bits are unpacked back into the lanes' elements, all
// rounds in registers.
#include <type_traits>

#include "launch.cuh"

namespace orqcu {

namespace {

struct RcaArgs {
    const void* a[3];
    const void* b[3];
    void* sum[3];
    StreamArg pair[3];     // nonces at the first carry round
    unsigned long long n;  // elements
    unsigned long long cw; // packed words (ceil(n / 8W))
    unsigned long long C;  // nonces per carry round (an AND over cw words)
    int carry_in;          // subtraction: the carry starts as all ones (inplace_invert)
};

// A warp owns the WPW = 16 / W consecutive packed words that one keystream
// block of a carry round covers (4 words of 32 elements for int32, 2 of 64
// for int64); lane l holds element 32h + l of each of them (four elements a
// lane). Before the rounds, the warp computes every keystream block it needs
// once, spread over the lanes: stream q's block of round i is computed by
// lane i % 32 into slot q * RPL + i / 32; round i then takes it by shuffle.
template <int W>
__global__ void __launch_bounds__(kAesThreads, 1) k_rca(RcaArgs a) {
    using T = typename std::conditional<W == 4, uint32_t, unsigned long long>::type;
    constexpr int B = 8 * W;              // elements per packed word
    constexpr int H = B / 32;             // elements per lane and word
    constexpr int WPW = 16 / W;           // words per warp (one keystream block)
    constexpr int RPL = (B - 1 + 31) / 32;  // rounds per lane and stream
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const int lane = threadIdx.x & 31;
    const unsigned long long groups = (a.cw + WPW - 1) / WPW;
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
    for (unsigned long long gi = (unsigned long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
         gi < groups; gi += warps) {
        const unsigned long long c0 = gi * WPW;
        // keystream of all rounds: ks[q * RPL + r] = stream q, round 32 r + lane
        uint4 ks[3 * RPL];
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int r = 0; r < RPL; r++) {
                const int i = 32 * r + lane;
                ks[q * RPL + r] = make_uint4(0, 0, 0, 0);
                if (i < B - 1)
                    ks[q * RPL + r] = keystream_block_n(S, a.pair[q].rk, a.pair[q].nonce + (unsigned long long)i * a.C,
                                                        c0 * W / 16);
            }
        T x[WPW][H][3], ab[WPW][H][3], sum[WPW][H][3];
#pragma unroll
        for (int j = 0; j < WPW; j++)
#pragma unroll
            for (int h = 0; h < H; h++) {
                const unsigned long long e = (c0 + j) * B + 32ull * h + lane;
                const bool ok = e < a.n;
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    x[j][h][p] = ok ? reinterpret_cast<const T*>(a.a[p])[e] : (T)0;
                    ab[j][h][p] = x[j][h][p] ^ (ok ? reinterpret_cast<const T*>(a.b[p])[e] : (T)0);
                    sum[j][h][p] = 0;
                }
            }
        const T cin = a.carry_in ? ~(T)0 : (T)0;
        T carry[WPW][3];
#pragma unroll
        for (int j = 0; j < WPW; j++) carry[j][0] = carry[j][1] = carry[j][2] = cin;
#pragma unroll 1
        for (int i = 0; i < B; i++) {
            // this round's keystream words: block of stream q from lane i % 32
            uint32_t kb[3][4];
            if (i < B - 1) {
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    uint4 blk = ks[q * RPL];
                    if constexpr (RPL > 1) {
                        if (i >= 32) blk = ks[q * RPL + 1];
                    }
                    kb[q][0] = __shfl_sync(0xffffffffu, blk.x, i & 31);
                    kb[q][1] = __shfl_sync(0xffffffffu, blk.y, i & 31);
                    kb[q][2] = __shfl_sync(0xffffffffu, blk.z, i & 31);
                    kb[q][3] = __shfl_sync(0xffffffffu, blk.w, i & 31);
                }
            }
#pragma unroll
            for (int j = 0; j < WPW; j++) {
                T axb[3], ai[3];
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    axb[p] = ai[p] = 0;
#pragma unroll
                    for (int h = 0; h < H; h++) {
                        axb[p] |= (T)__ballot_sync(0xffffffffu, (ab[j][h][p] >> i) & 1) << (32 * h);
                        ai[p] |= (T)__ballot_sync(0xffffffffu, (x[j][h][p] >> i) & 1) << (32 * h);
                    }
                }
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const T s = axb[p] ^ carry[j][p];
#pragma unroll
                    for (int h = 0; h < H; h++) sum[j][h][p] |= ((s >> (32 * h + lane)) & 1) << i;
                }
                if (i == B - 1) continue;  // no carry out of the top bit
                // word c0 + j of each stream's round-i draw: W bytes at j*W of the block
                T K[3];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    if constexpr (W == 4) K[q] = (T)kb[q][j];
                    else K[q] = (T)(((unsigned long long)kb[q][2 * j + 1] << 32) | kb[q][2 * j]);
                }
                // c_i = ((c ^ a_i) & axb_i) ^ a_i, the AND with r_p = K[p-1] ^ K[p]
                T u[3], z[3];
#pragma unroll
                for (int p = 0; p < 3; p++) u[p] = carry[j][p] ^ ai[p];
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const int q = (p + 1) % 3, pm = (p + 2) % 3;
                    z[p] = (K[pm] ^ K[p]) ^ (u[p] & axb[p]) ^ (u[p] & axb[q]) ^ (u[q] & axb[p]);
                }
#pragma unroll
                for (int p = 0; p < 3; p++) carry[j][p] = z[p] ^ ai[p];
            }
        }
#pragma unroll
        for (int j = 0; j < WPW; j++)
#pragma unroll
            for (int h = 0; h < H; h++) {
                const unsigned long long e = (c0 + j) * B + 32ull * h + lane;
                if (e < a.n) {
#pragma unroll
                    for (int p = 0; p < 3; p++) reinterpret_cast<T*>(a.sum[p])[e] = sum[j][h][p];
                }
            }
    }
}

// S0 + S1 (party 0's local value x(0) + x(1)) mod 2^(8W)
template <typename T>
__global__ void k_add01(CSh3 x, T* out, unsigned long long n) {
    for (unsigned long long i = gtid(); i < n; i += gstride())
        out[i] = reinterpret_cast<const T*>(x.p[0])[i] + reinterpret_cast<const T*>(x.p[1])[i];
}

}  // namespace

// ripple_carry_adder (operators/circuits.h:35-76) of two boolean sharings
void op_rca(Ctx& c, int w, size_t n, CSh3 A, CSh3 Bv, Sh3 sum, bool carry_in) {
    if (w != 4 && w != 8) throw std::invalid_argument("the boolean adder supports 4 and 8-byte shares");
    const unsigned long long B = 8ull * w, cw = (n + B - 1) / B;
    RcaArgs a;
    for (int j = 0; j < 3; j++) {
        a.a[j] = A.p[j];
        a.b[j] = Bv.p[j];
        a.sum[j] = sum.p[j];
        a.pair[j] = c.stream_arg(PAIR0 + j);
    }
    a.n = n;
    a.cw = cw;
    a.C = chunks_of(cw * (unsigned long long)w);
    a.carry_in = carry_in;
    if (n) {
        // one warp per 16 / W words; each computes 3 (B - 1) blocks
        const unsigned long long groups = (cw + 16 / w - 1) / (16 / w);
        const double blocks = 3.0 * (double)(B - 1) * (double)groups;
        if (w == 4) launch_aes(c, "boolean_adder", 9.0 * w * n, blocks, k_rca<4>, groups * 32, a);
        else launch_aes(c, "boolean_adder", 9.0 * w * n, blocks, k_rca<8>, groups * 32, a);
    }
    for (int q = 0; q < 3; q++) c.nonce[PAIR0 + q] += (B - 1) * a.C;
}

// BSharedVector::operator- (b_shared_vector.h:620-622): a + ~b + 1
void op_sub_b(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 z) {
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch nb(c, 3 * n1 * w);
    Sh3 NY;
    for (int j = 0; j < 3; j++) NY.p[j] = nb.as<uint8_t>() + j * n1 * w;
    op_not(c, w, n, y, NY);
    op_rca(c, w, n, x, CSh3{{NY.p[0], NY.p[1], NY.p[2]}}, z, true);
}

void op_a2b(Ctx& c, int w, size_t n, CSh3 x, Sh3 y) {
    if (w != 4 && w != 8) throw std::invalid_argument("a2b supports 4 and 8-byte shares");
    const size_t n1 = std::max<size_t>(n, 1);
    Scratch v(c, n1 * w), fb(c, 3 * n1 * w), sb(c, 3 * n1 * w);
    Sh3 F, G;
    for (int j = 0; j < 3; j++) {
        F.p[j] = fb.as<uint8_t>() + j * n1 * w;
        G.p[j] = sb.as<uint8_t>() + j * n1 * w;
    }
    if (n) {
        if (w == 4) k_add01<uint32_t><<<plain_grid(c, n), 256, 0, c.stream>>>(x, v.as<uint32_t>(), n);
        else k_add01<unsigned long long><<<plain_grid(c, n), 256, 0, c.stream>>>(x, v.as<unsigned long long>(), n);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched++;
    }
    // redistribute_shares_b: party 0 shares x(0) + x(1), then party 2 its x(0)
    op_secret_share(c, false, w, n, v.p, 0, F);
    op_secret_share(c, false, w, n, x.p[2], 2, G);
    op_rca(c, w, n, CSh3{{F.p[0], F.p[1], F.p[2]}}, CSh3{{G.p[0], G.p[1], G.p[2]}}, y, false);
}

}  // namespace orqcu
