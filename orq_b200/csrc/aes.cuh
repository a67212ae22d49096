// aes.cuh — AES-256 keystream on sm_100a, laid out for ORQ's PRG.
//
// ORQ's AESPRGAlgorithm (include/core/random/prg/prg_algorithm.h:161-231) fills
// a buffer by AES-256-GCM-encrypting zeros in 1 MiB chunks; chunk c uses the
// 96-bit IV (nonce0 + c as 8 little-endian bytes, then 4 zero bytes) and, as
// GCM specifies (NIST SP 800-38D), block j of the chunk is
// AES_K(IV || BE32(j + 2)). Byte o of a stream draw is therefore keystream
// block (o >> 4) of chunk (o >> 20), an affine function of the element index:
// every thread can produce exactly the keystream its elements need.
//
// Implementation: the 32-bit "T-table" formulation of the AES round (FIPS-197
// §5.1 SubBytes+ShiftRows+MixColumns folded into four 256-entry tables).
// Tables live in shared memory replicated once per lane (entry x of table t
// for lane l at word  region(t)*16384 + x*64 + (t&1)*32 + l), so every lookup
// of a warp hits 32 distinct banks whatever the byte values are. The byte
// extraction and the lane offset fuse into one byte-permute: the lookup
// address is (byte << 8) | (lane << 2). Round keys come from kernel parameters
// (constant bank), so AddRoundKey costs no loads.
#pragma once
#include <cstdint>

namespace orqcu {

struct AesRK {
    uint32_t k[60];  // FIPS-197 key schedule, word i = key-schedule bytes 4i..4i+3 (LE)
};

// One PRG stream as a kernel sees it: key schedule + nonce of its first chunk.
struct StreamArg {
    AesRK rk;
    unsigned long long nonce;
};

constexpr int kAesSmemBytes = 2 * 256 * 256;  // 4 tables x 256 entries x 32 lanes x 4 B

// Global copy of T0..T3 (4 x 256 words). Each translation unit that launches
// AES kernels owns one copy (no device linking); common.cuh registers an
// uploader per unit and the runtime fills every copy once per device.
static __device__ uint32_t g_aes_T[4 * 256];

// The 32 lane copies of one entry are 128 contiguous bytes; a thread writes 4
// of them with one 128-bit store, so a quarter-warp store phase covers one
// 128-byte row (conflict-free) and each global word is read by 8 threads.
__device__ __forceinline__ void aes_stage_tables(uint32_t* sm) {
    constexpr int kStores = 4 * 256 * 8;
    for (int base = 0; base < kStores; base += 16 * blockDim.x) {
        uint32_t v[16];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int idx = base + u * blockDim.x + threadIdx.x;
            v[u] = idx < kStores ? __ldg(&g_aes_T[idx >> 3]) : 0u;
        }
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int idx = base + u * blockDim.x + threadIdx.x;
            if (idx < kStores) {
                const int e = idx >> 3, t = e >> 8, x = e & 255;
                reinterpret_cast<uint4*>(sm + (t >> 1) * 16384 + x * 64 + (t & 1) * 32)[idx & 7] =
                    make_uint4(v[u], v[u], v[u], v[u]);
            }
        }
    }
    __syncthreads();
}

struct AesSmem {
    const char* base;  // shared base + lane*4 folded into the permute, see lk()
    uint32_t lane4;
    __device__ __forceinline__ explicit AesSmem(const uint32_t* sm)
        : base(reinterpret_cast<const char*>(sm)), lane4((threadIdx.x & 31u) << 2) {}
    // table t, byte j of word w
    template <int T, int J>
    __device__ __forceinline__ uint32_t lk(uint32_t w) const {
        const uint32_t a = __byte_perm(w, lane4, 0x5504u | (J << 4));
        return *reinterpret_cast<const uint32_t*>(base + a + (T >> 1) * 65536 + (T & 1) * 128);
    }
};

// Encrypt one block (4 little-endian column words) in place.
__device__ __forceinline__ void aes256_encrypt(const AesSmem& S, const AesRK& rk, uint32_t& s0,
                                               uint32_t& s1, uint32_t& s2, uint32_t& s3) {
    s0 ^= rk.k[0];
    s1 ^= rk.k[1];
    s2 ^= rk.k[2];
    s3 ^= rk.k[3];
#pragma unroll
    for (int r = 1; r < 14; r++) {
        const uint32_t n0 = S.lk<0, 0>(s0) ^ S.lk<1, 1>(s1) ^ S.lk<2, 2>(s2) ^ S.lk<3, 3>(s3) ^ rk.k[4 * r + 0];
        const uint32_t n1 = S.lk<0, 0>(s1) ^ S.lk<1, 1>(s2) ^ S.lk<2, 2>(s3) ^ S.lk<3, 3>(s0) ^ rk.k[4 * r + 1];
        const uint32_t n2 = S.lk<0, 0>(s2) ^ S.lk<1, 1>(s3) ^ S.lk<2, 2>(s0) ^ S.lk<3, 3>(s1) ^ rk.k[4 * r + 2];
        const uint32_t n3 = S.lk<0, 0>(s3) ^ S.lk<1, 1>(s0) ^ S.lk<2, 2>(s1) ^ S.lk<3, 3>(s2) ^ rk.k[4 * r + 3];
        s0 = n0;
        s1 = n1;
        s2 = n2;
        s3 = n3;
    }
    // last round: S-box bytes read out of the T tables (T2 byte0, T3 byte1,
    // T0 byte2 and T1 byte3 all hold S[x])
    const uint32_t n0 = (S.lk<2, 0>(s0) & 0xffu) | (S.lk<3, 1>(s1) & 0xff00u) |
                        (S.lk<0, 2>(s2) & 0xff0000u) | (S.lk<1, 3>(s3) & 0xff000000u);
    const uint32_t n1 = (S.lk<2, 0>(s1) & 0xffu) | (S.lk<3, 1>(s2) & 0xff00u) |
                        (S.lk<0, 2>(s3) & 0xff0000u) | (S.lk<1, 3>(s0) & 0xff000000u);
    const uint32_t n2 = (S.lk<2, 0>(s2) & 0xffu) | (S.lk<3, 1>(s3) & 0xff00u) |
                        (S.lk<0, 2>(s0) & 0xff0000u) | (S.lk<1, 3>(s1) & 0xff000000u);
    const uint32_t n3 = (S.lk<2, 0>(s3) & 0xffu) | (S.lk<3, 1>(s0) & 0xff00u) |
                        (S.lk<0, 2>(s1) & 0xff0000u) | (S.lk<1, 3>(s2) & 0xff000000u);
    s0 = n0 ^ rk.k[56];
    s1 = n1 ^ rk.k[57];
    s2 = n2 ^ rk.k[58];
    s3 = n3 ^ rk.k[59];
}

// Keystream block `blk` of a draw that starts at nonce `nonce0` of the stream
// keyed by rk.
__device__ __forceinline__ uint4 keystream_block_n(const AesSmem& S, const AesRK& rk,
                                                   unsigned long long nonce0, unsigned long long blk) {
    const unsigned long long nonce = nonce0 + (blk >> 16);
    uint32_t s0 = (uint32_t)nonce, s1 = (uint32_t)(nonce >> 32), s2 = 0u;
    uint32_t s3 = __byte_perm((uint32_t)(blk & 0xffffu) + 2u, 0, 0x0123);
    aes256_encrypt(S, rk, s0, s1, s2, s3);
    return make_uint4(s0, s1, s2, s3);
}

// Keystream block `blk` (16-byte unit) of a draw that starts at nonce `nonce0`.
__device__ __forceinline__ uint4 keystream_block(const AesSmem& S, const StreamArg& st,
                                                 unsigned long long blk) {
    const unsigned long long nonce = st.nonce + (blk >> 16);
    uint32_t s0 = (uint32_t)nonce, s1 = (uint32_t)(nonce >> 32), s2 = 0u;
    uint32_t s3 = __byte_perm((uint32_t)(blk & 0xffffu) + 2u, 0, 0x0123);
    aes256_encrypt(S, st.rk, s0, s1, s2, s3);
    return make_uint4(s0, s1, s2, s3);
}

}  // namespace orqcu
