// common.cuh — shared helpers for the ORQ loopback kernels.
//
// A 3PC shared vector of n elements of W bytes is three device arrays S[0..2]
// (the distinct shares; party p holds S[p], S[(p+1)%3]). Kernels work on
// 16-byte units because one AES block of a PRG stream covers exactly 16 bytes
// of the elements it randomises.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "aes.cuh"

namespace orqcu {

#define ORQ_CUDA_CHECK(expr)                                                              \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess)                                                            \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + \
                                     " at " __FILE__ ":" + std::to_string(__LINE__));     \
    } while (0)

typedef unsigned __int128 u128;

// Registry of per-translation-unit AES table uploaders (see aes.cuh).
typedef void (*AesTableUploader)(const uint32_t* T);
int register_aes_table_uploader(AesTableUploader f);
namespace {
inline void upload_tables_of_this_unit(const uint32_t* T) {
    ORQ_CUDA_CHECK(cudaMemcpyToSymbol(g_aes_T, T, 4 * 256 * sizeof(uint32_t)));
}
[[maybe_unused]] const int k_aes_tables_registered =
    register_aes_table_uploader(&upload_tables_of_this_unit);
}  // namespace

// Shares of one vector, as raw device pointers.
struct Sh3 {
    void* p[3];
};
struct CSh3 {
    const void* p[3];
};

__host__ __device__ inline unsigned long long ceil_div(unsigned long long a, unsigned long long b) {
    return (a + b - 1) / b;
}

// Number of AES nonces one getNext(Vector<T>) of nbytes consumes
// (1 MiB chunks, prg_algorithm.h:161-172).
__host__ __device__ inline unsigned long long chunks_of(unsigned long long nbytes) {
    return (nbytes + (1ull << 20) - 1) >> 20;
}

// ---- 16-byte unit load/store with a ragged tail --------------------------
__device__ __forceinline__ uint4 ld16(const void* base, unsigned long long blk,
                                      unsigned long long nbytes) {
    const unsigned long long off = blk << 4;
    const uint8_t* p = reinterpret_cast<const uint8_t*>(base) + off;
    if (off + 16 <= nbytes && ((reinterpret_cast<uintptr_t>(p) & 15) == 0))
        return __ldg(reinterpret_cast<const uint4*>(p));
    union {
        uint4 v;
        uint8_t b[16];
    } u;
    u.v = make_uint4(0, 0, 0, 0);
    const unsigned long long lim = nbytes > off ? (nbytes - off < 16 ? nbytes - off : 16) : 0;
    for (unsigned i = 0; i < lim; i++) u.b[i] = p[i];
    return u.v;
}

__device__ __forceinline__ void st16(void* base, unsigned long long blk, unsigned long long nbytes,
                                     uint4 v) {
    const unsigned long long off = blk << 4;
    uint8_t* p = reinterpret_cast<uint8_t*>(base) + off;
    if (off + 16 <= nbytes && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
        *reinterpret_cast<uint4*>(p) = v;
        return;
    }
    union {
        uint4 v;
        uint8_t b[16];
    } u;
    u.v = v;
    const unsigned long long lim = nbytes > off ? (nbytes - off < 16 ? nbytes - off : 16) : 0;
    for (unsigned i = 0; i < lim; i++) p[i] = u.b[i];
}

__device__ __forceinline__ uint4 operator^(uint4 a, uint4 b) {
    return make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
}
__device__ __forceinline__ uint4 operator&(uint4 a, uint4 b) {
    return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w);
}

// ---- lane-wise ring arithmetic on a 16-byte unit holding 16/W elements ----
template <int W>
struct Ring;

template <>
struct Ring<1> {
    static __device__ __forceinline__ uint32_t mulw(uint32_t a, uint32_t b) {
        uint32_t r = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) r |= (((a >> (8 * k)) * (b >> (8 * k))) & 0xffu) << (8 * k);
        return r;
    }
    static __device__ __forceinline__ uint4 add(uint4 a, uint4 b) {
        return make_uint4(__vadd4(a.x, b.x), __vadd4(a.y, b.y), __vadd4(a.z, b.z), __vadd4(a.w, b.w));
    }
    static __device__ __forceinline__ uint4 sub(uint4 a, uint4 b) {
        return make_uint4(__vsub4(a.x, b.x), __vsub4(a.y, b.y), __vsub4(a.z, b.z), __vsub4(a.w, b.w));
    }
    static __device__ __forceinline__ uint4 mul(uint4 a, uint4 b) {
        return make_uint4(mulw(a.x, b.x), mulw(a.y, b.y), mulw(a.z, b.z), mulw(a.w, b.w));
    }
};
template <>
struct Ring<2> {
    static __device__ __forceinline__ uint32_t mulw(uint32_t a, uint32_t b) {
        return ((a * b) & 0xffffu) | (((a >> 16) * (b >> 16)) << 16);
    }
    static __device__ __forceinline__ uint4 add(uint4 a, uint4 b) {
        return make_uint4(__vadd2(a.x, b.x), __vadd2(a.y, b.y), __vadd2(a.z, b.z), __vadd2(a.w, b.w));
    }
    static __device__ __forceinline__ uint4 sub(uint4 a, uint4 b) {
        return make_uint4(__vsub2(a.x, b.x), __vsub2(a.y, b.y), __vsub2(a.z, b.z), __vsub2(a.w, b.w));
    }
    static __device__ __forceinline__ uint4 mul(uint4 a, uint4 b) {
        return make_uint4(mulw(a.x, b.x), mulw(a.y, b.y), mulw(a.z, b.z), mulw(a.w, b.w));
    }
};
template <>
struct Ring<4> {
    static __device__ __forceinline__ uint4 add(uint4 a, uint4 b) {
        return make_uint4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
    }
    static __device__ __forceinline__ uint4 sub(uint4 a, uint4 b) {
        return make_uint4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
    }
    static __device__ __forceinline__ uint4 mul(uint4 a, uint4 b) {
        return make_uint4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
    }
};
__device__ __forceinline__ unsigned long long lo64(uint4 a) {
    return (unsigned long long)a.x | ((unsigned long long)a.y << 32);
}
__device__ __forceinline__ unsigned long long hi64(uint4 a) {
    return (unsigned long long)a.z | ((unsigned long long)a.w << 32);
}
__device__ __forceinline__ uint4 mk4(unsigned long long lo, unsigned long long hi) {
    return make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}
template <>
struct Ring<8> {
    static __device__ __forceinline__ uint4 add(uint4 a, uint4 b) {
        return mk4(lo64(a) + lo64(b), hi64(a) + hi64(b));
    }
    static __device__ __forceinline__ uint4 sub(uint4 a, uint4 b) {
        return mk4(lo64(a) - lo64(b), hi64(a) - hi64(b));
    }
    static __device__ __forceinline__ uint4 mul(uint4 a, uint4 b) {
        return mk4(lo64(a) * lo64(b), hi64(a) * hi64(b));
    }
};
template <>
struct Ring<16> {
    static __device__ __forceinline__ u128 w(uint4 a) { return ((u128)hi64(a) << 64) | lo64(a); }
    static __device__ __forceinline__ uint4 v(u128 x) {
        return mk4((unsigned long long)x, (unsigned long long)(x >> 64));
    }
    static __device__ __forceinline__ uint4 add(uint4 a, uint4 b) { return v(w(a) + w(b)); }
    static __device__ __forceinline__ uint4 sub(uint4 a, uint4 b) { return v(w(a) - w(b)); }
    static __device__ __forceinline__ uint4 mul(uint4 a, uint4 b) { return v(w(a) * w(b)); }
};

// Binary (XOR) or arithmetic (+ mod 2^8W) combination used by zero-sharings.
template <int W, bool ARITH>
struct Share {
    static __device__ __forceinline__ uint4 plus(uint4 a, uint4 b) {
        if constexpr (ARITH) return Ring<W>::add(a, b);
        else return a ^ b;
    }
    static __device__ __forceinline__ uint4 minus(uint4 a, uint4 b) {
        if constexpr (ARITH) return Ring<W>::sub(a, b);
        else return a ^ b;
    }
    static __device__ __forceinline__ uint4 times(uint4 a, uint4 b) {
        if constexpr (ARITH) return Ring<W>::mul(a, b);
        else return a & b;
    }
};

}  // namespace orqcu
