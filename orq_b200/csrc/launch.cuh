// launch.cuh — launch helpers shared by the kernel files.
#pragma once
#include "runtime.h"

namespace orqcu {

constexpr int kAesThreads = 512;

__device__ __forceinline__ unsigned long long gtid() {
    return (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ unsigned long long gstride() {
    return (unsigned long long)gridDim.x * blockDim.x;
}

inline unsigned aes_grid(const Ctx& c, unsigned long long units, int reserve_sms = 0) {
    unsigned long long g = ceil_div(units ? units : 1, kAesThreads);
    unsigned long long cap = (unsigned long long)(c.num_sms - reserve_sms);
    return (unsigned)(g < cap ? g : cap);
}
inline unsigned plain_grid(const Ctx& c, unsigned long long units, int threads = 256) {
    unsigned long long g = ceil_div(units ? units : 1, threads);
    unsigned long long cap = (unsigned long long)c.num_sms * 16;
    return (unsigned)(g < cap ? g : cap);
}

template <typename K>
inline void prep_aes_kernel(K kern) {
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kAesSmemBytes));
}

// Launch an AES kernel over `units` thread work items; name/bytes/blocks feed
// the optional per-kernel profile.
template <typename K, typename... Args>
inline void launch_aes(Ctx& c, const char* name, double bytes, double aes_blocks, K kern,
                       unsigned long long units, Args... args) {
    prep_aes_kernel(kern);
    ProfScope ps(c, name, bytes, aes_blocks);
    kern<<<aes_grid(c, units), kAesThreads, kAesSmemBytes, c.stream>>>(args...);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

#define ORQ_DISPATCH_W(w, ...)                                                              \
    switch (w) {                                                                             \
        case 1: { constexpr int W = 1; __VA_ARGS__; } break;                                        \
        case 2: { constexpr int W = 2; __VA_ARGS__; } break;                                        \
        case 4: { constexpr int W = 4; __VA_ARGS__; } break;                                        \
        case 8: { constexpr int W = 8; __VA_ARGS__; } break;                                        \
        case 16: { constexpr int W = 16; __VA_ARGS__; } break;                                      \
        default: throw std::invalid_argument("share width must be 1, 2, 4, 8 or 16 bytes");  \
    }

// Block-wide exclusive sum for blockDim.x <= 1024; `red` is >= 33 words of smem.
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t v, uint32_t* red, uint32_t& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) red[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < nw ? red[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        red[lane] = t;  // inclusive warp prefix
    }
    __syncthreads();
    const uint32_t warp_base = wid ? red[wid - 1] : 0u;
    total = red[nw - 1];
    __syncthreads();
    return warp_base + x - v;
}

}  // namespace orqcu
