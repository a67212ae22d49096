// scan.cu — inclusive prefix sum of arithmetic shares.
//
// SharedVector::prefix_sum (include/core/containers/shared_vector.h:249) scans
// each party's share columns locally (addition is linear, no communication);
// in loopback that is an inclusive scan mod 2^(8W) of each distinct share array
// S[0], S[1], S[2]. Reduce-then-scan over 4096-element tiles: per-tile sums,
// a scan of the tile sums per share, then each tile rescanned with its offset.
#include <memory>
#include <mutex>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr int kTile = 4096;
constexpr int kThreads = 256;
constexpr int kPer = kTile / kThreads;

template <typename T>
__device__ __forceinline__ T block_excl_sum_t(T v, T* red, T& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) red[wid] = x;
    __syncthreads();
    if (wid == 0) {
        T t = lane < nw ? red[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        red[lane] = t;
    }
    __syncthreads();
    const T base = wid ? red[wid - 1] : T(0);
    total = red[nw - 1];
    __syncthreads();
    return base + x - v;
}

template <typename T>
struct ScanArgs3 {
    T* s[3];
    T* tsum;  // [3][tiles]
    unsigned long long n;
    uint32_t tiles;
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_up(ScanArgs3<T> a) {
    __shared__ T red[32];
    const int j = blockIdx.y;
    for (uint32_t t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        T s = 0;
        for (int u = 0; u < kPer; u++) {
            const unsigned long long i = (unsigned long long)t * kTile + u * kThreads + threadIdx.x;
            if (i < a.n) s += a.s[j][i];
        }
        T tot;
        block_excl_sum_t<T>(s, red, tot);
        if (threadIdx.x == 0) a.tsum[(size_t)j * a.tiles + t] = tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_mid(ScanArgs3<T> a) {
    __shared__ T red[32];
    T* ts = a.tsum + (size_t)blockIdx.x * a.tiles;
    T carry = 0;
    for (uint32_t b0 = 0; b0 < a.tiles; b0 += 1024) {
        const uint32_t k = b0 + threadIdx.x;
        const T v = k < a.tiles ? ts[k] : T(0);
        T tot;
        const T pre = block_excl_sum_t<T>(v, red, tot);
        if (k < a.tiles) ts[k] = carry + pre;
        carry += tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_down(ScanArgs3<T> a) {
    __shared__ T red[32];
    const int j = blockIdx.y;
    for (uint32_t t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        const unsigned long long base = (unsigned long long)t * kTile + threadIdx.x * kPer;
        T v[kPer], s = 0;
#pragma unroll
        for (int u = 0; u < kPer; u++) {
            v[u] = base + u < a.n ? a.s[j][base + u] : T(0);
            s += v[u];
        }
        T tot;
        T pre = block_excl_sum_t<T>(s, red, tot) + a.tsum[(size_t)j * a.tiles + t];
#pragma unroll
        for (int u = 0; u < kPer; u++) {
            pre += v[u];
            if (base + u < a.n) a.s[j][base + u] = pre;
        }
    }
}

template <typename T>
void run_scan(Ctx& c, size_t n, Sh3 s, T* tsum, uint32_t tiles, bool profile = true) {
    ScanArgs3<T> a;
    for (int j = 0; j < 3; j++) a.s[j] = reinterpret_cast<T*>(s.p[j]);
    a.tsum = tsum;
    a.n = n;
    a.tiles = tiles;
    const dim3 grid(std::min<uint32_t>(tiles, (uint32_t)c.num_sms * 8), 3);
    std::unique_ptr<ProfScope> ps;
    if (profile) ps.reset(new ProfScope(c, "prefix_sum", 3.0 * 3.0 * n * sizeof(T)));
    k_up<T><<<grid, kThreads, 0, c.stream>>>(a);
    k_mid<T><<<3, 1024, 0, c.stream>>>(a);
    k_down<T><<<grid, kThreads, 0, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched += 3;
}

}  // namespace

uint32_t prefix_sum_tiles(size_t n) { return (uint32_t)ceil_div(n ? n : 1, kTile); }

// Tile sums live in `tsum` (3 * prefix_sum_tiles(n) words of W bytes).
void op_prefix_sum_into(Ctx& c, int w, size_t n, Sh3 s, void* tsum) {
    if (n == 0) return;
    const uint32_t tiles = prefix_sum_tiles(n);
    if (w == 4) run_scan<uint32_t>(c, n, s, reinterpret_cast<uint32_t*>(tsum), tiles);
    else if (w == 8) run_scan<unsigned long long>(c, n, s, reinterpret_cast<unsigned long long*>(tsum), tiles);
    else throw std::invalid_argument("prefix sum supports 4 and 8-byte shares");
}

// ---------------------------------------------------------------------------
// Prefix sum without any device allocation.
//
// Some callers cannot allocate device memory at the moment they call us: a
// host program that reserved the GPU's memory up front for its own pool (so a
// cudaMalloc would fail or break its budget), or a service loop that must not
// pay cudaMalloc's implicit device-wide synchronisation while other requests
// are running. For them the tile sums live in this fixed array instead of the
// runtime's pool. It holds 3 x 16384 tile sums of 8 bytes (384 KiB per device,
// kept until the process exits), which limits a call to 2^26 elements. Every
// call reuses the same array, so two such calls must not run at the same time
// on the GPU (different streams included): their tile sums would mix. Each
// call writes every tile sum it reads, so nothing needs clearing between calls.
constexpr size_t kNoAllocMaxElems = size_t(1) << 26;
constexpr size_t kNoAllocTiles = kNoAllocMaxElems / kTile;
static __device__ __align__(256) unsigned long long g_noalloc_tsum[3 * kNoAllocTiles];

// Device address of g_noalloc_tsum on `device`, looked up once per device with
// that device current (host code may not pass the symbol itself to a kernel).
// The address is remembered with the device's epoch: once the last runtime on
// the device is destroyed (after which the context may have been reset and
// the array moved) the next call looks it up again.
static void* noalloc_scratch(int device) {
    static std::mutex mu;
    static void* ptrs[kMaxDevices] = {};
    static unsigned long long epoch[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lk(mu);
    const unsigned long long ep = device_epoch(device);
    if (ptrs[device] && epoch[device] == ep) return ptrs[device];
    int cur = -1;
    ORQ_CUDA_CHECK(cudaGetDevice(&cur));
    if (cur != device) throw std::runtime_error("the runtime's device is not the current device");
    void* p = nullptr;
    ORQ_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_tsum));
    ptrs[device] = p;
    epoch[device] = ep;
    return p;
}

void op_prefix_sum_noalloc(Ctx& c, int w, size_t n, Sh3 s) {
    if (w != 4 && w != 8) throw std::invalid_argument("prefix sum supports 4 and 8-byte shares");
    if (n > kNoAllocMaxElems)
        throw std::invalid_argument("orqcu_prefix_sum_a_noalloc handles at most 2^26 elements per call");
    if (n == 0) return;
    void* ts = noalloc_scratch(c.device);
    const uint32_t tiles = prefix_sum_tiles(n);
    if (w == 4) run_scan<uint32_t>(c, n, s, reinterpret_cast<uint32_t*>(ts), tiles, false);
    else run_scan<unsigned long long>(c, n, s, reinterpret_cast<unsigned long long*>(ts), tiles, false);
}

void op_prefix_sum(Ctx& c, int w, size_t n, Sh3 s) {
    if (n == 0) return;
    if (w != 4 && w != 8) throw std::invalid_argument("prefix sum supports 4 and 8-byte shares");
    // released to the pool right away: later users of the buffer run on the
    // same stream, after these kernels
    Scratch ts(c, 3 * (size_t)prefix_sum_tiles(n) * w);
    op_prefix_sum_into(c, w, n, s, ts.p);
}

}  // namespace orqcu
