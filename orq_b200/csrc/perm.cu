// perm.cu — sharded permutations: generation (Fisher–Yates from the group
// PRGs, bit-exact with ORQ) and their oblivious application fused with the
// group reshare.
//
// Generation restates gen_perm (include/core/random/permutations/
// hm_sharded_permutation_generator.h:70-108): draws are u32 words of the group
// stream taken from getNext buffers of 2^20 words (4 nonces each), reduced by
// mask = 2^bit_width(n) - 1; draw values above n-1-i are rejected; the i-th
// accepted value v gives swap(p[i], p[i+v]). A permutation starts on a fresh
// buffer, so consecutive permutations of one group form a chain whose start
// nonces depend on how many draws the previous one used.
//
// GPU design:
//  * fy_gen  (all SMs but three): AES keystream of a window of buffers; per
//    32768-draw tile, nested lists (in draw order) of the draws below n/4^L,
//    and the tile's last draw.
//  * fy_scan (one 1024-thread CTA per group): replays the sequential
//    acceptance exactly over the sparsest level that holds every candidate; an
//    entry is certainly accepted if v + (its index in the step) <= n-1-i,
//    certainly rejected if v > n-1-i, and the few in between are decided in
//    order by one warp. Windows are generated up to five ahead of the scans.
//  * fy_small (M <= 2^17, a predictable number of buffers per permutation):
//    every (permutation, group) in its own CTA at once from predicted start
//    buffers, re-run from the first wrong prediction until all are verified.
//  * fy_finalize: turns the accepted offsets into the final permutation in
//    parallel and writes its inverse.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "launch.cuh"

namespace orqcu {

namespace {

constexpr uint32_t kTileDraws = 32768;        // draws per tile
constexpr uint32_t kTileBlocks = kTileDraws / 4;
constexpr uint32_t kTilesPerRefill = (1u << 20) / kTileDraws;  // 32
constexpr int kGenThreads = 512;
constexpr int kBlocksPerThread = kTileBlocks / kGenThreads;     // 16 blocks = 64 draws
constexpr int kMaxLevels = 16;
constexpr int kScanThreads = 1024;
constexpr uint32_t kMaxWindowTiles = 1024;

// Level L of a tile keeps, in draw order, the draws with v < n >> 2L (level 0:
// every draw that can ever be accepted). Entries are (position << 32) | v.
__host__ __device__ inline uint32_t level_threshold(uint32_t n, int L) { return n >> (2 * L); }
__host__ inline uint32_t level_capacity(int L) {
    // twice the largest expected count (mask >= n) plus slack; overflow is
    // reported as an error, never truncated silently
    return L == 0 ? kTileDraws : ((kTileDraws >> (2 * L)) * 2 + 256);
}

struct FyState {
    unsigned long long start_tile;  // absolute tile where the current permutation starts
    uint32_t m;                     // index of the permutation being scanned
    uint32_t i;                     // accepted so far
    uint32_t done;
    uint32_t pad;
};

struct FyLayout {
    uint32_t nl;               // levels in use
    uint32_t off[kMaxLevels];  // entry offset of each level list inside a tile slot
    uint32_t cap[kMaxLevels];
    uint32_t slot;             // entries per tile slot
};

struct FyGenArgs {
    StreamArg st[3];  // nonce = chain start nonce + 4 * (window start buffer)
    uint32_t n, mask, tiles;
    FyLayout lay;
    uint32_t* ev;    // [3][tiles][slot] entry values v
    uint32_t* last;  // [3][tiles] masked value of each tile's last draw
    uint32_t* cnt;  // [3][tiles][kMaxLevels]
    const FyState* state;
    int* err;
};

constexpr int kHalfBlocks = kBlocksPerThread / 2;  // blocks per thread per half tile

__global__ void __launch_bounds__(kGenThreads, 1) k_fy_gen(FyGenArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t sdone;
    __shared__ uint32_t sbase[kMaxLevels];
    __shared__ uint32_t wsum[kGenThreads / 32][kMaxLevels / 2];  // per-warp packed level counts
    __shared__ uint32_t htot[kMaxLevels / 2];                    // half-tile totals
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const uint32_t total = 3 * a.tiles;
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const uint32_t g = item / a.tiles, tile = item % a.tiles;
        // the scanner may be updating the flag concurrently: read it once per CTA
        if (threadIdx.x == 0) sdone = *(volatile const uint32_t*)&a.state[g].done;
        if (threadIdx.x < kMaxLevels) sbase[threadIdx.x] = 0;
        __syncthreads();
        if (sdone) continue;
        const size_t slot = (size_t)g * a.tiles + tile;
        uint32_t* ov = a.ev + slot * a.lay.slot;
        for (int half = 0; half < 2; half++) {
            // this thread's 32 consecutive draws of the half tile
            uint32_t v[4 * kHalfBlocks];
            const uint32_t blk0 = half * (kTileBlocks / 2) + threadIdx.x * kHalfBlocks;
#pragma unroll
            for (int b = 0; b < kHalfBlocks; b++) {
                const uint4 ks = keystream_block(S, a.st[g], (unsigned long long)tile * kTileBlocks + blk0 + b);
                v[4 * b + 0] = ks.x & a.mask;
                v[4 * b + 1] = ks.y & a.mask;
                v[4 * b + 2] = ks.z & a.mask;
                v[4 * b + 3] = ks.w & a.mask;
            }
            if (half == 1 && threadIdx.x == kGenThreads - 1) a.last[slot] = v[4 * kHalfBlocks - 1];
            // every level at once (nested lists: level L keeps v < n >> 2L):
            // per-thread counts two levels per word (16-bit fields; half-tile
            // totals <= 16384), one block-wide scan for all of them
            constexpr int kPk = kMaxLevels / 2;
            uint32_t pc[kPk], ex[kPk];
#pragma unroll
            for (int j = 0; j < kPk; j++) pc[j] = 0;
#pragma unroll
            for (int L = 0; L < kMaxLevels; L++) {
                if (L < (int)a.lay.nl) {
                    const uint32_t th = level_threshold(a.n, L);
                    uint32_t c = 0;
#pragma unroll
                    for (int k = 0; k < 4 * kHalfBlocks; k++) c += v[k] < th;
                    pc[L >> 1] |= c << (16 * (L & 1));
                }
            }
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
            for (int j = 0; j < kPk; j++) {
                uint32_t inc = pc[j];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += y;
                }
                ex[j] = inc - pc[j];
                if (lane == 31) wsum[warp][j] = inc;
            }
            __syncthreads();
            if (threadIdx.x < kPk) {  // exclusive offsets of the warps, and the totals
                uint32_t run = 0;
                for (int w = 0; w < kGenThreads / 32; w++) {
                    const uint32_t t = wsum[w][threadIdx.x];
                    wsum[w][threadIdx.x] = run;
                    run += t;
                }
                htot[threadIdx.x] = run;
            }
            __syncthreads();
#pragma unroll
            for (int L = 0; L < kMaxLevels; L++) {
                if (L >= (int)a.lay.nl) break;
                const int sh = 16 * (L & 1);
                const uint32_t mine = (pc[L >> 1] >> sh) & 0xffffu;
                const uint32_t pre = ((ex[L >> 1] + wsum[warp][L >> 1]) >> sh) & 0xffffu;
                const uint32_t tt = (htot[L >> 1] >> sh) & 0xffffu;
                const uint32_t base = sbase[L];
                if (base + tt > a.lay.cap[L]) {
                    if (threadIdx.x == 0) atomicOr(a.err, 16);
                    continue;
                }
                if (mine) {
                    const uint32_t th = level_threshold(a.n, L);
                    uint32_t* olv = ov + a.lay.off[L] + base + pre;
                    uint32_t o = 0;
#pragma unroll
                    for (int k = 0; k < 4 * kHalfBlocks; k++)
                        if (v[k] < th) olv[o++] = v[k];
                }
            }
            __syncthreads();  // every thread has read sbase
            if (threadIdx.x < a.lay.nl) sbase[threadIdx.x] += (htot[threadIdx.x >> 1] >> (16 * (threadIdx.x & 1))) & 0xffffu;
            __syncthreads();
        }
        // an overflowing level was flagged above; its count is clamped so the
        // scanner never reads past the level's list
        if (threadIdx.x < a.lay.nl)
            a.cnt[slot * kMaxLevels + threadIdx.x] = min(sbase[threadIdx.x], a.lay.cap[threadIdx.x]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Small permutations (M = 2^bit_width(n) <= 2^17). A permutation then takes
// d ≈ M·H_n draws (std ≈ 1.3·M) and 1 + floor(d / 2^20) getNext buffers, a
// count that is predictable: permutation m of a group is assumed to start at
// buffer m·b̂ of the chain, and every (permutation, group) pair runs at once,
// one CTA each, with no host round trip. Warps 1.. generate the draws chunk
// by chunk into shared memory (two chunk buffers), warp 0 replays the
// acceptance 32 draws at a time (lane j is certainly accepted if v + j <= T,
// rejected if v > T, and the rest are decided in order) and reports the
// buffers the permutation used. The host then checks the assumed starts
// against the used counts; from the first permutation of a group whose start
// was wrong, the rest are run again from the corrected start (each pass
// fixes at least that one). A permutation needing more than `max_chunks`
// chunks sets `overflow`, and the general chain redoes everything.
constexpr uint32_t kSmallChunk = 8192;  // draws per chunk
constexpr int kSmallThreads = 512;
constexpr uint32_t kSmallMaxM = 1u << 17;
constexpr uint32_t kChunksPerBuffer = (1u << 20) / kSmallChunk;  // 128
constexpr size_t kSmallSmem = (size_t)kAesSmemBytes + 2 * kSmallChunk * 4;

struct FySmallArgs {
    StreamArg st[3];  // chain start of each group (buffer 0)
    uint32_t n, mask, count, max_chunks;
    uint32_t m0[3];        // per group, the first permutation to run
    const uint32_t* start;  // [3][count] assumed start buffer
    uint32_t* used;         // [3][count] buffers used
    uint32_t* acc;          // [count][3][n] accepted offsets v_i
    uint32_t* overflow;     // set when a permutation needs more than max_chunks
};

__global__ void __launch_bounds__(kSmallThreads, 1) k_fy_small(FySmallArgs a) {
    const uint32_t m = blockIdx.x / 3, g = blockIdx.x % 3;
    if (m < a.m0[g]) return;  // already verified (uniform per CTA)
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_dlast;
    aes_stage_tables(sm);
    const AesSmem S(sm);
    uint32_t* buf = sm + kAesSmemBytes / 4;  // [2][kSmallChunk]
    StreamArg st = a.st[g];
    st.nonce += 4ull * a.start[g * a.count + m];  // 4 nonces per buffer
    const uint32_t n = a.n;
    uint32_t* acc = a.acc + ((size_t)m * 3 + g) * n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t i = 0;  // accepted so far (warp 0)
    // iteration k produces chunk k into buf[k & 1] and consumes chunk k - 1
    // from buf[(k - 1) & 1]; the barrier that opens an iteration publishes
    // chunk k - 1, frees the buffer chunk k - 2 held, and stops every thread
    // at once when the permutation is complete
    for (uint32_t k = 0; k <= a.max_chunks; k++) {
        if (__syncthreads_or(warp == 0 && i >= n)) break;
        if (warp > 0) {
            if (k < a.max_chunks) {
                uint4* dst = reinterpret_cast<uint4*>(buf + (k & 1) * kSmallChunk);
                const unsigned long long blk0 = (unsigned long long)k * (kSmallChunk / 4);
                for (uint32_t b = threadIdx.x - 32; b < kSmallChunk / 4; b += kSmallThreads - 32) {
                    const uint4 ks = keystream_block(S, st, blk0 + b);
                    dst[b] = make_uint4(ks.x & a.mask, ks.y & a.mask, ks.z & a.mask, ks.w & a.mask);
                }
            }
        } else if (k > 0) {
            const uint32_t* src = buf + ((k - 1) & 1) * kSmallChunk;
            const uint32_t d0 = (k - 1) * kSmallChunk;  // draw index of the chunk's first draw
            // 128 draws at a time (lane l holds draws 32u + l): T only
            // decreases, so a group with no draw <= T now has no acceptance
            // and is skipped whole (most groups, late in a permutation)
            for (uint32_t base = 0; base < kSmallChunk && i < n; base += 128) {
                uint32_t v4[4];
#pragma unroll
                for (int u = 0; u < 4; u++) v4[u] = src[base + 32u * u + lane];
                const uint32_t mn = min(min(v4[0], v4[1]), min(v4[2], v4[3]));
                const uint32_t T0 = n - 1 - i;
                if (!__any_sync(0xffffffffu, mn <= T0)) continue;
                // draw q = 32u + l of the group is certainly accepted if
                // v + q <= T0 (at most q acceptances precede it) and rejected if
                // v > T0; when no draw lies in between, every fate is known and
                // the ranks are prefix counts in draw order (one pass, no
                // dependence between the four rounds)
                uint32_t cm[4];
                bool und = false;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const uint32_t q = 32u * u + (uint32_t)lane;
                    const bool cert = v4[u] + q <= T0;
                    cm[u] = __ballot_sync(0xffffffffu, cert);
                    und = und || (!cert && v4[u] <= T0);
                }
                if (!__any_sync(0xffffffffu, und)) {
                    uint32_t run = i;
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if ((cm[u] >> lane) & 1u) {
                            const uint32_t r = run + (uint32_t)__popc(cm[u] & lt);
                            if (r < n) {
                                acc[r] = v4[u];
                                if (r == n - 1) s_dlast = d0 + base + 32u * u + (uint32_t)lane;
                            }
                        }
                        run += (uint32_t)__popc(cm[u]);
                    }
                    i = run;
                    continue;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (i >= n) break;
                    const uint32_t v = v4[u];  // v <= mask < 2^17: v + lane cannot wrap
                    const uint32_t T = n - 1 - i;
                    const bool cert = v + (uint32_t)lane <= T;
                    uint32_t ok = __ballot_sync(0xffffffffu, cert);
                    uint32_t pend = __ballot_sync(0xffffffffu, !cert && v <= T);
                    while (pend) {
                        const int j = __ffs(pend) - 1;
                        pend &= pend - 1;
                        const uint32_t vj = __shfl_sync(0xffffffffu, v, j);
                        if (vj + (uint32_t)__popc(ok & ((1u << j) - 1u)) <= T) ok |= 1u << j;
                    }
                    if ((ok >> lane) & 1u) {
                        const uint32_t r = i + (uint32_t)__popc(ok & lt);
                        if (r < n) {
                            acc[r] = v;
                            if (r == n - 1) s_dlast = d0 + base + 32u * u + (uint32_t)lane;
                        }
                    }
                    i += (uint32_t)__popc(ok);
                }
            }
        }
    }
    __syncwarp();
    if (threadIdx.x == 0) {
        // gen_perm refills each time its index reaches the end of a buffer,
        // the last accepted draw included: 1 + floor(draws / 2^20) buffers
        if (i >= n) a.used[g * a.count + m] = 1u + (s_dlast + 1u) / (1u << 20);
        else atomicOr(a.overflow, 1u);
    }
}

struct FyScanArgs {
    uint32_t n, count, tiles;
    uint32_t g0;                   // group of block 0 (one launch per group)
    unsigned long long win_tile0;  // absolute index of the window's first tile
    FyLayout lay;
    const uint32_t* ev;
    const uint32_t* last;  // [3][tiles] masked value of each tile's last draw
    const uint32_t* cnt;
    FyState* state;     // [3]
    uint32_t* acc;      // [count][3][n] accepted offsets v_i (swap with i + v_i)
    uint32_t* refills;  // [3][count] getNext buffers used
    unsigned long long* stats;  // optional [3][kFyStats] diagnostic counters (ORQ_FY_STATS)
};


// ---------------------------------------------------------------------------
// The scanner. One 1024-thread CTA per group replays the acceptance of its
// chain exactly. A step takes the next cs entries (<= 32768) of the current
// level; warp w owns entries [1024w, 1024w + 1024) and at iteration u its lane
// l holds entry q = 1024w + 32u + l, so loads, ranks and the stores of
// accepted values are all lane-parallel (ballots and popcounts, no per-thread
// serial loops) and coalesced. Level 1: entry q is certainly accepted if
// v + q <= T (at most q acceptances precede it), certainly rejected if v > T,
// otherwise uncertain. Level 2 (warp 0, 32 uncertain entries at a time):
// with c = certain accepts before an uncertain entry and a = uncertain accepts
// before it, it is accepted iff a <= T - c - v ("slack"); lane j of a chunk is
// certain if slack >= a_chunk + j, rejected if slack < a_chunk, and only the
// rest is decided lane by lane. A step with more uncertain entries than the
// list holds is halved until they fit (a step of at most kUncCap entries
// always does).
constexpr uint32_t kMaxStepEntries = 32768;
constexpr int kPerThread = kMaxStepEntries / kScanThreads;  // 32
constexpr int kScanWarps = kScanThreads / 32;
constexpr int kFyStats = 10;  // diagnostic counters per group
constexpr int kQuads = kPerThread / 4;  // lane-quads per thread and step
constexpr uint32_t kUncCap = 2048;
// dynamic shared memory: the step's entries, then the lane-quad classes and
// prefixes (cq below)
constexpr size_t kScanSmem = (size_t)kMaxStepEntries * 4 + (size_t)kScanWarps * kQuads * 32 * 4;

// entries per step at level L: uncertain entries of a step are about
// cs^2 / (2 n/4^L); keep that near 512
__device__ __forceinline__ uint32_t step_entries(uint32_t n, uint32_t L) {
    const unsigned long long t = level_threshold(n, L);
    uint32_t s = kMaxStepEntries;
    while (s > 1024 && (unsigned long long)s * s > 1024ull * t) s >>= 1;
    return s;
}

// 4-byte global -> shared copy that completes asynchronously (cp.async);
// dst is a shared-window address
__device__ __forceinline__ void cp_async4(uint32_t dst, const uint32_t* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// bulk prefetch of [addr, addr + bytes) into L2; addr and bytes multiples of 16
// (the range may round a list out to 16 bytes: list buffers carry slack)
__device__ __forceinline__ void prefetch_l2(uintptr_t addr, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(addr), "r"(bytes) : "memory");
}

// class of entry q with value v in a step of cs entries at bound T: bit 0
// certainly accepted (v + q <= T: at most q acceptances precede it), bit 4
// uncertain (v <= T but not certain); rejected otherwise
// (v < n < 2^31 and q < 2^15 for real entries, so v + q fits 32 bits; the
// padding entries beyond cs are excluded first)
__device__ __forceinline__ uint32_t fy_class(uint32_t q, uint32_t v, uint32_t cs, uint32_t T) {
    const bool in = q < cs;
    const bool cert = in && v + q <= T;
    const bool unc = in && !cert && v <= T;
    return (uint32_t)cert | ((uint32_t)unc << 4);
}

// exclusive warp prefix and warp total of a lane-quad's (certain | uncertain << 16)
__device__ __forceinline__ void quad_prefix(uint32_t code, int lane, uint32_t& excl, uint32_t& total) {
    const uint32_t x = __popc(code & 0xfu) | (__popc(code >> 4) << 16);
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    total = __shfl_sync(0xffffffffu, inc, 31);
    excl = inc - x;
}

// tile holding entry e, searching P[lo..hi] (P[lo] <= e < P[hi+1])
__device__ __forceinline__ uint32_t tile_in(const uint32_t* P, uint32_t lo, uint32_t hi, uint32_t e) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (P[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// quads (128 entries) of warp w's range [1024w, 1024w + 1024) below cs
__device__ __forceinline__ int wquads(int w, uint32_t cs) {
    const uint32_t b = (uint32_t)w * 1024u;
    return b >= cs ? 0 : (int)min((uint32_t)kQuads, (cs - b + 127u) / 128u);
}

__global__ void __launch_bounds__(kScanThreads, 1) k_fy_scan(FyScanArgs a) {
    extern __shared__ __align__(16) uint32_t sv[];  // step entries, sv[q]
    __shared__ uint32_t red[33];
    __shared__ uint32_t P[kMaxWindowTiles + 1];  // prefix of level-L counts over the window
    __shared__ uint32_t unc_v[kUncCap], unc_cp[kUncCap], unc_pre[kUncCap + 1];
    __shared__ uint32_t wtot[kScanWarps], wpre[kScanWarps];
    // per warp, quad iteration and lane: bits 0-7 the four entries' classes,
    // bits 8-18 the certain and bits 19-29 the uncertain entries of the warp
    // before this lane-quad (at most 1024 each); in the dynamic allocation
    // after the entries (static shared memory is limited to 48 KB)
    auto cq = reinterpret_cast<uint32_t (*)[kQuads][32]>(sv + kMaxStepEntries);
    __shared__ uint32_t s_last_q, s_uacc, s_tot;
    const uint32_t g = a.g0 + blockIdx.x;
    const uint32_t n = a.n;
    const uint32_t tiles = a.tiles;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    // scan state, identical in every thread
    uint32_t i = a.state[g].i, m = a.state[g].m, done = a.state[g].done;
    unsigned long long start = a.state[g].start_tile;
    uint32_t tau = 0, ix = 0, L = 0, Lp = 0xffffffffu;
    const uint32_t* EV = a.ev + (size_t)g * tiles * a.lay.slot;
    const uint32_t* LAST = a.last + (size_t)g * tiles;
    const uint32_t* C = a.cnt + (size_t)g * tiles * kMaxLevels;
    unsigned long long st_steps = 0, st_unc_steps = 0, st_ent = 0, st_unc = 0,
                       st_cyc_load = 0, st_cyc_unc = 0, st_cyc_all = 0, st_cyc_list = 0, st_cyc_acc = 0;
    const unsigned long long t_begin = clock64();
    for (int guard = 0; guard < (1 << 24) && !done; guard++) {
        // never look before the current permutation's first tile
        if (a.win_tile0 + tau < start) {
            const unsigned long long d = start - a.win_tile0;
            tau = d > tiles ? tiles : (uint32_t)d;
            ix = 0;
        }
        if (tau >= tiles) break;
        const uint32_t T = n - 1 - i;
        // sparsest level still holding every candidate v <= T
        uint32_t want = 0;
        while (want + 1 < a.lay.nl && T < level_threshold(n, want + 1)) want++;
        if (ix == 0) L = want;  // levels change only at tile starts
        if (L != Lp) {
            uint32_t tot;
            const uint32_t c = threadIdx.x < tiles ? C[threadIdx.x * kMaxLevels + L] : 0u;
            const uint32_t pre = block_excl_sum(c, red, tot);
            if (threadIdx.x < tiles) P[threadIdx.x] = pre;
            if (threadIdx.x == 0) P[tiles] = tot;
            __syncthreads();
            Lp = L;
        }
        const uint32_t e0 = P[tau] + ix;
        const uint32_t eend = (ix != 0 && want != L) ? P[tau + 1] : P[tiles];
        if (e0 >= eend) {
            if (eend == P[tiles]) tau = tiles;
            else {
                tau++;
                ix = 0;
            }
            continue;
        }
        uint32_t cs = min(step_entries(n, L), eend - e0);
        const unsigned long long t_l0 = clock64();
        if (warp == 0) {
            // warm L2 with the entries of the next two steps (a hint: the
            // staging of a later step then reads L2 instead of DRAM); lane j
            // covers the j-th tile of that range
            const uint32_t pf0 = e0 + cs, pf1 = min(P[tiles], e0 + cs + 2 * step_entries(n, L));
            if (pf0 < pf1) {
                const uint32_t t = tile_in(P, tau, tiles - 1, pf0) + lane;
                if (t < tiles && P[t] < pf1) {
                    const uint32_t s0 = max(P[t], pf0), s1 = min(P[t + 1], pf1);
                    if (s0 < s1) {
                        const uint32_t* src = EV + (size_t)t * a.lay.slot + a.lay.off[L] + (s0 - P[t]);
                        const uintptr_t lo = (uintptr_t)src & ~(uintptr_t)15;
                        const uintptr_t hi = ((uintptr_t)(src + (s1 - s0)) + 15) & ~(uintptr_t)15;
                        prefetch_l2(lo, (uint32_t)(hi - lo));
                    }
                }
            }
        }
        const uint32_t qw = (uint32_t)warp * 1024u + lane;  // staging: this thread's entry at u = 0
        // ---- stage the step's entries into shared memory at sv[q] with
        // asynchronous copies: no registers hold them, so all of a thread's
        // loads are in flight at once (coalesced per iteration; each lane walks
        // its tile cursor forward). Warp w stages and then processes entries
        // [1024w, 1024w + 1024), so a warp-level sync publishes them.
        {
            // the lane's current tile: entry e lives at EV[boff + e] while
            // e < tend; the tile advances only when a lane crosses into the next
            const size_t off = a.lay.off[L];
            uint32_t t = tau;
            uint32_t tend = P[t + 1];
            size_t boff = (size_t)t * a.lay.slot + off - (size_t)P[t];  // wraps; boff + e does not
            const uint32_t sv_sh = (uint32_t)__cvta_generic_to_shared(sv);
            // entries past cs are never read as entries (their class is
            // forced to rejected), so they are not staged
#pragma unroll
            for (int u = 0; u < kPerThread; u++) {
                if ((uint32_t)warp * 1024u + 32u * u >= cs) break;  // warp-uniform
                const uint32_t q = qw + 32u * u;
                if (q < cs) {
                    const uint32_t e = e0 + q;
                    if (e >= tend) {
                        do {
                            t++;
                        } while (P[t + 1] <= e);
                        tend = P[t + 1];
                        boff = (size_t)t * a.lay.slot + off - (size_t)P[t];
                    }
                    cp_async4(sv_sh + 4u * q, EV + (boff + e));
                }
            }
            cp_async_wait_all();
        }
        __syncwarp();
        // In the passes below lane l of warp w holds, at iteration u, the four
        // consecutive entries q = 1024w + 128u + 4l + r (r = 0..3); cq[w][u][l]
        // keeps their classification (bit r: certainly accepted, bit 4 + r:
        // uncertain): a lane-quad is one 16-byte shared load, and ranks come
        // from one packed warp scan per 128 entries.
        const uint32_t q0 = (uint32_t)warp * 1024u + 4u * (uint32_t)lane;
        // ---- level 1 counts per warp, block prefix over warps; halve the step
        // while the uncertain entries do not fit the list
        uint32_t tot_c, tot_u;
        for (;;) {
            uint32_t x = 0;  // the warp's (certain | uncertain << 16) so far
            // the warp's quads holding entries (warp-uniform; the passes below
            // skip the rest, whose classes would all be zero)
            const int nq = wquads(warp, cs);
#pragma unroll
            for (int u = 0; u < kQuads; u++) {
                if (u >= nq) break;
                const uint32_t q = q0 + 128u * u;
                const uint4 v4 = *reinterpret_cast<const uint4*>(sv + q);
                const uint32_t code = fy_class(q, v4.x, cs, T) | (fy_class(q + 1, v4.y, cs, T) << 1) |
                                      (fy_class(q + 2, v4.z, cs, T) << 2) | (fy_class(q + 3, v4.w, cs, T) << 3);
                uint32_t ex, tot;
                quad_prefix(code, lane, ex, tot);
                const uint32_t pre = x + ex;
                cq[warp][u][lane] = code | ((pre & 0xffffu) << 8) | ((pre >> 16) << 19);
                x += tot;
            }
            if (lane == 0) wtot[warp] = x;
            __syncthreads();
            if (warp == 0) {
                const uint32_t y = wtot[lane];
                uint32_t inc = y;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t z = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += z;
                }
                wpre[lane] = inc - y;
                if (lane == 31) s_tot = inc;
            }
            __syncthreads();
            tot_c = s_tot & 0xffffu;
            tot_u = s_tot >> 16;
            if (tot_u <= kUncCap) break;
            cs >>= 1;  // uniform: every thread read the same total
            __syncthreads();
        }
        const uint32_t cbase = wpre[warp] & 0xffffu, ubase = wpre[warp] >> 16;
        st_steps++;
        st_ent += cs;
        st_cyc_load += clock64() - t_l0;
        const unsigned long long t_li0 = clock64();
        // ---- list the uncertain entries in order, with the certain accepts
        // before each
        const int nq = wquads(warp, cs);
        if (tot_u) {
#pragma unroll
            for (int u = 0; u < kQuads; u++) {
                if (u >= nq) break;
                const uint32_t cw = cq[warp][u][lane];
                const uint32_t code = cw & 0xffu;
                if (code >> 4) {
                    const uint32_t q = q0 + 128u * u;
                    uint32_t c = cbase + ((cw >> 8) & 0x7ffu), k = ubase + (cw >> 19);
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        if ((code >> (4 + r)) & 1u) {
                            unc_v[k] = sv[q + r];
                            unc_cp[k] = c;
                            k++;
                        }
                        c += (code >> r) & 1u;
                    }
                }
            }
        }
        __syncthreads();
        const unsigned long long t_u0 = clock64();
        st_cyc_list += t_u0 - t_li0;
        if (warp == 0) {
            // level 2 over the listed uncertain entries
            uint32_t acc_so_far = 0;
            for (uint32_t base = 0; base < tot_u; base += 32) {
                const uint32_t k = base + lane;
                const bool valid = k < tot_u;
                long long slack = -1;
                if (valid) slack = (long long)T - unc_cp[k] - unc_v[k];
                const bool cert = valid && slack >= (long long)acc_so_far + lane;
                const bool und = valid && !cert && slack >= (long long)acc_so_far;
                uint32_t okmask = __ballot_sync(0xffffffffu, cert);
                const uint32_t undmask = __ballot_sync(0xffffffffu, und);
                if (undmask) {
                    // decide the undetermined lanes in order; the certain ones
                    // (already in okmask) and the rejected ones do not depend
                    // on the lanes before them
                    uint32_t pend = undmask;
                    while (pend) {
                        const int j = __ffs(pend) - 1;
                        pend &= pend - 1;
                        const long long sj = __shfl_sync(0xffffffffu, slack, j);
                        const uint32_t before = acc_so_far + __popc(okmask & ((1u << j) - 1u));
                        if (sj >= (long long)before) okmask |= 1u << j;
                    }
                }
                if (valid) {
                    unc_pre[k] = acc_so_far + __popc(okmask & lt);
                    unc_cp[k] = (okmask >> lane) & 1u;  // reuse as the decision
                }
                acc_so_far += __popc(okmask);
            }
            if (lane == 0) {
                unc_pre[tot_u] = acc_so_far;
                s_uacc = acc_so_far;
            }
        }
        __syncthreads();
        if (tot_u) {
            st_unc_steps++;
            st_unc += tot_u;
            st_cyc_unc += clock64() - t_u0;
        }
        // ---- accept, rank, store (a lane's accepted entries go to consecutive
        // ranks, consecutive lanes to consecutive runs)
        const unsigned long long t_a0 = clock64();
        const uint32_t tot_a = tot_c + s_uacc;
        const uint32_t need = n - i;
        uint32_t* acc = a.acc + ((size_t)m * 3 + g) * (size_t)n;
        {
            uint32_t* acci = acc + i;
#pragma unroll
            for (int u = 0; u < kQuads; u++) {
                if (u >= nq) break;
                const uint32_t cw = cq[warp][u][lane];
                const uint32_t code = cw & 0xffu;
                if (code) {
                    const uint32_t q = q0 + 128u * u;
                    const uint4 v4 = *reinterpret_cast<const uint4*>(sv + q);
                    const uint32_t vv[4] = {v4.x, v4.y, v4.z, v4.w};
                    // certain / uncertain entries before q + r
                    uint32_t c = cbase + ((cw >> 8) & 0x7ffu), k = ubase + (cw >> 19);
                    if ((code >> 4) == 0) {
                        // no uncertain entry in the quad: one lookup of the
                        // uncertain acceptances before it serves all four
                        const uint32_t up = unc_pre[k];
#pragma unroll
                        for (int r = 0; r < 4; r++) {
                            if ((code >> r) & 1u) {
                                const uint32_t rank = c + up;
                                if (rank < need) {
                                    acci[rank] = vv[r];
                                    if (rank == need - 1) s_last_q = q + r;
                                }
                                c++;
                            }
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < 4; r++) {
                            const bool cert = (code >> r) & 1u, unc = (code >> (4 + r)) & 1u;
                            if (cert || (unc && unc_cp[k])) {
                                const uint32_t rank = c + unc_pre[k];
                                if (rank < need) {
                                    acci[rank] = vv[r];
                                    if (rank == need - 1) s_last_q = q + r;
                                }
                            }
                            c += cert;
                            k += unc;
                        }
                    }
                }
            }
        }
        if (tot_a >= need) {
            __syncthreads();
            // permutation complete: locate its last draw, count the getNext buffers
            const uint32_t e = e0 + s_last_q;
            const uint32_t t = tile_in(P, tau, tiles - 1, e);
            // only a last draw at the very end of a getNext buffer changes the
            // count below: that is the tile's last draw, and then it is the
            // last entry of the tile's list
            const bool tile_end = e + 1 == P[t + 1] && LAST[t] < level_threshold(n, L);
            const unsigned long long kend =
                (a.win_tile0 + t - start) * (unsigned long long)kTileDraws + (tile_end ? kTileDraws - 1 : 0);
            const unsigned long long R = 1 + ((kend + 1) >> 20);
            if (threadIdx.x == 0) a.refills[(size_t)g * a.count + m] = (uint32_t)R;
            start = (start / kTilesPerRefill + R) * kTilesPerRefill;
            m++;
            i = 0;
            ix = 0;
            if (m >= a.count) done = 1;
        } else {
            i += tot_a;
            const uint32_t enew = e0 + cs;
            if (enew >= P[tiles]) {
                tau = tiles;
                ix = 0;
            } else {
                tau = tile_in(P, tau, tiles - 1, enew);
                ix = enew - P[tau];
            }
        }
        __syncthreads();  // the lists and counters are reused by the next step
        st_cyc_acc += clock64() - t_a0;
    }
    if (threadIdx.x == 0) {
        a.state[g].i = i;
        a.state[g].m = m;
        a.state[g].done = done;
        a.state[g].start_tile = start;
        if (a.stats) {
            st_cyc_all = clock64() - t_begin;
            unsigned long long* st = a.stats + g * kFyStats;
            st[0] += st_steps;
            st[1] += st_unc_steps;
            st[3] += st_ent;
            st[4] += st_unc;
            st[5] += st_cyc_load;
            st[6] += st_cyc_unc;
            st[7] += st_cyc_all;
            st[8] += st_cyc_list;
            st[9] += st_cyc_acc;
        }
    }
}

// ---- finalize: accepted offsets -> permutation -----------------------------
// Step i swaps positions i and j_i = i + v_i (j_i >= i), so position i is final
// after step i. The steps s != k with j_s = k (all s < k) form the bucket of
// position k, s_1 < ... < s_c in step order. Position k holds k until step s_1
// and A(s_m) after step s_m, where A(s) is the value at position s just before
// step s. So step s_m outputs p[s_m] = A(s_{m-1}) (k for m = 1), and A(k) =
// A(s_c) (k for an empty bucket): A(k) is the root of k in the forest of links
// k -> max(bucket(k)). A self-swap (j_k = k) outputs p[k] = A(k).
// Buckets are built by a counting sort: counts per target, an exclusive scan
// per permutation, then an atomic cursor per target places the steps (the
// cursor ends at the bucket's end, which is also the next bucket's start).
constexpr int kFinThreads = 1024;
constexpr uint32_t kFinChunk = kFinThreads * 8;  // scan chunk

struct FinArgs {
    const uint32_t* acc;  // [P][n]
    uint32_t n, P, chunks;
    uint32_t* cur;        // [P][n] bucket sizes, then starts (scan), then ends (place)
    uint32_t* part;       // [P][chunks] chunk sums, then their exclusive scan
    int32_t* bucket;      // [P][n] steps grouped by target
    int32_t* par;         // [P][n] max(bucket(k)), -1 when empty
    int32_t* A;           // [P][n]
    int32_t* const* perm_out;  // [P] -> n
    int32_t* const* inv_out;   // [P] -> n
    int* err;
};

// target of step i; an out-of-range offset (never produced by a correct scan)
// is flagged and treated as a self-swap so no access leaves the arrays
__device__ __forceinline__ uint32_t fin_target(const FinArgs& a, size_t t, uint32_t i) {
    const unsigned long long j = (unsigned long long)i + a.acc[t];
    if (j >= a.n) {
        atomicOr(a.err, 1);
        return i;
    }
    return (uint32_t)j;
}

__global__ void k_fin_count(FinArgs a) {
    const size_t tot = (size_t)a.P * a.n;
    for (size_t t = gtid(); t < tot; t += gstride()) {
        const size_t pm = t / a.n;
        const uint32_t i = (uint32_t)(t % a.n);
        const uint32_t j = fin_target(a, t, i);
        if (j != i) atomicAdd(&a.cur[pm * a.n + j], 1u);
    }
}

// sum of chunk (blockIdx.x % chunks) of permutation (blockIdx.x / chunks)
__global__ void __launch_bounds__(kFinThreads) k_fin_part(FinArgs a) {
    __shared__ uint32_t red[33];
    const size_t pm = blockIdx.x / a.chunks, ch = blockIdx.x % a.chunks;
    const uint32_t* c = a.cur + pm * a.n;
    uint32_t s = 0;
#pragma unroll
    for (int u = 0; u < 8; u++) {
        const size_t k = ch * kFinChunk + (size_t)u * kFinThreads + threadIdx.x;
        s += k < a.n ? c[k] : 0u;
    }
    uint32_t tot;
    block_excl_sum(s, red, tot);
    if (threadIdx.x == 0) a.part[pm * a.chunks + ch] = tot;
}

// exclusive scan of one permutation's chunk sums (one CTA per permutation)
__global__ void __launch_bounds__(kFinThreads) k_fin_top(FinArgs a) {
    __shared__ uint32_t red[33];
    uint32_t* p = a.part + (size_t)blockIdx.x * a.chunks;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < a.chunks; b0 += kFinThreads) {
        const uint32_t k = b0 + threadIdx.x;
        const uint32_t v = k < a.chunks ? p[k] : 0u;
        uint32_t tot;
        const uint32_t pre = block_excl_sum(v, red, tot);
        if (k < a.chunks) p[k] = carry + pre;
        carry += tot;
    }
}

// bucket starts: exclusive scan of the sizes, in place
__global__ void __launch_bounds__(kFinThreads) k_fin_starts(FinArgs a) {
    __shared__ uint32_t red[33];
    const size_t pm = blockIdx.x / a.chunks, ch = blockIdx.x % a.chunks;
    uint32_t* c = a.cur + pm * a.n;
    const size_t k0 = ch * kFinChunk + (size_t)threadIdx.x * 8;  // 8 consecutive per thread
    uint32_t v[8], s = 0;
#pragma unroll
    for (int u = 0; u < 8; u++) {
        v[u] = k0 + u < a.n ? c[k0 + u] : 0u;
        s += v[u];
    }
    uint32_t tot;
    uint32_t pre = block_excl_sum(s, red, tot) + a.part[pm * a.chunks + ch];
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (k0 + u < a.n) c[k0 + u] = pre;
        pre += v[u];
    }
}

__global__ void k_fin_place(FinArgs a) {
    const size_t tot = (size_t)a.P * a.n;
    for (size_t t = gtid(); t < tot; t += gstride()) {
        const size_t pm = t / a.n;
        const uint32_t i = (uint32_t)(t % a.n);
        const uint32_t j = fin_target(a, t, i);
        if (j != i) {
            const uint32_t slot = atomicAdd(&a.cur[pm * a.n + j], 1u);
            if (slot < a.n) a.bucket[pm * a.n + slot] = (int32_t)i;
            else atomicOr(a.err, 2);
        }
    }
}

// bucket of position k after placement: [end(k-1), end(k)), clamped to n
__device__ __forceinline__ void fin_bucket(const FinArgs& a, size_t pm, uint32_t k, uint32_t& b, uint32_t& e) {
    const uint32_t* cur = a.cur + pm * a.n;
    e = min(cur[k], a.n);
    b = k ? min(cur[k - 1], e) : 0u;
}

__global__ void k_fin_par(FinArgs a) {
    const size_t tot = (size_t)a.P * a.n;
    for (size_t t = gtid(); t < tot; t += gstride()) {
        const size_t pm = t / a.n;
        const uint32_t k = (uint32_t)(t % a.n);
        uint32_t b, e;
        fin_bucket(a, pm, k, b, e);
        const int32_t* bk = a.bucket + pm * a.n;
        int32_t mx = -1;
        for (uint32_t m = b; m < e; m++) mx = max(mx, bk[m]);
        // bucket entries are steps before k; anything else is corruption
        if (mx >= (int32_t)k) {
            atomicOr(a.err, 8);
            mx = -1;
        }
        a.par[t] = mx;
    }
}

__global__ void k_fin_roots(FinArgs a) {
    const size_t tot = (size_t)a.P * a.n;
    for (size_t t = gtid(); t < tot; t += gstride()) {
        const size_t pm = t / a.n;
        const int32_t* par = a.par + pm * a.n;
        int32_t k = (int32_t)(t % a.n);
        int32_t p = par[k];
        while (p >= 0) {  // strictly decreasing links: ends at a root
            k = p;
            p = par[k];
        }
        a.A[t] = k;
    }
}

__device__ __forceinline__ void fin_emit(const FinArgs& a, size_t pm, uint32_t s, int32_t val) {
    if ((uint32_t)val >= a.n) {
        atomicOr(a.err, 4);
        val = (int32_t)s;
    }
    a.perm_out[pm][s] = val;
    a.inv_out[pm][val] = (int32_t)s;
}

// per position k: its own step if it is a self-swap, and every step of its
// bucket (predecessor found by a scan of the small bucket)
__global__ void k_fin_final(FinArgs a) {
    const size_t tot = (size_t)a.P * a.n;
    for (size_t t = gtid(); t < tot; t += gstride()) {
        const size_t pm = t / a.n;
        const uint32_t k = (uint32_t)(t % a.n);
        const int32_t* A = a.A + pm * a.n;
        if (fin_target(a, t, k) == k) fin_emit(a, pm, k, A[k]);
        uint32_t b, e;
        fin_bucket(a, pm, k, b, e);
        const int32_t* bk = a.bucket + pm * a.n;
        for (uint32_t m = b; m < e; m++) {
            const int32_t s = bk[m];
            int32_t pred = -1;
            for (uint32_t q = b; q < e; q++) {
                const int32_t x = bk[q];
                if (x < s && x > pred) pred = x;
            }
            fin_emit(a, pm, (uint32_t)s, pred >= 0 ? A[pred] : (int32_t)k);
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Generate `count` sharded permutations of size n from the three 2-party group
// streams, in ORQ's order: permutation-major, groups {0,1},{0,2},{1,2}
// (generateBatch, hm_sharded_permutation_generator.h:178-194).
namespace {
FyRes& fy_res(Ctx& c) {
    FyRes& R = c.fy;
    if (R.ready) return R;
    // the scanners' streams have the highest priority: when generator CTAs
    // (which fill an SM's registers and shared memory) retire, pending scans
    // are dispatched before the next generator window
    int prio_lo = 0, prio_hi = 0;
    ORQ_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    ORQ_CUDA_CHECK(cudaStreamCreateWithPriority(&R.gs, cudaStreamNonBlocking, prio_lo));
    for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamCreateWithPriority(&R.ss[g], cudaStreamNonBlocking, prio_hi));
    ORQ_CUDA_CHECK(cudaStreamCreateWithPriority(&R.fs, cudaStreamNonBlocking, prio_lo));
    ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&R.ev_start, cudaEventDisableTiming));
    ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&R.fin_done, cudaEventDisableTiming));
    for (int k = 0; k < kFyRingMax; k++) {
        ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&R.gen_done[k], cudaEventDisableTiming));
        for (int g = 0; g < 3; g++) {
            ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&R.scan_done[g][k], cudaEventDisableTiming));
            ORQ_CUDA_CHECK(cudaEventCreateWithFlags(&R.st_ev[g][k], cudaEventDisableTiming));
        }
    }
    ORQ_CUDA_CHECK(cudaMallocHost(&R.hst, (size_t)kFyRingMax * 3 * sizeof(FyState)));
    R.ready = true;
    return R;
}
}  // namespace

void release_fy(Ctx& c) {
    FyRes& R = c.fy;
    if (!R.ready) return;
    cudaStreamSynchronize(R.gs);
    for (int g = 0; g < 3; g++) cudaStreamSynchronize(R.ss[g]);
    cudaStreamSynchronize(R.fs);
    cudaEventDestroy(R.ev_start);
    cudaEventDestroy(R.fin_done);
    for (int k = 0; k < kFyRingMax; k++) {
        cudaEventDestroy(R.gen_done[k]);
        for (int g = 0; g < 3; g++) {
            cudaEventDestroy(R.scan_done[g][k]);
            cudaEventDestroy(R.st_ev[g][k]);
        }
    }
    cudaStreamDestroy(R.gs);
    for (int g = 0; g < 3; g++) cudaStreamDestroy(R.ss[g]);
    cudaStreamDestroy(R.fs);
    cudaFreeHost(R.hst);
    R = FyRes{};
}

void gen_sharded_perms(Ctx& c, size_t n, size_t count, std::vector<ShardedPerm>& out) {
    out.clear();
    if (count == 0) return;
    if (n >= (1ull << 31)) throw std::invalid_argument("permutation size must be < 2^31");
    out.resize(count);
    for (auto& sp : out) {
        sp.n = n;
        for (int g = 0; g < 3; g++) {
            sp.perm[g] = (int32_t*)c.alloc(std::max<size_t>(n, 1) * 4);
            sp.inv[g] = (int32_t*)c.alloc(std::max<size_t>(n, 1) * 4);
        }
    }
    if (n == 0) {
        // gen_perm still draws one buffer (4 nonces) per permutation
        for (int g = 0; g < 3; g++) c.nonce[G01 + g] += 4ull * count;
        return;
    }
    int bitsw = 0;
    while (bitsw < 64 && (n >> bitsw)) bitsw++;
    const uint32_t mask = (uint32_t)((1ull << bitsw) - 1);

    // window of buffers generated per pipeline step
    const double M = (double)(1ull << bitsw);
    double H = 0;
    for (size_t k = 1; k <= std::min<size_t>(n, 1 << 16); k++) H += 1.0 / k;
    if (n > (1u << 16)) H += std::log((double)n / (1 << 16));
    const double per_perm = M * H / (double)(1 << 20) + 1.0;  // expected buffers
    uint32_t W = (uint32_t)std::clamp(per_perm * count / 8.0, 2.0, (double)(kMaxWindowTiles / kTilesPerRefill));
    const uint32_t tiles = W * kTilesPerRefill;

    FyLayout lay{};
    {
        // levels down to a threshold of 256: sparser ones would hold almost
        // nothing, and the scan of a permutation's last steps reads at most a
        // few thousand entries of the last level instead
        uint32_t nl = 1;
        while (nl < (uint32_t)kMaxLevels && level_threshold((uint32_t)n, nl) >= 256) nl++;
        lay.nl = nl;
        uint32_t o = 0;
        for (uint32_t L = 0; L < nl; L++) {
            lay.off[L] = o;
            lay.cap[L] = level_capacity(L);
            o += lay.cap[L];
        }
        lay.slot = o;
    }
    const size_t ents_b = (size_t)3 * tiles * lay.slot * 4;
    const size_t cnt_b = (size_t)3 * tiles * kMaxLevels * 4;
    // Ring of window buffers: the draws of a window do not depend on the scan
    // (windows are consecutive buffers of the group streams), so the generator
    // runs up to kRing-1 windows ahead. It stays ahead through the dense start
    // of a permutation (scan-bound) and the scanner catches up through the
    // sparse tail (generation-bound). The three groups are scanned on three
    // streams: their dense phases fall in different windows, and a shared
    // launch per window would cost the slowest group every time.
    // (allocated below, after the small-permutation path, which needs none)
    constexpr int kRing = 6;
    Scratch acc(c, (size_t)3 * count * n * 4);
    const bool want_stats = std::getenv("ORQ_FY_STATS") != nullptr;
    const auto t_start = std::chrono::steady_clock::now();

    // generator and scanner run on private non-blocking streams so they overlap
    // whatever the caller's stream is (the legacy default stream included)
    // the scanner's stream has the highest priority: when generator CTAs
    // (which fill an SM's registers and shared memory) retire, a pending scan
    // is dispatched before the next generator window
    FyRes& R = fy_res(c);
    cudaStream_t gs = R.gs;
    cudaStream_t* ss = R.ss;
    cudaEvent_t ev_start = R.ev_start;
    auto& gen_done = R.gen_done;
    auto& scan_done = R.scan_done;
    auto& st_ev = R.st_ev;
    static_assert(kRing <= kFyRingMax, "ring deeper than the cached events");
    // On every exit path (an exception included) the generator and scanner
    // streams are drained before the ring, state and output scratch above go
    // back to the pool: a later call on the runtime's stream could otherwise
    // be handed memory those kernels are still writing. Declared after the
    // scratch buffers, so it runs before their destructors.
    //
    // Finalize runs on its own low-priority stream for the permutations the
    // scanners have completed, while the chain goes on (the generator leaves
    // SMs idle while the scanners work through dense windows). acc is laid out
    // [permutation][group], so B permutations of all three groups are one
    // contiguous batch; the scratch holds one batch.
    const size_t fin_b = std::max<size_t>(1, std::min<size_t>({(size_t)4, count,
                                                               ((size_t)1 << 27) / (3 * std::max<size_t>(n, 1))}));
    const size_t fin_el = 3 * fin_b * n;
    const uint32_t fin_chunks = (uint32_t)ceil_div(n, (size_t)kFinChunk);
    Scratch f_cur(c, fin_el * 4), f_part(c, 3 * fin_b * fin_chunks * 4), f_bucket(c, fin_el * 4),
        f_par(c, fin_el * 4), f_A(c, fin_el * 4), f_ptrs(c, 2 * 3 * count * sizeof(void*));
    {
        std::vector<int32_t*> hp(2 * 3 * count);
        for (size_t m = 0; m < count; m++)
            for (int g = 0; g < 3; g++) {
                hp[3 * m + g] = out[m].perm[g];
                hp[3 * count + 3 * m + g] = out[m].inv[g];
            }
        ORQ_CUDA_CHECK(cudaMemcpyAsync(f_ptrs.p, hp.data(), hp.size() * sizeof(void*), cudaMemcpyHostToDevice,
                                       c.stream));
        ORQ_CUDA_CHECK(cudaStreamSynchronize(c.stream));  // hp is pageable and leaves scope
    }
    cudaStream_t fs = R.fs;
    size_t fin_next = 0;  // permutations [0, fin_next) are queued for finalize
    auto launch_fin = [&](size_t m0, size_t m1) {
        const size_t P = 3 * (m1 - m0);
        const size_t el = P * n;
        FinArgs fa;
        fa.acc = acc.as<uint32_t>() + 3 * m0 * n;
        fa.n = (uint32_t)n;
        fa.P = (uint32_t)P;
        fa.chunks = fin_chunks;
        fa.cur = f_cur.as<uint32_t>();
        fa.part = f_part.as<uint32_t>();
        fa.bucket = f_bucket.as<int32_t>();
        fa.par = f_par.as<int32_t>();
        fa.A = f_A.as<int32_t>();
        fa.perm_out = f_ptrs.as<int32_t*>() + 3 * m0;
        fa.inv_out = f_ptrs.as<int32_t*>() + 3 * count + 3 * m0;
        fa.err = c.d_err;
        const unsigned gg = plain_grid(c, el);
        const unsigned gc = (unsigned)(P * fin_chunks);
        ProfScope ps(c, "fy_finalize", 0.0, 0.0, fs);
        ORQ_CUDA_CHECK(cudaMemsetAsync(f_cur.p, 0, el * 4, fs));
        k_fin_count<<<gg, 256, 0, fs>>>(fa);
        k_fin_part<<<gc, kFinThreads, 0, fs>>>(fa);
        k_fin_top<<<(unsigned)P, kFinThreads, 0, fs>>>(fa);
        k_fin_starts<<<gc, kFinThreads, 0, fs>>>(fa);
        k_fin_place<<<gg, 256, 0, fs>>>(fa);
        k_fin_par<<<gg, 256, 0, fs>>>(fa);
        k_fin_roots<<<gg, 256, 0, fs>>>(fa);
        k_fin_final<<<gg, 256, 0, fs>>>(fa);
        ORQ_CUDA_CHECK(cudaGetLastError());
        c.kernels_launched += 8;
    };
    struct DrainSideStreams {
        FyRes& r;
        ~DrainSideStreams() {
            cudaStreamSynchronize(r.gs);
            for (int g = 0; g < 3; g++) cudaStreamSynchronize(r.ss[g]);
            cudaStreamSynchronize(r.fs);
        }
    } drain{R};
    ORQ_CUDA_CHECK(cudaEventRecord(ev_start, c.stream));
    ORQ_CUDA_CHECK(cudaStreamWaitEvent(gs, ev_start, 0));
    for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamWaitEvent(ss[g], ev_start, 0));
    ORQ_CUDA_CHECK(cudaStreamWaitEvent(fs, ev_start, 0));

    if ((1ull << bitsw) <= kSmallMaxM) {
        // every permutation of every group at once from predicted start
        // buffers, corrected pass by pass (k_fy_small)
        const uint32_t bhat = 1u + (uint32_t)(M * H / (double)(1u << 20));
        std::vector<uint32_t> hstart(3 * count), hused(3 * count);
        for (int g = 0; g < 3; g++)
            for (size_t m = 0; m < count; m++) hstart[g * count + m] = (uint32_t)m * bhat;
        Scratch d_start(c, hstart.size() * 4), d_used(c, hused.size() * 4), ovf(c, 4);
        // the pool hands out memory in the runtime stream's order
        ORQ_CUDA_CHECK(cudaEventRecord(ev_start, c.stream));
        ORQ_CUDA_CHECK(cudaStreamWaitEvent(gs, ev_start, 0));
        ORQ_CUDA_CHECK(cudaMemsetAsync(ovf.p, 0, 4, gs));
        ORQ_CUDA_CHECK(cudaFuncSetAttribute(k_fy_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem));
        FySmallArgs sa;
        for (int g = 0; g < 3; g++) {
            sa.st[g] = c.stream_arg(G01 + g);
            sa.m0[g] = 0;
        }
        sa.n = (uint32_t)n;
        sa.mask = mask;
        sa.count = (uint32_t)count;
        sa.max_chunks = (bhat + 6) * kChunksPerBuffer;
        sa.start = d_start.as<uint32_t>();
        sa.used = d_used.as<uint32_t>();
        sa.acc = acc.as<uint32_t>();
        sa.overflow = ovf.as<uint32_t>();
        bool ok = false;
        for (int pass = 0; pass < 64; pass++) {
            ORQ_CUDA_CHECK(cudaMemcpyAsync(d_start.p, hstart.data(), hstart.size() * 4, cudaMemcpyHostToDevice, gs));
            {
                ProfScope ps(c, "fy_small", 0.0, 0.0, gs);
                k_fy_small<<<(unsigned)(3 * count), kSmallThreads, kSmallSmem, gs>>>(sa);
            }
            ORQ_CUDA_CHECK(cudaGetLastError());
            c.kernels_launched++;
            uint32_t overflow = 0;
            ORQ_CUDA_CHECK(cudaMemcpyAsync(hused.data(), d_used.p, hused.size() * 4, cudaMemcpyDeviceToHost, gs));
            ORQ_CUDA_CHECK(cudaMemcpyAsync(&overflow, ovf.p, 4, cudaMemcpyDeviceToHost, gs));
            ORQ_CUDA_CHECK(cudaStreamSynchronize(gs));
            if (overflow) break;
            // permutations before m0[g] are verified, and so is m0[g]'s start;
            // the first one whose assumed start differs from the true one is
            // where the next pass begins
            bool again = false;
            for (int g = 0; g < 3; g++) {
                uint32_t* st = hstart.data() + g * count;
                const uint32_t* us = hused.data() + g * count;
                size_t m = sa.m0[g];
                if (m >= count) continue;
                uint32_t expect = st[m];
                for (; m < count; m++) {
                    if (st[m] != expect) break;
                    expect = st[m] + us[m];
                }
                sa.m0[g] = (uint32_t)m;
                if (m < count) {
                    again = true;
                    for (size_t k = m; k < count; k++) st[k] = expect + (uint32_t)(k - m) * bhat;
                }
            }
            if (!again) {
                ok = true;
                break;
            }
        }
        if (ok) {
            for (int g = 0; g < 3; g++)
                c.nonce[G01 + g] += 4ull * (hstart[g * count + count - 1] + hused[g * count + count - 1]);
            for (; fin_next < count; fin_next += fin_b) launch_fin(fin_next, std::min(count, fin_next + fin_b));
            ORQ_CUDA_CHECK(cudaEventRecord(R.fin_done, fs));
            ORQ_CUDA_CHECK(cudaStreamWaitEvent(c.stream, R.fin_done, 0));
            c.check_device_error();
            return;
        }
        // a permutation ran past max_chunks (or the passes did not settle):
        // the general chain below redoes all of them (no nonce was consumed)
    }

    std::vector<std::unique_ptr<Scratch>> ring_ev, ring_last, ring_cnt;
    for (int k = 0; k < kRing; k++) {
        ring_ev.emplace_back(new Scratch(c, ents_b + 256));  // slack for 16-byte rounded prefetches
        ring_last.emplace_back(new Scratch(c, (size_t)3 * tiles * 4));
        ring_cnt.emplace_back(new Scratch(c, cnt_b));
    }
    Scratch state(c, 3 * sizeof(FyState));
    Scratch refills(c, (size_t)3 * count * 4);
    ORQ_CUDA_CHECK(cudaMemsetAsync(state.p, 0, 3 * sizeof(FyState), c.stream));
    Scratch stats(c, 3 * kFyStats * 8);
    if (want_stats) ORQ_CUDA_CHECK(cudaMemsetAsync(stats.p, 0, 3 * kFyStats * 8, c.stream));
    // the side streams start after these allocations and memsets, and are
    // drained before the buffers above go back to the pool (declared after them)
    ORQ_CUDA_CHECK(cudaEventRecord(ev_start, c.stream));
    ORQ_CUDA_CHECK(cudaStreamWaitEvent(gs, ev_start, 0));
    for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamWaitEvent(ss[g], ev_start, 0));
    DrainSideStreams drain_ring{R};

    prep_aes_kernel(k_fy_gen);
    ORQ_CUDA_CHECK(cudaFuncSetAttribute(k_fy_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScanSmem));

    const unsigned gen_grid = (unsigned)std::max(1, c.num_sms - 3);
    uint32_t* evp[kRing];
    uint32_t* lastp[kRing];
    uint32_t* cntp[kRing];
    for (int k = 0; k < kRing; k++) {
        evp[k] = ring_ev[k]->as<uint32_t>();
        lastp[k] = ring_last[k]->as<uint32_t>();
        cntp[k] = ring_cnt[k]->as<uint32_t>();
    }

    const unsigned long long limit_windows =
        (unsigned long long)(count * (per_perm * 4.0 + 64.0) / W + 16);
    std::vector<cudaEvent_t> tl;  // stats mode: [gen start, gen end, scan start, scan end] per window
    auto tl_event = [&](cudaStream_t st) -> int {
        if (!want_stats) return -1;
        cudaEvent_t e;
        ORQ_CUDA_CHECK(cudaEventCreate(&e));
        ORQ_CUDA_CHECK(cudaEventRecord(e, st));
        tl.push_back(e);
        return (int)tl.size() - 1;
    };
    std::vector<std::array<int, 4>> tl_idx;
    auto launch_gen = [&](unsigned long long w) {
        const int b = (int)(w % kRing);
        // buffer b was last read by the three scans of window w-kRing
        if (w >= (unsigned long long)kRing)
            for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamWaitEvent(gs, scan_done[g][b], 0));
        FyGenArgs ga;
        for (int g = 0; g < 3; g++) ga.st[g] = c.stream_arg(G01 + g, 4ull * W * w);
        ga.n = (uint32_t)n;
        ga.mask = mask;
        ga.tiles = tiles;
        ga.lay = lay;
        ga.ev = evp[b];
        ga.last = lastp[b];
        ga.cnt = cntp[b];
        ga.state = state.as<FyState>();
        ga.err = c.d_err;
        if (tl_idx.size() <= w) tl_idx.resize(w + 1, {-1, -1, -1, -1});
        tl_idx[w][0] = tl_event(gs);
        {
            ProfScope ps(c, "fy_gen", 0.0, 3.0 * tiles * kTileBlocks, gs);
            k_fy_gen<<<gen_grid, kGenThreads, kAesSmemBytes, gs>>>(ga);
        }
        tl_idx[w][1] = tl_event(gs);
        ORQ_CUDA_CHECK(cudaGetLastError());
        ORQ_CUDA_CHECK(cudaEventRecord(gen_done[b], gs));
        c.kernels_launched++;
    };
    // Each group's scans are queued up to kRing-1 windows ahead of the host's
    // completion check, so a scan stream always holds its next scan (its CTA
    // takes the SM the previous one frees before any generator CTA can, by
    // stream priority) and no host round trip idles a scanner. A scan queued
    // after its group's last permutation completed sees `done` and returns.
    FyState* hst = static_cast<FyState*>(R.hst);
    auto launch_scan = [&](unsigned long long w, int g) {
        const int b = (int)(w % kRing);
        ORQ_CUDA_CHECK(cudaStreamWaitEvent(ss[g], gen_done[b], 0));
        FyScanArgs sa;
        sa.n = (uint32_t)n;
        sa.count = (uint32_t)count;
        sa.tiles = tiles;
        sa.g0 = (uint32_t)g;
        sa.win_tile0 = (unsigned long long)w * tiles;
        sa.lay = lay;
        sa.ev = evp[b];
        sa.last = lastp[b];
        sa.cnt = cntp[b];
        sa.state = state.as<FyState>();
        sa.acc = acc.as<uint32_t>();
        sa.refills = refills.as<uint32_t>();
        sa.stats = want_stats ? stats.as<unsigned long long>() : nullptr;
        if (tl_idx.size() <= w) tl_idx.resize(w + 1, {-1, -1, -1, -1});
        if (g == 0) tl_idx[w][2] = tl_event(ss[0]);
        {
            ProfScope ps(c, "fy_scan", 0.0, 0.0, ss[g]);
            k_fy_scan<<<1, kScanThreads, kScanSmem, ss[g]>>>(sa);
        }
        if (g == 0) tl_idx[w][3] = tl_event(ss[0]);
        ORQ_CUDA_CHECK(cudaGetLastError());
        ORQ_CUDA_CHECK(cudaEventRecord(scan_done[g][b], ss[g]));
        c.kernels_launched++;
        ORQ_CUDA_CHECK(cudaMemcpyAsync(hst + 3 * b + g, state.as<FyState>() + g, sizeof(FyState),
                                       cudaMemcpyDeviceToHost, ss[g]));
        ORQ_CUDA_CHECK(cudaEventRecord(st_ev[g][b], ss[g]));
    };
    // The host checks completion up to kRing-1 windows behind the launches
    // while more windows are expected (no idle scanner, no host round trip on
    // the critical path), then window by window, so a chain that ends early
    // does not leave a ring's worth of windows queued.
    const unsigned long long expect = (unsigned long long)std::ceil(per_perm * (double)count / W);
    unsigned long long checked = 0;
    bool finished = false;
    for (unsigned long long w = 0; !finished; w++) {
        if (w > limit_windows)
            throw std::runtime_error("permutation generation did not converge");
        launch_gen(w);
        for (int g = 0; g < 3; g++) launch_scan(w, g);
        const unsigned long long lag = (w + 1 < expect) ? (unsigned long long)(kRing - 1) : 0ull;
        while (!finished && checked + lag <= w) {
            const int pb = (int)(checked % kRing);
            bool all = true;
            size_t mmin = count;  // permutations every group has completed
            for (int g = 0; g < 3; g++) {
                ORQ_CUDA_CHECK(cudaEventSynchronize(st_ev[g][pb]));
                all = all && hst[3 * pb + g].done;
                mmin = std::min<size_t>(mmin, hst[3 * pb + g].done ? count : hst[3 * pb + g].m);
            }
            finished = all;
            checked++;
            if (!finished && fin_next + fin_b <= mmin) {
                // their accepted offsets were written before this window's states
                for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamWaitEvent(fs, st_ev[g][pb], 0));
                for (; fin_next + fin_b <= mmin; fin_next += fin_b) launch_fin(fin_next, fin_next + fin_b);
            }
        }
    }
    const unsigned long long w = tl_idx.size();
    ORQ_CUDA_CHECK(cudaStreamSynchronize(gs));
    for (int g = 0; g < 3; g++) ORQ_CUDA_CHECK(cudaStreamSynchronize(ss[g]));

    // nonce accounting: 4 nonces per getNext buffer
    std::vector<uint32_t> hr(3 * count);
    ORQ_CUDA_CHECK(cudaMemcpyAsync(hr.data(), refills.p, hr.size() * 4, cudaMemcpyDeviceToHost,
                                   c.stream));
    ORQ_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    for (int g = 0; g < 3; g++) {
        unsigned long long used = 0;
        for (size_t m = 0; m < count; m++) used += hr[g * count + m];
        c.nonce[G01 + g] += 4ull * used;
    }
    if (want_stats) {
        std::fprintf(stderr, "[fy] windows %llu of %u buffers, %.3f ms\n", w, W,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        for (size_t k = 0; k < tl_idx.size(); k++) {
            float g0 = 0, g1 = 0, s0 = 0, s1 = 0;
            if (tl_idx[k][0] >= 0) cudaEventElapsedTime(&g0, tl[0], tl[tl_idx[k][0]]);
            if (tl_idx[k][1] >= 0) cudaEventElapsedTime(&g1, tl[0], tl[tl_idx[k][1]]);
            if (tl_idx[k][2] >= 0) cudaEventElapsedTime(&s0, tl[0], tl[tl_idx[k][2]]);
            if (tl_idx[k][3] >= 0) cudaEventElapsedTime(&s1, tl[0], tl[tl_idx[k][3]]);
            std::fprintf(stderr, "[fy] window %zu: gen %.3f-%.3f scan %.3f-%.3f ms\n", k, g0, g1, s0, s1);
        }
        for (auto e : tl) cudaEventDestroy(e);
        unsigned long long hs[3 * kFyStats];
        ORQ_CUDA_CHECK(cudaMemcpy(hs, stats.p, sizeof(hs), cudaMemcpyDeviceToHost));
        for (int g = 0; g < 3; g++) {
            const unsigned long long* h = hs + g * kFyStats;
            std::fprintf(stderr,
                         "[fy] n=%zu perms=%zu windows=%llu group %d: steps %llu unc_steps %llu entries %llu "
                         "unc %llu cyc_load %llu cyc_list %llu cyc_unc %llu cyc_acc %llu cyc_all %llu\n",
                         n, count, w, g, h[0], h[1], h[3], h[4], h[5], h[8], h[6], h[9], h[7]);
        }
    }

    // the permutations completed since the last batch, then the runtime's
    // stream waits for the finalize stream
    for (; fin_next < count; fin_next += fin_b) launch_fin(fin_next, std::min(count, fin_next + fin_b));
    ORQ_CUDA_CHECK(cudaEventRecord(R.fin_done, fs));
    ORQ_CUDA_CHECK(cudaStreamWaitEvent(c.stream, R.fin_done, 0));
    c.check_device_error();

}

// PermutationManager::reserve (permutation_manager.h:102-181): keep a queue of
// permutations of one size; a size change empties it.
void reserve_perms(Ctx& c, size_t n, size_t count) {
    if (!c.perm_queue.empty() && c.perm_queue_n != n) {
        for (auto& sp : c.perm_queue) c.free_perm(sp);
        c.perm_queue.clear();
    }
    c.perm_queue_n = n;
    if (c.perm_queue.size() >= count) return;
    std::vector<ShardedPerm> fresh;
    gen_sharded_perms(c, n, count - c.perm_queue.size(), fresh);
    for (auto& sp : fresh) c.perm_queue.push_back(sp);
}

// PermutationManager::getNext / getNextPair for 3PC: pop the queue, or
// generate one on demand (hm generator getNext).
ShardedPerm next_perm(Ctx& c, size_t n) {
    if (!c.perm_queue.empty()) {
        if (c.perm_queue_n != n) throw std::runtime_error("queued permutation has the wrong size");
        ShardedPerm sp = c.perm_queue.front();
        c.perm_queue.pop_front();
        return sp;
    }
    std::vector<ShardedPerm> one;
    gen_sharded_perms(c, n, 1, one);
    return one[0];
}

// ---------------------------------------------------------------------------
// Application of one group's local permutation fused with that group's
// reshare, for up to two vectors that use the same permutation (ORQ applies
// the data vector and the permutation vector in turn with the same sharded
// permutation, shuffle.h:687-706). dst[k] = src[idx[k]] (+|^) r_j[k]:
// idx = inverse permutation for local_apply_perm (scatter new[pi[i]] = x[i],
// shuffle.h:113-133), idx = the permutation itself for
// local_apply_inverse_perm (shuffle.h:250-270).
//   MODE 0: store both results
//   MODE 2: open the second vector into sigma and scatter the first by it
//           (local_apply_perm of the opened permutation, shuffle.h:702-705)
//   MODE 3: open the first vector into sigma (no stores)
struct ApplyArgs {
    const void* src1[3];
    void* dst1[3];
    const void* src2[3];
    void* dst2[3];
    const int32_t* idx;
    StreamArg g1, g2;
    unsigned long long ch1, ch2;
    unsigned long long n;
    int32_t* sigma;
    int* err;
};

template <int W>
__device__ __forceinline__ void gather_elem(const void* src, int32_t k, uint8_t* dst) {
    if constexpr (W == 4) {
        *reinterpret_cast<uint32_t*>(dst) = __ldg(reinterpret_cast<const uint32_t*>(src) + k);
    } else if constexpr (W == 8) {
        *reinterpret_cast<uint2*>(dst) = __ldg(reinterpret_cast<const uint2*>(src) + k);
    } else {
        *reinterpret_cast<uint4*>(dst) = __ldg(reinterpret_cast<const uint4*>(src) + k);
    }
}
template <int W>
__device__ __forceinline__ void store_elem(void* dst, int32_t k, const uint8_t* v) {
    if constexpr (W == 4) {
        reinterpret_cast<uint32_t*>(dst)[k] = *reinterpret_cast<const uint32_t*>(v);
    } else if constexpr (W == 8) {
        reinterpret_cast<uint2*>(dst)[k] = *reinterpret_cast<const uint2*>(v);
    } else {
        reinterpret_cast<uint4*>(dst)[k] = *reinterpret_cast<const uint4*>(v);
    }
}

// the three shares of elements id[0..E) of src into E*W/16 16-byte words
// (element e at byte e*W); elements at or past n are left unchanged
template <int W, int E, int B>
__device__ __forceinline__ void gather3(const void* const* src, const int32_t (&id)[E], unsigned long long k0,
                                        unsigned long long n, uint4 (&v)[3][B]) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (k0 + e >= n) continue;
            if constexpr (W == 16) {
                v[j][e] = __ldg(reinterpret_cast<const uint4*>(src[j]) + id[e]);
            } else if constexpr (W == 8) {
                const uint2 x = __ldg(reinterpret_cast<const uint2*>(src[j]) + id[e]);
                if (e & 1) {
                    v[j][e >> 1].z = x.x;
                    v[j][e >> 1].w = x.y;
                } else {
                    v[j][e >> 1].x = x.x;
                    v[j][e >> 1].y = x.y;
                }
            } else {
                const uint32_t x = __ldg(reinterpret_cast<const uint32_t*>(src[j]) + id[e]);
                switch (e & 3) {
                    case 0: v[j][e >> 2].x = x; break;
                    case 1: v[j][e >> 2].y = x; break;
                    case 2: v[j][e >> 2].z = x; break;
                    default: v[j][e >> 2].w = x; break;
                }
            }
        }
}

template <int E>
__device__ __forceinline__ void load_idx(const int32_t* idx, unsigned long long k0, unsigned long long n,
                                         int32_t (&id)[E]) {
#pragma unroll
    for (int e = 0; e < E; e++) id[e] = (k0 + e < n) ? __ldg(idx + k0 + e) : 0;
}

// Zero-sharing of one 16-byte block of a vector: the keystreams of block blk in
// the group stream (r0) and at nonce offset ch (r1), r2 = -(r0 + r1) or
// r0 ^ r1, added to the three shares held at v[.][0]; then v[.][0..B) rotate
// left by one so the next block sits at index 0 (after B calls the order is
// restored). Called from loops kept rolled: two AES bodies per vector instead
// of two per block keep the kernel's loop inside the instruction cache (fully
// unrolled, ten AES-256 bodies stalled every warp on instruction fetch).
template <int W, bool A, int B>
__device__ __forceinline__ void reshare_block(const AesSmem& S, StreamArg gs, unsigned long long ch,
                                              unsigned long long blk, uint4 (&v)[3][B]) {
    const uint4 r0 = keystream_block(S, gs, blk);
    gs.nonce += ch;
    const uint4 r1 = keystream_block(S, gs, blk);
    uint4 r2;
    if constexpr (A) r2 = Ring<W>::sub(Ring<W>::sub(make_uint4(0, 0, 0, 0), r0), r1);
    else r2 = r0 ^ r1;
    v[0][0] = Share<W, A>::plus(v[0][0], r0);
    v[1][0] = Share<W, A>::plus(v[1][0], r1);
    v[2][0] = Share<W, A>::plus(v[2][0], r2);
    if constexpr (B > 1) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const uint4 x = v[j][0];
#pragma unroll
            for (int b = 0; b + 1 < B; b++) v[j][b] = v[j][b + 1];
            v[j][B - 1] = x;
        }
    }
}

// E elements per thread and unit; E*W1 and E*W2 are multiples of 16 bytes.
// Software-pipelined: a unit's gathers are issued in the previous iteration,
// right after that iteration has consumed the same registers, so each random
// gather has a whole iteration of keystream work to arrive in; the next unit's
// indices are loaded at the top of an iteration.
template <int W1, bool A1, int W2, bool A2, int MODE>
__global__ void __launch_bounds__(kAesThreads, 1) k_apply(ApplyArgs a) {
    constexpr int WMIN = (W2 && W2 < W1) ? W2 : W1;
    constexpr int E = 16 / WMIN;
    constexpr int B1 = E * W1 / 16;
    constexpr int B2 = W2 ? E * W2 / 16 : 1;
    extern __shared__ __align__(16) uint32_t sm[];
    aes_stage_tables(sm);
    const AesSmem S(sm);
    const unsigned long long units = ceil_div(a.n, E);
    unsigned long long t = gtid();
    if (t >= units) return;  // no barrier follows the table staging
    const unsigned long long stride = gstride();
    uint4 v1[3][B1], v2[3][B2];
    {
        int32_t id[E];
        load_idx<E>(a.idx, t * E, a.n, id);
        gather3<W1, E, B1>(a.src1, id, t * E, a.n, v1);
        if constexpr (W2 != 0) gather3<W2, E, B2>(a.src2, id, t * E, a.n, v2);
    }
    for (;;) {
        const unsigned long long k0 = t * E;
        const unsigned long long tn = t + stride;
        const bool more = tn < units;
        int32_t idn[E];
        load_idx<E>(a.idx, more ? tn * E : a.n, a.n, idn);
        // ---- vector 2 (the permutation vector in elementwise application)
        uint32_t sig[E];
        if constexpr (W2 != 0) {
#pragma unroll 1
            for (int bb = 0; bb < B2; bb++) reshare_block<W2, A2, B2>(S, a.g2, a.ch2, t * B2 + bb, v2);
            if constexpr (MODE == 0) {
#pragma unroll
                for (int j = 0; j < 3; j++)
#pragma unroll
                    for (int bb = 0; bb < B2; bb++) st16(a.dst2[j], t * B2 + bb, a.n * W2, v2[j][bb]);
            } else if constexpr (MODE == 2) {
                // open (W2 == 4): sigma = sum or xor of the three shares
                uint4 o[B2];
#pragma unroll
                for (int bb = 0; bb < B2; bb++)
                    o[bb] = Share<W2, A2>::plus(Share<W2, A2>::plus(v2[0][bb], v2[1][bb]), v2[2][bb]);
#pragma unroll
                for (int e = 0; e < E; e++) sig[e] = reinterpret_cast<const uint32_t*>(o)[e];
            }
            if (more) gather3<W2, E, B2>(a.src2, idn, tn * E, a.n, v2);
        }
        // ---- vector 1
#pragma unroll 1
        for (int bb = 0; bb < B1; bb++) reshare_block<W1, A1, B1>(S, a.g1, a.ch1, t * B1 + bb, v1);
        if constexpr (MODE == 0) {
#pragma unroll
            for (int j = 0; j < 3; j++)
#pragma unroll
                for (int bb = 0; bb < B1; bb++) st16(a.dst1[j], t * B1 + bb, a.n * W1, v1[j][bb]);
        } else if constexpr (MODE == 2) {
#pragma unroll
            for (int j = 0; j < 3; j++)
#pragma unroll
                for (int e = 0; e < E; e++)
                    if (k0 + e < a.n) {
                        // sigma is an opened permutation; a value outside [0, n)
                        // means corrupted shares: flag it, skip the store
                        if ((unsigned long long)sig[e] < a.n)
                            store_elem<W1>(a.dst1[j], (int32_t)sig[e],
                                           reinterpret_cast<const uint8_t*>(&v1[j][0]) + e * W1);
                        else
                            atomicOr(a.err, 8);
                    }
        } else if constexpr (MODE == 3) {
            uint4 o[B1];
#pragma unroll
            for (int bb = 0; bb < B1; bb++)
                o[bb] = Share<W1, A1>::plus(Share<W1, A1>::plus(v1[0][bb], v1[1][bb]), v1[2][bb]);
#pragma unroll
            for (int e = 0; e < E; e++)
                if (k0 + e < a.n) a.sigma[k0 + e] = reinterpret_cast<const int32_t*>(o)[e];
        }
        if (!more) break;
        gather3<W1, E, B1>(a.src1, idn, tn * E, a.n, v1);
        t = tn;
    }
}

namespace {

template <int W1, bool A1, int W2, bool A2, int MODE>
void launch_apply(Ctx& c, const ApplyArgs& a) {
    constexpr int WMIN = (W2 && W2 < W1) ? W2 : W1;
    constexpr int E = 16 / WMIN;
    auto kern = k_apply<W1, A1, W2, A2, MODE>;
    prep_aes_kernel(kern);
    const unsigned long long units = ceil_div(a.n, E);
    // idx + gathered shares + written shares (the second vector is only read
    // when its result is opened instead of stored)
    const double by = (double)a.n * (4.0 + 6.0 * W1 + (W2 ? (MODE == 0 ? 6.0 : 3.0) * W2 : 0.0));
    const double bl = 2.0 * ((double)ceil_div(a.n * W1, 16) + (W2 ? (double)ceil_div(a.n * W2, 16) : 0.0));
    ProfScope ps(c, "apply_group", by, bl);
    kern<<<aes_grid(c, units), kAesThreads, kAesSmemBytes, c.stream>>>(a);
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

// runtime dispatch over the (width, encoding) combinations used by the operators
template <int MODE>
void dispatch_apply(Ctx& c, int w1, bool a1, int w2, bool a2, const ApplyArgs& a) {
#define ORQ_AP(W1v, A1v, W2v, A2v)                                      \
    if (w1 == W1v && a1 == A1v && w2 == W2v && (W2v == 0 || a2 == A2v)) \
        return launch_apply<W1v, A1v, W2v, A2v, MODE>(c, a);
    ORQ_AP(4, false, 0, false)
    ORQ_AP(4, true, 0, false)
    ORQ_AP(8, false, 0, false)
    ORQ_AP(8, true, 0, false)
    ORQ_AP(16, false, 0, false)
    ORQ_AP(16, true, 0, false)
    ORQ_AP(16, false, 4, true)
    ORQ_AP(16, false, 4, false)
    ORQ_AP(8, false, 4, true)
    ORQ_AP(8, true, 4, true)
    ORQ_AP(8, false, 4, false)
    ORQ_AP(8, true, 4, false)
    ORQ_AP(4, true, 4, true)
    ORQ_AP(4, false, 4, true)
    ORQ_AP(4, true, 4, false)
    ORQ_AP(4, false, 4, false)
#undef ORQ_AP
    throw std::invalid_argument("unsupported share width/encoding for permutation application");
}

}  // namespace

// hm_oblivious_apply_sharded_perm / _inverse (shuffle.h:349-412) on one vector.
void op_apply_sharded(Ctx& c, bool arith, int w, size_t n, Sh3 s, const ShardedPerm& sp,
                      bool inverse) {
    if (w != 4 && w != 8 && w != 16)
        throw std::invalid_argument("permutation application supports 4, 8 and 16-byte shares");
    const unsigned long long ch = chunks_of((unsigned long long)n * w);
    if (n == 0) return;
    Scratch tmp(c, 3 * n * (size_t)w);
    void* other[3] = {tmp.as<uint8_t>(), tmp.as<uint8_t>() + n * (size_t)w,
                      tmp.as<uint8_t>() + 2 * n * (size_t)w};
    void* cur[3] = {s.p[0], s.p[1], s.p[2]};
    for (int step = 0; step < 3; step++) {
        const int g = inverse ? 2 - step : step;
        ApplyArgs a{};
        for (int j = 0; j < 3; j++) {
            a.src1[j] = cur[j];
            a.dst1[j] = other[j];
        }
        a.idx = inverse ? sp.perm[g] : sp.inv[g];
        a.g1 = c.stream_arg(G01 + g);
        a.ch1 = ch;
        a.n = n;
        dispatch_apply<0>(c, w, arith, 0, false, a);
        c.nonce[G01 + g] += 2 * ch;
        for (int j = 0; j < 3; j++) std::swap(cur[j], other[j]);
    }
    // three swaps leave the result in the scratch buffers
    for (int j = 0; j < 3; j++)
        ORQ_CUDA_CHECK(cudaMemcpyAsync(s.p[j], cur[j], n * (size_t)w, cudaMemcpyDeviceToDevice, c.stream));
}

// oblivious_apply_elementwise_perm (shuffle.h:687-706): shuffle x and a copy
// of the permutation with the same sharded permutation, open the shuffled
// permutation and scatter x with it. Three fused kernels, one per group.
void op_apply_elementwise(Ctx& c, bool x_arith, int xw, size_t n, Sh3 x, CSh3 perm) {
    if (n == 0) {
        ShardedPerm sp = next_perm(c, n);
        c.free_perm(sp);
        return;
    }
    ShardedPerm sp = next_perm(c, n);
    const unsigned long long chx = chunks_of((unsigned long long)n * xw);
    const unsigned long long chp = chunks_of((unsigned long long)n * 4);
    Scratch xa(c, 3 * n * (size_t)xw), xb(c, 3 * n * (size_t)xw), pa(c, 3 * n * 4), pb(c, 3 * n * 4);
    void* X[2][3];
    void* Pp[2][3];
    for (int j = 0; j < 3; j++) {
        X[0][j] = xa.as<uint8_t>() + j * n * (size_t)xw;
        X[1][j] = xb.as<uint8_t>() + j * n * (size_t)xw;
        Pp[0][j] = pa.as<uint8_t>() + j * n * 4;
        Pp[1][j] = pb.as<uint8_t>() + j * n * 4;
    }
    for (int g = 0; g < 3; g++) {
        ApplyArgs a{};
        for (int j = 0; j < 3; j++) {
            a.src1[j] = g == 0 ? x.p[j] : X[(g - 1) & 1][j];
            a.dst1[j] = g == 2 ? x.p[j] : X[g & 1][j];
            a.src2[j] = g == 0 ? perm.p[j] : Pp[(g - 1) & 1][j];
            a.dst2[j] = Pp[g & 1][j];
        }
        a.idx = sp.inv[g];
        a.err = c.d_err;
        // per group stream: the x reshare first, then the permutation's
        a.g1 = c.stream_arg(G01 + g);
        a.g2 = c.stream_arg(G01 + g, 2 * chx);
        a.ch1 = chx;
        a.ch2 = chp;
        a.n = n;
        if (g < 2) dispatch_apply<0>(c, xw, x_arith, 4, true, a);
        else dispatch_apply<2>(c, xw, x_arith, 4, true, a);
        c.nonce[G01 + g] += 2 * chx + 2 * chp;
    }
    c.free_perm(sp);
}

// shuffle (shuffle.h:752-757)
void op_shuffle(Ctx& c, bool arith, int w, size_t n, Sh3 s) {
    ShardedPerm sp = next_perm(c, n);
    op_apply_sharded(c, arith, w, n, s, sp, false);
    c.free_perm(sp);
}

// local_apply_perm with a public permutation: dst[sigma[i]] = src[i]
template <int W>
__global__ void k_scatter(CSh3 src, Sh3 dst, const int32_t* sigma, unsigned long long n, int* err) {
    for (unsigned long long i = gtid(); i < n; i += gstride()) {
        const int32_t d = __ldg(sigma + i);
        if ((unsigned long long)(uint32_t)d >= n) {
            atomicOr(err, 8);
            continue;
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
            uint8_t v[W];
            gather_elem<W>(src.p[j], (int32_t)i, v);
            store_elem<W>(dst.p[j], d, v);
        }
    }
}
void op_scatter(Ctx& c, int w, size_t n, CSh3 src, Sh3 dst, const int32_t* sigma) {
    if (!n) return;
    const unsigned g = plain_grid(c, n);
    if (w == 4) k_scatter<4><<<g, 256, 0, c.stream>>>(src, dst, sigma, n, c.d_err);
    else if (w == 8) k_scatter<8><<<g, 256, 0, c.stream>>>(src, dst, sigma, n, c.d_err);
    else if (w == 16) k_scatter<16><<<g, 256, 0, c.stream>>>(src, dst, sigma, n, c.d_err);
    else throw std::invalid_argument("scatter supports 4, 8, 16-byte shares");
    ORQ_CUDA_CHECK(cudaGetLastError());
    c.kernels_launched++;
}

}  // namespace orqcu
