// runtime.cu — context set-up: key schedule, AES tables, device buffer pool.
#include <cstring>

#include <algorithm>

#include "runtime.h"

namespace orqcu {

// ---------------------------------------------------------------------------
// Keys. The reference draws every AES-256 key from libsodium's keygen
// (include/core/random/prg/prg_algorithm.h:192-197). Reproducible runs replace
// that with SplitMix64 keyed by (seed, party, keygen-call index); the test shim
// that builds the reference does the same, so identical seeds give identical
// shares. Call order per party follows setup_random_generation
// (include/backend/common/rand_setup.h:306-381) — see init_ctx_keys.
static uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void derive_key(uint64_t seed, int party, int call, uint8_t key[32]) {
    uint64_t st = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(party + 1)) ^
                  (0xABC98388FB8FAC03ull * (uint64_t)(call + 1));
    for (int i = 0; i < 4; i++) {
        uint64_t v = splitmix64(st);
        for (int b = 0; b < 8; b++) key[8 * i + b] = (uint8_t)(v >> (8 * b));
    }
}

// AES (FIPS-197): S-box from the GF(2^8) inverse and affine map.
static uint8_t gmul(uint8_t a, uint8_t b) {
    uint8_t p = 0;
    while (b) {
        if (b & 1) p ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1B : 0));
        b >>= 1;
    }
    return p;
}
static const uint8_t* sbox() {
    static uint8_t s[256];
    static bool ready = false;
    if (!ready) {
        for (int x = 0; x < 256; x++) {
            uint8_t inv = 0;
            for (int y = 1; x && y < 256; y++)
                if (gmul((uint8_t)x, (uint8_t)y) == 1) {
                    inv = (uint8_t)y;
                    break;
                }
            uint8_t v = inv, r = inv;
            for (int i = 0; i < 4; i++) {
                r = (uint8_t)((r << 1) | (r >> 7));
                v ^= r;
            }
            s[x] = v ^ 0x63;
        }
        ready = true;
    }
    return s;
}

void aes256_expand(const uint8_t key[32], uint32_t rk[60]) {
    const uint8_t* S = sbox();
    auto subw = [&](uint32_t w) {
        return (uint32_t)S[w & 0xff] | ((uint32_t)S[(w >> 8) & 0xff] << 8) |
               ((uint32_t)S[(w >> 16) & 0xff] << 16) | ((uint32_t)S[w >> 24] << 24);
    };
    for (int i = 0; i < 8; i++)
        rk[i] = (uint32_t)key[4 * i] | ((uint32_t)key[4 * i + 1] << 8) |
                ((uint32_t)key[4 * i + 2] << 16) | ((uint32_t)key[4 * i + 3] << 24);
    uint8_t rcon = 1;
    for (int i = 8; i < 60; i++) {
        uint32_t t = rk[i - 1];
        if (i % 8 == 0) {
            t = subw((t >> 8) | (t << 24)) ^ rcon;
            rcon = gmul(rcon, 2);
        } else if (i % 8 == 4) {
            t = subw(t);
        }
        rk[i] = rk[i - 8] ^ t;
    }
}

// Which keygen call of which party keys each stream (rand_setup.h:21-146):
// call 0 = local PRG; lowest member draws group keys in the order {0,1},{0,2},
// {1,2},{0,1,2}; P0 draws a discarded duplicate everyone-group key; the last
// call is the pairwise key of setup_3pc_common_prgs.
void init_ctx_keys(Ctx& c, uint64_t seed) {
    static const int who[NSTREAMS][2] = {{0, 5}, {1, 2}, {2, 1}, {0, 1}, {0, 2},
                                         {1, 1}, {0, 3}, {0, 0}, {1, 0}, {2, 0}};
    c.seed = seed;
    for (int s = 0; s < NSTREAMS; s++) {
        uint8_t key[32];
        derive_key(seed, who[s][0], who[s][1], key);
        aes256_expand(key, c.rk[s].k);
        c.nonce[s] = 0;
    }
}

// Beaver 2PC (rand_setup.h:229-238,306-330): call 0 local PRG, call 1 the
// {0,1} group on P0 (P0's call 2, the everyone group of the same set, is
// discarded). Fantastic-4PC (rand_setup.h:154-221): call 0 local PRG, P0 draws
// the keys of {0,1,2}, {2,3,0}, {3,0,1} and the everyone group (calls 1-4),
// P1 that of {1,2,3}; setup_4pc_common_prgs then draws one key per party (P0
// call 5, P1 call 2, P2 call 1, P3 call 1): party q's key seeds the PRG of
// the three parties other than q+1.
void init_ctx_keys_np(Ctx& c, uint64_t seed, int nparties) {
    static const int who2[3][2] = {{0, 1}, {0, 0}, {1, 0}};
    static const int who4[8][2] = {{3, 1}, {0, 5}, {1, 2}, {2, 1}, {0, 0}, {1, 0}, {2, 0}, {3, 0}};
    if (nparties != 2 && nparties != 4) throw std::invalid_argument("parties must be 2 or 4");
    c.seed = seed;
    c.nparties = nparties;
    const int ns = nparties == 2 ? 3 : 8;
    for (int s = 0; s < NSTREAMS; s++) {
        c.nonce[s] = 0;
        std::memset(c.rk[s].k, 0, sizeof(c.rk[s].k));
    }
    for (int s = 0; s < ns; s++) {
        uint8_t key[32];
        const int* wh = nparties == 2 ? who2[s] : who4[s];
        derive_key(seed, wh[0], wh[1], key);
        aes256_expand(key, c.rk[s].k);
    }
}

static std::vector<AesTableUploader>& uploaders() {
    static std::vector<AesTableUploader> v;
    return v;
}
int register_aes_table_uploader(AesTableUploader f) {
    uploaders().push_back(f);
    return (int)uploaders().size();
}

namespace {
std::mutex g_dev_mu;
int g_dev_live[kMaxDevices] = {};
unsigned long long g_dev_epoch[kMaxDevices] = {};
}  // namespace

void device_runtime_opened(int device) {
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_dev_mu);
    g_dev_live[device]++;
}

void device_runtime_closed(int device) {
    if (device < 0 || device >= kMaxDevices) return;
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if (g_dev_live[device] > 0 && --g_dev_live[device] == 0) {
        g_dev_epoch[device]++;
        release_pool_memory(device);  // the last runtime on the device is gone
    }
}

unsigned long long device_epoch(int device) {
    std::lock_guard<std::mutex> lk(g_dev_mu);
    return (device >= 0 && device < kMaxDevices) ? g_dev_epoch[device] : 0ull;
}

void upload_aes_tables(int device) {
    // epoch + 1 of the last upload per device (0: never uploaded)
    static unsigned long long done[kMaxDevices] = {};
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
    const unsigned long long ep = device_epoch(device) + 1;
    if (done[device] == ep) return;
    const uint8_t* S = sbox();
    uint32_t T[4 * 256];
    for (int x = 0; x < 256; x++) {
        const uint32_t s = S[x], s2 = gmul((uint8_t)s, 2), s3 = gmul((uint8_t)s, 3);
        const uint32_t t0 = s2 | (s << 8) | (s << 16) | (s3 << 24);
        T[x] = t0;
        T[256 + x] = (t0 << 8) | (t0 >> 24);
        T[512 + x] = (t0 << 16) | (t0 >> 16);
        T[768 + x] = (t0 << 24) | (t0 >> 8);
    }
    for (AesTableUploader f : uploaders()) f(T);
    done[device] = ep;
}

// ---------------------------------------------------------------------------
// Pool: size-bucketed reuse of device allocations (above 1 MiB a bucket is a
// multiple of an eighth of the size's power of two, so at most 12.5 % is
// wasted on the multi-gigabyte buffers of large sorts; 256-byte multiples
// below), so the per-round temporaries of a sort do not go back to the
// allocator. New blocks come from the stream-ordered
// allocator on the runtime's stream and trim() returns cached blocks the same
// way, so neither ever synchronises the device (runtimes on different streams
// allocate and release independently).
static size_t bucket(size_t bytes) {
    if (bytes < 256) return 256;
    if (bytes <= (1u << 20)) return (bytes + 255) & ~size_t(255);
    size_t p = size_t(1) << 20;
    while (p * 2 <= bytes) p <<= 1;  // p <= bytes < 2p
    const size_t step = p / 8;
    return (bytes + step - 1) / step * step;
}

void* Pool::get(size_t bytes, cudaStream_t stream) {
    const size_t b = bucket(bytes);
    {
        std::lock_guard<std::mutex> lk(mu_);
        // the smallest cached block of at least b bytes, if it wastes at most half of b
        auto it = free_.lower_bound(b);
        if (it != free_.end() && it->first <= b + b / 2) {
            void* p = it->second;
            live_[p] = it->first;
            forget(it);
            return p;
        }
        // a miss with much memory cached in other sizes (a runtime that
        // serves requests of changing sizes): hand the least recently
        // released blocks back to the device's pool, stream-ordered, until
        // they cover the new block, which then reuses that memory instead of
        // growing the footprint (the device pool keeps it mapped, see
        // keep_pool_memory); blocks a steady workload keeps reusing stay
        if (cached_ >= kEvictBytes) {
            size_t freed = 0;
            while (freed < b && !lru_.empty()) {
                void* q = lru_.begin()->second;
                const size_t sz = meta_[q].first;
                auto r = free_.equal_range(sz);
                auto f = r.first;
                while (f != r.second && f->second != q) ++f;
                if (f == r.second) {  // not in the size index: drop the stale entry
                    lru_.erase(lru_.begin());
                    meta_.erase(q);
                    continue;
                }
                freed += sz;
                cudaFreeAsync(q, stream);
                forget(f);
            }
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, b, stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        trim(stream);
        ORQ_CUDA_CHECK(cudaStreamSynchronize(stream));
        ORQ_CUDA_CHECK(cudaMallocAsync(&p, b, stream));
    }
    std::lock_guard<std::mutex> lk(mu_);
    live_[p] = b;
    return p;
}

// drop a cached block from the size index, the release order and the count
void Pool::forget(std::multimap<size_t, void*>::iterator it) {
    void* p = it->second;
    auto m = meta_.find(p);
    if (m != meta_.end()) {
        lru_.erase(m->second.second);
        meta_.erase(m);
    }
    cached_ -= it->first;
    free_.erase(it);
}

void Pool::put(void* p) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = live_.find(p);
    if (it == live_.end()) return;
    const size_t sz = it->second;
    free_.emplace(sz, p);
    const uint64_t t = ++clock_;
    lru_.emplace(t, p);
    meta_[p] = {sz, t};
    cached_ += sz;
    live_.erase(it);
}

// The device's default memory pool keeps memory freed into it mapped (by
// default it returns it to the system at the next synchronisation, and the
// next allocation maps it again at a cost of milliseconds per gigabyte).
// Per process; set once per device.
void keep_pool_memory(int device) {
    static std::mutex mu;
    static bool done[kMaxDevices] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= kMaxDevices || done[device]) return;
    cudaMemPool_t pool;
    ORQ_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = ~0ull;
    ORQ_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    done[device] = true;
}

void release_pool_memory(int device) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
}

void Pool::trim(cudaStream_t stream) {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& kv : free_) cudaFreeAsync(kv.second, stream);
    free_.clear();
    lru_.clear();
    meta_.clear();
    cached_ = 0;
}

size_t Pool::cached_bytes() {
    std::lock_guard<std::mutex> lk(mu_);
    return cached_;
}

Pool::~Pool() {
    for (auto& kv : free_) cudaFree(kv.second);
    for (auto& kv : live_) cudaFree(kv.first);
}

void Ctx::release_graphs() {
    for (auto& kv : graphs) {
        BatchGraph& g = kv.second;
        if (g.done) cudaEventSynchronize(g.done);
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.work) cudaFree(g.work);
        if (g.items_dev) cudaFree(g.items_dev);
        if (g.items_host) cudaFreeHost(g.items_host);
        if (g.done) cudaEventDestroy(g.done);
    }
    graphs.clear();
    if (capture_stream) cudaStreamDestroy(capture_stream);
    capture_stream = nullptr;
}

void Ctx::check_device_error() {
    if (!d_err) return;
    int h = 0;
    ORQ_CUDA_CHECK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ORQ_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h) {
        ORQ_CUDA_CHECK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
        throw std::runtime_error("out-of-range index in a permutation (code " + std::to_string(h) + ")");
    }
}

ProfScope::ProfScope(Ctx& ctx, const char* name, double bytes, double aes_blocks, cudaStream_t st)
    : c(&ctx), s(st ? st : ctx.stream), on(ctx.profiling) {
    if (!on) return;
    ev.name = name;
    ev.bytes = bytes;
    ev.aes_blocks = aes_blocks;
    ORQ_CUDA_CHECK(cudaEventCreate(&ev.a));
    ORQ_CUDA_CHECK(cudaEventCreate(&ev.b));
    ORQ_CUDA_CHECK(cudaEventRecord(ev.a, s));
}
ProfScope::~ProfScope() {
    if (!on) return;
    cudaEventRecord(ev.b, s);
    c->prof_pending.push_back(ev);
}

void Ctx::prof_collect() {
    for (auto& e : prof_pending) {
        float ms = 0;
        ORQ_CUDA_CHECK(cudaEventSynchronize(e.b));
        ORQ_CUDA_CHECK(cudaEventElapsedTime(&ms, e.a, e.b));
        auto& g = prof_agg[e.name];
        g.launches++;
        g.ms += ms;
        g.bytes += e.bytes;
        g.aes_blocks += e.aes_blocks;
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    prof_pending.clear();
}

void Ctx::free_perm(ShardedPerm& sp) {
    for (int g = 0; g < 3; g++) {
        release(sp.perm[g]);
        release(sp.inv[g]);
        sp.perm[g] = sp.inv[g] = nullptr;
    }
}

}  // namespace orqcu
