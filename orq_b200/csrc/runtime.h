// runtime.h — the single-process loopback runtime that stands in for ORQ's
// RunTime + per-party protocol objects (include/backend/common/runtime.h,
// include/core/protocols/replicated_3pc.h) on one GPU.
//
// One Ctx holds all three parties: the 10 AES streams of a 3PC worker
// (3 pairwise, 4 group, 3 party-local; include/backend/common/rand_setup.h),
// their nonce counters, a CUDA stream, a device buffer pool and the queue of
// reserved sharded permutations (random/permutations/permutation_manager.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <deque>
#include <map>
#include <string>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace orqcu {

enum StreamId {
    PAIR0 = 0,  // shared by P0/P1 (P0's local key): P0 get(+1), P1 get(-1)
    PAIR1 = 1,
    PAIR2 = 2,
    G01 = 3,
    G02 = 4,
    G12 = 5,
    G012 = 6,
    LOCAL0 = 7,
    LOCAL1 = 8,
    LOCAL2 = 9,
    NSTREAMS = 10
};
// The same slots hold the streams of the other protocol classes:
// Beaver 2PC: the {0,1} PRG and the parties' local PRGs;
// Fantastic-4PC: the PRG of the three parties other than e (NOT0 + e) and the
// local PRGs (LOCAL0 + p).
enum { P2_COMMON = 0, P2_LOCAL0 = 1, P4_NOT0 = 0, P4_LOCAL0 = 4 };

// Device allocation that returns to the pool when dropped.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

class Pool {
   public:
    void* get(size_t bytes, cudaStream_t stream);
    void put(void* p);
    void trim(cudaStream_t stream);
    size_t cached_bytes();
    ~Pool();

    // on a miss with at least this much cached in other sizes, the least
    // recently released blocks are handed back to the device's pool first
    static constexpr size_t kEvictBytes = size_t(8) << 30;

   private:
    std::mutex mu_;
    std::multimap<size_t, void*> free_;               // cached blocks by size
    std::map<void*, size_t> live_;
    std::map<uint64_t, void*> lru_;                    // cached blocks by release time
    std::map<void*, std::pair<size_t, uint64_t>> meta_;  // cached block: size, release time
    size_t cached_ = 0;
    uint64_t clock_ = 0;
    void forget(std::multimap<size_t, void*>::iterator it);
};
// the device's default memory pool keeps freed memory mapped (once per device)
void keep_pool_memory(int device);
// returns the device pool's unused memory to the system
void release_pool_memory(int device);

// A sharded permutation: one local permutation per 2-party group
// ({0,1},{0,2},{1,2}), each with its inverse, all device-resident int32.
struct ShardedPerm {
    size_t n = 0;
    int32_t* perm[3] = {nullptr, nullptr, nullptr};
    int32_t* inv[3] = {nullptr, nullptr, nullptr};
};

// Per-launch timing records (enabled on demand): CUDA events around a launch on
// the stream it runs on, aggregated per kernel class with the launch's
// algorithmic bytes (distinct share arrays read once + outputs written once)
// and the AES-256 blocks it computes.
struct ProfEvent {
    std::string name;
    cudaEvent_t a, b;
    double bytes, aes_blocks;
};
struct ProfAgg {
    unsigned long long launches = 0;
    double ms = 0, bytes = 0, aes_blocks = 0;
};

// A captured batch of launches, cached per batch shape: the work lists and
// the item table live on the device; the item table is refreshed from the
// pinned host copy by the graph's first node on every replay.
struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    void* work = nullptr;        // device work lists (all rounds)
    void* items_dev = nullptr;   // device item table
    void* items_host = nullptr;  // pinned item table (source of the graph's copy)
    size_t items_bytes = 0;
    cudaEvent_t done = nullptr;  // last replay finished reading items_host
    int nt = 0;
    unsigned long long launches = 0;
};

// Streams, events and pinned state of the permutation generator, created on
// first use and kept for the runtime's life (creating them per call cost
// device-wide synchronisation when the pinned buffer was freed).
constexpr int kFyRingMax = 8;
struct FyRes {
    bool ready = false;
    cudaStream_t gs = nullptr;
    cudaStream_t ss[3] = {nullptr, nullptr, nullptr};
    cudaStream_t fs = nullptr;  // finalize of completed permutations, during the chain
    cudaEvent_t ev_start = nullptr;
    cudaEvent_t fin_done = nullptr;
    cudaEvent_t gen_done[kFyRingMax] = {};
    cudaEvent_t scan_done[3][kFyRingMax] = {};
    cudaEvent_t st_ev[3][kFyRingMax] = {};
    void* hst = nullptr;  // pinned scanner states, [ring slot][group]
};

struct Ctx {
    int device = 0;
    int nparties = 3;  // 3: replicated 3PC; 2: Beaver 2PC; 4: Fantastic-4PC
    int party = -1;    // >= 0: plays only this party of 3PC (party.cu); -1: all parties
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    uint64_t seed = 0;
    AesRK rk[NSTREAMS];
    unsigned long long nonce[NSTREAMS] = {0};
    Pool pool;
    std::deque<ShardedPerm> perm_queue;
    size_t perm_queue_n = 0;
    unsigned long long kernels_launched = 0;
    // device word set by kernels that meet an out-of-range data-dependent index
    // (they skip the access); checked at the synchronous points.
    int* d_err = nullptr;
    void check_device_error();
    FyRes fy;
    std::map<std::string, BatchGraph> graphs;  // batched launches by shape
    std::map<std::string, int> tuned;          // autotuned threads per CTA by size class
    cudaStream_t capture_stream = nullptr;     // private stream for graph capture
    void release_graphs();
    bool profiling = false;
    std::vector<ProfEvent> prof_pending;
    std::map<std::string, ProfAgg> prof_agg;
    void prof_collect();

    StreamArg stream_arg(int s, unsigned long long extra_nonces = 0) const {
        StreamArg a;
        a.rk = rk[s];
        a.nonce = nonce[s] + extra_nonces;
        return a;
    }
    void* alloc(size_t bytes) { return pool.get(bytes, stream); }
    void release(void* p) {
        if (p) pool.put(p);
    }
    void free_perm(ShardedPerm& sp);
};

// RAII scratch from the pool.
struct Scratch {
    Ctx* c;
    void* p;
    Scratch(Ctx& ctx, size_t bytes) : c(&ctx), p(ctx.alloc(bytes)) {}
    ~Scratch() { c->release(p); }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
};

struct ProfScope {
    Ctx* c;
    cudaStream_t s;
    ProfEvent ev;
    bool on;
    ProfScope(Ctx& ctx, const char* name, double bytes, double aes_blocks = 0,
              cudaStream_t st = nullptr);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;
};

// host-side key derivation (identical to the test shim / restatement)
void derive_key(uint64_t seed, int party, int call, uint8_t key[32]);
void aes256_expand(const uint8_t key[32], uint32_t rk[60]);
void init_ctx_keys(Ctx& c, uint64_t seed);
// keys of the Beaver-2PC (nparties 2) or Fantastic-4PC (4) streams
void init_ctx_keys_np(Ctx& c, uint64_t seed, int nparties);

// ---- Beaver 2PC / Fantastic-4PC local steps (proto24.cu) ----
void op_np_secret_share(Ctx& c, bool arith, int w, size_t n, const void* data, int party, void* const* s);
void op_np_open(Ctx& c, bool arith, int w, size_t n, const void* const* s, void* out);
void op_np_local(Ctx& c, int op, int w, size_t n, const void* const* x, const void* const* y, void* const* z);
void op_np_mult(Ctx& c, int mode, int w, size_t n, const void* const* x, const void* const* y, void* const* z);
void upload_aes_tables(int device);
// Per-device set-up (the AES tables, the address of the no-alloc scratch
// array) is done once per device and remembered with the device's epoch. The
// epoch advances when the last live runtime on the device is destroyed, so a
// cudaDeviceReset between runtimes (which drops the context's memory and can
// move its module globals) makes the next runtime redo the set-up. A reset
// while a runtime of that device is alive is not supported.
void device_runtime_opened(int device);
void device_runtime_closed(int device);
unsigned long long device_epoch(int device);
constexpr int kMaxDevices = 64;

// ---- primitives (prims.cu) ----
void launch_keystream(Ctx& c, int stream_id, unsigned long long nonce0, void* out, size_t nbytes);
void op_secret_share(Ctx& c, bool arith, int w, size_t n, const void* data_dev, int party, Sh3 s);
void op_public_share(Ctx& c, int w, size_t n, const void* data_dev, Sh3 s);
void op_open(Ctx& c, bool arith, int w, size_t n, CSh3 s, void* out_dev);
void op_mult(Ctx& c, bool arith, int w, size_t n, CSh3 x, CSh3 y, Sh3 z);
void op_local(Ctx& c, int op, int w, size_t n, CSh3 x, CSh3 y, Sh3 z);  // 0 xor,1 add,2 sub
// one party of 3PC (party.cu): local steps before the caller's exchange
void op_party_mult(Ctx& c, bool arith, int w, size_t n, const void* const x[2], const void* const y[2], void* z);
void op_party_b2a_pre(Ctx& c, int w, size_t n, const void* const x[2], void* s0, void* s1);
void op_party_b2a_post(Ctx& c, int w, size_t n, const void* const s0[2], const void* const s1[2], void* z);
void op_party_local(Ctx& c, int op, int w, size_t n, const void* const x[2], const void* const y[2], void* const z[2]);
void op_party_share(Ctx& c, bool arith, int w, size_t n, const void* data_dev, Sh3 s);
void op_party_open(Ctx& c, bool arith, int w, size_t n, const void* const x[2], const void* third, void* out_dev);
void op_not(Ctx& c, int w, size_t n, CSh3 x, Sh3 y);
void op_b2a_bit(Ctx& c, int w, size_t n, CSh3 x, Sh3 y);
void op_a2b(Ctx& c, int w, size_t n, CSh3 x, Sh3 y);
void op_rca(Ctx& c, int w, size_t n, CSh3 a, CSh3 b, Sh3 sum, bool carry_in);
void op_sub_b(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 z);
void op_zero_share(Ctx& c, bool arith, int w, size_t n, Sh3 r);
void op_reshare(Ctx& c, bool arith, int w, size_t n, int group, Sh3 s);

// ---- permutations (perm.cu) ----
void release_fy(Ctx& c);
void gen_sharded_perms(Ctx& c, size_t n, size_t count, std::vector<ShardedPerm>& out);
void reserve_perms(Ctx& c, size_t n, size_t count);
ShardedPerm next_perm(Ctx& c, size_t n);
// y = local permutation of x under one group's permutation followed by that
// group's reshare; idx gives dst[k] = src[idx[k]].
void op_apply_sharded(Ctx& c, bool arith, int w, size_t n, Sh3 s, const ShardedPerm& sp,
                      bool inverse);
void op_apply_elementwise(Ctx& c, bool x_arith, int xw, size_t n, Sh3 x, CSh3 perm /*int32 A*/);
void op_scatter(Ctx& c, int w, size_t n, CSh3 src, Sh3 dst, const int32_t* sigma);
void op_shuffle(Ctx& c, bool arith, int w, size_t n, Sh3 s);

// ---- prefix sum of arithmetic shares (scan.cu) ----
uint32_t prefix_sum_tiles(size_t n);
void op_prefix_sum_into(Ctx& c, int w, size_t n, Sh3 s, void* tsum);
void op_prefix_sum(Ctx& c, int w, size_t n, Sh3 s);
void op_prefix_sum_noalloc(Ctx& c, int w, size_t n, Sh3 s);

// ---- sorting (radix.cu) ----
void op_radix_sort(Ctx& c, int kw, size_t n, Sh3 key, int bits, bool desc, Sh3 perm_out /*int32*/);
// `count` radix sorts whose shares equal `count` op_radix_sort calls in list
// order, run back to back without host synchronisation between items.
void op_radix_sort_batch(Ctx& c, int kw, int count, const size_t* n, void* const* keys, const int* bits,
                         const int* desc, void* const* perms_out);

// ---- compare circuit and bitonic sort (cmp.cu) ----
void op_compare(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 eq, Sh3 gt);
void op_bitonic_sort(Ctx& c, int w, size_t n, Sh3 key, bool desc);
void op_equal(Ctx& c, int w, size_t n, CSh3 x, CSh3 y, Sh3 eq);
void op_not1(Ctx& c, int w, size_t n, CSh3 x, Sh3 y);
// pad_input -> body(padded rows, padded width) -> remove_padding -> invert;
// reserves `reserve` permutations first (radix sort and quicksort share it)
void sort_padded(Ctx& c, int kw, size_t n, Sh3 key, bool desc, Sh3 perm_out, size_t reserve,
                 const std::function<void(Sh3 P, int PW)>& body);
void op_quicksort(Ctx& c, int kw, size_t n, Sh3 key, bool desc, Sh3 perm_out);
void op_table_shuffle(Ctx& c, int w, size_t n, int na, const Sh3* data_a, int nb, const Sh3* data_b);
void op_mask_b(Ctx& c, int w, size_t n, Sh3 s, unsigned long long m);
void op_compare_rows(Ctx& c, int w, size_t n, int nkeys, const CSh3* x, const CSh3* y, const int* desc, Sh3 gt);
void op_swap(Ctx& c, int w, size_t n, bool arith, int ncols, const Sh3* x, const Sh3* y, CSh3 bits);
void op_extend_lsb(Ctx& c, int w, size_t n, CSh3 x, Sh3 y);
void op_bitonic_sort_rows(Ctx& c, int w, size_t n, int nkeys, const Sh3* keys, const int* desc, int na,
                          const Sh3* data_a, int nb, const Sh3* data_b);

// ---- aggregation network (agg.cu) ----
enum AggFunc { AGG_SUM = 0, AGG_COUNT = 1, AGG_COPY = 2, AGG_VALID = 3, AGG_BIT_OR = 4, AGG_MIN = 5, AGG_MAX = 6 };
struct AggSpec {  // same layout as orqcu_agg_spec
    const void* in[3];
    void* out[3];
    int func;
};
void op_aggregate(Ctx& c, int w, size_t n, int nkeys, const void* const* keys, int nb,
                  const AggSpec* bs, int na, const AggSpec* as, bool reverse, const void* const* sel);

// ---- table sort, permutation composition, distinct (tsort.cu) ----
void op_compose(Ctx& c, size_t n, Sh3 sigma, Sh3 rho);  // rho <- compose(sigma, rho)
void op_table_sort(Ctx& c, int w, size_t n, int ncols, const Sh3* cols, const int* desc,
                   const int* single_bit, int na, const Sh3* data_a, int nb, const Sh3* data_b, bool quick);
void op_distinct(Ctx& c, int w, size_t n, int nkeys, const CSh3* keys, Sh3 res);

// ---- batched bitonic sort (cmp.cu) ----
void op_bitonic_sort_batch(Ctx& c, int w, int count, const size_t* n, const Sh3* keys, const int* desc,
                           bool use_graph);

}  // namespace orqcu
