// capi.cu — extern "C" entry points (include/orq_cuda.h).
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/orq_cuda.h"
#include "runtime.h"

struct orqcu_runtime {
    orqcu::Ctx ctx;
};

namespace {

thread_local std::string g_err;

template <typename F>
int guard(F&& f) {
    try {
        f();
        return ORQCU_OK;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return ORQCU_EINVAL;
    } catch (const std::bad_alloc& e) {
        g_err = e.what();
        return ORQCU_ENOMEM;
    } catch (const std::runtime_error& e) {
        g_err = e.what();
        return std::strstr(e.what(), "CUDA error") ? ORQCU_ECUDA : ORQCU_ERUNTIME;
    } catch (...) {
        g_err = "unknown error";
        return ORQCU_ERUNTIME;
    }
}

void need(bool ok, const char* msg) {
    if (!ok) throw std::invalid_argument(msg);
}
// any runtime (memory, streams, profiling)
void need_rt_any(orqcu_runtime* rt) { need(rt != nullptr, "null runtime"); }
// a replicated-3PC runtime (every 3PC protocol and operator entry)
void need_rt(orqcu_runtime* rt) {
    need_rt_any(rt);
    need(rt->ctx.nparties == 3, "this runtime runs the 2PC/4PC protocol; use the orqcu_np_* entry points");
    need(rt->ctx.party < 0, "this runtime plays one party; use the orqcu_party_* entry points");
}
void need_w(int w) { need(w == 1 || w == 2 || w == 4 || w == 8 || w == 16, "width must be 1,2,4,8,16"); }
void need_sh(const void* const s[3], size_t n, const char* what) {
    if (n == 0) return;
    need(s != nullptr && s[0] && s[1] && s[2], what);
}
orqcu::CSh3 c3(const void* const s[3]) { return orqcu::CSh3{{s[0], s[1], s[2]}}; }
orqcu::Sh3 m3(void* const s[3]) { return orqcu::Sh3{{s[0], s[1], s[2]}}; }

}  // namespace

extern "C" {

int orqcu_version(void) { return 1; }
const char* orqcu_last_error(void) { return g_err.c_str(); }

static void create_runtime(uint64_t seed, int device, int nparties, orqcu_runtime** out, int party = -1) {
    need(out != nullptr, "null output");
    need(nparties == 2 || nparties == 3 || nparties == 4, "parties must be 2, 3 or 4");
    int ndev = 0;
    ORQ_CUDA_CHECK(cudaGetDeviceCount(&ndev));
    need(device >= 0 && device < ndev, "no such CUDA device");
    ORQ_CUDA_CHECK(cudaSetDevice(device));
    std::unique_ptr<orqcu_runtime> rt(new orqcu_runtime());
    rt->ctx.device = device;
    ORQ_CUDA_CHECK(cudaDeviceGetAttribute(&rt->ctx.num_sms, cudaDevAttrMultiProcessorCount, device));
    ORQ_CUDA_CHECK(cudaStreamCreateWithFlags(&rt->ctx.stream, cudaStreamNonBlocking));
    rt->ctx.owns_stream = true;
    ORQ_CUDA_CHECK(cudaMalloc(&rt->ctx.d_err, sizeof(int)));
    ORQ_CUDA_CHECK(cudaMemset(rt->ctx.d_err, 0, sizeof(int)));
    if (party >= 0) {
        // one party: its keys arrive through orqcu_party_set_key
        rt->ctx.party = party;
        for (int s = 0; s < orqcu::NSTREAMS; s++) std::memset(rt->ctx.rk[s].k, 0, sizeof(rt->ctx.rk[s].k));
    } else if (nparties == 3) {
        orqcu::init_ctx_keys(rt->ctx, seed);
    } else {
        orqcu::init_ctx_keys_np(rt->ctx, seed, nparties);
    }
    orqcu::keep_pool_memory(device);
    orqcu::device_runtime_opened(device);
    try {
        orqcu::upload_aes_tables(device);
    } catch (...) {
        orqcu::device_runtime_closed(device);
        throw;
    }
    *out = rt.release();
}

int orqcu_runtime_create(uint64_t seed, int device, orqcu_runtime** out) {
    return guard([&] { create_runtime(seed, device, 3, out); });
}

int orqcu_runtime_create_np(uint64_t seed, int device, int nparties, orqcu_runtime** out) {
    return guard([&] { create_runtime(seed, device, nparties, out); });
}

int orqcu_runtime_parties(orqcu_runtime* rt, int* nparties) {
    return guard([&] {
        need_rt_any(rt);
        need(nparties != nullptr, "null output");
        *nparties = rt->ctx.nparties;
    });
}

// ---- one party of 3PC --------------------------------------------------------
static void need_party_rt(orqcu_runtime* rt) {
    need_rt_any(rt);
    need(rt->ctx.party >= 0, "this runtime plays every party; create one with orqcu_party_runtime_create");
}
static void need2(const void* const* s, size_t n, const char* what) {
    if (n == 0) return;
    need(s != nullptr && s[0] && s[1], what);
}

int orqcu_party_runtime_create(int party, int device, orqcu_runtime** out) {
    return guard([&] {
        need(party >= 0 && party <= 2, "party must be 0, 1 or 2");
        create_runtime(0, device, 3, out, party);
    });
}

int orqcu_party_set_key(orqcu_runtime* rt, int slot, const uint8_t key[32]) {
    return guard([&] {
        need_party_rt(rt);
        need(key != nullptr, "null key");
        const int p = rt->ctx.party;
        int s;
        switch (slot) {
            case ORQCU_PKEY_LOCAL: s = orqcu::LOCAL0 + p; break;
            case ORQCU_PKEY_NEXT: s = orqcu::PAIR0 + p; break;
            case ORQCU_PKEY_PREV: s = orqcu::PAIR0 + (p + 2) % 3; break;
            case ORQCU_PKEY_G01: s = orqcu::G01; break;
            case ORQCU_PKEY_G02: s = orqcu::G02; break;
            case ORQCU_PKEY_G12: s = orqcu::G12; break;
            case ORQCU_PKEY_G012: s = orqcu::G012; break;
            default: throw std::invalid_argument("unknown key slot");
        }
        orqcu::aes256_expand(key, rt->ctx.rk[s].k);
        rt->ctx.nonce[s] = 0;
    });
}

int orqcu_keygen(uint64_t seed, int party, int call, uint8_t key[32]) {
    return guard([&] {
        need(key != nullptr, "null key");
        need(party >= 0 && call >= 0, "party and call must be non-negative");
        orqcu::derive_key(seed, party, call, key);
    });
}

int orqcu_party_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data_dev,
                             void* const s[3]) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need_sh(s, n, "null share pointer");
        need(n == 0 || data_dev != nullptr, "null data");
        orqcu::op_party_share(rt->ctx, arith != 0, width, n, data_dev, m3(s));
    });
}

static int party_mult(orqcu_runtime* rt, bool arith, int width, size_t n, const void* const x[2],
                      const void* const y[2], void* z) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need2(x, n, "null share pointer");
        need2(y, n, "null share pointer");
        need(n == 0 || z != nullptr, "null output");
        orqcu::op_party_mult(rt->ctx, arith, width, n, x, y, z);
    });
}
int orqcu_party_and_b(orqcu_runtime* rt, int width, size_t n, const void* const x[2], const void* const y[2],
                      void* z) {
    return party_mult(rt, false, width, n, x, y, z);
}
int orqcu_party_multiply_a(orqcu_runtime* rt, int width, size_t n, const void* const x[2],
                           const void* const y[2], void* z) {
    return party_mult(rt, true, width, n, x, y, z);
}

int orqcu_party_b2a_pre(orqcu_runtime* rt, int width, size_t n, const void* const x[2], void* s0, void* s1) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need2(x, n, "null share pointer");
        need(n == 0 || (s0 && s1), "null output");
        orqcu::op_party_b2a_pre(rt->ctx, width, n, x, s0, s1);
    });
}

int orqcu_party_b2a_post(orqcu_runtime* rt, int width, size_t n, const void* const s0[2],
                         const void* const s1[2], void* z) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need2(s0, n, "null share pointer");
        need2(s1, n, "null share pointer");
        need(n == 0 || z != nullptr, "null output");
        orqcu::op_party_b2a_post(rt->ctx, width, n, s0, s1, z);
    });
}

int orqcu_party_local(orqcu_runtime* rt, int op, int width, size_t n, const void* const x[2],
                      const void* const y[2], void* const z[2]) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need(op >= 0 && op <= 2, "op must be 0 (xor), 1 (add) or 2 (sub)");
        need2(x, n, "null share pointer");
        need2(y, n, "null share pointer");
        need2(z, n, "null output");
        orqcu::op_party_local(rt->ctx, op, width, n, x, y, z);
    });
}

int orqcu_party_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const x[2],
                     const void* third, void* out_dev) {
    return guard([&] {
        need_party_rt(rt);
        need_w(width);
        need2(x, n, "null share pointer");
        need(n == 0 || (third && out_dev), "null pointer");
        orqcu::op_party_open(rt->ctx, arith != 0, width, n, x, third, out_dev);
    });
}

// ---- Beaver 2PC / Fantastic-4PC ----------------------------------------------
static void need_np_rt(orqcu_runtime* rt) {
    need_rt_any(rt);
    need(rt->ctx.nparties == 2 || rt->ctx.nparties == 4,
         "this runtime runs replicated 3PC; create one with orqcu_runtime_create_np");
}
static void need_shares(const void* const* s, int np, size_t n, const char* what) {
    if (n == 0) return;
    need(s != nullptr, what);
    for (int k = 0; k < np; k++) need(s[k] != nullptr, what);
}

int orqcu_np_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data_dev,
                          int data_party, void* const* shares) {
    return guard([&] {
        need_np_rt(rt);
        need_shares(shares, rt->ctx.nparties, n, "null share pointer");
        need(n == 0 || data_dev != nullptr, "null data");
        orqcu::op_np_secret_share(rt->ctx, arith != 0, width, n, data_dev, data_party, shares);
    });
}

int orqcu_np_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const* shares, void* out_dev) {
    return guard([&] {
        need_np_rt(rt);
        need_shares(shares, rt->ctx.nparties, n, "null share pointer");
        need(n == 0 || out_dev != nullptr, "null output");
        orqcu::op_np_open(rt->ctx, arith != 0, width, n, shares, out_dev);
    });
}

static int np_bin(orqcu_runtime* rt, int mode, int width, size_t n, const void* const* x, const void* const* y,
                  void* const* z) {
    return guard([&] {
        need_np_rt(rt);
        need_shares(x, rt->ctx.nparties, n, "null x");
        if (mode != 2) need_shares(y, rt->ctx.nparties, n, "null y");
        need_shares(z, rt->ctx.nparties, n, "null z");
        orqcu::op_np_mult(rt->ctx, mode, width, n, x, y, z);
    });
}
int orqcu_np_and_b(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z) {
    return np_bin(rt, 0, width, n, x, y, z);
}
int orqcu_np_multiply_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                        void* const* z) {
    return np_bin(rt, 1, width, n, x, y, z);
}
int orqcu_np_b2a_bit(orqcu_runtime* rt, int width, size_t n, const void* const* x, void* const* y) {
    return np_bin(rt, 2, width, n, x, nullptr, y);
}

static int np_local(orqcu_runtime* rt, int op, int width, size_t n, const void* const* x, const void* const* y,
                    void* const* z) {
    return guard([&] {
        need_np_rt(rt);
        need_shares(x, rt->ctx.nparties, n, "null x");
        need_shares(y, rt->ctx.nparties, n, "null y");
        need_shares(z, rt->ctx.nparties, n, "null z");
        orqcu::op_np_local(rt->ctx, op, width, n, x, y, z);
    });
}
int orqcu_np_xor_b(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z) {
    return np_local(rt, 0, width, n, x, y, z);
}
int orqcu_np_add_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z) {
    return np_local(rt, 1, width, n, x, y, z);
}
int orqcu_np_sub_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z) {
    return np_local(rt, 2, width, n, x, y, z);
}

int orqcu_runtime_destroy(orqcu_runtime* rt) {
    return guard([&] {
        if (!rt) return;
        cudaSetDevice(rt->ctx.device);
        cudaStreamSynchronize(rt->ctx.stream);
        for (auto& sp : rt->ctx.perm_queue) rt->ctx.free_perm(sp);
        rt->ctx.perm_queue.clear();
        rt->ctx.release_graphs();
        orqcu::release_fy(rt->ctx);
        if (rt->ctx.owns_stream) cudaStreamDestroy(rt->ctx.stream);
        if (rt->ctx.d_err) cudaFree(rt->ctx.d_err);
        const int device = rt->ctx.device;
        delete rt;  // its pool's blocks go back to the device pool first
        orqcu::device_runtime_closed(device);
    });
}

int orqcu_runtime_set_stream(orqcu_runtime* rt, void* s) {
    return guard([&] {
        need_rt_any(rt);
        cudaSetDevice(rt->ctx.device);
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
        if (rt->ctx.owns_stream) cudaStreamDestroy(rt->ctx.stream);
        rt->ctx.stream = (cudaStream_t)s;  // NULL = the CUDA default stream
        rt->ctx.owns_stream = false;
    });
}

int orqcu_synchronize(orqcu_runtime* rt) {
    return guard([&] {
        need_rt_any(rt);
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
        rt->ctx.check_device_error();
    });
}

int orqcu_get_nonce(orqcu_runtime* rt, int stream, uint64_t* nonce) {
    return guard([&] {
        need_rt_any(rt);
        need(stream >= 0 && stream < orqcu::NSTREAMS && nonce, "bad stream id");
        *nonce = rt->ctx.nonce[stream];
    });
}

int orqcu_kernels_launched(orqcu_runtime* rt, uint64_t* count) {
    return guard([&] {
        need_rt_any(rt);
        need(count != nullptr, "null output");
        *count = rt->ctx.kernels_launched;
    });
}

int orqcu_profile_enable(orqcu_runtime* rt, int on) {
    return guard([&] {
        need_rt_any(rt);
        rt->ctx.prof_collect();
        rt->ctx.profiling = on != 0;
    });
}

int orqcu_profile_report(orqcu_runtime* rt, char* buf, size_t len) {
    return guard([&] {
        need_rt_any(rt);
        need(buf != nullptr && len > 0, "null buffer");
        rt->ctx.prof_collect();
        std::string out;
        for (auto& kv : rt->ctx.prof_agg) {
            char line[256];
            snprintf(line, sizeof(line), "%s %llu %.6f %.0f %.0f\n", kv.first.c_str(),
                     kv.second.launches, kv.second.ms, kv.second.bytes, kv.second.aes_blocks);
            out += line;
        }
        rt->ctx.prof_agg.clear();
        need(out.size() < len, "report buffer too small");
        std::memcpy(buf, out.c_str(), out.size() + 1);
    });
}

int orqcu_malloc(orqcu_runtime* rt, size_t bytes, void** dptr) {
    return guard([&] {
        need_rt_any(rt);
        need(dptr != nullptr, "null output");
        cudaSetDevice(rt->ctx.device);
        ORQ_CUDA_CHECK(cudaMalloc(dptr, bytes ? bytes : 1));
    });
}
int orqcu_free(orqcu_runtime* rt, void* dptr) {
    return guard([&] {
        need_rt_any(rt);
        ORQ_CUDA_CHECK(cudaFree(dptr));
    });
}
int orqcu_memcpy_h2d(orqcu_runtime* rt, void* dst, const void* src, size_t bytes) {
    return guard([&] {
        need_rt_any(rt);
        if (!bytes) return;
        ORQ_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, rt->ctx.stream));
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
    });
}
int orqcu_memcpy_d2h(orqcu_runtime* rt, void* dst, const void* src, size_t bytes) {
    return guard([&] {
        need_rt_any(rt);
        if (!bytes) return;
        ORQ_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, rt->ctx.stream));
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
    });
}

int orqcu_pool_alloc(orqcu_runtime* rt, size_t bytes, void** dptr) {
    return guard([&] {
        need_rt_any(rt);
        need(dptr != nullptr, "null output");
        cudaSetDevice(rt->ctx.device);
        *dptr = rt->ctx.alloc(bytes ? bytes : 1);
    });
}
int orqcu_pool_free(orqcu_runtime* rt, void* dptr) {
    return guard([&] {
        need_rt_any(rt);
        rt->ctx.release(dptr);
    });
}
int orqcu_memcpy_d2d(orqcu_runtime* rt, void* dst, const void* src, size_t bytes) {
    return guard([&] {
        need_rt_any(rt);
        if (!bytes) return;
        need(dst != nullptr && src != nullptr, "null pointer");
        ORQ_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, rt->ctx.stream));
    });
}
int orqcu_memset(orqcu_runtime* rt, void* dst, int byte, size_t bytes) {
    return guard([&] {
        need_rt_any(rt);
        if (!bytes) return;
        need(dst != nullptr, "null pointer");
        ORQ_CUDA_CHECK(cudaMemsetAsync(dst, byte & 0xff, bytes, rt->ctx.stream));
    });
}

int orqcu_keystream(orqcu_runtime* rt, int stream, uint64_t nonce0, size_t nbytes, void* out) {
    return guard([&] {
        need_rt_any(rt);
        need(stream >= 0 && stream < orqcu::NSTREAMS, "bad stream id");
        need(out != nullptr || nbytes == 0, "null output");
        orqcu::launch_keystream(rt->ctx, stream, nonce0, out, nbytes);
    });
}

int orqcu_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data,
                       int data_party, void* const shares[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh((const void* const*)shares, n, "null share pointer");
        need(data != nullptr || n == 0, "null data");
        orqcu::op_secret_share(rt->ctx, arith != 0, width, n, data, data_party, m3(shares));
    });
}

int orqcu_public_share(orqcu_runtime* rt, int width, size_t n, const void* data, void* const shares[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh((const void* const*)shares, n, "null share pointer");
        orqcu::op_public_share(rt->ctx, width, n, data, m3(shares));
    });
}

int orqcu_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const shares[3], void* out) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh(shares, n, "null share pointer");
        orqcu::op_open(rt->ctx, arith != 0, width, n, c3(shares), out);
    });
}

static int binop(orqcu_runtime* rt, int kind, int width, size_t n, const void* const x[3],
                 const void* const y[3], void* const z[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh(x, n, "null x");
        need_sh(y, n, "null y");
        need_sh((const void* const*)z, n, "null z");
        switch (kind) {
            case 0: orqcu::op_mult(rt->ctx, false, width, n, c3(x), c3(y), m3(z)); break;
            case 1: orqcu::op_mult(rt->ctx, true, width, n, c3(x), c3(y), m3(z)); break;
            case 2: orqcu::op_local(rt->ctx, 0, width, n, c3(x), c3(y), m3(z)); break;
            case 3: orqcu::op_local(rt->ctx, 1, width, n, c3(x), c3(y), m3(z)); break;
            case 4: orqcu::op_local(rt->ctx, 2, width, n, c3(x), c3(y), m3(z)); break;
        }
    });
}

int orqcu_and_b(orqcu_runtime* rt, int w, size_t n, const void* const x[3], const void* const y[3], void* const z[3]) {
    return binop(rt, 0, w, n, x, y, z);
}
int orqcu_multiply_a(orqcu_runtime* rt, int w, size_t n, const void* const x[3], const void* const y[3], void* const z[3]) {
    return binop(rt, 1, w, n, x, y, z);
}
int orqcu_xor_b(orqcu_runtime* rt, int w, size_t n, const void* const x[3], const void* const y[3], void* const z[3]) {
    return binop(rt, 2, w, n, x, y, z);
}
int orqcu_add_a(orqcu_runtime* rt, int w, size_t n, const void* const x[3], const void* const y[3], void* const z[3]) {
    return binop(rt, 3, w, n, x, y, z);
}
int orqcu_sub_a(orqcu_runtime* rt, int w, size_t n, const void* const x[3], const void* const y[3], void* const z[3]) {
    return binop(rt, 4, w, n, x, y, z);
}

int orqcu_not_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh(x, n, "null x");
        need_sh((const void* const*)y, n, "null y");
        orqcu::op_not(rt->ctx, width, n, c3(x), m3(y));
    });
}

int orqcu_b2a_bit(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh(x, n, "null x");
        need_sh((const void* const*)y, n, "null y");
        orqcu::op_b2a_bit(rt->ctx, width, n, c3(x), m3(y));
    });
}

int orqcu_zero_share(orqcu_runtime* rt, int arith, int width, size_t n, void* const r[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh((const void* const*)r, n, "null r");
        orqcu::op_zero_share(rt->ctx, arith != 0, width, n, m3(r));
    });
}

int orqcu_reshare(orqcu_runtime* rt, int arith, int width, size_t n, int group, void* const s[3]) {
    return guard([&] {
        need_rt(rt);
        need_w(width);
        need_sh((const void* const*)s, n, "null shares");
        orqcu::op_reshare(rt->ctx, arith != 0, width, n, group, m3(s));
    });
}

int orqcu_prefix_sum_a(orqcu_runtime* rt, int width, size_t n, void* const shares[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "prefix sum supports 4 and 8-byte shares");
        need_sh((const void* const*)shares, n, "null shares");
        orqcu::op_prefix_sum(rt->ctx, width, n, m3(shares));
    });
}

int orqcu_prefix_sum_a_noalloc(orqcu_runtime* rt, int width, size_t n, void* const shares[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "prefix sum supports 4 and 8-byte shares");
        need_sh((const void* const*)shares, n, "null shares");
        ORQ_CUDA_CHECK(cudaSetDevice(rt->ctx.device));
        orqcu::op_prefix_sum_noalloc(rt->ctx, width, n, m3(shares));
    });
}

int orqcu_reserve_permutations(orqcu_runtime* rt, size_t n, size_t count) {
    return guard([&] {
        need_rt(rt);
        orqcu::reserve_perms(rt->ctx, n, count);
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
    });
}

int orqcu_next_permutation(orqcu_runtime* rt, size_t n, int32_t* const perm_dev[3]) {
    return guard([&] {
        need_rt(rt);
        need(perm_dev != nullptr, "null output");
        orqcu::ShardedPerm sp = orqcu::next_perm(rt->ctx, n);
        for (int g = 0; g < 3; g++)
            if (n)
                ORQ_CUDA_CHECK(cudaMemcpyAsync(perm_dev[g], sp.perm[g], n * 4, cudaMemcpyDeviceToDevice,
                                               rt->ctx.stream));
        ORQ_CUDA_CHECK(cudaStreamSynchronize(rt->ctx.stream));
        rt->ctx.free_perm(sp);
    });
}

int orqcu_shuffle(orqcu_runtime* rt, int arith, int width, size_t n, void* const s[3]) {
    return guard([&] {
        need_rt(rt);
        need_sh((const void* const*)s, n, "null shares");
        orqcu::op_shuffle(rt->ctx, arith != 0, width, n, m3(s));
    });
}

int orqcu_apply_elementwise_perm(orqcu_runtime* rt, int x_arith, int x_width, size_t n,
                                 void* const x[3], const void* const perm[3]) {
    return guard([&] {
        need_rt(rt);
        need_sh((const void* const*)x, n, "null x");
        need_sh(perm, n, "null perm");
        orqcu::op_apply_elementwise(rt->ctx, x_arith != 0, x_width, n, m3(x), c3(perm));
    });
}

int orqcu_radix_sort(orqcu_runtime* rt, int key_width, size_t n, void* const key[3], int bits,
                     int descending, void* const perm_out[3]) {
    return guard([&] {
        need_rt(rt);
        need_sh((const void* const*)key, n, "null key");
        need_sh((const void* const*)perm_out, n, "null perm_out");
        orqcu::op_radix_sort(rt->ctx, key_width, n, m3(key), bits, descending != 0, m3(perm_out));
        rt->ctx.check_device_error();
    });
}


int orqcu_radix_sort_batch(orqcu_runtime* rt, int key_width, int count, const size_t* n, void* const* keys,
                           const int* bits, const int* descending, void* const* perms_out) {
    return guard([&] {
        need_rt(rt);
        need(count >= 0, "negative count");
        if (count == 0) return;
        need(n && keys && bits && descending && perms_out, "null argument");
        for (int k = 0; k < count; k++) {
            need_sh(keys + 3 * k, n[k], "null key share pointer");
            need_sh(perms_out + 3 * k, n[k], "null permutation share pointer");
        }
        orqcu::op_radix_sort_batch(rt->ctx, key_width, count, n, keys, bits, descending, perms_out);
    });
}

int orqcu_quicksort(orqcu_runtime* rt, int key_width, size_t n, void* const key[3], int descending,
                    void* const perm_out[3]) {
    return guard([&] {
        need_rt(rt);
        need(key_width == 4 || key_width == 8, "quicksort keys must be int32 or int64");
        need_sh((const void* const*)key, n, "null key");
        need_sh((const void* const*)perm_out, n, "null perm_out");
        orqcu::op_quicksort(rt->ctx, key_width, n, m3(key), descending != 0, m3(perm_out));
        rt->ctx.check_device_error();
    });
}

int orqcu_compare_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                    const void* const y[3], void* const eq[3], void* const gt[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8 || width == 16, "compare supports 4, 8 and 16-byte keys");
        need_sh(x, n, "null x");
        need_sh(y, n, "null y");
        need_sh((const void* const*)eq, n, "null eq");
        need_sh((const void* const*)gt, n, "null gt");
        orqcu::op_compare(rt->ctx, width, n, c3(x), c3(y), m3(eq), m3(gt));
    });
}

int orqcu_bitonic_sort(orqcu_runtime* rt, int width, size_t n, void* const key[3],
                       int descending) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "bitonic sort supports 4 and 8-byte keys");
        need((n & (n - 1)) == 0, "bitonic sort needs a power-of-two size");
        need_sh((const void* const*)key, n, "null key");
        orqcu::op_bitonic_sort(rt->ctx, width, n, m3(key), descending != 0);
    });
}

int orqcu_aggregate(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* keys,
                    int nb, const orqcu_agg_spec* b_specs, int na, const orqcu_agg_spec* a_specs,
                    int reverse, const void* const* sel) {
    static_assert(sizeof(orqcu_agg_spec) == sizeof(orqcu::AggSpec), "agg spec layout");
    return guard([&] {
        need_rt(rt);
        need(nkeys >= 0 && nb >= 0 && na >= 0, "negative column count");
        need(nkeys == 0 || keys != nullptr, "null keys");
        need(nb == 0 || b_specs != nullptr, "null boolean specs");
        need(na == 0 || a_specs != nullptr, "null arithmetic specs");
        for (int j = 0; j < nkeys; j++) need_sh(keys + 3 * j, n, "null key share");
        for (int s = 0; s < nb; s++) {
            need_sh(b_specs[s].in, n, "null spec input");
            need_sh((const void* const*)b_specs[s].out, n, "null spec output");
        }
        for (int s = 0; s < na; s++) {
            if (a_specs[s].func != ORQCU_AGG_COUNT) need_sh(a_specs[s].in, n, "null spec input");
            need_sh((const void* const*)a_specs[s].out, n, "null spec output");
        }
        if (sel) need_sh(sel, n, "null sel share");
        orqcu::op_aggregate(rt->ctx, width, n, nkeys, keys, nb,
                            reinterpret_cast<const orqcu::AggSpec*>(b_specs), na,
                            reinterpret_cast<const orqcu::AggSpec*>(a_specs), reverse != 0, sel);
    });
}

int orqcu_compose_permutations(orqcu_runtime* rt, size_t n, void* const sigma[3],
                               void* const rho[3]) {
    return guard([&] {
        need_rt(rt);
        need_sh((const void* const*)sigma, n, "null sigma");
        need_sh((const void* const*)rho, n, "null rho");
        orqcu::op_compose(rt->ctx, n, m3(sigma), m3(rho));
        rt->ctx.check_device_error();
    });
}

int orqcu_table_sort(orqcu_runtime* rt, int width, size_t n, int ncols, void* const* cols,
                     const int* descending, const int* single_bit, int na, void* const* data_a,
                     int nb, void* const* data_b, int protocol) {
    return guard([&] {
        need_rt(rt);
        need(protocol == ORQCU_SORT_QUICK || protocol == ORQCU_SORT_RADIX, "Unknown table sort protocol");
        need(ncols >= 1 && cols && descending && single_bit, "table sort needs key columns");
        need(na >= 0 && nb >= 0 && (na == 0 || data_a) && (nb == 0 || data_b), "bad data columns");
        need(n < (1ull << 31), "table sort supports n < 2^31");
        std::vector<orqcu::Sh3> k(ncols), a(na), b(nb);
        for (int i = 0; i < ncols; i++) {
            need_sh((const void* const*)cols + 3 * i, n, "null key column");
            k[i] = m3(cols + 3 * i);
        }
        for (int i = 0; i < na; i++) {
            need_sh((const void* const*)data_a + 3 * i, n, "null data column");
            a[i] = m3(data_a + 3 * i);
        }
        for (int i = 0; i < nb; i++) {
            need_sh((const void* const*)data_b + 3 * i, n, "null data column");
            b[i] = m3(data_b + 3 * i);
        }
        orqcu::op_table_sort(rt->ctx, width, n, ncols, k.data(), descending, single_bit, na, a.data(),
                             nb, b.data(), protocol == ORQCU_SORT_QUICK);
        rt->ctx.check_device_error();
    });
}

int orqcu_distinct(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* keys,
                   void* const res[3]) {
    return guard([&] {
        need_rt(rt);
        need(nkeys >= 1 && keys, "distinct needs key columns");
        std::vector<orqcu::CSh3> k(nkeys);
        for (int i = 0; i < nkeys; i++) {
            need_sh(keys + 3 * i, n, "null key column");
            k[i] = c3(keys + 3 * i);
        }
        need_sh((const void* const*)res, n, "null res");
        orqcu::op_distinct(rt->ctx, width, n, nkeys, k.data(), m3(res));
    });
}

int orqcu_bitonic_sort_batch(orqcu_runtime* rt, int width, int count, const size_t* n,
                             void* const* keys, const int* descending, int use_graph) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "bitonic sort supports 4 and 8-byte keys");
        need(count >= 0 && (count == 0 || (n && keys && descending)), "bad batch");
        std::vector<orqcu::Sh3> k(count);
        for (int i = 0; i < count; i++) {
            need((n[i] & (n[i] - 1)) == 0, "bitonic sort needs power-of-two sizes");
            need(n[i] < (1ull << 32), "bitonic batch items must have fewer than 2^32 rows");
            need_sh((const void* const*)keys + 3 * i, n[i], "null key share");
            k[i] = m3(keys + 3 * i);
        }
        orqcu::op_bitonic_sort_batch(rt->ctx, width, count, n, k.data(), descending, use_graph != 0);
    });
}

int orqcu_runtime_reseed(orqcu_runtime* rt, uint64_t seed) {
    return guard([&] {
        need_rt_any(rt);
        need(rt->ctx.party < 0, "a one-party runtime takes its keys from orqcu_party_set_key");
        for (auto& sp : rt->ctx.perm_queue) rt->ctx.free_perm(sp);
        rt->ctx.perm_queue.clear();
        rt->ctx.perm_queue_n = 0;
        if (rt->ctx.nparties == 3) orqcu::init_ctx_keys(rt->ctx, seed);
        else orqcu::init_ctx_keys_np(rt->ctx, seed, rt->ctx.nparties);
        for (int s = 0; s < orqcu::NSTREAMS; s++) rt->ctx.nonce[s] = 0;
    });
}

int orqcu_runtime_trim(orqcu_runtime* rt, size_t* cached_before) {
    return guard([&] {
        need_rt_any(rt);
        if (cached_before) *cached_before = rt->ctx.pool.cached_bytes();
        rt->ctx.pool.trim(rt->ctx.stream);
    });
}

int orqcu_runtime_set_sm_limit(orqcu_runtime* rt, int sms) {
    return guard([&] {
        need_rt_any(rt);
        int total = 0;
        ORQ_CUDA_CHECK(cudaDeviceGetAttribute(&total, cudaDevAttrMultiProcessorCount, rt->ctx.device));
        need(sms >= 0, "negative SM limit");
        rt->ctx.num_sms = (sms == 0 || sms > total) ? total : std::max(sms, 4);
    });
}

int orqcu_equal_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                  const void* const y[3], void* const eq[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8 || width == 16, "equality supports 4, 8 and 16-byte keys");
        need_sh(x, n, "null x");
        need_sh(y, n, "null y");
        need_sh((const void* const*)eq, n, "null eq");
        orqcu::op_equal(rt->ctx, width, n, c3(x), c3(y), m3(eq));
    });
}

int orqcu_not_b_1(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "not_b_1 supports 4 and 8-byte shares");
        need_sh(x, n, "null x");
        need_sh((const void* const*)y, n, "null y");
        orqcu::op_not1(rt->ctx, width, n, c3(x), m3(y));
    });
}

int orqcu_add_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], const void* const y[3],
                void* const z[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "the boolean adder supports 4 and 8-byte shares");
        need_sh(x, n, "null x");
        need_sh(y, n, "null y");
        need_sh((const void* const*)z, n, "null z");
        for (int j = 0; j < 3; j++) need(n == 0 || (z[j] != x[j] && z[j] != y[j]), "z must not alias x or y");
        orqcu::op_rca(rt->ctx, width, n, c3(x), c3(y), m3(z), false);
    });
}

int orqcu_sub_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], const void* const y[3],
                void* const z[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "the boolean adder supports 4 and 8-byte shares");
        need_sh(x, n, "null x");
        need_sh(y, n, "null y");
        need_sh((const void* const*)z, n, "null z");
        for (int j = 0; j < 3; j++) need(n == 0 || (z[j] != x[j] && z[j] != y[j]), "z must not alias x or y");
        orqcu::op_sub_b(rt->ctx, width, n, c3(x), c3(y), m3(z));
    });
}

int orqcu_a2b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "a2b supports 4 and 8-byte shares");
        need_sh(x, n, "null x");
        need_sh((const void* const*)y, n, "null y");
        for (int j = 0; j < 3; j++) need(n == 0 || x[j] != y[j], "a2b output must not alias its input");
        orqcu::op_a2b(rt->ctx, width, n, c3(x), m3(y));
    });
}

int orqcu_table_shuffle(orqcu_runtime* rt, int width, size_t n, int na, void* const* data_a, int nb,
                        void* const* data_b) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "table shuffle supports 4 and 8-byte columns");
        need(na >= 0 && nb >= 0 && (na == 0 || data_a) && (nb == 0 || data_b), "bad data columns");
        need(n < (1ull << 31), "table shuffle supports n < 2^31");
        std::vector<orqcu::Sh3> a(na), b(nb);
        for (int i = 0; i < na; i++) {
            need_sh((const void* const*)data_a + 3 * i, n, "null data column");
            a[i] = m3(data_a + 3 * i);
        }
        for (int i = 0; i < nb; i++) {
            need_sh((const void* const*)data_b + 3 * i, n, "null data column");
            b[i] = m3(data_b + 3 * i);
        }
        orqcu::op_table_shuffle(rt->ctx, width, n, na, a.data(), nb, b.data());
        rt->ctx.check_device_error();
    });
}

int orqcu_mask_b(orqcu_runtime* rt, int width, size_t n, void* const shares[3], uint64_t mask) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "mask supports 4 and 8-byte shares");
        need_sh((const void* const*)shares, n, "null shares");
        orqcu::op_mask_b(rt->ctx, width, n, m3(shares), mask);
    });
}

int orqcu_extend_lsb(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "extend_lsb supports 4 and 8-byte shares");
        need_sh(x, n, "null x");
        need_sh((const void* const*)y, n, "null y");
        orqcu::op_extend_lsb(rt->ctx, width, n, c3(x), m3(y));
    });
}

int orqcu_compare_rows(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* x,
                       const void* const* y, const int* descending, void* const gt[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "compare_rows supports 4 and 8-byte keys");
        need(nkeys >= 1 && nkeys <= 8, "compare_rows takes 1 to 8 key columns");
        need(x && y && descending, "null key arrays");
        std::vector<orqcu::CSh3> xs(nkeys), ys(nkeys);
        for (int k = 0; k < nkeys; k++) {
            need_sh(x + 3 * k, n, "null x key");
            need_sh(y + 3 * k, n, "null y key");
            xs[k] = c3(x + 3 * k);
            ys[k] = c3(y + 3 * k);
        }
        need_sh((const void* const*)gt, n, "null gt");
        orqcu::op_compare_rows(rt->ctx, width, n, nkeys, xs.data(), ys.data(), descending, m3(gt));
    });
}

int orqcu_swap(orqcu_runtime* rt, int arith, int width, size_t n, int ncols, void* const* x,
               void* const* y, const void* const bits[3]) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "swap supports 4 and 8-byte shares");
        need(ncols >= 0 && ncols <= 40, "swap takes 0 to 40 column pairs");
        need(ncols == 0 || (x && y), "null column arrays");
        need_sh(bits, n, "null bits");
        std::vector<orqcu::Sh3> xs(ncols), ys(ncols);
        for (int k = 0; k < ncols; k++) {
            need_sh((const void* const*)x + 3 * k, n, "null x column");
            need_sh((const void* const*)y + 3 * k, n, "null y column");
            for (int j = 0; j < 3; j++) need(x[3 * k + j] != y[3 * k + j], "swap columns x and y must differ");
            xs[k] = m3(x + 3 * k);
            ys[k] = m3(y + 3 * k);
        }
        orqcu::op_swap(rt->ctx, width, n, arith != 0, ncols, xs.data(), ys.data(), c3(bits));
    });
}

int orqcu_bitonic_sort_rows(orqcu_runtime* rt, int width, size_t n, int nkeys, void* const* keys,
                            const int* descending, int na, void* const* data_a, int nb,
                            void* const* data_b) {
    return guard([&] {
        need_rt(rt);
        need(width == 4 || width == 8, "bitonic sort supports 4 and 8-byte keys");
        need((n & (n - 1)) == 0, "bitonic sort needs a power-of-two size");
        need(nkeys >= 1 && nkeys <= 8, "bitonic sort takes 1 to 8 key columns");
        need(na >= 0 && nb >= 0 && nkeys + na + nb <= 40, "bitonic sort takes at most 40 columns");
        need(keys && descending && (na == 0 || data_a) && (nb == 0 || data_b), "null column arrays");
        std::vector<orqcu::Sh3> k(nkeys), a(na), b(nb);
        for (int i = 0; i < nkeys; i++) {
            need_sh((const void* const*)keys + 3 * i, n, "null key column");
            k[i] = m3(keys + 3 * i);
        }
        for (int i = 0; i < na; i++) {
            need_sh((const void* const*)data_a + 3 * i, n, "null A data column");
            a[i] = m3(data_a + 3 * i);
        }
        for (int i = 0; i < nb; i++) {
            need_sh((const void* const*)data_b + 3 * i, n, "null B data column");
            b[i] = m3(data_b + 3 * i);
        }
        orqcu::op_bitonic_sort_rows(rt->ctx, width, n, nkeys, k.data(), descending, na, a.data(), nb,
                                    b.data());
    });
}

}  // extern "C"
