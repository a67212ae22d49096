// runtime.hpp — the loopback RunTime: one process plays all three parties of
// replicated 3PC on one GPU, behind the C ABI of liborq_cuda.so.
//
// It stands in for ORQ's per-party RunTime (include/backend/common/
// runtime.h:123-144, whose generated protocol dispatchers and_b, multiply_a,
// b2a_bit, open_shares_*, secret_share_* ... each run one party's local step
// and a socket exchange). Here one call runs the local step of all parties
// and the exchange is a property of the share layout (party p holds S[p] and
// S[p+1]). Host code stays C++; every device operation is a C-ABI call.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../orq_cuda.h"

namespace orq {

// A failed C-ABI call: the reference's asserts and std::runtime_errors become
// this exception, carrying the library's message.
struct RuntimeError : std::runtime_error {
    int code;
    RuntimeError(int rc, const std::string& msg) : std::runtime_error(msg), code(rc) {}
};

inline void orqcu_check(int rc) {
    if (rc != ORQCU_OK) {
        const char* m = orqcu_last_error();
        throw RuntimeError(rc, m ? m : "liborq_cuda error");
    }
}

// Plaintext host vector (orq::Vector, core/containers/mapping_access_vector.h)
// with the elementwise arithmetic the reference's tests compare against.
template <typename T>
class Vector {
    std::vector<T> v_;

   public:
    using value_type = T;
    Vector() = default;
    explicit Vector(size_t n) : v_(n) {}
    Vector(size_t n, T fill) : v_(n, fill) {}
    Vector(std::initializer_list<T> l) : v_(l) {}
    explicit Vector(std::vector<T> v) : v_(std::move(v)) {}
    size_t size() const { return v_.size(); }
    T& operator[](size_t i) { return v_[i]; }
    const T& operator[](size_t i) const { return v_[i]; }
    T* data() { return v_.data(); }
    const T* data() const { return v_.data(); }
    auto begin() { return v_.begin(); }
    auto end() { return v_.end(); }
    auto begin() const { return v_.begin(); }
    auto end() const { return v_.end(); }
    void resize(size_t n) { v_.resize(n); }
    std::vector<T>& std() { return v_; }
    const std::vector<T>& std() const { return v_; }
    bool same_as(const Vector& o) const { return v_ == o.v_; }
    bool operator==(const Vector& o) const { return v_ == o.v_; }

#define ORQ_B200_VEC_BINOP(op)                                          \
    Vector operator op(const Vector& o) const {                         \
        if (o.size() != size()) throw std::invalid_argument("size mismatch"); \
        Vector r(size());                                               \
        for (size_t i = 0; i < size(); i++) r[i] = (T)(v_[i] op o.v_[i]); \
        return r;                                                       \
    }
    ORQ_B200_VEC_BINOP(&)
    ORQ_B200_VEC_BINOP(^)
    ORQ_B200_VEC_BINOP(|)
    ORQ_B200_VEC_BINOP(<)
    ORQ_B200_VEC_BINOP(>)
    ORQ_B200_VEC_BINOP(<=)
    ORQ_B200_VEC_BINOP(>=)
#undef ORQ_B200_VEC_BINOP
    // wrapping arithmetic, as the shares' ring mod 2^(8 sizeof T)
    Vector operator+(const Vector& o) const { return wrap(o, [](U a, U b) { return (U)(a + b); }); }
    Vector operator-(const Vector& o) const { return wrap(o, [](U a, U b) { return (U)(a - b); }); }
    Vector operator*(const Vector& o) const { return wrap(o, [](U a, U b) { return (U)(a * b); }); }
    Vector equal(const Vector& o) const {
        Vector r(size());
        for (size_t i = 0; i < size(); i++) r[i] = (T)(v_[i] == o.v_[i]);
        return r;
    }

   private:
    using U = std::make_unsigned_t<T>;
    template <typename F>
    Vector wrap(const Vector& o, F f) const {
        if (o.size() != size()) throw std::invalid_argument("size mismatch");
        Vector r(size());
        for (size_t i = 0; i < size(); i++) r[i] = (T)f((U)v_[i], (U)o.v_[i]);
        return r;
    }
};

template <typename T>
using DataTable = std::vector<Vector<T>>;

namespace service {

// The process-wide loopback runtime: keys for the ten PRG streams of the
// three parties, a CUDA stream and a device pool, owned by the library.
class LoopbackRunTime {
    orqcu_runtime* rt_ = nullptr;
    uint64_t seed_;
    int nparties_;
    std::mt19937_64 local_rng_;

   public:
    // nparties 3: replicated 3PC; 2: Beaver 2PC with dummy triples; 4:
    // Fantastic-4PC (the latter two run the protocols' local steps: sharing,
    // open, and_b, multiply_a, b2a_bit and the local ops)
    explicit LoopbackRunTime(uint64_t seed, int device = 0, int nparties = 3)
        : seed_(seed), nparties_(nparties), local_rng_(seed ^ 0x5DEECE66Dull) {
        if (nparties == 3) orqcu_check(orqcu_runtime_create(seed, device, &rt_));
        else orqcu_check(orqcu_runtime_create_np(seed, device, nparties, &rt_));
    }
    int nparties() const { return nparties_; }
    ~LoopbackRunTime() {
        if (rt_) orqcu_runtime_destroy(rt_);
    }
    LoopbackRunTime(const LoopbackRunTime&) = delete;
    LoopbackRunTime& operator=(const LoopbackRunTime&) = delete;

    orqcu_runtime* handle() const { return rt_; }
    uint64_t seed() const { return seed_; }

    // One process holds every party; opened values are available to it, so
    // checks written for "party 0" run here.
    int getPartyID() const { return 0; }
    int getNumParties() const { return nparties_; }

    // RunTime::populateLocalRandom (runtime.h): plaintext randomness for test
    // inputs, from a host generator seeded by the runtime seed.
    template <typename T>
    void populateLocalRandom(Vector<T>& v) {
        for (auto& x : v) x = (T)local_rng_();
    }

    void synchronize() { orqcu_check(orqcu_synchronize(rt_)); }
    uint64_t kernels_launched() const {
        uint64_t k = 0;
        orqcu_check(orqcu_kernels_launched(rt_, &k));
        return k;
    }
    // re-key as a fresh orq_init with `seed` (nonces at 0, reserved
    // permutations dropped), keeping the stream and cached memory
    void reseed(uint64_t seed) {
        orqcu_check(orqcu_runtime_reseed(rt_, seed));
        seed_ = seed;
    }
    void reserve_permutations(size_t n, size_t count) {
        orqcu_check(orqcu_reserve_permutations(rt_, n, count));
    }
};

// orq::service::runTime in the reference: the runtime every operator calls.
inline std::unique_ptr<LoopbackRunTime>& runtime_holder() {
    static std::unique_ptr<LoopbackRunTime> h;
    return h;
}
struct RunTimeRef {
    LoopbackRunTime* operator->() const {
        auto& h = runtime_holder();
        if (!h) throw std::logic_error("orq_init has not been called");
        return h.get();
    }
    LoopbackRunTime& operator*() const { return *operator->(); }
};
inline RunTimeRef runTime;

}  // namespace service

// ---------------------------------------------------------------------------
// Device storage: one pooled block holding the three share arrays of a vector
// (S0 | S1 | S2, `cap` elements each). Copies of a shared vector share it,
// like the reference's shallow Vector copies (mapping_access_vector.h:237-324).
struct ShareStore {
    orqcu_runtime* rt = nullptr;
    void* base = nullptr;
    size_t cap = 0;
    int width = 0;
    int np = 3;  // distinct share arrays: 3 (3PC), 2 (2PC) or 4 (4PC)
    ShareStore(orqcu_runtime* r, size_t n, int w, int parties) : rt(r), cap(n), width(w), np(parties) {
        orqcu_check(orqcu_pool_alloc(rt, (size_t)np * std::max<size_t>(n, 1) * (size_t)w, &base));
        orqcu_check(orqcu_memset(rt, base, 0, (size_t)np * std::max<size_t>(n, 1) * (size_t)w));
    }
    ~ShareStore() {
        if (base) orqcu_pool_free(rt, base);
    }
    ShareStore(const ShareStore&) = delete;
    ShareStore& operator=(const ShareStore&) = delete;
};

// A (possibly offset) view of n elements of a ShareStore: the share pointers
// the C ABI takes (three for 3PC, two or four for 2PC / 4PC).
struct Shares {
    std::shared_ptr<ShareStore> st;
    size_t off = 0, n = 0;
    int width = 0;

    Shares() = default;
    Shares(size_t n_, int w) : n(n_), width(w) {
        st = std::make_shared<ShareStore>(service::runTime->handle(), n_, w, service::runTime->nparties());
    }
    int np() const { return st ? st->np : 3; }
    void* ptr(int p) const {
        return static_cast<char*>(st->base) + ((size_t)p * st->cap + off) * (size_t)width;
    }
    struct P3 {
        void* p[4];
        operator void* const*() const { return p; }
        operator const void* const*() const { return const_cast<const void* const*>(p); }
    };
    P3 p3() const {
        P3 r{{nullptr, nullptr, nullptr, nullptr}};
        for (int p = 0; p < np(); p++) r.p[p] = ptr(p);
        return r;
    }
    Shares slice(size_t b, size_t e) const {
        if (b > e || e > n) throw std::out_of_range("slice out of range");
        Shares s = *this;
        s.off = off + b;
        s.n = e - b;
        return s;
    }
    // deep copy into fresh storage
    Shares clone() const {
        Shares c(n, width);
        c.assign(*this);
        return c;
    }
    // elementwise copy of o's shares into this view (Vector::operator=)
    void assign(const Shares& o) const {
        if (o.n != n || o.width != width || o.np() != np())
            throw std::invalid_argument("assignment of a different size or type");
        for (int p = 0; p < np(); p++)
            orqcu_check(orqcu_memcpy_d2d(st->rt, ptr(p), o.ptr(p), n * (size_t)width));
    }
    void zero() const {
        for (int p = 0; p < np(); p++) orqcu_check(orqcu_memset(st->rt, ptr(p), 0, n * (size_t)width));
    }
    // the distinct shares on the host, S[p][i] (tests and share files)
    template <typename T>
    std::vector<std::vector<T>> download() const {
        std::vector<std::vector<T>> h(np(), std::vector<T>(n));
        for (int p = 0; p < np(); p++)
            orqcu_check(orqcu_memcpy_d2h(st->rt, h[p].data(), ptr(p), n * sizeof(T)));
        return h;
    }
};

}  // namespace orq
