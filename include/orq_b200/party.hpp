// party.hpp — a GPU party of replicated 3PC among CPU parties of the reference.
//
// Party3PC plays party p = endpoint.rank() of Replicated_3PC: its setup sends
// and receives the PRG keys exactly as setup_random_generation does
// (backend/common/rand_setup.h:21-61,81-125,306-381, one worker thread), and
// each protocol call runs p's local step on the GPU (the orqcu_party_* entry
// points) and then the reference's exchange over the NoCopy wire
// (replicated_3pc.h: exchangeShares(local, remote, 2, 1) = send to p-1,
// receive from p+1). The CPU parties are unmodified reference programs run
// with one worker thread and batch size -1; shares are bit-identical to an
// all-CPU run with the same keys.
#pragma once

#include <algorithm>
#include <array>
#include <set>
#include <vector>

#include "nocopy.hpp"
#include "runtime.hpp"

namespace orq {
namespace gpu_party {

// p's two shares of a vector (S[p], S[p+1]) in pooled device memory
template <typename T>
class PShares {
    orqcu_runtime* rt_ = nullptr;
    void* base_ = nullptr;
    size_t n_ = 0;

   public:
    PShares(orqcu_runtime* rt, size_t n) : rt_(rt), n_(n) {
        orqcu_check(orqcu_pool_alloc(rt_, 2 * std::max<size_t>(n, 1) * sizeof(T), &base_));
    }
    ~PShares() {
        if (base_) orqcu_pool_free(rt_, base_);
    }
    PShares(PShares&& o) noexcept : rt_(o.rt_), base_(o.base_), n_(o.n_) { o.base_ = nullptr; }
    PShares(const PShares&) = delete;
    PShares& operator=(const PShares&) = delete;
    size_t size() const { return n_; }
    void* ptr(int k) const { return static_cast<char*>(base_) + (size_t)k * std::max<size_t>(n_, 1) * sizeof(T); }
    std::array<const void*, 2> c2() const { return {ptr(0), ptr(1)}; }
    std::array<void*, 2> m2() const { return {ptr(0), ptr(1)}; }
    // EVector::vector(k) on the host
    std::vector<T> download(int k) const {
        std::vector<T> h(n_);
        orqcu_check(orqcu_memcpy_d2h(rt_, h.data(), ptr(k), n_ * sizeof(T)));
        return h;
    }
};

// The keys party p holds after setup_random_generation: its local PRG key,
// its pairwise key (sent to p+1) and the one received from p-1, and the key of
// each randomness group it belongs to.
struct PartyKeys {
    std::array<uint8_t, 32> local{}, own{}, prev{};
    std::array<std::array<uint8_t, 32>, 4> group{};  // {0,1}, {0,2}, {1,2}, {0,1,2}
    std::array<bool, 4> have{};
};

// The key exchange of setup_random_generation (rand_setup.h:21-61,81-125,
// 306-381) for one worker thread. keygen(party, call, out) draws this party's
// keys in the reference's keygen order (call 0 the local PRG): orqcu_keygen
// reproduces a deterministic reference build, a deployment passes OS
// randomness.
template <typename KeyGen>
PartyKeys setup_keys(nocopy::Endpoint& ep, KeyGen keygen) {
    if (ep.count() != 3) throw std::invalid_argument("replicated 3PC needs three parties");
    const int p = ep.rank();
    PartyKeys K;
    int call = 0;
    keygen(p, call++, K.local.data());
    // create_common_prg_among_group over generateRandomnessGroups(3, 2, 1)
    // and then everyone once more: the lowest member draws the key and
    // exchanges 32 bytes with each other member (sending the key, receiving
    // an unused buffer); a group's first key is the one kept
    const std::vector<std::set<int>> groups = {{0, 1}, {0, 2}, {1, 2}, {0, 1, 2}, {0, 1, 2}};
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const auto& g = groups[gi];
        if (!g.count(p)) continue;
        const int lowest = *g.begin();
        std::array<uint8_t, 32> k{}, scratch{};
        if (p == lowest) {
            keygen(p, call++, k.data());
            for (int other : g)
                if (other != p) ep.exchange(other, k.data(), other, scratch.data(), 32);
        } else {
            std::array<uint8_t, 32> empty{};
            ep.exchange(lowest, empty.data(), lowest, k.data(), 32);
        }
        const int slot = gi < 3 ? (int)gi : 3;
        if (!K.have[slot]) {
            K.group[slot] = k;
            K.have[slot] = true;
        }
    }
    // setup_3pc_common_prgs: own key to p+1, p-1's key back
    keygen(p, call++, K.own.data());
    ep.exchange(ep.abs(1), K.own.data(), ep.abs(2), K.prev.data(), 32);
    return K;
}

class Party3PC {
    nocopy::Endpoint& ep_;
    orqcu_runtime* rt_ = nullptr;
    int p_;

    // host staging of one exchange: send `dev` to p-1, receive into `out` from p+1
    template <typename T>
    void exchange_dev(const void* dev, void* out, size_t n) {
        std::vector<T> s(n), r(n);
        orqcu_check(orqcu_memcpy_d2h(rt_, s.data(), dev, n * sizeof(T)));
        ep_.exchange(ep_.abs(2), s.data(), ep_.abs(1), r.data(), n * sizeof(T));
        orqcu_check(orqcu_memcpy_h2d(rt_, out, r.data(), n * sizeof(T)));
    }
    template <typename T>
    void send_dev(int to, const void* dev, size_t n) {
        std::vector<T> s(n);
        orqcu_check(orqcu_memcpy_d2h(rt_, s.data(), dev, n * sizeof(T)));
        ep_.send(to, s.data(), n * sizeof(T));
    }
    template <typename T>
    void recv_dev(int from, void* dev, size_t n) {
        std::vector<T> r(n);
        ep_.recv(from, r.data(), n * sizeof(T));
        orqcu_check(orqcu_memcpy_h2d(rt_, dev, r.data(), n * sizeof(T)));
    }
    template <typename T>
    static int w() {
        return (int)sizeof(T);
    }

   public:
    // keygen as for setup_keys
    template <typename KeyGen>
    Party3PC(nocopy::Endpoint& ep, int device, KeyGen keygen) : ep_(ep), p_(ep.rank()) {
        const PartyKeys K = setup_keys(ep, keygen);
        orqcu_check(orqcu_party_runtime_create(p_, device, &rt_));
        try {
            orqcu_check(orqcu_party_set_key(rt_, ORQCU_PKEY_LOCAL, K.local.data()));
            orqcu_check(orqcu_party_set_key(rt_, ORQCU_PKEY_NEXT, K.own.data()));
            orqcu_check(orqcu_party_set_key(rt_, ORQCU_PKEY_PREV, K.prev.data()));
            const int gslot[4] = {ORQCU_PKEY_G01, ORQCU_PKEY_G02, ORQCU_PKEY_G12, ORQCU_PKEY_G012};
            for (int g = 0; g < 4; g++)
                if (K.have[g]) orqcu_check(orqcu_party_set_key(rt_, gslot[g], K.group[g].data()));
        } catch (...) {
            orqcu_runtime_destroy(rt_);
            throw;
        }
    }
    ~Party3PC() {
        if (rt_) orqcu_runtime_destroy(rt_);
    }
    Party3PC(const Party3PC&) = delete;
    Party3PC& operator=(const Party3PC&) = delete;

    int party() const { return p_; }
    orqcu_runtime* handle() const { return rt_; }

    // secret_share_b / secret_share_a (replicated_3pc.h:401-448)
    template <typename T>
    PShares<T> secret_share(const Vector<T>& data, int owner, bool arith) {
        const size_t n = data.size();
        PShares<T> r(rt_, n);
        if (p_ == owner) {
            void* all = nullptr;
            orqcu_check(orqcu_pool_alloc(rt_, 4 * std::max<size_t>(n, 1) * sizeof(T), &all));
            auto at = [&](int k) { return static_cast<char*>(all) + (size_t)k * std::max<size_t>(n, 1) * sizeof(T); };
            try {
                orqcu_check(orqcu_memcpy_h2d(rt_, at(3), data.data(), n * sizeof(T)));
                void* s[3] = {at(0), at(1), at(2)};  // absolute S[0..2]
                orqcu_check(orqcu_party_secret_share(rt_, arith, w<T>(), n, at(3), s));
                const int a = p_, b = (p_ + 1) % 3, c = (p_ + 2) % 3;
                send_dev<T>(ep_.abs(1), s[b], n);
                send_dev<T>(ep_.abs(1), s[c], n);
                send_dev<T>(ep_.abs(2), s[c], n);
                send_dev<T>(ep_.abs(2), s[a], n);
                orqcu_check(orqcu_memcpy_d2d(rt_, r.ptr(0), s[a], n * sizeof(T)));
                orqcu_check(orqcu_memcpy_d2d(rt_, r.ptr(1), s[b], n * sizeof(T)));
            } catch (...) {
                orqcu_pool_free(rt_, all);
                throw;
            }
            orqcu_pool_free(rt_, all);
        } else {
            recv_dev<T>(owner, r.ptr(0), n);
            recv_dev<T>(owner, r.ptr(1), n);
        }
        return r;
    }
    template <typename T>
    PShares<T> secret_share_b(const Vector<T>& data, int owner = 0) {
        return secret_share<T>(data, owner, false);
    }
    template <typename T>
    PShares<T> secret_share_a(const Vector<T>& data, int owner = 0) {
        return secret_share<T>(data, owner, true);
    }

    // and_b / multiply_a (replicated_3pc.h:44-67,166-191)
    template <typename T>
    PShares<T> mult(const PShares<T>& x, const PShares<T>& y, bool arith) {
        if (x.size() != y.size()) throw std::invalid_argument("vector sizes differ");
        const size_t n = x.size();
        PShares<T> z(rt_, n);
        const auto xs = x.c2(), ys = y.c2();
        orqcu_check(arith ? orqcu_party_multiply_a(rt_, w<T>(), n, xs.data(), ys.data(), z.ptr(0))
                          : orqcu_party_and_b(rt_, w<T>(), n, xs.data(), ys.data(), z.ptr(0)));
        exchange_dev<T>(z.ptr(0), z.ptr(1), n);
        return z;
    }
    template <typename T>
    PShares<T> and_b(const PShares<T>& x, const PShares<T>& y) {
        return mult(x, y, false);
    }
    template <typename T>
    PShares<T> multiply_a(const PShares<T>& x, const PShares<T>& y) {
        return mult(x, y, true);
    }

    // xor_b / add_a / sub_a: local
    template <typename T>
    PShares<T> local(const PShares<T>& x, const PShares<T>& y, int op) {
        if (x.size() != y.size()) throw std::invalid_argument("vector sizes differ");
        PShares<T> z(rt_, x.size());
        const auto xs = x.c2(), ys = y.c2();
        const auto zs = z.m2();
        orqcu_check(orqcu_party_local(rt_, op, w<T>(), x.size(), xs.data(), ys.data(), zs.data()));
        return z;
    }
    template <typename T>
    PShares<T> xor_b(const PShares<T>& x, const PShares<T>& y) {
        return local(x, y, 0);
    }
    template <typename T>
    PShares<T> add_a(const PShares<T>& x, const PShares<T>& y) {
        return local(x, y, 1);
    }
    template <typename T>
    PShares<T> sub_a(const PShares<T>& x, const PShares<T>& y) {
        return local(x, y, 2);
    }

    // b2a_bit (replicated_3pc.h:220-251): two exchanges of the masked zero
    // shares, then multiply_a(s0 - s1, s0 - s1)
    template <typename T>
    PShares<T> b2a_bit(const PShares<T>& x) {
        const size_t n = x.size();
        PShares<T> s0(rt_, n), s1(rt_, n), y(rt_, n);
        const auto xs = x.c2();
        orqcu_check(orqcu_party_b2a_pre(rt_, w<T>(), n, xs.data(), s0.ptr(0), s1.ptr(0)));
        exchange_dev<T>(s0.ptr(0), s0.ptr(1), n);
        exchange_dev<T>(s1.ptr(0), s1.ptr(1), n);
        const auto a = s0.c2(), b = s1.c2();
        orqcu_check(orqcu_party_b2a_post(rt_, w<T>(), n, a.data(), b.data(), y.ptr(0)));
        exchange_dev<T>(y.ptr(0), y.ptr(1), n);
        return y;
    }

    // open_shares_b / open_shares_a (replicated_3pc.h:310-330)
    template <typename T>
    Vector<T> open(const PShares<T>& x, bool arith) {
        const size_t n = x.size();
        Vector<T> out(n);
        if (!n) return out;
        void* buf = nullptr;
        orqcu_check(orqcu_pool_alloc(rt_, 2 * n * sizeof(T), &buf));
        void* third = buf;
        void* res = static_cast<char*>(buf) + n * sizeof(T);
        try {
            exchange_dev<T>(x.ptr(1), third, n);
            const auto xs = x.c2();
            orqcu_check(orqcu_party_open(rt_, arith, w<T>(), n, xs.data(), third, res));
            orqcu_check(orqcu_memcpy_d2h(rt_, out.data(), res, n * sizeof(T)));
        } catch (...) {
            orqcu_pool_free(rt_, buf);
            throw;
        }
        orqcu_pool_free(rt_, buf);
        return out;
    }
    template <typename T>
    Vector<T> open_b(const PShares<T>& x) {
        return open(x, false);
    }
    template <typename T>
    Vector<T> open_a(const PShares<T>& x) {
        return open(x, true);
    }
};

}  // namespace gpu_party
}  // namespace orq
