// shared_vector.hpp — BSharedVector / ASharedVector on the loopback runtime.
//
// The API of ORQ's share containers (core/containers/b_shared_vector.h,
// a_shared_vector.h, encoded_vector.h:85-154): operators return
// std::unique_ptr of the vector type, compound assignments work in place,
// copies share storage and operator= copies elements. Each operator is one
// C-ABI call that runs the protocol's local step for all three parties.
#pragma once

#include "runtime.hpp"

namespace orq {

template <typename T>
class ASharedVector;
template <typename T>
class BSharedVector;

template <typename T>
constexpr int share_width() {
    static_assert(sizeof(T) == 1 || sizeof(T) == 2 || sizeof(T) == 4 || sizeof(T) == 8,
                  "shares are 1, 2, 4 or 8 bytes");
    return (int)sizeof(T);
}

// EVector in the reference: the replicated shares a secret_share_* call
// returns, convertible to either vector type.
template <typename T>
struct EVector {
    Shares s;
};

namespace detail {
// input on the device for secret_share / public_share
template <typename T>
struct DeviceInput {
    void* p = nullptr;
    orqcu_runtime* rt;
    DeviceInput(const Vector<T>& v) : rt(service::runTime->handle()) {
        orqcu_check(orqcu_pool_alloc(rt, std::max<size_t>(v.size(), 1) * sizeof(T), &p));
        if (v.size()) orqcu_check(orqcu_memcpy_h2d(rt, p, v.data(), v.size() * sizeof(T)));
    }
    ~DeviceInput() { orqcu_pool_free(rt, p); }
};
}  // namespace detail

// Common part of both vector types: a view of three share arrays.
template <typename T, typename Derived, bool Arith>
class SharedVectorBase {
   protected:
    Shares s_;

    using U = std::unique_ptr<Derived>;
    template <typename F>
    U binary(const Derived& o, F f) const {
        need_same(o);
        auto r = std::make_unique<Derived>(size());
        orqcu_check(f(rt(), share_width<T>(), size(), s_.p3(), o.shares().p3(), r->shares().p3()));
        return r;
    }
    template <typename F>
    Derived& in_place(const Derived& o, F f) {
        need_same(o);
        orqcu_check(f(rt(), share_width<T>(), size(), s_.p3(), o.shares().p3(), s_.p3()));
        return static_cast<Derived&>(*this);
    }
    void need_same(const SharedVectorBase& o) const {
        if (o.size() != size()) throw std::invalid_argument("vector sizes differ");
    }
    // replicated 3PC, or the 2PC / 4PC runtime (orqcu_np_* entry points)
    bool np3() const { return s_.np() == 3; }

   public:
    using value_type = T;
    static constexpr bool arithmetic = Arith;

    SharedVectorBase() = default;
    explicit SharedVectorBase(size_t n) : s_(n, share_width<T>()) {}
    explicit SharedVectorBase(Shares s) : s_(std::move(s)) {
        if (s_.width != share_width<T>()) throw std::invalid_argument("share width does not match the type");
    }
    SharedVectorBase(const EVector<T>& e) : SharedVectorBase(e.s) {}

    size_t size() const { return s_.n; }
    const Shares& shares() const { return s_; }
    Shares& shares() { return s_; }
    orqcu_runtime* rt() const { return s_.st ? s_.st->rt : service::runTime->handle(); }

    // Vector::operator= (mapping_access_vector.h:1263): elementwise copy into
    // this vector's storage (an empty vector adopts a copy)
    Derived& operator=(const Derived& o) {
        if (!s_.st) s_ = o.shares().clone();
        else if (o.shares().st != s_.st || o.shares().off != s_.off) s_.assign(o.shares());
        return static_cast<Derived&>(*this);
    }
    Derived& operator=(const std::unique_ptr<Derived>& o) { return *this = *o; }

    // open_shares_a / open_shares_b (replicated_3pc.h:310-330)
    Vector<T> open() const {
        Vector<T> out(size());
        if (!size()) return out;
        void* d = nullptr;
        orqcu_check(orqcu_pool_alloc(rt(), size() * sizeof(T), &d));
        int rc = np3() ? orqcu_open(rt(), Arith, share_width<T>(), size(), s_.p3(), d)
                       : orqcu_np_open(rt(), Arith, share_width<T>(), size(), s_.p3(), d);
        if (rc == ORQCU_OK) rc = orqcu_memcpy_d2h(rt(), out.data(), d, size() * sizeof(T));
        orqcu_pool_free(rt(), d);
        orqcu_check(rc);
        return out;
    }

    // views sharing storage (Vector::slice, mapping_access_vector.h)
    Derived slice(size_t begin, size_t end) const { return Derived(s_.slice(begin, end)); }
    Derived slice(size_t begin) const { return slice(begin, size()); }
    // a deep copy
    Derived deepcopy() const { return Derived(s_.clone()); }
    void zero() { s_.zero(); }
};

// ---------------------------------------------------------------------------
template <typename T>
class BSharedVector : public SharedVectorBase<T, BSharedVector<T>, false> {
    using Base = SharedVectorBase<T, BSharedVector<T>, false>;
    using typename Base::U;

   public:
    using Base::Base;
    using Base::operator=;
    BSharedVector() = default;
    BSharedVector(const BSharedVector&) = default;
    BSharedVector(BSharedVector&&) = default;
    BSharedVector& operator=(const BSharedVector& o) { return Base::operator=(o); }
    BSharedVector(std::unique_ptr<BSharedVector>&& p) : Base(p->shares()) {}
    BSharedVector(const std::unique_ptr<BSharedVector>& p) : Base(p->shares()) {}

    // and_b (replicated_3pc.h:166-191) fused with the zero-sharing
    U operator&(const BSharedVector& o) const { return this->binary(o, this->np3() ? orqcu_and_b : orqcu_np_and_b); }
    U operator^(const BSharedVector& o) const { return this->binary(o, this->np3() ? orqcu_xor_b : orqcu_np_xor_b); }
    BSharedVector& operator&=(const BSharedVector& o) { return *this = *(*this & o); }
    BSharedVector& operator^=(const BSharedVector& o) { return this->in_place(o, this->np3() ? orqcu_xor_b : orqcu_np_xor_b); }
    BSharedVector& operator&=(const U& o) { return *this &= *o; }
    BSharedVector& operator^=(const U& o) { return *this ^= *o; }
    // operator| (b_shared_vector.h:438-441): ~(~a & ~b)
    U operator|(const BSharedVector& o) const { return ~*(*~*this & *~o); }
    BSharedVector& operator|=(const BSharedVector& o) { return *this = *(*this | o); }
    // not_b (replicated_3pc.h:199)
    U operator~() const {
        auto r = std::make_unique<BSharedVector>(this->size());
        orqcu_check(orqcu_not_b(this->rt(), share_width<T>(), this->size(), this->s_.p3(), r->shares().p3()));
        return r;
    }
    // not_b_1 (replicated_3pc.h:207): logical NOT of the LSB
    U operator!() const {
        auto r = std::make_unique<BSharedVector>(this->size());
        orqcu_check(orqcu_not_b_1(this->rt(), share_width<T>(), this->size(), this->s_.p3(), r->shares().p3()));
        return r;
    }
    // operator+ / operator- (b_shared_vector.h:588-622): the ripple-carry adder
    U operator+(const BSharedVector& o) const { return this->binary(o, orqcu_add_b); }
    U operator-(const BSharedVector& o) const { return this->binary(o, orqcu_sub_b); }
    BSharedVector& operator+=(const BSharedVector& o) { return *this = *(*this + o); }
    BSharedVector& operator-=(const BSharedVector& o) { return *this = *(*this - o); }

    // _compare (circuits.h:231-295): eq and gt bits, signed order
    std::pair<BSharedVector, BSharedVector> _compare(const BSharedVector& o) const {
        this->need_same(o);
        BSharedVector eq(this->size()), gt(this->size());
        orqcu_check(orqcu_compare_b(this->rt(), share_width<T>(), this->size(), this->s_.p3(), o.shares().p3(),
                                    eq.shares().p3(), gt.shares().p3()));
        return {eq, gt};
    }
    // operator== (b_shared_vector.h:493-504): bit_same then mask(1)
    U operator==(const BSharedVector& o) const { return this->binary(o, orqcu_equal_b); }
    U operator!=(const BSharedVector& o) const { return !*(*this == o); }
    U operator>(const BSharedVector& o) const { return std::make_unique<BSharedVector>(_compare(o).second); }
    U operator<(const BSharedVector& o) const { return o > *this; }
    U operator>=(const BSharedVector& o) const { return !*(*this < o); }
    U operator<=(const BSharedVector& o) const { return !*(*this > o); }

    // mask (b_shared_vector.h:462-464): every share &= m, in place
    void mask(const T& m) {
        using UT = std::make_unsigned_t<T>;
        orqcu_check(orqcu_mask_b(this->rt(), share_width<T>(), this->size(), this->s_.p3(), (uint64_t)(UT)m));
    }
    // extend_lsb (b_shared_vector.h:145-147): all ones where in's LSB is set
    void extend_lsb(const BSharedVector& in) {
        this->need_same(in);
        orqcu_check(orqcu_extend_lsb(this->rt(), share_width<T>(), this->size(), in.shares().p3(), this->s_.p3()));
    }
    // b2a_bit (b_shared_vector.h:279-284, replicated_3pc.h:220-251)
    ASharedVector<T> b2a_bit() const;
};

// ---------------------------------------------------------------------------
template <typename T>
class ASharedVector : public SharedVectorBase<T, ASharedVector<T>, true> {
    using Base = SharedVectorBase<T, ASharedVector<T>, true>;
    using typename Base::U;

   public:
    using Base::Base;
    using Base::operator=;
    ASharedVector() = default;
    ASharedVector(const ASharedVector&) = default;
    ASharedVector(ASharedVector&&) = default;
    ASharedVector& operator=(const ASharedVector& o) { return Base::operator=(o); }
    ASharedVector(std::unique_ptr<ASharedVector>&& p) : Base(p->shares()) {}
    ASharedVector(const std::unique_ptr<ASharedVector>& p) : Base(p->shares()) {}

    // multiply_a (replicated_3pc.h:44-67); add_a / sub_a are local
    U operator*(const ASharedVector& o) const { return this->binary(o, this->np3() ? orqcu_multiply_a : orqcu_np_multiply_a); }
    U operator+(const ASharedVector& o) const { return this->binary(o, this->np3() ? orqcu_add_a : orqcu_np_add_a); }
    U operator-(const ASharedVector& o) const { return this->binary(o, this->np3() ? orqcu_sub_a : orqcu_np_sub_a); }
    ASharedVector& operator*=(const ASharedVector& o) { return *this = *(*this * o); }
    ASharedVector& operator+=(const ASharedVector& o) { return this->in_place(o, this->np3() ? orqcu_add_a : orqcu_np_add_a); }
    ASharedVector& operator-=(const ASharedVector& o) { return this->in_place(o, this->np3() ? orqcu_sub_a : orqcu_np_sub_a); }
    ASharedVector& operator*=(const U& o) { return *this *= *o; }
    ASharedVector& operator+=(const U& o) { return *this += *o; }
    ASharedVector& operator-=(const U& o) { return *this -= *o; }

    // a2b (a_shared_vector.h:138-144)
    std::unique_ptr<BSharedVector<T>> a2b() const {
        auto r = std::make_unique<BSharedVector<T>>(this->size());
        orqcu_check(orqcu_a2b(this->rt(), share_width<T>(), this->size(), this->s_.p3(), r->shares().p3()));
        return r;
    }
    // SharedVector::prefix_sum (shared_vector.h:249): in place, local
    void prefix_sum() {
        orqcu_check(orqcu_prefix_sum_a(this->rt(), share_width<T>(), this->size(), this->s_.p3()));
    }
};

template <typename T>
ASharedVector<T> BSharedVector<T>::b2a_bit() const {
    ASharedVector<T> r(this->size());
    if (this->np3())
        orqcu_check(orqcu_b2a_bit(this->rt(), share_width<T>(), this->size(), this->s_.p3(), r.shares().p3()));
    else
        orqcu_check(orqcu_np_b2a_bit(this->rt(), share_width<T>(), this->size(), this->s_.p3(), r.shares().p3()));
    return r;
}

template <typename T>
std::unique_ptr<BSharedVector<T>> operator~(const std::unique_ptr<BSharedVector<T>>& x) {
    return ~*x;
}
template <typename T>
std::unique_ptr<BSharedVector<T>> operator!(const std::unique_ptr<BSharedVector<T>>& x) {
    return !*x;
}

// The sorting permutation (core/containers/permutation.h:205-280): A-shared
// int32 destination indices.
class ElementwisePermutation : public ASharedVector<int32_t> {
   public:
    using ASharedVector<int32_t>::ASharedVector;
    ElementwisePermutation(const ASharedVector<int32_t>& a) : ASharedVector<int32_t>(a) {}
    ASharedVector<int32_t>& getASharedPerm() { return *this; }
    const ASharedVector<int32_t>& getASharedPerm() const { return *this; }
};

// ---------------------------------------------------------------------------
// secret_share_b / secret_share_a (replicated_3pc.h:401-448): the owner
// `party` shares its plaintext with its local PRG.
namespace detail {
template <typename T>
EVector<T> share(const Vector<T>& data, int party, int arith) {
    EVector<T> e{Shares(data.size(), share_width<T>())};
    DeviceInput<T> in(data);
    if (e.s.np() == 3)
        orqcu_check(orqcu_secret_share(e.s.st->rt, arith, share_width<T>(), data.size(), in.p, party, e.s.p3()));
    else
        orqcu_check(orqcu_np_secret_share(e.s.st->rt, arith, share_width<T>(), data.size(), in.p, party, e.s.p3()));
    return e;
}
}  // namespace detail
template <typename T>
EVector<T> secret_share_b(const Vector<T>& data, int party = 0) {
    return detail::share(data, party, 0);
}
template <typename T>
EVector<T> secret_share_a(const Vector<T>& data, int party = 0) {
    return detail::share(data, party, 1);
}
// secret_share_vec(x, sx) of the reference's tests: share into an existing
// vector, boolean or arithmetic by its type
template <typename T>
void secret_share_vec(const Vector<T>& data, BSharedVector<T>& out, int party = 0) {
    out = BSharedVector<T>(secret_share_b(data, party));
}
template <typename T>
void secret_share_vec(const Vector<T>& data, ASharedVector<T>& out, int party = 0) {
    out = ASharedVector<T>(secret_share_a(data, party));
}
// public_share (replicated_3pc.h:456-470): S0 = x, S1 = S2 = 0; for 2PC
// (beaver_2pc.h:262-270) S0 = x, S1 = 0; for 4PC (dalskov_4pc.h:786-797)
// X0 = x and the other shares 0
template <typename T>
EVector<T> public_share(const Vector<T>& data) {
    EVector<T> e{Shares(data.size(), share_width<T>())};
    detail::DeviceInput<T> in(data);
    if (e.s.np() == 3)
        orqcu_check(orqcu_public_share(e.s.st->rt, share_width<T>(), data.size(), in.p, e.s.p3()));
    else if (data.size())
        orqcu_check(orqcu_memcpy_d2d(e.s.st->rt, e.s.ptr(0), in.p, data.size() * sizeof(T)));
    return e;
}

}  // namespace orq
