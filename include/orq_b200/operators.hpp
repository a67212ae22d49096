// operators.hpp — ORQ's oblivious operators (core/operators/*.h) on the
// loopback runtime: sorts, shuffles, permutation application, compare_rows /
// swap / multiplex, table_sort, distinct and the aggregation network. Each is
// one C-ABI call (the library runs every round of the operator on the GPU).
#pragma once

#include <optional>
#include <tuple>

#include "shared_vector.hpp"

namespace orq {

// SortingProtocol (core/operators/sorting.h:15-22). A reference build fixes
// DEFAULT with DEFAULT_SORT_PROTO; here it is QUICKSORT (the reference's own
// default) unless ORQ_B200_DEFAULT_SORT_PROTO names another.
#ifndef ORQ_B200_DEFAULT_SORT_PROTO
#define ORQ_B200_DEFAULT_SORT_PROTO QUICKSORT
#endif
typedef enum { BITONICSORT = 0, QUICKSORT = 1, RADIXSORT = 2, DEFAULT = ORQ_B200_DEFAULT_SORT_PROTO } SortingProtocol;

namespace operators {

enum SortOrder { ASC, DESC };

namespace detail {
template <typename V>
std::vector<void*> flat(const std::vector<V*>& cols) {
    std::vector<void*> f;
    f.reserve(3 * cols.size() + 1);
    for (auto* c : cols)
        for (int p = 0; p < 3; p++) f.push_back(c->shares().ptr(p));
    if (f.empty()) f.push_back(nullptr);
    return f;
}
template <typename T>
constexpr size_t digits() {
    return std::numeric_limits<std::make_unsigned_t<T>>::digits;
}
inline std::vector<int> desc_flags(const std::vector<SortOrder>& o) {
    std::vector<int> d;
    for (auto x : o) d.push_back(x == DESC);
    if (d.empty()) d.push_back(0);
    return d;
}
}  // namespace detail

// radix_sort (radixsort.h:205-229): v sorted in place on its low `bits` bits
// (signed order at the full width); returns the sorting permutation.
template <typename T>
ElementwisePermutation radix_sort(BSharedVector<T>& v, SortOrder order = ASC, size_t bits = detail::digits<T>()) {
    ElementwisePermutation perm(v.size());
    orqcu_check(orqcu_radix_sort(v.rt(), share_width<T>(), v.size(), v.shares().p3(), (int)bits, order == DESC,
                                 perm.shares().p3()));
    return perm;
}

// quicksort (quicksort.h:214-246)
template <typename T>
ElementwisePermutation quicksort(BSharedVector<T>& v, SortOrder order = ASC) {
    ElementwisePermutation perm(v.size());
    orqcu_check(orqcu_quicksort(v.rt(), share_width<T>(), v.size(), v.shares().p3(), order == DESC,
                                perm.shares().p3()));
    return perm;
}

// bitonic_sort (sorting.h:394-399): one key column, n a power of two
template <typename T>
void bitonic_sort(BSharedVector<T>& v, SortOrder order = ASC) {
    orqcu_check(orqcu_bitonic_sort(v.rt(), share_width<T>(), v.size(), v.shares().p3(), order == DESC));
}

// bitonic_sort (sorting.h:266-353): key columns (most significant first) with
// A- and B-shared data columns moved along
template <typename T>
void bitonic_sort(std::vector<BSharedVector<T>*> columns, std::vector<ASharedVector<T>*> data_a,
                  std::vector<BSharedVector<T>*> data_b, std::vector<SortOrder> order) {
    if (columns.empty() || order.size() != columns.size())
        throw std::invalid_argument("bitonic_sort needs one order per key column");
    auto fc = detail::flat(columns), fa = detail::flat(data_a), fb = detail::flat(data_b);
    auto d = detail::desc_flags(order);
    orqcu_check(orqcu_bitonic_sort_rows(columns[0]->rt(), share_width<T>(), columns[0]->size(), (int)columns.size(),
                                        fc.data(), d.data(), (int)data_a.size(), fa.data(), (int)data_b.size(),
                                        fb.data()));
}

// shuffle (shuffle.h:752-757): x permuted in place by a fresh sharded
// permutation
template <typename V>
void shuffle(V& x) {
    orqcu_check(orqcu_shuffle(x.rt(), V::arithmetic, share_width<typename V::value_type>(), x.size(),
                              x.shares().p3()));
}

// shuffle(data_a, data_b, size) (shuffle.h:769-786): every column permuted by
// one random elementwise permutation
template <typename T>
void shuffle(std::vector<ASharedVector<T>*> data_a, std::vector<BSharedVector<T>*> data_b, size_t size) {
    auto fa = detail::flat(data_a), fb = detail::flat(data_b);
    orqcu_check(orqcu_table_shuffle(service::runTime->handle(), share_width<T>(), size, (int)data_a.size(),
                                    fa.data(), (int)data_b.size(), fb.data()));
}

// oblivious_apply_elementwise_perm (shuffle.h:687-706): x permuted in place
template <typename V>
void oblivious_apply_elementwise_perm(V& x, const ElementwisePermutation& perm) {
    if (perm.size() != x.size()) throw std::invalid_argument("permutation size differs");
    orqcu_check(orqcu_apply_elementwise_perm(x.rt(), V::arithmetic, share_width<typename V::value_type>(), x.size(),
                                             x.shares().p3(), perm.shares().p3()));
}

// compose_permutations (shuffle.h:717-743): rho <- rho * sigma; sigma is
// consumed
inline ElementwisePermutation compose_permutations(ElementwisePermutation& sigma, ElementwisePermutation& rho) {
    orqcu_check(orqcu_compose_permutations(rho.rt(), rho.size(), sigma.shares().p3(), rho.shares().p3()));
    return rho;
}

// compare_rows (sorting.h:80-108): row i of x > row i of y, lexicographically
template <typename T>
BSharedVector<T> compare_rows(const std::vector<BSharedVector<T>*>& x_vec, const std::vector<BSharedVector<T>*>& y_vec,
                              const std::vector<SortOrder>& order) {
    if (x_vec.empty() || x_vec.size() != y_vec.size() || order.size() != x_vec.size())
        throw std::invalid_argument("compare_rows needs matching key lists and one order per key");
    BSharedVector<T> gt(x_vec[0]->size());
    auto fx = detail::flat(x_vec), fy = detail::flat(y_vec);
    auto d = detail::desc_flags(order);
    orqcu_check(orqcu_compare_rows(gt.rt(), share_width<T>(), gt.size(), (int)x_vec.size(),
                                   const_cast<const void* const*>(fx.data()),
                                   const_cast<const void* const*>(fy.data()), d.data(), gt.shares().p3()));
    return gt;
}

// swap (sorting.h:146-212): rows exchanged where bits is 1 (B columns with B
// bits, A columns with A bits)
template <typename V>
void swap(std::vector<V*>& x_vec, std::vector<V*>& y_vec, const V& bits) {
    auto fx = detail::flat(x_vec), fy = detail::flat(y_vec);
    orqcu_check(orqcu_swap(bits.rt(), V::arithmetic, share_width<typename V::value_type>(), bits.size(),
                           (int)x_vec.size(), fx.data(), fy.data(), bits.shares().p3()));
}

// multiplex (operators/common.h:20-49): b where sel is 1, else a
template <typename T>
BSharedVector<T> multiplex(const BSharedVector<T>& sel, const BSharedVector<T>& a, const BSharedVector<T>& b) {
    BSharedVector<T> ext(sel.size());
    ext.extend_lsb(sel);
    return BSharedVector<T>(a ^ *(ext & *(b ^ a)));
}
template <typename T>
ASharedVector<T> multiplex(const ASharedVector<T>& sel, const ASharedVector<T>& a, const ASharedVector<T>& b) {
    return ASharedVector<T>(a + *(sel * *(b - a)));
}

// table_sort (sorting.h:509-612) with the quicksort or radix protocol
template <typename T>
void table_sort(std::vector<BSharedVector<T>*> columns, std::vector<ASharedVector<T>*> data_a,
                std::vector<BSharedVector<T>*> data_b, const std::vector<SortOrder>& order,
                const std::vector<bool>& single_bit, SortingProtocol protocol = DEFAULT) {
    if (columns.empty() || order.size() != columns.size() || single_bit.size() != columns.size())
        throw std::invalid_argument("table_sort needs one order and one single_bit flag per key column");
    auto fc = detail::flat(columns), fa = detail::flat(data_a), fb = detail::flat(data_b);
    auto d = detail::desc_flags(order);
    std::vector<int> sb(single_bit.begin(), single_bit.end());
    orqcu_check(orqcu_table_sort(columns[0]->rt(), share_width<T>(), columns[0]->size(), (int)columns.size(),
                                 fc.data(), d.data(), sb.data(), (int)data_a.size(), fa.data(), (int)data_b.size(),
                                 fb.data(), (int)protocol));
}

// distinct (distinct.h:20-53): res[i] = 1 where row i differs from row i-1
template <typename T>
void distinct(std::vector<BSharedVector<T>*>& keys, BSharedVector<T>* res) {
    if (keys.empty()) throw std::invalid_argument("distinct needs a key column");
    auto fk = detail::flat(keys);
    orqcu_check(orqcu_distinct(res->rt(), share_width<T>(), res->size(), (int)keys.size(),
                               const_cast<const void* const*>(fk.data()), res->shares().p3()));
}

}  // namespace operators

// ---------------------------------------------------------------------------
// orq::aggregators (aggregation.h:27-346). The functions are the reference's
// names; a spec passes them as function pointers, which select the device
// aggregation (the network itself runs in the library, one launch a level).
namespace aggregators {

enum class Direction { Forward, Reverse };

template <typename A>
void sum(const A&, A&, const A&) {}
template <typename A>
void count(const A&, A&, const A&) {}
template <typename T>
void copy(const T&, T&, const T&) {}
template <typename B>
void valid(const B&, B&, const B&) {}
template <typename B>
void bit_or(const B&, B&, const B&) {}
template <typename B>
void min(const B&, B&, const B&) {}
template <typename B>
void max(const B&, B&, const B&) {}

template <typename V>
using agg_fn = void (*)(const V&, V&, const V&);

// ORQCU_AGG_* code of an aggregation function
template <typename V>
int agg_code(agg_fn<V> f) {
    if (f == &sum<V>) return ORQCU_AGG_SUM;
    if (f == &count<V>) return ORQCU_AGG_COUNT;
    if (f == &copy<V>) return ORQCU_AGG_COPY;
    if (f == &valid<V>) return ORQCU_AGG_VALID;
    if (f == &bit_or<V>) return ORQCU_AGG_BIT_OR;
    if (f == &min<V>) return ORQCU_AGG_MIN;
    if (f == &max<V>) return ORQCU_AGG_MAX;
    throw std::invalid_argument("not an orq::aggregators function");
}

template <typename T>
using BSpec = std::tuple<BSharedVector<T>, BSharedVector<T>, agg_fn<BSharedVector<T>>>;
template <typename T>
using ASpec = std::tuple<ASharedVector<T>, ASharedVector<T>, agg_fn<ASharedVector<T>>>;

// aggregate (aggregation.h:167-346): the odd-even aggregation network over
// keys; each spec (input, output, function) overwrites its output
template <typename T>
void aggregate(std::vector<BSharedVector<T>>& keys, const std::vector<BSpec<T>>& agg_spec_b,
               const std::vector<ASpec<T>>& agg_spec_a, Direction dir = Direction::Forward,
               std::optional<BSharedVector<T>> sel_b = {}) {
    size_t n = 0;
    orqcu_runtime* rt = service::runTime->handle();
    if (!keys.empty()) n = keys[0].size();
    else if (!agg_spec_b.empty()) n = std::get<1>(agg_spec_b[0]).size();
    else if (!agg_spec_a.empty()) n = std::get<1>(agg_spec_a[0]).size();
    std::vector<const void*> kp;
    for (auto& k : keys)
        for (int p = 0; p < 3; p++) kp.push_back(k.shares().ptr(p));
    if (kp.empty()) kp.push_back(nullptr);
    auto specs = [](const auto& lst) {
        std::vector<orqcu_agg_spec> v(std::max<size_t>(lst.size(), 1));
        for (size_t i = 0; i < lst.size(); i++) {
            for (int p = 0; p < 3; p++) {
                v[i].in[p] = std::get<0>(lst[i]).shares().ptr(p);
                v[i].out[p] = std::get<1>(lst[i]).shares().ptr(p);
            }
            v[i].func = agg_code(std::get<2>(lst[i]));
        }
        return v;
    };
    auto sb = specs(agg_spec_b);
    auto sa = specs(agg_spec_a);
    Shares::P3 sel{};
    if (sel_b) sel = sel_b->shares().p3();
    orqcu_check(orqcu_aggregate(rt, share_width<T>(), n, (int)keys.size(), kp.data(), (int)agg_spec_b.size(),
                                sb.data(), (int)agg_spec_a.size(), sa.data(), dir == Direction::Reverse,
                                sel_b ? (const void* const*)sel : nullptr));
}

}  // namespace aggregators
}  // namespace orq
