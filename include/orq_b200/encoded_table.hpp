// encoded_table.hpp — EncodedTable and its join on the loopback runtime.
//
// ORQ's relational layer (core/containers/tabular/encoded_table.h and
// core/operators/join.h:32-233) as host C++ over the C ABI: the schema,
// padding, concatenation and projection are host bookkeeping; every protocol
// step is a library call made in the reference's order, so each column's
// shares equal the reference run's with the same keys and sort protocol.
//
// Column names follow the reference: a name containing '[' is a boolean-
// shared column, anything else arithmetic. The schema is a std::map, so data
// columns are permuted in byte order of their names, which fixes the PRG use.
#pragma once

#include <algorithm>
#include <map>
#include <set>
#include <string>

#include "operators.hpp"

namespace orq {
namespace relational {

using operators::SortOrder;
using operators::ASC;
using operators::DESC;

inline const std::string ENC_TABLE_JOIN_ID = "[##TID]";
inline const std::string ENC_TABLE_VALID = "[##V]";
inline const std::string ENC_TABLE_UNIQ = "[##UNIQ]";
inline const std::string ENC_TABLE_VALID_TEMP = "[##VALID_TEMP]";

// EncodedColumn (encoded_column.h:147): one shared column, boolean or
// arithmetic by its name, with the vector operators dispatched on its kind.
class EncodedColumn {
   public:
    Shares s;
    bool arith = false;
    std::string name;

    EncodedColumn() = default;
    EncodedColumn(Shares sh, bool a, std::string nm = "") : s(std::move(sh)), arith(a), name(std::move(nm)) {}
    // copies share storage (the reference's shallow Vector copies)
    EncodedColumn(const EncodedColumn&) = default;

    size_t size() const { return s.n; }
    template <typename T>
    BSharedVector<T> asB() const {
        if (arith) throw std::invalid_argument("column " + name + " is not boolean-shared");
        return BSharedVector<T>(s);
    }
    template <typename T>
    ASharedVector<T> asA() const {
        if (!arith) throw std::invalid_argument("column " + name + " is not arithmetic-shared");
        return ASharedVector<T>(s);
    }

    // elementwise assignment of another column's shares (Vector::operator=)
    EncodedColumn& operator=(const EncodedColumn& o) {
        if (!s.st) {
            s = o.s.clone();
            arith = o.arith;
        } else {
            if (o.arith != arith) throw std::invalid_argument("assignment between boolean and arithmetic columns");
            s.assign(o.s);
        }
        return *this;
    }
    EncodedColumn& operator=(const std::unique_ptr<EncodedColumn>& o) { return *this = *o; }

   private:
    template <typename F>
    auto typed(F f) const {
        if (s.width == 4) return f(int32_t{});
        if (s.width == 8) return f(int64_t{});
        throw std::invalid_argument("table columns are 4 or 8 bytes");
    }
    using UC = std::unique_ptr<EncodedColumn>;
    UC wrapB(const Shares& r) const { return std::make_unique<EncodedColumn>(r, false); }
    UC wrapA(const Shares& r) const { return std::make_unique<EncodedColumn>(r, true); }

   public:
#define ORQ_B200_COL_OP(op, allowA, allowB)                                                         \
    UC operator op(const EncodedColumn& o) const {                                                  \
        if (o.arith != arith) throw std::invalid_argument("operands of different sharing");         \
        return typed([&](auto t) -> UC {                                                             \
            using T = decltype(t);                                                                   \
            if (arith) {                                                                             \
                if constexpr (allowA) return wrapA((asA<T>() op o.asA<T>())->shares());              \
                else throw std::invalid_argument("operator " #op " needs boolean-shared columns");  \
            } else {                                                                                 \
                if constexpr (allowB) return wrapB((asB<T>() op o.asB<T>())->shares());              \
                else throw std::invalid_argument("operator " #op " needs arithmetic-shared columns"); \
            }                                                                                        \
        });                                                                                          \
    }                                                                                                \
    UC operator op(const UC& o) const { return *this op *o; }
    ORQ_B200_COL_OP(+, true, true)
    ORQ_B200_COL_OP(-, true, true)
    ORQ_B200_COL_OP(*, true, false)
    ORQ_B200_COL_OP(&, false, true)
    ORQ_B200_COL_OP(^, false, true)
    ORQ_B200_COL_OP(|, false, true)
    ORQ_B200_COL_OP(==, false, true)
    ORQ_B200_COL_OP(!=, false, true)
    ORQ_B200_COL_OP(<, false, true)
    ORQ_B200_COL_OP(>, false, true)
    ORQ_B200_COL_OP(<=, false, true)
    ORQ_B200_COL_OP(>=, false, true)
#undef ORQ_B200_COL_OP
    UC operator~() const {
        return typed([&](auto t) -> UC { return wrapB((~asB<decltype(t)>())->shares()); });
    }
    UC operator!() const {
        return typed([&](auto t) -> UC { return wrapB((!asB<decltype(t)>())->shares()); });
    }
    EncodedColumn& operator&=(const EncodedColumn& o) { return *this = *(*this & o); }
    EncodedColumn& operator^=(const EncodedColumn& o) { return *this = *(*this ^ o); }
    EncodedColumn& operator|=(const EncodedColumn& o) { return *this = *(*this | o); }
    EncodedColumn& operator+=(const EncodedColumn& o) { return *this = *(*this + o); }
    EncodedColumn& operator-=(const EncodedColumn& o) { return *this = *(*this - o); }
    EncodedColumn& operator*=(const EncodedColumn& o) { return *this = *(*this * o); }
};

inline std::unique_ptr<EncodedColumn> operator~(const std::unique_ptr<EncodedColumn>& x) { return ~*x; }
inline std::unique_ptr<EncodedColumn> operator!(const std::unique_ptr<EncodedColumn>& x) { return !*x; }

// AggregationSelector (aggregation_selector.h:14-70) for a table of T
template <typename T>
class AggregationSelector {
    aggregators::agg_fn<BSharedVector<T>> b_ = nullptr;
    aggregators::agg_fn<ASharedVector<T>> a_ = nullptr;

   public:
    AggregationSelector(aggregators::agg_fn<BSharedVector<T>> f) : b_(f) {}
    AggregationSelector(aggregators::agg_fn<ASharedVector<T>> f) : a_(f) {}
    bool boolean() const { return b_ != nullptr; }
    aggregators::agg_fn<BSharedVector<T>> getB() const {
        if (!b_) throw std::invalid_argument("requested a boolean aggregation, but the function is arithmetic");
        return b_;
    }
    aggregators::agg_fn<ASharedVector<T>> getA() const {
        if (!a_) throw std::invalid_argument("requested an arithmetic aggregation, but the function is boolean");
        return a_;
    }
    int code() const { return b_ ? aggregators::agg_code(b_) : aggregators::agg_code(a_); }
    // true for an aggregation, false for copy / valid (isAggregation)
    bool isAggregation() const {
        const int c = code();
        return c != ORQCU_AGG_COPY && c != ORQCU_AGG_VALID;
    }
};

// JoinOptions / AggregationOptions (encoded_table.h:91-119)
struct JoinOptions {
    bool left_outer = false;
    bool right_outer = false;
    bool anti = false;
    bool trim_invalid = true;
};
struct AggregationOptions {
    bool reverse = false;
    bool do_sort = true;
    bool mark_valid = true;
    std::optional<std::string> table_id = {};
};

inline bool isBShared(const std::string& name) { return name.find('[') != std::string::npos; }

namespace detail {
// a vector of n copies of a one-element share vector (per party), on the device
inline Shares broadcast(const Shares& one, size_t n) {
    Shares r(n, one.width);
    std::vector<char> host(std::max<size_t>(n, 1) * (size_t)one.width);
    for (int p = 0; p < 3; p++) {
        char v[8];
        orqcu_check(orqcu_memcpy_d2h(one.st->rt, v, one.ptr(p), (size_t)one.width));
        for (size_t i = 0; i < n; i++) std::memcpy(host.data() + i * one.width, v, (size_t)one.width);
        if (n) orqcu_check(orqcu_memcpy_h2d(one.st->rt, r.ptr(p), host.data(), n * (size_t)one.width));
    }
    return r;
}
// rows [b, e) of s as a fresh array
inline Shares copy_rows(const Shares& s, size_t b, size_t e) { return s.slice(b, e).clone(); }
}  // namespace detail

// ---------------------------------------------------------------------------
// EncodedTable<T> (encoded_table.h:123-1640): T is int32_t or int64_t.
template <typename T>
class EncodedTable {
   public:
    using A = ASharedVector<T>;
    using B = BSharedVector<T>;
    using AggregationSpec = std::vector<std::tuple<std::string, std::string, AggregationSelector<T>>>;
    using LabeledDataTable = std::pair<DataTable<T>, std::vector<std::string>>;

    std::string tableName;
    // SortingProtocol of this table's sorts; derived tables inherit it
    SortingProtocol protocol = DEFAULT;

   private:
    std::map<std::string, EncodedColumn> schema_;
    size_t rows_ = 0;

    static constexpr int W = share_width<T>();
    EncodedColumn zeros(const std::string& nm, size_t n) const {
        return EncodedColumn(Shares(n, W), !isBShared(nm), nm);
    }
    // public_share of 1: S0 = 1, S1 = S2 = 0
    EncodedColumn ones(const std::string& nm, size_t n) const {
        return EncodedColumn(orq::public_share(Vector<T>(n, (T)1)).s, !isBShared(nm), nm);
    }
    // bind a column (shares storage) under a name, replacing any old one
    void put(const std::string& nm, const EncodedColumn& c) {
        schema_.erase(nm);
        auto it = schema_.emplace(nm, c).first;
        it->second.name = nm;
    }
    void configure_valid() { put(ENC_TABLE_VALID, ones(ENC_TABLE_VALID, rows_)); }
    std::vector<B> key_vecs(const std::vector<std::string>& keys) {
        std::vector<B> v;
        for (auto& k : keys) v.push_back(asBSharedVector(k));
        return v;
    }

   public:
    EncodedTable() = default;
    // EncodedTable(name, schema, size) (encoded_table.h:244-250): zero columns,
    // every row valid
    EncodedTable(const std::string& name, const std::vector<std::string>& columns, size_t rows)
        : tableName(name), rows_(rows) {
        configure_valid();
        addColumns(columns, rows);
    }
    // EncodedTable(contents) (encoded_table.h:252-265): the columns that
    // secret_share returns, every row valid
    EncodedTable(std::vector<std::shared_ptr<EncodedColumn>>&& contents) {
        rows_ = contents.empty() ? 0 : contents[0]->size();
        for (auto& c : contents) {
            if (c->size() != rows_) throw std::invalid_argument("columns of different sizes");
            put(c->name, *c);
        }
        configure_valid();
    }

    size_t size() const { return rows_; }
    std::vector<std::string> getColumnNames() const {
        std::vector<std::string> v;
        for (auto& kv : schema_) v.push_back(kv.first);
        return v;
    }
    bool hasColumn(const std::string& n) const { return schema_.count(n) > 0; }
    EncodedColumn& operator[](const std::string& name) {
        auto it = schema_.find(name);
        if (it == schema_.end()) throw std::invalid_argument("column '" + name + "' not found");
        return it->second;
    }
    B asBSharedVector(const std::string& name) { return (*this)[name].template asB<T>(); }
    A asASharedVector(const std::string& name) { return (*this)[name].template asA<T>(); }

    void addColumns(const std::vector<std::string>& cols, size_t rows) {
        for (auto& nm : cols) {
            if (schema_.count(nm)) throw std::invalid_argument("Table column with name " + nm + " already exists.");
            put(nm, zeros(nm, rows));
        }
    }
    void addColumns(const std::vector<std::string>& cols) { addColumns(cols, rows_); }
    void deleteColumns(const std::vector<std::string>& cols) {
        for (auto& nm : cols) schema_.erase(nm);
    }
    // project (encoded_table.h:792-805): keep cols and the reserved columns
    void project(const std::vector<std::string>& cols) {
        std::set<std::string> keep(cols.begin(), cols.end());
        keep.insert({ENC_TABLE_JOIN_ID, ENC_TABLE_VALID, ENC_TABLE_UNIQ});
        std::vector<std::string> del;
        for (auto& kv : schema_)
            if (!keep.count(kv.first)) del.push_back(kv.first);
        deleteColumns(del);
    }
    // resize (encoded_table.h:1426-1436): truncate, or extend with zero rows
    void resize(size_t n) {
        if (n == rows_) return;
        for (auto& kv : schema_) {
            EncodedColumn nc = zeros(kv.first, n);
            const size_t m = std::min(n, rows_);
            if (m) nc.s.slice(0, m).assign(kv.second.s.slice(0, m));
            kv.second.s = nc.s;
        }
        rows_ = n;
    }
    void head(size_t n) { resize(n); }
    void tail(size_t n) {
        for (auto& kv : schema_) kv.second.s = detail::copy_rows(kv.second.s, rows_ - n, rows_);
        rows_ = n;
    }
    // pad_power_of_two (encoded_table.h:1446-1468) with zero rows
    void pad_power_of_two() {
        size_t p = 1;
        while (p < rows_) p <<= 1;
        resize(p);
    }
    // filter (encoded_table.h:299-316): valid &= bits
    void filter(const EncodedColumn& bits) { (*this)[ENC_TABLE_VALID] &= bits; }
    void filter(const std::unique_ptr<EncodedColumn>& bits) { filter(*bits); }

    // concatenate (encoded_table.h:1548-1610): rows of this table, then of
    // other; the table id column is 1 (one secret-shared 1) for other's rows
    EncodedTable concatenate(EncodedTable& other) {
        std::vector<std::string> cols{ENC_TABLE_JOIN_ID};
        for (auto& c : getColumnNames())
            if (c != ENC_TABLE_JOIN_ID) cols.push_back(c);
        for (auto& c : other.getColumnNames())
            if (!schema_.count(c)) cols.push_back(c);
        const size_t n = rows_ + other.rows_;
        EncodedTable t;
        t.tableName = tableName + "+" + other.tableName;
        t.protocol = protocol;
        t.rows_ = n;
        t.configure_valid();
        for (auto& c : cols)
            if (!t.schema_.count(c)) t.addColumns({c});
        for (auto& kv : schema_) t.schema_[kv.first].s.slice(0, rows_).assign(kv.second.s);
        for (auto& kv : other.schema_) t.schema_[kv.first].s.slice(rows_, n).assign(kv.second.s);
        auto one = secret_share_b(Vector<T>(1, (T)1), 0);
        t.schema_[ENC_TABLE_JOIN_ID].s.slice(rows_, n).assign(detail::broadcast(one.s, other.rows_));
        return t;
    }

    // ---- sort (encoded_table.h:841-998) ----------------------------------
    // QUICKSORT and RADIXSORT go through table_sort (the valid and table-id
    // columns on one bit); BITONICSORT pads to a power of two, runs the
    // multi-column network with every other column as data, and cuts the
    // padding again when the sort was on the valid column.
    EncodedTable& sort(const std::vector<std::pair<std::string, SortOrder>>& spec, SortingProtocol proto) {
        const size_t original = rows_;
        if (proto == BITONICSORT) pad_power_of_two();
        std::vector<std::string> keys;
        std::vector<SortOrder> orders;
        std::vector<bool> single_bit;
        bool can_unpad = false, unpad_from_top = true;
        for (auto& kv : spec) {
            keys.push_back(kv.first);
            orders.push_back(kv.second);
            single_bit.push_back(kv.first == ENC_TABLE_VALID || kv.first == ENC_TABLE_JOIN_ID);
            if (kv.first == ENC_TABLE_VALID) {
                can_unpad = true;
                unpad_from_top = kv.second == ASC;
            }
        }
        std::vector<B> kv_ = key_vecs(keys);
        std::vector<A> da;
        std::vector<B> db;
        for (auto& nm : getColumnNames()) {
            if (std::find(keys.begin(), keys.end(), nm) != keys.end()) continue;
            if (isBShared(nm)) db.push_back(asBSharedVector(nm));
            else da.push_back(asASharedVector(nm));
        }
        std::vector<B*> kp;
        std::vector<A*> ap;
        std::vector<B*> bp;
        for (auto& v : kv_) kp.push_back(&v);
        for (auto& v : da) ap.push_back(&v);
        for (auto& v : db) bp.push_back(&v);
        if (proto == BITONICSORT) {
            operators::bitonic_sort(kp, ap, bp, orders);
            if (can_unpad) {
                if (unpad_from_top) tail(original);
                else resize(original);
            }
        } else {
            operators::table_sort(kp, ap, bp, orders, single_bit, proto);
        }
        return *this;
    }
    EncodedTable& sort(const std::vector<std::pair<std::string, SortOrder>>& spec) { return sort(spec, protocol); }
    EncodedTable& sort(const std::vector<std::string>& columns, SortOrder allOrder, SortingProtocol proto) {
        std::vector<std::pair<std::string, SortOrder>> spec;
        for (auto& c : columns) spec.push_back({c, allOrder});
        return sort(spec, proto);
    }
    EncodedTable& sort(const std::vector<std::string>& columns, SortOrder allOrder = ASC) {
        return sort(columns, allOrder, protocol);
    }

    // ---- shuffle, mask, finalize (encoded_table.h:170-222,645-652,1003-1018)
    EncodedTable& shuffle() {
        std::vector<A> da;
        std::vector<B> db;
        for (auto& nm : getColumnNames()) {
            if (isBShared(nm)) db.push_back(asBSharedVector(nm));
            else da.push_back(asASharedVector(nm));
        }
        std::vector<A*> ap;
        std::vector<B*> bp;
        for (auto& v : da) ap.push_back(&v);
        for (auto& v : db) bp.push_back(&v);
        operators::shuffle(ap, bp, rows_);
        return *this;
    }
    // rows whose mask bit is 0 get MASK_VALUE (the type's maximum) in every
    // other column: multiplex on the bit (on its b2a_bit for arithmetic
    // columns); MASK_VALUE is secret-shared once, arithmetic sharing first
    EncodedTable& mask(const std::string& mask_column, const std::vector<std::string>& keys) {
        B sel_b = asBSharedVector(mask_column);
        A sel_a = sel_b.b2a_bit();
        const Vector<T> mv(1, std::numeric_limits<T>::max());
        auto one_a = secret_share_a(mv, 0);
        auto one_b = secret_share_b(mv, 0);
        A full_a(detail::broadcast(one_a.s, rows_));
        B full_b(detail::broadcast(one_b.s, rows_));
        for (auto& nm : keys) {
            if (nm == mask_column) continue;
            if (isBShared(nm)) put(nm, EncodedColumn(operators::multiplex(sel_b, full_b, asBSharedVector(nm)).shares(), false));
            else put(nm, EncodedColumn(operators::multiplex(sel_a, full_a, asASharedVector(nm)).shares(), true));
        }
        return *this;
    }
    EncodedTable& mask(const std::string& mask_column = ENC_TABLE_VALID) { return mask(mask_column, getColumnNames()); }
    void finalize(bool do_shuffle = true) {
        if (do_shuffle) shuffle();
        mask();
    }

    // ---- distinct (encoded_table.h:1198-1212) -----------------------------
    EncodedTable& distinct(const std::vector<std::string>& keys, const std::string& res) {
        std::vector<B> kv_ = key_vecs(keys);
        std::vector<B*> kp;
        for (auto& v : kv_) kp.push_back(&v);
        B r(rows_);
        operators::distinct(kp, &r);
        put(res, EncodedColumn(r.shares(), false));
        return *this;
    }

    // ---- aggregate (encoded_table.h:1059-1186) ----------------------------
    EncodedTable& aggregate(const std::vector<std::string>& keys_in, const AggregationSpec& agg_spec,
                            AggregationOptions opt = {}) {
        std::vector<std::string> keys = keys_in;
        if (opt.do_sort) {
            keys.insert(keys.begin(), ENC_TABLE_VALID);
            sort(keys, ASC);
        }
        const size_t original = rows_;
        pad_power_of_two();
        std::vector<B> keys_vec = key_vecs(keys);
        std::vector<aggregators::BSpec<T>> b_agg;
        std::vector<aggregators::ASpec<T>> a_agg;
        bool has_agg = false;
        for (auto& sp : agg_spec) {
            const std::string& data = std::get<0>(sp);
            const std::string& result = std::get<1>(sp);
            const AggregationSelector<T>& f = std::get<2>(sp);
            if (isBShared(data) != isBShared(result)) throw std::invalid_argument("aggregation mixes sharings");
            if (f.isAggregation()) has_agg = true;
            if (isBShared(data)) b_agg.emplace_back(asBSharedVector(data), asBSharedVector(result), f.getB());
            else a_agg.emplace_back(asASharedVector(data), asASharedVector(result), f.getA());
        }
        std::optional<B> sel;
        if (opt.mark_valid) {
            addColumns({ENC_TABLE_UNIQ});
            distinct(keys, ENC_TABLE_UNIQ);
            if (opt.table_id) sel = asBSharedVector(*opt.table_id);
        }
        aggregators::aggregate(keys_vec, b_agg, a_agg,
                               opt.reverse ? aggregators::Direction::Reverse : aggregators::Direction::Forward, sel);
        if (original < rows_) resize(original);
        if (opt.mark_valid) {
            if (has_agg) {
                if (opt.reverse) {
                    // the bottom row of each group stays valid
                    const size_t n = rows_;
                    if (n > 1) {
                        B head(detail::copy_rows((*this)[ENC_TABLE_VALID].s, 0, n - 1));
                        B nxt(detail::copy_rows((*this)[ENC_TABLE_UNIQ].s, 1, n));
                        head &= nxt;
                        (*this)[ENC_TABLE_VALID].s.slice(0, n - 1).assign(head.shares());
                    }
                } else {
                    filter((*this)[ENC_TABLE_UNIQ]);
                }
            }
            deleteColumns({ENC_TABLE_UNIQ});
        }
        return *this;
    }

    // ---- join (join.h:32-233) ---------------------------------------------
    // concatenate, project, sort on valid | keys | table id, distinct, the
    // VALID_TEMP rules of each join kind, a reverse aggregation restricted
    // by the table id, filter, and the trim heuristic for inner joins
    EncodedTable _join(EncodedTable& right, std::vector<std::string> keys, AggregationSpec agg_spec,
                       JoinOptions opt) {
        EncodedTable concat = concatenate(right);
        std::set<std::string> out_cols(keys.begin(), keys.end());
        for (auto& c : right.getColumnNames()) out_cols.insert(c);
        for (auto& sp : agg_spec) {
            out_cols.insert(std::get<0>(sp));
            out_cols.insert(std::get<1>(sp));
        }
        if (opt.left_outer)
            for (auto& c : getColumnNames()) out_cols.insert(c);
        concat.project(std::vector<std::string>(out_cols.begin(), out_cols.end()));
        keys.insert(keys.begin(), ENC_TABLE_VALID);
        std::vector<std::string> sort_keys = keys;
        sort_keys.push_back(ENC_TABLE_JOIN_ID);
        concat.sort(sort_keys, ASC);
        concat.addColumns({ENC_TABLE_UNIQ, ENC_TABLE_VALID_TEMP});
        if (!opt.right_outer) {
            agg_spec.emplace_back(ENC_TABLE_VALID_TEMP, ENC_TABLE_VALID_TEMP,
                                  AggregationSelector<T>(&aggregators::valid<B>));
            concat.distinct(keys, ENC_TABLE_UNIQ);
        }
        EncodedColumn& valid = concat[ENC_TABLE_VALID];
        if (opt.left_outer) {
            if (opt.right_outer) {
                concat.put(ENC_TABLE_VALID_TEMP, EncodedColumn(valid.s.clone(), false));
            } else {
                EncodedColumn& tid = concat[ENC_TABLE_JOIN_ID];
                EncodedColumn& uniq = concat[ENC_TABLE_UNIQ];
                concat.put(ENC_TABLE_VALID_TEMP, *(valid & *~*(tid & uniq)));
                const size_t n = concat.rows_;
                if (n > 1) {
                    EncodedColumn& vt = concat[ENC_TABLE_VALID_TEMP];
                    B head(detail::copy_rows(vt.s, 0, n - 1));
                    B t(detail::copy_rows(tid.s, 0, n - 1));
                    B u(detail::copy_rows(uniq.s, 1, n));
                    head &= *(t | u);
                    vt.s.slice(0, n - 1).assign(head.shares());
                }
            }
        } else {
            if (opt.right_outer) concat.put(ENC_TABLE_VALID_TEMP, *(valid & concat[ENC_TABLE_JOIN_ID]));
            else concat.put(ENC_TABLE_VALID_TEMP, *(valid & *~concat[ENC_TABLE_UNIQ]));
        }
        if (opt.anti)
            agg_spec.emplace_back(ENC_TABLE_VALID_TEMP, ENC_TABLE_VALID_TEMP,
                                  AggregationSelector<T>(&aggregators::copy<B>));
        concat.deleteColumns({ENC_TABLE_UNIQ});
        AggregationOptions ao;
        ao.reverse = true;
        ao.do_sort = false;
        ao.table_id = ENC_TABLE_JOIN_ID;
        concat.aggregate(keys, agg_spec, ao);
        concat.filter(concat[ENC_TABLE_VALID_TEMP]);
        concat.deleteColumns({ENC_TABLE_VALID_TEMP, ENC_TABLE_JOIN_ID});
        if (opt.trim_invalid && !opt.left_outer) {
            const size_t L = rows_, R = right.rows_;
            const size_t w = 8 * sizeof(T);
            const size_t c = schema_.size() - 1;
            if (R < (L * (w + c - 1)) / (c + 2)) {
                concat.sort(std::vector<std::string>{ENC_TABLE_VALID}, DESC);
                concat.head(R);
            }
        }
        return concat;
    }
    EncodedTable inner_join(EncodedTable& right, std::vector<std::string> keys, AggregationSpec agg_spec = {},
                            JoinOptions opt = {}) {
        return _join(right, keys, agg_spec, opt);
    }
    EncodedTable left_outer_join(EncodedTable& right, std::vector<std::string> keys, AggregationSpec agg_spec = {},
                                 JoinOptions opt = {}) {
        opt.left_outer = true;
        return _join(right, keys, agg_spec, opt);
    }
    EncodedTable right_outer_join(EncodedTable& right, std::vector<std::string> keys, AggregationSpec agg_spec = {},
                                  JoinOptions opt = {}) {
        opt.right_outer = true;
        return _join(right, keys, agg_spec, opt);
    }
    EncodedTable full_outer_join(EncodedTable& right, std::vector<std::string> keys, AggregationSpec agg_spec = {},
                                 JoinOptions opt = {}) {
        opt.left_outer = opt.right_outer = true;
        return _join(right, keys, agg_spec, opt);
    }

    // ---- output (encoded_table.h:672-711) ---------------------------------
    // opened columns in schema order; with remove_invalid the valid column is
    // left out and only valid rows are kept
    LabeledDataTable open_with_schema(bool remove_invalid = true) {
        LabeledDataTable out;
        Vector<T> valid;
        bool have_valid = false;
        for (auto& nm : getColumnNames()) {
            Vector<T> o = isBShared(nm) ? asBSharedVector(nm).open() : asASharedVector(nm).open();
            if (remove_invalid && nm == ENC_TABLE_VALID) {
                valid = o;
                have_valid = true;
            } else {
                out.first.push_back(o);
                out.second.push_back(nm);
            }
        }
        if (remove_invalid && have_valid) {
            for (auto& col : out.first) {
                Vector<T> kept;
                for (size_t i = 0; i < col.size(); i++)
                    if (valid[i] != 0) kept.std().push_back(col[i]);
                col = kept;
            }
        }
        return out;
    }
};

// secret_share(data_table, schema, party) (mpc.h): one column per name,
// boolean-shared when the name contains '[', arithmetic otherwise
template <typename T>
std::vector<std::shared_ptr<EncodedColumn>> secret_share(const DataTable<T>& data, const std::vector<std::string>& schema,
                                                         int party = 0) {
    if (data.size() != schema.size()) throw std::invalid_argument("one name per column");
    std::vector<std::shared_ptr<EncodedColumn>> cols;
    for (size_t k = 0; k < data.size(); k++) {
        const bool b = isBShared(schema[k]);
        EVector<T> e = b ? secret_share_b(data[k], party) : secret_share_a(data[k], party);
        cols.push_back(std::make_shared<EncodedColumn>(e.s, !b, schema[k]));
    }
    return cols;
}
}  // namespace relational
}  // namespace orq
