// test_loopback.cpp — a program written against ORQ's C++ API, compiled
// against the loopback orq.h (include/orq_b200) and linked with
// liborq_cuda.so. Run by tests/test_cpp_boundary.py.
//
//   test_loopback check
//       the checks of ORQ's own tests (tests/test_primitives.cpp,
//       test_sorting.cpp, test_operators.cpp, test_join.cpp): opened results
//       against plaintext computed here; prints one line per check.
//   test_loopback dump <op> <n> <seed> <out.bin> [bits]
//       the "prims", "radix" and "join_agg" sequences of the reference driver
//       (oracle/ref_driver.cpp) with the same inputs, dumping the three
//       distinct shares of every vector so their digests can be compared with
//       the reference's (run with ORQ_SEED = the reference's key seed, and
//       compiled with -DORQ_B200_DEFAULT_SORT_PROTO=RADIXSORT like the
//       reference driver). Compiled with -DPROTOCOL_NUM=2 or 4, "prims" is
//       the sequence of oracle/ref_driver_np.cpp and dumps the 2 or 4
//       distinct shares.
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <map>
#include <numeric>
#include <string>

#include "orq.h"

using namespace orq::debug;
using namespace orq::service;
using namespace COMPILED_MPC_PROTOCOL_NAMESPACE;

static uint64_t sm64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename T>
static orq::Vector<T> gen(size_t n, uint64_t& st, uint64_t mask) {
    orq::Vector<T> v(n);
    for (size_t i = 0; i < n; i++) v[i] = (T)(sm64(st) & mask);
    return v;
}

static int failures = 0;
#define CHECK(cond, what)                                    \
    do {                                                     \
        if (cond) {                                          \
            single_cout("OK " << what);                      \
        } else {                                             \
            single_cout("FAIL " << what);                    \
            failures++;                                      \
        }                                                    \
    } while (0)

// ---- dumps: name, width, n, then S0, S1, S2 (little-endian) --------------
struct Dumper {
    std::ofstream f;
    explicit Dumper(const std::string& path) : f(path, std::ios::binary) {}
    void rec(const std::string& name, uint32_t w, uint64_t n, const std::vector<const void*>& arrays) {
        uint32_t nl = name.size(), k = arrays.size();
        f.write((const char*)&nl, 4);
        f.write(name.data(), nl);
        f.write((const char*)&w, 4);
        f.write((const char*)&n, 8);
        f.write((const char*)&k, 4);
        for (auto* a : arrays) f.write((const char*)a, n * w);
    }
    template <typename SV>
    void shares(const std::string& name, const SV& v) {
        using T = typename SV::value_type;
        auto h = v.shares().template download<T>();
        std::vector<const void*> a;
        for (auto& col : h) a.push_back(col.data());
        rec(name, sizeof(T), v.size(), a);
    }
    template <typename T>
    void plain(const std::string& name, const orq::Vector<T>& a) {
        rec(name, sizeof(T), a.size(), {a.data()});
    }
};

// ---- the reference driver's sequences -------------------------------------
// xa_owner: 2 in the 3PC driver (oracle/ref_driver.cpp), 1 in the 2PC / 4PC
// driver (oracle/ref_driver_np.cpp)
template <typename T>
static void run_prims(size_t n, uint64_t seed, Dumper& d, const std::string& tag, int xa_owner) {
    uint64_t st = seed;
    auto x = gen<T>(n, st, ~0ull);
    auto y = gen<T>(n, st, ~0ull);
    BSharedVector<T> xb = secret_share_b(x, 0);
    BSharedVector<T> yb = secret_share_b(y, 1);
    d.shares(tag + "xb", xb);
    d.shares(tag + "yb", yb);
    BSharedVector<T> zb = xb & yb;
    d.shares(tag + "and", zb);
    BSharedVector<T> xo = xb ^ yb;
    d.shares(tag + "xor", xo);
    ASharedVector<T> xa = secret_share_a(x, xa_owner);
    ASharedVector<T> ya = secret_share_a(y, 0);
    d.shares(tag + "xa", xa);
    d.shares(tag + "ya", ya);
    ASharedVector<T> za = xa * ya;
    d.shares(tag + "mul", za);
    ASharedVector<T> sa = xa + ya;
    d.shares(tag + "add", sa);
    ASharedVector<T> ba = xb.b2a_bit();
    d.shares(tag + "b2a", ba);
    auto o1 = zb.open();
    auto o2 = za.open();
    auto o3 = ba.open();
    d.plain(tag + "open_and", o1);
    d.plain(tag + "open_mul", o2);
    d.plain(tag + "open_b2a", o3);
}

static void run_radix(size_t n, uint64_t seed, int bits, Dumper& d) {
    uint64_t st = seed;
    uint64_t km = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    auto key = gen<int64_t>(n, st, km);
    auto p1 = gen<int64_t>(n, st, 0xffffffffull);
    auto p2 = gen<int64_t>(n, st, 0xffffffffull);
    BSharedVector<int64_t> kb = secret_share_b(key, 0);
    ASharedVector<int64_t> a1 = secret_share_a(p1, 0);
    ASharedVector<int64_t> a2 = secret_share_a(p2, 0);
    auto perm = orq::operators::radix_sort(kb, orq::operators::SortOrder::ASC, bits);
    orq::operators::oblivious_apply_elementwise_perm(a1, perm);
    orq::operators::oblivious_apply_elementwise_perm(a2, perm);
    d.shares("key", kb);
    d.shares("pay1", a1);
    d.shares("pay2", a2);
    auto pa = perm.getASharedPerm();
    d.shares("perm", pa);
    d.plain("open_key", kb.open());
    d.plain("open_pay1", a1.open());
    d.plain("open_pay2", a2.open());
}

static void run_join_agg(size_t n, uint64_t seed, Dumper& d) {
    uint64_t st = seed;
    const size_t na = n, nb = 2 * n;
    orq::Vector<int64_t> pk(na), g(na), v(na), fk(nb), q(nb);
    for (size_t i = 0; i < na; i++) pk[i] = (int64_t)i;
    for (size_t i = na; i-- > 1;) {
        size_t j = sm64(st) % (i + 1);
        std::swap(pk[i], pk[j]);
    }
    for (size_t i = 0; i < na; i++) g[i] = (int64_t)(sm64(st) % 5);
    for (size_t i = 0; i < na; i++) v[i] = (int64_t)(sm64(st) % 1000000);
    for (size_t i = 0; i < nb; i++) fk[i] = (int64_t)(sm64(st) % na);
    for (size_t i = 0; i < nb; i++) q[i] = (int64_t)(1 + sm64(st) % 50);
    std::vector<orq::Vector<int64_t>> ca = {pk, g, v};
    std::vector<orq::Vector<int64_t>> cb = {fk, q};
    EncodedTable<int64_t> A = secret_share(ca, {"[K]", "[G]", "V"});
    EncodedTable<int64_t> B = secret_share(cb, {"[K]", "Q"});
    auto J = A.inner_join(B, {"[K]"}, {{"[G]", "[G]", copy<BSharedVector<int64_t>>},
                                       {"V", "V", copy<ASharedVector<int64_t>>}});
    J.addColumns(std::vector<std::string>{"VQ", "CNT"});
    J["VQ"] = J["V"] * J["Q"];
    J.aggregate({"[G]"}, {{"VQ", "VQ", sum<ASharedVector<int64_t>>}, {"CNT", "CNT", count<ASharedVector<int64_t>>}});
    for (auto& name : J.getColumnNames()) {
        if (isBShared(name)) d.shares(name, J.asBSharedVector(name));
        else d.shares(name, J.asASharedVector(name));
    }
    auto T = J.open_with_schema();
    for (size_t k = 0; k < T.second.size(); k++) d.plain("open_" + T.second[k], T.first[k]);
}

// ---- checks in the style of the reference's tests ---------------------------
template <typename T>
static void check_primitives(size_t n) {
    const int L = 8 * sizeof(T);
    orq::Vector<T> x(n), y(n);
    runTime->populateLocalRandom(x);
    runTime->populateLocalRandom(y);
    for (size_t i = 0; i < n; i += 7) y[i] = x[i];  // some equal pairs
    BSharedVector<T> bx = secret_share_b(x, 0), by = secret_share_b(y, 1);
    ASharedVector<T> ax = secret_share_a(x, 0), ay = secret_share_a(y, 2);
    CHECK((bx & by)->open().same_as(x & y), L << "-bit and");
    CHECK((bx ^ by)->open().same_as(x ^ y), L << "-bit xor");
    CHECK((bx | by)->open().same_as(x | y), L << "-bit or");
    CHECK((ax * ay)->open().same_as(x * y), L << "-bit multiplication");
    CHECK((ax + ay)->open().same_as(x + y), L << "-bit addition");
    CHECK((ax - ay)->open().same_as(x - y), L << "-bit subtraction");
    if (sizeof(T) >= 4) {
        CHECK((bx + by)->open().same_as(x + y), L << "-bit binary add");
        CHECK((bx - by)->open().same_as(x - y), L << "-bit binary subtract");
        CHECK(ax.a2b()->open().same_as(x), L << "-bit a2b");
    }
    if (sizeof(T) >= 4) {  // the compare circuits take 4-, 8- and 16-byte shares
        CHECK((bx == by)->open().same_as(x.equal(y)), L << "-bit equality");
        CHECK((bx != by)->open().same_as(x.equal(y) ^ orq::Vector<T>(n, (T)1)), L << "-bit inequality");
        CHECK((bx > by)->open().same_as(x > y), L << "-bit greater than");
        CHECK((bx < by)->open().same_as(x < y), L << "-bit less than");
        CHECK((bx >= by)->open().same_as(x >= y), L << "-bit greater or equal");
        CHECK((bx <= by)->open().same_as(x <= y), L << "-bit less or equal");
    }
    orq::Vector<T> lsb(n);
    for (size_t i = 0; i < n; i++) lsb[i] = x[i] & 1;
    if (sizeof(T) >= 4) {  // mask takes 4- and 8-byte shares
        BSharedVector<T> bits = secret_share_b(x, 0);
        bits.mask(1);
        CHECK(bits.b2a_bit().open().same_as(lsb), L << "-bit b2a_bit of a masked bit");
    }
    CHECK(bx.b2a_bit().open().same_as(lsb), L << "-bit b2a_bit");
    BSharedVector<T> acc = secret_share_b(x, 0);
    acc &= by;
    CHECK(acc.open().same_as(x & y), L << "-bit compound and");
}

template <typename T>
static void check_sorting(size_t n) {
    const int L = 8 * sizeof(T);
    orq::Vector<T> key(n), pay(n);
    runTime->populateLocalRandom(key);
    for (size_t i = 0; i < n; i++) pay[i] = (T)i;
    auto sorted = key.std();
    std::sort(sorted.begin(), sorted.end());
    {
        BSharedVector<T> k = secret_share_b(key, 0);
        ASharedVector<T> p = secret_share_a(pay, 0);
        auto perm = orq::operators::radix_sort(k, orq::operators::SortOrder::ASC);
        orq::operators::oblivious_apply_elementwise_perm(p, perm);
        auto ko = k.open(), po = p.open();
        bool carried = true;
        for (size_t i = 0; i < n; i++) carried = carried && key[(size_t)po[i]] == ko[i];
        CHECK(ko.std() == sorted && carried, L << "-bit radix_sort + payload apply");
    }
    {
        BSharedVector<T> k = secret_share_b(key, 0);
        auto perm = orq::operators::quicksort(k, orq::operators::SortOrder::DESC);
        auto ko = k.open();
        CHECK(std::equal(ko.begin(), ko.end(), sorted.rbegin()), L << "-bit quicksort DESC");
    }
    {
        BSharedVector<T> k = secret_share_b(key, 0);
        orq::operators::bitonic_sort(k, orq::operators::SortOrder::ASC);
        CHECK(k.open().std() == sorted, L << "-bit bitonic_sort");
    }
    {
        BSharedVector<T> k = secret_share_b(key, 0);
        orq::operators::shuffle(k);
        auto ko = k.open().std();
        std::sort(ko.begin(), ko.end());
        CHECK(ko == sorted, L << "-bit shuffle keeps the multiset");
    }
}

static void check_tables(size_t n) {
    // group-by: SUM(v), COUNT(*) per g, checked against a plaintext map
    orq::Vector<int64_t> g(n), v(n);
    uint64_t st = 99;
    for (size_t i = 0; i < n; i++) g[i] = (int64_t)(sm64(st) % 37);
    for (size_t i = 0; i < n; i++) v[i] = (int64_t)(sm64(st) % 1000);
    std::vector<orq::Vector<int64_t>> cols = {g, v};
    EncodedTable<int64_t> t = secret_share(cols, {"[G]", "V"});
    t.addColumns(std::vector<std::string>{"S", "C"});
    t["S"] = t["V"];
    t.aggregate({"[G]"}, {{"S", "S", sum<ASharedVector<int64_t>>}, {"C", "C", count<ASharedVector<int64_t>>}});
    t.deleteColumns({"V"});
    auto out = t.open_with_schema();
    std::map<int64_t, std::pair<int64_t, int64_t>> want, got;
    for (size_t i = 0; i < n; i++) {
        want[g[i]].first += v[i];
        want[g[i]].second += 1;
    }
    // columns in schema order: C, S, [G]
    for (size_t i = 0; i < out.first[0].size(); i++) got[out.first[2][i]] = {out.first[1][i], out.first[0][i]};
    CHECK(got == want, "EncodedTable aggregate (group-by sum, count)");

    // table sort on two key columns, DESC then ASC
    orq::Vector<int64_t> a(n), b(n);
    for (size_t i = 0; i < n; i++) a[i] = (int64_t)(sm64(st) % 5), b[i] = (int64_t)(sm64(st) % 1000);
    std::vector<orq::Vector<int64_t>> c2 = {a, b};
    EncodedTable<int64_t> s = secret_share(c2, {"[A]", "[B]"});
    s.sort(std::vector<std::pair<std::string, orq::operators::SortOrder>>{{"[A]", DESC}, {"[B]", ASC}});
    auto so = s.open_with_schema();
    std::vector<std::pair<int64_t, int64_t>> rows;
    for (size_t i = 0; i < n; i++) rows.push_back({-a[i], b[i]});
    std::sort(rows.begin(), rows.end());
    bool ok = so.first[0].size() == n;
    for (size_t i = 0; ok && i < n; i++) ok = so.first[0][i] == -rows[i].first && so.first[1][i] == rows[i].second;
    CHECK(ok, "EncodedTable sort ([A] DESC, [B] ASC)");
}

static void check_join(size_t n) {
    // PK-FK inner join then group-by SUM(V*Q), COUNT (the relational pipeline)
    uint64_t st = 7;
    const size_t na = n, nb = 4 * n;
    orq::Vector<int64_t> pk(na), g(na), v(na), fk(nb), q(nb);
    for (size_t i = 0; i < na; i++) pk[i] = (int64_t)i;
    for (size_t i = na; i-- > 1;) std::swap(pk[i], pk[sm64(st) % (i + 1)]);
    for (size_t i = 0; i < na; i++) g[i] = (int64_t)(sm64(st) % 11);
    for (size_t i = 0; i < na; i++) v[i] = (int64_t)(sm64(st) % 1000000);
    for (size_t i = 0; i < nb; i++) fk[i] = (int64_t)(sm64(st) % na);
    for (size_t i = 0; i < nb; i++) q[i] = (int64_t)(1 + sm64(st) % 50);
    std::vector<orq::Vector<int64_t>> ca = {pk, g, v}, cb = {fk, q};
    EncodedTable<int64_t> A = secret_share(ca, {"[K]", "[G]", "V"});
    EncodedTable<int64_t> B = secret_share(cb, {"[K]", "Q"});
    auto J = A.inner_join(B, {"[K]"}, {{"[G]", "[G]", copy<BSharedVector<int64_t>>},
                                       {"V", "V", copy<ASharedVector<int64_t>>}});
    J.addColumns(std::vector<std::string>{"VQ", "CNT"});
    J["VQ"] = J["V"] * J["Q"];
    J.aggregate({"[G]"}, {{"VQ", "VQ", sum<ASharedVector<int64_t>>}, {"CNT", "CNT", count<ASharedVector<int64_t>>}});
    J.deleteColumns({"V", "Q", "[K]"});
    auto out = J.open_with_schema();  // CNT, VQ, [G]
    std::vector<int64_t> gv(na), vv(na);
    for (size_t i = 0; i < na; i++) gv[pk[i]] = g[i], vv[pk[i]] = v[i];
    std::map<int64_t, std::pair<int64_t, int64_t>> want, got;
    for (size_t j = 0; j < nb; j++) {
        auto& w = want[gv[fk[j]]];
        w.first += vv[fk[j]] * q[j];
        w.second += 1;
    }
    for (size_t i = 0; i < out.first[0].size(); i++) got[out.first[2][i]] = {out.first[1][i], out.first[0][i]};
    CHECK(got == want, "inner_join + aggregate (A " << na << " rows, B " << nb << " rows)");
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: test_loopback check | dump <op> <n> <seed> <out> [bits]\n");
        return 2;
    }
    const std::string mode = argv[1];
    try {
        orq_init(argc, argv);
        if (mode == "check") {
            check_primitives<int32_t>(1 << 16);
            check_primitives<int64_t>(1 << 16);
            check_primitives<int8_t>(4096);
            check_sorting<int32_t>(1 << 14);
            check_sorting<int64_t>(1 << 14);
            check_tables(3000);
            check_join(2000);
            single_cout("kernels " << runTime->kernels_launched());
        } else if (mode == "dump" && argc >= 6) {
            const std::string op = argv[2];
            const size_t n = std::stoull(argv[3]);
            const uint64_t seed = std::stoull(argv[4]);
            const int bits = argc > 6 ? std::atoi(argv[6]) : 40;
            Dumper d(argv[5]);
            if (op == "prims") {
                const int xa_owner = PROTOCOL_NUM == 3 ? 2 : 1;
                run_prims<int32_t>(n, seed, d, "w4_", xa_owner);
                run_prims<int64_t>(n, seed + 1, d, "w8_", xa_owner);
                run_prims<int8_t>(n, seed + 2, d, "w1_", xa_owner);
            } else if (op == "radix") {
                run_radix(n, seed, bits, d);
            } else if (op == "join_agg") {
                run_join_agg(n, seed, d);
            } else {
                std::fprintf(stderr, "unknown op %s\n", op.c_str());
                return 2;
            }
        } else {
            std::fprintf(stderr, "bad arguments\n");
            return 2;
        }
        orq_finalize();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return failures ? 1 : 0;
}
