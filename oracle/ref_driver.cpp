// ref_driver.cpp — runs ORQ's own 3PC code on seeded inputs and dumps every
// party's local shares, so the loopback GPU path and the C restatement can be
// compared with the reference share by share.
//
// TEST INFRASTRUCTURE ONLY: built from the ORQ headers by oracle/Makefile into
// oracle/_ref/ (never shipped), launched as three local party processes by
// oracle/run_ref.py over ORQ's NoCopy socket communicator.
//
// usage: ref_driver <threads> <p_factor> <batch> <op> <n> <data_seed> <outdir> [bits]
//   threads=1 and batch=-1 give one protocol call per runtime operation, the
//   schedule the device runtime reproduces.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
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

struct Dumper {
    std::ofstream f;
    explicit Dumper(const std::string& path) : f(path, std::ios::binary) {}
    template <typename T>
    void rec(const std::string& name, const orq::Vector<T>& a, const orq::Vector<T>& b) {
        uint32_t nl = name.size(), w = sizeof(T);
        uint64_t n = a.size();
        f.write((const char*)&nl, 4);
        f.write(name.data(), nl);
        f.write((const char*)&w, 4);
        f.write((const char*)&n, 8);
        for (uint64_t i = 0; i < n; i++) {
            T v = a[i];
            f.write((const char*)&v, sizeof(T));
        }
        for (uint64_t i = 0; i < n; i++) {
            T v = b[i];
            f.write((const char*)&v, sizeof(T));
        }
    }
    template <typename SV>
    void shares(const std::string& name, SV& v) {
        rec(name, v.vector(0), v.vector(1));
    }
    template <typename T>
    void plain(const std::string& name, const orq::Vector<T>& a) {
        rec(name, a, a);
    }
};

template <typename T>
static orq::Vector<T> gen(size_t n, uint64_t& st, uint64_t mask) {
    orq::Vector<T> v(n);
    for (size_t i = 0; i < n; i++) v[i] = (T)(sm64(st) & mask);
    return v;
}

// Sequence of primitives on width T. The restatement replays exactly this
// sequence, so every PRG stream is consumed in the same order.
template <typename T>
static void run_prims(size_t n, uint64_t seed, Dumper& d, const std::string& tag) {
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
    ASharedVector<T> xa = secret_share_a(x, 2);
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

int main(int argc, char** argv) {
    orq_init(argc, argv);
    int pid = runTime->getPartyID();
    if (argc < 8) {
        fprintf(stderr, "usage: ref_driver t p batch op n seed outdir [bits]\n");
        return 2;
    }
    std::string op = argv[4];
    size_t n = std::stoull(argv[5]);
    uint64_t seed = std::stoull(argv[6]);
    std::string outdir = argv[7];
    int bits = argc > 8 ? atoi(argv[8]) : 40;
    Dumper d(outdir + "/p" + std::to_string(pid) + ".bin");

    auto t0 = std::chrono::steady_clock::now();
    double secs = 0;
    if (op == "prims") {
        run_prims<int32_t>(n, seed, d, "w4_");
        run_prims<int64_t>(n, seed + 1, d, "w8_");
        run_prims<int8_t>(n, seed + 2, d, "w1_");
    } else if (op == "join_time") {
        // Timing only: the relational pipeline of join_agg on n A rows and 4n B
        // rows with the distributions of the 2^22 x 2^24 configuration (group
        // key Zipf s=1.1 over 10^4 values by inverse CDF).
        uint64_t st = seed;
        const size_t na = n, nb = 4 * n;
        std::vector<double> cdf(10000);
        double acc = 0;
        for (int k = 0; k < 10000; k++) cdf[k] = (acc += 1.0 / std::pow(k + 1.0, 1.1));
        for (auto& c : cdf) c /= acc;
        orq::Vector<int64_t> pk(na), g(na), v(na), fk(nb), q(nb);
        for (size_t i = 0; i < na; i++) pk[i] = (int64_t)i;
        for (size_t i = na; i-- > 1;) std::swap(pk[i], pk[sm64(st) % (i + 1)]);
        for (size_t i = 0; i < na; i++) {
            double u = (double)(sm64(st) >> 11) * (1.0 / 9007199254740992.0);
            size_t k = std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin();
            g[i] = (int64_t)std::min<size_t>(k, 9999);
        }
        for (size_t i = 0; i < na; i++) v[i] = (int64_t)(sm64(st) % 1000000);
        for (size_t i = 0; i < nb; i++) fk[i] = (int64_t)(sm64(st) % na);
        for (size_t i = 0; i < nb; i++) q[i] = (int64_t)(1 + sm64(st) % 50);
        std::vector<orq::Vector<int64_t>> ca = {pk, g, v};
        std::vector<orq::Vector<int64_t>> cb = {fk, q};
        EncodedTable<int64_t> A = secret_share(ca, {"[K]", "[G]", "V"});
        EncodedTable<int64_t> B = secret_share(cb, {"[K]", "Q"});
        t0 = std::chrono::steady_clock::now();
        auto J = A.inner_join(B, {"[K]"}, {{"[G]", "[G]", copy<BSharedVector<int64_t>>},
                                           {"V", "V", copy<ASharedVector<int64_t>>}});
        J.addColumns(std::vector<std::string>{"VQ", "CNT"});
        J["VQ"] = J["V"] * J["Q"];
        J.aggregate({"[G]"}, {{"VQ", "VQ", sum<ASharedVector<int64_t>>},
                              {"CNT", "CNT", count<ASharedVector<int64_t>>}});
        secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        auto T = J.open_with_schema();
    } else if (op == "join_agg") {
        // The relational pipeline on small tables: A(n rows) = {[K] pk (a
        // Fisher-Yates permutation of 0..n-1), [G] group (0..4), V value
        // (< 10^6)}; B(2n rows) = {[K] fk (uniform over pk), Q quantity
        // (1..50)}. J = A.inner_join(B, [K], copy [G] and V); J.VQ = V*Q;
        // J.aggregate([G], sum VQ, count CNT). Every column of J is dumped.
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
        J.aggregate({"[G]"}, {{"VQ", "VQ", sum<ASharedVector<int64_t>>},
                              {"CNT", "CNT", count<ASharedVector<int64_t>>}});
        for (auto& name : J.getColumnNames()) {
            if (EncodedTable<int64_t>::isBShared(name)) {
                auto c = J.asBSharedVector(name);
                d.shares(name, c);
            } else {
                auto c = J.asASharedVector(name);
                d.shares(name, c);
            }
        }
        auto T = J.open_with_schema();
        for (size_t k = 0; k < T.second.size(); k++) d.plain("open_" + T.second[k], T.first[k]);
    } else if (op == "badd32" || op == "badd64") {
        // BSharedVector operator+ and operator- (the ripple-carry adder)
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            auto x = gen<T>(n, st, ~0ull);
            auto y = gen<T>(n, st, ~0ull);
            BSharedVector<T> xb = secret_share_b(x, 0);
            BSharedVector<T> yb = secret_share_b(y, 1);
            auto s = xb + yb;
            auto df = xb - yb;
            d.shares("sum", *s);
            d.shares("diff", *df);
            auto os = s->open(), od = df->open();
            d.plain("open_sum", os);
            d.plain("open_diff", od);
        };
        if (op == "badd32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "a2b32" || op == "a2b64") {
        // ASharedVector::a2b of values over all bits, shared by party 1
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            auto x = gen<T>(n, st, ~0ull);
            ASharedVector<T> xa = secret_share_a(x, 1);
            auto xb = xa.a2b();
            d.shares("xa", xa);
            d.shares("xb", *xb);
            auto o = xb->open();
            d.plain("open_xb", o);
        };
        if (op == "a2b32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "tshuffle") {
        // EncodedTable<int64_t> {[A], [B] (< 256), V (u32), [F] (bits)}:
        // filter on [F] (those rows invalid), then finalize(): shuffle() and
        // mask() of every column; each column dumped, and the open
        uint64_t st = seed;
        auto a = gen<int64_t>(n, st, ~0ull);
        auto b = gen<int64_t>(n, st, 0xff);
        auto v = gen<int64_t>(n, st, 0xffffffffull);
        auto f = gen<int64_t>(n, st, 1);
        std::vector<orq::Vector<int64_t>> cols = {a, b, v, f};
        EncodedTable<int64_t> T = secret_share(cols, {"[A]", "[B]", "V", "[F]"});
        T.filter(T["[F]"]);
        T.finalize();
        for (auto& name : T.getColumnNames()) {
            if (EncodedTable<int64_t>::isBShared(name)) {
                auto c = T.asBSharedVector(name);
                d.shares(name, c);
            } else {
                auto c = T.asASharedVector(name);
                d.shares(name, c);
            }
        }
        auto O = T.open_with_schema(false);
        for (size_t k = 0; k < O.second.size(); k++) d.plain("open_" + O.second[k], O.first[k]);
    } else if (op == "tsort" || op == "tsort_qs" || op == "distinct") {
        // tsort (tsort_qs): operators::table_sort with the radix (quicksort)
        // protocol on three key columns [bit ASC, small-int DESC, bit ASC] plus
        // one A and one B data column. distinct: operators::distinct over two
        // sorted key columns.
        using B = BSharedVector<int64_t>;
        using A = ASharedVector<int64_t>;
        uint64_t st = seed;
        auto v0 = gen<int64_t>(n, st, 1);
        auto v1 = gen<int64_t>(n, st, 7);
        auto v2 = gen<int64_t>(n, st, 1);
        auto va = gen<int64_t>(n, st, 0xffffffffull);
        auto vb = gen<int64_t>(n, st, ~0ull);
        B b0 = secret_share_b(v0, 0), b1 = secret_share_b(v1, 0), b2 = secret_share_b(v2, 0);
        A a0 = secret_share_a(va, 0);
        B b3 = secret_share_b(vb, 0);
        if (op != "distinct") {
            std::vector<B*> cols = {&b0, &b1, &b2};
            std::vector<A*> da = {&a0};
            std::vector<B*> db = {&b3};
            orq::operators::table_sort(cols, da, db,
                                       {orq::operators::SortOrder::ASC, orq::operators::SortOrder::DESC,
                                        orq::operators::SortOrder::ASC},
                                       {true, false, true},
                                       op == "tsort" ? orq::SortingProtocol::RADIXSORT
                                                     : orq::SortingProtocol::QUICKSORT);
            d.shares("c0", b0);
            d.shares("c1", b1);
            d.shares("c2", b2);
            d.shares("da", a0);
            d.shares("db", b3);
            auto o0 = b0.open(), o1 = b1.open(), o2 = b2.open();
            auto oa = a0.open();
            d.plain("open_c0", o0);
            d.plain("open_c1", o1);
            d.plain("open_c2", o2);
            d.plain("open_da", oa);
        } else {
            std::vector<B*> keys = {&b0, &b1};
            B res(n);
            orq::operators::distinct(keys, &res);
            d.shares("res", res);
            auto o = res.open();
            d.plain("open_res", o);
        }
    } else if (op == "radix" || op == "radix_time" || op == "radix_desc") {
        // radix_sort(key, ASC, bits) then apply the permutation to two
        // A-shared payloads (key uniform in [0, 2^bits), payloads u32).
        uint64_t st = seed;
        uint64_t km = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
        auto key = gen<int64_t>(n, st, km);
        auto p1 = gen<int64_t>(n, st, 0xffffffffull);
        auto p2 = gen<int64_t>(n, st, 0xffffffffull);
        BSharedVector<int64_t> kb = secret_share_b(key, 0);
        ASharedVector<int64_t> a1 = secret_share_a(p1, 0);
        ASharedVector<int64_t> a2 = secret_share_a(p2, 0);
        t0 = std::chrono::steady_clock::now();
        auto perm = orq::operators::radix_sort(
            kb, op == "radix_desc" ? orq::operators::SortOrder::DESC : orq::operators::SortOrder::ASC,
            bits);
        orq::operators::oblivious_apply_elementwise_perm(a1, perm);
        orq::operators::oblivious_apply_elementwise_perm(a2, perm);
        secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (op != "radix_time") {
            d.shares("key", kb);
            d.shares("pay1", a1);
            d.shares("pay2", a2);
            auto pa = perm.getASharedPerm();
            d.shares("perm", pa);
        }
        auto ko = kb.open();
        auto o1 = a1.open();
        auto o2 = a2.open();
        if (op != "radix_time") {
            d.plain("open_key", ko);
            d.plain("open_pay1", o1);
            d.plain("open_pay2", o2);
        }
    } else if (op == "bitonic32" || op == "bitonic64" || op == "bitonic32_desc" ||
               op == "bitonic_time") {
        // bitonic_sort(key) of one B-shared column (n a power of two), keys
        // uniform over all bits (sorted in the signed order)
        uint64_t st = seed;
        const bool desc = op == "bitonic32_desc";
        const auto order = desc ? orq::operators::SortOrder::DESC : orq::operators::SortOrder::ASC;
        if (op == "bitonic64") {
            auto key = gen<int64_t>(n, st, ~0ull);
            BSharedVector<int64_t> kb = secret_share_b(key, 0);
            orq::operators::bitonic_sort(kb, order);
            d.shares("key", kb);
            auto o = kb.open();
            d.plain("open_key", o);
        } else {
            auto key = gen<int32_t>(n, st, ~0ull);
            BSharedVector<int32_t> kb = secret_share_b(key, 0);
            t0 = std::chrono::steady_clock::now();
            orq::operators::bitonic_sort(kb, order);
            secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (op != "bitonic_time") {
                d.shares("key", kb);
                auto o = kb.open();
                d.plain("open_key", o);
            }
        }
    } else if (op == "qsort" || op == "qsort_desc" || op == "qsort32" || op == "qsort_time") {
        // quicksort(key, order) then the permutation applied to two A-shared
        // payloads of the key's type (int64 keys uniform in [0, 2^bits);
        // int32 keys over all 32 bits; payloads u32)
        uint64_t st = seed;
        const auto order =
            op == "qsort_desc" ? orq::operators::SortOrder::DESC : orq::operators::SortOrder::ASC;
        auto run = [&](auto tag, uint64_t km) {
            using T = decltype(tag);
            auto key = gen<T>(n, st, km);
            auto p1 = gen<T>(n, st, 0xffffffffull);
            auto p2 = gen<T>(n, st, 0xffffffffull);
            BSharedVector<T> kb = secret_share_b(key, 0);
            ASharedVector<T> a1 = secret_share_a(p1, 0);
            ASharedVector<T> a2 = secret_share_a(p2, 0);
            t0 = std::chrono::steady_clock::now();
            auto perm = orq::operators::quicksort(kb, order);
            orq::operators::oblivious_apply_elementwise_perm(a1, perm);
            orq::operators::oblivious_apply_elementwise_perm(a2, perm);
            secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (op == "qsort_time") return;
            d.shares("key", kb);
            d.shares("pay1", a1);
            d.shares("pay2", a2);
            auto pa = perm.getASharedPerm();
            d.shares("perm", pa);
            auto ko = kb.open(), o1 = a1.open(), o2 = a2.open();
            d.plain("open_key", ko);
            d.plain("open_pay1", o1);
            d.plain("open_pay2", o2);
        };
        if (op == "qsort32") run(int32_t{}, ~0ull);
        else run(int64_t{}, bits >= 64 ? ~0ull : ((1ull << bits) - 1));
    } else if (op == "rows32" || op == "rows64") {
        // bitonic_sort over two key columns (k0 in [-4, 3], so rows tie on
        // it, ASC; k1 over all bits, DESC) with one B and two A data columns
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            using B = BSharedVector<T>;
            using A = ASharedVector<T>;
            using orq::operators::SortOrder;
            auto k0 = gen<T>(n, st, 7);
            for (size_t i = 0; i < n; i++) k0[i] = (T)(k0[i] - 4);
            auto k1 = gen<T>(n, st, ~0ull);
            auto b0 = gen<T>(n, st, ~0ull);
            auto a0 = gen<T>(n, st, 0xffffffffull);
            auto a1 = gen<T>(n, st, 0xffffull);
            B K0 = secret_share_b(k0, 0), K1 = secret_share_b(k1, 1), B0 = secret_share_b(b0, 2);
            A A0 = secret_share_a(a0, 0), A1 = secret_share_a(a1, 1);
            orq::operators::bitonic_sort(std::vector<B*>{&K0, &K1}, std::vector<A*>{&A0, &A1},
                                         std::vector<B*>{&B0}, {SortOrder::ASC, SortOrder::DESC});
            d.shares("k0", K0);
            d.shares("k1", K1);
            d.shares("b0", B0);
            d.shares("a0", A0);
            d.shares("a1", A1);
            auto o0 = K0.open(), o1 = K1.open(), ob = B0.open(), oa0 = A0.open(), oa1 = A1.open();
            d.plain("open_k0", o0);
            d.plain("open_k1", o1);
            d.plain("open_b0", ob);
            d.plain("open_a0", oa0);
            d.plain("open_a1", oa1);
        };
        if (op == "rows32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "cmprows32" || op == "cmprows64") {
        // compare_rows of (x0, x1) vs (y0, y1), x0/y0 in [0, 3] (ties), key 0
        // ASC and key 1 DESC; then extend_lsb, multiplex (B and A), and swap
        // of the key columns and of two A columns with b2a_bit of the bits
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            using B = BSharedVector<T>;
            using A = ASharedVector<T>;
            using orq::operators::SortOrder;
            auto x0 = gen<T>(n, st, 3);
            auto y0 = gen<T>(n, st, 3);
            auto x1 = gen<T>(n, st, ~0ull);
            auto y1 = gen<T>(n, st, ~0ull);
            for (size_t i = 0; i < n; i += 4) y1[i] = x1[i];
            auto u = gen<T>(n, st, 0xffffffffull);
            auto v = gen<T>(n, st, 0xffffffffull);
            B X0 = secret_share_b(x0, 0), X1 = secret_share_b(x1, 0);
            B Y0 = secret_share_b(y0, 1), Y1 = secret_share_b(y1, 1);
            A U = secret_share_a(u, 2), V = secret_share_a(v, 2);
            B gt = orq::operators::compare_rows(std::vector<B*>{&X0, &X1}, std::vector<B*>{&Y0, &Y1},
                                                {SortOrder::ASC, SortOrder::DESC});
            d.shares("gt", gt);
            auto gta = gt.b2a_bit();
            d.shares("gta", *gta);
            B ext(n);
            ext.extend_lsb(gt);
            d.shares("ext", ext);
            B mb = orq::operators::multiplex(gt, X1, Y1);
            d.shares("mux_b", mb);
            A ma = orq::operators::multiplex(*gta, U, V);
            d.shares("mux_a", ma);
            std::vector<B*> px{&X0, &X1}, py{&Y0, &Y1};
            orq::operators::swap(px, py, gt);
            std::vector<A*> pu{&U}, pv{&V};
            orq::operators::swap(pu, pv, *gta);
            d.shares("x0", X0);
            d.shares("x1", X1);
            d.shares("y0", Y0);
            d.shares("y1", Y1);
            d.shares("u", U);
            d.shares("v", V);
            auto og = gt.open(), ox1 = X1.open(), oy1 = Y1.open(), ou = U.open(), ov = V.open();
            d.plain("open_gt", og);
            d.plain("open_x1", ox1);
            d.plain("open_y1", oy1);
            d.plain("open_u", ou);
            d.plain("open_v", ov);
        };
        if (op == "cmprows32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "relops32" || op == "relops64") {
        // operator== != >= <= of B-shared x vs y, in that order; a quarter of
        // the pairs are equal
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            auto x = gen<T>(n, st, ~0ull);
            auto y = gen<T>(n, st, ~0ull);
            for (size_t i = 0; i < n; i += 4) y[i] = x[i];
            BSharedVector<T> xb = secret_share_b(x, 0);
            BSharedVector<T> yb = secret_share_b(y, 1);
            auto e = xb == yb;
            auto ne = xb != yb;
            auto ge = xb >= yb;
            auto le = xb <= yb;
            d.shares("eq", *e);
            d.shares("ne", *ne);
            d.shares("ge", *ge);
            d.shares("le", *le);
            auto oe = e->open(), one = ne->open(), oge = ge->open(), ole = le->open();
            d.plain("open_eq", oe);
            d.plain("open_ne", one);
            d.plain("open_ge", oge);
            d.plain("open_le", ole);
        };
        if (op == "relops32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "compare32" || op == "compare64") {
        // BSharedVector::_compare of x vs y; a quarter of the pairs are equal
        uint64_t st = seed;
        auto run = [&](auto tag) {
            using T = decltype(tag);
            auto x = gen<T>(n, st, ~0ull);
            auto y = gen<T>(n, st, ~0ull);
            for (size_t i = 0; i < n; i += 4) y[i] = x[i];
            BSharedVector<T> xb = secret_share_b(x, 0);
            BSharedVector<T> yb = secret_share_b(y, 1);
            BSharedVector<T> eq(n), gt(n);
            xb._compare(yb, eq, gt);
            d.shares("xb", xb);
            d.shares("yb", yb);
            d.shares("eq", eq);
            d.shares("gt", gt);
            auto oe = eq.open();
            auto og = gt.open();
            d.plain("open_eq", oe);
            d.plain("open_gt", og);
        };
        if (op == "compare32") run(int32_t{});
        else run(int64_t{});
    } else if (op == "agg_fwd" || op == "agg_rev" || op == "agg_nokey") {
        // orq::aggregators::aggregate over n (power of two) int64 rows.
        // key0: sorted, values in [0, n/4]; key1 (agg_rev): sorted within
        // key0 runs, values in {0, 1}; sel (agg_rev): random table-id bits.
        // A specs: sum, count, copy; B specs: copy, valid, bit_or, max, min.
        using B = BSharedVector<int64_t>;
        using A = ASharedVector<int64_t>;
        namespace ag = orq::aggregators;
        uint64_t st = seed;
        std::vector<std::pair<int64_t, int64_t>> kv(n);
        for (size_t i = 0; i < n; i++)
            kv[i] = {(int64_t)(sm64(st) % (n / 4 + 1)), (int64_t)(sm64(st) & 1)};
        std::sort(kv.begin(), kv.end());
        orq::Vector<int64_t> k0(n), k1(n);
        for (size_t i = 0; i < n; i++) {
            k0[i] = kv[i].first;
            k1[i] = kv[i].second;
        }
        auto va1 = gen<int64_t>(n, st, 0xffffffffull);
        auto va3 = gen<int64_t>(n, st, 0xffffffffull);
        auto vb1 = gen<int64_t>(n, st, ~0ull);
        auto vb2 = gen<int64_t>(n, st, 1);
        auto vb3 = gen<int64_t>(n, st, ~0ull);
        auto vb4 = gen<int64_t>(n, st, ~0ull);
        auto vb5 = gen<int64_t>(n, st, ~0ull);
        auto sv = gen<int64_t>(n, st, 1);
        std::vector<B> keys;
        if (op != "agg_nokey") keys.push_back(secret_share_b(k0, 0));
        if (op == "agg_rev") keys.push_back(secret_share_b(k1, 0));
        A a1 = secret_share_a(va1, 0), a3 = secret_share_a(va3, 0);
        B b1 = secret_share_b(vb1, 0), b2 = secret_share_b(vb2, 0), b3 = secret_share_b(vb3, 0);
        B b4 = secret_share_b(vb4, 0), b5 = secret_share_b(vb5, 0);
        B sel = secret_share_b(sv, 0);
        A o1(n), o2(n), o3(n);
        B q1(n), q2(n), q3(n), q4(n), q5(n);
        std::vector<std::tuple<B, B, void (*)(const B&, B&, const B&)>> bs = {
            {b1, q1, &ag::copy<B>}, {b2, q2, &ag::valid<B>}, {b3, q3, &ag::bit_or<B>},
            {b4, q4, &ag::max<B>}, {b5, q5, &ag::min<B>}};
        std::vector<std::tuple<A, A, void (*)(const A&, A&, const A&)>> as = {
            {a1, o1, &ag::sum<A>}, {a1, o2, &ag::count<A>}, {a3, o3, &ag::copy<A>}};
        if (op == "agg_nokey") {
            bs.erase(bs.begin() + 1, bs.end());
            as.erase(as.begin() + 1, as.end());
        }
        if (op == "agg_rev")
            ag::aggregate(keys, bs, as, ag::Direction::Reverse, std::optional<B>(sel));
        else
            ag::aggregate(keys, bs, as, ag::Direction::Forward);
        d.shares("o1", o1);
        d.shares("q1", q1);
        if (op != "agg_nokey") {
            d.shares("o2", o2);
            d.shares("o3", o3);
            d.shares("q2", q2);
            d.shares("q3", q3);
            d.shares("q4", q4);
            d.shares("q5", q5);
        }
        auto x1 = o1.open();
        d.plain("open_o1", x1);
    } else if (op == "prims_time") {
        // ORQ's micro_primitives sequence on n 32-bit elements: AND, MULT, EQ,
        // GR, RCA (binary +), each timed; prints one JSON line of seconds
        uint64_t st = seed;
        auto x = gen<int32_t>(n, st, ~0ull);
        auto y = gen<int32_t>(n, st, ~0ull);
        BSharedVector<int32_t> xb = secret_share_b(x, 0), yb = secret_share_b(y, 1);
        ASharedVector<int32_t> xa = secret_share_a(x, 0), ya = secret_share_a(y, 1);
        double t[5];
        auto tick = [] { return std::chrono::steady_clock::now(); };
        auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
        auto a0 = tick();
        auto r0 = xb & yb;
        auto a1 = tick();
        auto r1 = xa * ya;
        auto a2 = tick();
        auto r2 = xb == yb;
        auto a3 = tick();
        auto r3 = xb > yb;
        auto a4 = tick();
        auto r4 = xb + yb;
        auto a5 = tick();
        t[0] = sec(a0, a1), t[1] = sec(a1, a2), t[2] = sec(a2, a3), t[3] = sec(a3, a4), t[4] = sec(a4, a5);
        secs = sec(a0, a5);
        if (pid == 0)
            printf("{\"prims\": {\"AND\": %.6f, \"MULT\": %.6f, \"EQ\": %.6f, \"GR\": %.6f, \"RCA\": %.6f}}\n",
                   t[0], t[1], t[2], t[3], t[4]);
        (void)r0, (void)r1, (void)r2, (void)r3, (void)r4;
    } else if (op == "shuffle") {
        uint64_t st = seed;
        auto x = gen<int32_t>(n, st, ~0ull);
        BSharedVector<int32_t> xb = secret_share_b(x, 0);
        orq::operators::shuffle(xb);
        d.shares("shuffled", xb);
        auto o = xb.open();
        d.plain("open_shuffled", o);
    } else if (op == "setup") {
        // orq_init alone: the key exchange of setup_random_generation
    } else {
        fprintf(stderr, "unknown op %s\n", op.c_str());
        return 2;
    }
    if (pid == 0) printf("{\"op\": \"%s\", \"n\": %zu, \"seconds\": %.6f}\n", op.c_str(), n, secs);
    return 0;
}
