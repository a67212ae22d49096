// ref_driver_np.cpp — runs ORQ's own Beaver-2PC (dummy triples) or
// Fantastic-4PC code on seeded inputs and dumps every party's local shares,
// so the loopback GPU path can be compared with the reference share by share.
//
// TEST INFRASTRUCTURE ONLY: built from the ORQ headers by oracle/Makefile
// (PROTOCOL_NUM=2 or 4) into oracle/_ref/, launched as two or four local party
// processes by oracle/run_ref.py over ORQ's NoCopy socket communicator.
//
// usage: ref_driver_np <threads> <p_factor> <batch> prims <n> <data_seed> <outdir>
// Record format: u32 name length, name, u32 width, u64 n, u32 k, then the k
// local share columns of this party (k = 1 for 2PC, 3 for 4PC; 1 for opened
// values).
#include <cstdio>
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

#if PROTOCOL_NUM == 4
constexpr int kLocal = 3;
#else
constexpr int kLocal = 1;
#endif

struct Dumper {
    std::ofstream f;
    explicit Dumper(const std::string& path) : f(path, std::ios::binary) {}
    template <typename T>
    void head(const std::string& name, uint64_t n, uint32_t k) {
        uint32_t nl = name.size(), w = sizeof(T);
        f.write((const char*)&nl, 4);
        f.write(name.data(), nl);
        f.write((const char*)&w, 4);
        f.write((const char*)&n, 8);
        f.write((const char*)&k, 4);
    }
    template <typename T>
    void col(const orq::Vector<T>& a) {
        for (uint64_t i = 0; i < a.size(); i++) {
            T v = a[i];
            f.write((const char*)&v, sizeof(T));
        }
    }
    template <typename SV>
    void shares(const std::string& name, SV& v) {
        using T = std::remove_cv_t<std::remove_reference_t<decltype(v.vector(0)[0])>>;
        head<T>(name, v.size(), kLocal);
        for (int k = 0; k < kLocal; k++) col(v.vector(k));
    }
    template <typename T>
    void plain(const std::string& name, const orq::Vector<T>& a) {
        head<T>(name, a.size(), 1);
        col(a);
    }
};

template <typename T>
static orq::Vector<T> gen(size_t n, uint64_t& st) {
    orq::Vector<T> v(n);
    for (size_t i = 0; i < n; i++) v[i] = (T)sm64(st);
    return v;
}

// The primitive sequence: shares from two owners, and_b, xor_b, multiply_a,
// add_a, b2a_bit, opens.
template <typename T>
static void run_prims(size_t n, uint64_t seed, Dumper& d, const std::string& tag) {
    uint64_t st = seed;
    auto x = gen<T>(n, st);
    auto y = gen<T>(n, st);
    BSharedVector<T> xb = secret_share_b(x, 0);
    BSharedVector<T> yb = secret_share_b(y, 1);
    d.shares(tag + "xb", xb);
    d.shares(tag + "yb", yb);
    BSharedVector<T> zb = xb & yb;
    d.shares(tag + "and", zb);
    BSharedVector<T> xo = xb ^ yb;
    d.shares(tag + "xor", xo);
    ASharedVector<T> xa = secret_share_a(x, 1);
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
        fprintf(stderr, "usage: ref_driver_np t p batch op n seed outdir\n");
        return 2;
    }
    std::string op = argv[4];
    size_t n = std::stoull(argv[5]);
    uint64_t seed = std::stoull(argv[6]);
    std::string outdir = argv[7];
    Dumper d(outdir + "/p" + std::to_string(pid) + ".bin");
    if (op == "prims") {
        run_prims<int32_t>(n, seed, d, "w4_");
        run_prims<int64_t>(n, seed + 1, d, "w8_");
        run_prims<int8_t>(n, seed + 2, d, "w1_");
    } else {
        fprintf(stderr, "unknown op %s\n", op.c_str());
        return 2;
    }
    d.f.close();
#ifdef MALICIOUS_PROTOCOL
    // the honest run's transcript hashes agree
    runTime->malicious_check();
#endif
    return 0;
}
