// gpu_party.cpp — one party of replicated 3PC on the GPU, run among CPU
// parties of the reference (oracle/_ref/ref_driver) over ORQ's NoCopy wire.
// Run by tests/test_nocopy_party.py.
//
//   gpu_party <threads> <p_factor> <batch> <op> <n> <seed> <outdir> [bits]
//
// takes ref_driver's arguments and startmpc's environment (STARTMPC_*), and
// the key seed from ORQ_SEED (the reference build's deterministic key seed).
//   op "setup": only the setup of random generation; writes the party's keys
//               (local, own pairwise, received pairwise, groups) as hex to
//               <outdir>/p<rank>.keys — needs no GPU.
//   op "prims": ref_driver's prims sequence on int32, int64, int8, dumping
//               this party's two shares of every vector to <outdir>/p<rank>.bin
//               in ref_driver's record format.
#include <cstdio>
#include <fstream>
#include <string>

#include "party.hpp"

using orq::gpu_party::Party3PC;
using orq::gpu_party::PShares;

static uint64_t sm64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// ref_driver's Dumper: name, width, n, first column, second column
struct Dumper {
    std::ofstream f;
    explicit Dumper(const std::string& path) : f(path, std::ios::binary) {}
    template <typename T>
    void rec(const std::string& name, const std::vector<T>& a, const std::vector<T>& b) {
        uint32_t nl = name.size(), w = sizeof(T);
        uint64_t n = a.size();
        f.write((const char*)&nl, 4);
        f.write(name.data(), nl);
        f.write((const char*)&w, 4);
        f.write((const char*)&n, 8);
        f.write((const char*)a.data(), n * sizeof(T));
        f.write((const char*)b.data(), n * sizeof(T));
    }
    template <typename T>
    void shares(const std::string& name, const PShares<T>& v) {
        rec(name, v.download(0), v.download(1));
    }
    template <typename T>
    void plain(const std::string& name, const orq::Vector<T>& a) {
        rec(name, a.std(), a.std());
    }
};

template <typename T>
static orq::Vector<T> gen(size_t n, uint64_t& st) {
    orq::Vector<T> v(n);
    for (size_t i = 0; i < n; i++) v[i] = (T)sm64(st);
    return v;
}

// the sequence of ref_driver.cpp's run_prims, party-local
template <typename T>
static void run_prims(Party3PC& P, size_t n, uint64_t seed, Dumper& d, const std::string& tag) {
    uint64_t st = seed;
    auto x = gen<T>(n, st);
    auto y = gen<T>(n, st);
    auto xb = P.secret_share_b(x, 0);
    auto yb = P.secret_share_b(y, 1);
    d.shares(tag + "xb", xb);
    d.shares(tag + "yb", yb);
    auto zb = P.and_b(xb, yb);
    d.shares(tag + "and", zb);
    auto xo = P.xor_b(xb, yb);
    d.shares(tag + "xor", xo);
    auto xa = P.secret_share_a(x, 2);
    auto ya = P.secret_share_a(y, 0);
    d.shares(tag + "xa", xa);
    d.shares(tag + "ya", ya);
    auto za = P.multiply_a(xa, ya);
    d.shares(tag + "mul", za);
    auto sa = P.add_a(xa, ya);
    d.shares(tag + "add", sa);
    auto ba = P.b2a_bit(xb);
    d.shares(tag + "b2a", ba);
    auto o1 = P.open_b(zb);
    auto o2 = P.open_a(za);
    auto o3 = P.open_a(ba);
    d.plain(tag + "open_and", o1);
    d.plain(tag + "open_mul", o2);
    d.plain(tag + "open_b2a", o3);
}

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: gpu_party t p batch op n seed outdir [bits]\n");
        return 2;
    }
    const std::string op = argv[4];
    const size_t n = std::stoull(argv[5]);
    const uint64_t seed = std::stoull(argv[6]);
    const std::string outdir = argv[7];
    const char* ks = std::getenv("ORQ_SEED");
    const uint64_t key_seed = ks ? std::strtoull(ks, nullptr, 10) : 1ull;
    auto keygen = [&](int party, int call, uint8_t* key) { orq::orqcu_check(orqcu_keygen(key_seed, party, call, key)); };
    try {
        auto ep = orq::nocopy::Endpoint::from_env(3);
        const int rank = ep.rank();
        if (op == "setup") {
            const auto K = orq::gpu_party::setup_keys(ep, keygen);
            std::ofstream f(outdir + "/p" + std::to_string(rank) + ".keys");
            auto hex = [&](const char* name, const std::array<uint8_t, 32>& k) {
                f << name << " ";
                for (uint8_t b : k) {
                    char h[3];
                    std::snprintf(h, sizeof(h), "%02x", b);
                    f << h;
                }
                f << "\n";
            };
            hex("local", K.local);
            hex("own", K.own);
            hex("prev", K.prev);
            const char* gname[4] = {"g01", "g02", "g12", "g012"};
            for (int g = 0; g < 4; g++)
                if (K.have[g]) hex(gname[g], K.group[g]);
            return 0;
        }
        int device = 0;
        if (const char* d = std::getenv("ORQ_DEVICE")) device = std::atoi(d);
        Party3PC P(ep, device, keygen);
        Dumper d(outdir + "/p" + std::to_string(rank) + ".bin");
        if (op == "prims") {
            run_prims<int32_t>(P, n, seed, d, "w4_");
            run_prims<int64_t>(P, n, seed + 1, d, "w8_");
            run_prims<int8_t>(P, n, seed + 2, d, "w1_");
        } else {
            std::fprintf(stderr, "unknown op %s\n", op.c_str());
            return 2;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
