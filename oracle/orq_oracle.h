/*
 * orq_oracle.h — CPU restatement of ORQ's replicated-3PC share computation.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product (orq_b200/, liborq_cuda.so) never links or calls it.
 *
 * Layout: all three parties live in one process ("loopback"). A 3PC shared
 * vector is stored as its three distinct share arrays S[0], S[1], S[2]; party p
 * holds the replicated pair (S[p], S[(p+1)%3]) exactly as get_shares_b/a hand
 * them out (reference: include/core/protocols/replicated_3pc.h:353-392).
 *
 * Parity is pinned two ways:
 *   - the AES-256 / GCM keystream against NIST-style known answers produced by
 *     Python `cryptography` (tests/golden/aes_gcm_kat.json);
 *   - every primitive and the radix sort against per-party share dumps of the
 *     reference itself, built from its own headers with a deterministic
 *     libsodium shim (oracle/ref_shim, oracle/Makefile) — tests/golden/*.bin.
 */
#ifndef ORQ_ORACLE_H
#define ORQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- deterministic key derivation (shared with the shim and the device) ---- */
uint64_t oro_splitmix64(uint64_t* state);
/* 32-byte AES key for keygen call `call` of party `party` under `seed`. */
void oro_derive_key(uint64_t seed, int party, int call, uint8_t key[32]);

/* ---- AES-256 (FIPS-197) ---- */
void oro_aes256_expand(const uint8_t key[32], uint32_t rk[60]);
void oro_aes256_encrypt(const uint32_t rk[60], const uint8_t in[16], uint8_t out[16]);

/* ---- GCM-mode keystream as ORQ's AESPRGAlgorithm consumes it ----
 * (include/core/random/prg/prg_algorithm.h:161-172,214-231): the buffer is cut
 * into 1 MiB chunks, chunk c is AES-GCM over zeros under nonce (nonce0 + c)
 * written little-endian into the 12-byte IV; block j of a chunk is
 * AES_K(IV || BE32(j + 2)). Returns the number of nonces consumed. */
uint64_t oro_keystream(const uint32_t rk[60], uint64_t nonce0, uint8_t* out, size_t nbytes);

/* ---- loopback context ---- */
enum {
    ORO_PAIR0 = 0, /* stream shared by P0/P1, keyed by P0's local key */
    ORO_PAIR1 = 1, /* P1/P2 */
    ORO_PAIR2 = 2, /* P2/P0 */
    ORO_G01 = 3,
    ORO_G02 = 4,
    ORO_G12 = 5,
    ORO_G012 = 6,
    ORO_LOCAL0 = 7,
    ORO_LOCAL1 = 8,
    ORO_LOCAL2 = 9,
    ORO_NSTREAMS = 10
};

typedef struct {
    uint32_t rk[ORO_NSTREAMS][60];
    uint64_t nonce[ORO_NSTREAMS];
} oro_ctx;

void oro_ctx_init(oro_ctx* c, uint64_t seed);
/* getNext(Vector<T>) of n elements of w bytes from stream s. */
void oro_stream_fill(oro_ctx* c, int s, void* out, size_t n, int w);

/* ---- primitives; x, y, z are arrays of three share pointers ----
 * w in {1,2,4,8,16} bytes. Arithmetic is mod 2^(8w). */
void oro_secret_share(oro_ctx* c, int arith, int w, size_t n, const void* data, int data_party,
                      void* s[3]);
void oro_public_share(int w, size_t n, const void* data, void* s[3]);
void oro_open(int arith, int w, size_t n, void* const s[3], void* out);
void oro_xor_b(int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_and_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_add_a(int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_sub_a(int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_mul_a(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_b2a_bit(oro_ctx* c, int w, size_t n, void* const x[3], void* y[3]);
void oro_reshare(oro_ctx* c, int arith, int w, size_t n, int group, void* s[3]);
void oro_zero_share(oro_ctx* c, int arith, int w, size_t n, void* r[3]);

/* Fisher–Yates from a group stream (hm_sharded_permutation_generator.h:70-108).
 * Returns the number of u32 draws consumed. */
uint64_t oro_gen_perm(oro_ctx* c, int stream, int32_t* perm, size_t n);
void oro_shuffle(oro_ctx* c, int arith, int w, size_t n, void* s[3]);
void oro_prefix_sum(int w, size_t n, void* s[3]);

/* radix_sort(v, ASC|DESC, bits) on an int32/int64 B-shared key followed by
 * oblivious_apply_elementwise_perm of each A-shared payload (64-bit) with the
 * returned permutation (radixsort.h:116-229, shuffle.h:687-706). The key is
 * sorted in place; the returned elementwise permutation (A-shared int32) is
 * written to perm_out if non-NULL. */
void oro_radix_sort(oro_ctx* c, int kw, size_t n, void* key[3], int bits, int desc,
                    int npayload, void** payloads /* npayload x 3 pointers, int64 */,
                    int32_t* perm_out[3]);

/* BSharedVector::_compare (circuits.h:231-295) of int32/int64 B-shared keys:
 * eq = (x == y), gt = (x > y) signed, each as B-shared bits in the LSB. */
void oro_compare(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* eq[3],
                 void* gt[3]);
/* bitonic_sort (sorting.h:266-353) of one B-shared int32/int64 key column in
 * place; n a power of two. */
void oro_bitonic_sort(oro_ctx* c, int w, size_t n, void* key[3], int desc);

/* aggregation functions (operators/aggregation.h:27-140) */
enum { ORO_AGG_SUM = 0, ORO_AGG_COUNT = 1, ORO_AGG_COPY = 2, ORO_AGG_VALID = 3, ORO_AGG_BIT_OR = 4,
       ORO_AGG_MIN = 5, ORO_AGG_MAX = 6 };
/* orq::aggregators::aggregate (aggregation.h:167-346) over n (a power of two)
 * rows of w-byte shares: keys are nkeys B-shared columns (3 pointers each),
 * b_in/b_out/b_func the boolean specs (copy/valid/bit_or/min/max), a_in/a_out/
 * a_func the arithmetic specs (sum/count/copy); sel (3 pointers) or NULL. */
void oro_aggregate(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys, int nb,
                   void* const* b_in, void* const* b_out, const int* b_func, int na,
                   void* const* a_in, void* const* a_out, const int* a_func, int reverse,
                   void* const* sel);

/* compose_permutations (shuffle.h:717-743) of two A-shared int32 elementwise
 * permutations; sigma is consumed, the result is written to rho. */
void oro_compose_permutations(oro_ctx* c, size_t n, int32_t* sigma[3], int32_t* rho[3]);
/* table_sort (sorting.h:509-612) with the radix sort protocol: ncols key
 * columns (3 pointers each) with per-column order and single-bit flags, then
 * na arithmetic and nb boolean data columns permuted along. */
void oro_table_sort(oro_ctx* c, int w, size_t n, int ncols, void* const* cols, const int* desc,
                    const int* single_bit, int na, void* const* data_a, int nb,
                    void* const* data_b, int quick);
/* distinct (distinct.h:20-53): res marks the first row of every run of equal
 * keys (adjacent rows only). */
void oro_distinct(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys, void* res[3]);

/* operator== (b_shared_vector.h:493-504) and not_b_1 (replicated_3pc.h:207). */
void oro_equal(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* eq[3]);
void oro_not_b1(int w, size_t n, void* const x[3], void* y[3]);
void oro_extend_lsb(int w, size_t n, void* const x[3], void* y[3]);
void oro_a2b(oro_ctx* c, int w, size_t n, void* const x[3], void* y[3]);
void oro_add_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_sub_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]);
void oro_quicksort(oro_ctx* c, int kw, size_t n, void* key[3], int desc, int npayload,
                   void** payloads, int32_t* perm_out[3]);
void oro_compare_rows(oro_ctx* c, int w, size_t n, int nkeys, void* const* x, void* const* y,
                      const int* desc, void* gt[3]);
void oro_swap(oro_ctx* c, int arith, int w, size_t n, int ncols, void* const* x, void* const* y,
              void* const bits[3]);
void oro_bitonic_sort_rows(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys,
                           const int* desc, int na, void* const* data_a, int nb,
                           void* const* data_b);

/* ---- Beaver 2PC with dummy triples and Fantastic-4PC: the local steps ----
 * A context for `nparties` = 2 or 4 holds that protocol's streams:
 *   2PC: ORO_P2_COMMON (group {0,1}, P0's keygen call 1), ORO_P2_LOCAL0/1;
 *   4PC: ORO_P4_NOT0..3 (the PRG shared by the three parties other than e,
 *        keyed by party e-1's setup_4pc_common_prgs key), ORO_P4_LOCAL0..3.
 * A 2PC vector is S[0], S[1] (party p holds S[p]); a 4PC vector is X[0..3]
 * where X[j] is the share party j lacks (party p holds X[p+1], X[p+2],
 * X[p+3] as its local shares 0, 1, 2). */
enum { ORO_P2_COMMON = 0, ORO_P2_LOCAL0 = 1, ORO_P2_LOCAL1 = 2 };
enum { ORO_P4_NOT0 = 0, ORO_P4_LOCAL0 = 4 };
void oro_ctx_init_np(oro_ctx* c, uint64_t seed, int nparties);
void oro_np_secret_share(oro_ctx* c, int np, int arith, int w, size_t n, const void* data, int d,
                         void* const* s);
void oro_np_open(int np, int arith, int w, size_t n, void* const* s, void* out);
void oro_np_mult(oro_ctx* c, int np, int arith, int w, size_t n, void* const* x, void* const* y,
                 void* const* z);
void oro_np_b2a_bit(oro_ctx* c, int np, int w, size_t n, void* const* x, void* const* y);
void oro_np_local(int np, int op, int w, size_t n, void* const* x, void* const* y, void* const* z);

#ifdef __cplusplus
}
#endif
#endif
