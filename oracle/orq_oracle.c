/*
 * orq_oracle.c — CPU restatement of ORQ's replicated-3PC local share computation.
 *
 * TEST INFRASTRUCTURE ONLY (see orq_oracle.h). Plain C, one thread, all three
 * parties in one process. Each function cites the reference lines it restates;
 * paths are relative to the ORQ source tree.
 */
#include "orq_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__)
#include <immintrin.h>
#define ORO_HAVE_AESNI 1
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* Key derivation. The reference draws every AES key from libsodium's
 * crypto_aead_aes256gcm_keygen (prg_algorithm.h:192-197). For reproducible
 * runs, the test shim and this library replace that with SplitMix64 (Steele,
 * Lea, Flood, OOPSLA 2014) keyed by (seed, party, keygen call index). */
uint64_t oro_splitmix64(uint64_t* state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void oro_derive_key(uint64_t seed, int party, int call, uint8_t key[32]) {
    uint64_t st = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(party + 1)) ^
                  (0xABC98388FB8FAC03ull * (uint64_t)(call + 1));
    for (int i = 0; i < 4; i++) {
        uint64_t v = oro_splitmix64(&st);
        for (int b = 0; b < 8; b++) key[8 * i + b] = (uint8_t)(v >> (8 * b));
    }
}

/* ------------------------------------------------------------------------- */
/* AES-256 from FIPS-197: S-box built from the GF(2^8) inverse and the affine
 * map, byte-oriented rounds. */
static uint8_t g_sbox[256];
static int g_sbox_ready = 0;

static uint8_t gf_mul(uint8_t a, uint8_t b) {
    uint8_t p = 0;
    while (b) {
        if (b & 1) p ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1B : 0));
        b >>= 1;
    }
    return p;
}

static void build_sbox(void) {
    if (g_sbox_ready) return;
    for (int x = 0; x < 256; x++) {
        uint8_t inv = 0;
        if (x) {
            for (int y = 1; y < 256; y++)
                if (gf_mul((uint8_t)x, (uint8_t)y) == 1) {
                    inv = (uint8_t)y;
                    break;
                }
        }
        uint8_t s = inv;
        uint8_t r = inv;
        for (int i = 0; i < 4; i++) {
            r = (uint8_t)((r << 1) | (r >> 7));
            s ^= r;
        }
        g_sbox[x] = s ^ 0x63;
    }
    g_sbox_ready = 1;
}

static uint32_t sub_word(uint32_t w) {
    return (uint32_t)g_sbox[w & 0xff] | ((uint32_t)g_sbox[(w >> 8) & 0xff] << 8) |
           ((uint32_t)g_sbox[(w >> 16) & 0xff] << 16) | ((uint32_t)g_sbox[w >> 24] << 24);
}

/* Round keys as little-endian words: word i holds key bytes 4i..4i+3. */
void oro_aes256_expand(const uint8_t key[32], uint32_t rk[60]) {
    build_sbox();
    for (int i = 0; i < 8; i++)
        rk[i] = (uint32_t)key[4 * i] | ((uint32_t)key[4 * i + 1] << 8) |
                ((uint32_t)key[4 * i + 2] << 16) | ((uint32_t)key[4 * i + 3] << 24);
    uint8_t rcon = 1;
    for (int i = 8; i < 60; i++) {
        uint32_t t = rk[i - 1];
        if (i % 8 == 0) {
            t = (t >> 8) | (t << 24); /* RotWord on the byte order */
            t = sub_word(t) ^ rcon;
            rcon = gf_mul(rcon, 2);
        } else if (i % 8 == 4) {
            t = sub_word(t);
        }
        rk[i] = rk[i - 8] ^ t;
    }
}

void oro_aes256_encrypt(const uint32_t rk[60], const uint8_t in[16], uint8_t out[16]) {
    uint8_t s[16], t[16];
    for (int i = 0; i < 16; i++) s[i] = in[i] ^ (uint8_t)(rk[i / 4] >> (8 * (i % 4)));
    for (int round = 1; round <= 14; round++) {
        /* SubBytes + ShiftRows: state byte (row r, col c) is s[4c + r] */
        for (int c = 0; c < 4; c++)
            for (int r = 0; r < 4; r++) t[4 * c + r] = g_sbox[s[4 * ((c + r) % 4) + r]];
        if (round != 14) {
            for (int c = 0; c < 4; c++) {
                uint8_t a0 = t[4 * c], a1 = t[4 * c + 1], a2 = t[4 * c + 2], a3 = t[4 * c + 3];
                s[4 * c + 0] = gf_mul(a0, 2) ^ gf_mul(a1, 3) ^ a2 ^ a3;
                s[4 * c + 1] = a0 ^ gf_mul(a1, 2) ^ gf_mul(a2, 3) ^ a3;
                s[4 * c + 2] = a0 ^ a1 ^ gf_mul(a2, 2) ^ gf_mul(a3, 3);
                s[4 * c + 3] = gf_mul(a0, 3) ^ a1 ^ a2 ^ gf_mul(a3, 2);
            }
        } else {
            memcpy(s, t, 16);
        }
        for (int i = 0; i < 16; i++) s[i] ^= (uint8_t)(rk[4 * round + i / 4] >> (8 * (i % 4)));
    }
    memcpy(out, s, 16);
}

#ifdef ORO_HAVE_AESNI
/* Same cipher on the x86 AES instructions (only a speed-up for the checker;
 * the round keys are the FIPS-197 schedule above, read as bytes). */
__attribute__((target("aes,sse4.1"))) static void aesni_ctr_chunk(const uint32_t rk[60],
                                                                   uint64_t nonce, uint8_t* out,
                                                                   size_t len) {
    __m128i k[15];
    for (int r = 0; r < 15; r++) k[r] = _mm_loadu_si128((const __m128i*)(rk + 4 * r));
    uint8_t blk[16];
    for (int b = 0; b < 8; b++) blk[b] = (uint8_t)(nonce >> (8 * b));
    blk[8] = blk[9] = blk[10] = blk[11] = 0;
    for (size_t j = 0; j * 16 < len; j++) {
        uint32_t ctr = (uint32_t)(j + 2);
        blk[12] = (uint8_t)(ctr >> 24);
        blk[13] = (uint8_t)(ctr >> 16);
        blk[14] = (uint8_t)(ctr >> 8);
        blk[15] = (uint8_t)ctr;
        __m128i s = _mm_xor_si128(_mm_loadu_si128((const __m128i*)blk), k[0]);
        for (int r = 1; r < 14; r++) s = _mm_aesenc_si128(s, k[r]);
        s = _mm_aesenclast_si128(s, k[14]);
        size_t take = len - j * 16 < 16 ? len - j * 16 : 16;
        if (take == 16)
            _mm_storeu_si128((__m128i*)(out + j * 16), s);
        else {
            uint8_t t[16];
            _mm_storeu_si128((__m128i*)t, s);
            memcpy(out + j * 16, t, take);
        }
    }
}
#endif

/* prg_algorithm.h:161-172 (1 MiB split) and :214-231 (nonce bytes, GCM). */
uint64_t oro_keystream(const uint32_t rk[60], uint64_t nonce0, uint8_t* out, size_t nbytes) {
    const size_t CH = (size_t)1 << 20;
    uint64_t used = 0;
    for (size_t off = 0; off < nbytes; off += CH, used++) {
        size_t len = nbytes - off < CH ? nbytes - off : CH;
        uint64_t nonce = nonce0 + used;
#ifdef ORO_HAVE_AESNI
        if (__builtin_cpu_supports("aes")) {
            aesni_ctr_chunk(rk, nonce, out + off, len);
            continue;
        }
#endif
        uint8_t blk[16], ks[16];
        for (int b = 0; b < 8; b++) blk[b] = (uint8_t)(nonce >> (8 * b));
        blk[8] = blk[9] = blk[10] = blk[11] = 0;
        for (size_t j = 0; j * 16 < len; j++) {
            uint32_t ctr = (uint32_t)(j + 2);
            blk[12] = (uint8_t)(ctr >> 24);
            blk[13] = (uint8_t)(ctr >> 16);
            blk[14] = (uint8_t)(ctr >> 8);
            blk[15] = (uint8_t)ctr;
            oro_aes256_encrypt(rk, blk, ks);
            size_t take = len - j * 16 < 16 ? len - j * 16 : 16;
            memcpy(out + off + j * 16, ks, take);
        }
    }
    return used;
}

/* ------------------------------------------------------------------------- */
/* Context: which keygen call of which party keys each stream. This follows
 * setup_random_generation (backend/common/rand_setup.h:306-381): call 0 is the
 * local PRG; the lowest member draws each group key in the order of
 * generateRandomnessGroups(3,2,1) = {0,1},{0,2},{1,2},{0,1,2}
 * (core/protocols/protocol.h:309-375); P0 draws a second, discarded
 * everyone-group key (rand_setup.h:321-325, map::insert keeps the first); the
 * last call is the pairwise local key of setup_3pc_common_prgs
 * (rand_setup.h:90-146): party p's get(+1) stream is keyed by its own local
 * key and p+1's get(-1) stream by the same key. */
void oro_ctx_init(oro_ctx* c, uint64_t seed) {
    static const int who[ORO_NSTREAMS][2] = {
        {0, 5}, {1, 2}, {2, 1},         /* PAIR0, PAIR1, PAIR2 */
        {0, 1}, {0, 2}, {1, 1}, {0, 3}, /* G01, G02, G12, G012 */
        {0, 0}, {1, 0}, {2, 0}          /* LOCAL0..2 */
    };
    for (int s = 0; s < ORO_NSTREAMS; s++) {
        uint8_t key[32];
        oro_derive_key(seed, who[s][0], who[s][1], key);
        oro_aes256_expand(key, c->rk[s]);
        c->nonce[s] = 0;
    }
}

/* PRGAlgorithm::getNextBuffered (prg_algorithm.h:86-104): elements are filled
 * in batches of at most 1 MiB; with power-of-two element sizes each batch is
 * exactly one AES-GCM call, so the stream is the plain keystream of n*w bytes. */
void oro_stream_fill(oro_ctx* c, int s, void* out, size_t n, int w) {
    c->nonce[s] += oro_keystream(c->rk[s], c->nonce[s], (uint8_t*)out, n * (size_t)w);
}

/* ------------------------------------------------------------------------- */
/* element helpers */
static inline u128 ld(const void* p, size_t i, int w) {
    u128 v = 0;
    memcpy(&v, (const uint8_t*)p + i * (size_t)w, (size_t)w);
    return v;
}
static inline void st(void* p, size_t i, int w, u128 v) {
    memcpy((uint8_t*)p + i * (size_t)w, &v, (size_t)w);
}
static inline u128 sext(u128 v, int w) { /* sign-extend a w-byte value to 128 bits */
    if (w == 16) return v;
    int sh = 128 - 8 * w;
    return (u128)(((__int128)(v << sh)) >> sh);
}

static void* xalloc(size_t bytes) {
    void* p = calloc(bytes ? bytes : 1, 1);
    if (!p) abort();
    return p;
}

/* ZeroSharingGenerator::getNextBinary/Arithmetic (zero_sharing_generator.h:101-148):
 * party p: prev = get(-1) = PAIR[p-1], next = get(+1) = PAIR[p];
 * r_p = prev ^ next  or  prev - next. Each pairwise stream is drawn once per
 * call (both holders consume it in lock-step). */
void oro_zero_share(oro_ctx* c, int arith, int w, size_t n, void* r[3]) {
    void* k[3];
    for (int q = 0; q < 3; q++) {
        k[q] = xalloc(n * (size_t)w);
        oro_stream_fill(c, ORO_PAIR0 + q, k[q], n, w);
    }
    for (int p = 0; p < 3; p++) {
        void* prev = k[(p + 2) % 3];
        void* next = k[p];
        for (size_t i = 0; i < n; i++) {
            u128 a = ld(prev, i, w), b = ld(next, i, w);
            st(r[p], i, w, arith ? a - b : a ^ b);
        }
    }
    for (int q = 0; q < 3; q++) free(k[q]);
}

/* secret_share_b/a on the data owner (replicated_3pc.h:353-448): share_1 and
 * share_2 from the owner's local PRG, share_3 = data ^ s1 ^ s2 (or data - s1 -
 * s2); owner d holds (share_1, share_2), so S[(d+k)%3] = share_{k+1}. */
void oro_secret_share(oro_ctx* c, int arith, int w, size_t n, const void* data, int d,
                      void* s[3]) {
    void* a = s[d % 3];
    void* b = s[(d + 1) % 3];
    void* e = s[(d + 2) % 3];
    oro_stream_fill(c, ORO_LOCAL0 + d, a, n, w);
    oro_stream_fill(c, ORO_LOCAL0 + d, b, n, w);
    for (size_t i = 0; i < n; i++) {
        u128 x = ld(data, i, w), u = ld(a, i, w), v = ld(b, i, w);
        st(e, i, w, arith ? x - u - v : x ^ u ^ v);
    }
}

/* public_share (replicated_3pc.h:456-470): P0 (x,0), P1 (0,0), P2 (0,x). */
void oro_public_share(int w, size_t n, const void* data, void* s[3]) {
    memcpy(s[0], data, n * (size_t)w);
    memset(s[1], 0, n * (size_t)w);
    memset(s[2], 0, n * (size_t)w);
}

/* open_shares_a/b (replicated_3pc.h:310-330). */
void oro_open(int arith, int w, size_t n, void* const s[3], void* out) {
    for (size_t i = 0; i < n; i++) {
        u128 a = ld(s[0], i, w), b = ld(s[1], i, w), e = ld(s[2], i, w);
        st(out, i, w, arith ? a + b + e : a ^ b ^ e);
    }
}

void oro_xor_b(int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    for (int p = 0; p < 3; p++)
        for (size_t i = 0; i < n; i++) st(z[p], i, w, ld(x[p], i, w) ^ ld(y[p], i, w));
}
void oro_add_a(int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    for (int p = 0; p < 3; p++)
        for (size_t i = 0; i < n; i++) st(z[p], i, w, ld(x[p], i, w) + ld(y[p], i, w));
}
void oro_sub_a(int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    for (int p = 0; p < 3; p++)
        for (size_t i = 0; i < n; i++) st(z[p], i, w, ld(x[p], i, w) - ld(y[p], i, w));
}

/* Replicated_3PC::and_b / multiply_a (replicated_3pc.h:44-67, 166-191):
 * z_p = r_p ^ x_p&y_p ^ x_p&y_{p+1} ^ x_{p+1}&y_p, then the exchange hands
 * z_{p+1} to party p as its second share (exchangeShares(local, remote, 2, 1)). */
static void mult_like(oro_ctx* c, int arith, int w, size_t n, void* const x[3], void* const y[3],
                      void* z[3]) {
    void* r[3];
    void* o[3];
    for (int p = 0; p < 3; p++) {
        r[p] = xalloc(n * (size_t)w);
        o[p] = xalloc(n * (size_t)w);
    }
    oro_zero_share(c, arith, w, n, r);
    for (int p = 0; p < 3; p++) {
        int q = (p + 1) % 3;
        for (size_t i = 0; i < n; i++) {
            u128 xp = ld(x[p], i, w), xq = ld(x[q], i, w);
            u128 yp = ld(y[p], i, w), yq = ld(y[q], i, w);
            u128 v = ld(r[p], i, w);
            if (arith)
                v = v + xp * yp + xp * yq + xq * yp;
            else
                v = v ^ (xp & yp) ^ (xp & yq) ^ (xq & yp);
            st(o[p], i, w, v);
        }
    }
    for (int p = 0; p < 3; p++) {
        memcpy(z[p], o[p], n * (size_t)w);
        free(r[p]);
        free(o[p]);
    }
}
void oro_and_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    mult_like(c, 0, w, n, x, y, z);
}
void oro_mul_a(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    mult_like(c, 1, w, n, x, y, z);
}

/* Replicated_3PC::b2a_bit (replicated_3pc.h:220-251), in the distinct-share
 * view: A = (r0 + ((x0^x1)&1), r1, r2), B = (r'0, r'1 + (x2&1), r'2) from two
 * arithmetic zero-sharings, D = A - B, y = D*D (one multiply_a). */
void oro_b2a_bit(oro_ctx* c, int w, size_t n, void* const x[3], void* y[3]) {
    void* A[3];
    void* B[3];
    for (int p = 0; p < 3; p++) {
        A[p] = xalloc(n * (size_t)w);
        B[p] = xalloc(n * (size_t)w);
    }
    oro_zero_share(c, 1, w, n, A);
    oro_zero_share(c, 1, w, n, B);
    for (size_t i = 0; i < n; i++) {
        u128 a = (ld(x[0], i, w) ^ ld(x[1], i, w)) & 1;
        u128 b = ld(x[2], i, w) & 1;
        st(A[0], i, w, ld(A[0], i, w) + a);
        st(B[1], i, w, ld(B[1], i, w) + b);
    }
    for (int p = 0; p < 3; p++)
        for (size_t i = 0; i < n; i++) st(A[p], i, w, ld(A[p], i, w) - ld(B[p], i, w));
    oro_mul_a(c, w, n, A, A, y);
    for (int p = 0; p < 3; p++) {
        free(A[p]);
        free(B[p]);
    }
}

/* Protocol::reshare (protocol.h:500-541) with groupGetNextBinary/Arithmetic
 * (zero_sharing_generator.h:158-183): r0, r1 from the group stream, r2 =
 * r0^r1 (or -r0-r1); every distinct share j is re-randomised by r_j (each is
 * held by a member of a 2-party group), the non-member receives the result. */
void oro_reshare(oro_ctx* c, int arith, int w, size_t n, int group, void* s[3]) {
    int stream = ORO_G01 + group;
    void* r0 = xalloc(n * (size_t)w);
    void* r1 = xalloc(n * (size_t)w);
    oro_stream_fill(c, stream, r0, n, w);
    oro_stream_fill(c, stream, r1, n, w);
    for (size_t i = 0; i < n; i++) {
        u128 a = ld(r0, i, w), b = ld(r1, i, w);
        u128 e = arith ? (u128)0 - a - b : a ^ b;
        if (arith) {
            st(s[0], i, w, ld(s[0], i, w) + a);
            st(s[1], i, w, ld(s[1], i, w) + b);
            st(s[2], i, w, ld(s[2], i, w) + e);
        } else {
            st(s[0], i, w, ld(s[0], i, w) ^ a);
            st(s[1], i, w, ld(s[1], i, w) ^ b);
            st(s[2], i, w, ld(s[2], i, w) ^ e);
        }
    }
    free(r0);
    free(r1);
}

/* gen_perm (random/permutations/hm_sharded_permutation_generator.h:70-108):
 * draws are u32 from buffers of 2^20 elements (one getNext of 4 MiB each);
 * mask = (1 << bit_width(n)) - 1; reject r > n-1-i; swap(p[i], p[i+r]). */
uint64_t oro_gen_perm(oro_ctx* c, int stream, int32_t* perm, size_t n) {
    const size_t BUF = (size_t)1 << 20;
    uint32_t* rnd = (uint32_t*)xalloc(BUF * 4);
    for (size_t i = 0; i < n; i++) perm[i] = (int32_t)i;
    oro_stream_fill(c, stream, rnd, BUF, 4);
    int bits = 0;
    while (bits < 64 && (n >> bits)) bits++;
    uint32_t mask = (uint32_t)((1ull << bits) - 1);
    size_t ri = 0;
    uint64_t draws = 0;
    for (size_t i = 0; i < n; i++) {
        uint32_t r = (uint32_t)n;
        while ((size_t)r > n - i - 1) {
            r = rnd[ri] & mask;
            ri++;
            draws++;
            if (ri == BUF) {
                oro_stream_fill(c, stream, rnd, BUF, 4);
                ri = 0;
            }
        }
        size_t loc = i + r;
        int32_t t = perm[i];
        perm[i] = perm[loc];
        perm[loc] = t;
    }
    free(rnd);
    return draws;
}

/* ------------------------------------------------------------------------- */
/* permutation plumbing */

/* a sharded permutation: one local permutation per 2-party group */
typedef struct {
    int32_t* g[3];
} sperm;

static void sperm_gen(oro_ctx* c, sperm* sp, size_t n) {
    /* HMShardedPermutationGenerator::generateBatch (hm_...generator.h:178-194):
     * groups in order {0,1},{0,2},{1,2}. */
    for (int g = 0; g < 3; g++) {
        sp->g[g] = (int32_t*)xalloc(n * 4);
        oro_gen_perm(c, ORO_G01 + g, sp->g[g], n);
    }
}
static void sperm_free(sperm* sp) {
    for (int g = 0; g < 3; g++) free(sp->g[g]);
}

/* local_apply_perm (operators/shuffle.h:113-133): new[pi[i]] = x[i] */
static void scatter(int w, size_t n, void* x, const int32_t* pi) {
    uint8_t* t = (uint8_t*)xalloc(n * (size_t)w);
    for (size_t i = 0; i < n; i++) memcpy(t + (size_t)pi[i] * w, (uint8_t*)x + i * w, (size_t)w);
    memcpy(x, t, n * (size_t)w);
    free(t);
}
/* local_apply_inverse_perm (shuffle.h:250-270): new[i] = x[pi[i]] */
static void gather(int w, size_t n, void* x, const int32_t* pi) {
    uint8_t* t = (uint8_t*)xalloc(n * (size_t)w);
    for (size_t i = 0; i < n; i++) memcpy(t + i * w, (uint8_t*)x + (size_t)pi[i] * w, (size_t)w);
    memcpy(x, t, n * (size_t)w);
    free(t);
}

/* hm_oblivious_apply_sharded_perm (shuffle.h:349-368): per group, members
 * permute the shares they hold, then the group reshares. */
static void apply_sharded(oro_ctx* c, int arith, int w, size_t n, void* s[3], const sperm* sp) {
    for (int g = 0; g < 3; g++) {
        for (int j = 0; j < 3; j++) scatter(w, n, s[j], sp->g[g]);
        oro_reshare(c, arith, w, n, g, s);
    }
}
/* hm_oblivious_apply_inverse_sharded_perm (shuffle.h:392-412): groups in
 * reverse order, inverse (gather) application. */
static void apply_inverse_sharded(oro_ctx* c, int arith, int w, size_t n, void* s[3],
                                  const sperm* sp) {
    for (int g = 2; g >= 0; g--) {
        for (int j = 0; j < 3; j++) gather(w, n, s[j], sp->g[g]);
        oro_reshare(c, arith, w, n, g, s);
    }
}

/* PermutationManager queue (random/permutations/permutation_manager.h:102-181,
 * 246-284): reserve() generates ahead; an empty queue generates on demand. */
typedef struct {
    sperm* q;
    size_t head, tail, cap, n;
} pqueue;

static void pq_reserve(oro_ctx* c, pqueue* pq, size_t n, size_t count) {
    if (pq->tail - pq->head >= count) return;
    size_t need = count - (pq->tail - pq->head);
    if (pq->tail + need > pq->cap) {
        pq->cap = pq->tail + need + 8;
        pq->q = (sperm*)realloc(pq->q, pq->cap * sizeof(sperm));
    }
    pq->n = n;
    for (size_t k = 0; k < need; k++) sperm_gen(c, &pq->q[pq->tail++], n);
}
static sperm pq_next(oro_ctx* c, pqueue* pq, size_t n) {
    sperm sp;
    if (pq->tail > pq->head) return pq->q[pq->head++];
    sperm_gen(c, &sp, n);
    return sp;
}

/* oblivious_apply_elementwise_perm (shuffle.h:687-706): shuffle x and a copy
 * of the (A-shared int32) permutation with the same sharded permutation, open
 * the shuffled permutation, scatter x with it. */
static void apply_elementwise(oro_ctx* c, pqueue* pq, int x_arith, int w, size_t n, void* x[3],
                              int32_t* const perm[3]) {
    int32_t* pc[3];
    for (int j = 0; j < 3; j++) {
        pc[j] = (int32_t*)xalloc(n * 4);
        memcpy(pc[j], perm[j], n * 4);
    }
    sperm sp = pq_next(c, pq, n);
    apply_sharded(c, x_arith, w, n, x, &sp);
    apply_sharded(c, 1, 4, n, (void**)pc, &sp);
    int32_t* opened = (int32_t*)xalloc(n * 4);
    oro_open(1, 4, n, (void* const*)pc, opened);
    for (int j = 0; j < 3; j++) scatter(w, n, x[j], opened);
    sperm_free(&sp);
    free(opened);
    for (int j = 0; j < 3; j++) free(pc[j]);
}

/* ------------------------------------------------------------------------- */
/* radix_sort (operators/radixsort.h:116-229) with pad_input/remove_padding
 * (operators/sorting.h:405-495) and ElementwisePermutation::b2a/invert
 * (containers/permutation.h:205-258). */
static void sort_pq(oro_ctx* c, pqueue* pqp, int proto, int kw, size_t n, void* key[3], int bits,
                    int desc, int npayload, int payw, void** payloads, int32_t* perm_out[3]);
#define radix_sort_pq(c, pqp, kw, n, key, bits, desc, np, pl, po) \
    sort_pq(c, pqp, 0, kw, n, key, bits, desc, np, 8, pl, po)

void oro_radix_sort(oro_ctx* c, int kw, size_t n, void* key[3], int bits, int desc,
                    int npayload, void** payloads, int32_t* perm_out[3]) {
    pqueue pq = {0};
    radix_sort_pq(c, &pq, kw, n, key, bits, desc, npayload, payloads, perm_out);
    while (pq.head < pq.tail) sperm_free(&pq.q[pq.head++]);
    free(pq.q);
}

/* quicksort (operators/quicksort.h:214-246): the same padding, permutation
 * extraction and inversion as radix_sort around quicksort_body; payloads are
 * kw-byte A-shared columns permuted with the result. */
void oro_quicksort(oro_ctx* c, int kw, size_t n, void* key[3], int desc, int npayload,
                   void** payloads, int32_t* perm_out[3]) {
    pqueue pq = {0};
    sort_pq(c, &pq, 1, kw, n, key, 0, desc, npayload, kw, payloads, perm_out);
    while (pq.head < pq.tail) sperm_free(&pq.q[pq.head++]);
    free(pq.q);
}

static void compare_pairs(oro_ctx* c, int w, size_t m, u128* const xa[3], u128* const ya[3],
                          u128* eq[3], u128* gt[3]);

/* partition (quicksort.h:28-49): Lomuto partition of rows [start, end] around
 * the row at start, driven by the opened comparisons (0: row <= pivot) */
static void qs_partition(int pw, void* P[3], const uint8_t* cmp, long start, long end, long* piv) {
    long i = start;
    for (long j = start + 1; j <= end; j++)
        if (cmp[j] == 0) {
            i++;
            for (int k = 0; k < 3; k++) {
                u128 a = ld(P[k], (size_t)j, pw), b = ld(P[k], (size_t)i, pw);
                st(P[k], (size_t)j, pw, b);
                st(P[k], (size_t)i, pw, a);
            }
        }
    for (int k = 0; k < 3; k++) {
        u128 a = ld(P[k], (size_t)start, pw), b = ld(P[k], (size_t)i, pw);
        st(P[k], (size_t)start, pw, b);
        st(P[k], (size_t)i, pw, a);
    }
    piv[i] = i;
    if (i + 1 <= end) piv[i + 1] = i + 1;
}

/* quicksort_body (quicksort.h:61-200): shuffle, then rounds of comparing every
 * non-pivot row with the pivot heading its segment (_compare, opened) and
 * partitioning each segment, until every row is a pivot */
static void quicksort_body(oro_ctx* c, pqueue* pq, int pw, size_t n, void* P[3]) {
    sperm sp = pq_next(c, pq, n);
    apply_sharded(c, 0, pw, n, P, &sp);
    sperm_free(&sp);
    if (n == 0) return;
    long* piv = (long*)xalloc(n * sizeof(long));
    uint8_t* cmp = (uint8_t*)xalloc(n);
    for (size_t q = 0; q < n; q++) piv[q] = -1;
    piv[0] = 0;
    size_t num_pivots = 1;
    u128 *R[3], *PV[3], *e[3], *g[3];
    for (int j = 0; j < 3; j++) {
        R[j] = (u128*)xalloc(n * 16 + 16);
        PV[j] = (u128*)xalloc(n * 16 + 16);
        e[j] = (u128*)xalloc(n * 16 + 16);
        g[j] = (u128*)xalloc(n * 16 + 16);
    }
    for (;;) {
        const size_t size = n - num_pivots;
        long head = 0;
        size_t k = 0;
        for (size_t q = 0; q < n; q++) {
            if (piv[q] >= 0) {
                head = piv[q] > head ? piv[q] : head;
                continue;
            }
            for (int j = 0; j < 3; j++) {
                R[j][k] = ld(P[j], q, pw);
                PV[j][k] = ld(P[j], (size_t)head, pw);
            }
            k++;
        }
        /* reduced._compare(pivot): gt = row > pivot */
        compare_pairs(c, pw, size, R, PV, e, g);
        k = 0;
        for (size_t q = 0; q < n; q++)
            if (piv[q] < 0) {
                cmp[q] = (uint8_t)((g[0][k] ^ g[1][k] ^ g[2][k]) & 1);
                k++;
            }
        long index = -1;
        for (long p = 0; p < (long)n; p++) {
            if (piv[p] < 0) continue;
            if (p - index == 1) {
                index++;
                continue;
            }
            qs_partition(pw, P, cmp, index, p - 1, piv);
            index = p;
        }
        qs_partition(pw, P, cmp, index, (long)n - 1, piv);
        num_pivots = 0;
        for (size_t q = 0; q < n; q++) num_pivots += piv[q] >= 0;
        if (num_pivots >= n) break;
    }
    for (int j = 0; j < 3; j++) {
        free(R[j]);
        free(PV[j]);
        free(e[j]);
        free(g[j]);
    }
    free(piv);
    free(cmp);
}

/* radix_sort (proto 0) or quicksort (proto 1) with the caller's
 * PermutationManager queue */
static void sort_pq(oro_ctx* c, pqueue* pqp, int proto, int kw, size_t n, void* key[3], int bits,
                    int desc, int npayload, int payw, void** payloads, int32_t* perm_out[3]) {
#define pq (*pqp)
    const int pw = (kw == 8) ? 16 : 8; /* PadWidth: int64 -> int128, else int64 */
    const int full_width = (kw * 8 == bits);
    void* P[3];
    for (int j = 0; j < 3; j++) P[j] = xalloc(n * (size_t)pw);

    /* pad_input: (v << 32) | idx, idx public-shared into S0 only */
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) {
            u128 v = sext(ld(key[j], i, kw), kw) << 32;
            if (j == 0) v |= (uint32_t)(desc ? (-1 - (int64_t)i) : (int64_t)i);
            st(P[j], i, pw, v);
        }
    if (desc)
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < n / 2; i++) {
                u128 a = ld(P[j], i, pw), b = ld(P[j], n - 1 - i, pw);
                st(P[j], i, pw, b);
                st(P[j], n - 1 - i, pw, a);
            }

    /* radix_sort_body: reserve 1 permutation + (bits + 1) pairs; quicksort:
     * 2 permutations (shuffle, remove_padding) + 1 pair (invert) */
    pq_reserve(c, &pq, n, proto ? 3 : (size_t)bits + 2);
    if (proto) {
        quicksort_body(c, &pq, pw, n, P);
        bits = 0; /* no radix passes */
    }
    int32_t* vp[3];
    int32_t* f1[3];
    int32_t* s[3];
    int32_t* s1v[3];
    int32_t* t[3];
    for (int j = 0; j < 3; j++) {
        vp[j] = (int32_t*)xalloc(n * 4);
        f1[j] = (int32_t*)xalloc(n * 4);
        s[j] = (int32_t*)xalloc(2 * n * 4 + 4);
        s1v[j] = (int32_t*)xalloc(n * 4);
        t[j] = (int32_t*)xalloc(n * 4);
    }
    for (int b = 0; b < bits; b++) {
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < n; i++) {
                u128 v = sext(ld(P[j], i, pw), pw);
                v = (u128)(((__int128)v) >> (32 + b));
                if (full_width && b == bits - 1) v = ~v; /* inplace_invert on every share */
                vp[j][i] = (int32_t)(uint32_t)v;
            }
        oro_b2a_bit(c, 4, n, (void* const*)vp, (void**)f1);
        /* s0 = one - f1 ; s1 = f1 ; s[0] -= 1 ; prefix_sum(s) */
        for (int j = 0; j < 3; j++) {
            for (size_t i = 0; i < n; i++) {
                uint32_t one = (j == 0) ? 1u : 0u;
                s[j][i] = (int32_t)(one - (uint32_t)f1[j][i]);
                s[j][n + i] = f1[j][i];
            }
            if (j == 0 && n) s[j][0] = (int32_t)((uint32_t)s[j][0] - 1u);
            uint32_t acc = 0;
            for (size_t i = 0; i < 2 * n; i++) {
                acc += (uint32_t)s[j][i];
                s[j][i] = (int32_t)acc;
            }
        }
        /* s1 -= s0 ; f1 *= s1 ; s0 += f1 */
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < n; i++)
                s1v[j][i] = (int32_t)((uint32_t)s[j][n + i] - (uint32_t)s[j][i]);
        oro_mul_a(c, 4, n, (void* const*)f1, (void* const*)s1v, (void**)t);
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < n; i++)
                t[j][i] = (int32_t)((uint32_t)s[j][i] + (uint32_t)t[j][i]);
        apply_elementwise(c, &pq, 0, pw, n, P, t);
    }

    if (desc)
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < n / 2; i++) {
                u128 a = ld(P[j], i, pw), b = ld(P[j], n - 1 - i, pw);
                st(P[j], i, pw, b);
                st(P[j], n - 1 - i, pw, a);
            }

    /* remove_padding: perm = low 32 bits (B-shared); key = padded >> 32 */
    int32_t* pm[3];
    for (int j = 0; j < 3; j++) {
        pm[j] = (int32_t*)xalloc(n * 4);
        for (size_t i = 0; i < n; i++) {
            u128 v = sext(ld(P[j], i, pw), pw);
            pm[j][i] = (int32_t)(uint32_t)v;
            st(key[j], i, kw, (u128)(((__int128)v) >> 32));
        }
    }
    /* ElementwisePermutation::b2a (permutation.h:222-258) */
    {
        int32_t* pc[3];
        for (int j = 0; j < 3; j++) {
            pc[j] = (int32_t*)xalloc(n * 4);
            memcpy(pc[j], pm[j], n * 4);
        }
        sperm sp = pq_next(c, &pq, n);
        apply_sharded(c, 0, 4, n, (void**)pc, &sp);
        int32_t* opened = (int32_t*)xalloc(n * 4);
        oro_open(0, 4, n, (void* const*)pc, opened);
        oro_public_share(4, n, opened, (void**)pm);
        apply_inverse_sharded(c, 1, 4, n, (void**)pm, &sp);
        sperm_free(&sp);
        free(opened);
        for (int j = 0; j < 3; j++) free(pc[j]);
    }
    if (desc) {
        /* negate(): v *= -1 (multiply_a with a public -1) ; v += -1 */
        int32_t* m1[3];
        for (int j = 0; j < 3; j++) {
            m1[j] = (int32_t*)xalloc(n * 4);
            for (size_t i = 0; i < n; i++) m1[j][i] = (j == 0) ? -1 : 0;
        }
        oro_mul_a(c, 4, n, (void* const*)pm, (void* const*)m1, (void**)pm);
        oro_add_a(4, n, (void* const*)pm, (void* const*)m1, (void**)pm);
        for (int j = 0; j < 3; j++) free(m1[j]);
    }
    /* invert(): apply the permutation to a public identity */
    {
        int32_t* inv[3];
        for (int j = 0; j < 3; j++) inv[j] = (int32_t*)xalloc(n * 4);
        for (size_t i = 0; i < n; i++) inv[0][i] = (int32_t)i;
        apply_elementwise(c, &pq, 1, 4, n, (void**)inv, pm);
        for (int j = 0; j < 3; j++) {
            memcpy(pm[j], inv[j], n * 4);
            free(inv[j]);
        }
    }
    for (int k = 0; k < npayload; k++) apply_elementwise(c, &pq, 1, payw, n, &payloads[3 * k], pm);
    if (perm_out)
        for (int j = 0; j < 3; j++) memcpy(perm_out[j], pm[j], n * 4);

    for (int j = 0; j < 3; j++) {
        free(P[j]);
        free(vp[j]);
        free(f1[j]);
        free(s[j]);
        free(s1v[j]);
        free(t[j]);
        free(pm[j]);
    }
#undef pq
}

/* shuffle (operators/shuffle.h:752-757): one on-demand sharded permutation
 * (permutation_manager.h:190-209 with an empty queue) applied with resharing. */
void oro_shuffle(oro_ctx* c, int arith, int w, size_t n, void* s[3]) {
    sperm sp;
    sperm_gen(c, &sp, n);
    apply_sharded(c, arith, w, n, s, &sp);
    sperm_free(&sp);
}

/* SharedVector::prefix_sum (containers/shared_vector.h:249): inclusive scan
 * of each share array, mod 2^(8w). */
void oro_prefix_sum(int w, size_t n, void* s[3]) {
    for (int j = 0; j < 3; j++) {
        u128 acc = 0;
        for (size_t i = 0; i < n; i++) {
            acc += ld(s[j], i, w);
            st(s[j], i, w, acc);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Compare circuit and bitonic sort on B-shared int32/int64 keys. */

/* arithmetic right shift of a w-byte two's-complement value */
static u128 ashr(u128 v, int w, int s) {
    return (u128)(((__int128)sext(v, w)) >> s);
}
static u128 wmask(int w) { return w == 16 ? ~(u128)0 : (((u128)1 << (8 * w)) - 1); }

/* BSharedVector::_compare (operators/circuits.h:231-295) with bit_same
 * (containers/b_shared_vector.h:164-178), for m pairs of w-byte keys; xa[j][p]
 * plays `this`. eq and gt come out masked to their LSB (one call sequence:
 * log2(8w) ANDs, gt &= this, and the packed OR on ceil(m/8w) words). */
static void compare_pairs(oro_ctx* c, int w, size_t m, u128* const xa[3], u128* const ya[3],
                          u128* eq[3], u128* gt[3]) {
    const int B = 8 * w;
    int L = 0;
    while ((1 << L) < B) L++; /* bit_width(B - 1) */
    const u128 M = wmask(w);
    void* S[3];
    void* Tm[3];
    for (int j = 0; j < 3; j++) {
        S[j] = xalloc(m * (size_t)w);
        Tm[j] = xalloc(m * (size_t)w);
        for (size_t p = 0; p < m; p++) st(S[j], p, w, ~(xa[j][p] ^ ya[j][p]) & M);
    }
    for (int lev = 0; lev < L; lev++) {
        for (int j = 0; j < 3; j++)
            for (size_t p = 0; p < m; p++) st(Tm[j], p, w, ashr(ld(S[j], p, w), w, 1 << lev) & M);
        oro_and_b(c, w, m, S, Tm, S);
    }
    /* gt = ((eq >> 1) ^ eq) & this, then parity of every share */
    void* G[3];
    void* X[3];
    for (int j = 0; j < 3; j++) {
        G[j] = xalloc(m * (size_t)w);
        X[j] = xalloc(m * (size_t)w);
        for (size_t p = 0; p < m; p++) {
            u128 e = ld(S[j], p, w);
            st(G[j], p, w, (ashr(e, w, 1) ^ e) & M);
            st(X[j], p, w, xa[j][p]);
        }
    }
    oro_and_b(c, w, m, G, X, G);
    /* sign fix-up on packed bits */
    const size_t cw = m / B + (m % B > 0);
    void* s1[3];
    void* s2[3];
    void* r[3];
    for (int j = 0; j < 3; j++) {
        s1[j] = xalloc(cw * (size_t)w);
        s2[j] = xalloc(cw * (size_t)w);
        r[j] = xalloc(cw * (size_t)w);
        for (size_t word = 0; word < cw; word++) {
            u128 a = 0, b = 0, e = 0;
            for (int k = 0; k < B && word * B + k < m; k++) {
                size_t p = word * B + k;
                u128 gv = ld(G[j], p, w);
                int par = 0;
                for (int bit = 0; bit < B; bit++) par ^= (int)((gv >> bit) & 1);
                a |= ((xa[j][p] >> (B - 1)) & 1) << k;
                b |= ((ya[j][p] >> (B - 1)) & 1) << k;
                e |= (u128)par << k;
            }
            /* r ^= s2 ; s2 ^= s1 ; then s2 |= r as ~(~s2 & ~r) */
            e ^= b;
            b ^= a;
            st(s1[j], word, w, a);
            st(s2[j], word, w, ~b & M);
            st(r[j], word, w, ~e & M);
        }
    }
    oro_and_b(c, w, cw, s2, r, s2);
    for (int j = 0; j < 3; j++) {
        for (size_t word = 0; word < cw; word++) {
            u128 o = ~ld(s2[j], word, w) & M;
            st(s1[j], word, w, ld(s1[j], word, w) ^ o);
        }
        for (size_t p = 0; p < m; p++) {
            eq[j][p] = ld(S[j], p, w) & 1;
            gt[j][p] = (ld(s1[j], p / B, w) >> (p % B)) & 1;
        }
        free(S[j]);
        free(Tm[j]);
        free(G[j]);
        free(X[j]);
        free(s1[j]);
        free(s2[j]);
        free(r[j]);
    }
}

void oro_compare(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* eq[3],
                 void* gt[3]) {
    u128* xa[3];
    u128* ya[3];
    u128* e[3];
    u128* g[3];
    for (int j = 0; j < 3; j++) {
        xa[j] = (u128*)xalloc(n * 16);
        ya[j] = (u128*)xalloc(n * 16);
        e[j] = (u128*)xalloc(n * 16);
        g[j] = (u128*)xalloc(n * 16);
        for (size_t p = 0; p < n; p++) {
            xa[j][p] = ld(x[j], p, w);
            ya[j][p] = ld(y[j], p, w);
        }
    }
    compare_pairs(c, w, n, xa, ya, e, g);
    for (int j = 0; j < 3; j++) {
        for (size_t p = 0; p < n; p++) {
            st(eq[j], p, w, e[j][p]);
            st(gt[j], p, w, g[j][p]);
        }
        free(xa[j]);
        free(ya[j]);
        free(e[j]);
        free(g[j]);
    }
}

/* bitonic_sort (operators/sorting.h:266-353,394-399) of one B-shared key
 * column: stage (i, j) with h = 2^(i-j) compares x[c*h+k] = c*2h+k with
 * y = c*2h+2h-1-k (j == 0, the reversed subset) or c*2h+h+k, then swaps with
 * two multiplexes (operators/common.h:20-28). */
void oro_bitonic_sort(oro_ctx* c, int w, size_t n, void* key[3], int desc) {
    if (n < 2) return;
    int rounds = 0;
    while (((size_t)1 << rounds) < n) rounds++;
    const size_t m = n / 2;
    const u128 M = wmask(w);
    u128* xa[3];
    u128* ya[3];
    u128* e[3];
    u128* g[3];
    size_t* xi = (size_t*)xalloc(m * sizeof(size_t));
    size_t* yi = (size_t*)xalloc(m * sizeof(size_t));
    for (int j = 0; j < 3; j++) {
        xa[j] = (u128*)xalloc(m * 16);
        ya[j] = (u128*)xalloc(m * 16);
        e[j] = (u128*)xalloc(m * 16);
        g[j] = (u128*)xalloc(m * 16);
    }
    void* E[3];
    void* D[3];
    void* Z[3];
    for (int j = 0; j < 3; j++) {
        E[j] = xalloc(m * (size_t)w);
        D[j] = xalloc(m * (size_t)w);
        Z[j] = xalloc(m * (size_t)w);
    }
    for (int i = 0; i < rounds; i++) {
        for (int jj = 0; jj <= i; jj++) {
            const size_t h = (size_t)1 << (i - jj);
            for (size_t p = 0; p < m; p++) {
                size_t cb = p / h, k = p % h;
                xi[p] = cb * 2 * h + k;
                yi[p] = jj == 0 ? cb * 2 * h + 2 * h - 1 - k : cb * 2 * h + h + k;
            }
            for (int j = 0; j < 3; j++)
                for (size_t p = 0; p < m; p++) {
                    xa[j][p] = ld(key[j], xi[p], w);
                    ya[j][p] = ld(key[j], yi[p], w);
                }
            /* ASC: x > y ; DESC: y > x (compare_rows, sorting.h:80-108) */
            if (desc)
                compare_pairs(c, w, m, ya, xa, e, g);
            else
                compare_pairs(c, w, m, xa, ya, e, g);
            /* tmp = multiplex(b, x, y) = x ^ (ext(b) & (y ^ x)) ; y' = y ^ (ext(b) & (x ^ y)) */
            for (int j = 0; j < 3; j++)
                for (size_t p = 0; p < m; p++) {
                    st(E[j], p, w, (g[j][p] & 1) ? M : 0);
                    st(D[j], p, w, (xa[j][p] ^ ya[j][p]) & M);
                }
            oro_and_b(c, w, m, E, D, Z);
            for (int j = 0; j < 3; j++)
                for (size_t p = 0; p < m; p++) st(key[j], xi[p], w, xa[j][p] ^ ld(Z[j], p, w));
            oro_and_b(c, w, m, E, D, Z);
            for (int j = 0; j < 3; j++)
                for (size_t p = 0; p < m; p++) st(key[j], yi[p], w, ya[j][p] ^ ld(Z[j], p, w));
        }
    }
    for (int j = 0; j < 3; j++) {
        free(xa[j]);
        free(ya[j]);
        free(e[j]);
        free(g[j]);
        free(E[j]);
        free(D[j]);
        free(Z[j]);
    }
    free(xi);
    free(yi);
}

/* ------------------------------------------------------------------------- */
/* Aggregation network (operators/aggregation.h:27-140,167-346). */

static void** sl3(void* const s[3], size_t off, int w, void* out[3]) {
    for (int j = 0; j < 3; j++) out[j] = (uint8_t*)s[j] + off * (size_t)w;
    return out;
}
static void alloc3(void* v[3], size_t n, int w) {
    for (int j = 0; j < 3; j++) v[j] = xalloc(n * (size_t)w + 16);
}
static void free3(void* v[3]) {
    for (int j = 0; j < 3; j++) free(v[j]);
}
static void copy3(void* dst[3], void* const src[3], size_t n, int w) {
    for (int j = 0; j < 3; j++) memmove(dst[j], src[j], n * (size_t)w);
}
/* public constant 1 repeated (public_share: S0 = 1, S1 = S2 = 0) */
static void one3(void* v[3], size_t n, int w) {
    for (size_t i = 0; i < n; i++) {
        st(v[0], i, w, 1);
        st(v[1], i, w, 0);
        st(v[2], i, w, 0);
    }
}
/* extend_lsb: every share becomes -(s & 1) */
static void ext3(void* dst[3], void* const src[3], size_t n, int w) {
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) st(dst[j], i, w, (ld(src[j], i, w) & 1) ? ~(u128)0 : 0);
}
static void not3(void* v[3], size_t n, int w) {
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) st(v[j], i, w, ~ld(v[j], i, w));
}
static void mask3(void* v[3], size_t n, int w, u128 m) {
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) st(v[j], i, w, ld(v[j], i, w) & m);
}
/* operator== : bit_same then mask(1) (b_shared_vector.h:164-178,493-504) */
static void eq3(oro_ctx* c, int w, size_t m, void* const x[3], void* const y[3], void* out[3]) {
    const int B = 8 * w;
    int L = 0;
    while ((1 << L) < B) L++;
    const u128 M = wmask(w);
    void* T[3];
    alloc3(T, m, w);
    for (int j = 0; j < 3; j++)
        for (size_t p = 0; p < m; p++) st(out[j], p, w, ~(ld(x[j], p, w) ^ ld(y[j], p, w)) & M);
    for (int lev = 0; lev < L; lev++) {
        for (int j = 0; j < 3; j++)
            for (size_t p = 0; p < m; p++) st(T[j], p, w, ashr(ld(out[j], p, w), w, 1 << lev) & M);
        oro_and_b(c, w, m, out, T, out);
    }
    mask3(out, m, w, 1);
    free3(T);
}
/* multiplex(sel, a, b) = a ^ (ext(sel) & (b ^ a)) (operators/common.h:20-28) */
static void mux_b(oro_ctx* c, int w, size_t m, void* const sel[3], void* const a[3],
                  void* const b[3], void* res[3]) {
    void* E[3];
    void* D[3];
    alloc3(E, m, w);
    alloc3(D, m, w);
    ext3(E, sel, m, w);
    oro_xor_b(w, m, b, a, D);
    oro_and_b(c, w, m, E, D, D);
    oro_xor_b(w, m, a, D, res);
    free3(E);
    free3(D);
}

/* func(g, a, b) for the boolean aggregations; writes the new a to res */
static void agg_b(oro_ctx* c, int func, int w, size_t m, void* const g[3], void* const a[3],
                  void* const b[3], void* res[3]) {
    void* t[3];
    alloc3(t, m, w);
    switch (func) {
        case ORO_AGG_COPY:
            mux_b(c, w, m, g, a, b, res);
            break;
        case ORO_AGG_VALID: /* agg = a & b ; a = multiplex(g, a, agg) */
            oro_and_b(c, w, m, a, b, t);
            mux_b(c, w, m, g, a, t, res);
            break;
        case ORO_AGG_BIT_OR: { /* a | (ext(g) & b), | = ~(~a & ~x) */
            void* na[3];
            alloc3(na, m, w);
            ext3(t, g, m, w);
            oro_and_b(c, w, m, t, b, t);
            copy3(na, a, m, w);
            not3(na, m, w);
            not3(t, m, w);
            oro_and_b(c, w, m, na, t, res);
            not3(res, m, w);
            free3(na);
            break;
        }
        case ORO_AGG_MAX:
        case ORO_AGG_MIN: { /* bg = b > a (! for min); a = mux(g, a, mux(bg, a, b)) */
            void* eq[3];
            void* gt[3];
            alloc3(eq, m, w);
            alloc3(gt, m, w);
            oro_compare(c, w, m, b, a, eq, gt);
            if (func == ORO_AGG_MIN)
                for (int j = 0; j < 3; j++)
                    for (size_t i = 0; i < m; i++) st(gt[j], i, w, (ld(gt[j], i, w) & 1) ^ 1);
            mux_b(c, w, m, gt, a, b, t);
            mux_b(c, w, m, g, a, t, res);
            free3(eq);
            free3(gt);
            break;
        }
        default:
            fprintf(stderr, "oro_aggregate: bad boolean aggregation %d\n", func);
            abort();
    }
    free3(t);
}

/* func(g, a, b) for the arithmetic aggregations: sum/count a + g*b, copy
 * a + g*(b - a) */
static void agg_a(oro_ctx* c, int func, int w, size_t m, void* const g[3], void* const a[3],
                  void* const b[3], void* res[3]) {
    void* t[3];
    alloc3(t, m, w);
    if (func == ORO_AGG_COPY) {
        oro_sub_a(w, m, b, a, t);
        oro_mul_a(c, w, m, g, t, t);
    } else {
        oro_mul_a(c, w, m, g, b, t);
    }
    oro_add_a(w, m, a, t, res);
    free3(t);
}

void oro_aggregate(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys, int nb,
                   void* const* b_in, void* const* b_out, const int* b_func, int na,
                   void* const* a_in, void* const* a_out, const int* a_func, int reverse,
                   void* const* sel) {
    int a_copy = 0, a_noncopy = 0, b_copy = 0, b_noncopy = 0;
    (void)b_copy;
    for (int s = 0; s < na; s++) {
        void* out[3] = {a_out[3 * s], a_out[3 * s + 1], a_out[3 * s + 2]};
        if (a_func[s] == ORO_AGG_COUNT) {
            if (sel) oro_b2a_bit(c, w, n, sel, out);
            else one3(out, n, w);
        } else {
            void* in[3] = {a_in[3 * s], a_in[3 * s + 1], a_in[3 * s + 2]};
            copy3(out, in, n, w);
        }
        if (a_func[s] == ORO_AGG_COPY) a_copy = 1;
        else a_noncopy = 1;
    }
    for (int s = 0; s < nb; s++) {
        void* out[3] = {b_out[3 * s], b_out[3 * s + 1], b_out[3 * s + 2]};
        void* in[3] = {b_in[3 * s], b_in[3 * s + 1], b_in[3 * s + 2]};
        copy3(out, in, n, w);
        if (b_func[s] == ORO_AGG_COPY) b_copy = 1;
        else b_noncopy = 1;
    }
    int log_size = 0;
    while (((size_t)2 << log_size) <= n) log_size++;
    for (int i = 1; i <= log_size; i++) {
        size_t d = n >> i;
        if (reverse) d = n >> (log_size - i + 1);
        const size_t dr = n - d;
        void *G[3], *JG[3], *GA[3], *JGA[3], *X[3], *Y[3], *R[3], *E[3];
        alloc3(G, dr, w);
        alloc3(JG, dr, w);
        alloc3(GA, dr, w);
        alloc3(JGA, dr, w);
        alloc3(X, dr, w);
        alloc3(Y, dr, w);
        alloc3(R, dr, w);
        alloc3(E, dr, w);
        if (nkeys == 0) {
            one3(G, dr, w);
            one3(GA, dr, w);
        } else {
            for (int k = 0; k < nkeys; k++) {
                void* kk[3] = {keys[3 * k], keys[3 * k + 1], keys[3 * k + 2]};
                void *lo[3], *hi[3];
                sl3(kk, 0, w, lo);
                sl3(kk, d, w, hi);
                if (k == 0) {
                    eq3(c, w, dr, lo, hi, G);
                } else {
                    eq3(c, w, dr, lo, hi, E);
                    oro_and_b(c, w, dr, G, E, G);
                }
            }
            for (int j = 0; j < 3; j++) memset(GA[j], 0, dr * (size_t)w);
        }
        copy3(JG, G, dr, w);
        copy3(JGA, GA, dr, w);
        if (sel && (a_noncopy || b_noncopy)) {
            void *lo[3], *hi[3];
            sl3(sel, 0, w, lo);
            sl3(sel, d, w, hi);
            oro_xor_b(w, dr, hi, lo, E);
            not3(E, dr, w);
            oro_and_b(c, w, dr, G, E, G);
        }
        mask3(G, dr, w, 1);
        for (int s = 0; s < nb; s++) {
            void* out[3] = {b_out[3 * s], b_out[3 * s + 1], b_out[3 * s + 2]};
            void *lo[3], *hi[3];
            sl3(out, 0, w, lo);
            sl3(out, d, w, hi);
            copy3(X, lo, dr, w);
            copy3(Y, hi, dr, w);
            void** g = b_func[s] == ORO_AGG_COPY ? JG : G;
            if (reverse) {
                agg_b(c, b_func[s], w, dr, g, Y, X, R);
                copy3(hi, R, dr, w);
            } else {
                agg_b(c, b_func[s], w, dr, g, X, Y, R);
                copy3(lo, R, dr, w);
            }
        }
        if (nkeys > 0 && na > 0) {
            if (a_noncopy) oro_b2a_bit(c, w, dr, G, GA);
            if (a_copy) oro_b2a_bit(c, w, dr, JG, JGA);
        }
        for (int s = 0; s < na; s++) {
            void* out[3] = {a_out[3 * s], a_out[3 * s + 1], a_out[3 * s + 2]};
            void *lo[3], *hi[3];
            sl3(out, 0, w, lo);
            sl3(out, d, w, hi);
            copy3(X, lo, dr, w);
            copy3(Y, hi, dr, w);
            void** g = a_func[s] == ORO_AGG_COPY ? JGA : GA;
            if (reverse) {
                agg_a(c, a_func[s], w, dr, g, Y, X, R);
                copy3(hi, R, dr, w);
            } else {
                agg_a(c, a_func[s], w, dr, g, X, Y, R);
                copy3(lo, R, dr, w);
            }
        }
        free3(G);
        free3(JG);
        free3(GA);
        free3(JGA);
        free3(X);
        free3(Y);
        free3(R);
        free3(E);
    }
}


/* ------------------------------------------------------------------------- */
/* Permutation composition, table sort and distinct. */

/* compose_permutations (operators/shuffle.h:717-743): pi from the queue;
 * sigma' = pi(sigma) (sharded apply, sigma modified), opened; rho gathered
 * by it (local_apply_inverse_perm), then pi undone on rho. Result in rho. */
static void compose_pq(oro_ctx* c, pqueue* pq, size_t n, int32_t* sigma[3], int32_t* rho[3]) {
    sperm sp = pq_next(c, pq, n);
    apply_sharded(c, 1, 4, n, (void**)sigma, &sp);
    int32_t* opened = (int32_t*)xalloc(n * 4 + 4);
    oro_open(1, 4, n, (void* const*)sigma, opened);
    for (int j = 0; j < 3; j++) gather(4, n, rho[j], opened);
    apply_inverse_sharded(c, 1, 4, n, (void**)rho, &sp);
    sperm_free(&sp);
    free(opened);
}

void oro_compose_permutations(oro_ctx* c, size_t n, int32_t* sigma[3], int32_t* rho[3]) {
    pqueue pq = {0};
    compose_pq(c, &pq, n, sigma, rho);
    free(pq.q);
}

/* table_sort (operators/sorting.h:509-612) with SortingProtocol::RADIXSORT:
 * reserve every permutation up front, sort the last key column, then each
 * earlier column after applying the running permutation to it, composing the
 * permutations; finally apply the total permutation to the key columns, the
 * arithmetic data columns and the boolean data columns, in that order. */
/* sort_sub (sorting.h:565-576): single-bit columns by a 1-bit radix sort,
 * the rest by quicksort (quick) or a full-width radix sort */
static void table_sort_sub(oro_ctx* c, pqueue* pq, int quick, int w, size_t n, void* col[3], int single,
                           int desc, int32_t* perm[3]) {
    if (single || !quick) radix_sort_pq(c, pq, w, n, col, single ? 1 : 8 * w, desc, 0, NULL, perm);
    else sort_pq(c, pq, 1, w, n, col, 0, desc, 0, w, NULL, perm);
}

void oro_table_sort(oro_ctx* c, int w, size_t n, int ncols, void* const* cols, const int* desc,
                    const int* single_bit, int na, void* const* data_a, int nb,
                    void* const* data_b, int quick) {
    int ns = 0;
    for (int k = 0; k < ncols; k++) ns += single_bit[k] != 0;
    const int nk = ncols - ns, nc = na + nb, L = 8 * w;
    const size_t perms = (size_t)(nk + ns - 1) + (size_t)(nk + ns) + (quick ? (size_t)nk : 0);
    const size_t pairs = (size_t)(4 * ns + 3 * nk + nc - 1) + (quick ? 0 : (size_t)nk * L);
    pqueue pq = {0};
    pq_reserve(c, &pq, n, perms + pairs);
    void* orig[3];
    alloc3(orig, n, w);
    int32_t* sp[3];
    int32_t* np_[3];
    for (int j = 0; j < 3; j++) {
        sp[j] = (int32_t*)xalloc(n * 4 + 4);
        np_[j] = (int32_t*)xalloc(n * 4 + 4);
    }
    int C = ncols - 1;
    {
        void* col[3] = {cols[3 * C], cols[3 * C + 1], cols[3 * C + 2]};
        copy3(orig, col, n, w);
        table_sort_sub(c, &pq, quick, w, n, col, single_bit[C], desc[C], sp);
        copy3(col, orig, n, w);
    }
    for (C--; C >= 0; C--) {
        void* col[3] = {cols[3 * C], cols[3 * C + 1], cols[3 * C + 2]};
        copy3(orig, col, n, w);
        apply_elementwise(c, &pq, 0, w, n, col, sp);
        table_sort_sub(c, &pq, quick, w, n, col, single_bit[C], desc[C], np_);
        copy3(col, orig, n, w);
        compose_pq(c, &pq, n, sp, np_);
        for (int j = 0; j < 3; j++) {
            int32_t* t = sp[j];
            sp[j] = np_[j];
            np_[j] = t;
        }
    }
    for (int k = 0; k < ncols; k++) {
        void* col[3] = {cols[3 * k], cols[3 * k + 1], cols[3 * k + 2]};
        apply_elementwise(c, &pq, 0, w, n, col, sp);
    }
    for (int k = 0; k < na; k++) {
        void* col[3] = {data_a[3 * k], data_a[3 * k + 1], data_a[3 * k + 2]};
        apply_elementwise(c, &pq, 1, w, n, col, sp);
    }
    for (int k = 0; k < nb; k++) {
        void* col[3] = {data_b[3 * k], data_b[3 * k + 1], data_b[3 * k + 2]};
        apply_elementwise(c, &pq, 0, w, n, col, sp);
    }
    free3(orig);
    for (int j = 0; j < 3; j++) {
        free(sp[j]);
        free(np_[j]);
    }
    while (pq.head < pq.tail) sperm_free(&pq.q[pq.head++]);
    free(pq.q);
}

/* distinct (operators/distinct.h:20-53): res = 0; res[0] = public 1; for
 * every key, res[1:] |= (key[:-1] != key[1:]) where != is !(bit_same & 1)
 * and |= is ~(~res & ~x) (b_shared_vector.h:450-455). */
void oro_distinct(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys, void* res[3]) {
    for (int j = 0; j < 3; j++) memset(res[j], 0, n * (size_t)w);
    if (n == 0) return;
    st(res[0], 0, w, 1);
    const size_t m = n - 1;
    void *E[3], *R[3];
    alloc3(E, m, w);
    sl3(res, 1, w, R);
    for (int k = 0; k < nkeys; k++) {
        void* kk[3] = {keys[3 * k], keys[3 * k + 1], keys[3 * k + 2]};
        void *lo[3], *hi[3];
        sl3(kk, 0, w, lo);
        sl3(kk, 1, w, hi);
        eq3(c, w, m, lo, hi, E);
        for (int j = 0; j < 3; j++)
            for (size_t i = 0; i < m; i++) st(E[j], i, w, (ld(E[j], i, w) & 1) ^ 1);
        not3(R, m, w);
        not3(E, m, w);
        oro_and_b(c, w, m, R, E, R);
        not3(R, m, w);
    }
    free3(E);
}

/* BSharedVector::operator== (b_shared_vector.h:493-504): bit_same, mask(1). */
void oro_equal(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* eq[3]) {
    eq3(c, w, n, x, y, eq);
}

/* not_b_1 (replicated_3pc.h:207): every share becomes !(s & 1). */
void oro_not_b1(int w, size_t n, void* const x[3], void* y[3]) {
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) st(y[j], i, w, (ld(x[j], i, w) & 1) ^ 1);
}

/* ------------------------------------------------------------------------- */
/* compare_rows, swap and multi-column bitonic sort (operators/sorting.h:80-353,
 * operators/common.h:20-49). */

/* BSharedVector::extend_lsb (b_shared_vector.h:145-147) */
void oro_extend_lsb(int w, size_t n, void* const x[3], void* y[3]) { ext3(y, x, n, w); }

/* multiplex(sel, a, b) = a + sel * (b - a) on A-shared columns (common.h:43-49) */
static void mux_a(oro_ctx* c, int w, size_t m, void* const sel[3], void* const a[3],
                  void* const b[3], void* res[3]) {
    void* t[3];
    alloc3(t, m, w);
    oro_sub_a(w, m, b, a, t);
    oro_mul_a(c, w, m, sel, t, t);
    oro_add_a(w, m, a, t, res);
    free3(t);
}

/* compare_rows (sorting.h:80-108) of m row pairs over nkeys key columns given
 * as widened arrays xa[3k+j], ya[3k+j]: gt of key 0, then per further key
 * gt ^= new_gt & eq and eq &= new_eq; gt comes out masked to its LSB. */
static void compare_rows_u(oro_ctx* c, int w, size_t m, int nkeys, u128* const* xa,
                           u128* const* ya, const int* desc, void* gt[3]) {
    u128 *e[3], *g[3];
    void *EQ[3], *NE[3], *NG[3];
    for (int j = 0; j < 3; j++) {
        e[j] = (u128*)xalloc(m * 16 + 16);
        g[j] = (u128*)xalloc(m * 16 + 16);
    }
    alloc3(EQ, m, w);
    alloc3(NE, m, w);
    alloc3(NG, m, w);
    for (int k = 0; k < nkeys; k++) {
        u128* const* t = desc[k] ? ya + 3 * k : xa + 3 * k;
        u128* const* o = desc[k] ? xa + 3 * k : ya + 3 * k;
        compare_pairs(c, w, m, t, o, e, g);
        void** G = k ? NG : gt;
        void** Q = k ? NE : EQ;
        for (int j = 0; j < 3; j++)
            for (size_t p = 0; p < m; p++) {
                st(G[j], p, w, g[j][p]);
                st(Q[j], p, w, e[j][p]);
            }
        if (k) {
            oro_and_b(c, w, m, NG, EQ, NG);
            oro_xor_b(w, m, gt, NG, gt);
            oro_and_b(c, w, m, EQ, NE, EQ);
        }
    }
    mask3(gt, m, w, 1);
    for (int j = 0; j < 3; j++) {
        free(e[j]);
        free(g[j]);
    }
    free3(EQ);
    free3(NE);
    free3(NG);
}

void oro_compare_rows(oro_ctx* c, int w, size_t n, int nkeys, void* const* x, void* const* y,
                      const int* desc, void* gt[3]) {
    u128** xa = (u128**)xalloc(sizeof(u128*) * 3 * (size_t)nkeys);
    u128** ya = (u128**)xalloc(sizeof(u128*) * 3 * (size_t)nkeys);
    for (int k = 0; k < 3 * nkeys; k++) {
        xa[k] = (u128*)xalloc(n * 16 + 16);
        ya[k] = (u128*)xalloc(n * 16 + 16);
        for (size_t p = 0; p < n; p++) {
            xa[k][p] = ld(x[k], p, w);
            ya[k][p] = ld(y[k], p, w);
        }
    }
    compare_rows_u(c, w, n, nkeys, xa, ya, desc, gt);
    for (int k = 0; k < 3 * nkeys; k++) {
        free(xa[k]);
        free(ya[k]);
    }
    free(xa);
    free(ya);
}

/* swap (sorting.h:146-212): per column tmp = multiplex(bits, x, y),
 * y = multiplex(bits, y, x), x = tmp; boolean or arithmetic multiplex. */
static void swap_cols(oro_ctx* c, int arith, int w, size_t m, int ncols, void* const* x,
                      void* const* y, void* const bits[3]) {
    void* tmp[3];
    alloc3(tmp, m, w);
    for (int k = 0; k < ncols; k++) {
        void* X[3] = {x[3 * k], x[3 * k + 1], x[3 * k + 2]};
        void* Y[3] = {y[3 * k], y[3 * k + 1], y[3 * k + 2]};
        if (arith) {
            mux_a(c, w, m, bits, X, Y, tmp);
            mux_a(c, w, m, bits, Y, X, Y);
        } else {
            mux_b(c, w, m, bits, X, Y, tmp);
            mux_b(c, w, m, bits, Y, X, Y);
        }
        copy3(X, tmp, m, w);
    }
    free3(tmp);
}

void oro_swap(oro_ctx* c, int arith, int w, size_t n, int ncols, void* const* x, void* const* y,
              void* const bits[3]) {
    swap_cols(c, arith, w, n, ncols, x, y, bits);
}

/* bitonic_sort (sorting.h:266-353) over nkeys key columns with na A-shared and
 * nb B-shared data columns: per stage compare_rows on the pair rows of every
 * key, swap of the keys, swap of the B data with the same bits, and (when there
 * is A data) b2a_bit of the bits and an arithmetic swap of the A data. */
void oro_bitonic_sort_rows(oro_ctx* c, int w, size_t n, int nkeys, void* const* keys,
                           const int* desc, int na, void* const* data_a, int nb,
                           void* const* data_b) {
    if (n < 2) return;
    int rounds = 0;
    while (((size_t)1 << rounds) < n) rounds++;
    const size_t m = n / 2;
    const int ncol = nkeys + nb + na;
    void** cols = (void**)xalloc(sizeof(void*) * 3 * (size_t)ncol);
    for (int k = 0; k < 3 * nkeys; k++) cols[k] = keys[k];
    for (int k = 0; k < 3 * nb; k++) cols[3 * nkeys + k] = data_b[k];
    for (int k = 0; k < 3 * na; k++) cols[3 * (nkeys + nb) + k] = data_a[k];
    void** X = (void**)xalloc(sizeof(void*) * 3 * (size_t)ncol);
    void** Y = (void**)xalloc(sizeof(void*) * 3 * (size_t)ncol);
    u128** xa = (u128**)xalloc(sizeof(u128*) * 3 * (size_t)nkeys);
    u128** ya = (u128**)xalloc(sizeof(u128*) * 3 * (size_t)nkeys);
    for (int k = 0; k < 3 * ncol; k++) {
        X[k] = xalloc(m * (size_t)w + 16);
        Y[k] = xalloc(m * (size_t)w + 16);
    }
    for (int k = 0; k < 3 * nkeys; k++) {
        xa[k] = (u128*)xalloc(m * 16 + 16);
        ya[k] = (u128*)xalloc(m * 16 + 16);
    }
    size_t* xi = (size_t*)xalloc(m * sizeof(size_t));
    size_t* yi = (size_t*)xalloc(m * sizeof(size_t));
    void *bits[3], *bits_a[3];
    alloc3(bits, m, w);
    alloc3(bits_a, m, w);
    for (int i = 0; i < rounds; i++) {
        for (int jj = 0; jj <= i; jj++) {
            const size_t h = (size_t)1 << (i - jj);
            for (size_t p = 0; p < m; p++) {
                size_t cb = p / h, k = p % h;
                xi[p] = cb * 2 * h + k;
                yi[p] = jj == 0 ? cb * 2 * h + 2 * h - 1 - k : cb * 2 * h + h + k;
            }
            for (int k = 0; k < 3 * ncol; k++)
                for (size_t p = 0; p < m; p++) {
                    st(X[k], p, w, ld(cols[k], xi[p], w));
                    st(Y[k], p, w, ld(cols[k], yi[p], w));
                }
            for (int k = 0; k < 3 * nkeys; k++)
                for (size_t p = 0; p < m; p++) {
                    xa[k][p] = ld(X[k], p, w);
                    ya[k][p] = ld(Y[k], p, w);
                }
            compare_rows_u(c, w, m, nkeys, xa, ya, desc, bits);
            swap_cols(c, 0, w, m, nkeys + nb, X, Y, bits);
            if (na) {
                oro_b2a_bit(c, w, m, bits, bits_a);
                swap_cols(c, 1, w, m, na, X + 3 * (nkeys + nb), Y + 3 * (nkeys + nb), bits_a);
            }
            for (int k = 0; k < 3 * ncol; k++)
                for (size_t p = 0; p < m; p++) {
                    st(cols[k], xi[p], w, ld(X[k], p, w));
                    st(cols[k], yi[p], w, ld(Y[k], p, w));
                }
        }
    }
    for (int k = 0; k < 3 * ncol; k++) {
        free(X[k]);
        free(Y[k]);
    }
    for (int k = 0; k < 3 * nkeys; k++) {
        free(xa[k]);
        free(ya[k]);
    }
    free3(bits);
    free3(bits_a);
    free(xi);
    free(yi);
    free(X);
    free(Y);
    free(xa);
    free(ya);
    free(cols);
}

/* ------------------------------------------------------------------------- */
/* ripple_carry_adder (operators/circuits.h:35-76) of boolean sharings F and G
 * on bit-packed words of 8w elements; carry_in starts the carry at all ones
 * (inplace_invert, for subtraction) */
static void rca(oro_ctx* c, int w, size_t n, void* const F[3], void* const G[3], void* y[3], int carry_in) {
    const int B = 8 * w;
    const size_t cw = n / B + (n % B > 0);
    void *AX[3], *Ai[3], *Cr[3];
    alloc3(AX, cw, w);
    alloc3(Ai, cw, w);
    alloc3(Cr, cw, w);
    for (int j = 0; j < 3; j++) {
        for (size_t word = 0; word < cw; word++) st(Cr[j], word, w, carry_in ? wmask(w) : 0);
        for (size_t i = 0; i < n; i++) st(y[j], i, w, 0);
    }
    for (int b = 0; b < B; b++) {
        for (int j = 0; j < 3; j++)
            for (size_t word = 0; word < cw; word++) {
                u128 ax = 0, ai = 0;
                for (int k = 0; k < B && word * B + k < n; k++) {
                    const size_t e = word * B + k;
                    const u128 fa = ld(F[j], e, w), ga = ld(G[j], e, w);
                    ax |= (((fa ^ ga) >> b) & 1) << k;
                    ai |= ((fa >> b) & 1) << k;
                }
                st(AX[j], word, w, ax);
                st(Ai[j], word, w, ai);
                const u128 s = ax ^ ld(Cr[j], word, w);
                for (int k = 0; k < B && word * B + k < n; k++) {
                    const size_t e = word * B + k;
                    st(y[j], e, w, ld(y[j], e, w) | (((s >> k) & 1) << b));
                }
            }
        if (b == B - 1) break;
        /* c = ((c ^ a_i) & axb_i) ^ a_i */
        for (int j = 0; j < 3; j++)
            for (size_t word = 0; word < cw; word++) st(Cr[j], word, w, ld(Cr[j], word, w) ^ ld(Ai[j], word, w));
        oro_and_b(c, w, cw, Cr, AX, Cr);
        for (int j = 0; j < 3; j++)
            for (size_t word = 0; word < cw; word++) st(Cr[j], word, w, ld(Cr[j], word, w) ^ ld(Ai[j], word, w));
    }
    free3(AX);
    free3(Ai);
    free3(Cr);
}

/* BSharedVector::operator+ / operator- (b_shared_vector.h:588-622): the adder,
 * subtraction as x + ~y with carry-in */
void oro_add_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    rca(c, w, n, x, y, z, 0);
}
void oro_sub_b(oro_ctx* c, int w, size_t n, void* const x[3], void* const y[3], void* z[3]) {
    void* ny[3];
    alloc3(ny, n, w);
    for (int j = 0; j < 3; j++)
        for (size_t i = 0; i < n; i++) st(ny[j], i, w, ~ld(y[j], i, w));
    rca(c, w, n, x, ny, z, 1);
    free3(ny);
}

/* ASharedVector::a2b (a_shared_vector.h:138-144): redistribute_shares_b
 * (replicated_3pc.h:259-262: party 0 secret-shares x(0) + x(1) = S0 + S1,
 * then party 2 shares its x(0) = S2) and the adder. */
void oro_a2b(oro_ctx* c, int w, size_t n, void* const x[3], void* y[3]) {
    void *v, *F[3], *G[3];
    v = xalloc(n * (size_t)w + 16);
    for (size_t i = 0; i < n; i++) st(v, i, w, ld(x[0], i, w) + ld(x[1], i, w));
    alloc3(F, n, w);
    alloc3(G, n, w);
    oro_secret_share(c, 0, w, n, v, 0, F);
    oro_secret_share(c, 0, w, n, x[2], 2, G);
    rca(c, w, n, F, G, y, 0);
    free(v);
    free3(F);
    free3(G);
}

/* ========================================================================= */
/* Beaver 2PC (core/protocols/beaver_2pc.h) with dummy triples and
 * Fantastic-4PC (core/protocols/dalskov_4pc.h): the local steps of all
 * parties in one process. */

/* Keys (rand_setup.h:306-381). 2PC: call 0 local PRG, call 1 group {0,1} on
 * P0 (the everyone group is the same set and P0's call 2 is discarded).
 * 4PC: call 0 local PRG; P0 draws the group keys of {0,1,2}, {2,3,0},
 * {3,0,1} and the everyone group (calls 1-4), P1 that of {1,2,3} (call 1);
 * then setup_4pc_common_prgs (rand_setup.h:154-221) draws one more key per
 * party (P0 call 5, P1 call 2, P2 call 1, P3 call 1): party q's key seeds the
 * PRG of {q, q-1, q-2}, the one that excludes q+1. */
void oro_ctx_init_np(oro_ctx* c, uint64_t seed, int nparties) {
    static const int who2[3][2] = {{0, 1}, {0, 0}, {1, 0}};
    static const int who4[8][2] = {{3, 1}, {0, 5}, {1, 2}, {2, 1}, {0, 0}, {1, 0}, {2, 0}, {3, 0}};
    memset(c, 0, sizeof(*c));
    const int ns = nparties == 2 ? 3 : 8;
    for (int s = 0; s < ns; s++) {
        uint8_t key[32];
        const int* wh = nparties == 2 ? who2[s] : who4[s];
        oro_derive_key(seed, wh[0], wh[1], key);
        oro_aes256_expand(key, c->rk[s]);
    }
}

static u128 ar(int arith, u128 a, u128 b) { return arith ? a + b : a ^ b; }
static u128 sr(int arith, u128 a, u128 b) { return arith ? a - b : a ^ b; }
static u128 mr(int arith, u128 a, u128 b) { return arith ? a * b : a & b; }

/* 2PC secret_share_b/a (beaver_2pc.h:214-260): the owner d keeps
 * r = localPRG_d.getNext(n) and sends data - r (data ^ r).
 * 4PC (dalskov_4pc.h:152-201): s0, s1, s2 from the owner's local PRG,
 * s3 = data - s0 - s1 - s2; party d+k lacks s_k, so X[(d+k)%4] = s_k. */
void oro_np_secret_share(oro_ctx* c, int np, int arith, int w, size_t n, const void* data, int d,
                         void* const* s) {
    if (np == 2) {
        oro_stream_fill(c, ORO_P2_LOCAL0 + d, s[d], n, w);
        for (size_t i = 0; i < n; i++) st(s[1 - d], i, w, sr(arith, ld(data, i, w), ld(s[d], i, w)));
        return;
    }
    void* sk[4];
    for (int k = 0; k < 4; k++) sk[k] = s[(d + k) % 4];
    for (int k = 0; k < 3; k++) oro_stream_fill(c, ORO_P4_LOCAL0 + d, sk[k], n, w);
    for (size_t i = 0; i < n; i++) {
        u128 v = ld(data, i, w);
        for (int k = 0; k < 3; k++) v = sr(arith, v, ld(sk[k], i, w));
        st(sk[3], i, w, v);
    }
}

void oro_np_open(int np, int arith, int w, size_t n, void* const* s, void* out) {
    for (size_t i = 0; i < n; i++) {
        u128 v = 0;
        for (int k = 0; k < np; k++) v = ar(arith, v, ld(s[k], i, w));
        st(out, i, w, v);
    }
}

/* op: 0 xor, 1 add, 2 sub (local on every share) */
void oro_np_local(int np, int op, int w, size_t n, void* const* x, void* const* y, void* const* z) {
    for (int k = 0; k < np; k++)
        for (size_t i = 0; i < n; i++) {
            u128 a = ld(x[k], i, w), b = ld(y[k], i, w);
            st(z[k], i, w, op == 0 ? a ^ b : op == 1 ? a + b : a - b);
        }
}

/* next_party / excluded_party (dalskov_4pc.h:11-24) */
static int f4_next(int i, int j) {
    int a = i < j ? i : j, b = i < j ? j : i;
    return b == (a + 1) % 4 ? (b + 1) % 4 : (a + 1) % 4;
}

/* 4PC inp<E>(v, Pi, Pj, Pg, Ph) (dalskov_4pc.h:300-340) accumulated into r:
 * X'[g] = R from the PRG that excludes g, X'[h] = v - R (v ^ R), others 0. */
static void f4_inp_acc(oro_ctx* c, int arith, int w, size_t n, const void* v, int g, int h, void* r[4]) {
    void* R = xalloc(n * (size_t)w);
    oro_stream_fill(c, ORO_P4_NOT0 + g, R, n, w);
    for (size_t i = 0; i < n; i++) {
        u128 rr = ld(R, i, w);
        st(r[g], i, w, ar(arith, ld(r[g], i, w), rr));
        st(r[h], i, w, ar(arith, ld(r[h], i, w), sr(arith, ld(v, i, w), rr)));
    }
    free(R);
}

void oro_np_mult(oro_ctx* c, int np, int arith, int w, size_t n, void* const* x, void* const* y,
                 void* const* z) {
    if (np == 2) {
        /* DummyOLE::getNext(2n) (dummy_ole.h): B, C, D from the common PRG,
         * A = C*D - B (B ^ C&D); P0 gets (A, C), P1 (B, D). Beaver triple
         * (beaver_triple_generator.h:getNext): P0 a=C[:n] b=C[n:]
         * c=a*b+A[:n]+A[n:]; P1 a=D[n:] b=D[:n] c=a*b+B[:n]+B[n:].
         * multiply_a / and_b (beaver_2pc.h:50-59,108-117): A' = open(x+a),
         * B' = open(y+b), z_p = y_p*A' - a_p*B' + c_p. */
        const size_t m = 2 * n;
        uint8_t* B = xalloc(m * (size_t)w);
        uint8_t* C = xalloc(m * (size_t)w);
        uint8_t* D = xalloc(m * (size_t)w);
        oro_stream_fill(c, ORO_P2_COMMON, B, m, w);
        oro_stream_fill(c, ORO_P2_COMMON, C, m, w);
        oro_stream_fill(c, ORO_P2_COMMON, D, m, w);
        for (size_t i = 0; i < n; i++) {
            u128 Cl = ld(C, i, w), Cr = ld(C, n + i, w), Dl = ld(D, i, w), Dr = ld(D, n + i, w);
            u128 Bl = ld(B, i, w), Br = ld(B, n + i, w);
            u128 Al = sr(arith, mr(arith, Cl, Dl), Bl), Arr = sr(arith, mr(arith, Cr, Dr), Br);
            if (!arith) {
                Al = Bl ^ (Cl & Dl);
                Arr = Br ^ (Cr & Dr);
            }
            u128 a[2] = {Cl, Dr}, b[2] = {Cr, Dl};
            u128 cc[2] = {ar(arith, ar(arith, mr(arith, Cl, Cr), Al), Arr),
                          ar(arith, ar(arith, mr(arith, Dr, Dl), Bl), Br)};
            u128 x0 = ld(x[0], i, w), x1 = ld(x[1], i, w), y0 = ld(y[0], i, w), y1 = ld(y[1], i, w);
            u128 Ao = ar(arith, ar(arith, x0, a[0]), ar(arith, x1, a[1]));
            u128 Bo = ar(arith, ar(arith, y0, b[0]), ar(arith, y1, b[1]));
            u128 yy[2] = {y0, y1};
            for (int p = 0; p < 2; p++)
                st(z[p], i, w, ar(arith, sr(arith, mr(arith, yy[p], Ao), mr(arith, a[p], Bo)), cc[p]));
        }
        free(B);
        free(C);
        free(D);
        return;
    }
    /* 4PC multiply_a / and_b (dalskov_4pc.h:384-420,479-506): for the pairs
     * (0,1) (0,2) (0,3) (1,2) (1,3) (2,3), inp of X_h*Y_g + X_g*Y_h into the
     * result, then Z_k += X_k*Y_k. */
    void* r[4];
    void* v = xalloc(n * (size_t)w);
    for (int k = 0; k < 4; k++) r[k] = xalloc(n * (size_t)w);
    for (int i = 0; i < 4; i++)
        for (int j = i + 1; j < 4; j++) {
            int g = f4_next(i, j), h = 6 - i - j - g;
            for (size_t e = 0; e < n; e++) {
                u128 xh = ld(x[h], e, w), xg = ld(x[g], e, w), yh = ld(y[h], e, w), yg = ld(y[g], e, w);
                st(v, e, w, ar(arith, mr(arith, xh, yg), mr(arith, xg, yh)));
            }
            f4_inp_acc(c, arith, w, n, v, g, h, r);
        }
    for (int k = 0; k < 4; k++) {
        for (size_t e = 0; e < n; e++)
            st(z[k], e, w, ar(arith, ld(r[k], e, w), mr(arith, ld(x[k], e, w), ld(y[k], e, w))));
        free(r[k]);
    }
    free(v);
}

void oro_np_b2a_bit(oro_ctx* c, int np, int w, size_t n, void* const* x, void* const* y) {
    void* t[4];
    for (int k = 0; k < np; k++) t[k] = xalloc(n * (size_t)w);
    if (np == 2) {
        /* beaver_2pc.h:147-158: xm = x & 1, P1 negates its share, xm * xm */
        for (size_t i = 0; i < n; i++) {
            st(t[0], i, w, ld(x[0], i, w) & 1);
            st(t[1], i, w, (u128)0 - (ld(x[1], i, w) & 1));
        }
    } else {
        /* dalskov_4pc.h:562-590: s0 = X2^X3 (bits, held by P0 and P1) shared by
         * inp(s0, 1, 0) (g = 2, h = 3), s1 = X0^X1 shared by inp(s1, 3, 2)
         * (g = 0, h = 1); share0 - share1, squared */
        void* s0 = xalloc(n * (size_t)w);
        void* s1 = xalloc(n * (size_t)w);
        void* u[4];
        for (int k = 0; k < 4; k++) u[k] = xalloc(n * (size_t)w);
        for (size_t i = 0; i < n; i++) {
            st(s0, i, w, (ld(x[2], i, w) ^ ld(x[3], i, w)) & 1);
            st(s1, i, w, (ld(x[0], i, w) ^ ld(x[1], i, w)) & 1);
        }
        f4_inp_acc(c, 1, w, n, s0, 2, 3, t);
        f4_inp_acc(c, 1, w, n, s1, 0, 1, u);
        for (int k = 0; k < 4; k++) {
            for (size_t i = 0; i < n; i++) st(t[k], i, w, ld(t[k], i, w) - ld(u[k], i, w));
            free(u[k]);
        }
        free(s0);
        free(s1);
    }
    oro_np_mult(c, np, 1, w, n, t, t, y);
    for (int k = 0; k < np; k++) free(t[k]);
}
