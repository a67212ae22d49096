/*
 * sodium.h — test-only stand-in for the libsodium calls ORQ makes, used to
 * build the reference (include/ of CASP-Systems-BU/orq) as the parity oracle.
 *
 * libsodium is not installed in this image. The reference uses it for:
 *   - crypto_aead_aes256gcm_encrypt_detached (core/random/prg/prg_algorithm.h:228)
 *     -> implemented with OpenSSL's EVP AES-256-GCM (same standard, NIST SP 800-38D);
 *   - crypto_aead_aes256gcm_keygen (prg_algorithm.h:196)
 *     -> made deterministic: key = SplitMix64 stream keyed by (seed, party, call
 *        index), seed from ORQ_SHIM_SEED and party from STARTMPC_HOST_RANK, so
 *        the GPU runtime can derive the same keys (oro_derive_key);
 *   - crypto_generichash* (4PC transcript hashes) -> SHA-512 through OpenSSL
 *     (consistent between parties; shares never depend on it);
 *   - crypto_stream_xchacha20* -> abort (not on the path).
 */
#pragma once

#include <openssl/evp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define crypto_aead_aes256gcm_KEYBYTES 32U
#define crypto_aead_aes256gcm_NPUBBYTES 12U
#define crypto_aead_aes256gcm_ABYTES 16U
#define crypto_stream_xchacha20_KEYBYTES 32U
#define crypto_stream_xchacha20_NONCEBYTES 24U
#define crypto_generichash_BYTES 32U
#define crypto_generichash_BYTES_MAX 64U
#define crypto_generichash_KEYBYTES 32U
#define crypto_generichash_blake2b_BYTES 32U

typedef struct crypto_generichash_state {
    unsigned char opaque[384];
} crypto_generichash_state;

static inline int sodium_init(void) { return 0; }

static inline uint64_t orq_shim_splitmix64(uint64_t* state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline int* orq_shim_keygen_counter(void) {
    static int counter = 0;
    return &counter;
}

static inline void crypto_aead_aes256gcm_keygen(unsigned char k[32]) {
    const char* seed_env = getenv("ORQ_SHIM_SEED");
    const char* rank_env = getenv("STARTMPC_HOST_RANK");
    uint64_t seed = seed_env ? strtoull(seed_env, NULL, 0) : 0;
    int party = rank_env ? atoi(rank_env) : 0;
    int call = (*orq_shim_keygen_counter())++;
    uint64_t st = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(party + 1)) ^
                  (0xABC98388FB8FAC03ull * (uint64_t)(call + 1));
    for (int i = 0; i < 4; i++) {
        uint64_t v = orq_shim_splitmix64(&st);
        for (int b = 0; b < 8; b++) k[8 * i + b] = (unsigned char)(v >> (8 * b));
    }
    if (getenv("ORQ_SHIM_TRACE")) fprintf(stderr, "[shim] P%d keygen call %d\n", party, call);
}

static inline int crypto_aead_aes256gcm_encrypt_detached(
    unsigned char* c, unsigned char* mac, unsigned long long* maclen_p, const unsigned char* m,
    unsigned long long mlen, const unsigned char* ad, unsigned long long adlen,
    const unsigned char* nsec, const unsigned char* npub, const unsigned char* k) {
    (void)nsec;
    EVP_CIPHER_CTX* ctx = EVP_CIPHER_CTX_new();
    int len = 0;
    int ok = EVP_EncryptInit_ex(ctx, EVP_aes_256_gcm(), NULL, NULL, NULL);
    ok &= EVP_CIPHER_CTX_ctrl(ctx, EVP_CTRL_GCM_SET_IVLEN, 12, NULL);
    ok &= EVP_EncryptInit_ex(ctx, NULL, NULL, k, npub);
    if (ad && adlen) ok &= EVP_EncryptUpdate(ctx, NULL, &len, ad, (int)adlen);
    unsigned long long done = 0;
    while (done < mlen) {
        int chunk = (int)((mlen - done) > (1u << 30) ? (1u << 30) : (mlen - done));
        ok &= EVP_EncryptUpdate(ctx, c + done, &len, m + done, chunk);
        done += (unsigned long long)chunk;
    }
    ok &= EVP_EncryptFinal_ex(ctx, c + done, &len);
    ok &= EVP_CIPHER_CTX_ctrl(ctx, EVP_CTRL_GCM_GET_TAG, 16, mac);
    EVP_CIPHER_CTX_free(ctx);
    if (maclen_p) *maclen_p = 16;
    if (!ok) {
        fprintf(stderr, "[shim] AES-GCM failure\n");
        abort();
    }
    return 0;
}

static inline void crypto_stream_xchacha20_keygen(unsigned char k[32]) {
    (void)k;
    fprintf(stderr, "[shim] xchacha20 is not provided\n");
    abort();
}
static inline int crypto_stream_xchacha20(unsigned char* c, unsigned long long clen,
                                          const unsigned char* n, const unsigned char* k) {
    (void)c, (void)clen, (void)n, (void)k;
    fprintf(stderr, "[shim] xchacha20 is not provided\n");
    abort();
}
/* crypto_generichash* (the 4PC transcript hashes, dalskov_4pc.h:107-111):
 * here SHA-512 truncated to the requested length through OpenSSL. The hashes
 * only let honest parties compare their views; every party computes the same
 * function, so the checks pass and no share depends on it. */
static inline EVP_MD_CTX** orq_shim_hash_ctx(crypto_generichash_state* s) {
    return (EVP_MD_CTX**)(void*)s->opaque;
}
static inline int crypto_generichash_init(crypto_generichash_state* s, const unsigned char* key,
                                          size_t keylen, size_t outlen) {
    (void)outlen;
    EVP_MD_CTX** c = orq_shim_hash_ctx(s);
    *c = EVP_MD_CTX_new();
    if (!*c || !EVP_DigestInit_ex(*c, EVP_sha512(), NULL)) abort();
    if (key && keylen) EVP_DigestUpdate(*c, key, keylen);
    return 0;
}
static inline int crypto_generichash_update(crypto_generichash_state* s, const unsigned char* in,
                                            unsigned long long inlen) {
    EVP_MD_CTX** c = orq_shim_hash_ctx(s);
    if (inlen && !EVP_DigestUpdate(*c, in, (size_t)inlen)) abort();
    return 0;
}
static inline int crypto_generichash_final(crypto_generichash_state* s, unsigned char* out,
                                           size_t outlen) {
    EVP_MD_CTX** c = orq_shim_hash_ctx(s);
    unsigned char md[64];
    unsigned int len = 0;
    if (!EVP_DigestFinal_ex(*c, md, &len)) abort();
    EVP_MD_CTX_free(*c);
    *c = NULL;
    memcpy(out, md, outlen < 64 ? outlen : 64);
    return 0;
}
static inline int crypto_generichash(unsigned char* out, size_t outlen, const unsigned char* in,
                                     unsigned long long inlen, const unsigned char* key,
                                     size_t keylen) {
    crypto_generichash_state st;
    crypto_generichash_init(&st, key, keylen, outlen);
    crypto_generichash_update(&st, in, inlen);
    return crypto_generichash_final(&st, out, outlen);
}
