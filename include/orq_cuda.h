/*
 * orq_cuda.h — C ABI of liborq_cuda.so, the B200 loopback runtime for ORQ's
 * replicated-3PC share computation.
 *
 * The library replaces, for all three parties at once on one GPU, the
 * per-party protocol dispatch of ORQ's RunTime (include/backend/common/
 * runtime.h:123-144, generated by runtime_declare_protocol_functions) together
 * with the socket exchange that follows each round (the ±1 exchange becomes a
 * property of the share layout), and the operators built from them.
 *
 * Conventions
 *   - A shared vector of n elements of `width` bytes (1, 2, 4, 8 or 16) is
 *     three device arrays S[0], S[1], S[2]; party p of the reference holds
 *     (S[p], S[(p+1)%3]) — the layout of get_shares_b/a
 *     (include/core/protocols/replicated_3pc.h:353-392).
 *   - `arith` = 1 selects arithmetic shares mod 2^(8*width) (ASharedVector),
 *     0 boolean XOR shares (BSharedVector).
 *   - PRG keys are derived from the runtime seed exactly as the deterministic
 *     key generator used to build the reference; every call consumes the
 *     runtime's PRG streams in the order the reference consumes them with one
 *     worker thread and batch size -1, so shares are bit-identical to the
 *     reference's for the same call sequence.
 *   - Device pointers must be cudaMalloc'd (or orqcu_malloc'd); arrays of 16-byte
 *     elements must be 16-byte aligned. Calls are asynchronous on the runtime's
 *     stream unless stated; results are visible after orqcu_synchronize.
 *   - Every function returns 0 on success or a negative ORQCU_E* code;
 *     orqcu_last_error() gives the message of the last failure on this thread.
 */
#ifndef ORQ_CUDA_H
#define ORQ_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORQCU_OK 0
#define ORQCU_EINVAL (-1)   /* bad argument (reference: assert / std::runtime_error) */
#define ORQCU_ECUDA (-2)    /* CUDA runtime error */
#define ORQCU_ERUNTIME (-3) /* protocol-level failure */
#define ORQCU_ENOMEM (-4)

/* PRG stream ids (include/backend/common/rand_setup.h:90-146,306-381) */
#define ORQCU_STREAM_PAIR0 0  /* P0/P1 pairwise: P0's get(+1), P1's get(-1) */
#define ORQCU_STREAM_PAIR1 1
#define ORQCU_STREAM_PAIR2 2
#define ORQCU_STREAM_G01 3    /* group {0,1} common PRG */
#define ORQCU_STREAM_G02 4
#define ORQCU_STREAM_G12 5
#define ORQCU_STREAM_G012 6
#define ORQCU_STREAM_LOCAL0 7 /* party-local PRGs */
#define ORQCU_STREAM_LOCAL1 8
#define ORQCU_STREAM_LOCAL2 9

typedef struct orqcu_runtime orqcu_runtime;

int orqcu_version(void);
const char* orqcu_last_error(void);

/* orq_init (include/backend/common/setup.h:8-58,121-129) for all three
 * parties: keys for the 10 streams, nonces at 0. device = CUDA ordinal. */
int orqcu_runtime_create(uint64_t seed, int device, orqcu_runtime** out);
int orqcu_runtime_destroy(orqcu_runtime* rt);
/* Run subsequent work on an existing cudaStream_t; NULL selects the CUDA
 * default stream (as in the CUDA runtime API). */
int orqcu_runtime_set_stream(orqcu_runtime* rt, void* cuda_stream);
int orqcu_synchronize(orqcu_runtime* rt);
/* Nonce counter of a PRG stream (AESPRGAlgorithm::nonce, prg_algorithm.h:208). */
int orqcu_get_nonce(orqcu_runtime* rt, int stream, uint64_t* nonce);
/* Number of kernels this runtime has launched. */
int orqcu_kernels_launched(orqcu_runtime* rt, uint64_t* count);

/* Per-kernel timing, the device counterpart of ORQ's thread instrumentation
 * (include/profiling/thread_profiling.h:227-280): when enabled, every launch is
 * bracketed by CUDA events on its stream. The report (and reset) gives one line
 * per kernel class: "name launches total_ms algorithmic_bytes aes_blocks". */
int orqcu_profile_enable(orqcu_runtime* rt, int on);
int orqcu_profile_report(orqcu_runtime* rt, char* buf, size_t len);

/* device memory helpers */
int orqcu_malloc(orqcu_runtime* rt, size_t bytes, void** dptr);
int orqcu_free(orqcu_runtime* rt, void* dptr);
int orqcu_memcpy_h2d(orqcu_runtime* rt, void* dst_dev, const void* src_host, size_t bytes);
int orqcu_memcpy_d2h(orqcu_runtime* rt, void* dst_host, const void* src_dev, size_t bytes);
/* Stream-ordered device memory from the runtime's pool (the storage behind
 * ORQ's Vector / EVector, mapping_access_vector.h:208-260): a block freed here
 * is reused by later work on the runtime's stream without synchronising the
 * device. Only pointers from orqcu_pool_alloc may be passed to orqcu_pool_free. */
int orqcu_pool_alloc(orqcu_runtime* rt, size_t bytes, void** dptr);
int orqcu_pool_free(orqcu_runtime* rt, void* dptr);
/* Device-to-device copy and byte fill, asynchronous on the runtime's stream
 * (Vector's deep operator=, mapping_access_vector.h:1263, and zero-initialised
 * storage). */
int orqcu_memcpy_d2d(orqcu_runtime* rt, void* dst_dev, const void* src_dev, size_t bytes);
int orqcu_memset(orqcu_runtime* rt, void* dst_dev, int byte, size_t bytes);

/* Keystream of `stream` starting at nonce0 (AESPRGAlgorithm::fillBytes,
 * prg_algorithm.h:161-172); does not advance the stream. */
int orqcu_keystream(orqcu_runtime* rt, int stream, uint64_t nonce0, size_t nbytes, void* out_dev);

/* secret_share_b / secret_share_a (replicated_3pc.h:401-448) with the owner's
 * local PRG; data_dev is the owner's plaintext on the device. */
int orqcu_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data_dev,
                       int data_party, void* const shares[3]);
/* public_share (replicated_3pc.h:456-470): S0 = x, S1 = S2 = 0. */
int orqcu_public_share(orqcu_runtime* rt, int width, size_t n, const void* data_dev,
                       void* const shares[3]);
/* open_shares_a / open_shares_b (replicated_3pc.h:310-330). */
int orqcu_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const shares[3],
               void* out_dev);

/* and_b (replicated_3pc.h:166-191) fused with ZeroSharingGenerator::getNextBinary. */
int orqcu_and_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                const void* const y[3], void* const z[3]);
/* multiply_a (replicated_3pc.h:44-67) fused with getNextArithmetic. */
int orqcu_multiply_a(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                     const void* const y[3], void* const z[3]);
/* xor_b / add_a / sub_a (protocol.h:561-649): local, no randomness. */
int orqcu_xor_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                const void* const y[3], void* const z[3]);
int orqcu_add_a(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                const void* const y[3], void* const z[3]);
int orqcu_sub_a(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                const void* const y[3], void* const z[3]);
/* not_b (replicated_3pc.h:199). */
int orqcu_not_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]);
/* BSharedVector::operator+ / operator- (b_shared_vector.h:588-622): addition
 * and subtraction mod 2^(8*width) of boolean sharings by the ripple-carry
 * adder (circuits.h:35-76; subtraction adds ~y with a carry-in), 8W-1 AND
 * rounds on bit-packed words in one launch. width 4 or 8; z must not alias
 * x or y. */
int orqcu_add_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], const void* const y[3],
                void* const z[3]);
int orqcu_sub_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], const void* const y[3],
                void* const z[3]);
/* ASharedVector::a2b (a_shared_vector.h:138-144): arithmetic -> boolean
 * sharing of the full width (4 or 8): redistribute_shares_b
 * (replicated_3pc.h:259-262; party 0 secret-shares S0 + S1, party 2 shares S2)
 * then the boolean ripple-carry adder (circuits.h:35-76, 8W-1 AND rounds on
 * bit-packed words), one fused launch for the adder. y must not alias x. */
int orqcu_a2b(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]);
/* b2a_bit (replicated_3pc.h:220-251): LSB of a boolean sharing -> arithmetic. */
int orqcu_b2a_bit(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]);
/* Pairwise zero-sharing (zero_sharing_generator.h:101-148). */
int orqcu_zero_share(orqcu_runtime* rt, int arith, int width, size_t n, void* const r[3]);
/* Protocol::reshare (protocol.h:500-541), group 0={0,1}, 1={0,2}, 2={1,2}. */
int orqcu_reshare(orqcu_runtime* rt, int arith, int width, size_t n, int group,
                  void* const shares[3]);

/* SharedVector::prefix_sum (shared_vector.h:249): in-place inclusive scan of
 * each share array mod 2^(8*width); width 4 or 8. Local (no randomness). */
int orqcu_prefix_sum_a(orqcu_runtime* rt, int width, size_t n, void* const shares[3]);
/* The same prefix sum for callers that cannot allocate device memory when they
 * call: a host program that has already reserved the GPU's memory for its own
 * pool, or a service loop that cannot afford cudaMalloc's device-wide
 * synchronisation while other work runs. It has no counterpart in the
 * reference. Its scratch (the tile sums) is a fixed 384 KiB array in the
 * library, held on every GPU that loads it until the process exits, so n is
 * limited to 2^26 elements (larger n returns ORQCU_EINVAL and touches nothing).
 * The first call on a device looks up the array's device address, so make
 * that first call before any stream capture; the address is looked up again
 * after the last runtime on the device has been destroyed (a cudaDeviceReset
 * while a runtime of the device is alive is not supported). All calls share
 * the array: calls
 * that overlap on the GPU (on any streams) race and must be serialised. No
 * cudaMalloc, cudaFree or other allocating routine is called. */
int orqcu_prefix_sum_a_noalloc(orqcu_runtime* rt, int width, size_t n, void* const shares[3]);

/* PermutationManager::reserve (permutation_manager.h:102-181): generate
 * `count` sharded permutations of size n ahead of use. Synchronous. */
int orqcu_reserve_permutations(orqcu_runtime* rt, size_t n, size_t count);
/* Pop the next sharded permutation (PermutationManager::getNext) and copy its
 * three group-local permutations ({0,1},{0,2},{1,2}; gen_perm's output,
 * hm_sharded_permutation_generator.h:70-108) to perm_dev[g]. */
int orqcu_next_permutation(orqcu_runtime* rt, size_t n, int32_t* const perm_dev[3]);
/* shuffle (shuffle.h:752-757). width 4, 8 or 16. */
int orqcu_shuffle(orqcu_runtime* rt, int arith, int width, size_t n, void* const shares[3]);
/* oblivious_apply_elementwise_perm (shuffle.h:687-706): x permuted in place by
 * an A-shared int32 permutation. */
int orqcu_apply_elementwise_perm(orqcu_runtime* rt, int x_arith, int x_width, size_t n,
                                 void* const x[3], const void* const perm[3]);
/* radix_sort (radixsort.h:205-229): sorts the B-shared key (width 4 or 8) on its
 * low `bits` bits (signed order when bits = 8*width), ascending; writes the
 * A-shared int32 sorting permutation to perm_out. Synchronous. */
int orqcu_radix_sort(orqcu_runtime* rt, int key_width, size_t n, void* const key[3], int bits,
                     int descending, void* const perm_out[3]);

/* `count` independent radix sorts (keys[3*i+p], width key_width 4 or 8, n[i]
 * rows, bits[i], descending[i]); perms_out[3*i+p] receives item i's A-shared
 * int32 sorting permutation. The shares equal those of `count`
 * orqcu_radix_sort calls in list order (the same PRG draws in the same
 * order); items run back to back with one synchronisation at the end. No
 * reference counterpart (ORQ sorts one vector per call). Synchronous. */
int orqcu_radix_sort_batch(orqcu_runtime* rt, int key_width, int count, const size_t* n, void* const* keys,
                           const int* bits, const int* descending, void* const* perms_out);

/* quicksort (quicksort.h:214-246): sorts the B-shared key (width 4 or 8) in
 * the signed order, ascending or descending, and writes the A-shared int32
 * sorting permutation to perm_out. The protocol of quicksort_body
 * (quicksort.h:61-200): the padded rows are shuffled, then each round compares
 * every non-pivot row with its segment's pivot (opened) and partitions every
 * segment as the reference's Lomuto partition does, so the rounds, their
 * compare sizes and the PRG use equal the reference's. Reserves 2
 * permutations and 1 pair up front. Synchronous. */
int orqcu_quicksort(orqcu_runtime* rt, int key_width, size_t n, void* const key[3], int descending,
                    void* const perm_out[3]);
/* BSharedVector::_compare (circuits.h:231-295, bit_same at
 * b_shared_vector.h:164-178): eq = (x == y), gt = (x > y) in the signed order,
 * both as B-shared single bits (LSB of each share). width 4, 8 or 16 (the
 * padded int64 keys of the sorts). One fused launch: log2(8*width)+1 AND
 * rounds on every pair and the packed sign fix-up. */
int orqcu_compare_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                    const void* const y[3], void* const eq[3], void* const gt[3]);
/* BSharedVector::operator== (b_shared_vector.h:493-504): bit_same (log2(8W)
 * AND rounds, b_shared_vector.h:164-178) then mask(1); eq is a B-shared bit.
 * width 4, 8 or 16. */
int orqcu_equal_b(orqcu_runtime* rt, int width, size_t n, const void* const x[3],
                  const void* const y[3], void* const eq[3]);
/* not_b_1 (replicated_3pc.h:207), BSharedVector::operator!: every share
 * becomes !(s & 1), the logical NOT of a B-shared bit. Local. */
int orqcu_not_b_1(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]);
/* bitonic_sort (sorting.h:266-353) of one B-shared key column in place, in the
 * signed order; n a power of two, width 4 or 8. One launch per network stage
 * (compare + two multiplexes, operators/common.h:20-28). */
int orqcu_bitonic_sort(orqcu_runtime* rt, int width, size_t n, void* const key[3],
                       int descending);
/* bitonic_sort (sorting.h:266-353) over nkeys B-shared key columns (keys[3*k+p],
 * most significant first, each ascending or descending) with na A-shared and
 * nb B-shared data columns moved along, in place; n a power of two, width 4
 * or 8, at most 8 keys and 40 columns. Per network stage one compare_rows
 * launch and one swap launch (keys and B data with the bits, A data with
 * b2a_bit of them). One key and no data take the fused orqcu_bitonic_sort path. */
int orqcu_bitonic_sort_rows(orqcu_runtime* rt, int width, size_t n, int nkeys, void* const* keys,
                            const int* descending, int na, void* const* data_a, int nb,
                            void* const* data_b);
/* compare_rows (sorting.h:80-108): gt[i] = row i of the nkeys key columns x
 * (x[3*k+p]) is greater than row i of y in their lexicographic order, key k
 * ascending or descending; gt is a B-shared bit. One fused launch. */
int orqcu_compare_rows(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* x,
                       const void* const* y, const int* descending, void* const gt[3]);
/* swap (sorting.h:146-212): for each of ncols column pairs (x[3*k+p],
 * y[3*k+p]) exchange rows i where bits[i] is 1, with two multiplexes per
 * column (operators/common.h:20-49): B-shared columns with B-shared bits
 * (arith = 0), A-shared columns with A-shared bits (arith = 1). x and y must
 * not alias. One fused launch. */
int orqcu_swap(orqcu_runtime* rt, int arith, int width, size_t n, int ncols, void* const* x,
               void* const* y, const void* const bits[3]);
/* operators::shuffle(data_a, data_b, size) (shuffle.h:769-786), as
 * EncodedTable::shuffle uses it: one random elementwise permutation (the
 * public identity at the columns' width, B-shared, under a sharded
 * permutation) applied with oblivious_apply_elementwise_perm to every
 * A-shared column (data_a[3*k+p]) and then every B-shared column. Synchronous. */
int orqcu_table_shuffle(orqcu_runtime* rt, int width, size_t n, int na, void* const* data_a, int nb,
                        void* const* data_b);
/* BSharedVector::mask(m) (b_shared_vector.h:462-464): every share &= m (local). */
int orqcu_mask_b(orqcu_runtime* rt, int width, size_t n, void* const shares[3], uint64_t mask);
/* BSharedVector::extend_lsb (b_shared_vector.h:145-147): every share becomes
 * all ones where its LSB is set, else zero. Local. */
int orqcu_extend_lsb(orqcu_runtime* rt, int width, size_t n, const void* const x[3], void* const y[3]);

/* Aggregation functions (aggregation.h:27-140). */
enum {
    ORQCU_AGG_SUM = 0,    /* arithmetic: a + g*b */
    ORQCU_AGG_COUNT = 1,  /* arithmetic: sum over ones (or b2a_bit(sel) inside joins) */
    ORQCU_AGG_COPY = 2,   /* arithmetic or boolean: multiplex(g, a, b) */
    ORQCU_AGG_VALID = 3,  /* boolean: multiplex(g, a, a & b) */
    ORQCU_AGG_BIT_OR = 4, /* boolean: a | (ext(g) & b) */
    ORQCU_AGG_MIN = 5,
    ORQCU_AGG_MAX = 6
};
/* One aggregation: input column, output column (3 share pointers each), and
 * the function. The output is overwritten (out = in first, as the reference). */
typedef struct {
    const void* in[3];
    void* out[3];
    int func;
} orqcu_agg_spec;
/* orq::aggregators::aggregate (aggregation.h:167-346): the odd-even
 * aggregation network over n rows (a power of two) of width-byte shares (4 or
 * 8). keys: nkeys B-shared key columns, 3 pointers each (keys[3*j+p]); b_specs
 * are boolean aggregations (copy, valid, bit_or), a_specs arithmetic ones
 * (sum, count, copy) — min and max (boolean, by the compare circuit's packed
 * sign fix-up) are accepted among b_specs; reverse selects
 * Direction::Reverse; sel (3 pointers, or NULL) is the table-id column that
 * restricts non-copy aggregations to rows of the same table. One fused launch
 * per network level; at most 4 keys and 8 specs of each kind. */
int orqcu_aggregate(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* keys,
                    int nb, const orqcu_agg_spec* b_specs, int na, const orqcu_agg_spec* a_specs,
                    int reverse, const void* const* sel);

/* compose_permutations (shuffle.h:717-743) of two A-shared int32 elementwise
 * permutations of n rows: rho <- rho * sigma (sort by sigma's order, then
 * rho's). sigma is consumed (left shuffled). Synchronous. */
int orqcu_compose_permutations(orqcu_runtime* rt, size_t n, void* const sigma[3],
                               void* const rho[3]);
/* SortingProtocol (sorting.h:15-21), in the reference's order. */
enum { ORQCU_SORT_BITONIC = 0, ORQCU_SORT_QUICK = 1, ORQCU_SORT_RADIX = 2 };
/* table_sort (sorting.h:509-612) over n rows of width-byte columns (4 or 8):
 * ncols B-shared key columns (cols[3*k+p]), each ascending or descending and
 * sorted on 1 bit (single_bit, e.g. valid and table-id columns, by a 1-bit
 * radix sort) or on its full width by the protocol (ORQCU_SORT_QUICK or
 * ORQCU_SORT_RADIX; others are "Unknown table sort protocol"); na A-shared and
 * nb B-shared data columns are permuted along. Reserves its permutations up
 * front like the reference. Synchronous. */
int orqcu_table_sort(orqcu_runtime* rt, int width, size_t n, int ncols, void* const* cols,
                     const int* descending, const int* single_bit, int na, void* const* data_a,
                     int nb, void* const* data_b, int protocol);
/* distinct (distinct.h:20-53): res[0] = 1 and res[i] = 1 where row i differs
 * from row i-1 in any of the nkeys B-shared key columns (keys[3*k+p]); one
 * fused launch. */
int orqcu_distinct(orqcu_runtime* rt, int width, size_t n, int nkeys, const void* const* keys,
                   void* const res[3]);

/* Batched bitonic_sort: `count` independent B-shared key columns of
 * power-of-two sizes n[i] (keys[3*i+p]), each ascending or descending. The
 * shares produced are exactly those of `count` orqcu_bitonic_sort calls in
 * list order. Execution is batched: one persistent launch per network round
 * walks a ragged work list of every column that still has a stage, the
 * threads per CTA are autotuned once per size class, and with use_graph the
 * rounds are captured once per batch shape into a CUDA graph that later calls
 * replay. No reference counterpart: ORQ sorts one vector per call. */
int orqcu_bitonic_sort_batch(orqcu_runtime* rt, int width, int count, const size_t* n,
                             void* const* keys, const int* descending, int use_graph);

/* Re-key the runtime as orqcu_runtime_create(seed) would (fresh keys, nonces
 * at zero, reserved permutations dropped) while keeping its stream, its
 * cached device memory, tuned launch shapes and captured graphs. A serving
 * slot runs each request on its own seed this way, so a request's shares do
 * not depend on what ran before it. No reference counterpart (one
 * orq_init per process there). */
int orqcu_runtime_reseed(orqcu_runtime* rt, uint64_t seed);
/* Return the runtime's cached (unused) device memory to the device's memory
 * pool, ordered on the runtime's stream (no device-wide synchronisation),
 * where other runtimes' allocations reuse it without mapping it again; writes
 * the bytes that were cached to *cached_before when non-NULL. The pool gives
 * its unused memory back to the system when the last runtime on the device
 * is destroyed. A runtime that misses its cache while holding 8 GiB or more
 * of other sizes returns its least recently released blocks the same way,
 * as much as the new block needs, before allocating. */
int orqcu_runtime_trim(orqcu_runtime* rt, size_t* cached_before);

/* Size this runtime's grids for `sms` SMs (0 = all; at least 4) instead of the
 * whole device, so that runtimes working concurrently on one GPU (serving
 * slots) keep their kernels resident side by side instead of each filling
 * every SM in turn. Results do not depend on it. No reference counterpart. */
int orqcu_runtime_set_sm_limit(orqcu_runtime* rt, int sms);

/* ---- Beaver 2PC and Fantastic-4PC ------------------------------------------
 * The local steps of ORQ's other protocol classes, every party in this
 * process. A runtime made by orqcu_runtime_create_np runs one of them:
 *   nparties = 2: Beaver_2PC (include/core/protocols/beaver_2pc.h) with the
 *     dummy triples of a USE_DUMMY_TRIPLES build (random/correlation/
 *     dummy_ole.h, beaver_triple_generator.h); a vector is S[0], S[1] and
 *     party p holds S[p];
 *   nparties = 4: Fantastic_4PC (include/core/protocols/dalskov_4pc.h); a
 *     vector is X[0..3], X[j] being the share party j lacks (party p holds
 *     X[p+1], X[p+2], X[p+3] as its local shares 0, 1, 2, get_shares at
 *     dalskov_4pc.h:152-168).
 * Keys follow the same deterministic key generator as the 3PC runtime, in
 * each protocol's keygen order (rand_setup.h:154-238,306-381), so shares equal
 * the reference's with one worker and batch size -1. `shares`, `x`, `y`, `z`
 * are arrays of nparties device pointers; widths 1, 2, 4 or 8. The 3PC entry
 * points refuse such a runtime and these refuse a 3PC one (ORQCU_EINVAL). */
int orqcu_runtime_create_np(uint64_t seed, int device, int nparties, orqcu_runtime** out);
/* 2, 3 or 4 */
int orqcu_runtime_parties(orqcu_runtime* rt, int* nparties);
/* secret_share_b / secret_share_a (beaver_2pc.h:214-260, dalskov_4pc.h:152-201)
 * from data_party's local PRG; data_dev is its plaintext on the device. */
int orqcu_np_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data_dev,
                          int data_party, void* const* shares);
/* open_shares_a / open_shares_b (beaver_2pc.h:172-183, dalskov_4pc.h:660-676). */
int orqcu_np_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const* shares,
                  void* out_dev);
/* and_b / multiply_a (beaver_2pc.h:50-59,108-117 with the dummy triple of the
 * call; dalskov_4pc.h:384-420,479-506 with the six inp sharings), one fused
 * launch each; z must not alias x or y. */
int orqcu_np_and_b(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z);
int orqcu_np_multiply_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                        void* const* z);
/* b2a_bit (beaver_2pc.h:147-158, dalskov_4pc.h:562-590): LSB of a boolean
 * sharing to an arithmetic one, one fused launch; y must not alias x. */
int orqcu_np_b2a_bit(orqcu_runtime* rt, int width, size_t n, const void* const* x, void* const* y);
/* xor_b / add_a / sub_a: local on every share. */
int orqcu_np_xor_b(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z);
int orqcu_np_add_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z);
int orqcu_np_sub_a(orqcu_runtime* rt, int width, size_t n, const void* const* x, const void* const* y,
                   void* const* z);

/* ---- One party of replicated 3PC beside CPU parties ---------------------------
 * A party runtime plays ONE party p of Replicated_3PC: it holds p's two
 * shares x[0] = S[p], x[1] = S[p+1] and only the keys p holds, and each entry
 * computes p's local step of a primitive; the exchange that follows is the
 * caller's, over its own communicator (the NoCopy wire format of
 * core/communication/no_copy_communicator/no_copy_communicator.h:120-266 is
 * raw little-endian arrays; include/orq_b200/nocopy.hpp speaks it), so a GPU
 * party runs with CPU parties of the reference. Party runtimes refuse the
 * all-party entries above and those refuse a party runtime (ORQCU_EINVAL). */
int orqcu_party_runtime_create(int party, int device, orqcu_runtime** out);
/* The keys of setup_random_generation (backend/common/rand_setup.h:306-381)
 * that party p holds, as 32-byte AES-256 keys: */
enum {
    ORQCU_PKEY_LOCAL = 0, /* the local PRG (secret_share on the data owner) */
    ORQCU_PKEY_NEXT = 1,  /* p's pairwise key, sent to p+1 (zero sharing get(+1)) */
    ORQCU_PKEY_PREV = 2,  /* the pairwise key received from p-1 (get(-1)) */
    ORQCU_PKEY_G01 = 3,   /* group PRGs of the groups p belongs to */
    ORQCU_PKEY_G02 = 4,
    ORQCU_PKEY_G12 = 5,
    ORQCU_PKEY_G012 = 6
};
int orqcu_party_set_key(orqcu_runtime* rt, int slot, const uint8_t key[32]);
/* The deterministic key generator of reproducible runs (AESPRGAlgorithm::
 * aesKeyGen, prg/prg_algorithm.h:192-197, replaced by SplitMix64 of seed,
 * party and the party's keygen-call index; call 0 is the local PRG). A
 * deployment draws keys from the OS instead. */
int orqcu_keygen(uint64_t seed, int party, int call, uint8_t key[32]);
/* secret_share_b / secret_share_a on the data owner (replicated_3pc.h:401-448):
 * writes the three shares, s[j] = S[j]; the owner keeps (S[p], S[p+1]), sends
 * (S[p+1], S[p+2]) to p+1 and (S[p+2], S[p]) to p+2. */
int orqcu_party_secret_share(orqcu_runtime* rt, int arith, int width, size_t n, const void* data_dev,
                             void* const s[3]);
/* and_b / multiply_a (replicated_3pc.h:44-67,166-191): z = p's new share,
 * before the exchange (send z to p-1, receive S[p+1] from p+1). */
int orqcu_party_and_b(orqcu_runtime* rt, int width, size_t n, const void* const x[2], const void* const y[2],
                      void* z);
int orqcu_party_multiply_a(orqcu_runtime* rt, int width, size_t n, const void* const x[2],
                           const void* const y[2], void* z);
/* b2a_bit (replicated_3pc.h:220-251) in two local steps around the exchange
 * of s0 and s1 (each: send to p-1, receive from p+1): pre writes p's s0, s1;
 * post takes both exchanged pairs and writes p's share of (s0 - s1)^2 before
 * the final exchange. */
int orqcu_party_b2a_pre(orqcu_runtime* rt, int width, size_t n, const void* const x[2], void* s0, void* s1);
int orqcu_party_b2a_post(orqcu_runtime* rt, int width, size_t n, const void* const s0[2],
                         const void* const s1[2], void* z);
/* xor_b / add_a / sub_a on both local shares (op 0, 1, 2). */
int orqcu_party_local(orqcu_runtime* rt, int op, int width, size_t n, const void* const x[2],
                      const void* const y[2], void* const z[2]);
/* open_shares_b / open_shares_a (replicated_3pc.h:310-330) after sending x[1]
 * to p-1 and receiving `third` (S[p+2]) from p+1. */
int orqcu_party_open(orqcu_runtime* rt, int arith, int width, size_t n, const void* const x[2],
                     const void* third, void* out_dev);

#ifdef __cplusplus
}
#endif
#endif /* ORQ_CUDA_H */
