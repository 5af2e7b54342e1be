/* afhe.h -- C ABI of the B200-native CKKS evaluation core.
 *
 * Drop-in for the accelerator path of iheydardoost/ANNS_FHE:
 *   * afhe_dispatch() replaces the kernel ABI `extern "C" fhe_accel_top(...)`
 *     (hardware_fpga_model/hls/src/fhe_accel_top.h:6-56, op codes
 *     hardware_fpga_model/hls/src/hls_params.h:18-26) with identical op
 *     semantics over identical 64-bit word offsets into poly_gmem / key_gmem;
 *   * afhe_eval_*() replace the composite operators of FHEHostDriver
 *     (cpp_host_model/src/fhe_host_driver.h:78-110) with the same argument
 *     order (c0/c1 offsets separately, then a limb count);
 *   * the arenas replace SimMemoryBus (cpp_host_model/src/sim_memory_bus.h:10-34):
 *     they live in device memory (HBM) and are addressed in 64-bit words.
 *
 * Conventions: plain pointers and sizes only; every function returns an
 * afhe_status and never throws; work is queued on the context's CUDA stream
 * and ordered; afhe_sync() waits for it. One context is not safe to drive from
 * two host threads at once; separate contexts are independent.
 */
#ifndef AFHE_H
#define AFHE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AFHE_MAX_Q 64      /* Q primes (reference: 15 limbs total, hls_params.h:8) */
#define AFHE_MAX_P 16      /* P primes (reference: 4) */
#define AFHE_MAX_PARTS 16  /* key-switch digits (reference: 3) */

typedef enum afhe_status {
    AFHE_OK = 0,
    AFHE_E_ARG = 1,      /* malformed argument (bad op code, limb count, prime mismatch) */
    AFHE_E_RANGE = 2,    /* offset + length outside an arena (sim_memory_bus.cpp:13-15) */
    AFHE_E_NOKEY = 3,    /* no rotation key for a step (fhe_host_driver.cpp:337-339) */
    AFHE_E_LEVEL = 4,    /* level unsupported by the loaded tables / key */
    AFHE_E_BUDGET = 5,   /* admission budget exceeded */
    AFHE_E_TIMEOUT = 6,  /* a bounded device wait gave up */
    AFHE_E_CUDA = 7,     /* CUDA runtime error (message via afhe_last_error) */
    AFHE_E_STATE = 8     /* call order violated (e.g. op before context load) */
} afhe_status;

/* Op codes: hardware_fpga_model/hls/src/hls_params.h:18-26 */
#define AFHE_OP_NTT 1u
#define AFHE_OP_INTT 2u
#define AFHE_OP_POLY_ADD 3u
#define AFHE_OP_POLY_SUB 4u
#define AFHE_OP_POLY_MUL_NTT 5u
#define AFHE_OP_AUTOMORPHISM 6u
#define AFHE_OP_KEY_SWITCH 7u
#define AFHE_OP_RESCALE 8u
#define AFHE_OP_LOAD_CONTEXT 99u

typedef struct afhe_ctx afhe_ctx;

/* Parameters of a context. Replaces FHEContextConfig
 * (cpp_host_model/src/fhe_host_driver.h:17-53) as a runtime value. */
typedef struct afhe_params {
    uint32_t log_n;            /* ring degree N = 2^log_n, 10 <= log_n <= 16 */
    uint32_t num_q;            /* L, Q primes (ciphertext limbs at the top level) */
    uint32_t num_p;            /* K, special primes */
    uint32_t alpha;            /* Q limbs per key-switch digit */
    uint64_t q[AFHE_MAX_Q];    /* Q chain, q[0] first; each q == 1 mod 2N, < 2^61 */
    uint64_t p[AFHE_MAX_P];    /* P chain */
    uint64_t poly_words;       /* poly_gmem size in 64-bit words */
    uint64_t key_words;        /* key_gmem size in 64-bit words */
    int32_t device;            /* CUDA device ordinal */
    uint32_t max_batch;        /* ciphertexts per batched launch (context scratch lanes);
                                  0 selects 64 */
    /* Primitive 2N-th root per prime behind the twiddles (tw[j] = psi^bitrev(j));
     * 0 selects the smallest root. A package's own roots (its tw[N/2]) make
     * every NTT match the package's evaluation-form data. */
    uint64_t psi_q[AFHE_MAX_Q];
    uint64_t psi_p[AFHE_MAX_P];
} afhe_params;

/* Scalar and array registers of fhe_accel_top (fhe_accel_top.h:8-55), with
 * offsets widened to 64 bits, ap_uint<128> Barrett constants split into
 * (lo, hi) words, and up to AFHE_MAX_PARTS base-conversion table offsets. */
typedef struct afhe_accel_args {
    uint32_t op_code;
    uint32_t active_limbs;
    uint64_t src_a_offset, src_b_offset, dst_offset;
    uint64_t evk_offset;
    uint32_t prime_idx, galois_elt;         /* unused, as in the reference */
    uint32_t sizeQl, sizeP, numPartQ, alpha;
    uint64_t rns_primes[AFHE_MAX_Q];
    uint64_t p_primes[AFHE_MAX_P];
    uint64_t barrett_m_q_lo[AFHE_MAX_Q], barrett_m_q_hi[AFHE_MAX_Q];
    uint32_t barrett_k_q[AFHE_MAX_Q];
    uint64_t barrett_m_p_lo[AFHE_MAX_P], barrett_m_p_hi[AFHE_MAX_P];
    uint32_t barrett_k_p[AFHE_MAX_P];
    uint64_t n_inv_q[AFHE_MAX_Q];
    uint64_t n_inv_p[AFHE_MAX_P];
    uint64_t n_inv_mod_q_last;
    uint64_t twiddles_q_offset, inv_twiddles_q_offset, twiddles_p_offset, inv_twiddles_p_offset;
    uint64_t qhat_inv_offset[AFHE_MAX_PARTS];   /* qHatInvModq_j_offset */
    uint64_t qhat_modp_offset[AFHE_MAX_PARTS];  /* qHatModp_j_offset */
    uint64_t p_inv_mod_q_offset, p_hat_inv_mod_p_offset, p_hat_mod_q_offset;
    uint64_t qlql_offset, qlinv_offset;         /* QlQlInvModqlDivqlModq, qlInvModq */
} afhe_accel_args;

/* Where afhe_ctx_write_context_tables() put the context tables in key_gmem.
 * Same arrangement as FHEHostDriver::initialize_context_from_directory
 * (fhe_host_driver.cpp:46-86): twiddles Q then P from word 0, inverse twiddles
 * after them, CRT tables in 64-word-aligned slots, keys 512-word aligned after. */
typedef struct afhe_context_layout {
    uint64_t twiddles_q_offset, inv_twiddles_q_offset, twiddles_p_offset, inv_twiddles_p_offset;
    uint64_t qhat_inv_offset[AFHE_MAX_PARTS];
    uint64_t qhat_modp_offset[AFHE_MAX_PARTS];
    uint64_t p_inv_mod_q_offset, p_hat_inv_mod_p_offset, p_hat_mod_q_offset;
    uint64_t qlql_offset, qlinv_offset;
    uint64_t first_free_offset;   /* 512-word aligned: where keys may start */
    uint32_t level;               /* the sizeQl the tables were written for */
    uint32_t num_parts;
} afhe_context_layout;

/* One ciphertext in poly_gmem for the batched entry points. */
typedef struct afhe_ct_ref {
    uint64_t c0_offset;
    uint64_t c1_offset;
} afhe_ct_ref;

/* ---- host-only number theory (no GPU needed) ------------------------------ */
/* Replaces OpenFHE's parameter generation used by
 * integration_tools/test_vector_generator.cpp:80-177. */
int afhe_find_ntt_primes(uint32_t log_n, uint32_t bits, uint32_t count,
                         const uint64_t* exclude, uint32_t n_exclude, uint64_t* out);
uint64_t afhe_min_primitive_root(uint32_t log_n, uint64_t q);
int afhe_gen_twiddles(uint32_t log_n, uint64_t q, uint64_t psi, uint64_t* tw, uint64_t* itw);
void afhe_barrett_constant(uint64_t q, uint64_t* m_lo, uint64_t* m_hi, uint32_t* k);
uint64_t afhe_inv_mod(uint64_t a, uint64_t q);
/* FindAutomorphismIndex (generate_interactive_test_vectors.cpp:297) */
uint32_t afhe_galois_elt(uint32_t log_n, int32_t step);
/* AutomorphismTransform's evaluation-form permutation (test_vector_generator.cpp:262-288) */
int afhe_automorphism_map(uint32_t log_n, uint32_t galois_elt, uint32_t* map);
/* GetPartQlHatInvModq / GetPartQlHatModp (test_vector_generator.cpp:438-463) */
int afhe_part_qhat_tables(const uint64_t* q, uint32_t sizeQl, uint32_t alpha, uint32_t part,
                          const uint64_t* p, uint32_t num_p, uint64_t* qhat_inv, uint64_t* qhat_modp);
/* GetPInvModq / GetPHatInvModp / GetPHatModq (test_vector_generator.cpp:473-494) */
int afhe_moddown_tables(const uint64_t* q, uint32_t sizeQl, const uint64_t* p, uint32_t num_p,
                        uint64_t* p_inv_mod_q, uint64_t* p_hat_inv_mod_p, uint64_t* p_hat_mod_q);
/* GetQlQlInvModqlDivqlModq / GetqlInvModq (test_vector_generator.cpp:309-310) */
int afhe_rescale_tables(const uint64_t* q, uint32_t sizeQl, uint64_t* qlql, uint64_t* qlinv);

const char* afhe_status_string(int status);
const char* afhe_last_error(void);

/* ---- context and arenas --------------------------------------------------- */
/* Replaces SimMemoryBus construction (sim_memory_bus.cpp:5-10) plus the
 * FHEHostDriver constructor: allocates poly_gmem / key_gmem in HBM and builds
 * the per-prime and per-level device tables for the parameter set. */
int afhe_ctx_create(const afhe_params* params, afhe_ctx** out);
int afhe_ctx_destroy(afhe_ctx* ctx);
int afhe_sync(afhe_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t) and arena base device pointers. */
void* afhe_stream(afhe_ctx* ctx);
uint64_t* afhe_poly_gmem(afhe_ctx* ctx);
uint64_t* afhe_key_gmem(afhe_ctx* ctx);
/* Words of context-private device scratch (max_batch lanes) allocated after
 * poly_gmem; no counterpart in the reference (its composites use fixed
 * SCRATCH_* slots inside poly_gmem, fhe_host_driver.h:63-69). */
uint64_t afhe_scratch_words(afhe_ctx* ctx);

/* SimMemoryBus::write_poly / read_poly / write_key / read_key
 * (sim_memory_bus.cpp:12-62): host <-> arena word copies (synchronous). */
int afhe_write_poly(afhe_ctx* ctx, uint64_t word_offset, const uint64_t* src, uint64_t count);
int afhe_read_poly(afhe_ctx* ctx, uint64_t word_offset, uint64_t* dst, uint64_t count);
int afhe_write_key(afhe_ctx* ctx, uint64_t word_offset, const uint64_t* src, uint64_t count);
int afhe_read_key(afhe_ctx* ctx, uint64_t word_offset, uint64_t* dst, uint64_t count);
/* Asynchronous variants on the context stream; host buffers should be pinned. */
int afhe_write_poly_async(afhe_ctx* ctx, uint64_t word_offset, const uint64_t* src, uint64_t count);
int afhe_read_poly_async(afhe_ctx* ctx, uint64_t word_offset, uint64_t* dst, uint64_t count);
int afhe_copy_poly(afhe_ctx* ctx, uint64_t dst_offset, uint64_t src_offset, uint64_t count);
/* Run-time options of a context (no counterpart in the reference; the
 * autotuner, anns_fhe_b200/autotune.py, picks them per GPU and parameter set):
 *   AFHE_OPT_KS_FUSED  1: the one-kernel key switch (one CTA per ciphertext
 *                      at N <= 2^13, a cluster of N / 2^13 CTAs above), 0: the
 *                      multi-kernel pipeline. Same residues either way.
 *   AFHE_OPT_CHUNK     ciphertexts per launch of a batched call, 1..lanes
 *                      (0: all lanes). Same residues for any value. */
#define AFHE_OPT_KS_FUSED 1u
#define AFHE_OPT_CHUNK 2u
/*   AFHE_OPT_FUSED_MIN launches of fewer ciphertexts than this take the
 *                      multi-kernel key switch even where the one-kernel path
 *                      is on (it carries one ciphertext per CTA, or per
 *                      cluster above N = 2^13, so a small launch leaves most
 *                      SMs idle). Default: half a wave of SMs. Same residues. */
#define AFHE_OPT_FUSED_MIN 3u
/*   AFHE_OPT_KS_CAPACITY (read only) ciphertexts the one-kernel key switch
 *                      runs at once on this GPU (CTAs, or clusters above
 *                      N = 2^13, resident together): a launch of a multiple
 *                      of it fills its waves; 0 where it cannot run. */
#define AFHE_OPT_KS_CAPACITY 4u
/*   AFHE_OPT_KS_EPT    values per thread of the one-kernel key switch: 8
 *                      (N / 8 threads per CTA slice, the default) or 16 (half
 *                      the threads, twice the registers each). Same residues. */
#define AFHE_OPT_KS_EPT 5u
/*   AFHE_OPT_KS_SLICE  log2 of the slice each CTA of a cluster holds in the
 *                      one-kernel key switch at N = 2^14 and 2^15: 13 (the
 *                      default: clusters of N / 2^13 CTAs of 1024 threads, one
 *                      per SM) or 12 (clusters of N / 2^12 CTAs, two per SM:
 *                      512 threads with 8 values each, or 256 threads with 16
 *                      values each in radix-16 rounds). Ignored at other N.
 *                      Same residues. */
#define AFHE_OPT_KS_SLICE 6u
int afhe_ctx_set_option(afhe_ctx* ctx, uint32_t option, int64_t value);
int afhe_ctx_get_option(afhe_ctx* ctx, uint32_t option, int64_t* value);
/* Page-locked host memory for the transfers above (the reference's host
 * buffers are std::vectors; pinned ones let copies run at full PCIe speed).
 * afhe_host_free releases what afhe_host_alloc returned. No counterpart in
 * the reference. */
int afhe_host_alloc(uint64_t bytes, void** out);
int afhe_host_free(void* p);
/* Gather `rows` rows of `row_words` words, row r at word_offset + r * stride,
 * into dst (rows * row_words words, packed), in one copy; synchronous. Reads
 * one limb of many result ciphertexts, e.g. limb 0 of each, which is all a
 * client needs to decrypt a message smaller than q_0 / 2. Replaces the
 * reference host's word-by-word read-back of results from poly_gmem
 * (SimMemoryBus, sim_memory_bus.h:10-34). */
int afhe_read_poly_rows(afhe_ctx* ctx, uint64_t word_offset, uint64_t stride, uint64_t rows,
                        uint64_t row_words, uint64_t* dst);
/* afhe_read_poly_rows enqueued on the context's stream without waiting: dst
 * (page-locked, e.g. from afhe_host_alloc, for the copy to overlap) holds the
 * rows once a fence issued after this call has been waited on. Lets a client
 * take the results of one group of queries while the server works on the
 * next; the reference host reads results synchronously (sim_memory_bus.h:10-34). */
int afhe_read_poly_rows_async(afhe_ctx* ctx, uint64_t word_offset, uint64_t stride, uint64_t rows,
                              uint64_t row_words, uint64_t* dst);
/* Fences on the context's stream: afhe_fence marks all work enqueued so far;
 * afhe_fence_wait blocks the host until that work has finished. No reference
 * counterpart: the reference's accelerator call returns when the operation is
 * done (fhe_host_driver.cpp:177-204 calls fhe_accel_top synchronously). */
int afhe_fence(afhe_ctx* ctx, uint64_t* fence);
int afhe_fence_wait(afhe_ctx* ctx, uint64_t fence);

/* Writes the context tables for level `level` (twiddles for all Q and P primes,
 * CRT tables for that level) into key_gmem in the reference's arrangement and
 * reports the offsets (FHEHostDriver::initialize_context_from_directory,
 * fhe_host_driver.cpp:18-86). */
int afhe_ctx_write_context_tables(afhe_ctx* ctx, uint32_t level, afhe_context_layout* out);

/* ---- kernel ABI ------------------------------------------------------------ */
/* fhe_accel_top (fhe_accel_top.cpp:90-328): one op over the arenas. OP 99 copies
 * the tables named by the offsets from key_gmem into the context (the reference
 * keeps them in static on-chip arrays); ops 1-8 use those loaded tables.
 * Ops 1-8 allocate nothing and do not wait: they are enqueued on the context's
 * stream in call order (their small per-call descriptors go through pinned
 * staging) and return; afhe_read_poly / afhe_read_key / afhe_sync wait for
 * them. The reference's fhe_accel_top returns when the op is done; a caller
 * that reads the device arenas by other means calls afhe_sync first. OP 99,
 * a one-time set-up, waits for its copies. */
int afhe_dispatch(afhe_ctx* ctx, const afhe_accel_args* args);

/* ---- key directory (FHEHostDriver m_cfg.relin_key_offset / m_rot_keys) ---- */
/* Keys are stored at full level: [a_0 .. a_{d-1}][b_0 .. b_{d-1}], each digit
 * (L + K) * N words, d = ceil(L / alpha) -- the relinearisation-key layout of
 * fhe_host_driver.cpp:105-117. At level l digit j limb i reads key limb i
 * (Q limbs) or L + k (P limb k). */
int afhe_set_relin_key(afhe_ctx* ctx, uint64_t evk_offset);
/* RotationKeyMeta (fhe_host_driver.h:10-15); the map is computed here. */
int afhe_add_rotation_key(afhe_ctx* ctx, int32_t step, uint64_t evk_offset);
int afhe_has_rotation_key(afhe_ctx* ctx, int32_t step);

/* ---- composite operators (FHEHostDriver, fhe_host_driver.cpp:248-404) ---- */
/* The primitives (afhe_ntt .. afhe_automorphism) also accept polynomials over
 * all L + K primes (Q limbs, then P limbs), as key generation needs; the
 * ciphertext operators take 1..L limbs. */
int afhe_ntt(afhe_ctx* ctx, uint64_t src, uint64_t dst, uint32_t limbs);
int afhe_intt(afhe_ctx* ctx, uint64_t src, uint64_t dst, uint32_t limbs);
int afhe_poly_add(afhe_ctx* ctx, uint64_t a, uint64_t b, uint64_t dst, uint32_t limbs);
int afhe_poly_sub(afhe_ctx* ctx, uint64_t a, uint64_t b, uint64_t dst, uint32_t limbs);
int afhe_poly_mul_ntt(afhe_ctx* ctx, uint64_t a, uint64_t b, uint64_t dst, uint32_t limbs);
int afhe_automorphism(afhe_ctx* ctx, uint64_t src, uint32_t galois_elt, uint64_t dst, uint32_t limbs);
/* FHEHostDriver::automorphism with its own arguments (fhe_host_driver.h:82):
 * the permutation is read from poly_gmem at auto_map_offset (N 32-bit source
 * indices, two per word, as initialize_context_from_directory stores them,
 * fhe_host_driver.cpp:141-154); galois_elt is not used, as in the reference
 * (OP 6, fhe_accel_top.cpp:272-281). In place is allowed. */
int afhe_automorphism_from_map(afhe_ctx* ctx, uint64_t src, uint64_t auto_map_offset, uint64_t dst, uint32_t limbs,
                               uint32_t galois_elt);
/* rescale c0 and c1 from `limbs` to `limbs - 1` (fhe_host_driver.cpp:362-365) */
int afhe_rescale(afhe_ctx* ctx, uint64_t c0_in, uint64_t c1_in, uint64_t c0_out, uint64_t c1_out,
                 uint32_t limbs);
/* key switch one polynomial with the key at evk_offset (full-level layout):
 * writes ks0 (sum digit * b) to dst_c0 and ks1 (sum digit * a) to dst_c1 */
int afhe_key_switch(afhe_ctx* ctx, uint64_t src, uint64_t evk_offset, uint64_t dst_c0,
                    uint64_t dst_c1, uint32_t limbs);

int afhe_eval_add(afhe_ctx* ctx, uint64_t a_c0, uint64_t a_c1, uint64_t b_c0, uint64_t b_c1,
                  uint64_t dst_c0, uint64_t dst_c1, uint32_t limbs);
int afhe_eval_sub_plain(afhe_ctx* ctx, uint64_t a_c0, uint64_t a_c1, uint64_t pt,
                        uint64_t dst_c0, uint64_t dst_c1, uint32_t limbs);
int afhe_eval_mult_relin_rescale(afhe_ctx* ctx, uint64_t a_c0, uint64_t a_c1, uint64_t b_c0,
                                 uint64_t b_c1, uint64_t dst_c0, uint64_t dst_c1, uint32_t in_limbs);
int afhe_eval_mult_plain_rescale(afhe_ctx* ctx, uint64_t a_c0, uint64_t a_c1, uint64_t pt,
                                 uint64_t dst_c0, uint64_t dst_c1, uint32_t in_limbs);
int afhe_eval_rotate_single_step(afhe_ctx* ctx, uint64_t in_c0, uint64_t in_c1, uint64_t dst_c0,
                                 uint64_t dst_c1, int32_t step, uint32_t limbs);
int afhe_eval_rotate(afhe_ctx* ctx, uint64_t in_c0, uint64_t in_c1, uint64_t dst_c0,
                     uint64_t dst_c1, int32_t total_rot, uint32_t limbs);

/* Key switch with no allocation at call time (no counterpart in the
 * reference). For callers that cannot call cudaMalloc on their request path:
 * applications whose device memory already belongs to their own pool
 * allocator, or latency-bound threads that cannot take the synchronisation
 * cudaMalloc / cudaFree may cause. Same result as afhe_key_switch.
 *   io: device pointer to 3 * limbs * N words: the input polynomial, then ks0
 *       (sum digit * b), then ks1 (sum digit * a); the caller owns it.
 *   evk_offset: the key in key_gmem (full-level layout, as afhe_key_switch).
 * Working memory is a fixed 16 MiB array of static device memory in this
 * library (held on every GPU that loads it until exit); parameter sets whose
 * key switch needs more return AFHE_E_BUDGET. afhe_ctx_create loads that array
 * on the context's device and looks up its address (cudaGetSymbolAddress), so
 * the entry point itself neither allocates nor loads anything: create the
 * context before a pool allocator takes the GPU's memory. All calls on a
 * device share the array: calls that overlap on the GPU race and must be
 * ordered by the caller. It always runs the multi-kernel key switch (slower
 * than afhe_key_switch's one-kernel path at N <= 2^13, same residues), and it
 * leaves the caller's current device as it found it. */
int afhe_key_switch_noalloc(afhe_ctx* ctx, uint64_t* io, uint64_t evk_offset, uint32_t limbs);

/* ---- batched composite operators ------------------------------------------ */
/* The same operator applied to `count` independent ciphertexts in one pass of
 * launches; each output is bit-identical to the one-at-a-time call. */
int afhe_eval_mult_relin_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b,
                                       const afhe_ct_ref* dst, uint32_t count, uint32_t in_limbs);
int afhe_eval_rotate_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* dst,
                           uint32_t count, int32_t total_rot, uint32_t limbs);
/* In-place forward (inverse = 0) or inverse NTT of `count` polynomials of
 * `limbs` limbs each (limb i under prime i, Q then P), one launch per pass. */
int afhe_ntt_batch(afhe_ctx* ctx, const uint64_t* polys, uint32_t count, uint32_t limbs, int inverse);
/* Client-side decryption of `count` ciphertexts at `limbs` limbs with the
 * secret key s (evaluation form) at s_offset: writes INTT(c0 + c1 * s), the
 * plaintext's coefficients mod each q_i, to out_offset + i * limbs * N.
 * Replaces the arithmetic of OpenFHE's Decrypt
 * (generate_interactive_test_vectors.cpp:443-447); decoding is the caller's. */
int afhe_decrypt_batch(afhe_ctx* ctx, const afhe_ct_ref* cts, uint32_t count, uint64_t s_offset,
                       uint64_t out_offset, uint32_t limbs);
/* NTT tile shapes ("plans"), per ring degree 2^log_n, process-wide (every
 * context of that degree, from the next launch). Plans change only launch
 * shapes; every plan gives the same residues. N <= 2^13 (one pass over the
 * limb): 2 plans, values per thread 8 or 16. N >= 2^14 (two passes): 6 plans,
 * columns per CTA of the column pass (16, 8, 32) x words per tile of the
 * chunk pass (4096, 8192). Plan 0 is the default. The autotuner
 * (anns_fhe_b200/autotune.py) times them. The one-kernel key switch has its
 * own transform and ignores the plan. */
int afhe_ntt_plan_count(uint32_t log_n, uint32_t* count);
int afhe_ntt_plan_describe(uint32_t log_n, uint32_t plan, char* buf, uint32_t len);
int afhe_ntt_set_plan(uint32_t log_n, uint32_t plan);
int afhe_ntt_get_plan(uint32_t log_n, uint32_t* plan);
/* Kernels launched by this library so far (host-side count, all contexts). */
uint64_t afhe_kernel_launches(void);
/* acc[i] = acc[i] + rotate(in[i], total_rot), bit-identical to eval_rotate
 * into a temporary followed by eval_add; in[i] may equal acc[i] (the
 * rotate-and-sum step x += rot(x)). The last rotation step's key switch adds
 * into acc in its epilogue. */
int afhe_eval_rotate_accumulate_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* acc,
                                      uint32_t count, int32_t total_rot, uint32_t limbs);
/* afhe_eval_rotate_accumulate_batch for ciphertexts at different levels:
 * acc[i] = acc[i] + rotate(in[i], total_rot), each at levels[i] limbs, in one
 * launch per rotation step (the one-kernel key switch reads each entry's
 * level's tables; without it, or when entries' outputs overlap other
 * entries' inputs, one launch sequence per level). Each result equals the
 * single-level call's. The reference runs one ciphertext at a time
 * (fhe_host_driver.cpp:361-404, then eval_add :248-257). */
int afhe_eval_rotate_accumulate_levels_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* acc,
                                             const uint32_t* levels, uint32_t count, int32_t total_rot);
int afhe_eval_add_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* dst,
                        uint32_t count, uint32_t limbs);
/* dst[i] = eval_rotate_single_step(in[i], steps[i]) (fhe_host_driver.cpp:
 * 331-359): every ciphertext rotated by its own step, with that step's
 * registered key, in one launch sequence. Each step is applied as a single
 * key switch, however many bits it has (eval_rotate would split it into
 * powers of two). dst[i] may alias in[i]. */
int afhe_eval_rotate_steps_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* dst,
                                 const int32_t* steps, uint32_t count, uint32_t limbs);
/* dst[i] = the Galois automorphism galois[i] of the polynomial src[i] (`limbs`
 * limbs, evaluation form): a permutation of its coefficients in each limb, the
 * same gather afhe_automorphism applies, for many polynomials and elements in
 * one launch. On a plaintext it rotates the slots: the automorphism of an
 * encoded vector is the encoding of the rotated vector, exactly (a signed
 * permutation of the rounded coefficients). No destination may overlap a
 * source. Maps are computed on first use of an element and kept. */
int afhe_automorphism_batch(afhe_ctx* ctx, const uint64_t* src, const uint32_t* galois, const uint64_t* dst,
                            uint32_t count, uint32_t limbs);
/* Sums of plaintext-ciphertext products, each plaintext moved by its own
 * Galois automorphism: the inner products of the diagonal (baby-step
 * giant-step) method, sum_i diag_i * rot(ct, i). Each term is the two
 * poly_mul_ntt products eval_mult_plain_rescale makes before its rescale
 * (fhe_host_driver.cpp:308-317) with the plaintext first moved by
 * FHEHostDriver::automorphism (:230-232); the terms are summed as eval_add
 * does (:248-257). For each output j:
 *   out[j] (+)= sum over groups g in [first_group[j], first_group[j + 1]) of
 *               sum over terms t of g: automorphism(terms[t].pt, terms[t].galois) * groups[g].src
 * (both polynomials, `limbs` limbs, evaluation form; galois 1 is the identity;
 * a group whose src.c0_offset is AFHE_MAC_UNIT multiplies by the constant
 * ciphertext (1, 0), i.e. adds its plaintexts to c0). The sums are reduced
 * once, so the result is the exact residue of the sum of products: equal to
 * eval_mult_plain without rescale on every term and eval_add of them all.
 * With accumulate the existing out is added. No output may overlap another
 * output or any operand. first_group has count + 1 entries. */
#define AFHE_MAC_UNIT UINT64_MAX
typedef struct afhe_mac_term {
    uint64_t pt;        /* plaintext polynomial offset in poly_gmem */
    uint32_t galois;    /* odd, < 2N; 1: no automorphism */
    uint32_t reserved;
} afhe_mac_term;
typedef struct afhe_mac_group {
    afhe_ct_ref src;     /* the ciphertext the group's plaintexts multiply */
    uint32_t first_term, n_terms;
} afhe_mac_group;
int afhe_eval_mac_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* out, const uint32_t* first_group, uint32_t count,
                              const afhe_mac_group* groups, const afhe_mac_term* terms, uint32_t limbs,
                              uint32_t accumulate);
/* The diagonal method's inner products in a fixed shape, the form the
 * diagonal chain issues: for output j,
 *   out[j] (+)= sum over units k in [first_unit[j], first_unit[j + 1]) of
 *               sum over b < nb of automorphism(pt at unit_pt[k] + b pt_stride, unit_galois[k]) * src[j nb + b]
 * (nb = 1, 2, 4, 8 or 16 baby steps; a unit's nb plaintexts lie pt_stride
 * words apart). Equal to afhe_eval_mac_plain_batch with one group per baby
 * step and one term per unit; the baby-step ciphertexts stay in registers and
 * a unit's automorphism index is read once for its nb plaintexts. No output
 * may overlap another output or any operand; first_unit has count + 1 entries. */
int afhe_eval_diag_inner_batch(afhe_ctx* ctx, const afhe_ct_ref* out, uint32_t count, const afhe_ct_ref* src,
                               uint32_t nb, const uint64_t* unit_pt, const uint32_t* unit_galois,
                               const uint32_t* first_unit, uint64_t pt_stride, uint32_t limbs, uint32_t accumulate);
/* dst[i] = a[i] (both polynomials, `limbs` limbs): the slot-to-slot copies the
 * reference's host makes between operators (eval_sub_plain's c1 copy,
 * fhe_host_driver.cpp:259-270), for many ciphertexts in one launch. */
int afhe_eval_copy_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* dst, uint32_t count,
                         uint32_t limbs);
/* dst[i] = a[i] - b[i] (both polynomials) */
int afhe_eval_sub_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* dst,
                        uint32_t count, uint32_t limbs);
/* dst[i] = a[i] + pt[i] (c0 + pt, c1 copied), the add counterpart of eval_sub_plain */
int afhe_eval_add_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* dst,
                              uint32_t count, uint32_t limbs);
/* pt[i] is the plaintext polynomial offset for ciphertext i */
int afhe_eval_sub_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* dst,
                              uint32_t count, uint32_t limbs);
int afhe_eval_mult_plain_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt,
                                       const afhe_ct_ref* dst, uint32_t count, uint32_t in_limbs);
/* Rescale of `count` ciphertexts, in_limbs -> in_limbs - 1: OP 8 (RESCALE) on
 * c0 and c1 of each (fhe_accel_top.cpp:286-292, FHEHostDriver::rescale at
 * fhe_host_driver.cpp:239-242), with this level's tables. dst may alias a. */
int afhe_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* dst, uint32_t count,
                       uint32_t in_limbs);

/* ---- server-side plaintext encoding ---------------------------------------- */
/* CKKS encoding of `count` real slot vectors on the device: row i of `values`
 * (host, count x slots doubles, row-major; slots <= N/2, the rest zero) at
 * `scale` into the evaluation-form polynomial at pt[i] (level limbs). The
 * server's plaintexts of the reference are OpenFHE's MakeCKKSPackedPlaintext
 * (fhe_core/fhe_searcher.cpp:334-368; centroids and masks in
 * integration_tools/generate_interactive_test_vectors.cpp:461-521). Slot j is
 * the value at the root exp(i pi 5^j / N); the inverse embedding is a
 * double-precision special FFT, coefficients rounded to nearest (equal to the
 * exactly rounded ones but where a value lies within the transform's
 * rounding error of a half-integer). AFHE_E_ARG if a coefficient reaches
 * 2^62. */
int afhe_encode_batch(afhe_ctx* ctx, const double* values, uint32_t count, uint32_t slots, double scale,
                      uint32_t level, const uint64_t* pt);
/* An IVF-PQ index held in device memory, to build the dimension-major
 * candidate plaintexts of stage 3 there (fhe_searcher.cpp:334-368): candidate
 * = the centroid of its list + its PQ codewords (residual PQ). */
typedef struct afhe_pq_index {
    uint32_t n_list, d, M, K;     /* M sub-quantizers of d / M components, K codewords each (<= 256) */
    uint64_t n;                   /* vectors */
    const float* centroids;       /* n_list x d */
    const float* codebooks;       /* M x K x (d / M) */
    const uint8_t* codes;         /* n x M */
    const uint32_t* assignments;  /* n: the list of each vector */
} afhe_pq_index;
typedef struct afhe_pq afhe_pq;
/* The client's decoding on the device, the inverse of afhe_encode_batch's
 * transform: polynomial i (coefficient form, e.g. afhe_decrypt_batch's
 * output, limb 0 at poly_gmem offset coef[i], centred mod q_0 < 2^53) to the
 * real parts of slots 0 .. slots - 1, m(zeta^(5^j)) / scales[i], into host
 * `out` (count x slots doubles, row-major; page-locked memory copies
 * fastest). Double-precision special FFT; the reference's client decodes
 * with OpenFHE (Decrypt + GetRealPackedValue,
 * fhe_core/fhe_context_manager.cpp:505-507). */
int afhe_decode_batch(afhe_ctx* ctx, const uint64_t* coef, const double* scales, uint32_t count, uint32_t slots,
                      double* out);
int afhe_pq_create(afhe_ctx* ctx, const afhe_pq_index* index, afhe_pq** out);
int afhe_pq_destroy(afhe_pq* pq);
/* Batch b: candidates vids[first[b] .. first[b] + count[b]) (count <= N / 2d);
 * slot d' B + j (B = N / 2d) = component d' of candidate j, 0 past the count;
 * encoded as afhe_encode_batch does into pt[b]. */
int afhe_pq_encode_batches(afhe_pq* pq, const uint32_t* vids, const uint32_t* first, const uint32_t* count,
                           uint32_t batches, double scale, uint32_t level, const uint64_t* pt);
/* The same batches' squared norms: slot d' B + j = ||x_j||^2 in every row d',
 * 0 past the count (the term the expanded distance ||q||^2 - 2 <q, x_j> +
 * ||x_j||^2 adds after the tree sum). */
int afhe_pq_encode_norms(afhe_pq* pq, const uint32_t* vids, const uint32_t* first, const uint32_t* count,
                         uint32_t batches, double scale, uint32_t level, const uint64_t* pt);
/* The diagonal method's plaintexts of `units` units of up to N/2 candidates
 * (unit u: vids[first[u] .. first[u] + count[u])): pt[u dim + i], i = g n1 + b
 * (n1 divides dim), slot k = coef x_j[(j + i) mod dim] with j = (k - n1 g)
 * mod N/2 the unit's candidate, 0 past the count. The sum over i of
 * plaintext i times the query (repeated every dim slots) rotated by b, each
 * giant-step group g rotated back by n1 g, leaves coef <q, x_j> in slot j. */
int afhe_pq_encode_diagonals(afhe_pq* pq, const uint32_t* vids, const uint32_t* first, const uint32_t* count,
                             uint32_t units, uint32_t n1, double coef, double scale, uint32_t level,
                             const uint64_t* pt);
/* The units' squared norms: slot j = ||x_j||^2 of the unit's candidate j, 0
 * past the count, into pt[u]. */
int afhe_pq_encode_unit_norms(afhe_pq* pq, const uint32_t* vids, const uint32_t* first, const uint32_t* count,
                              uint32_t units, double scale, uint32_t level, const uint64_t* pt);

/* ---- encrypted IVF-PQ server stages ---------------------------------------- */
/* InteractiveQueryManager's server stages (cpp_host_model/src/
 * interactive_query_manager.cpp:85-303) for many queries at once: stage 1 +
 * 1b (coarse distances, compacted) and stage 3 (candidate distances, placed
 * in the query's result ciphertexts), each operator one batched call over up
 * to `lanes` ciphertexts. Every result ciphertext is word for word the one
 * the one-query-at-a-time chain writes. The plaintexts (centroids, index
 * batches, masks) are encoded by the caller into poly_gmem and registered by
 * offset; the handle holds offsets only. */
typedef struct afhe_ivfpq afhe_ivfpq;
typedef struct afhe_ivfpq_shape {
    uint32_t D;           /* vector dimension, a power of two */
    uint32_t n_list;      /* coarse lists */
    uint32_t slots;       /* N / 2 */
    uint32_t lanes;       /* ciphertexts per batched call, <= the context's lanes */
    uint32_t packed;      /* 0: the reference's compaction (one-hot masks, eval_rotate's
                             power-of-two steps); 1: centroids over ceil(n_list / (slots / D))
                             ciphertexts, one stride mask, one key switch per placement;
                             2: the diagonal chain (baby-step giant-step inner products,
                             afhe_ivfpq_set_units / _set_diagonals / _set_scratch) */
    uint32_t eval_level;  /* limbs the chain runs at (0: each query's own level) */
} afhe_ivfpq_shape;
typedef struct afhe_ivfpq_query {
    afhe_ct_ref ct_query;        /* the query, repeated every D slots (stage 1 input) */
    afhe_ct_ref ct_dim;          /* the query, dimension d in slots d B .. d B + B - 1 (stage 3 input);
                                    diagonal chain: ||q||^2 in every slot, encrypted by the client at the
                                    evaluation level - 1 and scale Delta^2 / q_{level-1} */
    afhe_ct_ref compact;         /* stage 1b output: the compacted coarse distances */
    afhe_ct_ref norm;            /* packed chain, stage 3 scratch (expanded distances): ||q||^2 at the level - 1 */
    const afhe_ct_ref* results;  /* stage 3 outputs, n_results ciphertexts */
    uint32_t n_results;
    uint32_t level;              /* limbs of the encrypted query (0: the top level) */
    const uint32_t* probes;      /* stage 3: the lists the client selected, in order */
    uint32_t nprobe;
    const afhe_ct_ref* baby;     /* diagonal chain: the query rotated by 1 .. n1 - 1 (stage 1 output,
                                    stage 3 input), n1 - 1 ciphertexts */
    uint32_t n_baby;
} afhe_ivfpq_query;
int afhe_ivfpq_create(afhe_ctx* ctx, const afhe_ivfpq_shape* shape, afhe_ivfpq** out);
int afhe_ivfpq_destroy(afhe_ivfpq* h);
/* One centroid plaintext per coarse ciphertext (1, or ceil(n_list D / slots) packed). */
int afhe_ivfpq_set_centroids(afhe_ivfpq* h, const uint64_t* pts, uint32_t count);
/* The compaction masks of queries evaluated at `level` limbs: n_list one-hot
 * masks (slot i D), or the one stride mask (packed). */
int afhe_ivfpq_set_level_masks(afhe_ivfpq* h, uint32_t level, const uint64_t* masks, uint32_t count);
/* The mask of the first `count` slots for queries evaluated at `level`. */
int afhe_ivfpq_set_prefix_mask(afhe_ivfpq* h, uint32_t level, uint32_t count, uint64_t pt);
/* List `list`'s candidate batches: plaintext offsets and candidates per batch. */
int afhe_ivfpq_set_list(afhe_ivfpq* h, uint32_t list, const uint64_t* pts, const uint32_t* counts,
                        uint32_t batches);
/* Working ciphertexts: work[4 j .. 4 j + 3] = lane j's diff, sq, sel and a
 * scratch slot whose c0 polynomial holds the lane's placed mask (packed
 * chain); cmp[j (n_list - 1) + i - 1] = lane j's stage-1b term i (reference
 * compaction). */
int afhe_ivfpq_set_lanes(afhe_ivfpq* h, const afhe_ct_ref* work, uint32_t lanes, const afhe_ct_ref* cmp);
/* Expanded distances for the packed chain at `level`: pts[g] is the squared
 * norms plaintext (afhe_pq_encode_norms, level - 1 limbs, scale Delta^2 /
 * q_{level-1}) of global batch g (lists in order, then their batches). With
 * them stage 3 computes ||q||^2 - 2 <q, x_j> + ||x_j||^2: ||q||^2 once per
 * query (one relinearisation into afhe_ivfpq_query.norm), a plaintext
 * product per batch instead of a square. */
int afhe_ivfpq_set_norms(afhe_ivfpq* h, uint32_t level, const uint64_t* pts, uint32_t batches);
/* Key-switch options applied around every operator the stages issue at
 * `level` limbs (afhe_ctx_set_option's AFHE_OPT_KS_FUSED, AFHE_OPT_CHUNK,
 * AFHE_OPT_KS_EPT, AFHE_OPT_KS_SLICE, AFHE_OPT_FUSED_MIN): fused -1 leaves
 * the context's setting, any other field 0 leaves it. */
typedef struct afhe_ks_options {
    int32_t fused;
    uint32_t chunk, ept, slice, fused_min;
} afhe_ks_options;
int afhe_ivfpq_set_tuning(afhe_ivfpq* h, uint32_t level, const afhe_ks_options* opts);
/* Diagonal chain (shape.packed = 2). Units: list c holds units
 * [list_first_unit[c], list_first_unit[c + 1]), unit u counts[u] candidates
 * (<= N/2); a query's units are placed in probe order at multiples of D,
 * starting a new result ciphertext where one would not fit. */
int afhe_ivfpq_set_units(afhe_ivfpq* h, const uint32_t* list_first_unit, const uint32_t* counts, uint32_t units);
/* The plaintexts of queries evaluated at `level` limbs: the centroids' D
 * diagonals from `centroids` (stride level N words) and their squared norms
 * (level - 1 limbs); per unit its D diagonals from unit_pts[u] (stride level
 * N) and its squared norms unit_norms[u] (afhe_pq_encode_diagonals,
 * afhe_pq_encode_unit_norms). */
int afhe_ivfpq_set_diagonals(afhe_ivfpq* h, uint32_t level, uint64_t centroids, uint64_t centroid_norms,
                             const uint64_t* unit_pts, const uint64_t* unit_norms, uint32_t units);
/* Working ciphertexts of the inner products (at least D / n1, a multiple of it
 * used at a time), each with room for the highest evaluation level. */
int afhe_ivfpq_set_scratch(afhe_ivfpq* h, const afhe_ct_ref* cts, uint32_t count);
int afhe_ivfpq_stage1(afhe_ivfpq* h, const afhe_ivfpq_query* queries, uint32_t count);
int afhe_ivfpq_stage3(afhe_ivfpq* h, const afhe_ivfpq_query* queries, uint32_t count);

#ifdef __cplusplus
}
#endif
#endif /* AFHE_H */
