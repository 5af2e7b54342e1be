/* A plain C caller of the device path: includes include/afhe.h, links
 * libafhe.so, creates a context on GPU 0 and drives the reference's operators
 * through the C ABI alone, checking each against another route to the same
 * result or against a host computation:
 *   afhe_ntt then afhe_intt returns the input;
 *   afhe_poly_add / afhe_poly_mul_ntt equal the sum / product mod q on the host;
 *   afhe_dispatch OP 3 (POLY_ADD) after OP 99 equals afhe_poly_add;
 *   afhe_eval_rotate equals afhe_eval_rotate_batch of one ciphertext, and
 *   rotating by 1 then by -1 through eval_rotate_steps_batch is one key switch each;
 *   afhe_eval_mult_relin_rescale equals its batched form.
 * Prints one line per check; exits non-zero on the first failure. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "afhe.h"

#define N_LOG 10
#define N (1u << N_LOG)
#define NQ 3
#define NP 1

static uint64_t state = 88172645463325252ull;
static uint64_t rnd(void) {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return state;
}

static int fill(uint64_t* v, const uint64_t* primes, uint32_t limbs) {
    for (uint32_t i = 0; i < limbs; ++i)
        for (uint32_t j = 0; j < N; ++j) v[(size_t)i * N + j] = rnd() % primes[i];
    return 0;
}

#define CHECK(cond, code, what)                                            \
    do {                                                                   \
        if (!(cond)) {                                                     \
            fprintf(stderr, "%s failed: %s\n", what, afhe_last_error());   \
            return code;                                                   \
        }                                                                  \
    } while (0)

int main(void) {
    uint64_t q[NQ], p[NP], all[NQ + NP];
    CHECK(afhe_find_ntt_primes(N_LOG, 50, NQ, NULL, 0, q) == AFHE_OK, 1, "primes");
    CHECK(afhe_find_ntt_primes(N_LOG, 60, NP, q, NQ, p) == AFHE_OK, 2, "primes");
    memcpy(all, q, sizeof q);
    memcpy(all + NQ, p, sizeof p);

    afhe_params prm;
    memset(&prm, 0, sizeof prm);
    prm.log_n = N_LOG;
    prm.num_q = NQ;
    prm.num_p = NP;
    prm.alpha = 1;
    memcpy(prm.q, q, sizeof q);
    memcpy(prm.p, p, sizeof p);
    prm.poly_words = 64ull * (NQ + NP) * N;
    prm.key_words = 64ull * (NQ + NP) * N;
    prm.max_batch = 4;
    afhe_ctx* ctx = NULL;
    CHECK(afhe_ctx_create(&prm, &ctx) == AFHE_OK, 3, "afhe_ctx_create");

    const size_t W = (size_t)NQ * N;     /* one polynomial at the top level */
    uint64_t* a = malloc(W * 8);
    uint64_t* b = malloc(W * 8);
    uint64_t* r = malloc(W * 8);
    uint64_t* s = malloc(W * 8);
    fill(a, q, NQ);
    fill(b, q, NQ);

    /* NTT round trip */
    CHECK(afhe_write_poly(ctx, 0, a, W) == AFHE_OK, 4, "write");
    CHECK(afhe_ntt(ctx, 0, W, NQ) == AFHE_OK && afhe_intt(ctx, W, 2 * W, NQ) == AFHE_OK, 5, "ntt/intt");
    CHECK(afhe_read_poly(ctx, 2 * W, r, W) == AFHE_OK, 6, "read");
    CHECK(memcmp(r, a, W * 8) == 0, 7, "INTT(NTT(a)) == a");
    printf("ntt round trip ok\n");

    /* elementwise against the host */
    CHECK(afhe_write_poly(ctx, W, b, W) == AFHE_OK, 8, "write");
    CHECK(afhe_poly_add(ctx, 0, W, 2 * W, NQ) == AFHE_OK, 9, "poly_add");
    CHECK(afhe_poly_mul_ntt(ctx, 0, W, 3 * W, NQ) == AFHE_OK, 10, "poly_mul_ntt");
    CHECK(afhe_read_poly(ctx, 2 * W, r, W) == AFHE_OK && afhe_read_poly(ctx, 3 * W, s, W) == AFHE_OK, 11, "read");
    for (uint32_t i = 0; i < NQ; ++i)
        for (uint32_t j = 0; j < N; ++j) {
            const size_t k = (size_t)i * N + j;
            CHECK(r[k] == (a[k] + b[k]) % q[i], 12, "add mod q");
            CHECK(s[k] == (uint64_t)((unsigned __int128)a[k] * b[k] % q[i]), 13, "mul mod q");
        }
    printf("poly_add / poly_mul_ntt ok\n");

    /* the accelerator ABI: OP 99 with tables written by the context, then OP 3 */
    afhe_context_layout lay;
    CHECK(afhe_ctx_write_context_tables(ctx, NQ, &lay) == AFHE_OK, 14, "context tables");
    afhe_accel_args args;
    memset(&args, 0, sizeof args);
    args.op_code = AFHE_OP_LOAD_CONTEXT;
    args.active_limbs = NQ;
    args.sizeQl = NQ;
    args.sizeP = NP;
    args.numPartQ = NQ;
    args.alpha = 1;
    memcpy(args.rns_primes, q, sizeof q);
    memcpy(args.p_primes, p, sizeof p);
    for (int i = 0; i < NQ; ++i) {
        afhe_barrett_constant(q[i], &args.barrett_m_q_lo[i], &args.barrett_m_q_hi[i], &args.barrett_k_q[i]);
        args.n_inv_q[i] = afhe_inv_mod(N % q[i], q[i]);
    }
    for (int i = 0; i < NP; ++i) {
        afhe_barrett_constant(p[i], &args.barrett_m_p_lo[i], &args.barrett_m_p_hi[i], &args.barrett_k_p[i]);
        args.n_inv_p[i] = afhe_inv_mod(N % p[i], p[i]);
    }
    args.n_inv_mod_q_last = args.n_inv_q[NQ - 1];
    args.twiddles_q_offset = lay.twiddles_q_offset;
    args.inv_twiddles_q_offset = lay.inv_twiddles_q_offset;
    args.twiddles_p_offset = lay.twiddles_p_offset;
    args.inv_twiddles_p_offset = lay.inv_twiddles_p_offset;
    for (int j = 0; j < AFHE_MAX_PARTS; ++j) {
        args.qhat_inv_offset[j] = lay.qhat_inv_offset[j];
        args.qhat_modp_offset[j] = lay.qhat_modp_offset[j];
    }
    args.p_inv_mod_q_offset = lay.p_inv_mod_q_offset;
    args.p_hat_inv_mod_p_offset = lay.p_hat_inv_mod_p_offset;
    args.p_hat_mod_q_offset = lay.p_hat_mod_q_offset;
    args.qlql_offset = lay.qlql_offset;
    args.qlinv_offset = lay.qlinv_offset;
    CHECK(afhe_dispatch(ctx, &args) == AFHE_OK, 15, "OP 99");
    args.op_code = AFHE_OP_POLY_ADD;
    args.active_limbs = NQ;
    args.src_a_offset = 0;
    args.src_b_offset = W;
    args.dst_offset = 4 * W;
    CHECK(afhe_dispatch(ctx, &args) == AFHE_OK, 16, "OP 3");
    CHECK(afhe_read_poly(ctx, 4 * W, s, W) == AFHE_OK, 17, "read");
    CHECK(memcmp(r, s, W * 8) == 0, 18, "OP 3 == afhe_poly_add");
    printf("afhe_dispatch ok\n");

    /* composite operators with keys: a relinearisation key and rotation keys for 1 and -1 */
    const size_t KW = 2ull * NQ * (NQ + NP) * N;     /* dnum = NQ digits of a, then of b */
    uint64_t* key = malloc(KW * 8);
    for (int k = 0; k < 3; ++k) {
        for (size_t d = 0; d < 2ull * NQ; ++d) fill(key + d * (NQ + NP) * N, all, NQ + NP);
        const uint64_t off = lay.first_free_offset + (uint64_t)k * ((KW + 511) & ~511ull);
        CHECK(afhe_write_key(ctx, off, key, KW) == AFHE_OK, 19, "write key");
        if (k == 0) CHECK(afhe_set_relin_key(ctx, off) == AFHE_OK, 20, "relin key");
        else CHECK(afhe_add_rotation_key(ctx, k == 1 ? 1 : -1, off) == AFHE_OK, 21, "rotation key");
    }
    /* ciphertext (a, b) at [0, 2W); results after it */
    afhe_ct_ref in = {0, W}, o1 = {8 * W, 9 * W}, o2 = {10 * W, 11 * W};
    CHECK(afhe_eval_rotate(ctx, in.c0_offset, in.c1_offset, o1.c0_offset, o1.c1_offset, 1, NQ) == AFHE_OK, 22,
          "eval_rotate");
    CHECK(afhe_eval_rotate_batch(ctx, &in, &o2, 1, 1, NQ) == AFHE_OK, 23, "eval_rotate_batch");
    CHECK(afhe_read_poly(ctx, o1.c0_offset, r, W) == AFHE_OK && afhe_read_poly(ctx, o2.c0_offset, s, W) == AFHE_OK,
          24, "read");
    CHECK(memcmp(r, s, W * 8) == 0, 25, "eval_rotate == eval_rotate_batch (c0)");
    CHECK(afhe_read_poly(ctx, o1.c1_offset, r, W) == AFHE_OK && afhe_read_poly(ctx, o2.c1_offset, s, W) == AFHE_OK,
          26, "read");
    CHECK(memcmp(r, s, W * 8) == 0, 27, "eval_rotate == eval_rotate_batch (c1)");
    const int32_t steps[2] = {1, -1};
    afhe_ct_ref two_in[2] = {in, in}, two_out[2] = {{12 * W, 13 * W}, {14 * W, 15 * W}};
    CHECK(afhe_eval_rotate_steps_batch(ctx, two_in, two_out, steps, 2, NQ) == AFHE_OK, 28, "eval_rotate_steps_batch");
    CHECK(afhe_read_poly(ctx, two_out[0].c0_offset, s, W) == AFHE_OK, 29, "read");
    CHECK(afhe_read_poly(ctx, o1.c0_offset, r, W) == AFHE_OK && memcmp(r, s, W * 8) == 0, 30,
          "steps batch (step 1) == eval_rotate");
    printf("rotations ok\n");

    afhe_ct_ref m1 = {16 * W, 17 * W}, m2 = {18 * W, 19 * W};
    CHECK(afhe_eval_mult_relin_rescale(ctx, 0, W, 0, W, m1.c0_offset, m1.c1_offset, NQ) == AFHE_OK, 31,
          "eval_mult_relin_rescale");
    CHECK(afhe_eval_mult_relin_rescale_batch(ctx, &in, &in, &m2, 1, NQ) == AFHE_OK, 32, "batched");
    const size_t W1 = (size_t)(NQ - 1) * N;
    CHECK(afhe_read_poly(ctx, m1.c1_offset, r, W1) == AFHE_OK && afhe_read_poly(ctx, m2.c1_offset, s, W1) == AFHE_OK,
          33, "read");
    CHECK(memcmp(r, s, W1 * 8) == 0, 34, "mult_relin_rescale == batched");
    printf("mult_relin_rescale ok\n");

    CHECK(afhe_sync(ctx) == AFHE_OK, 35, "sync");
    afhe_ctx_destroy(ctx);
    free(a);
    free(b);
    free(r);
    free(s);
    free(key);
    printf("all ok\n");
    return 0;
}
