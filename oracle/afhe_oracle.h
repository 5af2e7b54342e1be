/* afhe_oracle.h -- CPU restatement of the reference's CKKS evaluation arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY: the bit-exact checker for the CUDA path. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may load it;
 * the product never does.
 *
 * Each function restates one reference HLS function of iheydardoost/ANNS_FHE
 * (hardware_fpga_model/hls/src/...) for a general power-of-two ring degree n
 * and general limb counts; at n = 16384 with <= 15 limbs it is cross-checked
 * word for word against the reference compiled verbatim (oracle/_ref).
 * All values are canonical residues in [0, q).
 */
#ifndef AFHE_ORACLE_H
#define AFHE_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

uint64_t orc_mod_add(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_mod_sub(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_mod_mul(uint64_t a, uint64_t b, uint64_t q);

void orc_ntt_forward(uint64_t* a, const uint64_t* tw, uint32_t n, uint64_t q);
void orc_intt_inverse(uint64_t* a, const uint64_t* itw, uint64_t n_inv, uint32_t n, uint64_t q);

void orc_poly_add(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q);
void orc_poly_sub(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q);
void orc_poly_mul(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q);
void orc_automorphism(const uint64_t* a, uint64_t* out, const uint64_t* map64, uint32_t n);

void orc_rescale(const uint64_t* a_in, uint64_t* a_out, uint32_t num_limbs, const uint64_t* q,
                 const uint64_t* inv_tw_last, const uint64_t* tw, uint64_t n_inv_last,
                 const uint64_t* qlql, const uint64_t* qlinv, uint32_t n);

void orc_fast_bases_conv(const uint64_t* in, uint64_t* out, uint32_t n_in, uint32_t n_out,
                         const uint64_t* in_primes, const uint64_t* out_primes,
                         const uint64_t* qhat_inv, const uint64_t* qhat_modp, uint32_t n);

void orc_approx_mod_down(const uint64_t* in, uint64_t* out, uint32_t nq, uint32_t np,
                         const uint64_t* q, const uint64_t* p,
                         const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p,
                         const uint64_t* p_hat_mod_q, const uint64_t* inv_tw_p, const uint64_t* tw_q,
                         const uint64_t* n_inv_p, uint32_t n);

/* Hybrid key switch of one polynomial (no c0 add).
 * evk_a / evk_b point at digit 0 of each key half; digit `part`, limb i lives at
 *   evk_x + (part * key_digit_stride + (i < sizeQl ? i : key_p_base + i - sizeQl)) * n.
 * The reference's OP_KEY_SWITCH uses key_digit_stride = sizeQl + sizeP and
 * key_p_base = sizeQl; a full-level key uses (L + K, L).
 * qhat_inv[part] / qhat_modp[part]: the per-digit base-conversion tables. */
void orc_key_switch(const uint64_t* c_in, const uint64_t* evk_a, const uint64_t* evk_b,
                    uint32_t key_digit_stride, uint32_t key_p_base,
                    uint64_t* out0, uint64_t* out1,
                    uint32_t sizeQl, uint32_t sizeP, uint32_t numPartQ, uint32_t alpha,
                    const uint64_t* q, const uint64_t* p,
                    const uint64_t* tw_q, const uint64_t* itw_q, const uint64_t* tw_p, const uint64_t* itw_p,
                    const uint64_t* n_inv_q, const uint64_t* n_inv_p,
                    const uint64_t* const* qhat_inv, const uint64_t* const* qhat_modp,
                    const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p,
                    const uint64_t* p_hat_mod_q, uint32_t n);

/* fhe_accel_top restated over 64-bit word arenas with an explicit context in
 * place of the reference's static on-chip tables. Field meanings follow
 * hardware_fpga_model/hls/src/fhe_accel_top.h:6-56. */
#define ORC_MAX_Q 64
#define ORC_MAX_P 16
#define ORC_MAX_PARTS 16

typedef struct orc_top_args {
    uint32_t op_code;
    uint64_t src_a_offset, src_b_offset, dst_offset;
    uint64_t evk_offset;
    uint32_t active_limbs, prime_idx, galois_elt;
    uint32_t sizeQl, sizeP, numPartQ, alpha;
    uint64_t rns_primes[ORC_MAX_Q];
    uint64_t p_primes[ORC_MAX_P];
    uint64_t n_inv_q[ORC_MAX_Q];
    uint64_t n_inv_p[ORC_MAX_P];
    uint64_t n_inv_mod_q_last;
    uint64_t twiddles_q_offset, inv_twiddles_q_offset, twiddles_p_offset, inv_twiddles_p_offset;
    uint64_t qhat_inv_offset[ORC_MAX_PARTS];
    uint64_t qhat_modp_offset[ORC_MAX_PARTS];
    uint64_t p_inv_mod_q_offset, p_hat_inv_mod_p_offset, p_hat_mod_q_offset;
    uint64_t qlql_offset, qlinv_offset;
} orc_top_args;

typedef struct orc_ctx orc_ctx;
orc_ctx* orc_ctx_create(uint32_t n);
void orc_ctx_destroy(orc_ctx* c);
/* returns 0 on success, non-zero for an unknown op code */
int orc_accel_top(orc_ctx* c, uint64_t* poly, uint64_t* key, const orc_top_args* a);

#ifdef __cplusplus
}
#endif
#endif
