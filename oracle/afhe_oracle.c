/* afhe_oracle.c -- CPU restatement of the reference's CKKS evaluation arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY (see afhe_oracle.h). Plain C11 with unsigned
 * __int128; no attempt at speed beyond -O3. Every function below names the
 * reference function it restates (paths inside iheydardoost/ANNS_FHE).
 */
#include "afhe_oracle.h"
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* hardware_fpga_model/hls/src/mod_arith.cpp:3 */
uint64_t orc_mod_add(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return s >= q ? s - q : s;
}

/* hardware_fpga_model/hls/src/mod_arith.cpp:9 */
uint64_t orc_mod_sub(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

/* hardware_fpga_model/hls/src/mod_arith.cpp:15-25. The reference's Barrett
 * reduction (m = floor(2^k/q), k = 2*bits(q)+3, two corrections) returns the
 * exact residue a*b mod q for every product below 2^(2*bits(q)); every call
 * site on the path satisfies that bound, so the exact remainder is restated. */
uint64_t orc_mod_mul(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

/* hardware_fpga_model/hls/src/ntt.cpp:4-43: in-place Cooley-Tukey, twiddle
 * tw[m + i] for butterfly block i of stage m, natural in -> bit-reversed out. */
void orc_ntt_forward(uint64_t* a, const uint64_t* tw, uint32_t n, uint64_t q) {
    uint32_t t = n >> 1;
    for (uint32_t m = 1; m < n; m <<= 1) {
        for (uint32_t i = 0; i < m; i++) {
            uint32_t j1 = 2 * i * t;
            uint64_t w = tw[m + i];
            for (uint32_t j = j1; j < j1 + t; j++) {
                uint64_t lo = a[j];
                uint64_t hw = orc_mod_mul(a[j + t], w, q);
                a[j] = orc_mod_add(lo, hw, q);
                a[j + t] = orc_mod_sub(lo, hw, q);
            }
        }
        t >>= 1;
    }
}

/* hardware_fpga_model/hls/src/ntt.cpp:46-80: Gentleman-Sande with itw[m + i],
 * then a separate pass multiplying by n^-1. */
void orc_intt_inverse(uint64_t* a, const uint64_t* itw, uint64_t n_inv, uint32_t n, uint64_t q) {
    uint32_t t = 1;
    for (uint32_t m = n >> 1; m >= 1; m >>= 1) {
        for (uint32_t i = 0; i < m; i++) {
            uint32_t j1 = 2 * i * t;
            uint64_t w = itw[m + i];
            for (uint32_t j = j1; j < j1 + t; j++) {
                uint64_t lo = a[j], hi = a[j + t];
                a[j] = orc_mod_add(lo, hi, q);
                a[j + t] = orc_mod_mul(orc_mod_sub(lo, hi, q), w, q);
            }
        }
        t <<= 1;
    }
    for (uint32_t i = 0; i < n; i++) a[i] = orc_mod_mul(a[i], n_inv, q);
}

/* hardware_fpga_model/hls/src/poly_arith.cpp:3-38 */
void orc_poly_add(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q) {
    for (uint32_t i = 0; i < n; i++) out[i] = orc_mod_add(a[i], b[i], q);
}
void orc_poly_sub(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q) {
    for (uint32_t i = 0; i < n; i++) out[i] = orc_mod_sub(a[i], b[i], q);
}
void orc_poly_mul(const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n, uint64_t q) {
    for (uint32_t i = 0; i < n; i++) out[i] = orc_mod_mul(a[i], b[i], q);
}

/* hardware_fpga_model/hls/src/automorphism.cpp:3-12: out[i] = a[map[i]], the
 * map packed two u32 per u64 word (low half = even index). */
void orc_automorphism(const uint64_t* a, uint64_t* out, const uint64_t* map64, uint32_t n) {
    for (uint32_t i = 0; i < n; i++) {
        uint64_t packed = map64[i / 2];
        uint32_t idx = (i % 2 == 0) ? (uint32_t)(packed & 0xFFFFFFFFu) : (uint32_t)(packed >> 32);
        out[i] = a[idx];
    }
}

/* hardware_fpga_model/hls/src/rescale.cpp:3-72. Drops the last limb:
 * INTT(last); for each remaining limb i: centred lift (v > q_l>>1 -> v - q_l)
 * mod q_i, times QlQlInvModqlDivqlModq[i], NTT with q_i's twiddles, then
 * a_i * qlInvModq[i] + that. */
void orc_rescale(const uint64_t* a_in, uint64_t* a_out, uint32_t num_limbs, const uint64_t* q,
                 const uint64_t* inv_tw_last, const uint64_t* tw, uint64_t n_inv_last,
                 const uint64_t* qlql, const uint64_t* qlinv, uint32_t n) {
    uint32_t last = num_limbs - 1;
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * n);
    uint64_t* tmp_i = (uint64_t*)malloc(sizeof(uint64_t) * n);
    memcpy(tmp, a_in + (size_t)last * n, sizeof(uint64_t) * n);
    orc_intt_inverse(tmp, inv_tw_last, n_inv_last, n, q[last]);
    uint64_t ql = q[last], half = ql >> 1;
    for (uint32_t i = 0; i < last; i++) {
        uint64_t qi = q[i];
        uint64_t ql_mod_qi = ql % qi;
        for (uint32_t j = 0; j < n; j++) {
            uint64_t v = tmp[j];
            uint64_t vm = v % qi;
            uint64_t val = (v > half) ? orc_mod_sub(vm, ql_mod_qi, qi) : vm;
            tmp_i[j] = orc_mod_mul(val, qlql[i], qi);
        }
        orc_ntt_forward(tmp_i, tw + (size_t)i * n, n, qi);
        for (uint32_t j = 0; j < n; j++) {
            uint64_t s = orc_mod_mul(a_in[(size_t)i * n + j], qlinv[i], qi);
            a_out[(size_t)i * n + j] = orc_mod_add(s, tmp_i[j], qi);
        }
    }
    free(tmp);
    free(tmp_i);
}

/* hardware_fpga_model/hls/src/key_switch.cpp:7-60 (ApproxSwitchCRTBasis, no
 * overflow correction): y_j = sum_i [x_i * qHatInv_i]_{q_i} * qHat_{i,j} mod p_j,
 * qhat_modp row-major [i][j] with row length n_out. */
void orc_fast_bases_conv(const uint64_t* in, uint64_t* out, uint32_t n_in, uint32_t n_out,
                         const uint64_t* in_primes, const uint64_t* out_primes,
                         const uint64_t* qhat_inv, const uint64_t* qhat_modp, uint32_t n) {
    uint64_t* x = (uint64_t*)malloc(sizeof(uint64_t) * n_in * (size_t)n);
    for (uint32_t i = 0; i < n_in; i++)
        for (uint32_t r = 0; r < n; r++)
            x[(size_t)i * n + r] = orc_mod_mul(in[(size_t)i * n + r], qhat_inv[i], in_primes[i]);
    for (uint32_t j = 0; j < n_out; j++) {
        uint64_t pj = out_primes[j];
        for (uint32_t r = 0; r < n; r++) {
            uint64_t s = 0;
            for (uint32_t i = 0; i < n_in; i++) {
                uint64_t xm = x[(size_t)i * n + r] % pj;
                s = orc_mod_add(s, orc_mod_mul(xm, qhat_modp[(size_t)i * n_out + j], pj), pj);
            }
            out[(size_t)j * n + r] = s;
        }
    }
    free(x);
}

/* hardware_fpga_model/hls/src/key_switch.cpp:62-163: INTT of the P limbs,
 * base conversion P -> Q, NTT of the Q limbs, then (x_Q - y) * P^-1 mod q_i. */
void orc_approx_mod_down(const uint64_t* in, uint64_t* out, uint32_t nq, uint32_t np,
                         const uint64_t* q, const uint64_t* p,
                         const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p,
                         const uint64_t* p_hat_mod_q, const uint64_t* inv_tw_p, const uint64_t* tw_q,
                         const uint64_t* n_inv_p, uint32_t n) {
    uint64_t* bp = (uint64_t*)malloc(sizeof(uint64_t) * np * (size_t)n);
    uint64_t* sw = (uint64_t*)malloc(sizeof(uint64_t) * nq * (size_t)n);
    memcpy(bp, in + (size_t)nq * n, sizeof(uint64_t) * np * (size_t)n);
    for (uint32_t i = 0; i < np; i++) orc_intt_inverse(bp + (size_t)i * n, inv_tw_p + (size_t)i * n, n_inv_p[i], n, p[i]);
    orc_fast_bases_conv(bp, sw, np, nq, p, q, p_hat_inv_mod_p, p_hat_mod_q, n);
    for (uint32_t i = 0; i < nq; i++) orc_ntt_forward(sw + (size_t)i * n, tw_q + (size_t)i * n, n, q[i]);
    for (uint32_t i = 0; i < nq; i++)
        for (uint32_t r = 0; r < n; r++) {
            uint64_t d = orc_mod_sub(in[(size_t)i * n + r], sw[(size_t)i * n + r], q[i]);
            out[(size_t)i * n + r] = orc_mod_mul(d, p_inv_mod_q[i], q[i]);
        }
    free(bp);
    free(sw);
}

/* hardware_fpga_model/hls/src/key_switch.cpp:167-439. For each digit: INTT of
 * its limbs, base conversion to the complementary Q primes and all P primes,
 * NTT, assemble the digit (own limbs copied from the evaluation-form input),
 * multiply-accumulate with the key; then ApproxModDown of both accumulators. */
void orc_key_switch(const uint64_t* c_in, const uint64_t* evk_a, const uint64_t* evk_b,
                    uint32_t key_digit_stride, uint32_t key_p_base,
                    uint64_t* out0, uint64_t* out1,
                    uint32_t sizeQl, uint32_t sizeP, uint32_t numPartQ, uint32_t alpha,
                    const uint64_t* q, const uint64_t* p,
                    const uint64_t* tw_q, const uint64_t* itw_q, const uint64_t* tw_p, const uint64_t* itw_p,
                    const uint64_t* n_inv_q, const uint64_t* n_inv_p,
                    const uint64_t* const* qhat_inv, const uint64_t* const* qhat_modp,
                    const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p,
                    const uint64_t* p_hat_mod_q, uint32_t n) {
    uint32_t qp = sizeQl + sizeP;
    size_t W = (size_t)qp * n;
    uint64_t* ext0 = (uint64_t*)calloc(W, sizeof(uint64_t));
    uint64_t* ext1 = (uint64_t*)calloc(W, sizeof(uint64_t));
    uint64_t* parts = (uint64_t*)malloc(W * sizeof(uint64_t));
    uint64_t* compl_ = (uint64_t*)malloc(W * sizeof(uint64_t));
    uint64_t* digit = (uint64_t*)malloc(W * sizeof(uint64_t));
    uint64_t out_primes[ORC_MAX_Q + ORC_MAX_P];
    const uint64_t* out_tw[ORC_MAX_Q + ORC_MAX_P];

    for (uint32_t part = 0; part < numPartQ; part++) {
        uint32_t size_part = (part == numPartQ - 1) ? (sizeQl - alpha * part) : alpha;
        uint32_t start = alpha * part;
        for (uint32_t i = 0; i < size_part; i++) {
            memcpy(parts + (size_t)i * n, c_in + (size_t)(start + i) * n, sizeof(uint64_t) * n);
            orc_intt_inverse(parts + (size_t)i * n, itw_q + (size_t)(start + i) * n, n_inv_q[start + i], n, q[start + i]);
        }
        uint32_t n_out = 0;
        for (uint32_t i = 0; i < sizeQl; i++)
            if (i < start || i >= start + size_part) { out_tw[n_out] = tw_q + (size_t)i * n; out_primes[n_out++] = q[i]; }
        for (uint32_t i = 0; i < sizeP; i++) { out_tw[n_out] = tw_p + (size_t)i * n; out_primes[n_out++] = p[i]; }
        orc_fast_bases_conv(parts, compl_, size_part, n_out, q + start, out_primes, qhat_inv[part], qhat_modp[part], n);
        for (uint32_t k = 0; k < n_out; k++) orc_ntt_forward(compl_ + (size_t)k * n, out_tw[k], n, out_primes[k]);
        uint32_t oi = 0;
        for (uint32_t i = 0; i < sizeQl; i++) {
            const uint64_t* src = (i >= start && i < start + size_part) ? c_in + (size_t)i * n : compl_ + (size_t)(oi++) * n;
            memcpy(digit + (size_t)i * n, src, sizeof(uint64_t) * n);
        }
        for (uint32_t i = 0; i < sizeP; i++) memcpy(digit + (size_t)(sizeQl + i) * n, compl_ + (size_t)(oi++) * n, sizeof(uint64_t) * n);

        for (uint32_t i = 0; i < qp; i++) {
            uint64_t m = (i < sizeQl) ? q[i] : p[i - sizeQl];
            size_t klimb = (size_t)part * key_digit_stride + (i < sizeQl ? i : key_p_base + (i - sizeQl));
            const uint64_t* ka = evk_a + klimb * n;
            const uint64_t* kb = evk_b + klimb * n;
            for (uint32_t r = 0; r < n; r++) {
                uint64_t c = digit[(size_t)i * n + r];
                ext0[(size_t)i * n + r] = orc_mod_add(ext0[(size_t)i * n + r], orc_mod_mul(c, kb[r], m), m);
                ext1[(size_t)i * n + r] = orc_mod_add(ext1[(size_t)i * n + r], orc_mod_mul(c, ka[r], m), m);
            }
        }
    }
    orc_approx_mod_down(ext0, out0, sizeQl, sizeP, q, p, p_inv_mod_q, p_hat_inv_mod_p, p_hat_mod_q, itw_p, tw_q, n_inv_p, n);
    orc_approx_mod_down(ext1, out1, sizeQl, sizeP, q, p, p_inv_mod_q, p_hat_inv_mod_p, p_hat_mod_q, itw_p, tw_q, n_inv_p, n);
    free(ext0); free(ext1); free(parts); free(compl_); free(digit);
}

/* ---- fhe_accel_top over word arenas ---------------------------------------
 * hardware_fpga_model/hls/src/fhe_accel_top.cpp:90-328. The reference keeps the
 * OP_LOAD_CONTEXT tables in static on-chip arrays; here they live in orc_ctx. */
struct orc_ctx {
    uint32_t n;
    uint64_t *tw_q, *itw_q, *tw_p, *itw_p;
    uint64_t qhat_inv[ORC_MAX_PARTS][ORC_MAX_Q];
    uint64_t qhat_modp[ORC_MAX_PARTS][ORC_MAX_Q * (ORC_MAX_Q + ORC_MAX_P)];
    uint64_t p_inv_mod_q[ORC_MAX_Q], p_hat_inv_mod_p[ORC_MAX_P], p_hat_mod_q[ORC_MAX_P * ORC_MAX_Q];
    uint64_t qlql[ORC_MAX_Q], qlinv[ORC_MAX_Q];
};

orc_ctx* orc_ctx_create(uint32_t n) {
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->n = n;
    c->tw_q = (uint64_t*)calloc((size_t)ORC_MAX_Q * n, 8);
    c->itw_q = (uint64_t*)calloc((size_t)ORC_MAX_Q * n, 8);
    c->tw_p = (uint64_t*)calloc((size_t)ORC_MAX_P * n, 8);
    c->itw_p = (uint64_t*)calloc((size_t)ORC_MAX_P * n, 8);
    return c;
}

void orc_ctx_destroy(orc_ctx* c) {
    if (!c) return;
    free(c->tw_q); free(c->itw_q); free(c->tw_p); free(c->itw_p); free(c);
}

static void ld(const uint64_t* key, uint64_t off, uint64_t* dst, size_t words) {
    memcpy(dst, key + off, words * sizeof(uint64_t));
}

int orc_accel_top(orc_ctx* c, uint64_t* poly, uint64_t* key, const orc_top_args* a) {
    const uint32_t n = c->n;
    const uint32_t L = a->active_limbs;
    const size_t LN = (size_t)L * n;
    if (a->op_code == 99) {
        /* fhe_accel_top.cpp:194-218 */
        ld(key, a->twiddles_q_offset, c->tw_q, LN);
        ld(key, a->inv_twiddles_q_offset, c->itw_q, LN);
        ld(key, a->twiddles_p_offset, c->tw_p, (size_t)a->sizeP * n);
        ld(key, a->inv_twiddles_p_offset, c->itw_p, (size_t)a->sizeP * n);
        for (uint32_t j = 0; j < a->numPartQ; j++) {
            uint32_t sz = (j == a->numPartQ - 1) ? L - a->alpha * j : a->alpha;
            ld(key, a->qhat_inv_offset[j], c->qhat_inv[j], sz);
            ld(key, a->qhat_modp_offset[j], c->qhat_modp[j], (size_t)sz * (L - sz + a->sizeP));
        }
        ld(key, a->p_inv_mod_q_offset, c->p_inv_mod_q, L);
        ld(key, a->p_hat_inv_mod_p_offset, c->p_hat_inv_mod_p, a->sizeP);
        ld(key, a->p_hat_mod_q_offset, c->p_hat_mod_q, (size_t)a->sizeP * L);
        ld(key, a->qlql_offset, c->qlql, L);
        ld(key, a->qlinv_offset, c->qlinv, L);
        return 0;
    }
    uint64_t* A = poly + a->src_a_offset;
    uint64_t* B = poly + a->src_b_offset;
    uint64_t* D = poly + a->dst_offset;
    const uint64_t* qs = a->rns_primes;
    switch (a->op_code) {
    case 1: { /* :222-230 */
        uint64_t* w = (uint64_t*)malloc(LN * 8); memcpy(w, A, LN * 8);
        for (uint32_t l = 0; l < L; l++) orc_ntt_forward(w + (size_t)l * n, c->tw_q + (size_t)l * n, n, qs[l]);
        memcpy(D, w, LN * 8); free(w); return 0; }
    case 2: { /* :232-240 */
        uint64_t* w = (uint64_t*)malloc(LN * 8); memcpy(w, A, LN * 8);
        for (uint32_t l = 0; l < L; l++) orc_intt_inverse(w + (size_t)l * n, c->itw_q + (size_t)l * n, a->n_inv_q[l], n, qs[l]);
        memcpy(D, w, LN * 8); free(w); return 0; }
    case 3: case 4: case 5: { /* :242-270 */
        uint64_t* w = (uint64_t*)malloc(LN * 8);
        for (uint32_t l = 0; l < L; l++) {
            const uint64_t *x = A + (size_t)l * n, *y = B + (size_t)l * n;
            uint64_t* o = w + (size_t)l * n;
            if (a->op_code == 3) orc_poly_add(x, y, o, n, qs[l]);
            else if (a->op_code == 4) orc_poly_sub(x, y, o, n, qs[l]);
            else orc_poly_mul(x, y, o, n, qs[l]);
        }
        memcpy(D, w, LN * 8); free(w); return 0; }
    case 6: { /* :272-281 */
        uint64_t* w = (uint64_t*)malloc(LN * 8);
        uint64_t* map = (uint64_t*)malloc((size_t)n / 2 * 8); memcpy(map, B, (size_t)n / 2 * 8);
        for (uint32_t l = 0; l < L; l++) orc_automorphism(A + (size_t)l * n, w + (size_t)l * n, map, n);
        memcpy(D, w, LN * 8); free(w); free(map); return 0; }
    case 8: { /* :283-297 */
        size_t out = (size_t)(L - 1) * n;
        uint64_t* w0 = (uint64_t*)malloc(LN * 8); uint64_t* w1 = (uint64_t*)malloc(LN * 8);
        uint64_t* r0 = (uint64_t*)malloc(LN * 8); uint64_t* r1 = (uint64_t*)malloc(LN * 8);
        memcpy(w0, A, LN * 8); memcpy(w1, B, LN * 8);
        const uint64_t* itl = c->itw_q + (size_t)(L - 1) * n;
        orc_rescale(w0, r0, L, qs, itl, c->tw_q, a->n_inv_mod_q_last, c->qlql, c->qlinv, n);
        orc_rescale(w1, r1, L, qs, itl, c->tw_q, a->n_inv_mod_q_last, c->qlql, c->qlinv, n);
        memcpy(D, r0, out * 8); memcpy(D + out, r1, out * 8);
        free(w0); free(w1); free(r0); free(r1); return 0; }
    case 7: { /* :299-326 */
        uint32_t sq = a->sizeQl, sp = a->sizeP;
        size_t SQ = (size_t)sq * n;
        uint64_t* w = (uint64_t*)malloc(SQ * 8); memcpy(w, A, SQ * 8);
        uint64_t* o0 = (uint64_t*)malloc(SQ * 8); uint64_t* o1 = (uint64_t*)malloc(SQ * 8);
        const uint64_t* qi[ORC_MAX_PARTS]; const uint64_t* qm[ORC_MAX_PARTS];
        for (uint32_t j = 0; j < ORC_MAX_PARTS; j++) { qi[j] = c->qhat_inv[j]; qm[j] = c->qhat_modp[j]; }
        const uint64_t* ea = key + a->evk_offset;
        const uint64_t* eb = key + a->evk_offset + (size_t)a->numPartQ * (sq + sp) * n;
        orc_key_switch(w, ea, eb, sq + sp, sq, o0, o1, sq, sp, a->numPartQ, a->alpha, qs, a->p_primes,
                       c->tw_q, c->itw_q, c->tw_p, c->itw_p, a->n_inv_q, a->n_inv_p, qi, qm,
                       c->p_inv_mod_q, c->p_hat_inv_mod_p, c->p_hat_mod_q, n);
        memcpy(D, o0, SQ * 8); memcpy(D + SQ, o1, SQ * 8);
        free(w); free(o0); free(o1); return 0; }
    default:
        return 1;
    }
}
