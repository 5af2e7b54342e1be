// fhe_accel_top_shim.cpp -- the reference's accelerator symbol over this library.
//
// A host built against the reference's kernel ABI calls
//   extern "C" void fhe_accel_top(ap_uint<512>* poly_gmem, ap_uint<512>* key_gmem,
//                                 uint32_t op_code, ... 15 table offsets)
// (hardware_fpga_model/hls/src/fhe_accel_top.h:6-56), e.g. FHEHostDriver::dispatch
// (cpp_host_model/src/fhe_host_driver.cpp:177-204). Linking this file's library
// (lib/libafhe_accel_top.so) in place of the HLS kernel object runs every call
// on the GPU through afhe_dispatch, with the host program unchanged.
//
// That host keeps poly_gmem / key_gmem in its own memory (SimMemoryBus,
// cpp_host_model/src/sim_memory_bus.h:10-34) and writes them between calls, so
// each call mirrors what it touches: the op's operands are copied to the
// device arenas, the op runs, and its output is copied back before the call
// returns (the reference's call is synchronous). Tables are copied at OP 99;
// an evaluation key is copied the first time a key switch names it after an
// OP 99 (the reference's host loads keys before it loads the context). A host
// that keeps its arenas in HBM instead calls afhe_dispatch on them directly.
//
// The 512-bit beats are taken as eight little-endian 64-bit words (the layout
// of ap_uint<512> in C simulation); the Barrett constants the call carries are
// not read: they are recomputed from the primes (afhe_barrett_constant), so
// the ap_uint<128> representation does not matter.
//
// The reference's call returns nothing; a failed call is reported on stderr
// and by afhe_accel_top_last_status().
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "afhe.h"

namespace {

struct Binding {
    afhe_ctx* ctx = nullptr;
    uint32_t log_n = 14;                    // the reference's N = 16384 (hls_params.h:6)
    uint64_t poly_words = 8388608;          // SimMemoryBus's default arenas (sim_memory_bus.h:13)
    uint64_t key_words = 67108864;
    int device = 0;
    int status = AFHE_OK;
    std::vector<uint64_t> ctx_primes;       // Q then P primes the context was made for
    std::vector<std::pair<uint64_t, uint64_t>> keys;   // key ranges copied since the last OP 99
};

Binding& binding() {
    static Binding b;
    return b;
}

int report(int rc, const char* what) {
    Binding& b = binding();
    b.status = rc;
    if (rc != AFHE_OK) std::fprintf(stderr, "fhe_accel_top (afhe): %s: %s\n", what, afhe_last_error());
    return rc;
}

int put_poly(const uint64_t* host, uint64_t off, uint64_t words) {
    return words ? afhe_write_poly(binding().ctx, off, host + off, words) : AFHE_OK;
}

int put_key(const uint64_t* host, uint64_t off, uint64_t words) {
    if (off >= binding().key_words) return AFHE_E_RANGE;
    if (off + words > binding().key_words) words = binding().key_words - off;
    return words ? afhe_write_key(binding().ctx, off, host + off, words) : AFHE_OK;
}

// A context for the call's primes (made, or made again, at OP 99).
int ensure_context(uint32_t L, uint32_t K, uint32_t alpha, const uint64_t* q, const uint64_t* p) {
    Binding& b = binding();
    std::vector<uint64_t> want(q, q + L);
    want.insert(want.end(), p, p + K);
    if (b.ctx && want == b.ctx_primes) return AFHE_OK;
    if (b.ctx) afhe_ctx_destroy(b.ctx);
    b.ctx = nullptr;
    afhe_params prm{};
    prm.log_n = b.log_n;
    prm.num_q = L;
    prm.num_p = K;
    prm.alpha = alpha;
    for (uint32_t i = 0; i < L; ++i) prm.q[i] = q[i];
    for (uint32_t i = 0; i < K; ++i) prm.p[i] = p[i];
    prm.poly_words = b.poly_words;
    prm.key_words = b.key_words;
    prm.device = b.device;
    prm.max_batch = 1;
    int rc = afhe_ctx_create(&prm, &b.ctx);
    if (rc == AFHE_OK) b.ctx_primes = want;
    return rc;
}

}  // namespace

extern "C" {

// Ring degree, arena sizes (64-bit words) and device of the mirror; call it
// before the first fhe_accel_top if the host's differ from the reference's
// defaults (N = 16384, SimMemoryBus's 8 M / 64 M words, device 0).
int afhe_accel_top_configure(uint32_t log_n, uint64_t poly_words, uint64_t key_words, int device) {
    Binding& b = binding();
    if (b.ctx) afhe_ctx_destroy(b.ctx);
    b = Binding{};
    b.log_n = log_n;
    b.poly_words = poly_words;
    b.key_words = key_words;
    b.device = device;
    return AFHE_OK;
}

int afhe_accel_top_last_status(void) { return binding().status; }

// Releases the mirror (the next OP 99 makes a new one).
void afhe_accel_top_release(void) {
    Binding& b = binding();
    if (b.ctx) afhe_ctx_destroy(b.ctx);
    b.ctx = nullptr;
    b.ctx_primes.clear();
    b.keys.clear();
}

void fhe_accel_top(void* poly_gmem, void* key_gmem, uint32_t op_code, uint32_t src_a_offset, uint32_t src_b_offset,
                   uint32_t dst_offset, uint64_t evk_offset, uint32_t active_limbs, uint32_t prime_idx,
                   uint32_t galois_elt, uint32_t sizeQl, uint32_t sizeP, uint32_t numPartQ, uint32_t alpha,
                   const uint64_t* rns_primes, const uint64_t* p_primes, const void* barrett_m_q,
                   const uint32_t* barrett_k_q, const void* barrett_m_p, const uint32_t* barrett_k_p,
                   const uint64_t* n_inv_q, const uint64_t* n_inv_p, uint64_t n_inv_mod_q_last,
                   uint32_t twiddles_q_offset, uint32_t inv_twiddles_q_offset, uint32_t twiddles_p_offset,
                   uint32_t inv_twiddles_p_offset, uint32_t qHatInvModq_0_offset, uint32_t qHatModp_0_offset,
                   uint32_t qHatInvModq_1_offset, uint32_t qHatModp_1_offset, uint32_t qHatInvModq_2_offset,
                   uint32_t qHatModp_2_offset, uint32_t PInvModq_offset, uint32_t PHatInvModp_offset,
                   uint32_t PHatModq_offset, uint32_t QlQlInvModqlDivqlModq_offset, uint32_t qlInvModq_offset) {
    (void)barrett_m_q;
    (void)barrett_k_q;
    (void)barrett_m_p;
    (void)barrett_k_p;
    Binding& b = binding();
    const uint64_t* poly = static_cast<const uint64_t*>(poly_gmem);
    const uint64_t* key = static_cast<const uint64_t*>(key_gmem);
    const uint64_t n = 1ull << b.log_n;
    const uint32_t L = active_limbs;
    int rc;
    if (op_code == AFHE_OP_LOAD_CONTEXT) {
        if ((rc = ensure_context(L, sizeP, alpha, rns_primes, p_primes)) != AFHE_OK) {
            report(rc, "context");
            return;
        }
        b.keys.clear();
        // the tables OP 99 reads: twiddles, and the CRT tables' 64-word slots
        // (fhe_host_driver.cpp:63-86 places them back to back)
        const uint64_t tw[4] = {twiddles_q_offset, inv_twiddles_q_offset, twiddles_p_offset, inv_twiddles_p_offset};
        const uint64_t tw_words[4] = {L * n, L * n, sizeP * n, sizeP * n};
        for (int i = 0; i < 4; ++i)
            if ((rc = put_key(key, tw[i], tw_words[i])) != AFHE_OK) {
                report(rc, "copy twiddles");
                return;
            }
        const uint32_t crt[11] = {qHatInvModq_0_offset, qHatModp_0_offset, qHatInvModq_1_offset, qHatModp_1_offset,
                                  qHatInvModq_2_offset, qHatModp_2_offset, PInvModq_offset, PHatInvModp_offset,
                                  PHatModq_offset, QlQlInvModqlDivqlModq_offset, qlInvModq_offset};
        uint64_t lo = crt[0], hi = crt[0];
        for (uint32_t o : crt) {
            lo = o < lo ? o : lo;
            hi = o > hi ? o : hi;
        }
        if ((rc = put_key(key, lo, hi - lo + 128)) != AFHE_OK) {
            report(rc, "copy CRT tables");
            return;
        }
    }
    if (!b.ctx) {
        report(AFHE_E_STATE, "op before OP 99");
        return;
    }
    afhe_accel_args a{};
    a.op_code = op_code;
    a.active_limbs = active_limbs;
    a.src_a_offset = src_a_offset;
    a.src_b_offset = src_b_offset;
    a.dst_offset = dst_offset;
    a.evk_offset = evk_offset;
    a.prime_idx = prime_idx;
    a.galois_elt = galois_elt;
    a.sizeQl = sizeQl;
    a.sizeP = sizeP;
    a.numPartQ = numPartQ;
    a.alpha = alpha;
    // the reference's arrays hold 15 Q and 4 P entries (fhe_accel_top.h:22-31)
    for (uint32_t i = 0; i < 15 && i < AFHE_MAX_Q; ++i) {
        a.rns_primes[i] = rns_primes[i];
        a.n_inv_q[i] = n_inv_q[i];
        if (rns_primes[i] > 2) afhe_barrett_constant(rns_primes[i], &a.barrett_m_q_lo[i], &a.barrett_m_q_hi[i],
                                                     &a.barrett_k_q[i]);
    }
    for (uint32_t i = 0; i < 4 && i < AFHE_MAX_P; ++i) {
        a.p_primes[i] = p_primes[i];
        a.n_inv_p[i] = n_inv_p[i];
        if (p_primes[i] > 2) afhe_barrett_constant(p_primes[i], &a.barrett_m_p_lo[i], &a.barrett_m_p_hi[i],
                                                   &a.barrett_k_p[i]);
    }
    a.n_inv_mod_q_last = n_inv_mod_q_last;
    a.twiddles_q_offset = twiddles_q_offset;
    a.inv_twiddles_q_offset = inv_twiddles_q_offset;
    a.twiddles_p_offset = twiddles_p_offset;
    a.inv_twiddles_p_offset = inv_twiddles_p_offset;
    a.qhat_inv_offset[0] = qHatInvModq_0_offset;
    a.qhat_modp_offset[0] = qHatModp_0_offset;
    a.qhat_inv_offset[1] = qHatInvModq_1_offset;
    a.qhat_modp_offset[1] = qHatModp_1_offset;
    a.qhat_inv_offset[2] = qHatInvModq_2_offset;
    a.qhat_modp_offset[2] = qHatModp_2_offset;
    a.p_inv_mod_q_offset = PInvModq_offset;
    a.p_hat_inv_mod_p_offset = PHatInvModp_offset;
    a.p_hat_mod_q_offset = PHatModq_offset;
    a.qlql_offset = QlQlInvModqlDivqlModq_offset;
    a.qlinv_offset = qlInvModq_offset;
    if (op_code == AFHE_OP_LOAD_CONTEXT) {
        report(afhe_dispatch(b.ctx, &a), "OP 99");
        return;
    }
    // operands in, per op code (fhe_accel_top.cpp:220-326)
    const uint64_t LN = (uint64_t)L * n;
    uint64_t out_words = LN;
    rc = AFHE_OK;
    switch (op_code) {
    case AFHE_OP_NTT:
    case AFHE_OP_INTT:
        rc = put_poly(poly, src_a_offset, LN);
        break;
    case AFHE_OP_POLY_ADD:
    case AFHE_OP_POLY_SUB:
    case AFHE_OP_POLY_MUL_NTT:
        if ((rc = put_poly(poly, src_a_offset, LN)) == AFHE_OK) rc = put_poly(poly, src_b_offset, LN);
        break;
    case AFHE_OP_AUTOMORPHISM:
        if ((rc = put_poly(poly, src_a_offset, LN)) == AFHE_OK) rc = put_poly(poly, src_b_offset, n / 2);
        break;
    case AFHE_OP_RESCALE:
        if ((rc = put_poly(poly, src_a_offset, LN)) == AFHE_OK) rc = put_poly(poly, src_b_offset, LN);
        out_words = L >= 1 ? 2ull * (L - 1) * n : 0;
        break;
    case AFHE_OP_KEY_SWITCH: {
        const uint64_t SQ = (uint64_t)sizeQl * n;
        const uint64_t kw = 2ull * numPartQ * (sizeQl + sizeP) * n;
        bool have = false;
        for (auto& r : b.keys) have = have || (evk_offset >= r.first && evk_offset + kw <= r.first + r.second);
        if (!have) {
            if ((rc = put_key(key, evk_offset, kw)) != AFHE_OK) break;
            b.keys.push_back({evk_offset, kw});
        }
        rc = put_poly(poly, src_a_offset, SQ);
        out_words = 2 * SQ;
        break;
    }
    default:
        break;
    }
    if (rc != AFHE_OK) {
        report(rc, "copy operands");
        return;
    }
    if ((rc = afhe_dispatch(b.ctx, &a)) != AFHE_OK) {
        report(rc, "dispatch");
        return;
    }
    // the op's output back into the host arena (afhe_read_poly waits for it)
    report(afhe_read_poly(b.ctx, dst_offset, static_cast<uint64_t*>(poly_gmem) + dst_offset, out_words), "copy output");
}

}  // extern "C"
