// ref_shim.cpp -- extern "C" wrappers around the reference HLS C-simulation
// functions, compiled verbatim from the reference tree (see oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY. Built into oracle/_ref/libref_hls.so, which never
// enters git and is used only by tests/, smoke() and bench.py's CPU baseline
// legs as the bit-exact checker / timed reference. ap_uint<128> Barrett
// constants cross this boundary as (lo, hi) uint64_t pairs.
//
// Wrapped reference symbols (paths inside iheydardoost/ANNS_FHE):
//   mod_mul                 hardware_fpga_model/hls/src/mod_arith.cpp:15
//   ntt_forward             hardware_fpga_model/hls/src/ntt.cpp:4
//   intt_inverse            hardware_fpga_model/hls/src/ntt.cpp:46
//   poly_add/sub/mul        hardware_fpga_model/hls/src/poly_arith.cpp:3-38
//   automorphism            hardware_fpga_model/hls/src/automorphism.cpp:3
//   rescale                 hardware_fpga_model/hls/src/rescale.cpp:3
//   fast_bases_conv         hardware_fpga_model/hls/src/key_switch.cpp:7
//   approx_mod_down         hardware_fpga_model/hls/src/key_switch.cpp:62
//   key_switch              hardware_fpga_model/hls/src/key_switch.cpp:167
//   fhe_accel_top           hardware_fpga_model/hls/src/fhe_accel_top.cpp:90
//   SimMemoryBus            cpp_host_model/src/sim_memory_bus.h:10-34
//
// The same shim is built against the verbatim sources (N = 16384) and against
// copies whose ring-degree literals the recipe rewrites (N = 8192, 32768); it
// takes the ring degree from the sources' own hls_params.h.
#include <cstdint>
#include <cstring>
#include <vector>

#include "mod_arith.h"
#include "ntt.h"
#include "poly_arith.h"
#include "automorphism.h"
#include "rescale.h"
#include "key_switch.h"
#include "fhe_accel_top.h"
#include "sim_memory_bus.h"

static inline ap_uint<128> mk128(uint64_t lo, uint64_t hi) {
    return (ap_uint<128>(hi) << 64) | ap_uint<128>(lo);
}

static void pack_beats(const uint64_t* words, size_t n_words, std::vector<ap_uint<512>>& beats) {
    beats.assign((n_words + 7) / 8, ap_uint<512>(0));
    for (size_t i = 0; i < n_words; ++i) beats[i / 8].w[i % 8] = words[i];
}

static void unpack_beats(const std::vector<ap_uint<512>>& beats, uint64_t* words, size_t n_words) {
    for (size_t i = 0; i < n_words; ++i) words[i] = beats[i / 8].w[i % 8];
}

// Scalar / array registers of fhe_accel_top, in one plain struct.
struct ref_top_args {
    uint32_t op_code;
    uint32_t src_a_offset, src_b_offset, dst_offset;
    uint64_t evk_offset;
    uint32_t active_limbs, prime_idx, galois_elt;
    uint32_t sizeQl, sizeP, numPartQ, alpha;
    uint64_t rns_primes[15];
    uint64_t p_primes[4];
    uint64_t barrett_m_q_lo[15], barrett_m_q_hi[15];
    uint32_t barrett_k_q[15];
    uint64_t barrett_m_p_lo[4], barrett_m_p_hi[4];
    uint32_t barrett_k_p[4];
    uint64_t n_inv_q[15];
    uint64_t n_inv_p[4];
    uint64_t n_inv_mod_q_last;
    uint32_t table_offsets[15];  // twiddles_q .. qlInvModq, in header order
};

extern "C" {

uint32_t ref_ring_degree(void) { return (uint32_t)N; }

uint64_t ref_mod_add(uint64_t a, uint64_t b, uint64_t q) { return mod_add(a, b, q); }
uint64_t ref_mod_sub(uint64_t a, uint64_t b, uint64_t q) { return mod_sub(a, b, q); }
uint64_t ref_mod_mul(uint64_t a, uint64_t b, uint64_t q, uint64_t m_lo, uint64_t m_hi, uint32_t k) {
    return mod_mul(a, b, q, mk128(m_lo, m_hi), k);
}

void ref_ntt_forward(uint64_t* a, const uint64_t* tw, uint64_t q, uint64_t m_lo, uint64_t m_hi, uint32_t k) {
    ntt_forward(a, tw, q, mk128(m_lo, m_hi), k);
}

void ref_intt_inverse(uint64_t* a, const uint64_t* itw, uint64_t n_inv, uint64_t q,
                      uint64_t m_lo, uint64_t m_hi, uint32_t k) {
    intt_inverse(a, itw, n_inv, q, mk128(m_lo, m_hi), k);
}

void ref_poly_add(const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t q) { poly_add(a, b, out, q); }
void ref_poly_sub(const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t q) { poly_sub(a, b, out, q); }
void ref_poly_mul(const uint64_t* a, const uint64_t* b, uint64_t* out, uint64_t q,
                  uint64_t m_lo, uint64_t m_hi, uint32_t k) {
    poly_mul(a, b, out, q, mk128(m_lo, m_hi), k);
}

void ref_automorphism(const uint64_t* a, uint64_t* out, const uint64_t* map64) { automorphism(a, out, map64); }

void ref_rescale(const uint64_t* a_in, uint64_t* a_out, uint32_t num_limbs, const uint64_t* q,
                 const uint64_t* m_lo, const uint64_t* m_hi, const uint32_t* k,
                 const uint64_t* inv_tw_last, const uint64_t* tw, uint64_t n_inv_last,
                 const uint64_t* qlql, const uint64_t* qlinv) {
    std::vector<ap_uint<128>> m(num_limbs);
    for (uint32_t i = 0; i < num_limbs; ++i) m[i] = mk128(m_lo[i], m_hi[i]);
    rescale(a_in, a_out, num_limbs, q, m.data(), k, inv_tw_last, tw, n_inv_last, qlql, qlinv);
}

void ref_fast_bases_conv(const uint64_t* in, uint64_t* out, uint32_t n_in, uint32_t n_out,
                         const uint64_t* in_primes, const uint64_t* out_primes,
                         const uint64_t* qhat_inv, const uint64_t* qhat_modp,
                         const uint64_t* m_in_lo, const uint64_t* m_in_hi, const uint32_t* k_in,
                         const uint64_t* m_out_lo, const uint64_t* m_out_hi, const uint32_t* k_out) {
    std::vector<ap_uint<128>> mi(n_in), mo(n_out);
    for (uint32_t i = 0; i < n_in; ++i) mi[i] = mk128(m_in_lo[i], m_in_hi[i]);
    for (uint32_t i = 0; i < n_out; ++i) mo[i] = mk128(m_out_lo[i], m_out_hi[i]);
    std::vector<uint64_t> buf((size_t)n_in * N);
    fast_bases_conv(in, out, n_in, n_out, in_primes, out_primes, qhat_inv, qhat_modp,
                    mi.data(), k_in, mo.data(), k_out, buf.data());
}

void ref_approx_mod_down(const uint64_t* in, uint64_t* out, uint32_t nq, uint32_t np,
                         const uint64_t* q, const uint64_t* p,
                         const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p, const uint64_t* p_hat_mod_q,
                         const uint64_t* inv_tw_p, const uint64_t* tw_q,
                         const uint64_t* mp_lo, const uint64_t* mp_hi, const uint32_t* kp,
                         const uint64_t* mq_lo, const uint64_t* mq_hi, const uint32_t* kq,
                         const uint64_t* n_inv_p) {
    std::vector<ap_uint<128>> mp(np), mq(nq);
    for (uint32_t i = 0; i < np; ++i) mp[i] = mk128(mp_lo[i], mp_hi[i]);
    for (uint32_t i = 0; i < nq; ++i) mq[i] = mk128(mq_lo[i], mq_hi[i]);
    std::vector<uint64_t> buf_p((size_t)np * N), part((size_t)nq * N), xq((size_t)np * N);
    approx_mod_down(in, out, nq, np, q, p, p_inv_mod_q, p_hat_inv_mod_p, p_hat_mod_q, inv_tw_p, tw_q,
                    mp.data(), kp, mq.data(), kq, n_inv_p, buf_p.data(), part.data(), xq.data());
}

// key_words: the evaluation-key arena as 64-bit words (packed into 512-bit beats here).
void ref_key_switch(const uint64_t* c_in, const uint64_t* key_words, uint64_t n_key_words,
                    uint64_t evk_a_offset, uint64_t evk_b_offset, uint64_t* out0, uint64_t* out1,
                    uint32_t sizeQl, uint32_t sizeP, uint32_t numPartQ, uint32_t alpha,
                    const uint64_t* q, const uint64_t* p,
                    const uint64_t* mq_lo, const uint64_t* mq_hi, const uint32_t* kq,
                    const uint64_t* mp_lo, const uint64_t* mp_hi, const uint32_t* kp,
                    const uint64_t* tw_q, const uint64_t* itw_q, const uint64_t* tw_p, const uint64_t* itw_p,
                    const uint64_t* n_inv_q, const uint64_t* n_inv_p,
                    const uint64_t* qhi0, const uint64_t* qhm0, const uint64_t* qhi1, const uint64_t* qhm1,
                    const uint64_t* qhi2, const uint64_t* qhm2,
                    const uint64_t* p_inv_mod_q, const uint64_t* p_hat_inv_mod_p, const uint64_t* p_hat_mod_q) {
    std::vector<ap_uint<128>> mq(sizeQl), mp(sizeP);
    for (uint32_t i = 0; i < sizeQl; ++i) mq[i] = mk128(mq_lo[i], mq_hi[i]);
    for (uint32_t i = 0; i < sizeP; ++i) mp[i] = mk128(mp_lo[i], mp_hi[i]);
    std::vector<ap_uint<512>> beats;
    pack_beats(key_words, n_key_words, beats);
    const size_t W = (size_t)MAX_LIMBS * N;
    std::vector<uint64_t> ext0(W), ext1(W), parts(W), compl_(W), digit(W);
    key_switch(c_in, beats.data(), evk_a_offset, evk_b_offset, out0, out1, sizeQl, sizeP, numPartQ, alpha,
               q, p, mq.data(), kq, mp.data(), kp, tw_q, itw_q, tw_p, itw_p, n_inv_q, n_inv_p,
               qhi0, qhm0, qhi1, qhm1, qhi2, qhm2, p_inv_mod_q, p_hat_inv_mod_p, p_hat_mod_q,
               ext0.data(), ext1.data(), parts.data(), compl_.data(), digit.data());
}

static void call_top(ap_uint<512>* pg, ap_uint<512>* kg, const ref_top_args* a) {
    uint64_t rns[15], pp[4], nq[15], np[4];
    ap_uint<128> mq[15], mp[4];
    uint32_t kq[15], kp[4];
    for (int i = 0; i < 15; ++i) {
        rns[i] = a->rns_primes[i]; nq[i] = a->n_inv_q[i]; kq[i] = a->barrett_k_q[i];
        mq[i] = mk128(a->barrett_m_q_lo[i], a->barrett_m_q_hi[i]);
    }
    for (int i = 0; i < 4; ++i) {
        pp[i] = a->p_primes[i]; np[i] = a->n_inv_p[i]; kp[i] = a->barrett_k_p[i];
        mp[i] = mk128(a->barrett_m_p_lo[i], a->barrett_m_p_hi[i]);
    }
    const uint32_t* o = a->table_offsets;
    fhe_accel_top(pg, kg, a->op_code, a->src_a_offset, a->src_b_offset, a->dst_offset,
                  a->evk_offset, a->active_limbs, a->prime_idx, a->galois_elt,
                  a->sizeQl, a->sizeP, a->numPartQ, a->alpha,
                  rns, pp, mq, kq, mp, kp, nq, np, a->n_inv_mod_q_last,
                  o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8], o[9], o[10], o[11], o[12], o[13], o[14]);
}

// The reference's own memory bus (cpp_host_model/src/sim_memory_bus.h:10-34)
// held across calls, so that a sequence of fhe_accel_top calls runs on
// resident arenas the way FHEHostDriver::dispatch (fhe_host_driver.cpp:177-204)
// drives them.
void* ref_bus_new(uint64_t poly_words, uint64_t key_words) { return new SimMemoryBus(poly_words, key_words); }
void ref_bus_free(void* bus) { delete static_cast<SimMemoryBus*>(bus); }
void ref_bus_write_poly(void* bus, uint64_t off, const uint64_t* src, uint64_t count) {
    static_cast<SimMemoryBus*>(bus)->write_poly((uint32_t)off, src, count);
}
void ref_bus_read_poly(void* bus, uint64_t off, uint64_t* dst, uint64_t count) {
    static_cast<SimMemoryBus*>(bus)->read_poly((uint32_t)off, dst, count);
}
void ref_bus_write_key(void* bus, uint64_t off, const uint64_t* src, uint64_t count) {
    static_cast<SimMemoryBus*>(bus)->write_key(off, src, count);
}
void ref_bus_accel_top(void* bus, const ref_top_args* a) {
    SimMemoryBus* b = static_cast<SimMemoryBus*>(bus);
    call_top(b->poly_gmem_ptr(), b->key_gmem_ptr(), a);
}

// One fhe_accel_top call over word arenas. The arenas are packed into 512-bit
// beats, the kernel runs, and both arenas are unpacked back in place.
void ref_fhe_accel_top(uint64_t* poly_words, uint64_t n_poly_words, uint64_t* key_words, uint64_t n_key_words,
                       const ref_top_args* a) {
    std::vector<ap_uint<512>> pg, kg;
    pack_beats(poly_words, n_poly_words, pg);
    pack_beats(key_words, n_key_words, kg);
    call_top(pg.data(), kg.data(), a);
    unpack_beats(pg, poly_words, n_poly_words);
    unpack_beats(kg, key_words, n_key_words);
}

}  // extern "C"
