// Test helper: the batched C-ABI operators and options that the native stage
// driver (anns_fhe_b200/csrc/ivfpq.cu) calls, as host stubs that record each
// call instead of running it. Linked with ivfpq.cu into a test library, it
// lets the CPU tests compare the native driver's operator sequence with the
// Python stage driver's (anns_fhe_b200/query.py, native=False), call by call.
#include <string>
#include <vector>

#include "internal.h"

namespace {
std::vector<std::string> g_log;
int64_t g_fused = 1, g_chunk = 0, g_ept = 8, g_slice = 13, g_fmin = 18;

void refs(std::string& s, const afhe_ct_ref* r, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i)
        s += " " + std::to_string(r[i].c0_offset) + ":" + std::to_string(r[i].c1_offset);
    s += " |";
}
void words(std::string& s, const uint64_t* p, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) s += " " + std::to_string(p[i]);
    s += " |";
}
std::string head(const char* name, uint32_t limbs, bool ks) {
    std::string s = std::string(name) + " " + std::to_string(limbs);
    if (ks)
        s += " fused=" + std::to_string(g_fused) + " chunk=" + std::to_string(g_chunk) + " ept=" + std::to_string(g_ept) +
             " slice=" + std::to_string(g_slice) + " fmin=" + std::to_string(g_fmin);
    return s + " |";
}
}  // namespace

namespace afhe {
int fail(afhe_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    g_log.push_back("error " + std::to_string(code) + " " + msg);
    return code;
}
}  // namespace afhe

extern "C" {

afhe_ctx* trace_ctx_new(uint32_t L, uint32_t n, uint32_t lanes) {
    afhe_ctx* c = new afhe_ctx();
    c->L = L;
    c->n = n;
    c->log_n = 0;
    while ((1u << c->log_n) < n) ++c->log_n;
    c->lanes = lanes;
    c->prm.poly_words = 1ull << 60;      // every recorded offset is in range
    g_log.clear();
    g_fused = 1;
    g_chunk = 0;
    g_ept = 8;
    g_slice = 13;
    g_fmin = 18;
    return c;
}
void trace_ctx_free(afhe_ctx* c) { delete c; }
uint32_t trace_count() { return (uint32_t)g_log.size(); }
const char* trace_line(uint32_t i) { return i < g_log.size() ? g_log[i].c_str() : ""; }

int afhe_ctx_set_option(afhe_ctx*, uint32_t option, int64_t value) {
    if (option == AFHE_OPT_KS_FUSED) g_fused = value;
    if (option == AFHE_OPT_CHUNK) g_chunk = value;
    if (option == AFHE_OPT_KS_EPT) g_ept = value;
    if (option == AFHE_OPT_KS_SLICE) g_slice = value;
    if (option == AFHE_OPT_FUSED_MIN) g_fmin = value;
    return AFHE_OK;
}
int afhe_ctx_get_option(afhe_ctx*, uint32_t option, int64_t* value) {
    *value = option == AFHE_OPT_KS_FUSED ? g_fused
             : option == AFHE_OPT_KS_EPT ? g_ept
             : option == AFHE_OPT_KS_SLICE ? g_slice
             : option == AFHE_OPT_FUSED_MIN ? g_fmin
                                            : g_chunk;
    return AFHE_OK;
}
int afhe_eval_add_batch(afhe_ctx*, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d, uint32_t n,
                        uint32_t limbs) {
    std::string s = head("add", limbs, false);
    refs(s, a, n), refs(s, b, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_sub_batch(afhe_ctx*, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d, uint32_t n,
                        uint32_t limbs) {
    std::string s = head("sub", limbs, false);
    refs(s, a, n), refs(s, b, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_add_plain_batch(afhe_ctx*, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d, uint32_t n,
                              uint32_t limbs) {
    std::string s = head("add_plain", limbs, false);
    refs(s, a, n), words(s, pt, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_copy_batch(afhe_ctx*, const afhe_ct_ref* a, const afhe_ct_ref* d, uint32_t n, uint32_t limbs) {
    std::string s = head("copy", limbs, false);
    refs(s, a, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_sub_plain_batch(afhe_ctx*, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d, uint32_t n,
                              uint32_t limbs) {
    std::string s = head("sub_plain", limbs, false);
    refs(s, a, n), words(s, pt, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_mult_plain_rescale_batch(afhe_ctx*, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d,
                                       uint32_t n, uint32_t limbs) {
    std::string s = head("mult_plain", limbs, false);
    refs(s, a, n), words(s, pt, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_mult_relin_rescale_batch(afhe_ctx*, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d,
                                       uint32_t n, uint32_t limbs) {
    std::string s = head("square", limbs, true);
    refs(s, a, n), refs(s, b, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_rotate_batch(afhe_ctx*, const afhe_ct_ref* in, const afhe_ct_ref* d, uint32_t n, int32_t rot,
                           uint32_t limbs) {
    std::string s = head("rotate", limbs, true) + " " + std::to_string(rot) + " |";
    refs(s, in, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_rotate_accumulate_batch(afhe_ctx*, const afhe_ct_ref* in, const afhe_ct_ref* acc, uint32_t n,
                                      int32_t rot, uint32_t limbs) {
    std::string s = head("rot_acc", limbs, true) + " " + std::to_string(rot) + " |";
    refs(s, in, n), refs(s, acc, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_automorphism_batch(afhe_ctx*, const uint64_t* src, const uint32_t* galois, const uint64_t* dst, uint32_t n,
                            uint32_t limbs) {
    std::string s = head("automorphism", limbs, false);
    words(s, src, n);
    for (uint32_t i = 0; i < n; ++i) s += " " + std::to_string(galois[i]);
    s += " |";
    words(s, dst, n);
    g_log.push_back(s);
    return AFHE_OK;
}
uint32_t afhe_galois_elt(uint32_t log_n, int32_t step) {
    // 5^step mod 2N (5^-1 for negative steps), as the library computes it
    const uint64_t m = 2ull << log_n;
    uint64_t g = 1, b = 5, e = (uint64_t)(step < 0 ? -(int64_t)step : step) % (m / 4);
    if (step < 0) {
        uint64_t inv = 1;
        for (uint64_t k = 0; k < m / 4 - 1; ++k) inv = inv * 5 % m;   // 5 has order N/2 mod 2N
        b = inv;
    }
    for (; e; e >>= 1, b = b * b % m)
        if (e & 1) g = g * b % m;
    return (uint32_t)g;
}
int afhe_eval_rotate_steps_batch(afhe_ctx*, const afhe_ct_ref* in, const afhe_ct_ref* d, const int32_t* steps,
                                 uint32_t n, uint32_t limbs) {
    std::string s = head("rotate_steps", limbs, true);
    for (uint32_t i = 0; i < n; ++i) s += " " + std::to_string(steps[i]);
    s += " |";
    refs(s, in, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}

int afhe_rescale_batch(afhe_ctx*, const afhe_ct_ref* a, const afhe_ct_ref* d, uint32_t n, uint32_t limbs) {
    std::string s = head("rescale", limbs, false);
    refs(s, a, n), refs(s, d, n);
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_diag_inner_batch(afhe_ctx*, const afhe_ct_ref* out, uint32_t n, const afhe_ct_ref* src, uint32_t nb,
                               const uint64_t* upt, const uint32_t* ugal, const uint32_t* first, uint64_t stride,
                               uint32_t limbs, uint32_t accumulate) {
    std::string s = head("diag_inner", limbs, false) + " nb=" + std::to_string(nb) + " stride=" +
                    std::to_string(stride) + " acc=" + std::to_string(accumulate) + " |";
    refs(s, out, n), refs(s, src, n * nb);
    for (uint32_t j = 0; j < n; ++j) {
        for (uint32_t k = first[j]; k < first[j + 1]; ++k) s += " " + std::to_string(upt[k]) + "@" + std::to_string(ugal[k]);
        s += " ;";
    }
    g_log.push_back(s);
    return AFHE_OK;
}
int afhe_eval_mac_plain_batch(afhe_ctx*, const afhe_ct_ref* out, const uint32_t* first, uint32_t n,
                              const afhe_mac_group* g, const afhe_mac_term* t, uint32_t limbs, uint32_t accumulate) {
    std::string s = head("mac", limbs, false) + " acc=" + std::to_string(accumulate) + " |";
    refs(s, out, n);
    for (uint32_t j = 0; j < n; ++j) {
        for (uint32_t k = first[j]; k < first[j + 1]; ++k) {
            s += " [" + std::to_string(g[k].src.c0_offset) + ":" + std::to_string(g[k].src.c1_offset);
            for (uint32_t x = g[k].first_term; x < g[k].first_term + g[k].n_terms; ++x)
                s += " " + std::to_string(t[x].pt) + "@" + std::to_string(t[x].galois);
            s += "]";
        }
        s += " ;";
    }
    g_log.push_back(s);
    return AFHE_OK;
}

}  // extern "C"
