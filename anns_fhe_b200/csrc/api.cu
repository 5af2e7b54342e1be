// api.cu -- C ABI of the CKKS evaluation core: context, arenas, the
// fhe_accel_top-compatible dispatcher and the FHEHostDriver composite operators.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "tables.h"
#include "lanes.h"

using namespace afhe;

namespace afhe {
thread_local std::string g_last_error;

int fail(afhe_ctx* ctx, int code, const std::string& msg) {
    g_last_error = msg;
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(afhe_ctx* ctx, cudaError_t e, const char* where) {
    // a failed runtime call (an out-of-memory cudaMalloc, say) also records
    // its error as the thread's last error: clear it here, or the launch
    // check of the next, unrelated call (cudaGetLastError) reports it again
    (void)cudaGetLastError();
    return fail(ctx, AFHE_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

u64 host_shoup(u64 w, u64 q) { return (u64)(((unsigned __int128)w << 64) / q); }

// The primitive 2N-th root behind prime i's twiddles (Q primes first, then
// P): the one the parameters name, else the smallest.
u64 root_of(const afhe_ctx* ctx, uint32_t i) {
    const u64 psi = i < ctx->L ? ctx->prm.psi_q[i] : ctx->prm.psi_p[i - ctx->L];
    const u64 q = i < ctx->L ? ctx->prm.q[i] : ctx->prm.p[i - ctx->L];
    return psi ? psi : min_primitive_root(ctx->log_n, q);
}

int ring_put(afhe_ctx* ctx, const void* src, size_t words, u64** dev) {
    DescRing& r = ctx->ring;
    if (words > r.seg_words) return fail(ctx, AFHE_E_ARG, "descriptor too large for the descriptor ring");
    if (r.pos + words > r.seg_words) {
        CK(cudaEventRecord(r.ev[r.cur], ctx->st));
        r.used[r.cur] = 1;
        r.cur = (r.cur + 1) % r.nseg;
        if (r.used[r.cur]) CK(cudaEventSynchronize(r.ev[r.cur]));
        r.pos = 0;
    }
    const size_t at = r.cur * r.seg_words + r.pos;
    std::memcpy(r.host + at, src, words * sizeof(u64));
    CK(cudaMemcpyAsync(r.dev + at, r.host + at, words * sizeof(u64), cudaMemcpyHostToDevice, ctx->st));
    *dev = r.dev + at;
    r.pos += (words + 31) & ~(size_t)31;
    return AFHE_OK;
}

int zf_from(afhe_ctx* ctx, const u64* vals, uint32_t n, ZField* out) {
    if (n == 0) { *out = zf_const(0); return AFHE_OK; }
    const u64 stride = n > 1 ? vals[1] - vals[0] : 0;
    bool prog = true;
    for (uint32_t i = 1; i < n && prog; ++i) prog = (vals[i] - vals[i - 1]) == stride;
    if (prog) { *out = zf_stride(vals[0], stride); return AFHE_OK; }
    if (n > ctx->ring.seg_words) return fail(ctx, AFHE_E_ARG, "batch too large for the descriptor ring");
    u64* dev = nullptr;
    int rc = ring_put(ctx, vals, n, &dev);
    if (rc != AFHE_OK) return rc;
    ZField f{};
    f.arr = dev;
    *out = f;
    return AFHE_OK;
}
}  // namespace afhe

namespace {

PrimeConst host_prime_const(u64 q, u64 ninv, u64 itw1) {
    PrimeConst c;
    c.q = q;
    ModConst m = make_modconst(q);
    c.r64 = m.r64;
    c.r64_sh = m.r64_sh;
    c.one_sh = m.one_sh;
    c.ninv = ninv % q;
    c.ninv_sh = host_shoup(c.ninv, q);
    c.w1ninv = (u64)((unsigned __int128)(itw1 % q) * c.ninv % q);
    c.w1ninv_sh = host_shoup(c.w1ninv, q);
    return c;
}

template <class T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

// ===========================================================================
// host-only number theory
// ===========================================================================
extern "C" {

int afhe_find_ntt_primes(uint32_t log_n, uint32_t bits, uint32_t count, const uint64_t* exclude, uint32_t n_exclude,
                         uint64_t* out) {
    try {
        std::vector<u64> ex(exclude, exclude + n_exclude);
        auto v = find_ntt_primes(log_n, bits, count, ex);
        std::copy(v.begin(), v.end(), out);
        return AFHE_OK;
    } catch (const std::exception& e) {
        return fail(nullptr, AFHE_E_ARG, e.what());
    }
}

uint64_t afhe_min_primitive_root(uint32_t log_n, uint64_t q) {
    try {
        return min_primitive_root(log_n, q);
    } catch (...) {
        return 0;
    }
}

int afhe_gen_twiddles(uint32_t log_n, uint64_t q, uint64_t psi, uint64_t* tw, uint64_t* itw) {
    if (log_n < 1 || log_n > 17 || q < 3) return fail(nullptr, AFHE_E_ARG, "gen_twiddles: bad arguments");
    gen_twiddles(log_n, q, psi, tw, itw);
    return AFHE_OK;
}

void afhe_barrett_constant(uint64_t q, uint64_t* m_lo, uint64_t* m_hi, uint32_t* k) { barrett_constant(q, m_lo, m_hi, k); }

uint64_t afhe_inv_mod(uint64_t a, uint64_t q) { return inv_mod(a, q); }

uint32_t afhe_galois_elt(uint32_t log_n, int32_t step) { return galois_elt_for_step(log_n, step); }

int afhe_automorphism_map(uint32_t log_n, uint32_t galois_elt, uint32_t* map) {
    if ((galois_elt & 1u) == 0) return fail(nullptr, AFHE_E_ARG, "galois element must be odd");
    automorphism_map(log_n, galois_elt, map);
    return AFHE_OK;
}

int afhe_part_qhat_tables(const uint64_t* q, uint32_t sizeQl, uint32_t alpha, uint32_t part, const uint64_t* p,
                          uint32_t num_p, uint64_t* qhat_inv, uint64_t* qhat_modp) {
    if (alpha == 0 || sizeQl == 0 || part >= (sizeQl + alpha - 1) / alpha)
        return fail(nullptr, AFHE_E_ARG, "part_qhat_tables: bad partition");
    part_qhat_tables(q, sizeQl, alpha, part, p, num_p, qhat_inv, qhat_modp);
    return AFHE_OK;
}

int afhe_moddown_tables(const uint64_t* q, uint32_t sizeQl, const uint64_t* p, uint32_t num_p, uint64_t* p_inv_mod_q,
                        uint64_t* p_hat_inv_mod_p, uint64_t* p_hat_mod_q) {
    moddown_tables(q, sizeQl, p, num_p, p_inv_mod_q, p_hat_inv_mod_p, p_hat_mod_q);
    return AFHE_OK;
}

int afhe_rescale_tables(const uint64_t* q, uint32_t sizeQl, uint64_t* qlql, uint64_t* qlinv) {
    if (sizeQl < 2) return fail(nullptr, AFHE_E_ARG, "rescale needs at least two limbs");
    rescale_tables(q, sizeQl, qlql, qlinv);
    return AFHE_OK;
}

const char* afhe_status_string(int s) {
    switch (s) {
    case AFHE_OK: return "ok";
    case AFHE_E_ARG: return "bad argument";
    case AFHE_E_RANGE: return "offset out of arena range";
    case AFHE_E_NOKEY: return "rotation key not found";
    case AFHE_E_LEVEL: return "level not supported by loaded tables or key";
    case AFHE_E_BUDGET: return "admission budget exceeded";
    case AFHE_E_TIMEOUT: return "bounded device wait timed out";
    case AFHE_E_CUDA: return "CUDA error";
    case AFHE_E_STATE: return "invalid call order";
    default: return "unknown status";
    }
}

const char* afhe_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

// ===========================================================================
// context
// ===========================================================================
namespace {

int build_native_tables(afhe_ctx* ctx) {
    const uint32_t n = ctx->n, L = ctx->L, K = ctx->K, np = L + K;
    std::vector<u64> primes(np);
    for (uint32_t i = 0; i < L; ++i) primes[i] = ctx->prm.q[i];
    for (uint32_t k = 0; k < K; ++k) primes[L + k] = ctx->prm.p[k];

    std::vector<u64> tw(n), itw(n);
    std::vector<ulonglong2> tw2((size_t)np * n), itw2((size_t)np * n);
    std::vector<PrimeConst> pc(np);
    for (uint32_t i = 0; i < np; ++i) {
        u64 q = primes[i];
        u64 psi = root_of(ctx, i);
        gen_twiddles(ctx->log_n, q, psi, tw.data(), itw.data());
        for (uint32_t j = 0; j < n; ++j) {
            tw2[(size_t)i * n + j] = make_ulonglong2(tw[j], host_shoup(tw[j], q));
            itw2[(size_t)i * n + j] = make_ulonglong2(itw[j], host_shoup(itw[j], q));
        }
        pc[i] = host_prime_const(q, inv_mod(n % q, q), itw[1]);
    }
    DevPrimeSet& s = ctx->nat;
    s.count = np;
    CK(dalloc(&s.pc, np));
    CK(dalloc(&s.tw2, (size_t)np * n));
    CK(dalloc(&s.itw2, (size_t)np * n));
    CK(cudaMemcpy(s.pc, pc.data(), np * sizeof(PrimeConst), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s.tw2, tw2.data(), tw2.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s.itw2, itw2.data(), itw2.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice));

    // per-level CRT tables, each followed by its Shoup companions
    std::vector<u64> buf;
    struct Ref { size_t v, sh; };
    auto push = [&](const std::vector<u64>& vals, const std::vector<u64>& mods) -> Ref {
        Ref r;
        r.v = buf.size();
        buf.insert(buf.end(), vals.begin(), vals.end());
        r.sh = buf.size();
        for (size_t i = 0; i < vals.size(); ++i) buf.push_back(host_shoup(vals[i], mods[i]));
        return r;
    };
    struct LvlRefs {
        Ref qi[AFHE_MAX_PARTS], qm[AFHE_MAX_PARTS], pinv, phinv, phq, qlql, qlinv;
        uint32_t parts;
    };
    std::vector<LvlRefs> refs(L + 1);
    const u64* q = primes.data();
    const u64* p = primes.data() + L;
    for (uint32_t lvl = 1; lvl <= L; ++lvl) {
        LvlRefs& R = refs[lvl];
        R.parts = (lvl + ctx->alpha - 1) / ctx->alpha;
        for (uint32_t j = 0; j < R.parts; ++j) {
            uint32_t start = j * ctx->alpha;
            uint32_t size = (j == R.parts - 1) ? lvl - start : ctx->alpha;
            uint32_t row = lvl - size + K;
            std::vector<u64> qi(size), qm((size_t)size * row), mi(size), mm((size_t)size * row);
            part_qhat_tables(q, lvl, ctx->alpha, j, p, K, qi.data(), qm.data());
            std::vector<u64> outp;
            for (uint32_t i = 0; i < lvl; ++i)
                if (i < start || i >= start + size) outp.push_back(q[i]);
            for (uint32_t k = 0; k < K; ++k) outp.push_back(p[k]);
            for (uint32_t i = 0; i < size; ++i) {
                mi[i] = q[start + i];
                for (uint32_t c = 0; c < row; ++c) mm[(size_t)i * row + c] = outp[c];
            }
            R.qi[j] = push(qi, mi);
            R.qm[j] = push(qm, mm);
        }
        std::vector<u64> pinv(lvl), phinv(K), phq((size_t)K * lvl), mq(lvl), mp(K), mphq((size_t)K * lvl);
        moddown_tables(q, lvl, p, K, pinv.data(), phinv.data(), phq.data());
        for (uint32_t i = 0; i < lvl; ++i) mq[i] = q[i];
        for (uint32_t k = 0; k < K; ++k) {
            mp[k] = p[k];
            for (uint32_t i = 0; i < lvl; ++i) mphq[(size_t)k * lvl + i] = q[i];
        }
        R.pinv = push(pinv, mq);
        R.phinv = push(phinv, mp);
        R.phq = push(phq, mphq);
        std::vector<u64> qlql(lvl > 1 ? lvl - 1 : 1, 0), qlinv(lvl > 1 ? lvl - 1 : 1, 0), mr(lvl > 1 ? lvl - 1 : 1, 3);
        if (lvl > 1) {
            rescale_tables(q, lvl, qlql.data(), qlinv.data());
            for (uint32_t i = 0; i + 1 < lvl; ++i) mr[i] = q[i];
        }
        R.qlql = push(qlql, mr);
        R.qlinv = push(qlinv, mr);
    }
    CK(dalloc(&ctx->lvbuf, buf.size()));
    CK(cudaMemcpy(ctx->lvbuf, buf.data(), buf.size() * 8, cudaMemcpyHostToDevice));
    ctx->lv.assign(L + 1, OpTabs{});
    for (uint32_t lvl = 1; lvl <= L; ++lvl) {
        OpTabs& t = ctx->lv[lvl];
        const LvlRefs& R = refs[lvl];
        const u64* b = ctx->lvbuf;
        t.pt = s.view();
        t.p_base = L;
        t.sizeQl = lvl;
        t.parts = R.parts;
        t.alpha = ctx->alpha;
        for (uint32_t j = 0; j < R.parts; ++j) {
            t.qhat_inv[j] = b + R.qi[j].v;
            t.qhat_inv_sh[j] = b + R.qi[j].sh;
            t.qhat_modp[j] = b + R.qm[j].v;
            t.qhat_modp_sh[j] = b + R.qm[j].sh;
        }
        t.p_inv_mod_q = b + R.pinv.v;
        t.p_inv_mod_q_sh = b + R.pinv.sh;
        t.phat_inv_modp = b + R.phinv.v;
        t.phat_inv_modp_sh = b + R.phinv.sh;
        t.phat_modq = b + R.phq.v;
        t.phat_modq_sh = b + R.phq.sh;
        t.qlql = b + R.qlql.v;
        t.qlql_sh = b + R.qlql.sh;
        t.qlinv = b + R.qlinv.v;
        t.qlinv_sh = b + R.qlinv.sh;
    }
    // the same tables as one device array, for launches whose entries run at
    // different levels
    CK(dalloc(&ctx->lv_dev, L + 1));
    CK(cudaMemcpy(ctx->lv_dev, ctx->lv.data(), (L + 1) * sizeof(OpTabs), cudaMemcpyHostToDevice));

    // job templates
    std::vector<LimbJob> jq(np);
    for (uint32_t i = 0; i < np; ++i) {
        LimbJob j{};
        j.src = j.dst = j.out = (u64)i * n;
        j.prime = i;
        j.aux = i < L ? i : i - L;
        jq[i] = j;
    }
    CK(dalloc(&ctx->jobs_qp, np));
    CK(cudaMemcpy(ctx->jobs_qp, jq.data(), np * sizeof(LimbJob), cudaMemcpyHostToDevice));
    ctx->lvjobs.assign(L + 1, LevelJobs{});
    const u64 S = (u64)L + K;
    for (uint32_t lvl = 1; lvl <= L; ++lvl) {
        std::vector<LimbJob> jm;
        uint32_t parts = (lvl + ctx->alpha - 1) / ctx->alpha;
        for (uint32_t j = 0; j < parts; ++j) {
            uint32_t start = j * ctx->alpha;
            uint32_t size = (j == parts - 1) ? lvl - start : ctx->alpha;
            uint32_t kpos = 0;
            for (uint32_t i = 0; i < lvl + K; ++i) {
                bool isq = i < lvl;
                if (isq && i >= start && i < start + size) continue;
                uint32_t slot = isq ? i : L + (i - lvl);
                LimbJob jb{};
                jb.src = 0;
                jb.dst = jb.out = ((u64)j * S + slot) * n;
                jb.prime = slot;
                jb.aux = (j << 16) | kpos++;
                jm.push_back(jb);
            }
        }
        LevelJobs& lj = ctx->lvjobs[lvl];
        lj.n_modup = (uint32_t)jm.size();
        CK(dalloc(&lj.modup, jm.size()));
        CK(cudaMemcpy(lj.modup, jm.data(), jm.size() * sizeof(LimbJob), cudaMemcpyHostToDevice));
    }
    return AFHE_OK;
}

}  // namespace

extern "C" {

int afhe_ctx_create(const afhe_params* prm, afhe_ctx** out) {
    if (!prm || !out) return fail(nullptr, AFHE_E_ARG, "null argument");
    *out = nullptr;
    if (prm->log_n < 10 || prm->log_n > 16) return fail(nullptr, AFHE_E_ARG, "log_n must be in [10, 16]");
    if (prm->num_q < 1 || prm->num_q > AFHE_MAX_Q || prm->num_p < 1 || prm->num_p > AFHE_MAX_P)
        return fail(nullptr, AFHE_E_ARG, "prime counts out of range");
    if (prm->alpha < 1 || (prm->num_q + prm->alpha - 1) / prm->alpha > AFHE_MAX_PARTS)
        return fail(nullptr, AFHE_E_ARG, "alpha gives too many digits");
    const u64 m2n = 2ull << prm->log_n;
    std::vector<u64> all;
    for (uint32_t i = 0; i < prm->num_q; ++i) all.push_back(prm->q[i]);
    for (uint32_t i = 0; i < prm->num_p; ++i) all.push_back(prm->p[i]);
    for (size_t i = 0; i < all.size(); ++i) {
        u64 q = all[i];
        if (q >= (1ull << 61) || q % m2n != 1 || !is_prime64(q))
            return fail(nullptr, AFHE_E_ARG, "every prime must be < 2^61, prime and == 1 mod 2N");
        for (size_t j = 0; j < i; ++j)
            if (all[j] == q) return fail(nullptr, AFHE_E_ARG, "primes must be distinct");
        const u64 psi = i < prm->num_q ? prm->psi_q[i] : prm->psi_p[i - prm->num_q];
        if (psi != 0 && (psi >= q || pow_mod(psi, 1ull << prm->log_n, q) != q - 1))
            return fail(nullptr, AFHE_E_ARG, "psi must be a primitive 2N-th root of unity mod its prime");
    }
    afhe_ctx* ctx = new afhe_ctx();
    ctx->prm = *prm;
    ctx->log_n = (int)prm->log_n;
    ctx->n = 1u << prm->log_n;
    ctx->L = prm->num_q;
    ctx->K = prm->num_p;
    ctx->alpha = prm->alpha;
    ctx->dnum = (ctx->L + ctx->alpha - 1) / ctx->alpha;
    ctx->device = prm->device;
    int rc = AFHE_OK;
    do {
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "cudaSetDevice"); break; }
        e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "cudaStreamCreate"); break; }
        // poly_gmem and the context-private scratch share one allocation so a
        // kernel can address both from one base: scratch word w is poly word
        // poly_words + w.
        ctx->lanes = prm->max_batch ? prm->max_batch : 64;
        {
            const char* v = std::getenv("AFHE_KS_FUSED");
            ctx->ks_fused = key_switch_fused_supported(ctx->log_n) && !(v && v[0] == '0');
            // the one-kernel path carries a ciphertext per CTA (per cluster of
            // N / 2^13 CTAs above N = 2^13): below half a wave of SMs a launch
            // leaves most of the GPU idle, and the limb-parallel multi-kernel
            // path is faster
            int sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
            const int cl = ctx->log_n > 13 ? 1 << (ctx->log_n - 13) : 1;
            ctx->fused_min = (uint32_t)std::max(1, sms / (2 * cl));
            const char* m = std::getenv("AFHE_FUSED_MIN");
            if (m && std::atoi(m) >= 1) ctx->fused_min = (uint32_t)std::atoi(m);
        }
        if (ctx->lanes > 4096) { rc = fail(ctx, AFHE_E_ARG, "max_batch must be <= 4096"); break; }
        ctx->scr_words = (size_t)ctx->lanes * lane_words(ctx);
        e = dalloc(&ctx->poly, prm->poly_words + ctx->scr_words);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "alloc poly_gmem + scratch"); break; }
        ctx->scr = ctx->poly + prm->poly_words;
        e = dalloc(&ctx->key, prm->key_words);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "alloc key_gmem"); break; }
        e = cudaMemset(ctx->poly, 0, (prm->poly_words + ctx->scr_words) * 8);
        if (e == cudaSuccess) e = cudaMemset(ctx->key, 0, std::max<u64>(prm->key_words, 1) * 8);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "clear arenas"); break; }
        rc = build_native_tables(ctx);
        if (rc != AFHE_OK) break;
        // afhe_key_switch_noalloc must allocate nothing when called; with
        // CUDA's lazy module loading the first lookup of its static array
        // loads (and so allocates) it, so the lookup happens here. A failure
        // is reported by that entry point, not by context creation.
        ctx->noalloc_err = noalloc_scratch_address(&ctx->noalloc_scr);
        if (ctx->noalloc_err != cudaSuccess) {
            ctx->noalloc_scr = nullptr;
            cudaGetLastError();
        }
        DescRing& r = ctx->ring;
        r.seg_words = 1u << 16;
        r.nseg = 32;
        e = cudaHostAlloc((void**)&r.host, r.seg_words * r.nseg * sizeof(u64), cudaHostAllocDefault);
        if (e == cudaSuccess) e = dalloc(&r.dev, r.seg_words * r.nseg);
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "alloc descriptor ring"); break; }
        r.ev.assign(r.nseg, nullptr);
        r.used.assign(r.nseg, 0);
        for (auto& ev : r.ev) {
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) break;
        }
        if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "descriptor ring events"); break; }
    } while (0);
    if (rc != AFHE_OK) {
        std::string msg = ctx->err;
        afhe_ctx_destroy(ctx);
        g_last_error = msg;
        return rc;
    }
    *out = ctx;
    return AFHE_OK;
}

int afhe_ctx_destroy(afhe_ctx* ctx) {
    if (!ctx) return AFHE_OK;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    auto fr = [](void* p) { if (p) cudaFree(p); };
    fr(ctx->poly); fr(ctx->key); fr(ctx->lvbuf); fr(ctx->lv_dev); fr(ctx->jobs_qp);
    for (auto& j : ctx->lvjobs) fr(j.modup);
    for (DevPrimeSet* s : {&ctx->nat, &ctx->ld}) { fr(s->pc); fr(s->tw); fr(s->itw); fr(s->tw2); fr(s->itw2); }
    fr(ctx->ld_crt); fr(ctx->ld_crt_sh); fr(ctx->ld_mod);
    for (auto& kv : ctx->rot) fr(kv.second.map);
    for (auto& kv : ctx->auto_maps) fr(kv.second);
    fr(ctx->dec_ws);
    free_key_preps(ctx);
    fr(ctx->ring.dev);
    if (ctx->ring.host) cudaFreeHost(ctx->ring.host);
    for (auto& ev : ctx->ring.ev) if (ev) cudaEventDestroy(ev);
    for (auto& ev : ctx->fences) if (ev) cudaEventDestroy(ev);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return AFHE_OK;
}

int afhe_sync(afhe_ctx* ctx) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    CK(cudaStreamSynchronize(ctx->st));
    return AFHE_OK;
}

void* afhe_stream(afhe_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }
uint64_t* afhe_poly_gmem(afhe_ctx* ctx) { return ctx ? ctx->poly : nullptr; }
uint64_t* afhe_key_gmem(afhe_ctx* ctx) { return ctx ? ctx->key : nullptr; }
uint64_t afhe_scratch_words(afhe_ctx* ctx) { return ctx ? (uint64_t)ctx->scr_words : 0; }

static int arena_copy(afhe_ctx* ctx, bool poly, bool to_dev, u64 off, void* host, u64 count, bool async) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    u64 size = poly ? ctx->prm.poly_words : ctx->prm.key_words;
    if (!range_ok(off, count, size)) return fail(ctx, AFHE_E_RANGE, "arena access out of range");
    if (count == 0) return AFHE_OK;
    if (!host) return fail(ctx, AFHE_E_ARG, "null host buffer");
    u64* base = (poly ? ctx->poly : ctx->key) + off;
    cudaError_t e = to_dev ? cudaMemcpyAsync(base, host, count * 8, cudaMemcpyHostToDevice, ctx->st)
                           : cudaMemcpyAsync(host, base, count * 8, cudaMemcpyDeviceToHost, ctx->st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "arena copy");
    if (!poly && to_dev) {
        int rc = refresh_key_preps(ctx, off, count);
        if (rc != AFHE_OK) return rc;
    }
    if (!async) CK(cudaStreamSynchronize(ctx->st));
    return AFHE_OK;
}

int afhe_write_poly(afhe_ctx* c, uint64_t o, const uint64_t* s, uint64_t n) { return arena_copy(c, true, true, o, (void*)s, n, false); }
int afhe_read_poly(afhe_ctx* c, uint64_t o, uint64_t* d, uint64_t n) { return arena_copy(c, true, false, o, d, n, false); }
int afhe_write_key(afhe_ctx* c, uint64_t o, const uint64_t* s, uint64_t n) { return arena_copy(c, false, true, o, (void*)s, n, false); }
int afhe_read_key(afhe_ctx* c, uint64_t o, uint64_t* d, uint64_t n) { return arena_copy(c, false, false, o, d, n, false); }
int afhe_write_poly_async(afhe_ctx* c, uint64_t o, const uint64_t* s, uint64_t n) { return arena_copy(c, true, true, o, (void*)s, n, true); }
int afhe_read_poly_async(afhe_ctx* c, uint64_t o, uint64_t* d, uint64_t n) { return arena_copy(c, true, false, o, d, n, true); }

static int read_rows(afhe_ctx* ctx, u64 off, u64 stride, u64 rows, u64 row_words, u64* dst, bool async) {
    if (!ctx || (rows && !dst)) return fail(ctx, AFHE_E_ARG, "null argument");
    if (rows == 0 || row_words == 0) return AFHE_OK;
    if (stride < row_words) return fail(ctx, AFHE_E_ARG, "row stride shorter than a row");
    if (rows > 1 && stride > (~0ull - row_words) / (rows - 1)) return fail(ctx, AFHE_E_RANGE, "rows out of range");
    const u64 span = (rows - 1) * stride + row_words;
    if (!range_ok(off, span, ctx->prm.poly_words)) return fail(ctx, AFHE_E_RANGE, "rows out of poly_gmem");
    if (stride == row_words)   // contiguous rows: one plain copy
        CK(cudaMemcpyAsync(dst, ctx->poly + off, span * 8, cudaMemcpyDeviceToHost, ctx->st));
    else
        CK(cudaMemcpy2DAsync(dst, row_words * 8, ctx->poly + off, stride * 8, row_words * 8, rows,
                             cudaMemcpyDeviceToHost, ctx->st));
    if (!async) CK(cudaStreamSynchronize(ctx->st));
    return AFHE_OK;
}

int afhe_read_poly_rows(afhe_ctx* ctx, uint64_t off, uint64_t stride, uint64_t rows, uint64_t row_words,
                        uint64_t* dst) {
    return read_rows(ctx, off, stride, rows, row_words, dst, false);
}

int afhe_read_poly_rows_async(afhe_ctx* ctx, uint64_t off, uint64_t stride, uint64_t rows, uint64_t row_words,
                              uint64_t* dst) {
    return read_rows(ctx, off, stride, rows, row_words, dst, true);
}

static constexpr size_t kFences = 64;

int afhe_fence(afhe_ctx* ctx, uint64_t* fence) {
    if (!ctx || !fence) return fail(ctx, AFHE_E_ARG, "null argument");
    if (ctx->fences.empty()) ctx->fences.assign(kFences, nullptr);
    cudaEvent_t& ev = ctx->fences[ctx->fence_next % kFences];
    if (!ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, ctx->st));
    *fence = ctx->fence_next++;
    return AFHE_OK;
}

int afhe_fence_wait(afhe_ctx* ctx, uint64_t fence) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    if (fence >= ctx->fence_next) return fail(ctx, AFHE_E_ARG, "fence not issued by this context");
    // a fence whose event was recorded again by a later fence waits for that
    // later point of the same stream, which is after the work it marks
    CK(cudaEventSynchronize(ctx->fences[fence % kFences]));
    return AFHE_OK;
}

int afhe_ctx_set_option(afhe_ctx* ctx, uint32_t option, int64_t value) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    switch (option) {
    case AFHE_OPT_KS_FUSED:
        if (value && !key_switch_fused_supported(ctx->log_n))
            return fail(ctx, AFHE_E_ARG, "the one-kernel key switch cannot run on this GPU at this ring degree");
        ctx->ks_fused = value != 0;
        return AFHE_OK;
    case AFHE_OPT_CHUNK:
        if (value < 0 || value > (int64_t)ctx->lanes) return fail(ctx, AFHE_E_ARG, "chunk must be in [0, lanes]");
        ctx->chunk = (uint32_t)value;
        return AFHE_OK;
    case AFHE_OPT_FUSED_MIN:
        if (value < 1 || value > 4096) return fail(ctx, AFHE_E_ARG, "fused minimum must be in [1, 4096]");
        ctx->fused_min = (uint32_t)value;
        return AFHE_OK;
    case AFHE_OPT_KS_EPT:
        if (value != 8 && value != 16) return fail(ctx, AFHE_E_ARG, "values per thread must be 8 or 16");
        ctx->ks_ept = (uint32_t)value;
        return AFHE_OK;
    case AFHE_OPT_KS_SLICE:
        if (value != 12 && value != 13) return fail(ctx, AFHE_E_ARG, "the slice must be 2^12 or 2^13 values");
        if (value == 12 && (ctx->log_n == 14 || ctx->log_n == 15)) {
            if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
            if (key_switch_fused_capacity(ctx->log_n, 8, 12) <= 0)
                return fail(ctx, AFHE_E_ARG, "clusters of 2^12-value slices cannot run on this GPU");
        }
        ctx->ks_slice = (uint32_t)value;
        return AFHE_OK;
    case AFHE_OPT_KS_CAPACITY:
        return fail(ctx, AFHE_E_ARG, "the key-switch capacity is read only");
    default:
        return fail(ctx, AFHE_E_ARG, "unknown option");
    }
}

int afhe_ctx_get_option(afhe_ctx* ctx, uint32_t option, int64_t* value) {
    if (!ctx || !value) return fail(ctx, AFHE_E_ARG, "null argument");
    switch (option) {
    case AFHE_OPT_KS_FUSED: *value = ctx->ks_fused ? 1 : 0; return AFHE_OK;
    case AFHE_OPT_CHUNK: *value = ctx->chunk ? ctx->chunk : ctx->lanes; return AFHE_OK;
    case AFHE_OPT_FUSED_MIN: *value = ctx->fused_min; return AFHE_OK;
    case AFHE_OPT_KS_EPT: *value = ctx->ks_ept; return AFHE_OK;
    case AFHE_OPT_KS_SLICE: *value = ctx->ks_slice; return AFHE_OK;
    case AFHE_OPT_KS_CAPACITY:
        if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
        *value = key_switch_fused_capacity(ctx->log_n, (int)ctx->ks_ept, (int)ctx->ks_slice);
        return AFHE_OK;
    default: return fail(ctx, AFHE_E_ARG, "unknown option");
    }
}

int afhe_host_alloc(uint64_t bytes, void** out) {
    if (!out) return fail(nullptr, AFHE_E_ARG, "null argument");
    *out = nullptr;
    if (bytes == 0) return AFHE_OK;
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaHostAlloc");
    return AFHE_OK;
}

int afhe_host_free(void* p) {
    if (!p) return AFHE_OK;
    cudaError_t e = cudaFreeHost(p);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaFreeHost");
    return AFHE_OK;
}

int afhe_automorphism_from_map(afhe_ctx* ctx, uint64_t src, uint64_t map_off, uint64_t dst, uint32_t limbs,
                               uint32_t /*galois_elt*/) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    const u64 n = ctx->n, LN = (u64)limbs * n, pw = ctx->prm.poly_words;
    if (limbs < 1 || limbs > ctx->L + ctx->K) return fail(ctx, AFHE_E_ARG, "limbs must be in [1, L + K]");
    if (!range_ok(src, LN, pw) || !range_ok(map_off, n / 2, pw) || !range_ok(dst, LN, pw))
        return fail(ctx, AFHE_E_RANGE, "automorphism operands out of range");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->st;
    // map and source staged in scratch first (a gather cannot run in place)
    CK(cudaMemcpyAsync(ctx->scr, ctx->poly + map_off, (n / 2) * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(ctx->scr + n, ctx->poly + src, LN * 8, cudaMemcpyDeviceToDevice, st));
    ZBases zb{};
    zb.src = zf_const(ctx->prm.poly_words + n);
    zb.out = zf_const(dst);
    CK(launch_automorphism(nullptr, ctx->scr, ctx->poly, n, limbs, 1, zb, st));
    return AFHE_OK;
}

int afhe_ntt_plan_count(uint32_t log_n, uint32_t* count) {
    if (!count) return fail(nullptr, AFHE_E_ARG, "null argument");
    *count = (uint32_t)ntt_plan_count((int)log_n);
    return *count ? AFHE_OK : fail(nullptr, AFHE_E_ARG, "log_n outside [10, 16]");
}

int afhe_ntt_plan_describe(uint32_t log_n, uint32_t plan, char* buf, uint32_t len) {
    if (!buf || !len) return fail(nullptr, AFHE_E_ARG, "null argument");
    if (plan >= (uint32_t)ntt_plan_count((int)log_n)) return fail(nullptr, AFHE_E_ARG, "no such plan");
    const NttPlan fwd = make_plan((int)log_n, false, (int)plan);
    if (fwd.npass == 1)
        snprintf(buf, len, "one pass, %d values per thread", fwd.ept[0]);
    else
        snprintf(buf, len, "columns %d per CTA (%d values per thread), chunk tiles %d words (%d values per thread)",
                 1 << fwd.g[0].log_c, fwd.ept[0], 1 << (fwd.g[1].P + fwd.g[1].log_c), fwd.ept[1]);
    return AFHE_OK;
}

int afhe_ntt_set_plan(uint32_t log_n, uint32_t plan) {
    if (plan >= (uint32_t)ntt_plan_count((int)log_n)) return fail(nullptr, AFHE_E_ARG, "no such plan");
    set_ntt_plan((int)log_n, (int)plan);
    return AFHE_OK;
}

int afhe_ntt_get_plan(uint32_t log_n, uint32_t* plan) {
    if (!plan) return fail(nullptr, AFHE_E_ARG, "null argument");
    if (!ntt_plan_count((int)log_n)) return fail(nullptr, AFHE_E_ARG, "log_n outside [10, 16]");
    *plan = (uint32_t)ntt_plan((int)log_n);
    return AFHE_OK;
}

int afhe_copy_poly(afhe_ctx* ctx, uint64_t dst, uint64_t src, uint64_t count) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    if (!range_ok(src, count, ctx->prm.poly_words) || !range_ok(dst, count, ctx->prm.poly_words))
        return fail(ctx, AFHE_E_RANGE, "copy out of range");
    if (count == 0 || dst == src) return AFHE_OK;
    CK(cudaMemcpyAsync(ctx->poly + dst, ctx->poly + src, count * 8, cudaMemcpyDeviceToDevice, ctx->st));
    return AFHE_OK;
}

int afhe_ctx_write_context_tables(afhe_ctx* ctx, uint32_t level, afhe_context_layout* out) {
    if (!ctx || !out) return fail(ctx, AFHE_E_ARG, "null argument");
    if (level < 1 || level > ctx->L) return fail(ctx, AFHE_E_LEVEL, "level out of range");
    const uint32_t n = ctx->n, L = ctx->L, K = ctx->K;
    std::vector<u64> q(ctx->prm.q, ctx->prm.q + L), p(ctx->prm.p, ctx->prm.p + K);
    afhe_context_layout lay{};
    lay.level = level;
    u64 cur = 0;
    std::vector<u64> tw((size_t)(L + K) * n), itw((size_t)(L + K) * n);
    for (uint32_t i = 0; i < L + K; ++i) {
        u64 qq = i < L ? q[i] : p[i - L];
        gen_twiddles(ctx->log_n, qq, root_of(ctx, i), &tw[(size_t)i * n], &itw[(size_t)i * n]);
    }
    // fhe_host_driver.cpp:63-86: twiddles (Q then P), inverse twiddles, CRT slots
    lay.twiddles_q_offset = cur;
    lay.twiddles_p_offset = cur + (u64)L * n;
    cur += (u64)(L + K) * n;
    lay.inv_twiddles_q_offset = cur;
    lay.inv_twiddles_p_offset = cur + (u64)L * n;
    cur += (u64)(L + K) * n;
    std::vector<std::pair<u64, std::vector<u64>>> writes;
    writes.push_back({lay.twiddles_q_offset, tw});
    writes.push_back({lay.inv_twiddles_q_offset, itw});
    auto slot = [&](const std::vector<u64>& v) {
        u64 at = cur;
        writes.push_back({at, v});
        u64 words = std::max<u64>(64, (v.size() + 63) / 64 * 64);
        cur += words;
        return at;
    };
    uint32_t parts = (level + ctx->alpha - 1) / ctx->alpha;
    lay.num_parts = parts;
    for (uint32_t j = 0; j < parts; ++j) {
        uint32_t start = j * ctx->alpha;
        uint32_t size = (j == parts - 1) ? level - start : ctx->alpha;
        std::vector<u64> qi(size), qm((size_t)size * (level - size + K));
        part_qhat_tables(q.data(), level, ctx->alpha, j, p.data(), K, qi.data(), qm.data());
        lay.qhat_inv_offset[j] = slot(qi);
        lay.qhat_modp_offset[j] = slot(qm);
    }
    std::vector<u64> pinv(level), phinv(K), phq((size_t)K * level);
    moddown_tables(q.data(), level, p.data(), K, pinv.data(), phinv.data(), phq.data());
    lay.p_inv_mod_q_offset = slot(pinv);
    lay.p_hat_inv_mod_p_offset = slot(phinv);
    lay.p_hat_mod_q_offset = slot(phq);
    std::vector<u64> qlql(level > 1 ? level - 1 : 1, 0), qlinv(level > 1 ? level - 1 : 1, 0);
    if (level > 1) rescale_tables(q.data(), level, qlql.data(), qlinv.data());
    lay.qlql_offset = slot(qlql);
    lay.qlinv_offset = slot(qlinv);
    lay.first_free_offset = (cur + 511) & ~511ull;
    if (lay.first_free_offset > ctx->prm.key_words) return fail(ctx, AFHE_E_RANGE, "key_gmem too small for tables");
    for (auto& w : writes) {
        int rc = afhe_write_key(ctx, w.first, w.second.data(), w.second.size());
        if (rc != AFHE_OK) return rc;
    }
    *out = lay;
    return AFHE_OK;
}

}  // extern "C"

// ===========================================================================
// fhe_accel_top dispatch
// ===========================================================================
namespace {

// Size of each base-conversion table as OP_LOAD_CONTEXT copies it
// (fhe_accel_top.cpp:200-209, generalised to numPartQ digits).
uint32_t part_size(uint32_t limbs, uint32_t alpha, uint32_t parts, uint32_t j) {
    return (j == parts - 1) ? limbs - alpha * j : alpha;
}

int load_context(afhe_ctx* ctx, const afhe_accel_args* a) {
    const uint32_t n = ctx->n;
    const uint32_t L = a->active_limbs, K = a->sizeP, parts = a->numPartQ, alpha = a->alpha;
    if (L < 1 || L > AFHE_MAX_Q || K > AFHE_MAX_P || parts < 1 || parts > AFHE_MAX_PARTS || alpha < 1)
        return fail(ctx, AFHE_E_ARG, "OP_LOAD_CONTEXT: sizes out of range");
    if ((u64)alpha * (parts - 1) >= L) return fail(ctx, AFHE_E_ARG, "OP_LOAD_CONTEXT: last digit would be empty");
    const u64 kw = ctx->prm.key_words;
    auto chk = [&](u64 off, u64 words) { return range_ok(off, words, kw); };
    if (!chk(a->twiddles_q_offset, (u64)L * n) || !chk(a->inv_twiddles_q_offset, (u64)L * n) ||
        !chk(a->twiddles_p_offset, (u64)K * n) || !chk(a->inv_twiddles_p_offset, (u64)K * n))
        return fail(ctx, AFHE_E_RANGE, "OP_LOAD_CONTEXT: twiddle offsets out of range");
    // validate the primes' constants against the loaded context (the
    // reference's Barrett reduction is exact only with m = floor(2^k/q), k = 2*bits+3)
    for (uint32_t i = 0; i < L + K; ++i) {
        u64 q = i < L ? a->rns_primes[i] : a->p_primes[i - L];
        u64 mlo, mhi;
        uint32_t k;
        if (q < 3 || q >= (1ull << 61) || (q & 1) == 0) return fail(ctx, AFHE_E_ARG, "OP_LOAD_CONTEXT: modulus out of range");
        barrett_constant(q, &mlo, &mhi, &k);
        u64 glo = i < L ? a->barrett_m_q_lo[i] : a->barrett_m_p_lo[i - L];
        u64 ghi = i < L ? a->barrett_m_q_hi[i] : a->barrett_m_p_hi[i - L];
        uint32_t gk = i < L ? a->barrett_k_q[i] : a->barrett_k_p[i - L];
        if (glo != mlo || ghi != mhi || gk != k) return fail(ctx, AFHE_E_ARG, "Barrett constant does not match its modulus");
    }
    // twiddles: (L + K) rows, Q then P
    DevPrimeSet& s = ctx->ld;
    if (s.count < L + K) {
        for (void* pp : {(void*)s.pc, (void*)s.tw, (void*)s.itw, (void*)s.tw2, (void*)s.itw2}) if (pp) cudaFree(pp);
        s = DevPrimeSet{};
        CK(dalloc(&s.pc, AFHE_MAX_Q + AFHE_MAX_P));
        CK(dalloc(&s.tw, (size_t)(AFHE_MAX_Q + AFHE_MAX_P) * n));
        CK(dalloc(&s.itw, (size_t)(AFHE_MAX_Q + AFHE_MAX_P) * n));
        CK(dalloc(&s.tw2, (size_t)(AFHE_MAX_Q + AFHE_MAX_P) * n));
        CK(dalloc(&s.itw2, (size_t)(AFHE_MAX_Q + AFHE_MAX_P) * n));
        s.count = AFHE_MAX_Q + AFHE_MAX_P;
    }
    cudaStream_t st = ctx->st;
    CK(cudaMemcpyAsync(s.tw, ctx->key + a->twiddles_q_offset, (size_t)L * n * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.tw + (size_t)L * n, ctx->key + a->twiddles_p_offset, (size_t)K * n * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.itw, ctx->key + a->inv_twiddles_q_offset, (size_t)L * n * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.itw + (size_t)L * n, ctx->key + a->inv_twiddles_p_offset, (size_t)K * n * 8, cudaMemcpyDeviceToDevice, st));
    std::vector<u64> qv(L + K), ninv(L + K);
    for (uint32_t i = 0; i < L + K; ++i) {
        qv[i] = i < L ? a->rns_primes[i] : a->p_primes[i - L];
        ninv[i] = i < L ? a->n_inv_q[i] : a->n_inv_p[i - L];
    }
    u64* dq = nullptr;
    u64* dn = nullptr;
    CK(dalloc(&dq, L + K));
    CK(dalloc(&dn, L + K));
    CK(cudaMemcpyAsync(dq, qv.data(), qv.size() * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dn, ninv.data(), ninv.size() * 8, cudaMemcpyHostToDevice, st));
    CK(launch_interleave(s.tw, dq, s.tw2, L + K, n, st));
    CK(launch_interleave(s.itw, dq, s.itw2, L + K, n, st));
    CK(launch_prime_consts(s.pc, dq, dn, s.itw, n, L + K, st));
    CK(cudaStreamSynchronize(st));
    cudaFree(dq); cudaFree(dn);

    // CRT tables, raw
    std::vector<std::pair<u64, u64>> regions;  // (key offset, words) in load order
    ctx->ld_off_qhat_inv.assign(parts, 0);
    ctx->ld_off_qhat_modp.assign(parts, 0);
    size_t cur = 0;
    for (uint32_t j = 0; j < parts; ++j) {
        uint32_t sz = part_size(L, alpha, parts, j);
        ctx->ld_off_qhat_inv[j] = cur; regions.push_back({a->qhat_inv_offset[j], sz}); cur += sz;
        u64 w = (u64)sz * (L - sz + K);
        ctx->ld_off_qhat_modp[j] = cur; regions.push_back({a->qhat_modp_offset[j], w}); cur += w;
    }
    ctx->ld_off_pinv = cur; regions.push_back({a->p_inv_mod_q_offset, L}); cur += L;
    ctx->ld_off_phatinv = cur; regions.push_back({a->p_hat_inv_mod_p_offset, K}); cur += K;
    ctx->ld_off_phatmodq = cur; regions.push_back({a->p_hat_mod_q_offset, (u64)K * L}); cur += (u64)K * L;
    ctx->ld_off_qlql = cur; regions.push_back({a->qlql_offset, L}); cur += L;
    ctx->ld_off_qlinv = cur; regions.push_back({a->qlinv_offset, L}); cur += L;
    for (auto& r : regions)
        if (!chk(r.first, r.second)) return fail(ctx, AFHE_E_RANGE, "OP_LOAD_CONTEXT: table offset out of range");
    if (ctx->ld_crt_words < cur) {
        if (ctx->ld_crt) cudaFree(ctx->ld_crt);
        if (ctx->ld_crt_sh) cudaFree(ctx->ld_crt_sh);
        if (ctx->ld_mod) cudaFree(ctx->ld_mod);
        ctx->ld_crt = ctx->ld_crt_sh = ctx->ld_mod = nullptr;
        CK(dalloc(&ctx->ld_crt, 2 * cur));   // raw, then a working copy
        CK(dalloc(&ctx->ld_crt_sh, cur));
        CK(dalloc(&ctx->ld_mod, cur));
        ctx->ld_crt_words = cur;
    }
    size_t at = 0;
    for (auto& r : regions) {
        if (r.second) CK(cudaMemcpyAsync(ctx->ld_crt + at, ctx->key + r.first, r.second * 8, cudaMemcpyDeviceToDevice, st));
        at += r.second;
    }
    CK(cudaStreamSynchronize(st));
    ctx->ld_nq = L;
    ctx->ld_np = K;
    ctx->ld_alpha = alpha;
    ctx->ld_parts = parts;
    ctx->ld_q.assign(a->rns_primes, a->rns_primes + L);
    ctx->ld_p.assign(a->p_primes, a->p_primes + K);
    ctx->ld_ninv_q.assign(a->n_inv_q, a->n_inv_q + L);
    ctx->ld_ninv_p.assign(a->n_inv_p, a->n_inv_p + K);
    std::fill(ctx->ld_tabs_key, ctx->ld_tabs_key + 4, -1);    // tables prepared from the old load are stale
    ctx->loaded = true;
    return AFHE_OK;
}

// The call's primes and N^-1 values must be the ones the tables were loaded for.
int check_call_primes(afhe_ctx* ctx, const afhe_accel_args* a, uint32_t nq, uint32_t np) {
    if (!ctx->loaded) return fail(ctx, AFHE_E_STATE, "op issued before OP_LOAD_CONTEXT");
    if (nq > ctx->ld_nq || np > ctx->ld_np) return fail(ctx, AFHE_E_LEVEL, "more limbs than the loaded context");
    for (uint32_t i = 0; i < nq; ++i)
        if (a->rns_primes[i] != ctx->ld_q[i] || a->n_inv_q[i] != ctx->ld_ninv_q[i])
            return fail(ctx, AFHE_E_ARG, "call primes differ from the loaded context");
    for (uint32_t i = 0; i < np; ++i)
        if (a->p_primes[i] != ctx->ld_p[i] || a->n_inv_p[i] != ctx->ld_ninv_p[i])
            return fail(ctx, AFHE_E_ARG, "call special primes differ from the loaded context");
    return AFHE_OK;
}

// Per-call working copy of the loaded CRT tables reduced by, and with
// companions for, the moduli each entry multiplies under at level sizeQl.
int prep_loaded_tables(afhe_ctx* ctx, uint32_t sizeQl, uint32_t parts, uint32_t alpha, bool ks, OpTabs* t) {
    const int key[4] = {(int)sizeQl, (int)parts, (int)alpha, ks ? 1 : 0};
    if (std::equal(key, key + 4, ctx->ld_tabs_key)) {   // prepared by an earlier call, in stream order
        *t = ctx->ld_tabs;
        return AFHE_OK;
    }
    const uint32_t K = ctx->ld_np, Lld = ctx->ld_nq;
    const size_t W = ctx->ld_crt_words;
    std::vector<u64> mods(W, 0);
    const u64* q = ctx->ld_q.data();
    const u64* p = ctx->ld_p.data();
    t->pt = ctx->ld.view();
    t->p_base = Lld;
    t->sizeQl = sizeQl;
    t->parts = parts;
    t->alpha = alpha;
    u64* work = ctx->ld_crt + W;
    if (ks) {
        if (parts > ctx->ld_parts) return fail(ctx, AFHE_E_LEVEL, "more digits than the loaded context");
        for (uint32_t j = 0; j < parts; ++j) {
            uint32_t start = alpha * j;
            uint32_t size = part_size(sizeQl, alpha, parts, j);
            uint32_t row = sizeQl - size + K;
            uint32_t ld_size = part_size(Lld, ctx->ld_alpha, ctx->ld_parts, j);
            u64 ld_w = (u64)ld_size * (Lld - ld_size + K);
            if (size > ld_size || (u64)size * row > ld_w)
                return fail(ctx, AFHE_E_LEVEL, "base-conversion tables loaded for a smaller level");
            std::vector<u64> outp;
            for (uint32_t i = 0; i < sizeQl; ++i)
                if (i < start || i >= start + size) outp.push_back(q[i]);
            for (uint32_t k = 0; k < K; ++k) outp.push_back(p[k]);
            for (uint32_t i = 0; i < size; ++i) {
                mods[ctx->ld_off_qhat_inv[j] + i] = q[start + i];
                for (uint32_t c = 0; c < row; ++c) mods[ctx->ld_off_qhat_modp[j] + (size_t)i * row + c] = outp[c];
            }
            t->qhat_inv[j] = work + ctx->ld_off_qhat_inv[j];
            t->qhat_inv_sh[j] = ctx->ld_crt_sh + ctx->ld_off_qhat_inv[j];
            t->qhat_modp[j] = work + ctx->ld_off_qhat_modp[j];
            t->qhat_modp_sh[j] = ctx->ld_crt_sh + ctx->ld_off_qhat_modp[j];
        }
        for (uint32_t i = 0; i < sizeQl; ++i) mods[ctx->ld_off_pinv + i] = q[i];
        for (uint32_t k = 0; k < K; ++k) {
            mods[ctx->ld_off_phatinv + k] = p[k];
            for (uint32_t i = 0; i < sizeQl; ++i) mods[ctx->ld_off_phatmodq + (size_t)k * sizeQl + i] = q[i];
        }
    } else {
        for (uint32_t i = 0; i + 1 < sizeQl; ++i) {
            mods[ctx->ld_off_qlql + i] = q[i];
            mods[ctx->ld_off_qlinv + i] = q[i];
        }
    }
    t->p_inv_mod_q = work + ctx->ld_off_pinv;
    t->p_inv_mod_q_sh = ctx->ld_crt_sh + ctx->ld_off_pinv;
    t->phat_inv_modp = work + ctx->ld_off_phatinv;
    t->phat_inv_modp_sh = ctx->ld_crt_sh + ctx->ld_off_phatinv;
    t->phat_modq = work + ctx->ld_off_phatmodq;
    t->phat_modq_sh = ctx->ld_crt_sh + ctx->ld_off_phatmodq;
    t->qlql = work + ctx->ld_off_qlql;
    t->qlql_sh = ctx->ld_crt_sh + ctx->ld_off_qlql;
    t->qlinv = work + ctx->ld_off_qlinv;
    t->qlinv_sh = ctx->ld_crt_sh + ctx->ld_off_qlinv;
    // the moduli go through the pinned descriptor ring: no host wait, and the
    // working copy is rewritten in stream order after every earlier use
    cudaStream_t st = ctx->st;
    u64* dmods = nullptr;
    int rc = ring_put(ctx, mods.data(), W, &dmods);
    if (rc != AFHE_OK) return rc;
    CK(cudaMemcpyAsync(work, ctx->ld_crt, W * 8, cudaMemcpyDeviceToDevice, st));
    CK(launch_companions(work, ctx->ld_crt_sh, dmods, W, st));
    ctx->ld_tabs = *t;
    std::copy(key, key + 4, ctx->ld_tabs_key);
    return AFHE_OK;
}

// The call's job list, staged through the descriptor ring (no host wait).
int upload_jobs(afhe_ctx* ctx, const std::vector<LimbJob>& jobs, const LimbJob** dev) {
    static_assert(sizeof(LimbJob) % sizeof(u64) == 0, "LimbJob is staged as words");
    u64* d = nullptr;
    int rc = ring_put(ctx, jobs.data(), jobs.size() * sizeof(LimbJob) / sizeof(u64), &d);
    *dev = (const LimbJob*)d;
    return rc;
}

bool overlap(u64 a, u64 aw, u64 b, u64 bw) { return a < b + bw && b < a + aw; }

// If [src, src + w) overlaps [dst, dst + w2) and is not the same start, copy
// src into scratch (the reference loads every operand into on-chip buffers
// before writing, so any aliasing is legal there). Returns the offset to read
// and whether it is in scratch.
int stage(afhe_ctx* ctx, u64 src, u64 w, u64 dst, u64 w2, u64 scr_off, u64* eff, bool* in_scr) {
    *eff = src;
    *in_scr = false;
    if (w && w2 && overlap(src, w, dst, w2) && src != dst) {
        CK(cudaMemcpyAsync(ctx->scr + scr_off, ctx->poly + src, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
        *eff = scr_off;
        *in_scr = true;
    }
    return AFHE_OK;
}

}  // namespace

extern "C" int afhe_dispatch(afhe_ctx* ctx, const afhe_accel_args* a) {
    if (!ctx || !a) return fail(ctx, AFHE_E_ARG, "null argument");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
    if (a->op_code == AFHE_OP_LOAD_CONTEXT) return load_context(ctx, a);
    const uint32_t n = ctx->n;
    const u64 pw = ctx->prm.poly_words;
    const uint32_t L = a->active_limbs;
    const u64 LN = (u64)L * n;
    cudaStream_t st = ctx->st;
    int rc;
    switch (a->op_code) {
    case AFHE_OP_NTT:
    case AFHE_OP_INTT: {
        if (L < 1) return fail(ctx, AFHE_E_ARG, "active_limbs must be >= 1");
        if ((rc = check_call_primes(ctx, a, L, 0)) != AFHE_OK) return rc;
        if (!range_ok(a->src_a_offset, LN, pw) || !range_ok(a->dst_offset, LN, pw))
            return fail(ctx, AFHE_E_RANGE, "NTT operands out of range");
        std::vector<LimbJob> jobs(L);
        for (uint32_t i = 0; i < L; ++i) { jobs[i].src = jobs[i].dst = jobs[i].out = (u64)i * n; jobs[i].prime = i; jobs[i].aux = i; }
        const LimbJob* djobs = nullptr;
        if ((rc = upload_jobs(ctx, jobs, &djobs)) != AFHE_OK) return rc;
        u64 src; bool in_scr;
        if ((rc = stage(ctx, a->src_a_offset, LN, a->dst_offset, LN, 0, &src, &in_scr)) != AFHE_OK) return rc;
        ZBases zb{};
        zb.src = zf_const(src);
        zb.mid = zf_const(a->dst_offset);
        zb.out = zf_const(a->dst_offset);
        CK(launch_ntt_plain(a->op_code == AFHE_OP_INTT, ctx->log_n, ctx->ld.view(), djobs, L,
                            in_scr ? ctx->scr : ctx->poly, ctx->poly, 1, zb, st));
        break;
    }
    case AFHE_OP_POLY_ADD:
    case AFHE_OP_POLY_SUB:
    case AFHE_OP_POLY_MUL_NTT: {
        if (L < 1 || L > AFHE_MAX_Q) return fail(ctx, AFHE_E_ARG, "active_limbs out of range");
        if (!range_ok(a->src_a_offset, LN, pw) || !range_ok(a->src_b_offset, LN, pw) || !range_ok(a->dst_offset, LN, pw))
            return fail(ctx, AFHE_E_RANGE, "poly operands out of range");
        // these ops need only the call's primes (fhe_accel_top.cpp:242-270)
        std::vector<PrimeConst> pc(L);
        for (uint32_t i = 0; i < L; ++i) {
            if (a->rns_primes[i] < 3 || a->rns_primes[i] >= (1ull << 61)) return fail(ctx, AFHE_E_ARG, "modulus out of range");
            pc[i] = host_prime_const(a->rns_primes[i], 1, 1);
        }
        static_assert(sizeof(PrimeConst) % sizeof(u64) == 0, "PrimeConst is staged as words");
        u64* dpc_words = nullptr;
        if ((rc = ring_put(ctx, pc.data(), L * sizeof(PrimeConst) / sizeof(u64), &dpc_words)) != AFHE_OK) return rc;
        const PrimeConst* dpc = (const PrimeConst*)dpc_words;
        // operands that partially overlap the output are staged (scratch words [0, 2LN))
        u64 sa, sb; bool ia, ib;
        if ((rc = stage(ctx, a->src_a_offset, LN, a->dst_offset, LN, 0, &sa, &ia)) != AFHE_OK) return rc;
        if ((rc = stage(ctx, a->src_b_offset, LN, a->dst_offset, LN, LN, &sb, &ib)) != AFHE_OK) return rc;
        ElemOp op = a->op_code == AFHE_OP_POLY_ADD ? EW_ADD : (a->op_code == AFHE_OP_POLY_SUB ? EW_SUB : EW_MUL);
        if (ia || ib) {
            // bring both operands into scratch so one arena base serves the kernel
            if (!ia) CK(cudaMemcpyAsync(ctx->scr, ctx->poly + sa, LN * 8, cudaMemcpyDeviceToDevice, st));
            if (!ib) CK(cudaMemcpyAsync(ctx->scr + LN, ctx->poly + sb, LN * 8, cudaMemcpyDeviceToDevice, st));
            ZBases zb{};
            zb.src = zf_const(0); zb.aux = zf_const(LN); zb.out = zf_const(2 * LN);
            CK(launch_elementwise(op, dpc, 0, ctx->scr, n, L, 1, zb, st));
            CK(cudaMemcpyAsync(ctx->poly + a->dst_offset, ctx->scr + 2 * LN, LN * 8, cudaMemcpyDeviceToDevice, st));
        } else {
            ZBases zb{};
            zb.src = zf_const(sa); zb.aux = zf_const(sb); zb.out = zf_const(a->dst_offset);
            CK(launch_elementwise(op, dpc, 0, ctx->poly, n, L, 1, zb, st));
        }
        break;
    }
    case AFHE_OP_AUTOMORPHISM: {
        if (L < 1) return fail(ctx, AFHE_E_ARG, "active_limbs must be >= 1");
        if (!range_ok(a->src_a_offset, LN, pw) || !range_ok(a->src_b_offset, n / 2, pw) || !range_ok(a->dst_offset, LN, pw))
            return fail(ctx, AFHE_E_RANGE, "automorphism operands out of range");
        // fhe_accel_top.cpp:272-281: the map is read once into a work buffer
        CK(cudaMemcpyAsync(ctx->scr, ctx->poly + a->src_b_offset, (n / 2) * 8, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ctx->scr + n, ctx->poly + a->src_a_offset, LN * 8, cudaMemcpyDeviceToDevice, st));
        ZBases zb{};
        zb.src = zf_const(n); zb.out = zf_const(n + LN);
        CK(launch_automorphism(nullptr, ctx->scr, ctx->scr, n, L, 1, zb, st));
        CK(cudaMemcpyAsync(ctx->poly + a->dst_offset, ctx->scr + n + LN, LN * 8, cudaMemcpyDeviceToDevice, st));
        break;
    }
    case AFHE_OP_RESCALE: {
        if (L < 2) return fail(ctx, AFHE_E_ARG, "rescale needs active_limbs >= 2");
        if ((rc = check_call_primes(ctx, a, L, 0)) != AFHE_OK) return rc;
        if (a->n_inv_mod_q_last != ctx->ld_ninv_q[L - 1]) return fail(ctx, AFHE_E_ARG, "n_inv_mod_q_last mismatch");
        const u64 out = (u64)(L - 1) * n;
        if (!range_ok(a->src_a_offset, LN, pw) || !range_ok(a->src_b_offset, LN, pw) || !range_ok(a->dst_offset, 2 * out, pw))
            return fail(ctx, AFHE_E_RANGE, "rescale operands out of range");
        OpTabs t;
        if ((rc = prep_loaded_tables(ctx, L, 1, 1, false, &t)) != AFHE_OK) return rc;
        std::vector<LimbJob> jobs(L);
        for (uint32_t i = 0; i < L; ++i) { jobs[i].src = jobs[i].dst = jobs[i].out = (u64)i * n; jobs[i].prime = i; jobs[i].aux = i; }
        const LimbJob* djobs = nullptr;
        if ((rc = upload_jobs(ctx, jobs, &djobs)) != AFHE_OK) return rc;
        // fhe_accel_top.cpp:283-297: both inputs are loaded before anything is stored
        const u64 s_in = 0, s_tmp = 2 * LN, s_out = 4 * LN;
        CK(cudaMemcpyAsync(ctx->scr + s_in, ctx->poly + a->src_a_offset, LN * 8, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ctx->scr + s_in + LN, ctx->poly + a->src_b_offset, LN * 8, cudaMemcpyDeviceToDevice, st));
        ZBases zb{};
        zb.src = zf_stride(s_in, LN);
        zb.out = zf_stride(s_out, out);
        zb.mid = zf_stride(s_tmp, LN);
        CK(launch_rescale(ctx->log_n, t, djobs, L, ctx->scr, ctx->scr, 2, zb, st));
        CK(cudaMemcpyAsync(ctx->poly + a->dst_offset, ctx->scr + s_out, 2 * out * 8, cudaMemcpyDeviceToDevice, st));
        break;
    }
    case AFHE_OP_KEY_SWITCH: {
        const uint32_t sq = a->sizeQl, K = a->sizeP, parts = a->numPartQ, alpha = a->alpha;
        if (sq < 1 || K < 1 || parts < 1 || parts > AFHE_MAX_PARTS || alpha < 1)
            return fail(ctx, AFHE_E_ARG, "key switch sizes out of range");
        if ((u64)alpha * (parts - 1) >= sq) return fail(ctx, AFHE_E_ARG, "key switch: last digit would be empty");
        if ((rc = check_call_primes(ctx, a, sq, K)) != AFHE_OK) return rc;
        const u64 SQ = (u64)sq * n;
        const u64 key_words = 2ull * parts * (sq + K) * n;
        if (!range_ok(a->src_a_offset, SQ, pw) || !range_ok(a->dst_offset, 2 * SQ, pw))
            return fail(ctx, AFHE_E_RANGE, "key switch operands out of range");
        if (!range_ok(a->evk_offset, key_words, ctx->prm.key_words)) return fail(ctx, AFHE_E_RANGE, "evk out of key_gmem");
        OpTabs t;
        if ((rc = prep_loaded_tables(ctx, sq, parts, alpha, true, &t)) != AFHE_OK) return rc;
        // jobs: Q slots [0, sq), special slots [sq, sq + K) -> primes ld_nq + k, then ModUp jobs
        std::vector<LimbJob> jobs;
        for (uint32_t i = 0; i < sq + K; ++i) {
            LimbJob j{};
            j.src = j.dst = j.out = (u64)i * n;
            j.prime = i < sq ? i : ctx->ld_nq + (i - sq);
            j.aux = i < sq ? i : i - sq;
            jobs.push_back(j);
        }
        const u64 S = (u64)sq + K;
        uint32_t n_modup = 0;
        for (uint32_t j = 0; j < parts; ++j) {
            uint32_t start = j * alpha, size = part_size(sq, alpha, parts, j), kpos = 0;
            for (uint32_t i = 0; i < sq + K; ++i) {
                if (i < sq && i >= start && i < start + size) continue;
                LimbJob jb{};
                jb.dst = jb.out = ((u64)j * S + i) * n;
                jb.prime = i < sq ? i : ctx->ld_nq + (i - sq);
                jb.aux = (j << 16) | kpos++;
                jobs.push_back(jb);
                ++n_modup;
            }
        }
        const LimbJob* djobs = nullptr;
        if ((rc = upload_jobs(ctx, jobs, &djobs)) != AFHE_OK) return rc;
        const u64 kw = ks_scratch_words(n, sq, K, parts);
        if (SQ + kw > ctx->scr_words) return fail(ctx, AFHE_E_ARG, "scratch too small for this key switch");
        // input staged into scratch (fhe_accel_top.cpp:299-300 loads it first)
        CK(cudaMemcpyAsync(ctx->scr, ctx->poly + a->src_a_offset, SQ * 8, cudaMemcpyDeviceToDevice, st));
        // the kernel reads the input and writes the outputs through one arena
        // base; the input lives in scratch, so the outputs go via scratch too
        const u64 o_scr = SQ + kw;
        if (o_scr + 2 * SQ > ctx->scr_words) return fail(ctx, AFHE_E_ARG, "scratch too small for this key switch");
        ZBases zb{};
        zb.src = zf_const(0);
        zb.mid = zf_const(SQ);
        zb.out = zf_const(o_scr);        // ks0
        zb.aux = zf_const(o_scr + SQ);   // ks1
        CK(launch_key_switch(ctx->log_n, t, djobs, djobs + sq + K, n_modup, sq, sq, K, ctx->key,
                             a->evk_offset, a->evk_offset + (u64)parts * (sq + K) * n, sq + K, sq, ctx->scr, ctx->scr,
                             1, zb, st));
        CK(cudaMemcpyAsync(ctx->poly + a->dst_offset, ctx->scr + o_scr, 2 * SQ * 8, cudaMemcpyDeviceToDevice, st));
        break;
    }
    default:
        return fail(ctx, AFHE_E_ARG, "unknown op code");
    }
    // enqueued on the context stream; afhe_read_* and afhe_sync wait for it
    return AFHE_OK;
}
