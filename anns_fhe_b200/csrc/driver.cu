// driver.cu -- FHEHostDriver composite operators on the device arenas
// (cpp_host_model/src/fhe_host_driver.cpp:248-404), plus batched variants.
//
// Every composite runs entirely on the context stream; intermediates live in
// the context-private scratch (one lane per ciphertext of a batch) instead of
// the reference's fixed SCRATCH_* slots of poly_gmem
// (cpp_host_model/src/fhe_host_driver.h:63-69), so caller-visible memory is
// never clobbered. Keys use the full-level layout: digit j, limb i of a key at
// evk lives at evk + (j * (L + K) + (i < l ? i : L + i - l)) * N, evk_b after
// all d digits of evk_a (fhe_host_driver.cpp:105-117, fhe_accel_top.cpp:304-305).
//
// A batched call processes up to ctx->lanes ciphertexts per launch; the
// per-ciphertext offsets reach the kernels as ZFields (strided when regular,
// else a small array staged through the context's descriptor ring).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <vector>

#include "internal.h"
#include "lanes.h"
#include "tables.h"

using namespace afhe;

namespace {

typedef std::vector<u64> Offs;

int check_limbs(afhe_ctx* ctx, uint32_t limbs, uint32_t min_limbs) {
    if (limbs < min_limbs || limbs > ctx->L) return fail(ctx, AFHE_E_LEVEL, "limb count outside [min, L]");
    return AFHE_OK;
}

// Primitive operators also accept "extended" polynomials over all L + K
// primes (Q limbs then P limbs), as key generation needs.
int check_limbs_ext(afhe_ctx* ctx, uint32_t limbs) {
    if (limbs < 1 || limbs > ctx->L + ctx->K) return fail(ctx, AFHE_E_LEVEL, "limb count outside [1, L + K]");
    return AFHE_OK;
}

int check_poly(afhe_ctx* ctx, u64 off, uint32_t limbs) {
    if (!range_ok(off, (u64)limbs * ctx->n, ctx->prm.poly_words)) return fail(ctx, AFHE_E_RANGE, "operand out of poly_gmem");
    return AFHE_OK;
}

int check_key(afhe_ctx* ctx, u64 evk) {
    u64 words = 2ull * ctx->dnum * (ctx->L + ctx->K) * ctx->n;
    if (!range_ok(evk, words, ctx->prm.key_words)) return fail(ctx, AFHE_E_RANGE, "key out of key_gmem");
    return AFHE_OK;
}

int check_cts(afhe_ctx* ctx, const afhe_ct_ref* v, uint32_t count, uint32_t limbs) {
    int rc;
    for (uint32_t i = 0; i < count; ++i)
        if ((rc = check_poly(ctx, v[i].c0_offset, limbs)) || (rc = check_poly(ctx, v[i].c1_offset, limbs))) return rc;
    return AFHE_OK;
}

// The device copy of the evaluation-form automorphism map of `galois`
// (computed on first use, kept until the context is destroyed).
int cached_map(afhe_ctx* ctx, uint32_t galois, const uint32_t** out) {
    auto it = ctx->auto_maps.find(galois);
    if (it != ctx->auto_maps.end()) {
        *out = it->second;
        return AFHE_OK;
    }
    std::vector<uint32_t> map(ctx->n);
    automorphism_map(ctx->log_n, galois, map.data());
    uint32_t* d = nullptr;
    CK(cudaMalloc(&d, (size_t)ctx->n * sizeof(uint32_t)));
    cudaError_t e = cudaMemcpy(d, map.data(), (size_t)ctx->n * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(ctx, e, "automorphism map upload");
    }
    bool local = true;
    for (uint32_t i = 0; i < ctx->n && local; ++i) local = (map[i] >> 8) == (i >> 8);
    ctx->auto_maps[galois] = d;
    ctx->auto_map_local[galois] = local;
    *out = d;
    return AFHE_OK;
}

#define ZF(dst, vec)                                                                    \
    do {                                                                                \
        int _rc = zf_from(ctx, (vec).data(), (uint32_t)(vec).size(), &(dst));           \
        if (_rc != AFHE_OK) return _rc;                                                 \
    } while (0)

// Key switch nz polynomials (poly_gmem-relative offsets) with one key, with
// optional fusion (automorphism gather, c0 add, accumulate; see KsFuse).
// `fused_ok` is false when an entry's outputs may overlap another entry's
// inputs, which the one-kernel key switch cannot order.
// With lvz (mixed levels, one-kernel key switch only), entry z runs at level
// lvz.at(z) and `limbs` is the largest of them.
int ks_batch(afhe_ctx* ctx, const ZField& in, const ZField& out0, const ZField& out1, uint32_t nz, u64 evk,
             uint32_t limbs, const KsFuse* fuse = nullptr, bool fused_ok = true, const ulonglong2* prep = nullptr,
             const ZField* lvz = nullptr) {
    const u64 n = ctx->n, S = (u64)ctx->L + ctx->K;
    const OpTabs& t = ctx->lv[limbs];
    const LevelJobs& lj = ctx->lvjobs[limbs];
    ZBases zb{};
    zb.src = in;
    zb.out = out0;
    zb.aux = out1;
    zb.mid = lane_field(ctx, &Lane::ks);
    if (lvz && !(ctx->ks_fused && fused_ok)) return fail(ctx, AFHE_E_STATE, "mixed levels need the one-kernel key switch");
    if (ctx->ks_fused && fused_ok && (lvz || nz >= ctx->fused_min)) {
        CK(launch_key_switch_fused(ctx->log_n, t, limbs, ctx->K, ctx->key, evk, evk + (u64)ctx->dnum * S * n,
                                   (uint32_t)S, ctx->L, ctx->poly, ctx->scr, nz, zb, ctx->st, fuse, prep,
                                   lvz ? ctx->lv_dev : nullptr, lvz, (int)ctx->ks_ept, (int)ctx->ks_slice));
        return AFHE_OK;
    }
    CK(launch_key_switch(ctx->log_n, t, ctx->jobs_qp, lj.modup, lj.n_modup, ctx->L, limbs, ctx->K, ctx->key, evk,
                         evk + (u64)ctx->dnum * S * n, (uint32_t)S, ctx->L, ctx->poly, ctx->scr, nz, zb, ctx->st,
                         fuse));
    return AFHE_OK;
}

// Rescale nz ciphertexts (in0, in1) -> (out0, out1), level limbs -> limbs - 1.
// The two polynomials of ciphertext z run as z' = 2z, 2z + 1.
int rescale_batch(afhe_ctx* ctx, const Offs& in0, const Offs& in1, const Offs& out0, const Offs& out1,
                  uint32_t limbs) {
    const uint32_t nz = (uint32_t)in0.size();
    Offs src(2 * nz), out(2 * nz);
    for (uint32_t z = 0; z < nz; ++z) {
        src[2 * z] = in0[z]; src[2 * z + 1] = in1[z];
        out[2 * z] = out0[z]; out[2 * z + 1] = out1[z];
    }
    ZBases zb{};
    ZF(zb.src, src);
    ZF(zb.out, out);
    zb.mid = zf_pair(lane_field(ctx, &Lane::resc), (u64)ctx->L * ctx->n);
    CK(launch_rescale(ctx->log_n, ctx->lv[limbs], ctx->jobs_qp, limbs, ctx->poly, ctx->scr, 2 * nz, zb, ctx->st));
    return AFHE_OK;
}

int ew_fields(afhe_ctx* ctx, ElemOp op, const ZField& a, const ZField& b, const ZField& o, uint32_t nz,
              uint32_t limbs) {
    ZBases zb{};
    zb.src = a;
    zb.aux = b;
    zb.out = o;
    CK(launch_elementwise(op, ctx->nat.pc, 0, ctx->poly, ctx->n, limbs, nz, zb, ctx->st));
    return AFHE_OK;
}

int ew_batch(afhe_ctx* ctx, ElemOp op, const Offs& a, const Offs* b, const Offs& o, uint32_t limbs) {
    ZField fa, fb, fo;
    ZF(fa, a);
    if (b) ZF(fb, *b); else fb = fa;
    ZF(fo, o);
    return ew_fields(ctx, op, fa, fb, fo, (uint32_t)a.size(), limbs);
}

bool overlap(u64 a, u64 aw, u64 b, u64 bw) { return a < b + bw && b < a + aw; }

// eval_mult_relin_rescale on nz ciphertexts (lane z for ciphertext z).
int mult_relin_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d,
                             uint32_t nz, uint32_t limbs) {
    if (!ctx->has_relin) return fail(ctx, AFHE_E_NOKEY, "no relinearisation key set");
    Offs a0(nz), a1(nz), b0(nz), b1(nz), o0(nz), o1(nz), t0(nz), t1(nz);
    for (uint32_t z = 0; z < nz; ++z) {
        a0[z] = a[z].c0_offset; a1[z] = a[z].c1_offset;
        b0[z] = b[z].c0_offset; b1[z] = b[z].c1_offset;
        o0[z] = d[z].c0_offset; o1[z] = d[z].c1_offset;
        t0[z] = lane_temp(ctx, z, 0);
        t1[z] = lane_temp(ctx, z, 1);
    }
    // 1. tensor product (fhe_host_driver.cpp:280-286) into lane temps 0, 1, 2
    TensorArgs ta{};
    ZF(ta.a0, a0); ZF(ta.a1, a1); ZF(ta.b0, b0); ZF(ta.b1, b1);
    ta.d0 = lane_temp_field(ctx, 0);
    ta.d1 = lane_temp_field(ctx, 1);
    ta.d2 = lane_temp_field(ctx, 2);
    CK(launch_tensor(ctx->nat.pc, ctx->poly, ctx->n, limbs, nz, ta, ctx->st));
    // 2-3. relinearise d2 and add (:288-293): d0 += ks0, d1 += ks1 in the
    //      key switch's ModDown epilogue
    KsFuse f{};
    f.has_acc = 1;
    f.acc0 = ta.d0;
    f.acc1 = ta.d1;
    int rc = ks_batch(ctx, ta.d2, ta.d0, ta.d1, nz, ctx->relin_off, limbs, &f, true, ctx->relin_prep);
    if (rc != AFHE_OK) return rc;
    // 4. rescale into the destination (:296-305)
    return rescale_batch(ctx, t0, t1, o0, o1, limbs);
}

// One rotation step on nz ciphertexts (fhe_host_driver.cpp:331-359):
//   dst = (auto(c0) + ks0, ks1), ks = KS(auto(c1)),
// or, with acc, dst = acc + that. One fused key switch: the automorphism is
// applied on the key switch's loads and the additions in its epilogue.
// Inputs may alias outputs; acc may alias dst.
int rotate_step_batch(afhe_ctx* ctx, const ZField& in0, const ZField& in1, const ZField& d0, const ZField& d1,
                      uint32_t nz, int32_t step, uint32_t limbs, const ZField* acc0 = nullptr,
                      const ZField* acc1 = nullptr, bool fused_ok = true, const ZField* lvz = nullptr) {
    auto it = ctx->rot.find(step);
    if (it == ctx->rot.end()) return fail(ctx, AFHE_E_NOKEY, "rotation key not found for step " + std::to_string(step));
    const RotKey& rk = it->second;
    KsFuse f{};
    f.map = rk.map;
    f.has_c0 = 1;
    f.c0 = in0;
    f.has_acc = acc0 != nullptr;
    if (acc0) { f.acc0 = *acc0; f.acc1 = *acc1; }
    return ks_batch(ctx, in1, d0, d1, nz, rk.evk_offset, limbs, &f, fused_ok, rk.prep, lvz);
}

// Whether the one-kernel key switch may run a rotation batch: its entries run
// concurrently and each reads input limb i up to the point where it writes
// output limb i, so every input polynomial must either be disjoint from every
// output polynomial or coincide exactly with an output of its own entry (all
// polynomials span w words).
bool fused_rotation_safe(const Offs& i0, const Offs& i1, const Offs& o0, const Offs& o1, u64 w) {
    const size_t nz = i0.size();
    std::vector<std::pair<u64, uint32_t>> outs;
    outs.reserve(2 * nz);
    for (uint32_t z = 0; z < nz; ++z) {
        outs.emplace_back(o0[z], z);
        outs.emplace_back(o1[z], z);
    }
    std::sort(outs.begin(), outs.end());
    for (uint32_t z = 0; z < nz; ++z)
        for (u64 a : {i0[z], i1[z]}) {
            // outputs starting in (a - w, a + w) overlap [a, a + w)
            const u64 lo = a >= w ? a - w + 1 : 0;
            auto it = std::lower_bound(outs.begin(), outs.end(), std::make_pair(lo, 0u));
            for (; it != outs.end() && it->first < a + w; ++it)
                if (it->second != z || it->first != a) return false;
        }
    return true;
}

// eval_rotate on nz ciphertexts by the same amount (fhe_host_driver.cpp:361-404):
// |r| decomposed into descending powers of two, sign kept. With `accumulate`,
// dst += rotate(in) instead (the last step adds into dst in its epilogue).
int rotate_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* dst, uint32_t nz, int32_t total,
                 uint32_t limbs, bool accumulate = false) {
    Offs i0(nz), i1(nz), o0(nz), o1(nz);
    for (uint32_t z = 0; z < nz; ++z) {
        i0[z] = in[z].c0_offset; i1[z] = in[z].c1_offset;
        o0[z] = dst[z].c0_offset; o1[z] = dst[z].c1_offset;
    }
    if (total == 0 && accumulate) {   // dst += in
        Offs A(2 * nz), B(2 * nz);
        for (uint32_t z = 0; z < nz; ++z) {
            A[2 * z] = o0[z]; A[2 * z + 1] = o1[z];
            B[2 * z] = i0[z]; B[2 * z + 1] = i1[z];
        }
        return ew_batch(ctx, EW_ADD, A, &B, A, limbs);
    }
    if (total == 0) {
        for (uint32_t z = 0; z < nz; ++z) {
            CK(cudaMemcpyAsync(ctx->poly + o0[z], ctx->poly + i0[z], (u64)limbs * ctx->n * 8, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(ctx->poly + o1[z], ctx->poly + i1[z], (u64)limbs * ctx->n * 8, cudaMemcpyDeviceToDevice, ctx->st));
        }
        return AFHE_OK;
    }
    // every step's key must exist before anything is launched
    long long rem = std::llabs((long long)total);
    const int sign = total > 0 ? 1 : -1;
    std::vector<int32_t> steps;
    while (rem > 0) {
        long long s = 1;
        while ((s << 1) <= rem) s <<= 1;
        steps.push_back((int32_t)(sign * s));
        rem -= s;
    }
    for (int32_t s : steps)
        if (!ctx->rot.count(s)) return fail(ctx, AFHE_E_NOKEY, "rotation key not found for step " + std::to_string(s));
    const bool fused_ok = fused_rotation_safe(i0, i1, o0, o1, (u64)limbs * ctx->n);
    ZField fi0, fi1, fo0, fo1;
    ZF(fi0, i0); ZF(fi1, i1); ZF(fo0, o0); ZF(fo1, o1);
    // chain temporaries (lane temps 2 and 5 are unused by a single step)
    const ZField x0 = lane_temp_field(ctx, 2), x1 = lane_temp_field(ctx, 5);
    ZField c0 = fi0, c1 = fi1;
    for (size_t k = 0; k < steps.size(); ++k) {
        const bool last = k + 1 == steps.size();
        const ZField& n0 = last ? fo0 : x0;
        const ZField& n1 = last ? fo1 : x1;
        int rc = (last && accumulate)
                     ? rotate_step_batch(ctx, c0, c1, n0, n1, nz, steps[k], limbs, &fo0, &fo1, fused_ok)
                     : rotate_step_batch(ctx, c0, c1, n0, n1, nz, steps[k], limbs, nullptr, nullptr, fused_ok);
        if (rc != AFHE_OK) return rc;
        c0 = n0;
        c1 = n1;
    }
    return AFHE_OK;
}

u64 key_region_words(const afhe_ctx* ctx) { return 2ull * ctx->dnum * (ctx->L + ctx->K) * ctx->n; }

// The one-kernel key switch reads a registered key through a prepared copy:
// (k mod q, Shoup companion) per key word, derived on the device.
int prep_key(afhe_ctx* ctx, u64 evk, ulonglong2** prep) {
    if (!ctx->ks_fused) return AFHE_OK;
    const u64 words = key_region_words(ctx);
    if (!*prep) CK(cudaMalloc((void**)prep, words * sizeof(ulonglong2)));
    CK(launch_key_prep(ctx->key + evk, *prep, ctx->nat.pc, ctx->n, ctx->L + ctx->K, words, ctx->st));
    return AFHE_OK;
}

template <class F>
int for_chunks(afhe_ctx* ctx, uint32_t count, F f) {
    const uint32_t w = ctx->chunk ? ctx->chunk : ctx->lanes;
    for (uint32_t s = 0; s < count; s += w) {
        uint32_t m = count - s < w ? count - s : w;
        int rc = f(s, m);
        if (rc != AFHE_OK) return rc;
    }
    return AFHE_OK;
}

}  // namespace

int afhe::refresh_key_preps(afhe_ctx* ctx, u64 off, u64 count) {
    const u64 words = key_region_words(ctx);
    auto hit = [&](u64 evk) { return count && off < evk + words && evk < off + count; };
    int rc;
    if (ctx->has_relin && ctx->relin_prep && hit(ctx->relin_off))
        if ((rc = prep_key(ctx, ctx->relin_off, &ctx->relin_prep)) != AFHE_OK) return rc;
    for (auto& kv : ctx->rot)
        if (kv.second.prep && hit(kv.second.evk_offset))
            if ((rc = prep_key(ctx, kv.second.evk_offset, &kv.second.prep)) != AFHE_OK) return rc;
    return AFHE_OK;
}

void afhe::free_key_preps(afhe_ctx* ctx) {
    if (ctx->relin_prep) cudaFree(ctx->relin_prep);
    ctx->relin_prep = nullptr;
    for (auto& kv : ctx->rot) {
        if (kv.second.prep) cudaFree(kv.second.prep);
        kv.second.prep = nullptr;
    }
}

extern "C" {

// ---- key directory ----------------------------------------------------------
int afhe_set_relin_key(afhe_ctx* ctx, uint64_t evk) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc = check_key(ctx, evk);
    if (rc != AFHE_OK) return rc;
    cudaSetDevice(ctx->device);
    if ((rc = prep_key(ctx, evk, &ctx->relin_prep)) != AFHE_OK) return rc;
    ctx->relin_off = evk;
    ctx->has_relin = true;
    return AFHE_OK;
}

int afhe_add_rotation_key(afhe_ctx* ctx, int32_t step, uint64_t evk) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc = check_key(ctx, evk);
    if (rc != AFHE_OK) return rc;
    cudaSetDevice(ctx->device);
    RotKey rk;
    rk.step = step;
    rk.galois = galois_elt_for_step(ctx->log_n, step);
    rk.evk_offset = evk;
    std::vector<uint32_t> map(ctx->n);
    automorphism_map(ctx->log_n, rk.galois, map.data());
    auto old = ctx->rot.find(step);
    if (old != ctx->rot.end()) {
        rk.map = old->second.map;
        rk.prep = old->second.prep;
    } else {
        CK(cudaMalloc((void**)&rk.map, ctx->n * sizeof(uint32_t)));
    }
    CK(cudaMemcpy(rk.map, map.data(), ctx->n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    rc = prep_key(ctx, evk, &rk.prep);
    ctx->rot[step] = rk;
    return rc;
}

int afhe_has_rotation_key(afhe_ctx* ctx, int32_t step) { return ctx && ctx->rot.count(step) ? 1 : 0; }

// ---- primitives (native tables) ------------------------------------------------
static int ntt_native(afhe_ctx* ctx, bool inv, uint64_t src, uint64_t dst, uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs_ext(ctx, limbs)) || (rc = check_poly(ctx, src, limbs)) || (rc = check_poly(ctx, dst, limbs))) return rc;
    const u64 w = (u64)limbs * ctx->n;
    u64 s = src;
    if (src != dst && overlap(src, w, dst, w)) {
        CK(cudaMemcpyAsync(ctx->scr, ctx->poly + src, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
        s = ctx->prm.poly_words;
    }
    ZBases zb{};
    zb.src = zf_const(s);
    zb.mid = zf_const(dst);
    zb.out = zf_const(dst);
    CK(launch_ntt_plain(inv, ctx->log_n, ctx->nat.view(), ctx->jobs_qp, limbs, ctx->poly, ctx->poly, 1, zb, ctx->st));
    return AFHE_OK;
}

int afhe_ntt(afhe_ctx* ctx, uint64_t src, uint64_t dst, uint32_t limbs) { return ntt_native(ctx, false, src, dst, limbs); }
int afhe_intt(afhe_ctx* ctx, uint64_t src, uint64_t dst, uint32_t limbs) { return ntt_native(ctx, true, src, dst, limbs); }

static int ew_single(afhe_ctx* ctx, ElemOp op, uint64_t a, uint64_t b, uint64_t dst, uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs_ext(ctx, limbs)) || (rc = check_poly(ctx, a, limbs)) || (rc = check_poly(ctx, b, limbs)) ||
        (rc = check_poly(ctx, dst, limbs)))
        return rc;
    const u64 w = (u64)limbs * ctx->n;
    u64 aa = a, bb = b;
    if (a != dst && overlap(a, w, dst, w)) {
        CK(cudaMemcpyAsync(ctx->scr, ctx->poly + a, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
        aa = ctx->prm.poly_words;
    }
    if (b != dst && overlap(b, w, dst, w)) {
        CK(cudaMemcpyAsync(ctx->scr + w, ctx->poly + b, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
        bb = ctx->prm.poly_words + w;
    }
    return ew_fields(ctx, op, zf_const(aa), zf_const(bb), zf_const(dst), 1, limbs);
}

int afhe_poly_add(afhe_ctx* c, uint64_t a, uint64_t b, uint64_t d, uint32_t l) { return ew_single(c, EW_ADD, a, b, d, l); }
int afhe_poly_sub(afhe_ctx* c, uint64_t a, uint64_t b, uint64_t d, uint32_t l) { return ew_single(c, EW_SUB, a, b, d, l); }
int afhe_poly_mul_ntt(afhe_ctx* c, uint64_t a, uint64_t b, uint64_t d, uint32_t l) { return ew_single(c, EW_MUL, a, b, d, l); }

int afhe_automorphism(afhe_ctx* ctx, uint64_t src, uint32_t galois, uint64_t dst, uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs_ext(ctx, limbs)) || (rc = check_poly(ctx, src, limbs)) || (rc = check_poly(ctx, dst, limbs))) return rc;
    if ((galois & 1u) == 0 || galois >= 2 * ctx->n) return fail(ctx, AFHE_E_ARG, "galois element must be odd and < 2N");
    std::vector<uint32_t> map(ctx->n);
    automorphism_map(ctx->log_n, galois, map.data());
    const u64 w = (u64)limbs * ctx->n;
    // map in scratch words [0, N/2), the source copy after it (a gather cannot run in place)
    uint32_t* dmap = (uint32_t*)(ctx->scr);
    CK(cudaMemcpyAsync(dmap, map.data(), ctx->n * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->scr + ctx->n, ctx->poly + src, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
    ZBases zb{};
    zb.src = zf_const(ctx->prm.poly_words + ctx->n);
    zb.out = zf_const(dst);
    CK(launch_automorphism(dmap, nullptr, ctx->poly, ctx->n, limbs, 1, zb, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));   // the host map buffer goes out of scope
    return AFHE_OK;
}

int afhe_rescale(afhe_ctx* ctx, uint64_t c0_in, uint64_t c1_in, uint64_t c0_out, uint64_t c1_out, uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 2)) || (rc = check_poly(ctx, c0_in, limbs)) || (rc = check_poly(ctx, c1_in, limbs)) ||
        (rc = check_poly(ctx, c0_out, limbs - 1)) || (rc = check_poly(ctx, c1_out, limbs - 1)))
        return rc;
    // inputs go to lane temps first so that any aliasing with the outputs is safe
    const u64 w = (u64)limbs * ctx->n;
    u64 t0 = lane_temp(ctx, 0, 0), t1 = lane_temp(ctx, 0, 1);
    CK(cudaMemcpyAsync(ctx->poly + t0, ctx->poly + c0_in, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->poly + t1, ctx->poly + c1_in, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
    return rescale_batch(ctx, Offs{t0}, Offs{t1}, Offs{c0_out}, Offs{c1_out}, limbs);
}

int afhe_key_switch(afhe_ctx* ctx, uint64_t src, uint64_t evk, uint64_t d0, uint64_t d1, uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_poly(ctx, src, limbs)) || (rc = check_poly(ctx, d0, limbs)) ||
        (rc = check_poly(ctx, d1, limbs)) || (rc = check_key(ctx, evk)))
        return rc;
    const u64 w = (u64)limbs * ctx->n;
    u64 t = lane_temp(ctx, 0, 2);
    CK(cudaMemcpyAsync(ctx->poly + t, ctx->poly + src, w * 8, cudaMemcpyDeviceToDevice, ctx->st));
    // a registered key at this offset brings its prepared copy
    const ulonglong2* prep = nullptr;
    if (ctx->has_relin && ctx->relin_off == evk) prep = ctx->relin_prep;
    for (const auto& kv : ctx->rot)
        if (!prep && kv.second.evk_offset == evk) prep = kv.second.prep;
    return ks_batch(ctx, zf_const(t), zf_const(d0), zf_const(d1), 1, evk, limbs, nullptr, true, prep);
}

// ---- composite operators ------------------------------------------------------
int afhe_eval_add(afhe_ctx* ctx, uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1, uint64_t d0, uint64_t d1,
                  uint32_t limbs) {
    int rc = afhe_poly_add(ctx, a0, b0, d0, limbs);
    if (rc != AFHE_OK) return rc;
    return afhe_poly_add(ctx, a1, b1, d1, limbs);
}

int afhe_eval_sub_plain(afhe_ctx* ctx, uint64_t a0, uint64_t a1, uint64_t pt, uint64_t d0, uint64_t d1, uint32_t limbs) {
    int rc = afhe_poly_sub(ctx, a0, pt, d0, limbs);
    if (rc != AFHE_OK) return rc;
    if (a1 != d1) {
        if ((rc = check_poly(ctx, a1, limbs)) || (rc = check_poly(ctx, d1, limbs))) return rc;
        CK(cudaMemcpyAsync(ctx->poly + d1, ctx->poly + a1, (u64)limbs * ctx->n * 8, cudaMemcpyDeviceToDevice, ctx->st));
    }
    return AFHE_OK;
}

int afhe_eval_mult_relin_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d,
                                       uint32_t count, uint32_t limbs) {
    if (!ctx || (!a && count) || (!b && count) || (!d && count)) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 2)) || (rc = check_cts(ctx, a, count, limbs)) ||
        (rc = check_cts(ctx, b, count, limbs)) || (rc = check_cts(ctx, d, count, limbs - 1)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) { return mult_relin_rescale_batch(ctx, a + s, b + s, d + s, m, limbs); });
}

int afhe_eval_mult_relin_rescale(afhe_ctx* ctx, uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1, uint64_t d0,
                                 uint64_t d1, uint32_t limbs) {
    afhe_ct_ref a{a0, a1}, b{b0, b1}, d{d0, d1};
    return afhe_eval_mult_relin_rescale_batch(ctx, &a, &b, &d, 1, limbs);
}

int afhe_eval_mult_plain_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d,
                                       uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !pt || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 2)) || (rc = check_cts(ctx, a, count, limbs)) ||
        (rc = check_cts(ctx, d, count, limbs - 1)))
        return rc;
    for (uint32_t i = 0; i < count; ++i)
        if ((rc = check_poly(ctx, pt[i], limbs))) return rc;
    // fhe_host_driver.cpp:308-329: (c0 * pt, c1 * pt), then rescale
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(2 * m), P(2 * m), T(2 * m), t0(m), t1(m), o0(m), o1(m);
        for (uint32_t z = 0; z < m; ++z) {
            t0[z] = lane_temp(ctx, z, 0);
            t1[z] = lane_temp(ctx, z, 1);
            A[2 * z] = a[s + z].c0_offset; A[2 * z + 1] = a[s + z].c1_offset;
            P[2 * z] = pt[s + z]; P[2 * z + 1] = pt[s + z];
            T[2 * z] = t0[z]; T[2 * z + 1] = t1[z];
            o0[z] = d[s + z].c0_offset; o1[z] = d[s + z].c1_offset;
        }
        int r = ew_batch(ctx, EW_MUL, A, &P, T, limbs);
        if (r != AFHE_OK) return r;
        return rescale_batch(ctx, t0, t1, o0, o1, limbs);
    });
}

int afhe_rescale_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* d, uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 2)) || (rc = check_cts(ctx, a, count, limbs)) ||
        (rc = check_cts(ctx, d, count, limbs - 1)))
        return rc;
    // OP 8 on both polynomials (fhe_accel_top.cpp:286-292); the inputs go to
    // lane temps first, so outputs may alias any input
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(2 * m), T(2 * m), t0(m), t1(m), o0(m), o1(m);
        for (uint32_t z = 0; z < m; ++z) {
            t0[z] = lane_temp(ctx, z, 0);
            t1[z] = lane_temp(ctx, z, 1);
            A[2 * z] = a[s + z].c0_offset; A[2 * z + 1] = a[s + z].c1_offset;
            T[2 * z] = t0[z]; T[2 * z + 1] = t1[z];
            o0[z] = d[s + z].c0_offset; o1[z] = d[s + z].c1_offset;
        }
        int r = ew_batch(ctx, EW_COPY, A, nullptr, T, limbs);
        if (r != AFHE_OK) return r;
        return rescale_batch(ctx, t0, t1, o0, o1, limbs);
    });
}

int afhe_eval_mult_plain_rescale(afhe_ctx* ctx, uint64_t a0, uint64_t a1, uint64_t pt, uint64_t d0, uint64_t d1,
                                 uint32_t limbs) {
    afhe_ct_ref a{a0, a1}, d{d0, d1};
    return afhe_eval_mult_plain_rescale_batch(ctx, &a, &pt, &d, 1, limbs);
}

int afhe_eval_rotate_single_step(afhe_ctx* ctx, uint64_t i0, uint64_t i1, uint64_t d0, uint64_t d1, int32_t step,
                                 uint32_t limbs) {
    if (!ctx) return fail(nullptr, AFHE_E_ARG, "null context");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_poly(ctx, i0, limbs)) || (rc = check_poly(ctx, i1, limbs)) ||
        (rc = check_poly(ctx, d0, limbs)) || (rc = check_poly(ctx, d1, limbs)))
        return rc;
    const bool fused_ok = fused_rotation_safe(Offs{i0}, Offs{i1}, Offs{d0}, Offs{d1}, (u64)limbs * ctx->n);
    return rotate_step_batch(ctx, zf_const(i0), zf_const(i1), zf_const(d0), zf_const(d1), 1, step, limbs, nullptr,
                             nullptr, fused_ok);
}

int afhe_eval_rotate_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* dst, uint32_t count, int32_t total,
                           uint32_t limbs) {
    if (!ctx || (!in && count) || (!dst && count)) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, in, count, limbs)) ||
        (rc = check_cts(ctx, dst, count, limbs)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) { return rotate_batch(ctx, in + s, dst + s, m, total, limbs); });
}

int afhe_eval_rotate_accumulate_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* acc, uint32_t count,
                                      int32_t total, uint32_t limbs) {
    if (!ctx || (!in && count) || (!acc && count)) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, in, count, limbs)) ||
        (rc = check_cts(ctx, acc, count, limbs)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        return rotate_batch(ctx, in + s, acc + s, m, total, limbs, true);
    });
}

int afhe_eval_rotate_accumulate_levels_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* acc,
                                             const uint32_t* levels, uint32_t count, int32_t total) {
    if (!ctx || (count && (!in || !acc || !levels))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    uint32_t top = 1;
    for (uint32_t i = 0; i < count; ++i) {
        if ((rc = check_limbs(ctx, levels[i], 1)) || (rc = check_cts(ctx, in + i, 1, levels[i])) ||
            (rc = check_cts(ctx, acc + i, 1, levels[i])))
            return rc;
        top = std::max(top, levels[i]);
    }
    long long rem = std::llabs((long long)total);
    std::vector<int32_t> steps;
    while (rem > 0) {
        long long st = 1;
        while ((st << 1) <= rem) st <<= 1;
        steps.push_back((int32_t)(total > 0 ? st : -st));
        rem -= st;
    }
    for (int32_t st : steps)
        if (!ctx->rot.count(st)) return fail(ctx, AFHE_E_NOKEY, "rotation key not found for step " + std::to_string(st));
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) -> int {
        Offs i0(m), i1(m), o0(m), o1(m), lv(m);
        uint32_t mx = 1;
        for (uint32_t z = 0; z < m; ++z) {
            i0[z] = in[s + z].c0_offset; i1[z] = in[s + z].c1_offset;
            o0[z] = acc[s + z].c0_offset; o1[z] = acc[s + z].c1_offset;
            lv[z] = levels[s + z];
            mx = std::max(mx, levels[s + z]);
        }
        if (total == 0 || !ctx->ks_fused || !fused_rotation_safe(i0, i1, o0, o1, (u64)top * ctx->n)) {
            // one launch sequence per level, entries of a level together
            std::map<uint32_t, std::vector<uint32_t>> by;
            for (uint32_t z = 0; z < m; ++z) by[levels[s + z]].push_back(z);
            for (auto& kv : by) {
                std::vector<afhe_ct_ref> a, b;
                for (uint32_t z : kv.second) { a.push_back(in[s + z]); b.push_back(acc[s + z]); }
                int r = afhe_eval_rotate_accumulate_batch(ctx, a.data(), b.data(), (uint32_t)a.size(), total, kv.first);
                if (r != AFHE_OK) return r;
            }
            return AFHE_OK;
        }
        ZField fi0, fi1, fo0, fo1, flv;
        ZF(fi0, i0); ZF(fi1, i1); ZF(fo0, o0); ZF(fo1, o1); ZF(flv, lv);
        const ZField x0 = lane_temp_field(ctx, 2), x1 = lane_temp_field(ctx, 5);
        ZField c0 = fi0, c1 = fi1;
        for (size_t k = 0; k < steps.size(); ++k) {
            const bool last = k + 1 == steps.size();
            const ZField& n0 = last ? fo0 : x0;
            const ZField& n1 = last ? fo1 : x1;
            int r = rotate_step_batch(ctx, c0, c1, n0, n1, m, steps[k], mx, last ? &fo0 : nullptr,
                                      last ? &fo1 : nullptr, true, &flv);
            if (r != AFHE_OK) return r;
            c0 = n0;
            c1 = n1;
        }
        return AFHE_OK;
    });
}

int afhe_eval_rotate_steps_batch(afhe_ctx* ctx, const afhe_ct_ref* in, const afhe_ct_ref* dst, const int32_t* steps,
                                 uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!in || !dst || !steps))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, in, count, limbs)) ||
        (rc = check_cts(ctx, dst, count, limbs)))
        return rc;
    for (uint32_t i = 0; i < count; ++i)
        if (!ctx->rot.count(steps[i]))
            return fail(ctx, AFHE_E_NOKEY, "rotation key not found for step " + std::to_string(steps[i]));
    const u64 n = ctx->n, S = (u64)ctx->L + ctx->K;
    const OpTabs& t = ctx->lv[limbs];
    const LevelJobs& lj = ctx->lvjobs[limbs];
    // eval_rotate_single_step per entry (fhe_host_driver.cpp:331-359), each
    // with its own key and automorphism, in one key switch launch sequence.
    // The multi-kernel key switch reads every input before it writes any
    // output, so outputs may alias inputs anywhere; the one-kernel key switch
    // runs its entries concurrently, so it takes a chunk whose outputs alias
    // only their own entry's inputs.
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) -> int {
        Offs i0(m), i1(m), o0(m), o1(m), maps(m), keys(m), preps(m);
        bool all_prep = true;
        for (uint32_t z = 0; z < m; ++z) {
            const RotKey& rk = ctx->rot.at(steps[s + z]);
            i0[z] = in[s + z].c0_offset; i1[z] = in[s + z].c1_offset;
            o0[z] = dst[s + z].c0_offset; o1[z] = dst[s + z].c1_offset;
            maps[z] = (u64)(uintptr_t)rk.map;
            keys[z] = rk.evk_offset;
            preps[z] = (u64)(uintptr_t)rk.prep;
            all_prep = all_prep && rk.prep;
        }
        KsFuse f{};
        f.has_c0 = 1;
        f.per_z = 1;
        ZF(f.c0, i0);
        ZF(f.mapz, maps);
        ZF(f.keyz, keys);
        ZBases zb{};
        ZF(zb.src, i1);
        ZF(zb.out, o0);
        ZF(zb.aux, o1);
        zb.mid = lane_field(ctx, &Lane::ks);
        if (ctx->ks_fused && m >= ctx->fused_min && fused_rotation_safe(i0, i1, o0, o1, (u64)limbs * n)) {
            const ulonglong2* prep = nullptr;
            if (all_prep) {
                ZF(f.prepz, preps);
                prep = ctx->rot.at(steps[s]).prep;
            }
            CK(launch_key_switch_fused(ctx->log_n, t, limbs, ctx->K, ctx->key, 0, (u64)ctx->dnum * S * n, (uint32_t)S,
                                       ctx->L, ctx->poly, ctx->scr, m, zb, ctx->st, &f, prep, nullptr, nullptr,
                                       (int)ctx->ks_ept, (int)ctx->ks_slice));
            return AFHE_OK;
        }
        CK(launch_key_switch(ctx->log_n, t, ctx->jobs_qp, lj.modup, lj.n_modup, ctx->L, limbs, ctx->K, ctx->key, 0,
                             (u64)ctx->dnum * S * n, (uint32_t)S, ctx->L, ctx->poly, ctx->scr, m, zb, ctx->st, &f));
        return AFHE_OK;
    });
}

int afhe_eval_rotate(afhe_ctx* ctx, uint64_t i0, uint64_t i1, uint64_t d0, uint64_t d1, int32_t total, uint32_t limbs) {
    afhe_ct_ref in{i0, i1}, d{d0, d1};
    return afhe_eval_rotate_batch(ctx, &in, &d, 1, total, limbs);
}

// Batched elementwise composites: ciphertext i of the batch is computed
// exactly as the single call would; distinct batch entries must not overlap
// each other's outputs (in-place per entry is fine).
int afhe_eval_add_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d,
                        uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !b || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, a, count, limbs)) ||
        (rc = check_cts(ctx, b, count, limbs)) || (rc = check_cts(ctx, d, count, limbs)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(2 * m), B(2 * m), D(2 * m);
        for (uint32_t z = 0; z < m; ++z) {
            A[2 * z] = a[s + z].c0_offset; A[2 * z + 1] = a[s + z].c1_offset;
            B[2 * z] = b[s + z].c0_offset; B[2 * z + 1] = b[s + z].c1_offset;
            D[2 * z] = d[s + z].c0_offset; D[2 * z + 1] = d[s + z].c1_offset;
        }
        return ew_batch(ctx, EW_ADD, A, &B, D, limbs);
    });
}

int afhe_eval_sub_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* b, const afhe_ct_ref* d,
                        uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !b || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, a, count, limbs)) ||
        (rc = check_cts(ctx, b, count, limbs)) || (rc = check_cts(ctx, d, count, limbs)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(2 * m), B(2 * m), D(2 * m);
        for (uint32_t z = 0; z < m; ++z) {
            A[2 * z] = a[s + z].c0_offset; A[2 * z + 1] = a[s + z].c1_offset;
            B[2 * z] = b[s + z].c0_offset; B[2 * z + 1] = b[s + z].c1_offset;
            D[2 * z] = d[s + z].c0_offset; D[2 * z + 1] = d[s + z].c1_offset;
        }
        return ew_batch(ctx, EW_SUB, A, &B, D, limbs);
    });
}

int afhe_eval_add_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d,
                              uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !pt || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, a, count, limbs)) || (rc = check_cts(ctx, d, count, limbs)))
        return rc;
    for (uint32_t i = 0; i < count; ++i)
        if ((rc = check_poly(ctx, pt[i], limbs))) return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(m), P(m), D(m), A2, D2;
        for (uint32_t z = 0; z < m; ++z) { A[z] = a[s + z].c0_offset; P[z] = pt[s + z]; D[z] = d[s + z].c0_offset; }
        int r = ew_batch(ctx, EW_ADD, A, &P, D, limbs);
        if (r != AFHE_OK) return r;
        for (uint32_t z = 0; z < m; ++z)
            if (a[s + z].c1_offset != d[s + z].c1_offset) {
                A2.push_back(a[s + z].c1_offset);
                D2.push_back(d[s + z].c1_offset);
            }
        return A2.empty() ? AFHE_OK : ew_batch(ctx, EW_COPY, A2, nullptr, D2, limbs);
    });
}

int afhe_automorphism_batch(afhe_ctx* ctx, const uint64_t* src, const uint32_t* galois, const uint64_t* dst,
                            uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!src || !galois || !dst))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs_ext(ctx, limbs))) return rc;
    const u64 w = (u64)limbs * ctx->n;
    std::vector<std::pair<u64, int>> ends;    // interval ends: sources (+1 / -1) and destinations (+2 / -2)
    for (uint32_t i = 0; i < count; ++i) {
        if ((rc = check_poly(ctx, src[i], limbs)) || (rc = check_poly(ctx, dst[i], limbs))) return rc;
        if ((galois[i] & 1u) == 0 || galois[i] >= 2 * ctx->n)
            return fail(ctx, AFHE_E_ARG, "galois element must be odd and < 2N");
        ends.push_back({src[i], 1});
        ends.push_back({src[i] + w, -1});
        ends.push_back({dst[i], 2});
        ends.push_back({dst[i] + w, -2});
    }
    // a gather cannot run in place: no destination may overlap any source
    std::sort(ends.begin(), ends.end());
    int open_src = 0, open_dst = 0;
    for (const auto& e : ends) {
        if (e.second == 1) ++open_src;
        else if (e.second == -1) --open_src;
        else if (e.second == 2) ++open_dst;
        else --open_dst;
        if (open_src > 0 && open_dst > 0) return fail(ctx, AFHE_E_ARG, "a destination overlaps a source");
    }
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t* d = nullptr;
        if ((rc = cached_map(ctx, galois[i], &d))) return rc;
    }
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs S(m), D(m), M(m);
        for (uint32_t z = 0; z < m; ++z) {
            S[z] = src[s + z];
            D[z] = dst[s + z];
            M[z] = (u64)(uintptr_t)ctx->auto_maps.at(galois[s + z]);
        }
        ZBases zb{};
        ZField maps;
        ZF(zb.src, S);
        ZF(zb.out, D);
        ZF(maps, M);
        CK(launch_automorphism_z(maps, ctx->poly, ctx->n, limbs, m, zb, ctx->st));
        return (int)AFHE_OK;
    });
}

int afhe_eval_mac_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* out, const uint32_t* first_group, uint32_t count,
                              const afhe_mac_group* groups, const afhe_mac_term* terms, uint32_t limbs,
                              uint32_t accumulate) {
    if (!ctx || (count && (!out || !first_group || !groups || !terms))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, out, count, limbs))) return rc;
    const u64 w = (u64)limbs * ctx->n;
    // interval ends: operands read (+1 / -1) and outputs (+2 / -2); an output
    // may overlap nothing else of the call (its own accumulation is read in place)
    std::vector<std::pair<u64, int>> ends;
    auto read = [&](u64 off) {
        ends.push_back({off, 1});
        ends.push_back({off + w, -1});
    };
    for (uint32_t j = 0; j < count; ++j) {
        if (first_group[j + 1] < first_group[j]) return fail(ctx, AFHE_E_ARG, "group ranges must not decrease");
        for (uint32_t g = first_group[j]; g < first_group[j + 1]; ++g) {
            const afhe_mac_group& G = groups[g];
            if (G.src.c0_offset != AFHE_MAC_UNIT) {
                if ((rc = check_poly(ctx, G.src.c0_offset, limbs)) || (rc = check_poly(ctx, G.src.c1_offset, limbs)))
                    return rc;
                read(G.src.c0_offset);
                read(G.src.c1_offset);
            }
            for (uint32_t t = G.first_term; t < G.first_term + G.n_terms; ++t) {
                if ((rc = check_poly(ctx, terms[t].pt, limbs))) return rc;
                if ((terms[t].galois & 1u) == 0 || terms[t].galois >= 2 * ctx->n)
                    return fail(ctx, AFHE_E_ARG, "galois element must be odd and < 2N");
                read(terms[t].pt);
            }
        }
        ends.push_back({out[j].c0_offset, 2});
        ends.push_back({out[j].c0_offset + w, -2});
        ends.push_back({out[j].c1_offset, 2});
        ends.push_back({out[j].c1_offset + w, -2});
    }
    std::sort(ends.begin(), ends.end());
    int open_src = 0, open_dst = 0;
    for (const auto& e : ends) {
        if (e.second == 1) ++open_src;
        else if (e.second == -1) --open_src;
        else if (e.second == 2) ++open_dst;
        else --open_dst;
        if (open_dst > 1 || (open_src > 0 && open_dst > 0))
            return fail(ctx, AFHE_E_ARG, "an output overlaps another output or an operand");
    }
    // terms between folds of the 128-bit accumulators: each product < q^2
    u64 qmax = 0;
    for (uint32_t l = 0; l < limbs; ++l) qmax = std::max<u64>(qmax, ctx->prm.q[l]);
    const unsigned __int128 sq = (unsigned __int128)(qmax - 1) * (qmax - 1);
    const unsigned __int128 room = ~(unsigned __int128)0 / (sq ? sq : 1);
    const uint32_t reduce_every = room > 0x7fffffff ? 0x7fffffffu : (uint32_t)room;
    // launches of whole jobs whose descriptors fit one segment of the ring
    const size_t seg = ctx->ring.seg_words - 96;
    std::vector<MacJob> J;
    std::vector<MacGroup> G;
    std::vector<MacTerm> T;
    auto words = [&](size_t j, size_t g, size_t t) {
        return (j * sizeof(MacJob) + g * sizeof(MacGroup) + t * sizeof(MacTerm)) / sizeof(u64);
    };
    auto flush = [&]() -> int {
        if (J.empty()) return AFHE_OK;
        u64 *dj = nullptr, *dg = nullptr, *dt = nullptr;
        int r;
        if ((r = ring_put(ctx, J.data(), J.size() * sizeof(MacJob) / sizeof(u64), &dj))) return r;
        if ((r = ring_put(ctx, G.data(), std::max<size_t>(G.size(), 1) * sizeof(MacGroup) / sizeof(u64), &dg)))
            return r;
        if ((r = ring_put(ctx, T.data(), std::max<size_t>(T.size(), 1) * sizeof(MacTerm) / sizeof(u64), &dt)))
            return r;
        CK(launch_mac_plain(ctx->nat.pc, ctx->poly, ctx->n, limbs, (uint32_t)J.size(), (const MacJob*)dj,
                            (const MacGroup*)dg, (const MacTerm*)dt, reduce_every, accumulate ? 1 : 0, ctx->st));
        J.clear();
        G.clear();
        T.clear();
        return AFHE_OK;
    };
    G.reserve(1);
    T.reserve(1);
    for (uint32_t j = 0; j < count; ++j) {
        size_t ng = first_group[j + 1] - first_group[j], nt = 0;
        for (uint32_t g = first_group[j]; g < first_group[j + 1]; ++g) nt += groups[g].n_terms;
        if (words(1, std::max<size_t>(ng, 1), std::max<size_t>(nt, 1)) > seg / 3)
            return fail(ctx, AFHE_E_ARG, "too many terms in one output for the descriptor ring");
        if (words(J.size() + 1, G.size() + ng + 1, T.size() + nt + 1) > seg / 3 && (rc = flush())) return rc;
        MacJob mj{out[j].c0_offset, out[j].c1_offset, (uint32_t)G.size(), (uint32_t)(G.size() + ng)};
        J.push_back(mj);
        for (uint32_t g = first_group[j]; g < first_group[j + 1]; ++g) {
            const afhe_mac_group& src = groups[g];
            MacGroup mg{src.src.c0_offset, src.src.c1_offset, (uint32_t)T.size(), (uint32_t)(T.size() + src.n_terms)};
            G.push_back(mg);
            for (uint32_t t = src.first_term; t < src.first_term + src.n_terms; ++t) {
                const uint32_t* map = nullptr;
                if (terms[t].galois != 1 && (rc = cached_map(ctx, terms[t].galois, &map))) return rc;
                T.push_back(MacTerm{terms[t].pt, map});
            }
        }
    }
    return flush();
}

int afhe_eval_diag_inner_batch(afhe_ctx* ctx, const afhe_ct_ref* out, uint32_t count, const afhe_ct_ref* src,
                               uint32_t nb, const uint64_t* unit_pt, const uint32_t* unit_galois,
                               const uint32_t* first_unit, uint64_t pt_stride, uint32_t limbs, uint32_t accumulate) {
    if (!ctx || (count && (!out || !src || !first_unit))) return fail(ctx, AFHE_E_ARG, "null argument");
    if (nb != 1 && nb != 2 && nb != 4 && nb != 8 && nb != 16) return fail(ctx, AFHE_E_ARG, "nb must be 1, 2, 4, 8 or 16");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, out, count, limbs)) ||
        (rc = check_cts(ctx, src, count * nb, limbs)))
        return rc;
    const u64 w = (u64)limbs * ctx->n;
    const u64 span = (u64)(nb - 1) * pt_stride + w;       // a unit's nb plaintexts
    std::vector<std::pair<u64, int>> ends;
    auto read = [&](u64 off, u64 len) {
        ends.push_back({off, 1});
        ends.push_back({off + len, -1});
    };
    for (uint32_t j = 0; j < count; ++j) {
        if (first_unit[j + 1] < first_unit[j]) return fail(ctx, AFHE_E_ARG, "unit ranges must not decrease");
        if (first_unit[j + 1] > first_unit[j] && (!unit_pt || !unit_galois)) return fail(ctx, AFHE_E_ARG, "null argument");
        for (uint32_t k = first_unit[j]; k < first_unit[j + 1]; ++k) {
            if (!range_ok(unit_pt[k], span, ctx->prm.poly_words)) return fail(ctx, AFHE_E_RANGE, "plaintexts out of poly_gmem");
            if ((unit_galois[k] & 1u) == 0 || unit_galois[k] >= 2 * ctx->n)
                return fail(ctx, AFHE_E_ARG, "galois element must be odd and < 2N");
            read(unit_pt[k], span);
        }
        for (uint32_t b = 0; b < nb; ++b) {
            read(src[(u64)j * nb + b].c0_offset, w);
            read(src[(u64)j * nb + b].c1_offset, w);
        }
        ends.push_back({out[j].c0_offset, 2});
        ends.push_back({out[j].c0_offset + w, -2});
        ends.push_back({out[j].c1_offset, 2});
        ends.push_back({out[j].c1_offset + w, -2});
    }
    std::sort(ends.begin(), ends.end());
    int open_src = 0, open_dst = 0;
    for (const auto& e : ends) {
        if (e.second == 1) ++open_src;
        else if (e.second == -1) --open_src;
        else if (e.second == 2) ++open_dst;
        else --open_dst;
        if (open_dst > 1 || (open_src > 0 && open_dst > 0))
            return fail(ctx, AFHE_E_ARG, "an output overlaps another output or an operand");
    }
    u64 qmax = 0;
    for (uint32_t l = 0; l < limbs; ++l) qmax = std::max<u64>(qmax, ctx->prm.q[l]);
    const unsigned __int128 sq = (unsigned __int128)(qmax - 1) * (qmax - 1);
    const unsigned __int128 room = ~(unsigned __int128)0 / (sq ? sq : 1);
    const uint32_t reduce_every = room > 0x7fffffff ? 0x7fffffffu : (uint32_t)room;
    if (reduce_every < nb + 1) return fail(ctx, AFHE_E_ARG, "primes too large for the accumulators; use afhe_eval_mac_plain_batch");
    // the shared-memory form: tiles of 256 words stay put under every map,
    // 16-byte aligned plaintext tiles
    bool staged = ctx->n % 256 == 0 && pt_stride % 2 == 0;
    for (uint32_t j = 0; j < count && staged; ++j)
        for (uint32_t k = first_unit[j]; k < first_unit[j + 1] && staged; ++k) {
            const uint32_t* map = nullptr;
            if (unit_pt[k] % 2) staged = false;
            else if (unit_galois[k] != 1) {
                if ((rc = cached_map(ctx, unit_galois[k], &map))) return rc;
                staged = ctx->auto_map_local[unit_galois[k]];
            }
        }
    const size_t seg = ctx->ring.seg_words - 96;
    std::vector<DiagJob> J;
    std::vector<u64> S;
    std::vector<DiagUnit> U;
    auto flush = [&]() -> int {
        if (J.empty()) return AFHE_OK;
        u64 *dj = nullptr, *ds = nullptr, *du = nullptr;
        int r;
        if (U.empty()) U.push_back(DiagUnit{0, nullptr});
        if ((r = ring_put(ctx, J.data(), J.size() * sizeof(DiagJob) / sizeof(u64), &dj))) return r;
        if ((r = ring_put(ctx, S.data(), S.size(), &ds))) return r;
        if ((r = ring_put(ctx, U.data(), U.size() * sizeof(DiagUnit) / sizeof(u64), &du))) return r;
        CK(launch_diag_inner(ctx->nat.pc, ctx->poly, ctx->n, limbs, (uint32_t)J.size(), nb, (const DiagJob*)dj, ds,
                             (const DiagUnit*)du, pt_stride, reduce_every, accumulate ? 1 : 0, staged,
                             qmax < (1ull << 50), ctx->st));
        J.clear();
        S.clear();
        U.clear();
        return AFHE_OK;
    };
    for (uint32_t j = 0; j < count; ++j) {
        const size_t nu = first_unit[j + 1] - first_unit[j];
        if (3 + 2 * nb + 2 * nu + 2 > seg / 3) return fail(ctx, AFHE_E_ARG, "too many units in one output for the descriptor ring");
        if ((J.size() + 1) * 3 > seg / 3 || S.size() + 2 * nb > seg / 3 || (U.size() + nu + 1) * 2 > seg / 3)
            if ((rc = flush())) return rc;
        J.push_back(DiagJob{out[j].c0_offset, out[j].c1_offset, (uint32_t)U.size(), (uint32_t)(U.size() + nu)});
        for (uint32_t b = 0; b < nb; ++b) {
            S.push_back(src[(u64)j * nb + b].c0_offset);
            S.push_back(src[(u64)j * nb + b].c1_offset);
        }
        for (uint32_t k = first_unit[j]; k < first_unit[j + 1]; ++k) {
            const uint32_t* map = nullptr;
            if (unit_galois[k] != 1 && (rc = cached_map(ctx, unit_galois[k], &map))) return rc;
            U.push_back(DiagUnit{unit_pt[k], map});
        }
    }
    return flush();
}

int afhe_eval_copy_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const afhe_ct_ref* d, uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, a, count, limbs)) || (rc = check_cts(ctx, d, count, limbs)))
        return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(2 * m), D(2 * m);
        for (uint32_t z = 0; z < m; ++z) {
            A[2 * z] = a[s + z].c0_offset; A[2 * z + 1] = a[s + z].c1_offset;
            D[2 * z] = d[s + z].c0_offset; D[2 * z + 1] = d[s + z].c1_offset;
        }
        return ew_batch(ctx, EW_COPY, A, nullptr, D, limbs);
    });
}

int afhe_eval_sub_plain_batch(afhe_ctx* ctx, const afhe_ct_ref* a, const uint64_t* pt, const afhe_ct_ref* d,
                              uint32_t count, uint32_t limbs) {
    if (!ctx || (count && (!a || !pt || !d))) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, a, count, limbs)) || (rc = check_cts(ctx, d, count, limbs)))
        return rc;
    for (uint32_t i = 0; i < count; ++i)
        if ((rc = check_poly(ctx, pt[i], limbs))) return rc;
    return for_chunks(ctx, count, [&](uint32_t s, uint32_t m) {
        Offs A(m), P(m), D(m), A2, D2;
        for (uint32_t z = 0; z < m; ++z) { A[z] = a[s + z].c0_offset; P[z] = pt[s + z]; D[z] = d[s + z].c0_offset; }
        int r = ew_batch(ctx, EW_SUB, A, &P, D, limbs);
        if (r != AFHE_OK) return r;
        for (uint32_t z = 0; z < m; ++z)
            if (a[s + z].c1_offset != d[s + z].c1_offset) {
                A2.push_back(a[s + z].c1_offset);
                D2.push_back(d[s + z].c1_offset);
            }
        return A2.empty() ? AFHE_OK : ew_batch(ctx, EW_COPY, A2, nullptr, D2, limbs);
    });
}

int afhe_ntt_batch(afhe_ctx* ctx, const uint64_t* polys, uint32_t count, uint32_t limbs, int inverse) {
    if (!ctx || (count && !polys)) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs_ext(ctx, limbs))) return rc;
    for (uint32_t i = 0; i < count; ++i)
        if ((rc = check_poly(ctx, polys[i], limbs))) return rc;
    for (uint32_t s = 0; s < count; s += 4096) {
        uint32_t m = count - s < 4096u ? count - s : 4096u;
        Offs v(polys + s, polys + s + m);
        ZBases zb{};
        ZF(zb.src, v);
        zb.mid = zb.src;
        zb.out = zb.src;
        CK(launch_ntt_plain(inverse != 0, ctx->log_n, ctx->nat.view(), ctx->jobs_qp, limbs, ctx->poly, ctx->poly, m,
                            zb, ctx->st));
    }
    return AFHE_OK;
}

uint64_t afhe_kernel_launches(void) { return launches_so_far(); }

int afhe_decrypt_batch(afhe_ctx* ctx, const afhe_ct_ref* cts, uint32_t count, uint64_t s_offset, uint64_t out_offset,
                       uint32_t limbs) {
    if (!ctx || (count && !cts)) return fail(ctx, AFHE_E_ARG, "null argument");
    int rc;
    if ((rc = check_limbs(ctx, limbs, 1)) || (rc = check_cts(ctx, cts, count, limbs)) ||
        (rc = check_poly(ctx, s_offset, limbs)))
        return rc;
    const u64 w = (u64)limbs * ctx->n;
    if (!range_ok(out_offset, (u64)count * w, ctx->prm.poly_words)) return fail(ctx, AFHE_E_RANGE, "output out of range");
    for (uint32_t s0 = 0; s0 < count; s0 += 4096) {
        uint32_t m = count - s0 < 4096u ? count - s0 : 4096u;
        Offs C1(m), C0(m);
        for (uint32_t z = 0; z < m; ++z) { C1[z] = cts[s0 + z].c1_offset; C0[z] = cts[s0 + z].c0_offset; }
        ZField f1, f0;
        ZF(f1, C1);
        ZF(f0, C0);
        const ZField O = zf_stride(out_offset + (u64)s0 * w, w);
        if ((rc = ew_fields(ctx, EW_MUL, f1, zf_const(s_offset), O, m, limbs)) != AFHE_OK) return rc;   // c1 * s
        if ((rc = ew_fields(ctx, EW_ADD, O, f0, O, m, limbs)) != AFHE_OK) return rc;                    // + c0
        ZBases zb{};
        zb.src = zb.mid = zb.out = O;
        CK(launch_ntt_plain(true, ctx->log_n, ctx->nat.view(), ctx->jobs_qp, limbs, ctx->poly, ctx->poly, m, zb,
                            ctx->st));
    }
    return AFHE_OK;
}

}  // extern "C"
