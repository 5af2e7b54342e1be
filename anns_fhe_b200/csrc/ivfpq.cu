// ivfpq.cu -- the encrypted IVF-PQ query chain's server stages in C++.
//
// The reference's InteractiveQueryManager (cpp_host_model/src/
// interactive_query_manager.cpp:85-303, semantics fixed by integration_tools/
// generate_interactive_test_vectors.cpp:383-541) runs one query's stages one
// ciphertext at a time through FHEHostDriver. This driver runs the same
// stages for many queries at once: every operator is one batched call over
// up to `lanes` ciphertexts (queries in stage 1, (query, list, batch) items in
// stage 3), and every ciphertext's residues are the ones the one-at-a-time
// chain produces:
//
//   stage 1   ct_diff = ct_query - pt_centroids; ct_sq = rescale(ct_diff^2);
//             tree sum with rotations 1, 2, .., D/2
//   stage 1b  reference compaction: for list i, mask slot i D, rescale,
//             rotate by i (D - 1) (eval_rotate's power-of-two steps), sum;
//             packed compaction (centroids over several ciphertexts): mask
//             every centroid slot of coarse ciphertext k, rescale, rotate by
//             -k in one key switch, sum
//   stage 3   per candidate batch: ct_dim - pt_batch, square, rescale, tree
//             sum with rotations B, 2B, .., B D/2 (packed, with the norms
//             registered: ||q||^2 - 2 ct_dim pt_batch, ||q||^2 squared once
//             per query, then + ||x_j||^2 after the tree sum), mask the batch's slots,
//             rescale, place it at its slot offset (eval_rotate's steps; when
//             packed, the mask itself is moved to the batch's row, since the
//             tree sum leaves the sums in every row), accumulate into the
//             query's result ciphertext
//   diagonal  (shape.packed = 2) stage 1: the query rotated by 1 .. n1 - 1
//             (baby steps, kept for stage 3), the centroids' inner products
//             by their diagonals (one
//             afhe_eval_diag_inner_batch per giant step group), rescale,
//             giant-step rotations by n1 g, sum, + ||q||^2 (the client's
//             ciphertext in ct_dim) + ||c||^2;
//             stage 3: the same per result ciphertext over the query's units,
//             each unit's diagonals placed at its slot offset (a multiple of
//             D) by an automorphism folded into the product's loads, then
//             + ||q||^2 + the placed unit norms
//
// Plaintexts, masks and working ciphertexts stay resident in poly_gmem at the
// offsets the caller registers (anns_fhe_b200/query.py encodes them). Modular
// additions are exact, so summing a query's terms pairwise gives the
// reference's running sum word for word.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <vector>

#include "internal.h"
#include "lanes.h"

using namespace afhe;

struct afhe_ivfpq {
    afhe_ctx* ctx = nullptr;
    afhe_ivfpq_shape sh{};
    std::vector<u64> centroid_cts;                      // [n_coarse]
    std::map<uint32_t, std::vector<u64>> masks;         // level -> one-hot [n_list] or stride [1]
    std::map<std::pair<uint32_t, uint32_t>, u64> prefix;   // (level, count) -> mask of the first count slots
    std::map<uint32_t, std::vector<u64>> norms;         // level -> candidates' squared norms per global batch
    std::vector<std::vector<std::pair<u64, uint32_t>>> lists;   // list -> (plaintext, candidates) per batch
    std::vector<afhe_ct_ref> work;                      // diff, sq, sel per lane
    std::vector<afhe_ct_ref> cmp;                       // (n_list - 1) per lane: reference compaction terms
    std::map<uint32_t, afhe_ks_options> tuning;        // level -> key-switch options
    bool fused_ok = false;                              // the one-kernel key switch was on at creation
    // diagonal chain
    struct Diag {
        u64 cent = 0, cnorm = 0;                        // centroids' first diagonal, their norms
        std::vector<u64> unit_pts, unit_norms;          // per unit: first diagonal, norms
    };
    std::map<uint32_t, Diag> diag;                      // level -> plaintexts
    std::vector<uint32_t> list_first_unit;              // [n_list + 1]
    std::vector<uint32_t> unit_count;                   // candidates per unit
    std::vector<afhe_ct_ref> scratch;                   // inner-product ciphertexts
};

namespace {

typedef std::vector<afhe_ct_ref> Cts;

int fail_h(afhe_ivfpq* h, int code, const char* msg) { return fail(h ? h->ctx : nullptr, code, msg); }

uint32_t n_coarse(const afhe_ivfpq_shape& s) {
    if (s.packed == 2) return 1;
    const uint32_t per = s.slots / s.D;
    return (s.n_list + per - 1) / per;
}

bool diagonal(const afhe_ivfpq* h) { return h->sh.packed == 2; }

// Baby steps of the diagonal method: 2^ceil(log2(D) / 2); giant steps D / n1.
uint32_t baby_steps(uint32_t D) {
    uint32_t lg = 0;
    while ((1u << lg) < D) ++lg;
    return 1u << ((lg + 1) / 2);
}

uint32_t eval_at(const afhe_ivfpq* h, uint32_t level) {
    const uint32_t lv = level ? level : h->ctx->L;
    return h->sh.eval_level ? std::min(lv, h->sh.eval_level) : lv;
}

// The tuned options of the level an operator runs at (query.py _at).
void at(afhe_ivfpq* h, uint32_t limbs) {
    auto it = h->tuning.find(limbs);
    if (it == h->tuning.end()) return;
    const afhe_ks_options& o = it->second;
    if (o.fused == 0 || (o.fused > 0 && h->fused_ok)) afhe_ctx_set_option(h->ctx, AFHE_OPT_KS_FUSED, o.fused);
    if (o.chunk) afhe_ctx_set_option(h->ctx, AFHE_OPT_CHUNK, std::min<uint32_t>(o.chunk, h->ctx->lanes));
    if (o.ept) afhe_ctx_set_option(h->ctx, AFHE_OPT_KS_EPT, o.ept);
    if (o.slice) afhe_ctx_set_option(h->ctx, AFHE_OPT_KS_SLICE, o.slice);
    if (o.fused_min) afhe_ctx_set_option(h->ctx, AFHE_OPT_FUSED_MIN, o.fused_min);
}

#define RC(expr)                              \
    do {                                      \
        int _rc = (expr);                     \
        if (_rc != AFHE_OK) return _rc;       \
    } while (0)

int add(afhe_ivfpq* h, const Cts& a, const Cts& b, const Cts& d, uint32_t limbs) {
    return a.empty() ? AFHE_OK : afhe_eval_add_batch(h->ctx, a.data(), b.data(), d.data(), (uint32_t)a.size(), limbs);
}

int copy(afhe_ivfpq* h, const Cts& a, const Cts& d, uint32_t limbs) {
    return a.empty() ? AFHE_OK : afhe_eval_copy_batch(h->ctx, a.data(), d.data(), (uint32_t)a.size(), limbs);
}

int rot_acc(afhe_ivfpq* h, const Cts& src, const Cts& acc, int32_t r, uint32_t limbs) {
    at(h, limbs);
    return afhe_eval_rotate_accumulate_batch(h->ctx, src.data(), acc.data(), (uint32_t)src.size(), r, limbs);
}

int square(afhe_ivfpq* h, const Cts& a, const Cts& d, uint32_t limbs) {
    at(h, limbs);
    return afhe_eval_mult_relin_rescale_batch(h->ctx, a.data(), a.data(), d.data(), (uint32_t)a.size(), limbs);
}

// dst = rescale(a * pt) per entry
int mult_plain(afhe_ivfpq* h, const Cts& a, const std::vector<u64>& pts, const Cts& d, uint32_t limbs) {
    return afhe_eval_mult_plain_rescale_batch(h->ctx, a.data(), pts.data(), d.data(), (uint32_t)a.size(), limbs);
}

// Each (ct, step) rotated in place by its step in one key switch.
int rotate_direct(afhe_ivfpq* h, const std::vector<std::pair<afhe_ct_ref, int32_t>>& items, uint32_t limbs) {
    Cts cts;
    std::vector<int32_t> steps;
    for (auto& it : items)
        if (it.second) {
            cts.push_back(it.first);
            steps.push_back(it.second);
        }
    if (cts.empty()) return AFHE_OK;
    at(h, limbs);
    return afhe_eval_rotate_steps_batch(h->ctx, cts.data(), cts.data(), steps.data(), (uint32_t)cts.size(), limbs);
}

// Each (ct, shift) rotated in place as eval_rotate does it (fhe_host_driver.cpp:
// 361-404): |shift| in descending powers of two, sign kept; one batched call
// per (power, sign) over the items whose shift has that bit.
int rotate_grouped(afhe_ivfpq* h, const std::vector<std::pair<afhe_ct_ref, int32_t>>& items, uint32_t limbs) {
    uint32_t top = 0;
    for (auto& it : items) top = std::max<uint32_t>(top, (uint32_t)std::abs(it.second));
    if (!top) return AFHE_OK;
    int b = 31;
    while (!((top >> b) & 1u)) --b;
    for (; b >= 0; --b)
        for (int sign : {1, -1}) {
            Cts sel;
            for (auto& it : items) {
                const int32_t s = it.second;
                if (s && ((s > 0) == (sign > 0)) && ((((uint32_t)std::abs(s)) >> b) & 1u)) sel.push_back(it.first);
            }
            if (sel.empty()) continue;
            at(h, limbs);
            RC(afhe_eval_rotate_batch(h->ctx, sel.data(), sel.data(), (uint32_t)sel.size(), sign * (1 << b), limbs));
        }
    return AFHE_OK;
}

// groups[g][0] += groups[g][1] + ... by pairwise batched additions.
int sum_groups(afhe_ivfpq* h, std::vector<Cts> live, uint32_t limbs) {
    for (;;) {
        Cts a, b;
        for (auto& g : live)
            for (size_t j = 0; j + 1 < g.size(); j += 2) {
                a.push_back(g[j]);
                b.push_back(g[j + 1]);
            }
        if (a.empty()) return AFHE_OK;
        RC(add(h, a, b, a, limbs));
        for (auto& g : live) {
            Cts k;
            for (size_t j = 0; j < g.size(); j += 2) k.push_back(g[j]);
            g.swap(k);
        }
    }
}

bool same(const afhe_ct_ref& a, const afhe_ct_ref& b) { return a.c0_offset == b.c0_offset && a.c1_offset == b.c1_offset; }

// items (target, first, src): per target its sources summed pairwise, then
// copied into the target when one of them starts the target's sum, else added.
int accumulate(afhe_ivfpq* h, const std::vector<std::pair<std::pair<afhe_ct_ref, bool>, afhe_ct_ref>>& items,
               uint32_t limbs) {
    std::vector<afhe_ct_ref> targets;
    std::vector<bool> first;
    std::vector<Cts> groups;
    for (auto& it : items) {
        size_t g = 0;
        while (g < targets.size() && !same(targets[g], it.first.first)) ++g;
        if (g == targets.size()) {
            targets.push_back(it.first.first);
            first.push_back(false);
            groups.emplace_back();
        }
        first[g] = first[g] || it.first.second;
        groups[g].push_back(it.second);
    }
    RC(sum_groups(h, groups, limbs));
    Cts cs, ct, as, at_;
    for (size_t g = 0; g < targets.size(); ++g) {
        if (first[g]) { cs.push_back(groups[g][0]); ct.push_back(targets[g]); }
        else { as.push_back(groups[g][0]); at_.push_back(targets[g]); }
    }
    RC(copy(h, cs, ct, limbs));
    return add(h, at_, as, at_, limbs);
}

int sub_plain(afhe_ivfpq* h, const Cts& a, const std::vector<u64>& pts, const Cts& d, uint32_t limbs) {
    return afhe_eval_sub_plain_batch(h->ctx, a.data(), pts.data(), d.data(), (uint32_t)a.size(), limbs);
}

// queries by the level they run at, highest first (query.py _by_level)
std::vector<std::pair<uint32_t, std::vector<uint32_t>>> by_level(afhe_ivfpq* h, const afhe_ivfpq_query* q,
                                                                  uint32_t count) {
    std::map<uint32_t, std::vector<uint32_t>> g;
    for (uint32_t i = 0; i < count; ++i) g[eval_at(h, q[i].level)].push_back(i);
    return std::vector<std::pair<uint32_t, std::vector<uint32_t>>>(g.rbegin(), g.rend());
}

int stage1_packed(afhe_ivfpq* h, const afhe_ivfpq_query* q, const std::vector<uint32_t>& idx, uint32_t Ll) {
    const uint32_t D = h->sh.D, nc = n_coarse(h->sh), lanes = h->sh.lanes;
    std::vector<std::pair<uint32_t, uint32_t>> items;
    for (uint32_t qi : idx)
        for (uint32_t k = 0; k < nc; ++k) items.push_back({qi, k});
    for (size_t c0 = 0; c0 < items.size(); c0 += lanes) {
        const size_t m = std::min<size_t>(lanes, items.size() - c0);
        Cts diff(m), sq(m), sel(m), in(m);
        std::vector<u64> pts(m), stride(m, h->masks[Ll][0]);
        for (size_t j = 0; j < m; ++j) {
            diff[j] = h->work[4 * j];
            sq[j] = h->work[4 * j + 1];
            sel[j] = h->work[4 * j + 2];
            in[j] = q[items[c0 + j].first].ct_query;
            pts[j] = h->centroid_cts[items[c0 + j].second];
        }
        RC(sub_plain(h, in, pts, diff, Ll));
        RC(square(h, diff, sq, Ll));
        for (uint32_t s = 1; s < D; s <<= 1) RC(rot_acc(h, sq, sq, (int32_t)s, Ll - 1));
        RC(mult_plain(h, sq, stride, sel, Ll - 1));
        std::vector<std::pair<afhe_ct_ref, int32_t>> rot;
        std::vector<std::pair<std::pair<afhe_ct_ref, bool>, afhe_ct_ref>> acc;
        for (size_t j = 0; j < m; ++j) {
            const uint32_t k = items[c0 + j].second;
            rot.push_back({sel[j], -(int32_t)k});
            acc.push_back({{q[items[c0 + j].first].compact, k == 0}, sel[j]});
        }
        RC(rotate_direct(h, rot, Ll - 2));
        RC(accumulate(h, acc, Ll - 2));
    }
    return AFHE_OK;
}

int stage1_reference(afhe_ivfpq* h, const afhe_ivfpq_query* q, const std::vector<uint32_t>& idx, uint32_t Ll) {
    const uint32_t D = h->sh.D, nl = h->sh.n_list, lanes = h->sh.lanes;
    const std::vector<u64>& onehot = h->masks[Ll];
    for (size_t c0 = 0; c0 < idx.size(); c0 += lanes) {
        const size_t m = std::min<size_t>(lanes, idx.size() - c0);
        Cts diff(m), sq(m), in(m);
        std::vector<u64> pts(m, h->centroid_cts[0]);
        for (size_t j = 0; j < m; ++j) {
            diff[j] = h->work[4 * j];
            sq[j] = h->work[4 * j + 1];
            in[j] = q[idx[c0 + j]].ct_query;
        }
        RC(sub_plain(h, in, pts, diff, Ll));
        RC(square(h, diff, sq, Ll));
        for (uint32_t s = 1; s < D; s <<= 1) RC(rot_acc(h, sq, sq, (int32_t)s, Ll - 1));
        // stage 1b: every (query, list) term masked in one batched operator,
        // rotated step by step across the terms, summed pairwise
        Cts src, dst;
        std::vector<u64> masks;
        for (size_t k = 0; k < m; ++k)
            for (uint32_t i = 0; i < nl; ++i) {
                src.push_back(sq[k]);
                masks.push_back(onehot[i]);
                dst.push_back(i == 0 ? q[idx[c0 + k]].compact : h->cmp[k * (nl - 1) + i - 1]);
            }
        RC(mult_plain(h, src, masks, dst, Ll - 1));
        if (nl == 1) continue;
        std::vector<std::pair<afhe_ct_ref, int32_t>> rot;
        std::vector<Cts> groups;
        for (size_t k = 0; k < m; ++k) {
            Cts g{q[idx[c0 + k]].compact};
            for (uint32_t i = 1; i < nl; ++i) {
                rot.push_back({h->cmp[k * (nl - 1) + i - 1], (int32_t)(i * (D - 1))});
                g.push_back(h->cmp[k * (nl - 1) + i - 1]);
            }
            groups.push_back(g);
        }
        RC(rotate_grouped(h, rot, Ll - 2));
        RC(sum_groups(h, groups, Ll - 2));
    }
    return AFHE_OK;
}

struct Item {
    uint32_t qi;
    u64 pt;
    uint32_t cnt;
    u64 off;
    uint32_t gb;      // global batch number (lists in order, then batches)
};

int sub(afhe_ivfpq* h, const Cts& a, const Cts& b, const Cts& d, uint32_t limbs) {
    return a.empty() ? AFHE_OK : afhe_eval_sub_batch(h->ctx, a.data(), b.data(), d.data(), (uint32_t)a.size(), limbs);
}

int add_plain(afhe_ivfpq* h, const Cts& a, const std::vector<u64>& pts, const Cts& d, uint32_t limbs) {
    return afhe_eval_add_plain_batch(h->ctx, a.data(), pts.data(), d.data(), (uint32_t)a.size(), limbs);
}

int stage3_items(afhe_ivfpq* h, const afhe_ivfpq_query* q, const std::vector<Item>& items, uint32_t Ll) {
    const uint32_t D = h->sh.D, S = h->sh.slots, B = S / D, lanes = h->sh.lanes;
    // Expanded distances (packed chain, with the candidates' norms registered
    // for this level): ||q - x_j||^2 = ||q||^2 - 2 <q, x_j> + ||x_j||^2, the
    // query's ||q||^2 squared once per query instead of a square per batch.
    auto nit = h->norms.find(Ll);
    const bool expand = h->sh.packed && nit != h->norms.end();
    if (expand) {
        Cts qin, qnorm;
        std::vector<bool> seen;
        for (const Item& it : items) {
            if (it.qi >= seen.size()) seen.resize(it.qi + 1, false);
            if (seen[it.qi]) continue;
            seen[it.qi] = true;
            qin.push_back(q[it.qi].ct_dim);
            qnorm.push_back(q[it.qi].norm);
        }
        for (size_t c0 = 0; c0 < qin.size(); c0 += lanes) {
            const size_t m = std::min<size_t>(lanes, qin.size() - c0);
            RC(square(h, Cts(qin.begin() + c0, qin.begin() + c0 + m), Cts(qnorm.begin() + c0, qnorm.begin() + c0 + m),
                      Ll));
        }
    }
    for (size_t c0 = 0; c0 < items.size(); c0 += lanes) {
        const size_t m = std::min<size_t>(lanes, items.size() - c0);
        Cts diff(m), sq(m), sel(m), in(m);
        std::vector<u64> pts(m), prefix(m);
        for (size_t j = 0; j < m; ++j) {
            const Item& it = items[c0 + j];
            diff[j] = h->work[4 * j];
            sq[j] = h->work[4 * j + 1];
            sel[j] = h->work[4 * j + 2];
            in[j] = q[it.qi].ct_dim;
            pts[j] = it.pt;
            auto pm = h->prefix.find({Ll, it.cnt});
            if (pm == h->prefix.end()) return fail_h(h, AFHE_E_STATE, "no prefix mask for a candidate count at this level");
            prefix[j] = pm->second;
        }
        if (expand) {
            Cts qn(m);
            std::vector<u64> nx(m);
            for (size_t j = 0; j < m; ++j) {
                qn[j] = q[items[c0 + j].qi].norm;
                if (items[c0 + j].gb >= nit->second.size())
                    return fail_h(h, AFHE_E_STATE, "no norm plaintext for a candidate batch at this level");
                nx[j] = nit->second[items[c0 + j].gb];
            }
            RC(mult_plain(h, in, pts, diff, Ll));          // <q, x_j> per row (one rescale)
            RC(sub(h, qn, diff, sq, Ll - 1));              // ||q||^2 - <q, x_j>
            RC(sub(h, sq, diff, sq, Ll - 1));              //          - <q, x_j>
            for (uint32_t s = B; s < D * B; s <<= 1) RC(rot_acc(h, sq, sq, (int32_t)s, Ll - 1));
            RC(add_plain(h, sq, nx, sq, Ll - 1));          // + ||x_j||^2, in every row
        } else {
            RC(sub_plain(h, in, pts, diff, Ll));
            RC(square(h, diff, sq, Ll));
            for (uint32_t s = B; s < D * B; s <<= 1) RC(rot_acc(h, sq, sq, (int32_t)s, Ll - 1));
        }
        std::vector<std::pair<std::pair<afhe_ct_ref, bool>, afhe_ct_ref>> acc;
        for (size_t j = 0; j < m; ++j) {
            const Item& it = items[c0 + j];
            acc.push_back({{q[it.qi].results[it.off / S], it.off % S == 0}, sel[j]});
        }
        if (h->sh.packed) {
            // The tree sum runs over all D rows of B slots, so every row holds
            // the batch's sums. The prefix mask moved to row t = offset / B
            // (an automorphism of the plaintext: no key switch) both selects
            // and places them.
            std::vector<u64> masks(m);
            std::vector<uint32_t> gal(m);
            for (size_t j = 0; j < m; ++j) {
                masks[j] = h->work[4 * j + 3].c0_offset;
                gal[j] = afhe_galois_elt(h->ctx->log_n, -(int32_t)(items[c0 + j].off % S));
            }
            RC(afhe_automorphism_batch(h->ctx, prefix.data(), gal.data(), masks.data(), (uint32_t)m, Ll - 1));
            RC(mult_plain(h, sq, masks, sel, Ll - 1));
        } else {
            RC(mult_plain(h, sq, prefix, sel, Ll - 1));
            std::vector<std::pair<afhe_ct_ref, int32_t>> place;
            for (size_t j = 0; j < m; ++j) place.push_back({sel[j], -(int32_t)(items[c0 + j].off % S)});
            RC(rotate_grouped(h, place, Ll - 2));
        }
        RC(accumulate(h, acc, Ll - 2));
    }
    return AFHE_OK;
}

// ---- the diagonal chain ----------------------------------------------------
// One output of the inner products: its baby-step sources (n1 ciphertexts)
// and its placed units (first diagonal of the unit at giant step 0, galois).
struct InnerOut {
    const afhe_ct_ref* query;              // the query (baby step 0)
    const afhe_ct_ref* baby;               // baby steps 1 .. n1 - 1
    std::vector<std::pair<u64, uint32_t>> units;
};

// For each output k: giant step g's inner product into scr[k n2 + g] (Ll
// limbs), the sum over its units and b < n1 of diagonal g n1 + b (unit base +
// (g n1 + b) Ll N) moved by the unit's automorphism, times baby step b; then
// rescaled, giant step g rotated by n1 g, summed into scr[k n2] (Ll - 1 limbs).
int giant(afhe_ivfpq* h, const std::vector<InnerOut>& outs, const Cts& scr, uint32_t Ll) {
    const uint32_t n1 = baby_steps(h->sh.D), n2 = h->sh.D / n1;
    const u64 stride = (u64)Ll * h->ctx->n;
    const uint32_t count = (uint32_t)outs.size() * n2;
    Cts inner(scr.begin(), scr.begin() + count), src;
    std::vector<u64> upt;
    std::vector<uint32_t> ugal, first{0};
    for (const auto& o : outs)
        for (uint32_t g = 0; g < n2; ++g) {
            src.push_back(*o.query);
            for (uint32_t b = 1; b < n1; ++b) src.push_back(o.baby[b - 1]);
            for (const auto& u : o.units) {
                upt.push_back(u.first + (u64)g * n1 * stride);
                ugal.push_back(u.second);
            }
            first.push_back((uint32_t)upt.size());
        }
    if (n1 <= 16) {
        RC(afhe_eval_diag_inner_batch(h->ctx, inner.data(), count, src.data(), n1, upt.data(), ugal.data(),
                                      first.data(), stride, Ll, 0));
    } else {                                          // the generic form: one group per baby step
        std::vector<afhe_mac_group> G;
        std::vector<afhe_mac_term> T;
        std::vector<uint32_t> fg{0};
        for (uint32_t j = 0; j < count; ++j) {
            for (uint32_t b = 0; b < n1; ++b) {
                G.push_back(afhe_mac_group{src[(size_t)j * n1 + b], (uint32_t)T.size(), first[j + 1] - first[j]});
                for (uint32_t k = first[j]; k < first[j + 1]; ++k) T.push_back(afhe_mac_term{upt[k] + b * stride, ugal[k], 0});
            }
            fg.push_back((uint32_t)G.size());
        }
        RC(afhe_eval_mac_plain_batch(h->ctx, inner.data(), fg.data(), count, G.data(), T.data(), Ll, 0));
    }
    RC(afhe_rescale_batch(h->ctx, inner.data(), inner.data(), count, Ll));
    std::vector<std::pair<afhe_ct_ref, int32_t>> rot;
    std::vector<Cts> groups;
    for (size_t k = 0; k < outs.size(); ++k) {
        groups.push_back(Cts(inner.begin() + k * n2, inner.begin() + (k + 1) * n2));
        for (uint32_t g = 1; g < n2; ++g) rot.push_back({inner[k * n2 + g], (int32_t)(n1 * g)});
    }
    RC(rotate_direct(h, rot, Ll - 1));
    return sum_groups(h, groups, Ll - 1);
}

int stage1_diagonal(afhe_ivfpq* h, const afhe_ivfpq_query* q, const std::vector<uint32_t>& idx, uint32_t Ll) {
    const uint32_t D = h->sh.D, n1 = baby_steps(D), n2 = D / n1;
    const afhe_ivfpq::Diag& dg = h->diag.at(Ll);
    Cts src, dst;
    std::vector<int32_t> steps;
    for (uint32_t i : idx)
        for (uint32_t b = 1; b < n1; ++b) {
            src.push_back(q[i].ct_query);
            dst.push_back(q[i].baby[b - 1]);
            steps.push_back((int32_t)b);
        }
    if (!src.empty()) {
        at(h, Ll);
        RC(afhe_eval_rotate_steps_batch(h->ctx, src.data(), dst.data(), steps.data(), (uint32_t)src.size(), Ll));
    }
    const size_t per = h->scratch.size() / n2;
    for (size_t c0 = 0; c0 < idx.size(); c0 += per) {
        const size_t m = std::min(per, idx.size() - c0);
        std::vector<InnerOut> outs;
        Cts heads, norms, comp;
        for (size_t k = 0; k < m; ++k) {
            const afhe_ivfpq_query& x = q[idx[c0 + k]];
            outs.push_back(InnerOut{&x.ct_query, x.baby, {{dg.cent, 1u}}});
            heads.push_back(h->scratch[k * n2]);
            norms.push_back(x.ct_dim);                    // ||q||^2, the client's
            comp.push_back(x.compact);
        }
        RC(giant(h, outs, h->scratch, Ll));
        RC(add(h, heads, norms, comp, Ll - 1));
        RC(add_plain(h, comp, std::vector<u64>(m, dg.cnorm), comp, Ll - 1));
    }
    return AFHE_OK;
}

// The slot offsets of a query's units (probe order): spans of count rounded
// up to a multiple of D, back to back, a unit that would cross a result's end
// starting the next result. Returns false on a list out of range.
bool unit_layout(const afhe_ivfpq* h, const afhe_ivfpq_query& q, std::vector<std::pair<uint32_t, u64>>& out) {
    const u64 S = h->sh.slots, D = h->sh.D;
    u64 off = 0;
    out.clear();
    for (uint32_t p = 0; p < q.nprobe; ++p) {
        const uint32_t c = q.probes[p];
        if (c >= h->sh.n_list) return false;
        for (uint32_t u = h->list_first_unit[c]; u < h->list_first_unit[c + 1]; ++u) {
            const u64 span = (h->unit_count[u] + D - 1) / D * D;
            if (off % S + span > S) off = (off / S + 1) * S;
            out.push_back({u, off});
            off += span;
        }
    }
    return true;
}

int stage3_diagonal(afhe_ivfpq* h, const afhe_ivfpq_query* q, const std::vector<uint32_t>& idx, uint32_t Ll) {
    const uint32_t D = h->sh.D, n1 = baby_steps(D), n2 = D / n1;
    const u64 S = h->sh.slots;
    const afhe_ivfpq::Diag& dg = h->diag.at(Ll);
    struct It {
        uint32_t qi, r;
        std::vector<std::pair<uint32_t, uint32_t>> units;     // (unit, galois)
    };
    std::vector<It> items;
    std::vector<std::pair<uint32_t, u64>> lay;
    for (uint32_t i : idx) {
        unit_layout(h, q[i], lay);
        const uint32_t used = lay.empty() ? 1u : (uint32_t)(lay.back().second / S) + 1;
        for (uint32_t r = 0; r < used; ++r) {
            It it{i, r, {}};
            for (const auto& u : lay)
                if (u.second / S == r)
                    it.units.push_back({u.first, afhe_galois_elt((uint32_t)h->ctx->log_n, -(int32_t)(u.second % S))});
            items.push_back(std::move(it));
        }
    }
    const size_t per = h->scratch.size() / n2;
    for (size_t c0 = 0; c0 < items.size(); c0 += per) {
        const size_t m = std::min(per, items.size() - c0);
        std::vector<InnerOut> outs;
        Cts heads, norms, res;
        std::vector<afhe_mac_group> G;
        std::vector<afhe_mac_term> T;
        std::vector<uint32_t> fg{0};
        for (size_t k = 0; k < m; ++k) {
            const It& it = items[c0 + k];
            const afhe_ivfpq_query& x = q[it.qi];
            InnerOut o{&x.ct_query, x.baby, {}};
            G.push_back(afhe_mac_group{afhe_ct_ref{AFHE_MAC_UNIT, 0}, (uint32_t)T.size(), (uint32_t)it.units.size()});
            for (const auto& u : it.units) {
                o.units.push_back({dg.unit_pts[u.first], u.second});
                T.push_back(afhe_mac_term{dg.unit_norms[u.first], u.second, 0});
            }
            fg.push_back((uint32_t)G.size());
            outs.push_back(std::move(o));
            heads.push_back(h->scratch[k * n2]);
            norms.push_back(x.ct_dim);
            res.push_back(x.results[it.r]);
        }
        RC(giant(h, outs, h->scratch, Ll));
        RC(add(h, heads, norms, res, Ll - 1));            // + ||q||^2, then + the placed unit norms
        RC(afhe_eval_mac_plain_batch(h->ctx, res.data(), fg.data(), (uint32_t)m, G.data(), T.data(), Ll - 1, 1));
    }
    return AFHE_OK;
}

int check_query(afhe_ivfpq* h, const afhe_ivfpq_query& q) {
    if (diagonal(h)) {
        if (q.level > h->ctx->L || (q.level && q.level < 2)) return fail_h(h, AFHE_E_LEVEL, "query level outside [2, L]");
        if (!h->diag.count(eval_at(h, q.level))) return fail_h(h, AFHE_E_STATE, "no diagonals for the query's level");
        if (q.n_baby != baby_steps(h->sh.D) - 1 || (q.n_baby && !q.baby))
            return fail_h(h, AFHE_E_ARG, "a query needs n1 - 1 baby-step ciphertexts");
        return AFHE_OK;
    }
    if (q.level > h->ctx->L || (q.level && q.level < 3)) return fail_h(h, AFHE_E_LEVEL, "query level outside [3, L]");
    if (!h->masks.count(eval_at(h, q.level))) return fail_h(h, AFHE_E_STATE, "no masks for the query's level");
    return AFHE_OK;
}

}  // namespace

extern "C" {

int afhe_ivfpq_create(afhe_ctx* ctx, const afhe_ivfpq_shape* shape, afhe_ivfpq** out) {
    if (!ctx || !shape || !out) return fail(ctx, AFHE_E_ARG, "null argument");
    const afhe_ivfpq_shape& s = *shape;
    if (s.D < 2 || (s.D & (s.D - 1)) || s.slots != ctx->n / 2 || s.D > s.slots || s.n_list < 1 || s.lanes < 1 ||
        s.lanes > ctx->lanes)
        return fail(ctx, AFHE_E_ARG, "ivfpq shape: D a power of two <= N/2, slots = N/2, lanes in [1, context lanes]");
    if (s.packed > 2) return fail(ctx, AFHE_E_ARG, "compaction: 0 reference, 1 packed, 2 diagonal");
    if (s.packed == 0 && s.n_list * s.D > s.slots) return fail(ctx, AFHE_E_ARG, "centroids do not fit one ciphertext");
    if (s.packed == 1 && n_coarse(s) > s.D) return fail(ctx, AFHE_E_ARG, "packed compaction needs n_coarse <= D");
    if (s.packed == 2 && s.n_list > s.slots) return fail(ctx, AFHE_E_ARG, "the diagonal chain needs n_list <= N/2");
    const uint32_t min_level = s.packed == 2 ? 2 : 3;     // the chain's depth + 1
    if (s.eval_level && (s.eval_level < min_level || s.eval_level > ctx->L))
        return fail(ctx, AFHE_E_LEVEL, "eval_level in [depth + 1, L]");
    afhe_ivfpq* h = new afhe_ivfpq();
    h->ctx = ctx;
    h->sh = s;
    h->lists.resize(s.n_list);
    int64_t v = 0;
    h->fused_ok = afhe_ctx_get_option(ctx, AFHE_OPT_KS_FUSED, &v) == AFHE_OK && v == 1;
    *out = h;
    return AFHE_OK;
}

int afhe_ivfpq_destroy(afhe_ivfpq* h) {
    delete h;
    return AFHE_OK;
}

int afhe_ivfpq_set_centroids(afhe_ivfpq* h, const uint64_t* pts, uint32_t count) {
    if (!h || !pts) return fail_h(h, AFHE_E_ARG, "null argument");
    if (count != n_coarse(h->sh)) return fail_h(h, AFHE_E_ARG, "one centroid plaintext per coarse ciphertext");
    h->centroid_cts.assign(pts, pts + count);
    return AFHE_OK;
}

int afhe_ivfpq_set_level_masks(afhe_ivfpq* h, uint32_t level, const uint64_t* masks, uint32_t count) {
    if (!h || !masks) return fail_h(h, AFHE_E_ARG, "null argument");
    if (count != (h->sh.packed ? 1u : h->sh.n_list)) return fail_h(h, AFHE_E_ARG, "n_list one-hot masks, or one stride mask");
    h->masks[level].assign(masks, masks + count);
    return AFHE_OK;
}

int afhe_ivfpq_set_prefix_mask(afhe_ivfpq* h, uint32_t level, uint32_t count, uint64_t pt) {
    if (!h) return fail_h(h, AFHE_E_ARG, "null argument");
    h->prefix[{level, count}] = pt;
    return AFHE_OK;
}

int afhe_ivfpq_set_list(afhe_ivfpq* h, uint32_t list, const uint64_t* pts, const uint32_t* counts, uint32_t batches) {
    if (!h || (batches && (!pts || !counts))) return fail_h(h, AFHE_E_ARG, "null argument");
    if (list >= h->sh.n_list) return fail_h(h, AFHE_E_RANGE, "list out of range");
    auto& v = h->lists[list];
    v.clear();
    for (uint32_t b = 0; b < batches; ++b) {
        if (counts[b] < 1 || counts[b] > h->sh.slots / h->sh.D) return fail_h(h, AFHE_E_ARG, "batch count outside [1, B]");
        v.push_back({pts[b], counts[b]});
    }
    return AFHE_OK;
}

int afhe_ivfpq_set_lanes(afhe_ivfpq* h, const afhe_ct_ref* work, uint32_t lanes, const afhe_ct_ref* cmp) {
    if (!h || !work) return fail_h(h, AFHE_E_ARG, "null argument");
    if (lanes < h->sh.lanes) return fail_h(h, AFHE_E_ARG, "a diff / sq / sel / mask quadruple for every lane");
    h->work.assign(work, work + 4 * (size_t)lanes);
    if (!h->sh.packed && h->sh.n_list > 1) {
        if (!cmp) return fail_h(h, AFHE_E_ARG, "the reference compaction needs n_list - 1 term ciphertexts per lane");
        h->cmp.assign(cmp, cmp + (size_t)lanes * (h->sh.n_list - 1));
    }
    return AFHE_OK;
}

int afhe_ivfpq_set_norms(afhe_ivfpq* h, uint32_t level, const uint64_t* pts, uint32_t batches) {
    if (!h || (batches && !pts)) return fail_h(h, AFHE_E_ARG, "null argument");
    if (!h->sh.packed) return fail_h(h, AFHE_E_STATE, "expanded distances are for the packed chain");
    h->norms[level].assign(pts, pts + batches);
    return AFHE_OK;
}

int afhe_ivfpq_set_tuning(afhe_ivfpq* h, uint32_t level, const afhe_ks_options* o) {
    if (!h || !o) return fail_h(h, AFHE_E_ARG, "null argument");
    if (o->ept && o->ept != 8 && o->ept != 16) return fail_h(h, AFHE_E_ARG, "values per thread must be 8 or 16");
    if (o->slice && o->slice != 12 && o->slice != 13) return fail_h(h, AFHE_E_ARG, "the slice must be 2^12 or 2^13 values");
    if (o->fused_min > 4096) return fail_h(h, AFHE_E_ARG, "fused minimum must be in [1, 4096]");
    h->tuning[level] = *o;
    return AFHE_OK;
}

int afhe_ivfpq_set_units(afhe_ivfpq* h, const uint32_t* list_first_unit, const uint32_t* counts, uint32_t units) {
    if (!h || !list_first_unit || (units && !counts)) return fail_h(h, AFHE_E_ARG, "null argument");
    if (!diagonal(h)) return fail_h(h, AFHE_E_STATE, "units are for the diagonal chain");
    if (list_first_unit[0] != 0 || list_first_unit[h->sh.n_list] != units)
        return fail_h(h, AFHE_E_ARG, "list_first_unit must run from 0 to units");
    for (uint32_t c = 0; c < h->sh.n_list; ++c)
        if (list_first_unit[c + 1] < list_first_unit[c]) return fail_h(h, AFHE_E_ARG, "unit ranges must not decrease");
    for (uint32_t u = 0; u < units; ++u)
        if (counts[u] < 1 || counts[u] > h->sh.slots) return fail_h(h, AFHE_E_ARG, "unit count outside [1, N/2]");
    h->list_first_unit.assign(list_first_unit, list_first_unit + h->sh.n_list + 1);
    h->unit_count.assign(counts, counts + units);
    return AFHE_OK;
}

int afhe_ivfpq_set_diagonals(afhe_ivfpq* h, uint32_t level, uint64_t centroids, uint64_t centroid_norms,
                             const uint64_t* unit_pts, const uint64_t* unit_norms, uint32_t units) {
    if (!h || (units && (!unit_pts || !unit_norms))) return fail_h(h, AFHE_E_ARG, "null argument");
    if (!diagonal(h)) return fail_h(h, AFHE_E_STATE, "diagonals are for the diagonal chain");
    if (level < 2 || level > h->ctx->L) return fail_h(h, AFHE_E_LEVEL, "level in [2, L]");
    if (units != h->unit_count.size()) return fail_h(h, AFHE_E_ARG, "one set of diagonals per unit (set the units first)");
    const u64 w = (u64)level * h->ctx->n, span = (u64)h->sh.D * w;
    if (!range_ok(centroids, span, h->ctx->prm.poly_words) ||
        !range_ok(centroid_norms, (u64)(level - 1) * h->ctx->n, h->ctx->prm.poly_words))
        return fail_h(h, AFHE_E_RANGE, "centroid plaintexts out of poly_gmem");
    for (uint32_t u = 0; u < units; ++u)
        if (!range_ok(unit_pts[u], span, h->ctx->prm.poly_words) ||
            !range_ok(unit_norms[u], (u64)(level - 1) * h->ctx->n, h->ctx->prm.poly_words))
            return fail_h(h, AFHE_E_RANGE, "unit plaintexts out of poly_gmem");
    afhe_ivfpq::Diag& d = h->diag[level];
    d.cent = centroids;
    d.cnorm = centroid_norms;
    d.unit_pts.assign(unit_pts, unit_pts + units);
    d.unit_norms.assign(unit_norms, unit_norms + units);
    return AFHE_OK;
}

int afhe_ivfpq_set_scratch(afhe_ivfpq* h, const afhe_ct_ref* cts, uint32_t count) {
    if (!h || (count && !cts)) return fail_h(h, AFHE_E_ARG, "null argument");
    const uint32_t n2 = h->sh.D / baby_steps(h->sh.D);
    if (count < n2) return fail_h(h, AFHE_E_ARG, "at least D / n1 working ciphertexts");
    h->scratch.assign(cts, cts + count / n2 * n2);
    return AFHE_OK;
}

int afhe_ivfpq_stage1(afhe_ivfpq* h, const afhe_ivfpq_query* q, uint32_t count) {
    if (!h || (count && !q)) return fail_h(h, AFHE_E_ARG, "null argument");
    if (diagonal(h)) {
        if (h->scratch.empty()) return fail_h(h, AFHE_E_STATE, "scratch not set");
        for (uint32_t i = 0; i < count; ++i) RC(check_query(h, q[i]));
        for (auto& g : by_level(h, q, count)) RC(stage1_diagonal(h, q, g.second, g.first));
        return AFHE_OK;
    }
    if (h->work.empty() || h->centroid_cts.empty()) return fail_h(h, AFHE_E_STATE, "lanes and centroids not set");
    for (uint32_t i = 0; i < count; ++i) RC(check_query(h, q[i]));
    for (auto& g : by_level(h, q, count))
        RC(h->sh.packed ? stage1_packed(h, q, g.second, g.first) : stage1_reference(h, q, g.second, g.first));
    return AFHE_OK;
}

int afhe_ivfpq_stage3(afhe_ivfpq* h, const afhe_ivfpq_query* q, uint32_t count) {
    if (!h || (count && !q)) return fail_h(h, AFHE_E_ARG, "null argument");
    if (diagonal(h)) {
        if (h->scratch.empty() || h->list_first_unit.empty()) return fail_h(h, AFHE_E_STATE, "scratch and units not set");
        std::vector<std::pair<uint32_t, u64>> lay;
        for (uint32_t i = 0; i < count; ++i) {
            RC(check_query(h, q[i]));
            if (q[i].nprobe && !q[i].probes) return fail_h(h, AFHE_E_ARG, "null probes");
            if (!unit_layout(h, q[i], lay)) return fail_h(h, AFHE_E_RANGE, "probed list out of range");
            if (!lay.empty() && lay.back().second / h->sh.slots >= q[i].n_results)
                return fail_h(h, AFHE_E_RANGE, "more candidates than the result ciphertexts hold");
        }
        for (auto& g : by_level(h, q, count)) RC(stage3_diagonal(h, q, g.second, g.first));
        return AFHE_OK;
    }
    if (h->work.empty()) return fail_h(h, AFHE_E_STATE, "lanes not set");
    const uint32_t S = h->sh.slots, B = S / h->sh.D;
    std::vector<uint32_t> first_batch(h->sh.n_list + 1, 0);      // global number of each list's first batch
    for (uint32_t c = 0; c < h->sh.n_list; ++c) first_batch[c + 1] = first_batch[c] + (uint32_t)h->lists[c].size();
    std::map<uint32_t, std::vector<Item>> items;
    for (uint32_t qi = 0; qi < count; ++qi) {
        RC(check_query(h, q[qi]));
        if (q[qi].nprobe && !q[qi].probes) return fail_h(h, AFHE_E_ARG, "null probes");
        auto& lst = items[eval_at(h, q[qi].level)];
        u64 off = 0;
        uint32_t t = 0;
        for (uint32_t p = 0; p < q[qi].nprobe; ++p) {
            const uint32_t c = q[qi].probes[p];
            if (c >= h->sh.n_list) return fail_h(h, AFHE_E_RANGE, "probed list out of range");
            for (size_t bi = 0; bi < h->lists[c].size(); ++bi) {
                const auto& b = h->lists[c][bi];
                u64 at_;
                if (h->sh.packed) {
                    at_ = (u64)t * B;            // batch t at slot t B
                } else {
                    if (off % S + b.second > S) off = (off / S + 1) * S;   // no batch straddles two results
                    at_ = off;
                    off += b.second;
                }
                if (at_ / S >= q[qi].n_results) return fail_h(h, AFHE_E_RANGE, "more candidates than the result ciphertexts hold");
                lst.push_back({qi, b.first, b.second, at_, first_batch[c] + (uint32_t)bi});
                ++t;
            }
        }
    }
    for (auto it = items.rbegin(); it != items.rend(); ++it) RC(stage3_items(h, q, it->second, it->first));
    return AFHE_OK;
}

}  // extern "C"
