// internal.h -- context state and launch helpers shared by the CUDA sources.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/afhe.h"
#include "modarith.cuh"
#include "ntt.cuh"

namespace afhe {

// Table pointers an operator needs at one level (device memory). Every
// constant that multiplies through Shoup comes with its companion (_sh).
struct OpTabs {
    PrimeTables pt;
    uint32_t p_base;   // table index of special prime 0
    uint32_t sizeQl;   // level these tables are for
    uint32_t parts;    // digits at this level
    uint32_t alpha;
    const u64* qhat_inv[AFHE_MAX_PARTS];
    const u64* qhat_inv_sh[AFHE_MAX_PARTS];
    const u64* qhat_modp[AFHE_MAX_PARTS];
    const u64* qhat_modp_sh[AFHE_MAX_PARTS];
    const u64* p_inv_mod_q;
    const u64* p_inv_mod_q_sh;
    const u64* phat_inv_modp;
    const u64* phat_inv_modp_sh;
    const u64* phat_modq;       // [K][sizeQl]
    const u64* phat_modq_sh;
    const u64* qlql;
    const u64* qlql_sh;
    const u64* qlinv;
    const u64* qlinv_sh;
};

// Owned device storage for one twiddle table set. tw / itw hold raw tables
// (only for tables loaded by OP_LOAD_CONTEXT); tw2 / itw2 the (w, companion)
// pairs the kernels read.
struct DevPrimeSet {
    PrimeConst* pc = nullptr;
    u64* tw = nullptr;
    u64* itw = nullptr;
    ulonglong2* tw2 = nullptr;
    ulonglong2* itw2 = nullptr;
    uint32_t count = 0;
    PrimeTables view() const { return PrimeTables{pc, tw2, itw2}; }
};

// Ring of small per-launch descriptor arrays (ZField::arr): pinned host
// staging and device memory in segments; a segment is reused only after the
// event recorded when the stream moved past it has completed.
struct DescRing {
    u64* host = nullptr;
    u64* dev = nullptr;
    size_t seg_words = 0, nseg = 0, cur = 0, pos = 0;
    std::vector<cudaEvent_t> ev;
    std::vector<char> used;
};

struct RotKey {
    int32_t step;
    uint32_t galois;
    u64 evk_offset;
    uint32_t* map;              // device, N entries
    ulonglong2* prep = nullptr;  // (k mod q, Shoup companion) per key word, for the one-kernel key switch
};

// Key-switch job templates for one level (device arrays).
struct LevelJobs {
    LimbJob* modup = nullptr;   // per (digit, complementary limb)
    uint32_t n_modup = 0;
};

}  // namespace afhe

struct afhe_ctx {
    afhe_params prm;
    int log_n;
    uint32_t n, L, K, alpha, dnum;
    int device;
    cudaStream_t st = nullptr;
    afhe::u64* poly = nullptr;
    afhe::u64* key = nullptr;

    // native tables: primes q[0..L), p[0..K) at indices [0, L) and [L, L + K)
    afhe::DevPrimeSet nat;
    afhe::u64* lvbuf = nullptr;                 // per-level CRT tables
    std::vector<afhe::OpTabs> lv;                // index = level (1..L)
    afhe::OpTabs* lv_dev = nullptr;              // the same, in device memory (mixed-level launches)
    afhe::LimbJob* jobs_qp = nullptr;            // slot i -> prime i, offsets i*N, for i < L + K
    std::vector<afhe::LevelJobs> lvjobs;         // index = level

    // tables loaded by OP_LOAD_CONTEXT (dispatch path)
    bool loaded = false;
    afhe::DevPrimeSet ld;
    uint32_t ld_nq = 0, ld_np = 0, ld_alpha = 0, ld_parts = 0;
    std::vector<afhe::u64> ld_q, ld_p, ld_ninv_q, ld_ninv_p;
    afhe::u64* ld_crt = nullptr;       // raw CRT tables as loaded (device)
    afhe::u64* ld_crt_sh = nullptr;    // per-call companions (device)
    afhe::u64* ld_mod = nullptr;       // per-call moduli for companion prep (device)
    size_t ld_crt_words = 0;
    std::vector<size_t> ld_off_qhat_inv, ld_off_qhat_modp;
    size_t ld_off_pinv = 0, ld_off_phatinv = 0, ld_off_phatmodq = 0, ld_off_qlql = 0, ld_off_qlinv = 0;
    // loaded tables prepared for the last (sizeQl, parts, alpha, key switch)
    // a dispatched op used; reused while the next op has the same shape
    int ld_tabs_key[4] = {-1, -1, -1, -1};
    afhe::OpTabs ld_tabs{};

    // scratch for composite operators (context-private), `lanes` lanes
    afhe::u64* scr = nullptr;
    size_t scr_words = 0;
    uint32_t lanes = 64;
    afhe::DescRing ring;
    bool ks_fused = true;   // one-kernel key switch where supported (AFHE_KS_FUSED=0 turns it off)
    uint32_t chunk = 0;     // ciphertexts per launch of a batched call (0: all lanes)
    uint32_t fused_min = 1; // launches of fewer ciphertexts take the multi-kernel key switch
    uint32_t ks_ept = 8;    // values per thread of the one-kernel key switch (8 or 16)
    uint32_t ks_slice = 13; // log2 of the slice a CTA of a cluster holds (12: N = 2^14, 2^15 only)
    // afhe_fence: fence f is event fences[f % size], recorded on st
    std::vector<cudaEvent_t> fences;
    uint64_t fence_next = 0;

    // key directory
    bool has_relin = false;
    afhe::u64 relin_off = 0;
    ulonglong2* relin_prep = nullptr;
    std::map<int32_t, afhe::RotKey> rot;
    // device automorphism maps by Galois element (afhe_automorphism_batch)
    std::map<uint32_t, uint32_t*> auto_maps;
    // whether a map keeps every 256-word tile within itself (by Galois element)
    std::map<uint32_t, bool> auto_map_local;
    // afhe_decode_batch's working memory, grown on demand and kept (a
    // cudaFree per call would wait for every stream of the device)
    void* dec_ws = nullptr;
    size_t dec_ws_bytes = 0;

    // device address of the static working array of afhe_key_switch_noalloc
    // on this context's device, looked up when the context is created (null
    // if the lookup failed; noalloc_err then holds the CUDA error)
    afhe::u64* noalloc_scr = nullptr;
    cudaError_t noalloc_err = cudaSuccess;

    std::string err;
};

namespace afhe {

// ---- kernel launchers (kernels.cu) -----------------------------------------
uint64_t launches_so_far();
enum ElemOp { EW_ADD = 0, EW_SUB = 1, EW_MUL = 2, EW_COPY = 3 };

// out[l] = a[l] op b[l] for limbs l < limbs, primes from pc[prime0 + l]; z
// entries with per-z offsets in zb (src = a, aux = b, out = out).
cudaError_t launch_elementwise(ElemOp op, const PrimeConst* pc, uint32_t prime0, u64* arena, uint32_t n,
                               uint32_t limbs, uint32_t nz, const ZBases& zb, cudaStream_t st);

// Ciphertext tensor product operands, per z (word offsets into one arena).
struct TensorArgs {
    ZField a0, a1, b0, b1, d0, d1, d2;
};
cudaError_t launch_tensor(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t nz,
                          const TensorArgs& ta, cudaStream_t st);

// out[l][i] = a[l][map[i]]; map as u32[N] (device) or packed pairs in u64.
cudaError_t launch_automorphism(const uint32_t* map32, const u64* map64, u64* arena, uint32_t n, uint32_t limbs,
                                uint32_t nz, const ZBases& zb, cudaStream_t st);
// out_z = in_z through permutation maps.at(z) (a device address per polynomial)
cudaError_t launch_automorphism_z(const ZField& maps, u64* arena, uint32_t n, uint32_t limbs, uint32_t nz,
                                  const ZBases& zb, cudaStream_t st);

// Sums of plaintext-ciphertext products (afhe_eval_mac_plain_batch): job z
// writes out = sum over its groups of sum over the group's terms of
// pt[map[i]] * src (both polynomials), limbs l < limbs with prime l. A group
// whose src0 is kMacUnit multiplies by the constant ciphertext (1, 0). Terms
// are reduced once at the end (128-bit accumulators, folded every
// reduce_every terms); accumulate adds the existing out.
constexpr u64 kMacUnit = ~0ull;
struct MacJob {
    u64 out0, out1;
    uint32_t g0, g1;
};
struct MacGroup {
    u64 src0, src1;
    uint32_t t0, t1;
};
struct MacTerm {
    u64 pt;
    const uint32_t* map;   // null: identity
};
// The diagonal method's inner products (afhe_eval_diag_inner_batch): job z
// writes out = sum over its units k of sum over b < nb of
// pt_k[b stride + map_k[i]] * src_{z, b}, srcs[z nb + b] = (c0, c1) offsets.
// staged: every map keeps 256-word tiles within themselves, every plaintext
// offset and the stride are even and N is a multiple of 256 (the
// shared-memory form); halves (staged only): every prime is below 2^50
// (25-bit split products).
struct DiagJob {
    u64 out0, out1;
    uint32_t u0, u1;
};
struct DiagUnit {
    u64 pt;
    const uint32_t* map;   // null: identity
};
cudaError_t launch_diag_inner(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t jobs,
                              uint32_t nb, const DiagJob* job, const u64* srcs, const DiagUnit* unit, u64 stride,
                              uint32_t reduce_every, int accumulate, bool staged, bool halves, cudaStream_t st);
cudaError_t launch_mac_plain(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t jobs,
                             const MacJob* job, const MacGroup* group, const MacTerm* term, uint32_t reduce_every,
                             int accumulate, cudaStream_t st);

// Plain (I)NTT of `limbs` limbs laid out contiguously (limb i at +i*N), table
// index prime0 + i. src arena -> dst arena, per-z offsets zb.src / zb.out.
cudaError_t launch_ntt_plain(bool inverse, int log_n, const PrimeTables& pt, const LimbJob* jobs, uint32_t limbs,
                             u64* src_arena, u64* dst_arena, uint32_t nz, const ZBases& zb, cudaStream_t st);

// Rescale of nz polynomials at level sizeQl: zb.src = input polys (arena),
// zb.out = outputs (arena), zb.mid = scratch for the last limb's coefficients
// (scratch arena, N words each), zb.aux = scratch for pass intermediates
// ((sizeQl - 1) * N words each).
cudaError_t launch_rescale(int log_n, const OpTabs& t, const LimbJob* jobs_q, uint32_t sizeQl, u64* arena,
                           u64* scratch, uint32_t nz, const ZBases& zb, cudaStream_t st);

// Key switch of nz polynomials at level sizeQl. Per z: zb.src = input poly
// (arena), zb.out = ks0 output, zb.aux = ks1 output (arena), zb.mid = scratch
// region of ks_scratch_words(...) words. Key digit `part`, limb i lives at
// key + evk_a / evk_b + (part * key_stride + (i < sizeQl ? i : key_pbase + i - sizeQl)) * N.
// Optional fusion around a key switch (rotation and accumulation):
//   * map: the input is read through the automorphism, x -> in[map[x]];
//   * has_c0: ks0 output += c0[map[x]] (c0 gathered into scratch by the MAC);
//   * has_acc: ks0 output += acc0[x], ks1 output += acc1[x].
// So one call computes a whole rotation step, acc + rot(ct), or d + KS(d2).
// With per_z, entry z has its own rotation: its automorphism map at the
// device address mapz.at(z), its key at keyz.at(z) words past evk_a / evk_b,
// and (one-kernel key switch with prepared keys) that key's prepared copy at
// the device address prepz.at(z).
struct KsFuse {
    const uint32_t* map;
    int has_c0;
    int has_acc;
    ZField c0, acc0, acc1;
    int per_z;
    ZField mapz, keyz, prepz;
};
size_t ks_scratch_words(uint32_t n, uint32_t L, uint32_t K, uint32_t parts);
cudaError_t launch_key_switch(int log_n, const OpTabs& t, const LimbJob* jobs_qp, const LimbJob* jobs_modup,
                              uint32_t n_modup, uint32_t slots_q, uint32_t sizeQl, uint32_t K,
                              const u64* key, u64 evk_a, u64 evk_b, uint32_t key_stride, uint32_t key_pbase,
                              u64* arena, u64* scratch, uint32_t nz, const ZBases& zb, cudaStream_t st,
                              const KsFuse* fuse = nullptr);

// The same key switch as one kernel per polynomial: for N <= 2^13 one CTA,
// above that a cluster of N / 2^13 CTAs (distributed shared memory) keeps
// the limb being transformed and both accumulators in shared memory
// and needs ks_fused_scratch_words(...) words of scratch at zb.mid (the INTT
// of the input's limbs and of the special accumulators). Entries of one
// launch run concurrently, so an entry's outputs must not overlap another
// entry's inputs (in place within an entry is fine).
// `prep`, when given, holds the key (evk_a digits then evk_b digits, the key
// region's word order) as (k mod q, Shoup companion) pairs; the inner product
// then multiplies with Shoup's method instead of a full 128-bit reduction.
bool key_switch_fused_supported(int log_n);
// ciphertexts the one-kernel key switch holds at once on the current device
// (resident CTAs at N <= 2^13, resident clusters above; 0: cannot run)
int key_switch_fused_capacity(int log_n, int ept = 8, int slice = 13);
size_t ks_fused_scratch_words(uint32_t n, uint32_t sizeQl, uint32_t K);
cudaError_t launch_key_switch_fused(int log_n, const OpTabs& t, uint32_t sizeQl, uint32_t K, const u64* key, u64 evk_a,
                                    u64 evk_b, uint32_t key_stride, uint32_t key_pbase, u64* arena, u64* scratch,
                                    uint32_t nz, const ZBases& zb, cudaStream_t st, const KsFuse* fuse = nullptr,
                                    const ulonglong2* prep = nullptr, const OpTabs* lvtabs = nullptr,
                                    const ZField* lvz = nullptr, int ept = 8, int slice = 13);
// With lvtabs and lvz (mixed levels), entry z runs at level lvz->at(z) with
// the tables lvtabs[level] (a device copy of the context's per-level tables;
// sizeQl is then the largest level), each reading and writing that many limbs.
// prep[w] = (k mod q, companion) for k = key[w], w < words, where word w
// belongs to key limb slot (w / n) mod S and slot i uses prime pc[i].
cudaError_t launch_key_prep(const u64* key, ulonglong2* prep, const PrimeConst* pc, uint32_t n, uint32_t S, u64 words,
                            cudaStream_t st);

// Twiddle pairs: out2[r * n + j] = (w, companion of w), w = raw[r * n + j] mod q[r].
cudaError_t launch_interleave(const u64* raw, const u64* q, ulonglong2* out2, uint32_t rows, uint32_t n,
                              cudaStream_t st);
// Companion prep: sh[e] = shoup_companion(v[e] mod m[e], m[e]); v reduced in place.
cudaError_t launch_companions(u64* v, u64* sh, const u64* m, size_t count, cudaStream_t st);
// Loaded prime constants: fills pc[i] from q/ninv arrays (device) and itw.
cudaError_t launch_prime_consts(PrimeConst* pc, const u64* q, const u64* ninv, const u64* itw, uint32_t n,
                                uint32_t count, cudaStream_t st);

}  // namespace afhe
