// ksfused.cu -- the whole hybrid key switch in one kernel, N = 2^10 .. 2^16.
//
// Same arithmetic as launch_key_switch (key_switch.cpp:167-439 restated:
// INTT of the input's limbs, fast_bases_conv to each digit's complementary
// primes, NTT, inner product with evk_a / evk_b, approx_mod_down), but one
// polynomial is carried through every step by one CTA (N <= 2^13) or by a
// thread-block cluster of CL = N / 2^13 CTAs (N = 2^14, 2^15, 2^16: 2, 4 or
// 8 CTAs), with the limb being transformed held in shared memory:
//
//   phase 0  coef[i] = INTT(in[i]) * qHatInv_i for the input's Q limbs -> lane scratch
//   phase 1  for every special slot k: the MAC over digits (each digit's value
//            for the slot is the input itself when the slot is one of the
//            digit's own limbs, else BConv(coef) + NTT); INTT of both
//            accumulators -> lane scratch
//   phase 2  for every Q limb i: the MAC as above, then for each accumulator
//            BConv of the special limbs to q_i, NTT, (acc - that) * P^-1, plus
//            the fused extras (c0 through the automorphism, accumulate), and
//            the store of output limb i
//
// Shared memory: three padded limb buffers (W for transforms, A0 / A1 for the
// two accumulators). A cluster splits each buffer: CTA r holds elements
// [r QN, (r + 1) QN), QN = 2^13, so every CTA uses 3 * (QN + QN/16) words =
// 204 KB whatever N is. The transforms' low 13 butterfly stages run inside a
// CTA on its slice (the tile code of ntt.cuh, with the slice index as the
// index bits above the tile); the top log2(CL) stages combine the CL slices
// and run across the cluster through distributed shared memory, between two
// cluster barriers: forward NTTs start with them, inverse NTTs end with them
// (where the last one folds in N^-1). Element-wise work (base conversions,
// inner products, ModDown combine) runs on each CTA's own slice.
//
// The key limbs every CTA of a launch reads are the same, so they come from
// L2. A registered key comes as a prepared copy of (k mod q, Shoup
// companion) pairs, so each inner-product term is one Shoup multiplication.
//
// In place is safe: input limb i is read only while slot i is processed, and
// output limb i is written after every read of input limb i (the cluster
// barriers of the transforms in between) and of the gathered c0 limb i
// (staged in shared memory behind a barrier across the whole cluster).
#include <cooperative_groups.h>

#include <map>
#include <mutex>
#include <tuple>

#include "internal.h"

namespace cg = cooperative_groups;

namespace afhe {

namespace {

struct KsFusedArgs {
    OpTabs t;
    uint32_t sizeQl, K;
    const u64* key;
    u64 evk_a, evk_b;
    uint32_t key_stride, key_pbase;
    u64* arena;
    u64* scratch;
    ZField in, out0, out1, mid;
    KsFuse f;
    const ulonglong2* prep;   // prepared key (evk_a digits, then evk_b digits), or null
    u64 prep_b;               // offset of the evk_b digits in prep
    // mixed levels: entry z runs at level lvz.at(z) with the tables
    // lvtabs[level] (device copy of the context's per-level tables); null:
    // every entry at sizeQl with t
    const OpTabs* lvtabs;
    ZField lvz;
};

constexpr int kLogQ = 13;    // log2 of the slice a CTA holds at N >= 2^13 (12 on request at N = 2^14, 2^15)

// One polynomial per CTA (LOGCL = 0) or per cluster of 2^LOGCL CTAs; each CTA
// holds 2^LOGQ elements of every buffer. Local positions e < 2^LOGQ, global
// positions x = rank * 2^LOGQ + e.
template <int LOGQ, int LOGCL, int E = 8>
struct Geo {
    static constexpr int LOGN = LOGQ + LOGCL;
    static constexpr uint32_t QN = 1u << LOGQ;
    static constexpr uint32_t CL = 1u << LOGCL;
    static constexpr uint32_t THREADS = QN / E;
    __device__ __forceinline__ static uint32_t rank() {
        if constexpr (LOGCL == 0) return 0;
        else return cg::this_cluster().block_rank();
    }
    // every element of every CTA's slices is visible to every CTA after this
    __device__ __forceinline__ static void sync_all() {
        if constexpr (LOGCL == 0) __syncthreads();
        else cg::this_cluster().sync();
    }
    __device__ __forceinline__ static uint32_t z() { return blockIdx.x >> LOGCL; }
};

// digit j of a level-l key switch: limbs [start, start + size)
__device__ __forceinline__ void digit_range(const OpTabs& t, uint32_t j, uint32_t& start, uint32_t& size) {
    start = j * t.alpha;
    size = (j == t.parts - 1) ? t.sizeQl - start : t.alpha;
}

// The top LOGCL butterfly stages of a forward NTT, across the cluster: the
// CL elements x = k QN + j (k < CL) form a column of CL values, transformed
// by the stages of bits LOGN - 1 .. LOGQ (block b of stage s uses tw[2^s + b]).
// CTA r takes the columns j in [r QN / CL, (r + 1) QN / CL).
template <int LOGQ, int LOGCL, int NB, int E>
__device__ __forceinline__ void cross_fwd(u64* const (&bufs)[NB], const ulonglong2* __restrict__ tw,
                                          const PrimeConst& pc) {
    using G = Geo<LOGQ, LOGCL, E>;
    constexpr uint32_t CL = G::CL, PER = G::QN / CL;
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t r = cl.block_rank();
    const u64 q = pc.q, q2 = q << 1;
    ulonglong2 w[CL - 1];
#pragma unroll
    for (uint32_t i = 1; i < CL; ++i) w[i - 1] = __ldg(tw + i);
    u64* rb[NB][CL];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (uint32_t k = 0; k < CL; ++k) rb[b][k] = cl.map_shared_rank(bufs[b], k);
    for (uint32_t jj = threadIdx.x; jj < PER; jj += G::THREADS) {
        const uint32_t e = padix(r * PER + jj);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            u64 v[CL];
#pragma unroll
            for (uint32_t k = 0; k < CL; ++k) v[k] = rb[b][k][e];
#pragma unroll
            for (int s = 0; s < LOGCL; ++s) {
                const uint32_t m = 1u << s, t = CL >> (s + 1);
#pragma unroll
                for (uint32_t blk = 0; blk < m; ++blk)
#pragma unroll
                    for (uint32_t i = 0; i < t; ++i)
                        ct_bfly(v[blk * 2 * t + i], v[blk * 2 * t + i + t], w[m + blk - 1], q, q2);
            }
#pragma unroll
            for (uint32_t k = 0; k < CL; ++k) rb[b][k][e] = v[k];
        }
    }
}

// The top LOGCL stages of an inverse NTT (Gentleman-Sande, bits LOGQ ..
// LOGN - 1), the last one with N^-1 folded in; outputs canonical.
template <int LOGQ, int LOGCL, int NB, int E>
__device__ __forceinline__ void cross_inv(u64* const (&bufs)[NB], const ulonglong2* __restrict__ itw,
                                          const PrimeConst& pc) {
    using G = Geo<LOGQ, LOGCL, E>;
    constexpr uint32_t CL = G::CL, PER = G::QN / CL;
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t r = cl.block_rank();
    const u64 q = pc.q, q2 = q << 1;
    ulonglong2 w[CL > 2 ? CL - 1 : 1];
#pragma unroll
    for (uint32_t i = 2; i < CL; ++i) w[i - 1] = __ldg(itw + i);   // itw[1] enters through pc.w1ninv
    u64* rb[NB][CL];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (uint32_t k = 0; k < CL; ++k) rb[b][k] = cl.map_shared_rank(bufs[b], k);
    for (uint32_t jj = threadIdx.x; jj < PER; jj += G::THREADS) {
        const uint32_t e = padix(r * PER + jj);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            u64 v[CL];
#pragma unroll
            for (uint32_t k = 0; k < CL; ++k) v[k] = rb[b][k][e];
#pragma unroll
            for (int s = LOGCL - 1; s >= 0; --s) {
                const uint32_t m = 1u << s, t = CL >> (s + 1);
                if (s == 0) {
#pragma unroll
                    for (uint32_t i = 0; i < t; ++i) gs_bfly_last(v[i], v[i + t], pc, q2);
                } else {
#pragma unroll
                    for (uint32_t blk = 0; blk < m; ++blk)
#pragma unroll
                        for (uint32_t i = 0; i < t; ++i)
                            gs_bfly(v[blk * 2 * t + i], v[blk * 2 * t + i + t], w[m + blk - 1], q, q2);
                }
            }
#pragma unroll
            for (uint32_t k = 0; k < CL; ++k) rb[b][k][e] = v[k];
        }
    }
}

// Radix of a CTA's own transform rounds: 2^4 where 16 values per thread
// divide the slice's bits into whole rounds (2^12-value slices: three rounds
// instead of four), else 2^3.
template <int LOGQ, int E>
constexpr int round_bits() { return (E == 16 && LOGQ % 4 == 0) ? 4 : 3; }

// Forward NTT of one buffer. On entry this CTA's slice is written (and
// visible after a CTA barrier); on return the slice holds lazy residues in
// [0, 4q). Not inlined: each transform gets its own register allocation
// instead of competing with the caller's live state (1024 threads leave 64
// registers).
template <int LOGQ, int LOGCL, int E>
__device__ __noinline__ void fwd_ntt(u64* buf, const PrimeTables pt, uint32_t prime, const PrimeConst pc) {
    using G = Geo<LOGQ, LOGCL, E>;
    const ulonglong2* tw = pt.tw2 + ((u64)prime << G::LOGN);
    if constexpr (LOGCL > 0) {
        u64* const one[1] = {buf};
        G::sync_all();
        cross_fwd<LOGQ, LOGCL, 1, E>(one, tw, pc);
        G::sync_all();
    }
    ntt_rounds<false, LOGQ, 0, false, 0, E, round_bits<LOGQ, E>()>(buf, tw, pc, G::rank(), G::LOGN, 0, true);
}

// Inverse NTT of one buffer; on return the slice holds canonical residues.
template <int LOGQ, int LOGCL, int E>
__device__ __noinline__ void inv_ntt(u64* buf, const PrimeTables pt, uint32_t prime, const PrimeConst pc) {
    using G = Geo<LOGQ, LOGCL, E>;
    const ulonglong2* itw = pt.itw2 + ((u64)prime << G::LOGN);
    ntt_rounds<true, LOGQ, 0, false, 0, E, round_bits<LOGQ, E>()>(buf, itw, pc, G::rank(), G::LOGN, 0, LOGCL == 0);
    if constexpr (LOGCL > 0) {
        u64* const one[1] = {buf};
        G::sync_all();
        cross_inv<LOGQ, LOGCL, 1, E>(one, itw, pc);
        G::sync_all();
    }
}

// Two limbs of the same prime transformed together (shared twiddles).
template <bool INV, int LOGQ, int LOGCL, int E>
__device__ __noinline__ void ntt2(u64* b0, u64* b1, const PrimeTables pt, uint32_t prime, const PrimeConst pc) {
    using G = Geo<LOGQ, LOGCL, E>;
    u64* const bufs[2] = {b0, b1};
    const ulonglong2* tw = (INV ? pt.itw2 : pt.tw2) + ((u64)prime << G::LOGN);
    if constexpr (!INV && LOGCL > 0) {
        G::sync_all();
        cross_fwd<LOGQ, LOGCL, 2, E>(bufs, tw, pc);
        G::sync_all();
    }
    ntt_rounds_n<INV, LOGQ, 0, false, 0, E, 2, round_bits<LOGQ, E>()>(bufs, tw, pc, G::rank(), G::LOGN, 0,
                                                                       !INV || LOGCL == 0);
    if constexpr (INV && LOGCL > 0) {
        G::sync_all();
        cross_inv<LOGQ, LOGCL, 2, E>(bufs, tw, pc);
        G::sync_all();
    }
}

// Every element-wise pass below gives each of the QN / E threads the local
// positions e_k = threadIdx.x + k * QN/E, k < E (global x_k = rank * QN +
// e_k), and issues a chunk's global loads before its arithmetic, so several
// L2 round trips are in flight per thread. E (values per thread: 8, or 16
// with half the threads and twice the registers each) is the kernel's
// template parameter, picked at run time (AFHE_OPT_KS_EPT).
constexpr uint32_t kChunk = 4;   // positions whose loads are issued together

template <int LOGQ, int E>
__device__ __forceinline__ uint32_t lpos(uint32_t k) { return threadIdx.x + k * ((1u << LOGQ) / E); }

// gathered position of x: the automorphism's source index, or x itself
__device__ __forceinline__ uint32_t gpos(const uint32_t* map, uint32_t x) { return map ? __ldg(map + x) : x; }

// This entry's rotation (automorphism map, key offset, prepared key).
struct EntryKey {
    const uint32_t* map;
    u64 koff;
    const ulonglong2* prep;
};

__device__ __forceinline__ EntryKey entry_key(const KsFusedArgs& a, uint32_t z) {
    EntryKey k;
    if (a.f.per_z) {
        k.map = (const uint32_t*)a.f.mapz.at(z);
        k.koff = a.f.keyz.at(z);
        k.prep = a.prep ? (const ulonglong2*)a.f.prepz.at(z) : nullptr;
    } else {
        k.map = a.f.map;
        k.koff = 0;
        k.prep = a.prep;
    }
    return k;
}

// Inner product for one slot (Q limb `s` < l, or special limb s - l) into
// this CTA's slices of A0 / A1: A0 = sum_j d_j * evk_b[j], A1 = sum_j d_j *
// evk_a[j] (mod the slot's prime).
template <int LOGQ, int LOGCL, bool PREP, int E>
__device__ void mac_slot(const KsFusedArgs& a, const OpTabs& t, uint32_t l, const EntryKey& ek, uint32_t s, u64* W,
                         u64* A0, u64* A1,
                         const u64* __restrict__ in, const u64* __restrict__ coef) {
    using G = Geo<LOGQ, LOGCL, E>;
    constexpr int LOGN = G::LOGN;
    constexpr uint32_t N = 1u << LOGN;
    const uint32_t x0 = G::rank() * G::QN;
    const bool isq = s < l;
    const uint32_t prime = isq ? s : t.p_base + (s - l);
    const uint32_t klimb = isq ? s : a.key_pbase + (s - l);
    const PrimeConst pc = t.pt.pc[prime];
    const ModConst mc = modconst_of(pc);
    const u64 q = pc.q, p2 = q << 1;
    const uint32_t* map = ek.map;
    for (uint32_t j = 0; j < t.parts; ++j) {
        uint32_t start, size;
        digit_range(t, j, start, size);
        const bool own = isq && s >= start && s < start + size;
        const u64 kofs = ((u64)j * a.key_stride + klimb) * N;
        const u64* kb = a.key + a.evk_b + ek.koff + kofs;
        const u64* ka = a.key + a.evk_a + ek.koff + kofs;
        const ulonglong2* pb2 = PREP ? ek.prep + a.prep_b + kofs : nullptr;
        const ulonglong2* pa2 = PREP ? ek.prep + kofs : nullptr;
        if (!own) {
            // W = BConv_j(coef) at this slot's prime, then NTT
            const uint32_t row = l - size + a.K;
            const uint32_t kpos = isq ? (s < start ? s : s - size) : (l - size) + (s - l);
            u64 acc[E];
#pragma unroll
            for (uint32_t k = 0; k < E; ++k) acc[k] = 0;
            for (uint32_t i = 0; i < size; ++i) {
                const uint32_t limb = start + i;
                const u64 w1 = __ldg(t.qhat_modp[j] + i * row + kpos), w1s = __ldg(t.qhat_modp_sh[j] + i * row + kpos);
                const u64* src = coef + ((u64)limb << LOGN) + x0;     // [x * qHatInv]_{q_i} (phase 0)
                u64 v[E];
#pragma unroll
                for (uint32_t k = 0; k < E; ++k) v[k] = src[lpos<LOGQ, E>(k)];
#pragma unroll
                for (uint32_t k = 0; k < E; ++k) {
                    acc[k] += mul_shoup_lazy(v[k], w1, w1s, q);
                    acc[k] = acc[k] >= p2 ? acc[k] - p2 : acc[k];
                }
            }
#pragma unroll
            for (uint32_t k = 0; k < E; ++k) W[padix(lpos<LOGQ, E>(k))] = csub(acc[k], q);
            __syncthreads();
            fwd_ntt<LOGQ, LOGCL, E>(W, t.pt, prime, pc);
        }
        const u64* src = in + ((u64)s << LOGN);
        if (PREP) {
            // Shoup products with the prepared key; the accumulators stay lazy
            // in [0, 2q) (both consumers accept that range)
#pragma unroll
            for (uint32_t c = 0; c < E; c += kChunk) {
                u64 d[kChunk];
                ulonglong2 vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = x0 + lpos<LOGQ, E>(c + k);
                    vb[k] = __ldg(pb2 + x);
                    va[k] = __ldg(pa2 + x);
                    d[k] = own ? src[gpos(map, x)] : W[padix(lpos<LOGQ, E>(c + k))];   // any d < 2^64 is valid for Shoup
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t e = padix(lpos<LOGQ, E>(c + k));
                    u64 pb = mul_shoup_lazy(d[k], vb[k].x, vb[k].y, q);
                    u64 pa = mul_shoup_lazy(d[k], va[k].x, va[k].y, q);
                    if (j > 0) {
                        pb += A0[e];
                        pa += A1[e];
                        pb = pb >= p2 ? pb - p2 : pb;
                        pa = pa >= p2 ? pa - p2 : pa;
                    }
                    A0[e] = pb;
                    A1[e] = pa;
                }
            }
        } else {
#pragma unroll
            for (uint32_t c = 0; c < E; c += kChunk) {
                u64 d[kChunk], vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = x0 + lpos<LOGQ, E>(c + k);
                    vb[k] = __ldg(kb + x);
                    va[k] = __ldg(ka + x);
                    d[k] = own ? src[gpos(map, x)] : canon4(W[padix(lpos<LOGQ, E>(c + k))], q);
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t e = padix(lpos<LOGQ, E>(c + k));
                    u64 pb = mul_mod(d[k], vb[k], mc);
                    u64 pa = mul_mod(d[k], va[k], mc);
                    if (j > 0) {
                        pb = add_mod(pb, A0[e], q);
                        pa = add_mod(pa, A1[e], q);
                    }
                    A0[e] = pb;
                    A1[e] = pa;
                }
            }
        }
        __syncthreads();
    }
}

// The key switch at one Q limb with one special prime (a single digit), N <=
// 2^13: nothing leaves shared memory between the input load and the output
// store.
//   W = INTT_q0(in), W = BConv(W) to P, W = NTT_P(W); A_h = W * key_h[P];
//   (A0, A1) = INTT_P; BConv to q0 in place; (A0, A1) = NTT_q0;
//   out_h = (in * key_h[q0] - A_h) * P^-1 (+ extras), the own digit's product
//   computed in the same pass. Same residues as the general path.
template <int LOGN, bool PREP, int E>
__device__ __forceinline__ void ks_one_limb(const KsFusedArgs& a, const OpTabs& t, const EntryKey& ek, u64* W, u64* A0,
                                            u64* A1) {
    constexpr uint32_t N = 1u << LOGN;
    const uint32_t z = blockIdx.x;
    const uint32_t* map = ek.map;
    const u64* in = a.arena + a.in.at(z);
    const PrimeConst pq = t.pt.pc[0], pp = t.pt.pc[t.p_base];
    const u64 q = pq.q, p = pp.q;
    const u64* key = a.key + ek.koff;
    // W = INTT_q0(input through the automorphism)
    {
        uint32_t g[E];
        u64 v[E];
#pragma unroll
        for (uint32_t k = 0; k < E; ++k) g[k] = gpos(map, lpos<LOGN, E>(k));
#pragma unroll
        for (uint32_t k = 0; k < E; ++k) v[k] = in[g[k]];
#pragma unroll
        for (uint32_t k = 0; k < E; ++k) W[padix(lpos<LOGN, E>(k))] = v[k];
    }
    __syncthreads();
    inv_ntt<LOGN, 0, E>(W, t.pt, 0, pq);
    // BConv q0 -> P in place (digit 0's only limb), then NTT_P
    {
        const u64 w0 = __ldg(t.qhat_inv[0]), w0s = __ldg(t.qhat_inv_sh[0]);
        const u64 w1 = __ldg(t.qhat_modp[0]), w1s = __ldg(t.qhat_modp_sh[0]);
#pragma unroll
        for (uint32_t k = 0; k < E; ++k) {
            const uint32_t e = padix(lpos<LOGN, E>(k));
            W[e] = csub(mul_shoup_lazy(mul_shoup(W[e], w0, w0s, q), w1, w1s, p), p);
        }
    }
    __syncthreads();
    fwd_ntt<LOGN, 0, E>(W, t.pt, t.p_base, pp);
    // inner product at P
    {
        const u64 kofs = (u64)a.key_pbase * N;
        const ModConst mc = modconst_of(pp);
#pragma unroll 1
        for (uint32_t c = 0; c < E; c += kChunk) {
            u64 d[kChunk], rb[kChunk], ra[kChunk];
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) d[k] = W[padix(lpos<LOGN, E>(c + k))];
            if (PREP) {
                ulonglong2 vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = lpos<LOGN, E>(c + k);
                    vb[k] = __ldg(ek.prep + a.prep_b + kofs + x);
                    va[k] = __ldg(ek.prep + kofs + x);
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    rb[k] = mul_shoup_lazy(d[k], vb[k].x, vb[k].y, p);
                    ra[k] = mul_shoup_lazy(d[k], va[k].x, va[k].y, p);
                }
            } else {
                u64 vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = lpos<LOGN, E>(c + k);
                    vb[k] = __ldg(key + a.evk_b + kofs + x);
                    va[k] = __ldg(key + a.evk_a + kofs + x);
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    rb[k] = mul_mod(canon4(d[k], p), vb[k], mc);
                    ra[k] = mul_mod(canon4(d[k], p), va[k], mc);
                }
            }
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) {
                const uint32_t e = padix(lpos<LOGN, E>(c + k));
                A0[e] = rb[k];
                A1[e] = ra[k];
            }
        }
    }
    __syncthreads();
    ntt2<true, LOGN, 0, E>(A0, A1, t.pt, t.p_base, pp);
    // BConv P -> q0 in place on both, then NTT_q0 of both
    {
        const u64 w0 = __ldg(t.phat_inv_modp), w0s = __ldg(t.phat_inv_modp_sh);
        const u64 w1 = __ldg(t.phat_modq), w1s = __ldg(t.phat_modq_sh);
#pragma unroll
        for (uint32_t k = 0; k < E; ++k) {
            const uint32_t e = padix(lpos<LOGN, E>(k));
            A0[e] = csub(mul_shoup_lazy(mul_shoup(A0[e], w0, w0s, p), w1, w1s, q), q);
            A1[e] = csub(mul_shoup_lazy(mul_shoup(A1[e], w0, w0s, p), w1, w1s, q), q);
        }
    }
    __syncthreads();
    ntt2<false, LOGN, 0, E>(A0, A1, t.pt, 0, pq);
    // out_h = (in * key_h[q0] - A_h) * P^-1, staged in A_h: the input and the
    // gathered c0 may alias the outputs
    {
        const ModConst mc = modconst_of(pq);
        const u64 pinv = __ldg(t.p_inv_mod_q), pinv_sh = __ldg(t.p_inv_mod_q_sh);
        const u64* cb = a.arena + (a.f.has_c0 ? a.f.c0.at(z) : 0);
#pragma unroll 1
        for (uint32_t c = 0; c < E; c += kChunk) {
            u64 d[kChunk], cv[kChunk], rb[kChunk], ra[kChunk];
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) {
                const uint32_t g = gpos(map, lpos<LOGN, E>(c + k));
                d[k] = in[g];
                cv[k] = a.f.has_c0 ? cb[g] : 0;
            }
            if (PREP) {
                ulonglong2 vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = lpos<LOGN, E>(c + k);
                    vb[k] = __ldg(ek.prep + a.prep_b + x);
                    va[k] = __ldg(ek.prep + x);
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    rb[k] = mul_shoup_lazy(d[k], vb[k].x, vb[k].y, q);
                    ra[k] = mul_shoup_lazy(d[k], va[k].x, va[k].y, q);
                }
            } else {
                u64 vb[kChunk], va[kChunk];
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    const uint32_t x = lpos<LOGN, E>(c + k);
                    vb[k] = __ldg(key + a.evk_b + x);
                    va[k] = __ldg(key + a.evk_a + x);
                }
#pragma unroll
                for (uint32_t k = 0; k < kChunk; ++k) {
                    rb[k] = mul_mod(d[k], vb[k], mc);
                    ra[k] = mul_mod(d[k], va[k], mc);
                }
            }
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) {
                const uint32_t e = padix(lpos<LOGN, E>(c + k));
                u64 r0 = mul_shoup(sub_mod(rb[k], canon4(A0[e], q), q), pinv, pinv_sh, q);
                const u64 r1 = mul_shoup(sub_mod(ra[k], canon4(A1[e], q), q), pinv, pinv_sh, q);
                if (a.f.has_c0) r0 = add_mod(r0, cv[k], q);
                A0[e] = r0;
                A1[e] = r1;
            }
        }
    }
    __syncthreads();
    {
        u64* o0 = a.arena + a.out0.at(z);
        u64* o1 = a.arena + a.out1.at(z);
        const u64* x0 = a.arena + (a.f.has_acc ? a.f.acc0.at(z) : 0);
        const u64* x1 = a.arena + (a.f.has_acc ? a.f.acc1.at(z) : 0);
#pragma unroll 1
        for (uint32_t c = 0; c < E; c += kChunk) {
            u64 e0[kChunk], e1[kChunk];
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) {
                const uint32_t x = lpos<LOGN, E>(c + k);
                e0[k] = a.f.has_acc ? x0[x] : 0;
                e1[k] = a.f.has_acc ? x1[x] : 0;
            }
#pragma unroll
            for (uint32_t k = 0; k < kChunk; ++k) {
                const uint32_t x = lpos<LOGN, E>(c + k);
                u64 r0 = A0[padix(x)], r1 = A1[padix(x)];
                if (a.f.has_acc) {
                    r0 = add_mod(r0, e0[k], q);
                    r1 = add_mod(r1, e1[k], q);
                }
                o0[x] = r0;
                o1[x] = r1;
            }
        }
    }
}

// Slices of 2^12 in a cluster (N = 2^14, 2^15) take 104 KB of shared memory
// and 512 threads: two CTAs per SM, whose barriers interleave.
template <int LOGQ, int LOGCL, bool PREP, int E>
__global__ void __launch_bounds__((1u << LOGQ) / E, (LOGCL > 0 && LOGQ < 13) ? 2 : 1)
    ks_fused_kernel(const KsFusedArgs a) {
    using G = Geo<LOGQ, LOGCL, E>;
    constexpr int LOGN = G::LOGN;
    constexpr uint32_t PADQ = G::QN + G::QN / 16;
    extern __shared__ u64 smem[];
    u64* W = smem;
    u64* A0 = smem + PADQ;
    u64* A1 = smem + 2 * PADQ;
    const uint32_t z = G::z();
    const uint32_t x0 = G::rank() * G::QN;
    const uint32_t l = a.lvtabs ? (uint32_t)a.lvz.at(z) : a.sizeQl;
    const OpTabs& t = a.lvtabs ? a.lvtabs[l] : a.t;
    const uint32_t K = a.K;
    const EntryKey ek = entry_key(a, z);
    const uint32_t* map = ek.map;
    if constexpr (LOGCL == 0) {
        if (l == 1 && K == 1) {
            ks_one_limb<LOGN, PREP, E>(a, t, ek, W, A0, A1);
            return;
        }
    }
    const u64* in = a.arena + a.in.at(z);
    u64* coef = a.scratch + a.mid.at(z);          // l limbs
    u64* pcoef = coef + ((u64)l << LOGN);         // 2K limbs: INTT of the special accumulators

    // phase 0: coefficients of the input's limbs (read through the automorphism)
    for (uint32_t i = 0; i < l; ++i) {
        const PrimeConst pc = t.pt.pc[i];
        const u64* src = in + ((u64)i << LOGN);
        {
            uint32_t g[E];
            u64 v[E];
#pragma unroll
            for (uint32_t k = 0; k < E; ++k) g[k] = gpos(map, x0 + lpos<LOGQ, E>(k));
#pragma unroll
            for (uint32_t k = 0; k < E; ++k) v[k] = src[g[k]];
#pragma unroll
            for (uint32_t k = 0; k < E; ++k) W[padix(lpos<LOGQ, E>(k))] = v[k];
        }
        __syncthreads();
        inv_ntt<LOGQ, LOGCL, E>(W, t.pt, i, pc);
        // stored times qHatInv: the first factor of ModUp's base conversion,
        // once per limb instead of once per output slot
        {
            const uint32_t part = i / t.alpha, idx = i - part * t.alpha;
            const u64 w0 = __ldg(t.qhat_inv[part] + idx), w0s = __ldg(t.qhat_inv_sh[part] + idx);
#pragma unroll
            for (uint32_t k = 0; k < E; ++k)
                coef[((u64)i << LOGN) + x0 + lpos<LOGQ, E>(k)] = mul_shoup(W[padix(lpos<LOGQ, E>(k))], w0, w0s, pc.q);
        }
        __syncthreads();
    }
    // phase 1: special slots -> INTT of both accumulators
    for (uint32_t k = 0; k < K; ++k) {
        mac_slot<LOGQ, LOGCL, PREP, E>(a, t, l, ek, l + k, W, A0, A1, in, coef);
        const uint32_t prime = t.p_base + k;
        const PrimeConst pc = t.pt.pc[prime];
        ntt2<true, LOGQ, LOGCL, E>(A0, A1, t.pt, prime, pc);
        u64* d0 = pcoef + ((u64)(2 * k) << LOGN) + x0;
        u64* d1 = pcoef + ((u64)(2 * k + 1) << LOGN) + x0;
        // stored times PHatInv_k: the first factor of ModDown's base conversion
        const u64 w0 = __ldg(t.phat_inv_modp + k), w0s = __ldg(t.phat_inv_modp_sh + k);
#pragma unroll
        for (uint32_t e = 0; e < E; ++e) {
            const uint32_t x = lpos<LOGQ, E>(e);
            d0[x] = mul_shoup(A0[padix(x)], w0, w0s, pc.q);
            d1[x] = mul_shoup(A1[padix(x)], w0, w0s, pc.q);
        }
        __syncthreads();
    }
    // phase 2: Q limbs -> ModDown and outputs
    const u64 o0 = a.out0.at(z), o1 = a.out1.at(z);
    const u64 c0 = a.f.has_c0 ? a.f.c0.at(z) : 0;
    const u64 ac0 = a.f.has_acc ? a.f.acc0.at(z) : 0, ac1 = a.f.has_acc ? a.f.acc1.at(z) : 0;
    for (uint32_t i = 0; i < l; ++i) {
        mac_slot<LOGQ, LOGCL, PREP, E>(a, t, l, ek, i, W, A0, A1, in, coef);
        const PrimeConst pc = t.pt.pc[i];
        const u64 q = pc.q, q2 = q << 1;
        const u64 pinv = __ldg(t.p_inv_mod_q + i), pinv_sh = __ldg(t.p_inv_mod_q_sh + i);
        for (uint32_t h = 0; h < 2; ++h) {
            u64* A = h ? A1 : A0;
            // W = BConv of the special limbs to q_i (approx_mod_down's fast_bases_conv), then NTT
            {
                u64 acc[E];
#pragma unroll
                for (uint32_t e = 0; e < E; ++e) acc[e] = 0;
                for (uint32_t k = 0; k < K; ++k) {
                    const u64 w1 = __ldg(t.phat_modq + k * l + i), w1s = __ldg(t.phat_modq_sh + k * l + i);
                    const u64* src = pcoef + ((u64)(2 * k + h) << LOGN) + x0;   // [x * PHatInv]_{p_k} (phase 1)
                    u64 v[E];
#pragma unroll
                    for (uint32_t e = 0; e < E; ++e) v[e] = src[lpos<LOGQ, E>(e)];
#pragma unroll
                    for (uint32_t e = 0; e < E; ++e) {
                        acc[e] += mul_shoup_lazy(v[e], w1, w1s, q);
                        acc[e] = acc[e] >= q2 ? acc[e] - q2 : acc[e];
                    }
                }
#pragma unroll
                for (uint32_t e = 0; e < E; ++e) W[padix(lpos<LOGQ, E>(e))] = csub(acc[e], q);
            }
            __syncthreads();
            fwd_ntt<LOGQ, LOGCL, E>(W, t.pt, i, pc);
            // (x_Q - y) * P^-1 plus the fused extras. The gathered c0 limb i
            // is staged in A and stored after a barrier over every CTA of the
            // polynomial (c0 may alias out0, and the gather reads any slice);
            // every other output goes straight out (each element is read and
            // written by the same thread).
            const bool stage = h == 0 && a.f.has_c0;
            const u64 ob = (h ? o1 : o0) + ((u64)i << LOGN) + x0;
            const u64 ab = (h ? ac1 : ac0) + ((u64)i << LOGN) + x0;
            const u64* cb = a.arena + c0 + ((u64)i << LOGN);
#pragma unroll
            for (uint32_t c = 0; c < E; c += kChunk) {
                u64 ex[kChunk];
#pragma unroll
                for (uint32_t e = 0; e < kChunk; ++e) {
                    const uint32_t x = lpos<LOGQ, E>(c + e);
                    ex[e] = stage ? cb[gpos(map, x0 + x)] : (a.f.has_acc ? a.arena[ab + x] : 0);
                }
#pragma unroll
                for (uint32_t e = 0; e < kChunk; ++e) {
                    const uint32_t x = lpos<LOGQ, E>(c + e);
                    // A may be lazy in [0, 2q): the difference is then in
                    // [0, 2q) and mul_shoup returns it canonical
                    u64 r = mul_shoup(sub_mod(A[padix(x)], canon4(W[padix(x)], q), q), pinv, pinv_sh, q);
                    if (stage || a.f.has_acc) r = add_mod(r, ex[e], q);
                    if (stage) A[padix(x)] = r;
                    else a.arena[ob + x] = r;
                }
            }
            if (stage) {
                G::sync_all();
#pragma unroll
                for (uint32_t c = 0; c < E; c += kChunk) {
                    u64 ex[kChunk];
#pragma unroll
                    for (uint32_t e = 0; e < kChunk; ++e) ex[e] = a.f.has_acc ? a.arena[ab + lpos<LOGQ, E>(c + e)] : 0;
#pragma unroll
                    for (uint32_t e = 0; e < kChunk; ++e) {
                        const uint32_t x = lpos<LOGQ, E>(c + e);
                        u64 r = A[padix(x)];
                        if (a.f.has_acc) r = add_mod(r, ex[e], q);
                        a.arena[ob + x] = r;
                    }
                }
            }
            __syncthreads();
        }
    }
}

template <int LOGQ, int LOGCL, bool PREP, int E>
cudaError_t launch_fused_v(const KsFusedArgs& a, uint32_t nz, cudaStream_t st) {
    constexpr uint32_t QN = 1u << LOGQ;
    const size_t smem = 3ull * (QN + QN / 16) * sizeof(u64);
    auto kern = ks_fused_kernel<LOGQ, LOGCL, PREP, E>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if constexpr (LOGCL == 0) {
        kern<<<nz, QN / E, smem, st>>>(a);
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nz << LOGCL, 1, 1);
        cfg.blockDim = dim3(QN / E, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 1u << LOGCL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, a);
        if (e != cudaSuccess) return e;
    }
    count_launches(1);
    return cudaGetLastError();
}

template <int LOGQ, int LOGCL>
cudaError_t launch_fused(const KsFusedArgs& a, uint32_t nz, cudaStream_t st, int ept) {
    if (ept == 16)
        return a.prep ? launch_fused_v<LOGQ, LOGCL, true, 16>(a, nz, st) : launch_fused_v<LOGQ, LOGCL, false, 16>(a, nz, st);
    return a.prep ? launch_fused_v<LOGQ, LOGCL, true, 8>(a, nz, st) : launch_fused_v<LOGQ, LOGCL, false, 8>(a, nz, st);
}

// 2^12-value slices (clusters of 4 or 8 CTAs, two CTAs per SM): 8 values per
// thread (512 threads, radix-8 rounds) or 16 (256 threads, radix-16 rounds)
template <int LOGCL>
cudaError_t launch_slice12(const KsFusedArgs& a, uint32_t nz, cudaStream_t st, int ept) {
    if (ept == 16)
        return a.prep ? launch_fused_v<12, LOGCL, true, 16>(a, nz, st) : launch_fused_v<12, LOGCL, false, 16>(a, nz, st);
    return a.prep ? launch_fused_v<12, LOGCL, true, 8>(a, nz, st) : launch_fused_v<12, LOGCL, false, 8>(a, nz, st);
}

// Clusters the GPU can hold at once for the kernel at N = 2^(LOGQ + LOGCL)
// (0 when it cannot place even one: the multi-kernel path is used then).
template <int LOGCL, int E = 8, int LOGQ = kLogQ>
int cluster_capacity() {
    constexpr uint32_t QN = 1u << LOGQ;
    const size_t smem = 3ull * (QN + QN / 16) * sizeof(u64);
    auto kern = ks_fused_kernel<LOGQ, LOGCL, true, E>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1u << LOGCL, 1, 1);
    cfg.blockDim = dim3(QN / E, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1u << LOGCL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <class Kern>
cudaError_t occupancy_of(Kern kern, uint32_t threads, size_t smem, int* per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, (int)threads, smem);
}

__global__ void key_prep_kernel(const u64* __restrict__ key, ulonglong2* __restrict__ prep,
                                const PrimeConst* __restrict__ pc, uint32_t n, uint32_t S, u64 words) {
    for (u64 w = blockIdx.x * (u64)blockDim.x + threadIdx.x; w < words; w += (u64)gridDim.x * blockDim.x) {
        const u64 q = pc[(w / n) % S].q;
        const u64 k = key[w] % q;
        prep[w] = make_ulonglong2(k, shoup_companion(k, q));
    }
}

}  // namespace

namespace {
int capacity_uncached(int log_n, int ept, int slice) {
    if (slice == 12 && (log_n == 14 || log_n == 15)) {
        if (ept == 16) return log_n == 14 ? cluster_capacity<2, 16, 12>() : cluster_capacity<3, 16, 12>();
        return log_n == 14 ? cluster_capacity<2, 8, 12>() : cluster_capacity<3, 8, 12>();
    }
    if (log_n >= 14 && log_n <= 16) {
        if (ept == 16)
            return log_n == 14 ? cluster_capacity<1, 16>() : log_n == 15 ? cluster_capacity<2, 16>()
                                                                          : cluster_capacity<3, 16>();
        return log_n == 14 ? cluster_capacity<1>() : log_n == 15 ? cluster_capacity<2>() : cluster_capacity<3>();
    }
    if (log_n < 10 || log_n > 13) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const uint32_t qn = 1u << log_n;
    const size_t smem = 3ull * (qn + qn / 16) * sizeof(u64);
    cudaError_t e = cudaSuccess;
    if (ept == 16) {
        switch (log_n) {
        case 10: e = occupancy_of(ks_fused_kernel<10, 0, true, 16>, qn / 16, smem, &per); break;
        case 11: e = occupancy_of(ks_fused_kernel<11, 0, true, 16>, qn / 16, smem, &per); break;
        case 12: e = occupancy_of(ks_fused_kernel<12, 0, true, 16>, qn / 16, smem, &per); break;
        default: e = occupancy_of(ks_fused_kernel<13, 0, true, 16>, qn / 16, smem, &per); break;
        }
    } else {
        switch (log_n) {
        case 10: e = occupancy_of(ks_fused_kernel<10, 0, true, 8>, qn / 8, smem, &per); break;
        case 11: e = occupancy_of(ks_fused_kernel<11, 0, true, 8>, qn / 8, smem, &per); break;
        case 12: e = occupancy_of(ks_fused_kernel<12, 0, true, 8>, qn / 8, smem, &per); break;
        default: e = occupancy_of(ks_fused_kernel<13, 0, true, 8>, qn / 8, smem, &per); break;
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per * sms;
}

}  // namespace

// The occupancy queries behind the capacity cost tens of microseconds, and
// the options that consult them are set around every batched operator, so the
// answers are kept per (device, N, values per thread, slice).
int key_switch_fused_capacity(int log_n, int ept, int slice) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const auto key = std::make_tuple(dev, log_n, ept, slice);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    const int cap = capacity_uncached(log_n, ept, slice);
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = cap;
    return cap;
}

bool key_switch_fused_supported(int log_n) {
    if (log_n >= 10 && log_n <= 13) return true;
    return log_n <= 16 && key_switch_fused_capacity(log_n, 8, 13) > 0;
}

size_t ks_fused_scratch_words(uint32_t n, uint32_t sizeQl, uint32_t K) { return (size_t)n * (sizeQl + 2 * K); }

cudaError_t launch_key_prep(const u64* key, ulonglong2* prep, const PrimeConst* pc, uint32_t n, uint32_t S, u64 words,
                            cudaStream_t st) {
    if (words == 0) return cudaSuccess;
    u64 blocks = (words + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    key_prep_kernel<<<(unsigned)blocks, 256, 0, st>>>(key, prep, pc, n, S, words);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_key_switch_fused(int log_n, const OpTabs& t, uint32_t sizeQl, uint32_t K, const u64* key, u64 evk_a,
                                    u64 evk_b, uint32_t key_stride, uint32_t key_pbase, u64* arena, u64* scratch,
                                    uint32_t nz, const ZBases& zb, cudaStream_t st, const KsFuse* fuse,
                                    const ulonglong2* prep, const OpTabs* lvtabs, const ZField* lvz, int ept,
                                    int slice) {
    if (nz == 0) return cudaSuccess;
    KsFusedArgs a{};
    a.t = t;
    a.sizeQl = sizeQl;
    a.K = K;
    a.key = key;
    a.evk_a = evk_a;
    a.evk_b = evk_b;
    a.key_stride = key_stride;
    a.key_pbase = key_pbase;
    a.arena = arena;
    a.scratch = scratch;
    a.in = zb.src;
    a.out0 = zb.out;
    a.out1 = zb.aux;
    a.mid = zb.mid;
    if (fuse) a.f = *fuse;
    a.prep = prep;
    a.prep_b = evk_b - evk_a;
    if (lvtabs && lvz) {
        a.lvtabs = lvtabs;
        a.lvz = *lvz;
    }
    switch (log_n) {
    case 10: return launch_fused<10, 0>(a, nz, st, ept);
    case 11: return launch_fused<11, 0>(a, nz, st, ept);
    case 12: return launch_fused<12, 0>(a, nz, st, ept);
    case 13: return launch_fused<13, 0>(a, nz, st, ept);
    case 14: return slice == 12 ? launch_slice12<2>(a, nz, st, ept) : launch_fused<kLogQ, 1>(a, nz, st, ept);
    case 15: return slice == 12 ? launch_slice12<3>(a, nz, st, ept) : launch_fused<kLogQ, 2>(a, nz, st, ept);
    case 16: return launch_fused<kLogQ, 3>(a, nz, st, ept);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace afhe
