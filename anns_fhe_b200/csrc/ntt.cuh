// ntt.cuh -- negacyclic NTT / INTT passes for sm_100a.
//
// Computes exactly the transforms of hardware_fpga_model/hls/src/ntt.cpp:
//   forward (ntt.cpp:4-43): Cooley-Tukey, stage with block size t = 2^p uses
//     twiddle tw[N/2^(p+1) + (x >> (p+1))]; natural order in, bit-reversed out;
//   inverse (ntt.cpp:46-80): Gentleman-Sande with itw[...] on the same index,
//     stages in the opposite order, then x N^-1 (fused into the last stage here).
// Every butterfly is an exact operation mod q, so with the same twiddle tables
// the canonical outputs are bit-identical to the reference's.
//
// Layout: a limb is N contiguous uint64 words (limb-major ciphertexts). A
// transform is 1 or 2 passes; a pass covers the butterfly bits
// [lo_bit, lo_bit + P) of the coefficient index:
//   * column pass (lo_bit > 0): a CTA owns 2^logC adjacent low-index columns of
//     the 2^P rows, i.e. 2^P row segments of 2^logC * 8 bytes (coalesced);
//   * chunk pass (lo_bit == 0): a CTA owns 2^logC contiguous chunks of 2^P words.
// The tile (2^(P+logC) words) is staged in shared memory; the butterflies run
// in rounds of up to three consecutive stages on eight values held in
// registers (radix-8), with one shared-memory exchange per round.
// Values between stages are lazily reduced: forward in [0, 4q) (Harvey), inverse
// in [0, 2q); the last pass canonicalises before its epilogue.
#pragma once
#include <cstdint>
#include "modarith.cuh"

namespace afhe {

// Host-side count of kernels this library has launched (all contexts).
void count_launches(uint64_t k);

// Per-prime constants (64 bytes).
struct PrimeConst {
    u64 q;
    u64 ninv, ninv_sh;        // N^-1 mod q and its Shoup companion
    u64 w1ninv, w1ninv_sh;    // itw[1] * N^-1 (fused last inverse stage)
    u64 r64, r64_sh, one_sh;  // reduce128 constants
};

// One table set: primes [0, count) with twiddles for each. Twiddles are
// stored as (w, Shoup companion of w) pairs, one 16-byte load per twiddle.
struct PrimeTables {
    const PrimeConst* pc;    // [count]
    const ulonglong2* tw2;   // [count][N] forward  (psi^bitrev(j), companion)
    const ulonglong2* itw2;  // [count][N] inverse
};

AFHE_HD ModConst modconst_of(const PrimeConst& p) {
    ModConst m;
    m.q = p.q; m.r64 = p.r64; m.r64_sh = p.r64_sh; m.one_sh = p.one_sh;
    return m;
}

// A unit of NTT work: one limb. Word offsets: `src` is read by the prologue,
// `dst` holds the limb between passes (relative to the `mid` base), `out` is
// written by the epilogue; `prime` indexes the table set; `aux` is free for
// prologue / epilogue functors (e.g. a digit or output-limb index).
struct LimbJob {
    u64 src;
    u64 dst;
    u64 out;
    uint32_t prime;
    uint32_t aux;
};

struct NttGeom {
    int log_n;
    int lo_bit;   // first butterfly bit of this pass
    int P;        // number of butterfly bits in this pass
    int log_c;    // log2 of tiles per CTA
    int first;    // pass reads through the prologue
    int last;     // pass writes through the epilogue
};

// Word offset of one operand for polynomial z of a batched launch:
//   (arr ? arr[z >> shift] : base + (z >> shift) * stride) + add + (z & low) * hdelta,
// low = 2^shift - 1. A regular batch (operands at a fixed stride) needs no
// memory; an irregular one reads a small device array. shift = 1 describes the
// two polynomials (c0, c1) of ciphertext z >> 1 that differ by hdelta.
struct ZField {
    const u64* arr;
    u64 base, stride, add, hdelta;
    uint32_t shift;
    AFHE_HD u64 at(uint32_t z) const {
        const uint32_t zz = z >> shift;
        const u64 v = arr ? arr[zz] : base + (u64)zz * stride;
        return v + add + (u64)(z & ((1u << shift) - 1u)) * hdelta;
    }
};

inline ZField zf_const(u64 v) { ZField f{}; f.base = v; return f; }
inline ZField zf_stride(u64 base, u64 stride) { ZField f{}; f.base = base; f.stride = stride; return f; }
inline ZField zf_plus(ZField f, u64 add) { f.add += add; return f; }
inline ZField zf_pair(ZField f, u64 hdelta) { f.shift = 1; f.hdelta = hdelta; return f; }

// The operands of one batched launch: meaning of src / out / aux is the
// prologue's and epilogue's; mid is where a limb lives between the passes of
// a two-pass transform (in the `mid` arena).
struct ZBases {
    ZField src, mid, out, aux;
};

// Plain prologue / epilogue.
struct LoadPlain {
    const u64* base;
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst&) const {
        return base[zb.src.at(z) + j.src + x];
    }
};
struct StorePlain {
    u64* base;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst&) const {
        base[zb.out.at(z) + j.out + x] = v;
    }
};

// Forward (CT) butterfly, lazy [0, 4q).
__device__ __forceinline__ void ct_bfly(u64& x, u64& y, ulonglong2 w, u64 q, u64 q2) {
    u64 a = x >= q2 ? x - q2 : x;
    u64 t = mul_shoup_lazy(y, w.x, w.y, q);
    x = a + t;
    y = a - t + q2;
}

// Inverse (GS) butterfly, lazy [0, 2q).
__device__ __forceinline__ void gs_bfly(u64& x, u64& y, ulonglong2 w, u64 q, u64 q2) {
    u64 u = x + y;
    u64 v = x - y + q2;
    x = u >= q2 ? u - q2 : u;
    y = mul_shoup_lazy(v, w.x, w.y, q);
}

// Last inverse stage with N^-1 folded in; outputs canonical.
__device__ __forceinline__ void gs_bfly_last(u64& x, u64& y, const PrimeConst& pc, u64 q2) {
    u64 u = x + y;
    u64 v = x - y + q2;
    x = csub(mul_shoup_lazy(u, pc.ninv, pc.ninv_sh, pc.q), pc.q);
    y = csub(mul_shoup_lazy(v, pc.w1ninv, pc.w1ninv_sh, pc.q), pc.q);
}

__device__ __forceinline__ u64 canon4(u64 v, u64 q) {
    u64 q2 = q << 1;
    v = v >= q2 ? v - q2 : v;
    return v >= q ? v - q : v;
}

// Shared-memory layout: one pad word per 16 words, so the strided patterns of
// every round (8-byte elements, strides 1, 2, 8, 16, 64, ...) hit distinct banks.
__device__ __forceinline__ uint32_t padix(uint32_t e) { return e + (e >> 4); }

// One round: K consecutive stages on bits [RB, RB + K) of the pass index.
// Each of the TILE / EPT threads holds EPT values per round, as EPT / 2^K
// groups of 2^K; all shapes are compile-time.
template <bool INV, int P, int LOGC, bool COL, int RB, int K, int EPT>
struct NttRound {
    static constexpr uint32_t C = 1u << LOGC;
    static constexpr uint32_t T = (1u << (P + LOGC)) / EPT;
    static constexpr uint32_t NK = 1u << K;
    static constexpr uint32_t GROUPS = EPT >> K;
    static constexpr uint32_t STEP_E = COL ? (1u << (RB + LOGC)) : (1u << RB);

    // slot of twiddle m of stage s among a group's NK - 1 twiddles
    __device__ static constexpr uint32_t slot(int s, uint32_t m) { return (NK >> (s + 1)) - 1 + m; }

    // Rounds over NB buffers of the same prime at once: each group's
    // twiddles and addresses are computed once and applied to every buffer.
    template <int NB>
    __device__ __forceinline__ static void run_n(u64* const (&sms)[NB], const ulonglong2* __restrict__ tw,
                                                 const PrimeConst& pc, uint32_t tile0, int log_n, int lo_bit,
                                                 bool last_pass) {
        const u64 q = pc.q, q2 = q << 1;
#pragma unroll
        for (uint32_t gi = 0; gi < GROUPS; ++gi) {
            const uint32_t r = threadIdx.x + gi * T;
            uint32_t c, brest;
            if (COL) { c = r & (C - 1u); brest = r >> LOGC; }
            else { brest = r & ((1u << (P - K)) - 1u); c = r >> (P - K); }
            const uint32_t base_b = ((brest >> RB) << (RB + K)) | (brest & ((1u << RB) - 1u));
            const uint32_t base_e = COL ? ((base_b << LOGC) | c) : ((c << P) | base_b);
            const uint32_t hb = COL ? 0u : (tile0 + c);   // index bits above the pass
            // the group's twiddles, issued before its values are read
            ulonglong2 w[NK - 1];
#pragma unroll
            for (int s = 0; s < K; ++s) {
                const int pb = RB + s;
                const int p = lo_bit + pb;
                if (INV && last_pass && p == log_n - 1) continue;   // N^-1 stage: constants, no table
                const uint32_t tb = (1u << (log_n - 1 - p)) + (hb << (P - pb - 1)) + (base_b >> (pb + 1));
#pragma unroll
                for (uint32_t m = 0; m < (NK >> (s + 1)); ++m) w[slot(s, m)] = __ldg(tw + tb + m);
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                // base_e has zeros where j * STEP_E has ones, so
                // padix(base_e + j * STEP_E) = padix(base_e) + padix(j * STEP_E):
                // one address per group, compile-time offsets per element
                u64* const sp = sms[b] + padix(base_e);
                u64 v[NK];
#pragma unroll
                for (uint32_t j = 0; j < NK; ++j) v[j] = sp[padix(j * STEP_E)];
                if (!INV) {
#pragma unroll
                    for (int s = K - 1; s >= 0; --s) {
#pragma unroll
                        for (uint32_t m = 0; m < (NK >> (s + 1)); ++m) {
                            const ulonglong2 ww = w[slot(s, m)];
#pragma unroll
                            for (uint32_t jj = 0; jj < (1u << s); ++jj) {
                                const uint32_t j = (m << (s + 1)) | jj;
                                ct_bfly(v[j], v[j + (1u << s)], ww, q, q2);
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int s = 0; s < K; ++s) {
                        const int p = lo_bit + RB + s;
                        if (last_pass && p == log_n - 1) {
#pragma unroll
                            for (uint32_t j = 0; j < (NK >> 1); ++j) gs_bfly_last(v[j], v[j + (NK >> 1)], pc, q2);
                        } else {
#pragma unroll
                            for (uint32_t m = 0; m < (NK >> (s + 1)); ++m) {
                                const ulonglong2 ww = w[slot(s, m)];
#pragma unroll
                                for (uint32_t jj = 0; jj < (1u << s); ++jj) {
                                    const uint32_t j = (m << (s + 1)) | jj;
                                    gs_bfly(v[j], v[j + (1u << s)], ww, q, q2);
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (uint32_t j = 0; j < NK; ++j) sp[padix(j * STEP_E)] = v[j];
            }
        }
    }
};

// All rounds of a pass over NB tiles in shared memory (same prime), each
// round followed by a barrier: forward takes bits high to low, inverse low to
// high, in rounds of R bits (radix 2^R: R = 3, or 4 with 16 values per
// thread; the remainder round is smaller).
template <bool INV, int P, int LOGC, bool COL, int RD, int EPT, int NB, int R = 3>
__device__ __forceinline__ void ntt_rounds_n(u64* const (&sms)[NB], const ulonglong2* tw, const PrimeConst& pc,
                                             uint32_t tile0, int log_n, int lo_bit, bool last_pass) {
    static_assert((EPT >> R) >= 1, "a round needs 2^R values per thread");
    constexpr int NR = (P + R - 1) / R;
    if constexpr (RD < NR) {
        constexpr int HI = P - R * RD;                       // forward: bits [.., HI)
        constexpr int KF = HI >= R ? R : HI;
        constexpr int RBF = HI - KF;
        constexpr int RBI = R * RD;                          // inverse: bits [RBI, ..)
        constexpr int KI = (P - RBI) >= R ? R : (P - RBI);
        NttRound<INV, P, LOGC, COL, INV ? RBI : RBF, INV ? KI : KF, EPT>::template run_n<NB>(
            sms, tw, pc, tile0, log_n, lo_bit, last_pass);
        __syncthreads();
        ntt_rounds_n<INV, P, LOGC, COL, RD + 1, EPT, NB, R>(sms, tw, pc, tile0, log_n, lo_bit, last_pass);
    }
}

// One tile.
template <bool INV, int P, int LOGC, bool COL, int RD, int EPT = 8, int R = 3>
__device__ __forceinline__ void ntt_rounds(u64* sm, const ulonglong2* tw, const PrimeConst& pc, uint32_t tile0,
                                           int log_n, int lo_bit, bool last_pass) {
    u64* const one[1] = {sm};
    ntt_rounds_n<INV, P, LOGC, COL, RD, EPT, 1, R>(one, tw, pc, tile0, log_n, lo_bit, last_pass);
}

// One pass over 2^(P + LOGC)-word tiles: stage the tile in shared memory
// (through the prologue on the first pass), run the rounds, write it back
// (through the epilogue on the last pass, canonical residues). EPT values per
// thread (8 or 16); CTAs of 1024 threads are launched one per SM's register
// budget, smaller ones two.
constexpr uint32_t ntt_threads(int P, int LOGC, int EPT) { return (1u << (P + LOGC)) / EPT; }
constexpr int ntt_min_ctas(int P, int LOGC, int EPT) { return ntt_threads(P, LOGC, EPT) >= 1024 ? 1 : 2; }

template <bool INV, int P, int LOGC, bool COL, int EPT, class Pro, class Epi>
__global__ void __launch_bounds__(ntt_threads(P, LOGC, EPT), ntt_min_ctas(P, LOGC, EPT))
ntt_kernel(NttGeom g, PrimeTables pt, const LimbJob* __restrict__ jobs, u64* __restrict__ mid,
           const ZBases zb, Pro pro, Epi epi) {
    extern __shared__ u64 sm[];
    constexpr uint32_t C = 1u << LOGC;
    constexpr uint32_t TILE = 1u << (P + LOGC);
    constexpr uint32_t T = TILE / EPT;
    const LimbJob job = jobs[blockIdx.y];
    const uint32_t z = blockIdx.z;
    const u64 zm = zb.mid.at(z);
    const PrimeConst pc = pt.pc[job.prime];
    const uint32_t n = 1u << g.log_n;
    const ulonglong2* __restrict__ tw = (INV ? pt.itw2 : pt.tw2) + (u64)job.prime * n;
    const uint32_t tile0 = blockIdx.x << LOGC;

    auto gidx = [&](uint32_t e) -> uint32_t {
        if (!COL) return (tile0 << P) + e;
        const uint32_t b = e >> LOGC, c = e & (C - 1u);
        return (b << g.lo_bit) + tile0 + c;
    };

#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < TILE; e += T) {
        const uint32_t x = gidx(e);
        sm[padix(e)] = g.first ? pro(job, zb, z, x, pc) : mid[zm + job.dst + x];
    }
    __syncthreads();
    ntt_rounds<INV, P, LOGC, COL, 0, EPT>(sm, tw, pc, tile0, g.log_n, g.lo_bit, g.last != 0);
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < TILE; e += T) {
        const uint32_t x = gidx(e);
        u64 v = sm[padix(e)];
        if (g.last) {
            if (!INV) v = canon4(v, pc.q);
            epi(job, zb, z, x, v, pc);
        } else {
            mid[zm + job.dst + x] = v;
        }
    }
}

// Tile shapes of a transform ("plans"), chosen per ring degree at run time
// (afhe_ntt_set_plan; the autotuner times them). Every plan computes the
// same butterflies on the same values, so the residues do not depend on it.
//   N <= 2^13, one pass over the whole limb: plan 0 the default values per
//     thread (16 for 8192-word limbs, else 8), plan 1 the other choice;
//   N >= 2^14, two passes (high bits in columns, then low bits in chunks):
//     plan = 3 * t + c: columns per CTA 2^{4, 3, 5}[c] in the column pass,
//     chunk-pass tiles of 2^{12, 13}[t] words. Plan 0 is 16 columns and
//     4096-word tiles.
// Values per thread in a two-pass transform: 16 for 8192-word tiles, else 8.
constexpr int kNttPlansOnePass = 2;
constexpr int kNttPlansTwoPass = 6;
inline int ntt_plan_count(int log_n) {
    return log_n < 10 || log_n > 16 ? 0 : (log_n <= 13 ? kNttPlansOnePass : kNttPlansTwoPass);
}
// the plan in force per log_n, process-wide (kernels.cu)
int ntt_plan(int log_n);
void set_ntt_plan(int log_n, int plan);

struct NttPlan {
    int npass;
    int ept[2];
    NttGeom g[2];
};

inline NttPlan make_plan(int log_n, bool inverse, int plan) {
    NttPlan pl;
    if (log_n <= 13) {   // whole limb in shared memory (<= 68 KB)
        pl.npass = 1;
        NttGeom a{};
        a.log_n = log_n; a.lo_bit = 0; a.P = log_n; a.log_c = 0; a.first = 1; a.last = 1;
        pl.g[0] = a;
        const int def = log_n >= 13 ? 16 : 8;
        pl.ept[0] = plan == 1 ? 24 - def : def;
        return pl;
    }
    static const int col_c[3] = {4, 3, 5};
    const int c = col_c[plan % 3], tl = 12 + plan / 3;
    int pa = (log_n + 1) / 2;     // high (column) pass bits
    int pb = log_n - pa;          // low (chunk) pass bits
    NttGeom col{}, chk{};
    col.log_n = log_n; col.lo_bit = pb; col.P = pa; col.log_c = c;
    chk.log_n = log_n; chk.lo_bit = 0; chk.P = pb; chk.log_c = tl - pb;
    const int ept_col = pa + c >= 13 ? 16 : 8, ept_chk = tl >= 13 ? 16 : 8;
    pl.npass = 2;
    if (!inverse) { pl.g[0] = col; pl.g[1] = chk; pl.ept[0] = ept_col; pl.ept[1] = ept_chk; }
    else { pl.g[0] = chk; pl.g[1] = col; pl.ept[0] = ept_chk; pl.ept[1] = ept_col; }
    pl.g[0].first = 1; pl.g[0].last = 0;
    pl.g[1].first = 0; pl.g[1].last = 1;
    return pl;
}

template <bool INV, int P, int LOGC, bool COL, int EPT, class Pro, class Epi>
inline cudaError_t launch_pass(const NttGeom& g, const PrimeTables& pt, const LimbJob* jobs, uint32_t njobs,
                               uint32_t nz, u64* mid, const ZBases& zb, const Pro& pro, const Epi& epi,
                               cudaStream_t st) {
    constexpr uint32_t TILE = 1u << (P + LOGC);
    const uint32_t ctas = 1u << (g.log_n - P - LOGC);
    const size_t smem = (size_t)(TILE + TILE / 16) * sizeof(u64);
    auto kern = ntt_kernel<INV, P, LOGC, COL, EPT, Pro, Epi>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<dim3(ctas, njobs, nz), ntt_threads(P, LOGC, EPT), smem, st>>>(g, pt, jobs, mid, zb, pro, epi);
    count_launches(1);
    return cudaSuccess;
}

// The pass with geometry g and EPT values per thread, dispatched to its
// compile-time instance (every shape some plan uses).
template <bool INV, class Pro, class Epi>
inline cudaError_t launch_shape(const NttGeom& g, int ept, const PrimeTables& pt, const LimbJob* jobs,
                                uint32_t njobs, uint32_t nz, u64* mid, const ZBases& zb, const Pro& pro,
                                const Epi& epi, cudaStream_t st) {
#define AFHE_NTT_SHAPE(P_, C_, COL_, EPT_)                                                                  \
    if (g.P == P_ && g.log_c == C_ && (g.lo_bit > 0) == COL_ && ept == EPT_)                                \
        return launch_pass<INV, P_, C_, COL_, EPT_>(g, pt, jobs, njobs, nz, mid, zb, pro, epi, st);
    // one pass
    AFHE_NTT_SHAPE(10, 0, false, 8) AFHE_NTT_SHAPE(10, 0, false, 16)
    AFHE_NTT_SHAPE(11, 0, false, 8) AFHE_NTT_SHAPE(11, 0, false, 16)
    AFHE_NTT_SHAPE(12, 0, false, 8) AFHE_NTT_SHAPE(12, 0, false, 16)
    AFHE_NTT_SHAPE(13, 0, false, 8) AFHE_NTT_SHAPE(13, 0, false, 16)
    // column passes: 2^7 (N = 2^14) or 2^8 (2^15, 2^16) bits, 8 / 16 / 32 columns
    AFHE_NTT_SHAPE(7, 3, true, 8) AFHE_NTT_SHAPE(7, 4, true, 8) AFHE_NTT_SHAPE(7, 5, true, 8)
    AFHE_NTT_SHAPE(8, 3, true, 8) AFHE_NTT_SHAPE(8, 4, true, 8) AFHE_NTT_SHAPE(8, 5, true, 16)
    // chunk passes: 4096- or 8192-word tiles
    AFHE_NTT_SHAPE(7, 5, false, 8) AFHE_NTT_SHAPE(7, 6, false, 16)
    AFHE_NTT_SHAPE(8, 4, false, 8) AFHE_NTT_SHAPE(8, 5, false, 16)
#undef AFHE_NTT_SHAPE
    return cudaErrorInvalidValue;
}

// Launch a full transform over `njobs` limbs x `nz` polynomials. Between
// passes limb `job` of polynomial z lives at mid + zb.mid[z] + job.dst.
template <bool INV, class Pro, class Epi>
inline cudaError_t launch_ntt(int log_n, const PrimeTables& pt, const LimbJob* jobs, uint32_t njobs, uint32_t nz,
                              u64* mid, const ZBases& zb, Pro pro, Epi epi, cudaStream_t st) {
    if (njobs == 0 || nz == 0) return cudaSuccess;
    NttPlan pl = make_plan(log_n, INV, ntt_plan(log_n));
    for (int i = 0; i < pl.npass; ++i) {
        cudaError_t e = launch_shape<INV>(pl.g[i], pl.ept[i], pt, jobs, njobs, nz, mid, zb, pro, epi, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

}  // namespace afhe
