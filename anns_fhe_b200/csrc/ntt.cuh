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

// One table set: primes [0, count) with twiddles for each.
struct PrimeTables {
    const PrimeConst* pc;   // [count]
    const u64* tw;          // [count][N]
    const u64* tw_sh;
    const u64* itw;
    const u64* itw_sh;
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

constexpr int ZMAX = 128;  // polynomials per launch (blockIdx.z)

// Per-z word offsets of the operands of one launch (kernel parameter). The
// meaning of src / out / aux is the prologue's and epilogue's; mid is where a
// limb lives between the passes of a two-pass transform (in the `mid` arena).
struct ZBases {
    u64 src[ZMAX];
    u64 mid[ZMAX];
    u64 out[ZMAX];
    u64 aux[ZMAX];
};

// Plain prologue / epilogue.
struct LoadPlain {
    const u64* base;
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst&) const {
        return base[zb.src[z] + j.src + x];
    }
};
struct StorePlain {
    u64* base;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst&) const {
        base[zb.out[z] + j.out + x] = v;
    }
};

__device__ __forceinline__ uint32_t ins_bits(uint32_t rest, int rb, int k, uint32_t j) {
    uint32_t lo = rest & ((1u << rb) - 1u);
    uint32_t hi = rest >> rb;
    return (hi << (rb + k)) | (j << rb) | lo;
}

// Forward (CT) butterfly, lazy [0, 4q).
__device__ __forceinline__ void ct_bfly(u64& x, u64& y, u64 w, u64 wsh, u64 q, u64 q2) {
    u64 a = x >= q2 ? x - q2 : x;
    u64 t = mul_shoup_lazy(y, w, wsh, q);
    x = a + t;
    y = a - t + q2;
}

// Inverse (GS) butterfly, lazy [0, 2q).
__device__ __forceinline__ void gs_bfly(u64& x, u64& y, u64 w, u64 wsh, u64 q, u64 q2) {
    u64 u = x + y;
    u64 v = x - y + q2;
    x = u >= q2 ? u - q2 : u;
    y = mul_shoup_lazy(v, w, wsh, q);
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

template <bool INV, class Pro, class Epi>
__global__ void __launch_bounds__(1024) ntt_pass_kernel(NttGeom g, PrimeTables pt, const LimbJob* __restrict__ jobs,
                                                        u64* __restrict__ mid, const __grid_constant__ ZBases zb,
                                                        Pro pro, Epi epi) {
    extern __shared__ u64 sm[];
    const LimbJob job = jobs[blockIdx.y];
    const uint32_t z = blockIdx.z;
    const u64 zm = zb.mid[z];
    const PrimeConst pc = pt.pc[job.prime];
    const u64 q = pc.q, q2 = q << 1;
    const uint32_t n = 1u << g.log_n;
    const u64* __restrict__ tw = (INV ? pt.itw : pt.tw) + (u64)job.prime * n;
    const u64* __restrict__ twsh = (INV ? pt.itw_sh : pt.tw_sh) + (u64)job.prime * n;

    const int P = g.P, logc = g.log_c;
    const uint32_t C = 1u << logc;
    const uint32_t tile = 1u << (P + logc);
    const uint32_t T = blockDim.x;
    const bool chunk = (g.lo_bit == 0);
    const uint32_t tile0 = blockIdx.x << logc;   // first chunk (chunk mode) or column (column mode)

    // local index e -> global coefficient index
    auto gidx = [&](uint32_t e) -> uint32_t {
        if (chunk) return (tile0 << P) + e;
        uint32_t b = e >> logc, c = e & (C - 1u);
        return (b << g.lo_bit) + tile0 + c;
    };

    // ---- load tile ----
    for (uint32_t e = threadIdx.x; e < tile; e += T) {
        uint32_t x = gidx(e);
        u64 v;
        if (g.first) v = pro(job, zb, z, x, pc);
        else v = mid[zm + job.dst + x];
        sm[e] = v;
    }
    __syncthreads();

    // ---- rounds of up to 3 stages ----
    const int nrounds = (P + 2) / 3;
    for (int rd = 0; rd < nrounds; ++rd) {
        int rb, k;
        if (!INV) {  // forward: high bits first
            int hi = P - 3 * rd;
            k = hi >= 3 ? 3 : hi;
            rb = hi - k;
        } else {     // inverse: low bits first
            rb = 3 * rd;
            k = (P - rb) >= 3 ? 3 : (P - rb);
        }
        const uint32_t groups = 8u >> k;
        const uint32_t nk = 1u << k;
        for (uint32_t gi = 0; gi < groups; ++gi) {
            uint32_t r = threadIdx.x + gi * T;
            uint32_t c, brest;
            if (chunk) { brest = r & ((1u << (P - k)) - 1u); c = r >> (P - k); }
            else { c = r & (C - 1u); brest = r >> logc; }
            uint32_t hb = chunk ? (tile0 + c) : 0u;   // index bits above the pass
            u64 v[8];
            uint32_t bj[8];
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                if (j < nk) {
                    bj[j] = ins_bits(brest, rb, k, j);
                    uint32_t e = chunk ? ((c << P) | bj[j]) : ((bj[j] << logc) | c);
                    v[j] = sm[e];
                }
            }
            if (!INV) {
#pragma unroll
                for (int s = 2; s >= 0; --s) {
                    if (s >= k) continue;
                    const int pb = rb + s;             // bit within pass
                    const int p = g.lo_bit + pb;       // global bit
#pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) {
                        if (j >= nk || (j >> s) & 1u) continue;
                        uint32_t idx = (1u << (g.log_n - 1 - p)) + ((hb << (P - pb - 1)) | (bj[j] >> (pb + 1)));
                        ct_bfly(v[j], v[j | (1u << s)], __ldg(tw + idx), __ldg(twsh + idx), q, q2);
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < 3; ++s) {
                    if (s >= k) continue;
                    const int pb = rb + s;
                    const int p = g.lo_bit + pb;
                    const bool fuse_last = g.last && (p == g.log_n - 1);
#pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) {
                        if (j >= nk || (j >> s) & 1u) continue;
                        if (fuse_last) {
                            gs_bfly_last(v[j], v[j | (1u << s)], pc, q2);
                        } else {
                            uint32_t idx = (1u << (g.log_n - 1 - p)) + ((hb << (P - pb - 1)) | (bj[j] >> (pb + 1)));
                            gs_bfly(v[j], v[j | (1u << s)], __ldg(tw + idx), __ldg(twsh + idx), q, q2);
                        }
                    }
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                if (j < nk) {
                    uint32_t e = chunk ? ((c << P) | bj[j]) : ((bj[j] << logc) | c);
                    sm[e] = v[j];
                }
            }
        }
        __syncthreads();
    }

    // ---- store tile ----
    for (uint32_t e = threadIdx.x; e < tile; e += T) {
        uint32_t x = gidx(e);
        u64 v = sm[e];
        if (g.last) {
            if (!INV) v = canon4(v, q);
            epi(job, zb, z, x, v, pc);
        } else {
            mid[zm + job.dst + x] = v;
        }
    }
}

// Pass plan for a transform of size 2^log_n.
struct NttPlan {
    int npass;
    NttGeom g[2];
};

inline NttPlan make_plan(int log_n, bool inverse) {
    NttPlan pl;
    if (log_n <= 13) {   // whole limb in shared memory (<= 64 KB), N / 8 threads
        pl.npass = 1;
        NttGeom a{};
        a.log_n = log_n; a.lo_bit = 0; a.P = log_n; a.log_c = 0; a.first = 1; a.last = 1;
        pl.g[0] = a;
        return pl;
    }
    int pa = (log_n + 1) / 2;     // high (column) pass bits
    int pb = log_n - pa;          // low (chunk) pass bits
    NttGeom col{}, chk{};
    col.log_n = log_n; col.lo_bit = pb; col.P = pa; col.log_c = 12 - pa < 4 ? 12 - pa : 4;
    if (col.log_c < 0) col.log_c = 0;
    chk.log_n = log_n; chk.lo_bit = 0; chk.P = pb; chk.log_c = 12 - pb;
    pl.npass = 2;
    if (!inverse) { pl.g[0] = col; pl.g[1] = chk; }
    else { pl.g[0] = chk; pl.g[1] = col; }
    pl.g[0].first = 1; pl.g[0].last = 0;
    pl.g[1].first = 0; pl.g[1].last = 1;
    return pl;
}

// Launch a full transform over `njobs` limbs x `nz` polynomials. Between
// passes limb `job` of polynomial z lives at mid + zb.mid[z] + job.dst.
template <bool INV, class Pro, class Epi>
inline cudaError_t launch_ntt(int log_n, const PrimeTables& pt, const LimbJob* jobs, uint32_t njobs, uint32_t nz,
                              u64* mid, const ZBases& zb, Pro pro, Epi epi, cudaStream_t st) {
    if (njobs == 0 || nz == 0) return cudaSuccess;
    NttPlan pl = make_plan(log_n, INV);
    for (int i = 0; i < pl.npass; ++i) {
        NttGeom g = pl.g[i];
        uint32_t tile = 1u << (g.P + g.log_c);
        uint32_t threads = tile / 8;
        uint32_t ctas = 1u << (log_n - g.P - g.log_c);
        dim3 grid(ctas, njobs, nz);
        size_t smem = (size_t)tile * sizeof(u64);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(ntt_pass_kernel<INV, Pro, Epi>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        ntt_pass_kernel<INV, Pro, Epi><<<grid, threads, smem, st>>>(g, pt, jobs, mid, zb, pro, epi);
        count_launches(1);
    }
    return cudaGetLastError();
}

}  // namespace afhe
