// kernels.cu -- CUDA kernels and launchers for the CKKS evaluation core.
//
// Reference functions restated here (paths inside iheydardoost/ANNS_FHE):
//   poly_add / poly_sub / poly_mul      hardware_fpga_model/hls/src/poly_arith.cpp:3-38
//   automorphism                        hardware_fpga_model/hls/src/automorphism.cpp:3-12
//   rescale                             hardware_fpga_model/hls/src/rescale.cpp:3-72
//   fast_bases_conv / approx_mod_down   hardware_fpga_model/hls/src/key_switch.cpp:7-163
//   key_switch                          hardware_fpga_model/hls/src/key_switch.cpp:167-439
// Fusion: the base conversions run as the prologue of the NTT that consumes
// them; the rescale combine (a_i * q_l^-1 + NTT(...)) and the ModDown combine
// ((x_Q - y) * P^-1) run as the NTT epilogue; the evaluation-key inner product
// accumulates all digits of a limb in 128-bit registers and reduces once.
#include <atomic>

#include "internal.h"

namespace afhe {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
uint64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

static std::atomic<int> g_ntt_plan[17];
int ntt_plan(int log_n) { return log_n >= 0 && log_n <= 16 ? g_ntt_plan[log_n].load(std::memory_order_relaxed) : 0; }
void set_ntt_plan(int log_n, int plan) { g_ntt_plan[log_n].store(plan, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// elementwise
// ---------------------------------------------------------------------------
template <int OP>
__global__ void __launch_bounds__(256) elementwise_kernel(const PrimeConst* __restrict__ pc, uint32_t prime0,
                                                          u64* __restrict__ arena, uint32_t n, const ZBases zb) {
    const uint32_t l = blockIdx.y, z = blockIdx.z;
    const PrimeConst p = pc[prime0 + l];
    const u64 off = (u64)l * n;
    const u64* a = arena + zb.src.at(z) + off;
    const u64* b = arena + zb.aux.at(z) + off;
    u64* o = arena + zb.out.at(z) + off;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 x = a[i];
        u64 r;
        if (OP == EW_ADD) r = add_mod(x, b[i], p.q);
        else if (OP == EW_SUB) r = sub_mod(x, b[i], p.q);
        else if (OP == EW_MUL) r = mul_mod(x, b[i], modconst_of(p));
        else r = x;
        o[i] = r;
    }
}

cudaError_t launch_elementwise(ElemOp op, const PrimeConst* pc, uint32_t prime0, u64* arena, uint32_t n,
                               uint32_t limbs, uint32_t nz, const ZBases& zb, cudaStream_t st) {
    if (limbs == 0 || nz == 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, limbs, nz);
    switch (op) {
    case EW_ADD: elementwise_kernel<EW_ADD><<<grid, 256, 0, st>>>(pc, prime0, arena, n, zb); break;
    case EW_SUB: elementwise_kernel<EW_SUB><<<grid, 256, 0, st>>>(pc, prime0, arena, n, zb); break;
    case EW_MUL: elementwise_kernel<EW_MUL><<<grid, 256, 0, st>>>(pc, prime0, arena, n, zb); break;
    default: elementwise_kernel<EW_COPY><<<grid, 256, 0, st>>>(pc, prime0, arena, n, zb); break;
    }
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// ciphertext tensor product (fhe_host_driver.cpp:280-286):
//   d0 = a0*b0, d1 = a0*b1 + a1*b0, d2 = a1*b1  (d1 reduced once from 128 bits)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) tensor_kernel(const PrimeConst* __restrict__ pc, u64* __restrict__ arena,
                                                     uint32_t n, const TensorArgs ta) {
    const uint32_t l = blockIdx.y, z = blockIdx.z;
    const ModConst m = modconst_of(pc[l]);
    const u64 off = (u64)l * n;
    const u64* a0 = arena + ta.a0.at(z) + off;
    const u64* a1 = arena + ta.a1.at(z) + off;
    const u64* b0 = arena + ta.b0.at(z) + off;
    const u64* b1 = arena + ta.b1.at(z) + off;
    u64* d0 = arena + ta.d0.at(z) + off;
    u64* d1 = arena + ta.d1.at(z) + off;
    u64* d2 = arena + ta.d2.at(z) + off;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u64 x0 = a0[i], x1 = a1[i], y0 = b0[i], y1 = b1[i];
        Acc128 c;
        acc_init(c);
        acc_mad(c, x0, y1);
        acc_mad(c, x1, y0);
        d0[i] = mul_mod(x0, y0, m);
        d1[i] = acc_reduce(c, m);
        d2[i] = mul_mod(x1, y1, m);
    }
}

cudaError_t launch_tensor(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t nz,
                          const TensorArgs& ta, cudaStream_t st) {
    if (limbs == 0 || nz == 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, limbs, nz);
    tensor_kernel<<<grid, 256, 0, st>>>(pc, arena, n, ta);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// automorphism: out[i] = a[map[i]]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) automorphism_kernel(const uint32_t* __restrict__ map32,
                                                           const u64* __restrict__ map64, u64* __restrict__ arena,
                                                           uint32_t n, const ZBases zb) {
    const uint32_t l = blockIdx.y, z = blockIdx.z;
    const u64 off = (u64)l * n;
    const u64* a = arena + zb.src.at(z) + off;
    u64* o = arena + zb.out.at(z) + off;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t idx;
        if (map32) idx = map32[i];
        else {
            u64 packed = map64[i >> 1];
            idx = (i & 1u) ? (uint32_t)(packed >> 32) : (uint32_t)(packed & 0xFFFFFFFFull);
        }
        o[i] = idx < n ? a[idx] : 0ull;  // out-of-range map entries read nothing
    }
}

cudaError_t launch_automorphism(const uint32_t* map32, const u64* map64, u64* arena, uint32_t n, uint32_t limbs,
                                uint32_t nz, const ZBases& zb, cudaStream_t st) {
    if (limbs == 0 || nz == 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, limbs, nz);
    automorphism_kernel<<<grid, 256, 0, st>>>(map32, map64, arena, n, zb);
    count_launches(1);
    return cudaGetLastError();
}

// Every polynomial of a batch through its own permutation: maps.at(z) is the
// device address of polynomial z's map (N indices, each < N).
__global__ void __launch_bounds__(256) automorphism_z_kernel(const ZField maps, u64* __restrict__ arena, uint32_t n,
                                                            const ZBases zb) {
    const uint32_t l = blockIdx.y, z = blockIdx.z;
    const uint32_t* __restrict__ map = (const uint32_t*)maps.at(z);
    const u64 off = (u64)l * n;
    const u64* a = arena + zb.src.at(z) + off;
    u64* o = arena + zb.out.at(z) + off;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = a[__ldg(map + i)];
}

cudaError_t launch_automorphism_z(const ZField& maps, u64* arena, uint32_t n, uint32_t limbs, uint32_t nz,
                                  const ZBases& zb, cudaStream_t st) {
    if (limbs == 0 || nz == 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, limbs, nz);
    automorphism_z_kernel<<<grid, 256, 0, st>>>(maps, arena, n, zb);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// sums of plaintext-ciphertext products, each plaintext read through its own
// automorphism (the inner products of the diagonal method: a plaintext moved
// by a slot rotation is a permutation of its evaluation-form coefficients)
// ---------------------------------------------------------------------------
AFHE_HD void acc_fold(Acc128& a, const ModConst& m) {
    a.lo = acc_reduce(a, m);
    a.hi = 0;
}

__global__ void __launch_bounds__(256) mac_plain_kernel(const PrimeConst* __restrict__ pc, u64* __restrict__ arena,
                                                        uint32_t n, const MacJob* __restrict__ jobs,
                                                        const MacGroup* __restrict__ groups,
                                                        const MacTerm* __restrict__ terms, uint32_t reduce_every,
                                                        int accumulate) {
    const uint32_t l = blockIdx.y;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MacJob J = jobs[blockIdx.z];
    const ModConst m = modconst_of(pc[l]);
    const u64 off = (u64)l * n + i;
    Acc128 a0, a1;
    acc_init(a0);
    acc_init(a1);
    uint32_t cnt = 0;
    for (uint32_t g = J.g0; g < J.g1; ++g) {
        const MacGroup G = groups[g];
        const bool unit = G.src0 == kMacUnit;
        const u64 x0 = unit ? 1 : arena[G.src0 + off];
        const u64 x1 = unit ? 0 : arena[G.src1 + off];
        for (uint32_t t = G.t0; t < G.t1; ++t) {
            const MacTerm T = terms[t];
            const uint32_t j = T.map ? __ldg(T.map + i) : i;
            const u64 p = arena[T.pt + (u64)l * n + j];
            acc_mad(a0, p, x0);
            if (!unit) acc_mad(a1, p, x1);
            if (++cnt == reduce_every) {
                acc_fold(a0, m);
                acc_fold(a1, m);
                cnt = 1;
            }
        }
    }
    u64 r0 = acc_reduce(a0, m), r1 = acc_reduce(a1, m);
    if (accumulate) {
        r0 = add_mod(r0, arena[J.out0 + off], m.q);
        r1 = add_mod(r1, arena[J.out1 + off], m.q);
    }
    arena[J.out0 + off] = r0;
    arena[J.out1 + off] = r1;
}

// One coefficient per thread: the nb baby-step ciphertexts' coefficients stay
// in registers while the job's units stream through; a unit's automorphism
// index is loaded once for its nb plaintexts, which lie `stride` words apart.
template <int NB>
__global__ void __launch_bounds__(256) diag_inner_kernel(const PrimeConst* __restrict__ pc, u64* __restrict__ arena,
                                                         uint32_t n, const DiagJob* __restrict__ jobs,
                                                         const u64* __restrict__ srcs,
                                                         const DiagUnit* __restrict__ units, u64 stride,
                                                         uint32_t reduce_every, int accumulate) {
    const uint32_t l = blockIdx.y;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DiagJob J = jobs[blockIdx.z];
    const ModConst m = modconst_of(pc[l]);
    const u64 off = (u64)l * n;
    const u64* s = srcs + (u64)blockIdx.z * 2 * NB;
    u64 x0[NB], x1[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        x0[b] = arena[s[2 * b] + off + i];
        x1[b] = arena[s[2 * b + 1] + off + i];
    }
    Acc128 a0, a1;
    acc_init(a0);
    acc_init(a1);
    uint32_t cnt = 0;
    // the next unit's descriptor and automorphism index are loaded while the
    // current unit's plaintexts are read and multiplied
    DiagUnit Un{};
    uint32_t jn = i;
    if (J.u0 < J.u1) {
        Un = units[J.u0];
        jn = Un.map ? __ldg(Un.map + i) : i;
    }
    for (uint32_t k = J.u0; k < J.u1; ++k) {
        const u64* p = arena + Un.pt + off + jn;
        if (k + 1 < J.u1) {
            Un = units[k + 1];
            jn = Un.map ? __ldg(Un.map + i) : i;
        }
        if (cnt + NB > reduce_every) {
            acc_fold(a0, m);
            acc_fold(a1, m);
            cnt = 1;
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const u64 v = p[(u64)b * stride];
            acc_mad(a0, v, x0[b]);
            acc_mad(a1, v, x1[b]);
        }
        cnt += NB;
    }
    u64 r0 = acc_reduce(a0, m), r1 = acc_reduce(a1, m);
    if (accumulate) {
        r0 = add_mod(r0, arena[J.out0 + off + i], m.q);
        r1 = add_mod(r1, arena[J.out1 + off + i], m.q);
    }
    arena[J.out0 + off + i] = r0;
    arena[J.out1 + off + i] = r1;
}

// The same sums with the plaintexts staged through shared memory: every
// placement map of the launch keeps each 256-coefficient tile within itself
// (a slot rotation by a multiple of D permutes the evaluation form inside
// blocks of N / 2D words), so a CTA copies the tile of all nb plaintexts of
// its next unit with cp.async while it multiplies the current one
// (double-buffered), and gathers from shared memory. One coefficient per
// thread, 256 threads: tile t = coefficients [256 t, 256 t + 256).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

constexpr uint32_t kDiagTile = 256;

// Residues below 2^50: operands split into 25-bit halves, x = x1 2^25 + x0;
// the partial sums x0 y0, x0 y1 + x1 y0, x1 y1 of the products accumulate
// in 64-bit registers by single 32 x 32 + 64 multiply-adds (products of
// halves < 2^50: 4,096 products fit between folds); recombined in 128 bits.
constexpr uint32_t kHalfBits = 25, kHalfMask = (1u << kHalfBits) - 1, kHalfFold = 4096;
__device__ __forceinline__ void mad_wide(u64& acc, uint32_t a, uint32_t b) {
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc) : "r"(a), "r"(b));
}
struct Halves {
    u64 s00, s01, s11;
};
__device__ __forceinline__ void halves_mad(Halves& h, uint32_t v0, uint32_t v1, uint32_t x0, uint32_t x1) {
    mad_wide(h.s00, v0, x0);
    mad_wide(h.s01, v0, x1);
    mad_wide(h.s01, v1, x0);
    mad_wide(h.s11, v1, x1);
}
__device__ __forceinline__ u64 halves_reduce(const Halves& h, const ModConst& m) {
    u64 lo = h.s00, hi = 0;
    const u64 t1 = h.s01 << kHalfBits, t2 = h.s11 << (2 * kHalfBits);
    lo += t1;
    hi += (lo < t1 ? 1 : 0) + (h.s01 >> (64 - kHalfBits));
    lo += t2;
    hi += (lo < t2 ? 1 : 0) + (h.s11 >> (64 - 2 * kHalfBits));
    return reduce128(hi, lo, m);
}

template <int NB, bool HALVES>
__global__ void __launch_bounds__(kDiagTile) diag_inner_staged_kernel(
    const PrimeConst* __restrict__ pc, u64* __restrict__ arena, uint32_t n, const DiagJob* __restrict__ jobs,
    const u64* __restrict__ srcs, const DiagUnit* __restrict__ units, u64 stride, uint32_t reduce_every,
    int accumulate) {
    extern __shared__ u64 stage[];          // 2 buffers x NB plaintexts x kDiagTile words
    // jobs vary fastest across the grid: consecutive CTAs are other outputs
    // of the same tile, so outputs that share their baby steps (one query's
    // giant steps) read them from L2
    const uint32_t z = blockIdx.x, l = blockIdx.z, tid = threadIdx.x;
    const uint32_t base = blockIdx.y * kDiagTile, i = base + tid;
    const DiagJob J = jobs[z];
    const ModConst m = modconst_of(pc[l]);
    const u64 off = (u64)l * n;
    const u64* s = srcs + (u64)z * 2 * NB;
    u64 x0[HALVES ? 1 : NB], x1[HALVES ? 1 : NB];
    uint32_t h00[HALVES ? NB : 1], h01[HALVES ? NB : 1], h10[HALVES ? NB : 1], h11[HALVES ? NB : 1];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const u64 y0 = arena[s[2 * b] + off + i], y1 = arena[s[2 * b + 1] + off + i];
        if (HALVES) {
            h00[b] = (uint32_t)y0 & kHalfMask;
            h01[b] = (uint32_t)(y0 >> kHalfBits);
            h10[b] = (uint32_t)y1 & kHalfMask;
            h11[b] = (uint32_t)(y1 >> kHalfBits);
        } else {
            x0[b] = y0;
            x1[b] = y1;
        }
    }
    // unit k's tile of its NB plaintexts into buffer `buf`: NB x 128 chunks of 16 bytes
    auto issue = [&](uint32_t k, uint32_t buf) {
        const u64* g = arena + units[k].pt + off + base;
        u64* d = stage + (size_t)buf * NB * kDiagTile;
        for (uint32_t c = tid; c < NB * (kDiagTile / 2); c += kDiagTile) {
            const uint32_t b = c / (kDiagTile / 2), w = (c % (kDiagTile / 2)) * 2;
            cp_async16(d + b * kDiagTile + w, g + (u64)b * stride + w);
        }
        cp_async_commit();
    };
    Acc128 a0, a1;
    acc_init(a0);
    acc_init(a1);
    Halves c0{0, 0, 0}, c1{0, 0, 0};
    uint32_t cnt = 0;
    if (J.u0 < J.u1) issue(J.u0, 0);
    for (uint32_t k = J.u0; k < J.u1; ++k) {
        const uint32_t buf = (k - J.u0) & 1u;
        const uint32_t* map = units[k].map;
        const uint32_t j = (map ? __ldg(map + i) : i) - base;
        if (k + 1 < J.u1) {
            issue(k + 1, buf ^ 1u);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const u64* t = stage + (size_t)buf * NB * kDiagTile + j;
        if (HALVES) {
            if (cnt + NB > kHalfFold) {
                c0 = Halves{halves_reduce(c0, m), 0, 0};
                c1 = Halves{halves_reduce(c1, m), 0, 0};
                cnt = 1;
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const u64 v = t[b * kDiagTile];
                const uint32_t v0 = (uint32_t)v & kHalfMask, v1 = (uint32_t)(v >> kHalfBits);
                halves_mad(c0, v0, v1, h00[b], h01[b]);
                halves_mad(c1, v0, v1, h10[b], h11[b]);
            }
        } else {
            if (cnt + NB > reduce_every) {
                acc_fold(a0, m);
                acc_fold(a1, m);
                cnt = 1;
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const u64 v = t[b * kDiagTile];
                acc_mad(a0, v, x0[b]);
                acc_mad(a1, v, x1[b]);
            }
        }
        cnt += NB;
        __syncthreads();                    // the buffer is refilled two units later
    }
    u64 r0 = HALVES ? halves_reduce(c0, m) : acc_reduce(a0, m);
    u64 r1 = HALVES ? halves_reduce(c1, m) : acc_reduce(a1, m);
    if (accumulate) {
        r0 = add_mod(r0, arena[J.out0 + off + i], m.q);
        r1 = add_mod(r1, arena[J.out1 + off + i], m.q);
    }
    arena[J.out0 + off + i] = r0;
    arena[J.out1 + off + i] = r1;
}

cudaError_t launch_diag_inner(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t jobs,
                              uint32_t nb, const DiagJob* job, const u64* srcs, const DiagUnit* unit, u64 stride,
                              uint32_t reduce_every, int accumulate, bool staged, bool halves, cudaStream_t st) {
    if (limbs == 0 || jobs == 0) return cudaSuccess;
    if (staged) {
        if (n % kDiagTile) return cudaErrorInvalidValue;
        if (n / kDiagTile > 65535 || limbs > 65535) return cudaErrorInvalidValue;
        dim3 grid(jobs, n / kDiagTile, limbs);
        const size_t smem = 2ull * nb * kDiagTile * sizeof(u64);
#define DIAG_STAGED_H(NBV, H)                                                                                  \
    {                                                                                                          \
        cudaError_t e = cudaFuncSetAttribute(diag_inner_staged_kernel<NBV, H>,                                 \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);          \
        if (e != cudaSuccess) return e;                                                                        \
        diag_inner_staged_kernel<NBV, H><<<grid, kDiagTile, smem, st>>>(pc, arena, n, job, srcs, unit, stride, \
                                                                        reduce_every, accumulate);             \
    }
#define DIAG_STAGED(NBV)                \
    case NBV:                           \
        if (halves)                     \
            DIAG_STAGED_H(NBV, true)    \
        else                            \
            DIAG_STAGED_H(NBV, false)   \
        break;
        switch (nb) {
            DIAG_STAGED(1)
            DIAG_STAGED(2)
            DIAG_STAGED(4)
            DIAG_STAGED(8)
            DIAG_STAGED(16)
        default: return cudaErrorInvalidValue;
        }
#undef DIAG_STAGED
#undef DIAG_STAGED_H
        count_launches(1);
        return cudaGetLastError();
    }
    dim3 grid((n + 255) / 256, limbs, jobs);
    switch (nb) {
    case 1: diag_inner_kernel<1><<<grid, 256, 0, st>>>(pc, arena, n, job, srcs, unit, stride, reduce_every, accumulate); break;
    case 2: diag_inner_kernel<2><<<grid, 256, 0, st>>>(pc, arena, n, job, srcs, unit, stride, reduce_every, accumulate); break;
    case 4: diag_inner_kernel<4><<<grid, 256, 0, st>>>(pc, arena, n, job, srcs, unit, stride, reduce_every, accumulate); break;
    case 8: diag_inner_kernel<8><<<grid, 256, 0, st>>>(pc, arena, n, job, srcs, unit, stride, reduce_every, accumulate); break;
    case 16: diag_inner_kernel<16><<<grid, 256, 0, st>>>(pc, arena, n, job, srcs, unit, stride, reduce_every, accumulate); break;
    default: return cudaErrorInvalidValue;
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_mac_plain(const PrimeConst* pc, u64* arena, uint32_t n, uint32_t limbs, uint32_t jobs,
                             const MacJob* job, const MacGroup* group, const MacTerm* term, uint32_t reduce_every,
                             int accumulate, cudaStream_t st) {
    if (limbs == 0 || jobs == 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, limbs, jobs);
    mac_plain_kernel<<<grid, 256, 0, st>>>(pc, arena, n, job, group, term, reduce_every, accumulate);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// plain transforms
// ---------------------------------------------------------------------------
cudaError_t launch_ntt_plain(bool inverse, int log_n, const PrimeTables& pt, const LimbJob* jobs, uint32_t limbs,
                             u64* src_arena, u64* dst_arena, uint32_t nz, const ZBases& zb, cudaStream_t st) {
    LoadPlain pro{src_arena};
    StorePlain epi{dst_arena};
    if (inverse) return launch_ntt<true>(log_n, pt, jobs, limbs, nz, dst_arena, zb, pro, epi, st);
    return launch_ntt<false>(log_n, pt, jobs, limbs, nz, dst_arena, zb, pro, epi, st);
}

// ---------------------------------------------------------------------------
// rescale (rescale.cpp:3-72)
//   step 1: INTT of the last limb -> coefficients in scratch
//   step 2: NTT over limbs i < L-1 whose prologue is the centred lift of the
//           last limb times QlQlInvModqlDivqlModq[i], and whose epilogue is
//           a_i * qlInvModq[i] + NTT(...)
// ---------------------------------------------------------------------------
struct RescaleLoad {
    const u64* scratch;
    const u64* qlql;
    const u64* qlql_sh;
    const PrimeConst* pc_last;   // q_l, the prime being dropped
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst& pc) const {
        const u64 q = pc.q;
        const u64 ql = pc_last->q, ql_half = ql >> 1;
        u64 v = scratch[zb.aux.at(z) + x];                           // last limb coefficient, [0, q_l)
        u64 vm = csub(mul_shoup_lazy(v, 1, pc.one_sh, q), q);         // v mod q_i
        u64 qlm = csub(mul_shoup_lazy(ql, 1, pc.one_sh, q), q);       // q_l mod q_i
        u64 val = (v > ql_half) ? sub_mod(vm, qlm, q) : vm;           // rescale.cpp:50 tie rule
        return mul_shoup(val, __ldg(qlql + j.aux), __ldg(qlql_sh + j.aux), q);
    }
};

struct RescaleStore {
    u64* arena;
    const u64* qlinv;
    const u64* qlinv_sh;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst& pc) const {
        const u64 q = pc.q;
        u64 a = arena[zb.src.at(z) + j.src + x];
        u64 s = mul_shoup(a, __ldg(qlinv + j.aux), __ldg(qlinv_sh + j.aux), q);
        arena[zb.out.at(z) + j.out + x] = add_mod(s, v, q);
    }
};

// zb.src = input poly (arena), zb.out = output poly (arena), zb.mid = scratch
// region of sizeQl * N words per z: words [0, N) hold the last limb's
// coefficients, words [N, sizeQl * N) the step-2 intermediates.
cudaError_t launch_rescale(int log_n, const OpTabs& t, const LimbJob* jobs_q, uint32_t sizeQl, u64* arena,
                           u64* scratch, uint32_t nz, const ZBases& zb_in, cudaStream_t st) {
    if (sizeQl < 2 || nz == 0) return cudaSuccess;
    const u64 n = 1ull << log_n;
    const uint32_t last = sizeQl - 1;
    // step 1: INTT(last limb). jobs_q[last] has src = dst = out = last * N,
    // so shifting mid / out back by last * N lands it at scratch + mid(z).
    ZBases z1 = zb_in;
    z1.mid = zf_plus(zb_in.mid, (u64)0 - (u64)last * n);
    z1.out = z1.mid;
    cudaError_t e = launch_ntt<true>(log_n, t.pt, jobs_q + last, 1, nz, scratch, z1, LoadPlain{arena},
                                     StorePlain{scratch}, st);
    if (e != cudaSuccess) return e;
    // step 2
    ZBases z2 = zb_in;
    z2.aux = zb_in.mid;                      // coefficients of the last limb
    z2.mid = zf_plus(zb_in.mid, n);          // intermediates
    RescaleLoad pro{scratch, t.qlql, t.qlql_sh, t.pt.pc + last};
    RescaleStore epi{arena, t.qlinv, t.qlinv_sh};
    return launch_ntt<false>(log_n, t.pt, jobs_q, last, nz, scratch, z2, pro, epi, st);
}

// ---------------------------------------------------------------------------
// key switch (key_switch.cpp:167-439)
// ---------------------------------------------------------------------------
// Scratch layout per polynomial (S = slots_q + K limb slots, Q limb i at slot
// i, special limb k at slot slots_q + k):
//   coef   : slots_q * N   INTT of the input's Q limbs, times qHatInv (ModUp's first factor)
//   modup  : parts * S * N digit j's complementary limbs, evaluation form
//   ext0   : S * N         sum_j digit_j * evk_b   (then ModDown input)
//   ext1   : S * N         sum_j digit_j * evk_a
//   mid    : 2 * slots_q * N  two-pass intermediates of the ModDown NTTs
//   t0     : slots_q * N   c0 gathered through the automorphism (rotation)
size_t ks_scratch_words(uint32_t n, uint32_t slots_q, uint32_t K, uint32_t parts) {
    const size_t S = slots_q + K;
    return (size_t)n * (slots_q + parts * S + 2 * S + 3 * (size_t)slots_q);
}

// Input load through the automorphism: the key switch of auto(c1) reads
// c1[map[x]] (the reference applies automorphism() first, fhe_host_driver.cpp:342-350).
struct LoadGather {
    const u64* base;
    const uint32_t* map;
    ZField mapz;        // per-entry map addresses (per_z)
    int per_z;
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst&) const {
        const uint32_t* m = per_z ? (const uint32_t*)mapz.at(z) : map;
        return base[zb.src.at(z) + j.src + __ldg(m + x)];
    }
};

// Epilogue of the input's INTT: stores y_i = [x_i * qHatInv_i]_{q_i}, the
// first factor of ModUp's base conversion (key_switch.cpp:7-60), once per
// input limb instead of once per complementary output limb. job.aux = Q limb i.
struct StoreQhatInv {
    u64* scratch;
    OpTabs t;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst& pc) const {
        const uint32_t part = j.aux / t.alpha, idx = j.aux - part * t.alpha;
        scratch[zb.out.at(z) + j.out + x] =
            mul_shoup(v, __ldg(t.qhat_inv[part] + idx), __ldg(t.qhat_inv_sh[part] + idx), pc.q);
    }
};

// Epilogue of the special limbs' INTT before ModDown: stores
// [x_k * PHatInv_k]_{p_k}, the first factor of the P -> Q base conversion
// (key_switch.cpp:62-163), once per special limb. job.aux = special limb k.
struct StorePhatInv {
    u64* scratch;
    OpTabs t;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst& pc) const {
        scratch[zb.out.at(z) + j.out + x] =
            mul_shoup(v, __ldg(t.phat_inv_modp + j.aux), __ldg(t.phat_inv_modp_sh + j.aux), pc.q);
    }
};

// ModUp base conversion as the NTT prologue: job.aux = digit << 16 | k, where
// k is the output's position among the digit's complementary primes. Reads
// y_i = [x_i * qHatInv_i]_{q_i} (StoreQhatInv) and sums y_i * [qHat_i]_p.
struct ModUpLoad {
    const u64* scratch;   // coef region at zb.aux[z]
    OpTabs t;
    uint32_t K;
    uint32_t n;
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst& pc) const {
        const uint32_t part = j.aux >> 16, k = j.aux & 0xFFFFu;
        const uint32_t start = part * t.alpha;
        const uint32_t size = (part == t.parts - 1) ? t.sizeQl - start : t.alpha;
        const uint32_t row = t.sizeQl - size + K;   // complementary primes of this digit
        const u64 p = pc.q, p2 = p << 1;
        const u64* qm = t.qhat_modp[part];
        const u64* qmsh = t.qhat_modp_sh[part];
        u64 s = 0;
        for (uint32_t i = 0; i < size; ++i) {
            const uint32_t limb = start + i;
            const u64 y = scratch[zb.aux.at(z) + (u64)limb * n + x];            // [x * qHatInv]_{q_i}
            u64 w = mul_shoup_lazy(y, __ldg(qm + i * row + k), __ldg(qmsh + i * row + k), p);
            s += w;
            s = s >= p2 ? s - p2 : s;
        }
        return csub(s, p);
    }
};

struct StoreSlot {   // plain store into scratch
    u64* scratch;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst&) const {
        scratch[zb.out.at(z) + j.out + x] = v;
    }
};

// Inner product with the evaluation key. One thread per (slot, coefficient).
// slot s < sizeQl is Q limb s, slot slots_q + k is special limb k.
__global__ void __launch_bounds__(256) ks_mac_kernel(OpTabs t, uint32_t n, uint32_t slots_q, uint32_t sizeQl,
                                                     uint32_t K, const u64* __restrict__ key, u64 evk_a, u64 evk_b,
                                                     uint32_t key_stride, uint32_t key_pbase,
                                                     const u64* __restrict__ arena, u64* __restrict__ scratch,
                                                     u64 modup_off, u64 ext0_off, u64 ext1_off, u64 t0_off,
                                                     const ZBases zb, const KsFuse f) {
    const uint32_t sidx = blockIdx.y;   // 0..sizeQl+K-1
    const uint32_t z = blockIdx.z;
    const bool isq = sidx < sizeQl;
    const uint32_t slot = isq ? sidx : slots_q + (sidx - sizeQl);
    const uint32_t prime = isq ? sidx : t.p_base + (sidx - sizeQl);
    const uint32_t klimb_in_digit = isq ? sidx : key_pbase + (sidx - sizeQl);
    const PrimeConst pc = t.pt.pc[prime];
    const ModConst mc = modconst_of(pc);
    const u64 S = (u64)slots_q + K;
    const u64 base_scr = zb.mid.at(z);
    const u64* in = arena + zb.src.at(z) + (u64)sidx * n;   // only valid for Q limbs
    const u64 c0_off = f.has_c0 ? f.c0.at(z) : 0;
    const uint32_t* map = f.per_z ? (const uint32_t*)f.mapz.at(z) : f.map;
    const u64 koff = f.per_z ? f.keyz.at(z) : 0;           // this entry's key (per_z)
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
        const uint32_t xs = map ? __ldg(map + x) : x;         // position read through the automorphism
        if (isq && f.has_c0)
            scratch[base_scr + t0_off + (u64)sidx * n + x] = arena[c0_off + (u64)sidx * n + xs];
        Acc128 ab, aa;
        acc_init(ab);
        acc_init(aa);
        for (uint32_t part = 0; part < t.parts; ++part) {
            const uint32_t start = part * t.alpha;
            const uint32_t size = (part == t.parts - 1) ? sizeQl - start : t.alpha;
            u64 d;
            if (isq && sidx >= start && sidx < start + size) d = in[xs];
            else d = scratch[base_scr + modup_off + ((u64)part * S + slot) * n + x];
            const u64 kl = koff + ((u64)part * key_stride + klimb_in_digit) * n + x;
            acc_mad(ab, d, __ldg(key + evk_b + kl));
            acc_mad(aa, d, __ldg(key + evk_a + kl));
        }
        scratch[base_scr + ext0_off + (u64)slot * n + x] = acc_reduce(ab, mc);
        scratch[base_scr + ext1_off + (u64)slot * n + x] = acc_reduce(aa, mc);
    }
}

// ModDown base conversion P -> Q as the NTT prologue (job = Q limb i). Reads
// [x_k * PHatInv_k]_{p_k} (StorePhatInv) and sums it times [PHat_k]_{q_i}.
struct ModDownLoad {
    const u64* scratch;  // ext region at zb.aux[z]
    OpTabs t;
    uint32_t slots_q, K, n;
    __device__ __forceinline__ u64 operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x,
                                              const PrimeConst& pc) const {
        const u64 q = pc.q, q2 = q << 1;
        const uint32_t i = j.aux;
        u64 s = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const u64 y = scratch[zb.aux.at(z) + (u64)(slots_q + k) * n + x];
            u64 w = mul_shoup_lazy(y, __ldg(t.phat_modq + k * t.sizeQl + i), __ldg(t.phat_modq_sh + k * t.sizeQl + i), q);
            s += w;
            s = s >= q2 ? s - q2 : s;
        }
        return csub(s, q);
    }
};

// ModDown combine as the NTT epilogue: out = (x_Q - y) * P^-1 mod q_i.
// z' = 2z + h: h = 0 writes ks0 (+ gathered c0, + acc0), h = 1 writes ks1 (+ acc1).
struct ModDownStore {
    const u64* scratch;  // ext region at zb.src(z)
    u64* arena;          // outputs
    OpTabs t;
    uint32_t n;
    int has_c0, has_acc;
    ZField t0;           // scratch offset of the gathered c0, per ciphertext
    ZField out0, out1;   // ks0 / ks1 destinations, per ciphertext
    ZField acc0, acc1;
    __device__ __forceinline__ void operator()(const LimbJob& j, const ZBases& zb, uint32_t z, uint32_t x, u64 v,
                                               const PrimeConst& pc) const {
        const u64 q = pc.q;
        const uint32_t i = j.aux;
        const uint32_t h = z & 1u, zc = z >> 1;
        const u64 li = (u64)i * n + x;
        u64 xq = scratch[zb.src.at(z) + li];
        u64 d = sub_mod(xq, v, q);
        u64 r = mul_shoup(d, __ldg(t.p_inv_mod_q + i), __ldg(t.p_inv_mod_q_sh + i), q);
        if (h == 0 && has_c0) r = add_mod(r, scratch[t0.at(zc) + li], q);
        if (has_acc) r = add_mod(r, arena[(h ? acc1.at(zc) : acc0.at(zc)) + li], q);
        arena[(h ? out1.at(zc) : out0.at(zc)) + li] = r;
    }
};

cudaError_t launch_key_switch(int log_n, const OpTabs& t, const LimbJob* jobs_qp, const LimbJob* jobs_modup,
                              uint32_t n_modup, uint32_t slots_q, uint32_t sizeQl, uint32_t K, const u64* key,
                              u64 evk_a, u64 evk_b, uint32_t key_stride, uint32_t key_pbase, u64* arena,
                              u64* scratch, uint32_t nz, const ZBases& zb, cudaStream_t st, const KsFuse* fuse) {
    if (nz == 0) return cudaSuccess;
    if (2ull * nz > 65535ull) return cudaErrorInvalidValue;
    KsFuse f{};
    if (fuse) f = *fuse;
    const u64 n = 1ull << log_n;
    const u64 S = (u64)slots_q + K;
    const u64 off_coef = 0;
    const u64 off_modup = off_coef + (u64)slots_q * n;
    const u64 off_ext0 = off_modup + (u64)t.parts * S * n;
    const u64 off_ext1 = off_ext0 + S * n;
    const u64 off_mid = off_ext1 + S * n;
    const u64 off_t0 = off_mid + 2ull * slots_q * n;
    cudaError_t e;

    // 1. INTT of the input's Q limbs -> coef (slot i at coef + i*N)
    {
        ZBases a = zb;
        a.mid = zf_plus(zb.mid, off_coef);
        a.out = a.mid;
        if (f.map || f.per_z)
            e = launch_ntt<true>(log_n, t.pt, jobs_qp, sizeQl, nz, scratch, a,
                                 LoadGather{arena, f.map, f.mapz, f.per_z}, StoreQhatInv{scratch, t}, st);
        else
            e = launch_ntt<true>(log_n, t.pt, jobs_qp, sizeQl, nz, scratch, a, LoadPlain{arena},
                                 StoreQhatInv{scratch, t}, st);
        if (e != cudaSuccess) return e;
    }
    // 2. ModUp: base conversion + NTT for every (digit, complementary limb)
    {
        ZBases a = zb;
        a.aux = zf_plus(zb.mid, off_coef);
        a.mid = zf_plus(zb.mid, off_modup);
        a.out = a.mid;
        ModUpLoad pro{scratch, t, K, (uint32_t)n};
        e = launch_ntt<false>(log_n, t.pt, jobs_modup, n_modup, nz, scratch, a, pro, StoreSlot{scratch}, st);
        if (e != cudaSuccess) return e;
    }
    // 3. inner product with the key
    {
        dim3 grid((uint32_t)((n + 255) / 256), sizeQl + K, nz);
        ks_mac_kernel<<<grid, 256, 0, st>>>(t, (uint32_t)n, slots_q, sizeQl, K, key, evk_a, evk_b, key_stride,
                                            key_pbase, arena, scratch, off_modup, off_ext0, off_ext1, off_t0, zb, f);
        count_launches(1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // 4. ModDown of both accumulators: z' = 2z (ext0 -> ks0), 2z + 1 (ext1 -> ks1)
    {
        ZBases a{};
        a.src = zf_pair(zf_plus(zb.mid, off_ext0), off_ext1 - off_ext0);
        a.aux = a.src;
        a.mid = a.src;
        a.out = a.src;
        // 4a. INTT of the special limbs, in place, times PHatInv
        e = launch_ntt<true>(log_n, t.pt, jobs_qp + slots_q, K, 2 * nz, scratch, a, LoadPlain{scratch},
                             StorePhatInv{scratch, t}, st);
        if (e != cudaSuccess) return e;
        // 4b. NTT over Q limbs with base-conversion prologue and ModDown epilogue
        ZBases b = a;
        b.mid = zf_pair(zf_plus(zb.mid, off_mid), (u64)slots_q * n);
        ModDownLoad pro{scratch, t, slots_q, K, (uint32_t)n};
        ModDownStore epi{};
        epi.scratch = scratch;
        epi.arena = arena;
        epi.t = t;
        epi.n = (uint32_t)n;
        epi.has_c0 = f.has_c0;
        epi.has_acc = f.has_acc;
        epi.t0 = zf_plus(zb.mid, off_t0);
        epi.out0 = zb.out;
        epi.out1 = zb.aux;
        epi.acc0 = f.acc0;
        epi.acc1 = f.acc1;
        e = launch_ntt<false>(log_n, t.pt, jobs_qp, sizeQl, 2 * nz, scratch, b, pro, epi, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// table preparation
// ---------------------------------------------------------------------------
__global__ void companions_kernel(u64* v, u64* sh, const u64* m, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        u64 mod = m[i];
        if (mod == 0) { sh[i] = 0; continue; }
        u64 w = v[i] % mod;
        v[i] = w;
        sh[i] = shoup_companion(w, mod);
    }
}

cudaError_t launch_companions(u64* v, u64* sh, const u64* m, size_t count, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    unsigned blocks = (unsigned)((count + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    companions_kernel<<<blocks, 256, 0, st>>>(v, sh, m, count);
    count_launches(1);
    return cudaGetLastError();
}

__global__ void interleave_kernel(const u64* raw, const u64* q, ulonglong2* out2, uint32_t rows, uint32_t n) {
    const size_t total = (size_t)rows * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const u64 m = q[i / n];
        const u64 w = raw[i] % m;
        out2[i] = make_ulonglong2(w, shoup_companion(w, m));
    }
}

cudaError_t launch_interleave(const u64* raw, const u64* q, ulonglong2* out2, uint32_t rows, uint32_t n,
                              cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    size_t total = (size_t)rows * n;
    unsigned blocks = (unsigned)((total + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    interleave_kernel<<<blocks, 256, 0, st>>>(raw, q, out2, rows, n);
    count_launches(1);
    return cudaGetLastError();
}

__global__ void prime_consts_kernel(PrimeConst* pc, const u64* q, const u64* ninv, const u64* itw, uint32_t n,
                                    uint32_t count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    PrimeConst c;
    c.q = q[i];
    ModConst m = make_modconst(c.q);
    c.r64 = m.r64;
    c.r64_sh = m.r64_sh;
    c.one_sh = m.one_sh;
    c.ninv = ninv[i] % c.q;
    c.ninv_sh = shoup_companion(c.ninv, c.q);
    c.w1ninv = mul_mod(itw[(u64)i * n + 1] % c.q, c.ninv, m);
    c.w1ninv_sh = shoup_companion(c.w1ninv, c.q);
    pc[i] = c;
}

cudaError_t launch_prime_consts(PrimeConst* pc, const u64* q, const u64* ninv, const u64* itw, uint32_t n,
                                uint32_t count, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    prime_consts_kernel<<<(count + 63) / 64, 64, 0, st>>>(pc, q, ninv, itw, n, count);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace afhe
