// ksfused.cu -- the whole hybrid key switch in one kernel, for N <= 2^13.
//
// Same arithmetic as launch_key_switch (key_switch.cpp:167-439 restated:
// INTT of the input's limbs, fast_bases_conv to each digit's complementary
// primes, NTT, inner product with evk_a / evk_b, approx_mod_down), but one
// CTA carries one ciphertext polynomial through every step with the limb
// being transformed held in shared memory:
//
//   phase 0  coef[i] = INTT(in[i]) for the input's Q limbs -> lane scratch
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
// two accumulators), 3 * (N + N/16) words = 204 KB at N = 8192. The key limbs
// every CTA of a launch reads are the same, so they come from L2.
//
// In place is safe: input limb i is read only while slot i is processed, and
// output limb i is written after every read of input limb i and of the
// gathered c0 limb i (they are staged in shared memory first).
#include "internal.h"

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
};

// digit j of a level-l key switch: limbs [start, start + size)
__device__ __forceinline__ void digit_range(const OpTabs& t, uint32_t j, uint32_t& start, uint32_t& size) {
    start = j * t.alpha;
    size = (j == t.parts - 1) ? t.sizeQl - start : t.alpha;
}

// Not inlined: each transform gets its own register allocation instead of
// competing with the caller's live state (1024 threads leave 64 registers).
template <int LOGN>
__device__ __noinline__ void fwd_ntt(u64* buf, const PrimeTables pt, uint32_t prime, const PrimeConst pc) {
    ntt_rounds<false, LOGN, 0, false, 0>(buf, pt.tw2 + ((u64)prime << LOGN), pc, 0u, LOGN, 0, true);
}

template <int LOGN>
__device__ __noinline__ void inv_ntt(u64* buf, const PrimeTables pt, uint32_t prime, const PrimeConst pc) {
    ntt_rounds<true, LOGN, 0, false, 0>(buf, pt.itw2 + ((u64)prime << LOGN), pc, 0u, LOGN, 0, true);
}

// Inner product for one slot (Q limb `s` < l, or special limb s - l) into A0 / A1:
// A0 = sum_j d_j * evk_b[j], A1 = sum_j d_j * evk_a[j] (mod the slot's prime).
template <int LOGN>
__device__ void mac_slot(const KsFusedArgs& a, uint32_t z, uint32_t s, u64* W, u64* A0, u64* A1,
                         const u64* __restrict__ in, const u64* __restrict__ coef) {
    constexpr uint32_t N = 1u << LOGN, T = N / 8;
    const OpTabs& t = a.t;
    const uint32_t l = a.sizeQl;
    const bool isq = s < l;
    const uint32_t prime = isq ? s : t.p_base + (s - l);
    const uint32_t klimb = isq ? s : a.key_pbase + (s - l);
    const PrimeConst pc = t.pt.pc[prime];
    const ModConst mc = modconst_of(pc);
    const u64 p2 = pc.q << 1;
    for (uint32_t j = 0; j < t.parts; ++j) {
        uint32_t start, size;
        digit_range(t, j, start, size);
        const bool own = isq && s >= start && s < start + size;
        const u64* kb = a.key + a.evk_b + ((u64)j * a.key_stride + klimb) * N;
        const u64* ka = a.key + a.evk_a + ((u64)j * a.key_stride + klimb) * N;
        if (!own) {
            // W = BConv_j(coef) at this slot's prime, then NTT
            const uint32_t row = l - size + a.K;
            const uint32_t kpos = isq ? (s < start ? s : s - size) : (l - size) + (s - l);
            const u64* qi = t.qhat_inv[j];
            const u64* qish = t.qhat_inv_sh[j];
            const u64* qm = t.qhat_modp[j];
            const u64* qmsh = t.qhat_modp_sh[j];
#pragma unroll 2
            for (uint32_t x = threadIdx.x; x < N; x += T) {
                u64 acc = 0;
                for (uint32_t i = 0; i < size; ++i) {
                    const uint32_t limb = start + i;
                    const u64 qq = t.pt.pc[limb].q;
                    u64 y = mul_shoup(coef[((u64)limb << LOGN) + x], __ldg(qi + i), __ldg(qish + i), qq);
                    acc += mul_shoup_lazy(y, __ldg(qm + i * row + kpos), __ldg(qmsh + i * row + kpos), pc.q);
                    acc = acc >= p2 ? acc - p2 : acc;
                }
                W[padix(x)] = csub(acc, pc.q);
            }
            __syncthreads();
            fwd_ntt<LOGN>(W, t.pt, prime, pc);
        }
#pragma unroll 2
        for (uint32_t x = threadIdx.x; x < N; x += T) {
            u64 d;
            if (own) d = in[((u64)s << LOGN) + (a.f.map ? __ldg(a.f.map + x) : x)];
            else d = canon4(W[padix(x)], pc.q);
            u64 pb = mul_mod(d, __ldg(kb + x), mc);
            u64 pa = mul_mod(d, __ldg(ka + x), mc);
            if (j > 0) {
                pb = add_mod(pb, A0[padix(x)], pc.q);
                pa = add_mod(pa, A1[padix(x)], pc.q);
            }
            A0[padix(x)] = pb;
            A1[padix(x)] = pa;
        }
        __syncthreads();
    }
}

template <int LOGN>
__global__ void __launch_bounds__((1u << LOGN) / 8, 1) ks_fused_kernel(const KsFusedArgs a) {
    constexpr uint32_t N = 1u << LOGN, T = N / 8;
    constexpr uint32_t PADN = N + N / 16;
    extern __shared__ u64 smem[];
    u64* W = smem;
    u64* A0 = smem + PADN;
    u64* A1 = smem + 2 * PADN;
    const uint32_t z = blockIdx.x;
    const OpTabs& t = a.t;
    const uint32_t l = a.sizeQl, K = a.K;
    const u64* in = a.arena + a.in.at(z);
    u64* coef = a.scratch + a.mid.at(z);          // l limbs
    u64* pcoef = coef + ((u64)l << LOGN);         // 2K limbs: INTT of the special accumulators

    // phase 0: coefficients of the input's limbs (read through the automorphism)
    for (uint32_t i = 0; i < l; ++i) {
        const PrimeConst pc = t.pt.pc[i];
#pragma unroll 2
        for (uint32_t x = threadIdx.x; x < N; x += T)
            W[padix(x)] = in[((u64)i << LOGN) + (a.f.map ? __ldg(a.f.map + x) : x)];
        __syncthreads();
        inv_ntt<LOGN>(W, t.pt, i, pc);
#pragma unroll 2
        for (uint32_t x = threadIdx.x; x < N; x += T) coef[((u64)i << LOGN) + x] = W[padix(x)];
        __syncthreads();
    }
    // phase 1: special slots -> INTT of both accumulators
    for (uint32_t k = 0; k < K; ++k) {
        mac_slot<LOGN>(a, z, l + k, W, A0, A1, in, coef);
        const uint32_t prime = t.p_base + k;
        const PrimeConst pc = t.pt.pc[prime];
        inv_ntt<LOGN>(A0, t.pt, prime, pc);
        inv_ntt<LOGN>(A1, t.pt, prime, pc);
#pragma unroll 2
        for (uint32_t x = threadIdx.x; x < N; x += T) {
            pcoef[((u64)(2 * k) << LOGN) + x] = A0[padix(x)];
            pcoef[((u64)(2 * k + 1) << LOGN) + x] = A1[padix(x)];
        }
        __syncthreads();
    }
    // phase 2: Q limbs -> ModDown and outputs
    const u64 o0 = a.out0.at(z), o1 = a.out1.at(z);
    const u64 c0 = a.f.has_c0 ? a.f.c0.at(z) : 0;
    const u64 ac0 = a.f.has_acc ? a.f.acc0.at(z) : 0, ac1 = a.f.has_acc ? a.f.acc1.at(z) : 0;
    for (uint32_t i = 0; i < l; ++i) {
        mac_slot<LOGN>(a, z, i, W, A0, A1, in, coef);
        const PrimeConst pc = t.pt.pc[i];
        const u64 q = pc.q, q2 = q << 1;
        const u64 pinv = __ldg(t.p_inv_mod_q + i), pinv_sh = __ldg(t.p_inv_mod_q_sh + i);
        for (uint32_t h = 0; h < 2; ++h) {
            u64* A = h ? A1 : A0;
            // W = BConv of the special limbs to q_i (approx_mod_down's fast_bases_conv), then NTT
#pragma unroll 2
            for (uint32_t x = threadIdx.x; x < N; x += T) {
                u64 acc = 0;
                for (uint32_t k = 0; k < K; ++k) {
                    const PrimeConst& pk = t.pt.pc[t.p_base + k];
                    u64 y = mul_shoup(pcoef[((u64)(2 * k + h) << LOGN) + x], __ldg(t.phat_inv_modp + k),
                                      __ldg(t.phat_inv_modp_sh + k), pk.q);
                    acc += mul_shoup_lazy(y, __ldg(t.phat_modq + k * l + i), __ldg(t.phat_modq_sh + k * l + i), q);
                    acc = acc >= q2 ? acc - q2 : acc;
                }
                W[padix(x)] = csub(acc, q);
            }
            __syncthreads();
            fwd_ntt<LOGN>(W, t.pt, i, pc);
            // (x_Q - y) * P^-1, then the fused extras, staged in A before any store
#pragma unroll 2
            for (uint32_t x = threadIdx.x; x < N; x += T) {
                u64 r = mul_shoup(sub_mod(A[padix(x)], canon4(W[padix(x)], q), q), pinv, pinv_sh, q);
                if (h == 0 && a.f.has_c0)
                    r = add_mod(r, a.arena[c0 + ((u64)i << LOGN) + (a.f.map ? __ldg(a.f.map + x) : x)], q);
                A[padix(x)] = r;
            }
            __syncthreads();
            const u64 ob = (h ? o1 : o0) + ((u64)i << LOGN);
            const u64 ab = (h ? ac1 : ac0) + ((u64)i << LOGN);
#pragma unroll 2
            for (uint32_t x = threadIdx.x; x < N; x += T) {
                u64 r = A[padix(x)];
                if (a.f.has_acc) r = add_mod(r, a.arena[ab + x], q);
                a.arena[ob + x] = r;
            }
            __syncthreads();
        }
    }
}

template <int LOGN>
cudaError_t launch_fused(const KsFusedArgs& a, uint32_t nz, cudaStream_t st) {
    constexpr uint32_t N = 1u << LOGN;
    const size_t smem = 3ull * (N + N / 16) * sizeof(u64);
    cudaError_t e = cudaFuncSetAttribute(ks_fused_kernel<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    ks_fused_kernel<LOGN><<<nz, N / 8, smem, st>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace

bool key_switch_fused_supported(int log_n) { return log_n >= 10 && log_n <= 13; }

size_t ks_fused_scratch_words(uint32_t n, uint32_t sizeQl, uint32_t K) { return (size_t)n * (sizeQl + 2 * K); }

cudaError_t launch_key_switch_fused(int log_n, const OpTabs& t, uint32_t sizeQl, uint32_t K, const u64* key, u64 evk_a,
                                    u64 evk_b, uint32_t key_stride, uint32_t key_pbase, u64* arena, u64* scratch,
                                    uint32_t nz, const ZBases& zb, cudaStream_t st, const KsFuse* fuse) {
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
    switch (log_n) {
    case 10: return launch_fused<10>(a, nz, st);
    case 11: return launch_fused<11>(a, nz, st);
    case 12: return launch_fused<12>(a, nz, st);
    case 13: return launch_fused<13>(a, nz, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace afhe
