// encode.cu -- the server's plaintexts built and CKKS-encoded on the device.
//
// The reference's server encodes its plaintexts with OpenFHE
// (MakeCKKSPackedPlaintext: fhe_core/fhe_searcher.cpp:334-368 builds one
// dimension-major candidate plaintext per batch, slot d B + j = component d of
// candidate j; integration_tools/generate_interactive_test_vectors.cpp:461-521
// the centroid and mask plaintexts). Here:
//
//   values -> slot vectors    afhe_encode_batch: rows of host doubles;
//                             afhe_pq_encode_batches: built on the device from
//                             the IVF-PQ index (candidate = centroid of its list
//                             + its PQ codewords, in double precision)
//   slots -> coefficients     the inverse canonical embedding, slot j at the
//                             root zeta^(5^j), zeta = exp(i pi / N): a
//                             decimation-in-frequency special FFT over N/2
//                             complex values (radix 2, twiddle ksi^((4 len -
//                             5^j mod 4 len) 2N / (4 len)), ksi = exp(2 pi i /
//                             2N)), bit reversal, / (N/2); coefficient i =
//                             round(Re v_i * scale), i + N/2 = round(Im v_i *
//                             scale)
//   coefficients -> RNS, NTT  reduced mod each q_l into poly_gmem, then the
//                             forward NTT of the context (evaluation form)
//
// Double precision: the coefficients equal the exactly rounded ones except
// where the exact value lies within the transform's rounding error (about
// |c| 2^-50) of a half-integer, where they may differ by one (an encoding
// rounding difference, far below CKKS noise).
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "internal.h"
#include "lanes.h"

using namespace afhe;

struct afhe_pq {
    afhe_ctx* ctx = nullptr;
    uint32_t n_list = 0, d = 0, M = 0, K = 0;
    uint64_t n = 0;
    float* centroids = nullptr;     // n_list x d
    float* codebooks = nullptr;     // M x K x (d / M)
    uint8_t* codes = nullptr;       // n x M
    uint32_t* assign = nullptr;     // n
};

namespace afhe {
namespace {

constexpr uint32_t kTile = 4096;        // complex values per shared-memory tile (64 KB)
constexpr uint32_t kTileThreads = 512;
constexpr uint32_t kChunkPts = 256;     // plaintexts per pass of the pipeline

// Twiddle tables of one ring degree: ksi[k] = exp(2 pi i k / 2N), k <= 2N, and
// rot[j] = 5^j mod 2N, j < N/2 (device memory, cached per (device, N) for the
// life of the process).
struct FftTables {
    double2* ksi = nullptr;
    uint32_t* rot = nullptr;
};

std::mutex g_fft_mu;
std::map<std::pair<int, uint32_t>, FftTables> g_fft;

cudaError_t fft_tables(int device, uint32_t n, cudaStream_t st, FftTables* out) {
    std::lock_guard<std::mutex> lock(g_fft_mu);
    auto it = g_fft.find({device, n});
    if (it != g_fft.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    FftTables t;
    const uint32_t m = 2 * n, s = n / 2;
    const double two_pi = 6.283185307179586476925286766559;
    std::vector<double2> ksi(m + 1);
    for (uint32_t k = 0; k <= m; ++k) {
        const double a = two_pi * (double)k / (double)m;
        ksi[k] = make_double2(std::cos(a), std::sin(a));
    }
    std::vector<uint32_t> rot(s);
    uint64_t r = 1;
    for (uint32_t j = 0; j < s; ++j) {
        rot[j] = (uint32_t)r;
        r = r * 5 % m;
    }
    cudaError_t e = cudaMalloc(&t.ksi, ksi.size() * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&t.rot, rot.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.ksi, ksi.data(), ksi.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t.rot, rot.data(), rot.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(t.ksi);
        cudaFree(t.rot);
        return e;
    }
    g_fft[{device, n}] = t;
    *out = t;
    return cudaSuccess;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One radix-2 butterfly of the stage of block length `len` at global pair
// (i + j, i + j + len/2) of plaintext z.
__device__ __forceinline__ void special_bfly(double2& a, double2& b, uint32_t j, uint32_t len, uint32_t m,
                                             const double2* __restrict__ ksi, const uint32_t* __restrict__ rot) {
    const uint32_t lenq = len << 2;
    const uint32_t idx = (lenq - (__ldg(rot + j) & (lenq - 1))) * (m / lenq);
    const double2 u = make_double2(a.x + b.x, a.y + b.y);
    const double2 v = make_double2(a.x - b.x, a.y - b.y);
    a = u;
    b = cmul(v, __ldg(ksi + idx));
}

// Stages with blocks longer than a tile: one butterfly per thread-iteration
// over every plaintext of the chunk, in global memory.
__global__ void fft_global_stage(double2* __restrict__ v, uint32_t s, uint32_t len, uint32_t count,
                                 const double2* __restrict__ ksi, const uint32_t* __restrict__ rot) {
    const uint32_t half = s / 2, lenh = len >> 1, m = 4 * s;
    const u64 total = (u64)count * half;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t / half), b = (uint32_t)(t % half);
        const uint32_t blk = b / lenh, j = b % lenh;
        double2* p = v + (u64)z * s + (u64)blk * len + j;
        double2 a = p[0], c = p[lenh];
        special_bfly(a, c, j, len, m, ksi, rot);
        p[0] = a;
        p[lenh] = c;
    }
}

// The stages with blocks of up to a tile, one tile of `tile` values per CTA
// in shared memory (tile = min(s, kTile)).
__global__ void __launch_bounds__(kTileThreads) fft_tile_stages(double2* __restrict__ v, uint32_t s, uint32_t tile,
                                                                const double2* __restrict__ ksi,
                                                                const uint32_t* __restrict__ rot) {
    extern __shared__ double2 sm2[];
    const uint32_t m = 4 * s;
    double2* g = v + (u64)blockIdx.y * s + (u64)blockIdx.x * tile;
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) sm2[e] = g[e];
    __syncthreads();
    for (uint32_t len = tile; len >= 2; len >>= 1) {
        const uint32_t lenh = len >> 1;
        for (uint32_t b = threadIdx.x; b < tile / 2; b += blockDim.x) {
            const uint32_t blk = b / lenh, j = b % lenh;
            double2& a = sm2[blk * len + j];
            double2& c = sm2[blk * len + j + lenh];
            special_bfly(a, c, j, len, m, ksi, rot);
        }
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) g[e] = sm2[e];
}

// Bit reversal, / (N/2), * scale, rounding, and the residues mod q_0 ..
// q_{level-1} of both halves, into the plaintexts' polynomials.
__global__ void fft_finish(const double2* __restrict__ v, uint32_t log_s, double scale, const u64* __restrict__ q,
                           uint32_t level, u64* __restrict__ arena, const u64* __restrict__ pt, uint32_t count,
                           int* __restrict__ overflow) {
    const uint32_t s = 1u << log_s, n = 2 * s;
    const u64 total = (u64)count * s;
    const double inv = 1.0 / (double)s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t >> log_s), i = (uint32_t)(t & (s - 1));
        const uint32_t r = __brev(i) >> (32 - log_s);
        const double2 x = v[(u64)z * s + r];
        const double re = rint(x.x * inv * scale), im = rint(x.y * inv * scale);
        if (fabs(re) >= 4611686018427387904.0 || fabs(im) >= 4611686018427387904.0) {   // 2^62
            atomicOr(overflow, 1);
            continue;
        }
        const long long cr = (long long)re, ci = (long long)im;
        u64* out = arena + pt[z];
        for (uint32_t l = 0; l < level; ++l) {
            const long long ql = (long long)q[l];
            long long a = cr % ql, b = ci % ql;
            a += a < 0 ? ql : 0;
            b += b < 0 ? ql : 0;
            out[(u64)l * n + i] = (u64)a;
            out[(u64)l * n + i + s] = (u64)b;
        }
    }
}

// slot vectors from host rows (real parts; slots beyond `slots` are zero)
__global__ void fft_load_rows(double2* __restrict__ v, const double* __restrict__ rows, uint32_t s, uint32_t slots,
                              uint32_t count) {
    const u64 total = (u64)count * s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t / s), j = (uint32_t)(t % s);
        v[t] = make_double2(j < slots ? rows[(u64)z * slots + j] : 0.0, 0.0);
    }
}

// dimension-major candidate slot vectors: slot d B + j = component d of the
// batch's candidate j (centroid of its list + its PQ codewords), 0 past the
// batch's count
__global__ void fft_load_pq(double2* __restrict__ v, uint32_t s, uint32_t dim, uint32_t M, uint32_t K,
                            const float* __restrict__ cent, const float* __restrict__ cb, const uint8_t* __restrict__ codes,
                            const uint32_t* __restrict__ assign, const uint32_t* __restrict__ vids,
                            const uint32_t* __restrict__ first, const uint32_t* __restrict__ cnt, uint32_t count) {
    const uint32_t B = s / dim, sd = dim / M;
    const u64 total = (u64)count * s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t / s), slot = (uint32_t)(t % s);
        const uint32_t d = slot / B, j = slot % B;
        double x = 0.0;
        if (j < cnt[z]) {
            const uint32_t id = vids[first[z] + j];
            const uint32_t m = d / sd;
            x = (double)cent[(u64)assign[id] * dim + d] +
                (double)cb[((u64)m * K + codes[(u64)id * M + m]) * sd + (d - m * sd)];
        }
        v[t] = make_double2(x, 0.0);
    }
}

// The candidates' squared norms, slot d B + j = ||x_j||^2 for every row d
// (x_j the reconstruction of the batch's candidate j), 0 past the count: the
// plaintext the expanded distance ||q||^2 - 2 <q, x_j> + ||x_j||^2 adds after
// the tree sum has left its other two terms in every row. With B = N/2 (one
// row) slot j = ||x_j||^2: a unit of the diagonal method.
__global__ void fft_load_pq_norms(double2* __restrict__ v, uint32_t s, uint32_t dim, uint32_t M, uint32_t K,
                                  const float* __restrict__ cent, const float* __restrict__ cb,
                                  const uint8_t* __restrict__ codes, const uint32_t* __restrict__ assign,
                                  const uint32_t* __restrict__ vids, const uint32_t* __restrict__ first,
                                  const uint32_t* __restrict__ cnt, uint32_t B, uint32_t count) {
    const uint32_t sd = dim / M;
    const u64 total = (u64)count * s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t / s), j = (uint32_t)(t % s) % B;
        double x2 = 0.0;
        if (j < cnt[z]) {
            const uint32_t id = vids[first[z] + j];
            const float* c = cent + (u64)assign[id] * dim;
            for (uint32_t m = 0; m < M; ++m) {
                const float* w = cb + ((u64)m * K + codes[(u64)id * M + m]) * sd;
                for (uint32_t e = 0; e < sd; ++e) {
                    const double x = (double)c[m * sd + e] + (double)w[e];
                    x2 += x * x;
                }
            }
        }
        v[t] = make_double2(x2, 0.0);
    }
}

// The diagonals of a unit of up to N/2 candidates (the diagonal method's
// plaintexts): plaintext i = g n1 + b of unit z, slot k, holds coef x_j[(j +
// i) mod dim] for the candidate j = (k - n1 g) mod (N/2) of the unit (0 past
// its count). That is diagonal i of the (candidates x dim) matrix, whose
// slot j multiplies slot j of the query rotated by i, pre-rotated by -n1 g
// for the giant step that brings it back.
__global__ void fft_load_pq_diag(double2* __restrict__ v, uint32_t s, uint32_t dim, uint32_t M, uint32_t K,
                                 const float* __restrict__ cent, const float* __restrict__ cb,
                                 const uint8_t* __restrict__ codes, const uint32_t* __restrict__ assign,
                                 const uint32_t* __restrict__ vids, const uint32_t* __restrict__ first,
                                 const uint32_t* __restrict__ cnt, uint32_t n1, double coef, uint32_t pt0,
                                 uint32_t count) {
    const uint32_t sd = dim / M;
    const u64 total = (u64)count * s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = pt0 + (uint32_t)(t / s), slot = (uint32_t)(t % s);
        const uint32_t unit = z / dim, i = z % dim, g = i / n1;
        const uint32_t j = (slot + s - (n1 * g) % s) % s;
        double x = 0.0;
        if (j < cnt[unit]) {
            const uint32_t id = vids[first[unit] + j];
            const uint32_t d = (j + i) % dim, m = d / sd;
            x = coef * ((double)cent[(u64)assign[id] * dim + d] +
                        (double)cb[((u64)m * K + codes[(u64)id * M + m]) * sd + (d - m * sd)]);
        }
        v[t] = make_double2(x, 0.0);
    }
}

int grid_for(u64 work) {
    u64 b = (work + 255) / 256;
    return (int)(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

// The special FFT and the RNS store of `count` slot vectors already in v.
int finish_chunk(afhe_ctx* ctx, const FftTables& tb, double2* v, uint32_t count, double scale, uint32_t level,
                 const u64* pt_dev, const u64* pt_host, const u64* q_dev, int* overflow) {
    const uint32_t s = ctx->n / 2;
    const uint32_t tile = s < kTile ? s : kTile;
    for (uint32_t len = s; len > tile; len >>= 1) {
        fft_global_stage<<<grid_for((u64)count * s / 2), 256, 0, ctx->st>>>(v, s, len, count, tb.ksi, tb.rot);
        count_launches(1);
    }
    const size_t smem = tile * sizeof(double2);
    CK(cudaFuncSetAttribute(fft_tile_stages, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fft_tile_stages<<<dim3(s / tile, count), kTileThreads, smem, ctx->st>>>(v, s, tile, tb.ksi, tb.rot);
    count_launches(1);
    uint32_t log_s = 0;
    while ((1u << log_s) < s) ++log_s;
    fft_finish<<<grid_for((u64)count * s), 256, 0, ctx->st>>>(v, log_s, scale, q_dev, level, ctx->poly, pt_dev, count,
                                                               overflow);
    count_launches(1);
    CK(cudaGetLastError());
    return afhe_ntt_batch(ctx, pt_host, count, level, 0);
}

// Shared driver: `load(v, c0, m)` fills v with plaintexts [c0, c0 + m).
// ---- decoding (the client's side): the forward special FFT ----------------
// Slot j of m = sum c_k X^k is m(zeta^(5^j)). With v_i = (c_i + i c_{i+N/2}) /
// scale, the encoder's transform inverted: bit reversal, then the stages of
// block length 2 .. N/2, each (a, b) -> (a + w b, a - w b) with w =
// ksi^((5^j mod 4 len) 2N / (4 len)); slot j is then v_j.
__device__ __forceinline__ void special_bfly_fwd(double2& a, double2& b, uint32_t j, uint32_t len, uint32_t m,
                                                 const double2* __restrict__ ksi, const uint32_t* __restrict__ rot) {
    const uint32_t lenq = len << 2;
    const uint32_t idx = (__ldg(rot + j) & (lenq - 1)) * (m / lenq);
    const double2 t = cmul(b, __ldg(ksi + idx));
    b = make_double2(a.x - t.x, a.y - t.y);
    a = make_double2(a.x + t.x, a.y + t.y);
}

// limb 0 of each decrypted polynomial (coefficient form), centred mod q_0,
// / scale, paired (c_i, c_{i+N/2}) at the bit-reversed position of i
__global__ void dec_load(double2* __restrict__ v, const u64* __restrict__ arena, const u64* __restrict__ coef,
                         const double* __restrict__ scales, u64 q0, uint32_t log_s, uint32_t count) {
    const uint32_t s = 1u << log_s;
    const u64 total = (u64)count * s;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t >> log_s), i = (uint32_t)(t & (s - 1));
        const u64* c = arena + coef[z];
        const u64 a = c[i], b = c[i + s];
        const double inv = 1.0 / scales[z];
        const double re = (double)(a > q0 / 2 ? -(long long)(q0 - a) : (long long)a) * inv;
        const double im = (double)(b > q0 / 2 ? -(long long)(q0 - b) : (long long)b) * inv;
        v[(u64)z * s + (__brev(i) >> (32 - log_s))] = make_double2(re, im);
    }
}

// the stages of block length 2 .. tile in shared memory, one tile per CTA
__global__ void __launch_bounds__(kTileThreads) dec_tile_stages(double2* __restrict__ v, uint32_t s, uint32_t tile,
                                                                const double2* __restrict__ ksi,
                                                                const uint32_t* __restrict__ rot) {
    extern __shared__ double2 sm2[];
    const uint32_t m = 4 * s;
    double2* g = v + (u64)blockIdx.y * s + (u64)blockIdx.x * tile;
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) sm2[e] = g[e];
    __syncthreads();
    for (uint32_t len = 2; len <= tile; len <<= 1) {
        const uint32_t lenh = len >> 1;
        for (uint32_t b = threadIdx.x; b < tile / 2; b += blockDim.x) {
            const uint32_t blk = b / lenh, j = b % lenh;
            special_bfly_fwd(sm2[blk * len + j], sm2[blk * len + j + lenh], j, len, m, ksi, rot);
        }
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) g[e] = sm2[e];
}

// one stage of block length above a tile, in global memory
__global__ void dec_global_stage(double2* __restrict__ v, uint32_t s, uint32_t len, uint32_t count,
                                 const double2* __restrict__ ksi, const uint32_t* __restrict__ rot) {
    const uint32_t half = s / 2, lenh = len >> 1, m = 4 * s;
    const u64 total = (u64)count * half;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const uint32_t z = (uint32_t)(t / half), b = (uint32_t)(t % half);
        const uint32_t blk = b / lenh, j = b % lenh;
        double2* p = v + (u64)z * s + (u64)blk * len + j;
        double2 a = p[0], c = p[lenh];
        special_bfly_fwd(a, c, j, len, m, ksi, rot);
        p[0] = a;
        p[lenh] = c;
    }
}

// the real parts of slots 0 .. slots - 1
__global__ void dec_store(const double2* __restrict__ v, double* __restrict__ out, uint32_t s, uint32_t slots,
                          uint32_t count) {
    const u64 total = (u64)count * slots;
    for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x)
        out[t] = v[(t / slots) * s + t % slots].x;
}

template <class Load>
int encode_pipeline(afhe_ctx* ctx, uint32_t count, double scale, uint32_t level, const uint64_t* pt, Load load) {
    if (!(scale > 0.0) || !std::isfinite(scale)) return fail(ctx, AFHE_E_ARG, "scale must be positive and finite");
    if (level < 1 || level > ctx->L) return fail(ctx, AFHE_E_LEVEL, "level outside [1, L]");
    for (uint32_t i = 0; i < count; ++i)
        if (!range_ok(pt[i], (u64)level * ctx->n, ctx->prm.poly_words))
            return fail(ctx, AFHE_E_RANGE, "plaintext out of range");
    if (count == 0) return AFHE_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
    FftTables tb;
    CK(fft_tables(ctx->device, ctx->n, ctx->st, &tb));
    const uint32_t s = ctx->n / 2, chunk = count < kChunkPts ? count : kChunkPts;
    double2* v = nullptr;
    u64 *q_dev = nullptr, *pt_dev = nullptr;
    int* overflow = nullptr;
    int rc = AFHE_OK;
    cudaError_t e = cudaMalloc(&v, (size_t)chunk * s * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&q_dev, ctx->L * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&pt_dev, (size_t)count * sizeof(u64));
    if (e == cudaSuccess) e = cudaMalloc(&overflow, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyAsync(q_dev, ctx->prm.q, ctx->L * sizeof(u64), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pt_dev, pt, (size_t)count * sizeof(u64), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(overflow, 0, sizeof(int), ctx->st);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "encode buffers");
    for (uint32_t c0 = 0; rc == AFHE_OK && c0 < count; c0 += chunk) {
        const uint32_t m = count - c0 < chunk ? count - c0 : chunk;
        rc = load(v, c0, m);
        if (rc == AFHE_OK) rc = finish_chunk(ctx, tb, v, m, scale, level, pt_dev + c0, pt + c0, q_dev, overflow);
    }
    int of = 0;
    if (rc == AFHE_OK) {
        e = cudaMemcpyAsync(&of, overflow, sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "encode");
        else if (of) rc = fail(ctx, AFHE_E_ARG, "encoded coefficients exceed 62 bits; lower the scale");
    } else {
        cudaStreamSynchronize(ctx->st);
    }
    cudaFree(v);
    cudaFree(q_dev);
    cudaFree(pt_dev);
    cudaFree(overflow);
    return rc;
}

}  // namespace
}  // namespace afhe

extern "C" {

int afhe_decode_batch(afhe_ctx* ctx, const uint64_t* coef, const double* scales, uint32_t count, uint32_t slots,
                      double* out) {
    if (!ctx || (count && (!coef || !scales || !out))) return fail(ctx, AFHE_E_ARG, "null argument");
    const uint32_t s = ctx->n / 2;
    if (slots < 1 || slots > s) return fail(ctx, AFHE_E_ARG, "slots must be in [1, N/2]");
    if (ctx->prm.q[0] >= (1ull << 53)) return fail(ctx, AFHE_E_ARG, "q_0 must be below 2^53 (exact doubles)");
    for (uint32_t i = 0; i < count; ++i) {
        if (!range_ok(coef[i], ctx->n, ctx->prm.poly_words)) return fail(ctx, AFHE_E_RANGE, "polynomial out of range");
        if (!(scales[i] > 0.0) || !std::isfinite(scales[i])) return fail(ctx, AFHE_E_ARG, "scales must be positive");
    }
    if (count == 0) return AFHE_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
    FftTables tb;
    CK(fft_tables(ctx->device, ctx->n, ctx->st, &tb));
    uint32_t log_s = 0;
    while ((1u << log_s) < s) ++log_s;
    const uint32_t chunk = kChunkPts, tile = s < kTile ? s : kTile;
    // one workspace per context, grown on demand: v (chunk x s), res (chunk
    // x slots), the scales and offsets of the call
    const size_t need = (size_t)chunk * s * sizeof(double2) + (size_t)chunk * s * sizeof(double) +
                        (size_t)count * (sizeof(double) + sizeof(u64));
    int rc = AFHE_OK;
    cudaError_t e = cudaSuccess;
    if (ctx->dec_ws_bytes < need) {
        if (ctx->dec_ws) {
            cudaStreamSynchronize(ctx->st);
            cudaFree(ctx->dec_ws);
            ctx->dec_ws = nullptr;
            ctx->dec_ws_bytes = 0;
        }
        const size_t grow = std::max(need, 2 * ctx->dec_ws_bytes);
        e = cudaMalloc(&ctx->dec_ws, grow);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "decode workspace");
        ctx->dec_ws_bytes = grow;
    }
    double2* v = (double2*)ctx->dec_ws;
    double* res = (double*)(v + (size_t)chunk * s);
    double* sc = res + (size_t)chunk * s;
    u64* cf = (u64*)(sc + count);
    e = cudaMemcpyAsync(sc, scales, (size_t)count * sizeof(double), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cf, coef, (size_t)count * sizeof(u64), cudaMemcpyHostToDevice, ctx->st);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "decode buffers");
    const size_t smem = tile * sizeof(double2);
    if (rc == AFHE_OK) {
        e = cudaFuncSetAttribute(dec_tile_stages, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "decode smem");
    }
    for (uint32_t c0 = 0; rc == AFHE_OK && c0 < count; c0 += chunk) {
        const uint32_t m = count - c0 < chunk ? count - c0 : chunk;
        dec_load<<<grid_for((u64)m * s), 256, 0, ctx->st>>>(v, ctx->poly, cf + c0, sc + c0, ctx->prm.q[0], log_s, m);
        dec_tile_stages<<<dim3(s / tile, m), kTileThreads, smem, ctx->st>>>(v, s, tile, tb.ksi, tb.rot);
        for (uint32_t len = 2 * tile; len <= s; len <<= 1)
            dec_global_stage<<<grid_for((u64)m * s / 2), 256, 0, ctx->st>>>(v, s, len, m, tb.ksi, tb.rot);
        dec_store<<<grid_for((u64)m * slots), 256, 0, ctx->st>>>(v, res, s, slots, m);
        count_launches(3 + (s > tile ? log_s - (31 - __builtin_clz(tile)) : 0));
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out + (size_t)c0 * slots, res, (size_t)m * slots * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);    // res is reused by the next chunk
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "decode");
    }
    if (rc != AFHE_OK) cudaStreamSynchronize(ctx->st);
    return rc;
}

int afhe_encode_batch(afhe_ctx* ctx, const double* values, uint32_t count, uint32_t slots, double scale,
                      uint32_t level, const uint64_t* pt) {
    if (!ctx || (count && (!values || !pt))) return fail(ctx, AFHE_E_ARG, "null argument");
    if (slots > ctx->n / 2) return fail(ctx, AFHE_E_ARG, "more values than slots");
    double* rows = nullptr;
    auto load = [&](double2* v, uint32_t c0, uint32_t m) -> int {
        const size_t bytes = (size_t)m * slots * sizeof(double);
        if (!rows) CK(cudaMalloc(&rows, (size_t)(count < kChunkPts ? count : kChunkPts) * (slots ? slots : 1) *
                                            sizeof(double)));
        if (bytes) CK(cudaMemcpyAsync(rows, values + (size_t)c0 * slots, bytes, cudaMemcpyHostToDevice, ctx->st));
        fft_load_rows<<<grid_for((u64)m * ctx->n / 2), 256, 0, ctx->st>>>(v, rows, ctx->n / 2, slots, m);
        count_launches(1);
        // the next chunk's copy reuses `rows`: it is ordered after this load on the stream
        return AFHE_OK;
    };
    int rc = encode_pipeline(ctx, count, scale, level, pt, load);
    if (rows) cudaFree(rows);
    return rc;
}

int afhe_pq_create(afhe_ctx* ctx, const afhe_pq_index* ix, afhe_pq** out) {
    if (!ctx || !ix || !out || !ix->centroids || !ix->codebooks || (ix->n && (!ix->codes || !ix->assignments)))
        return fail(ctx, AFHE_E_ARG, "null argument");
    if (ix->M == 0 || ix->d % ix->M || ix->K == 0 || ix->K > 256 || ix->n_list == 0)
        return fail(ctx, AFHE_E_ARG, "index shape: M divides d, 1 <= K <= 256");
    for (uint64_t i = 0; i < ix->n; ++i)
        if (ix->assignments[i] >= ix->n_list) return fail(ctx, AFHE_E_ARG, "assignment outside the lists");
    for (uint64_t i = 0; i < ix->n * ix->M; ++i)
        if (ix->codes[i] >= ix->K) return fail(ctx, AFHE_E_ARG, "code outside the codebook");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AFHE_E_CUDA, "cudaSetDevice");
    afhe_pq* p = new afhe_pq();
    p->ctx = ctx;
    p->n_list = ix->n_list;
    p->d = ix->d;
    p->M = ix->M;
    p->K = ix->K;
    p->n = ix->n;
    const size_t cbytes = (size_t)ix->n_list * ix->d * sizeof(float), bbytes = (size_t)ix->K * ix->d * sizeof(float);
    cudaError_t e = cudaMalloc(&p->centroids, cbytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->codebooks, bbytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->codes, ix->n * ix->M + 1);
    if (e == cudaSuccess) e = cudaMalloc(&p->assign, ix->n * sizeof(uint32_t) + 4);
    if (e == cudaSuccess) e = cudaMemcpy(p->centroids, ix->centroids, cbytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->codebooks, ix->codebooks, bbytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ix->n) e = cudaMemcpy(p->codes, ix->codes, ix->n * ix->M, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ix->n)
        e = cudaMemcpy(p->assign, ix->assignments, ix->n * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        afhe_pq_destroy(p);
        return cuda_fail(ctx, e, "index upload");
    }
    *out = p;
    return AFHE_OK;
}

int afhe_pq_destroy(afhe_pq* p) {
    if (!p) return AFHE_OK;
    cudaFree(p->centroids);
    cudaFree(p->codebooks);
    cudaFree(p->codes);
    cudaFree(p->assign);
    delete p;
    return AFHE_OK;
}

namespace {
enum PqLayout { PQ_BATCHES, PQ_NORMS, PQ_DIAGONALS, PQ_UNIT_NORMS };
int pq_encode(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt, uint32_t batches,
              double scale, uint32_t level, const uint64_t* pt, PqLayout layout, uint32_t n1 = 0, double coef = 1.0);
}

int afhe_pq_encode_batches(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt,
                           uint32_t batches, double scale, uint32_t level, const uint64_t* pt) {
    return pq_encode(p, vids, first, cnt, batches, scale, level, pt, PQ_BATCHES);
}

int afhe_pq_encode_norms(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt,
                         uint32_t batches, double scale, uint32_t level, const uint64_t* pt) {
    return pq_encode(p, vids, first, cnt, batches, scale, level, pt, PQ_NORMS);
}

int afhe_pq_encode_diagonals(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt,
                             uint32_t units, uint32_t n1, double coef, double scale, uint32_t level,
                             const uint64_t* pt) {
    return pq_encode(p, vids, first, cnt, units, scale, level, pt, PQ_DIAGONALS, n1, coef);
}

int afhe_pq_encode_unit_norms(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt,
                              uint32_t units, double scale, uint32_t level, const uint64_t* pt) {
    return pq_encode(p, vids, first, cnt, units, scale, level, pt, PQ_UNIT_NORMS);
}

}  // extern "C"

namespace {
int pq_encode(afhe_pq* p, const uint32_t* vids, const uint32_t* first, const uint32_t* cnt, uint32_t batches,
              double scale, uint32_t level, const uint64_t* pt, PqLayout layout, uint32_t n1, double coef) {
    if (!p) return fail(nullptr, AFHE_E_ARG, "null argument");
    afhe_ctx* ctx = p->ctx;
    if (batches && (!vids || !first || !cnt || !pt)) return fail(ctx, AFHE_E_ARG, "null argument");
    const uint32_t s = ctx->n / 2;
    if (p->d > s || s % p->d) return fail(ctx, AFHE_E_ARG, "the dimension must divide N/2");
    const bool unit = layout == PQ_DIAGONALS || layout == PQ_UNIT_NORMS;
    const uint32_t B = unit ? s : s / p->d;
    if (layout == PQ_DIAGONALS && (n1 == 0 || p->d % n1))
        return fail(ctx, AFHE_E_ARG, "the baby steps must divide the dimension");
    if (layout == PQ_DIAGONALS && !std::isfinite(coef)) return fail(ctx, AFHE_E_ARG, "coefficient must be finite");
    uint64_t total = 0;
    for (uint32_t b = 0; b < batches; ++b) {
        if (cnt[b] > B) return fail(ctx, AFHE_E_ARG, unit ? "more candidates in a unit than N / 2"
                                                          : "more candidates in a batch than N / 2d");
        total = std::max<uint64_t>(total, (uint64_t)first[b] + cnt[b]);
    }
    std::vector<uint32_t> ids(vids, vids + total);
    for (uint32_t id : ids)
        if (id >= p->n) return fail(ctx, AFHE_E_ARG, "candidate id outside the index");
    uint32_t *vids_d = nullptr, *first_d = nullptr, *cnt_d = nullptr;
    auto release = [&]() {
        cudaFree(vids_d);
        cudaFree(first_d);
        cudaFree(cnt_d);
    };
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = cudaMalloc(&vids_d, (total + 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&first_d, ((size_t)batches + 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&cnt_d, ((size_t)batches + 1) * sizeof(uint32_t));
    if (e == cudaSuccess && total) e = cudaMemcpy(vids_d, ids.data(), total * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && batches) e = cudaMemcpy(first_d, first, batches * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && batches) e = cudaMemcpy(cnt_d, cnt, batches * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(ctx, e, "batch upload");
    }
    auto load = [&](double2* v, uint32_t c0, uint32_t m) -> int {
        if (layout == PQ_NORMS || layout == PQ_UNIT_NORMS)
            fft_load_pq_norms<<<grid_for((u64)m * s), 256, 0, ctx->st>>>(v, s, p->d, p->M, p->K, p->centroids,
                                                                         p->codebooks, p->codes, p->assign, vids_d,
                                                                         first_d + c0, cnt_d + c0, B, m);
        else if (layout == PQ_DIAGONALS)       // plaintexts c0 .. c0 + m - 1 of units x dim
            fft_load_pq_diag<<<grid_for((u64)m * s), 256, 0, ctx->st>>>(v, s, p->d, p->M, p->K, p->centroids,
                                                                        p->codebooks, p->codes, p->assign, vids_d,
                                                                        first_d, cnt_d, n1, coef, c0, m);
        else
            fft_load_pq<<<grid_for((u64)m * s), 256, 0, ctx->st>>>(v, s, p->d, p->M, p->K, p->centroids,
                                                                   p->codebooks, p->codes, p->assign, vids_d,
                                                                   first_d + c0, cnt_d + c0, m);
        count_launches(1);
        return AFHE_OK;
    };
    const uint64_t n_pts = layout == PQ_DIAGONALS ? (uint64_t)batches * p->d : batches;
    if (n_pts > 0xffffffffull) {
        release();
        return fail(ctx, AFHE_E_ARG, "too many plaintexts in one call");
    }
    int rc = encode_pipeline(ctx, (uint32_t)n_pts, scale, level, pt, load);
    release();
    return rc;
}
}  // namespace
