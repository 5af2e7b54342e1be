// noalloc.cu -- a key switch that allocates nothing at call time.
//
// Some callers cannot call cudaMalloc on their request path: an application
// whose device memory is already handed to its own pool allocator (so a fresh
// cudaMalloc fails or steals from the pool), or a latency-bound serving thread
// that cannot afford the device-wide synchronisation cudaMalloc / cudaFree may
// imply. afhe_key_switch_noalloc gives them the key switch with its working
// memory in a fixed array compiled into this library instead of allocated
// memory: the array below is static device memory, held by every GPU that
// loads this library's module until the process exits, so its size is kept
// modest (16 MiB).
//
// With CUDA's lazy module loading the array is created when its module is
// first used on a device, and creating it allocates. So its address is looked
// up when a context is created (afhe_ctx_create calls
// noalloc_scratch_address with the context's device current), never on the
// entry point's path: by the time a caller's pool takes the GPU's memory, a
// context on that device already exists and the array is in place.
//
// The array is shared by every call on a device and keeps the previous call's
// contents. The key switch writes every scratch word before reading it, so no
// clearing is needed. Calls whose execution overlaps on the GPU (different
// streams, or several contexts on one device) race on the array; the caller
// must order them. The entry point always runs the multi-kernel key switch
// (INTT, ModUp NTT, inner product, ModDown), whatever the context's
// AFHE_OPT_KS_FUSED setting; the residues are the same either way.
#include <cuda_runtime.h>

#include "internal.h"
#include "lanes.h"

using namespace afhe;

namespace {

constexpr size_t kNoallocScratchWords = size_t(1) << 21;   // 16 MiB of uint64_t

static __device__ __align__(256) u64 g_noalloc_scratch[kNoallocScratchWords];

// Restores the caller's current device when the entry point returns.
struct DeviceGuard {
    int prev = -1;
    cudaError_t enter(int dev) {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) { prev = -1; return e; }
        return prev == dev ? cudaSuccess : cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

// Host code must not use g_noalloc_scratch's name as an address (on the host
// it names a shadow variable, not device memory): the device address comes
// from cudaGetSymbolAddress with the device current.
cudaError_t afhe::noalloc_scratch_address(u64** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    *out = e == cudaSuccess ? (u64*)p : nullptr;
    return e;
}

extern "C" int afhe_key_switch_noalloc(afhe_ctx* ctx, uint64_t* io, uint64_t evk_offset, uint32_t limbs) {
    if (!ctx || !io) return fail(ctx, AFHE_E_ARG, "null argument");
    if (limbs < 1 || limbs > ctx->L) return fail(ctx, AFHE_E_LEVEL, "limb count outside [1, L]");
    const u64 key_words = 2ull * ctx->dnum * (ctx->L + ctx->K) * ctx->n;
    if (!range_ok(evk_offset, key_words, ctx->prm.key_words)) return fail(ctx, AFHE_E_RANGE, "key out of key_gmem");
    const size_t need = ks_scratch_words(ctx->n, ctx->L, ctx->K, ctx->dnum);
    if (need > kNoallocScratchWords)
        return fail(ctx, AFHE_E_BUDGET,
                    "afhe_key_switch_noalloc: this parameter set needs " + std::to_string(need) +
                        " scratch words, more than the fixed " + std::to_string(kNoallocScratchWords));
    if (!ctx->noalloc_scr) return cuda_fail(ctx, ctx->noalloc_err, "cudaGetSymbolAddress(noalloc scratch) at context creation");
    DeviceGuard dg;
    cudaError_t e = dg.enter(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    const u64 w = (u64)limbs * ctx->n;
    ZBases zb{};
    zb.src = zf_const(0);        // input at io[0, w)
    zb.out = zf_const(w);        // ks0 at io[w, 2w)
    zb.aux = zf_const(2 * w);    // ks1 at io[2w, 3w)
    zb.mid = zf_const(0);        // scratch from the start of the fixed array
    const u64 S = (u64)ctx->L + ctx->K;
    const LevelJobs& lj = ctx->lvjobs[limbs];
    e = launch_key_switch(ctx->log_n, ctx->lv[limbs], ctx->jobs_qp, lj.modup, lj.n_modup, ctx->L, limbs, ctx->K,
                          ctx->key, evk_offset, evk_offset + (u64)ctx->dnum * S * ctx->n, (uint32_t)S, ctx->L, io,
                          ctx->noalloc_scr, 1, zb, ctx->st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "afhe_key_switch_noalloc launch");
    return AFHE_OK;
}
