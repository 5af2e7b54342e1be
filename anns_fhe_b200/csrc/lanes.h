// lanes.h -- layout of the context-private scratch used by the composite
// operators, and small shared helpers.
#pragma once
#include <string>

#include "internal.h"

namespace afhe {

inline bool range_ok(u64 off, u64 words, u64 size) { return off <= size && words <= size - off; }

// Error reporting shared by the C ABI sources (defined in api.cu): records the
// message for afhe_last_error() and returns `code`.
extern thread_local std::string g_last_error;
int fail(afhe_ctx* ctx, int code, const std::string& msg);
int cuda_fail(afhe_ctx* ctx, cudaError_t e, const char* where);
u64 host_shoup(u64 w, u64 q);
// Re-derive the prepared copies of registered keys that overlap key words
// [off, off + count) after they were overwritten (driver.cu).
int refresh_key_preps(afhe_ctx* ctx, u64 off, u64 count);
void free_key_preps(afhe_ctx* ctx);
// Device address of afhe_key_switch_noalloc's static working array on the
// current device (noalloc.cu). Loads the array's module if lazy loading has
// not yet done so, which is why contexts call it once at creation.
cudaError_t noalloc_scratch_address(u64** out);

#define CK(expr)                                                        \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::afhe::cuda_fail(ctx, _e, #expr); \
    } while (0)

// Scratch lane b owns [b * lane_words, (b + 1) * lane_words) of ctx->scr. A
// batched composite operator gives ciphertext b of a launch lane b; a context
// has ctx->lanes lanes (afhe_params.max_batch).
constexpr uint32_t kTempPolys = 6;  // d0, d1, d2, ks0, ks1, t (each (L + K) * N words)

struct Lane {
    u64 ks;      // key-switch scratch
    u64 resc;    // rescale scratch: 2 polys x L * N
    u64 temp;    // kTempPolys polys
};

inline u64 ks_words_ctx(const afhe_ctx* c) { return ks_scratch_words(c->n, c->L, c->K, c->dnum); }
inline u64 lane_words(const afhe_ctx* c) {
    return ks_words_ctx(c) + 2ull * c->L * c->n + (u64)kTempPolys * (c->L + c->K) * c->n;
}
inline Lane lane_of(const afhe_ctx* c, uint32_t b) {
    Lane l;
    u64 base = (u64)b * lane_words(c);
    l.ks = base;
    l.resc = l.ks + ks_words_ctx(c);
    l.temp = l.resc + 2ull * c->L * c->n;
    return l;
}
// offset of temp polynomial t of lane b, relative to the poly_gmem base
inline u64 lane_temp(const afhe_ctx* c, uint32_t b, uint32_t t) {
    return c->prm.poly_words + lane_of(c, b).temp + (u64)t * (c->L + c->K) * c->n;
}
// the same for lanes 0, 1, 2, ... as a strided field
inline ZField lane_temp_field(const afhe_ctx* c, uint32_t t) {
    return zf_stride(lane_temp(c, 0, t), lane_words(c));
}
inline ZField lane_field(const afhe_ctx* c, u64 Lane::*member) {
    return zf_stride(lane_of(c, 0).*member, lane_words(c));
}

// Field for per-ciphertext offsets vals[0..n): strided when they form an
// arithmetic progression, else staged through the context's descriptor ring.
int zf_from(afhe_ctx* ctx, const u64* vals, uint32_t n, ZField* out);
// Copy `words` words through the context's pinned descriptor ring to device
// memory, enqueued on the context stream; *dev stays valid for the work
// enqueued after it (the ring reuses a segment only once the stream has
// passed it).
int ring_put(afhe_ctx* ctx, const void* src, size_t words, u64** dev);

}  // namespace afhe
