// ref_iqm_harness.cpp -- the reference's own host program behind a C interface.
//
// TEST INFRASTRUCTURE ONLY. SimMemoryBus, FHEHostDriver and
// InteractiveQueryManager (cpp_host_model/src/*.cpp) are compiled verbatim
// from the reference tree by oracle/Makefile, twice:
//   _ref/libref_iqm_cpu.so  with the reference's HLS fhe_accel_top (the CPU
//                           C-simulation, hardware_fpga_model/hls/src/*.cpp);
//   _ref/libref_iqm_gpu.so  with anns_fhe_b200/lib/libafhe_accel_top.so, this
//                           repository's fhe_accel_top over afhe_dispatch.
// The same unmodified host code then runs the reference's query stages on
// either, and tests/test_gpu_reference_host.py compares the arenas.
#include <cstdint>
#include <string>
#include <vector>

#include "sim_memory_bus.h"
#include "fhe_host_driver.h"
#include "interactive_query_manager.h"

namespace {
struct RefHost {
    SimMemoryBus bus;
    FHEHostDriver drv;
    InteractiveQueryManager iqm;
    explicit RefHost(uint64_t poly_words, uint64_t key_words)
        : bus(poly_words, key_words), drv(&bus), iqm(&drv) {}
};
}  // namespace

extern "C" {

// FHEHostDriver::initialize_context_from_directory (fhe_host_driver.cpp:18-175)
// then load_context_to_hardware (OP 99, :206-208).
void* rh_new(const char* vec_dir, uint64_t poly_words, uint64_t key_words) {
    RefHost* h = new RefHost(poly_words, key_words);
    h->drv.initialize_context_from_directory(vec_dir);
    h->drv.load_context_to_hardware();
    return h;
}

void rh_free(void* h) { delete static_cast<RefHost*>(h); }

void rh_write_poly(void* h, uint64_t off, const uint64_t* src, uint64_t count) {
    static_cast<RefHost*>(h)->bus.write_poly((uint32_t)off, src, count);
}

void rh_read_poly(void* h, uint64_t off, uint64_t* dst, uint64_t count) {
    static_cast<RefHost*>(h)->bus.read_poly((uint32_t)off, dst, count);
}

uint64_t rh_poly_words(void* h) { return static_cast<RefHost*>(h)->bus.poly_size_words(); }

// InteractiveQueryManager stage 1 (interactive_query_manager.cpp:85-119), as is.
void rh_stage1(void* h) { static_cast<RefHost*>(h)->iqm.stage1_coarse_centroid_distance(); }

// InteractiveQueryManager::stage1b_distance_compaction's loop
// (interactive_query_manager.cpp:121-178) through the same FHEHostDriver
// calls, with one change: mask i % 8 >= 4 is read from mask_hi + (i % 8 - 4) *
// 15N instead of SLOT_PT_MASK + (i % 8) * 15N. In the reference's map those
// four masks overlap SCRATCH_D0 .. SCRATCH_D2 (0x300000 + 4 * 15N > 0x400000),
// so scratch results overwrite them before they are read.
void rh_stage1b(void* h, uint32_t mask_hi) {
    RefHost* r = static_cast<RefHost*>(h);
    FHEHostDriver& d = r->drv;
    typedef InteractiveQueryManager Q;
    const uint32_t N = FHEHostDriver::N, D = 128, n_list = 32;
    bool first = true;
    std::vector<uint64_t> tmp(9 * N);
    for (uint32_t i = 0; i < n_list; ++i) {
        const uint32_t m = i % 8;
        const uint32_t mask = m < 4 ? Q::SLOT_PT_MASK + m * (15 * N) : mask_hi + (m - 4) * (15 * N);
        d.eval_mult_plain_rescale(Q::SLOT_CT_SQ_C0, Q::SLOT_CT_SQ_C1, mask, FHEHostDriver::SCRATCH_D0,
                                  FHEHostDriver::SCRATCH_D1, 10);
        const int shift = (int)(i * (D - 1));
        if (shift != 0) {
            d.eval_rotate(FHEHostDriver::SCRATCH_D0, FHEHostDriver::SCRATCH_D1, FHEHostDriver::SCRATCH_D2,
                          FHEHostDriver::SCRATCH_TMP, shift, 9);
        } else {
            r->bus.read_poly(FHEHostDriver::SCRATCH_D0, tmp.data(), tmp.size());
            r->bus.write_poly(FHEHostDriver::SCRATCH_D2, tmp.data(), tmp.size());
            r->bus.read_poly(FHEHostDriver::SCRATCH_D1, tmp.data(), tmp.size());
            r->bus.write_poly(FHEHostDriver::SCRATCH_TMP, tmp.data(), tmp.size());
        }
        if (first) {
            r->bus.read_poly(FHEHostDriver::SCRATCH_D2, tmp.data(), tmp.size());
            r->bus.write_poly(Q::SLOT_CT_COMPACT_C0, tmp.data(), tmp.size());
            r->bus.read_poly(FHEHostDriver::SCRATCH_TMP, tmp.data(), tmp.size());
            r->bus.write_poly(Q::SLOT_CT_COMPACT_C1, tmp.data(), tmp.size());
            first = false;
        } else {
            d.eval_add(Q::SLOT_CT_COMPACT_C0, Q::SLOT_CT_COMPACT_C1, FHEHostDriver::SCRATCH_D2,
                       FHEHostDriver::SCRATCH_TMP, Q::SLOT_CT_COMPACT_C0, Q::SLOT_CT_COMPACT_C1, 9);
        }
    }
}

// One FHEHostDriver composite (fhe_host_driver.cpp:272-306, :361-404).
void rh_eval_mult_relin_rescale(void* h, uint32_t a0, uint32_t a1, uint32_t d0, uint32_t d1, uint32_t limbs) {
    static_cast<RefHost*>(h)->drv.eval_mult_relin_rescale(a0, a1, a0, a1, d0, d1, limbs);
}

void rh_eval_rotate(void* h, uint32_t i0, uint32_t i1, uint32_t d0, uint32_t d1, int32_t total, uint32_t limbs) {
    static_cast<RefHost*>(h)->drv.eval_rotate(i0, i1, d0, d1, total, limbs);
}

}  // extern "C"
