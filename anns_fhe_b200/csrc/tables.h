// tables.h -- host-side number theory for the CKKS evaluation core: NTT-friendly
// primes, primitive 2N-th roots, twiddle tables and the RNS/CRT constants the
// reference reads from OpenFHE-generated files.
//
// The layouts follow what the reference's kernels index:
//   * twiddles tw[j] = psi^bitrev(j, log N), inverse itw[j] = psi^-bitrev(j)
//     (integration_tools/test_vector_generator.cpp:151-177);
//   * Barrett m = floor(2^k / q), k = 2*bits(q) + 3 (test_vector_generator.cpp:128-133);
//   * PartQlHatInvModq / PartQlHatModp per digit, row-major [i][j]
//     (hardware_fpga_model/hls/src/key_switch.cpp:7-60);
//   * PInvModq, PHatInvModp, PHatModq [k][i] (key_switch.cpp:62-163);
//   * QlQlInvModqlDivqlModq, qlInvModq (hardware_fpga_model/hls/src/rescale.cpp:3-72).
#pragma once
#include <cstdint>
#include <vector>

namespace afhe {

typedef uint64_t u64;

u64 pow_mod(u64 b, u64 e, u64 q);
u64 inv_mod(u64 a, u64 q);  // q prime
bool is_prime64(u64 n);
uint32_t bitrev(uint32_t x, int bits);

// The `count` largest primes q < 2^bits with q == 1 (mod 2N), in descending
// order, skipping any value listed in `exclude`.
std::vector<u64> find_ntt_primes(uint32_t log_n, uint32_t bits, uint32_t count,
                                 const std::vector<u64>& exclude);

// Smallest primitive 2N-th root of unity modulo q (minimum over all of them).
u64 min_primitive_root(uint32_t log_n, u64 q);

void gen_twiddles(uint32_t log_n, u64 q, u64 psi, u64* tw, u64* itw);

void barrett_constant(u64 q, u64* m_lo, u64* m_hi, uint32_t* k);

// Galois element 5^step mod 2N (step < 0 uses 5^-1), the rotation-by-step map.
uint32_t galois_elt_for_step(uint32_t log_n, int32_t step);

// Evaluation-form automorphism map for Galois element k on the bit-reversed
// NTT layout: out[i] = in[map[i]].
void automorphism_map(uint32_t log_n, uint32_t galois_elt, uint32_t* map);

// Digit `part` at level `sizeQl` (alpha limbs per digit, last digit shorter):
// qhat_inv[size_part], qhat_modp[size_part * (sizeQl - size_part + K)], the
// complementary primes ordered as the other Q primes ascending, then P.
void part_qhat_tables(const u64* q, uint32_t sizeQl, uint32_t alpha, uint32_t part,
                      const u64* p, uint32_t K, u64* qhat_inv, u64* qhat_modp);

// ModDown constants at level sizeQl: p_inv_mod_q[sizeQl], phat_inv_mod_p[K],
// phat_mod_q[K * sizeQl] (row k, column i).
void moddown_tables(const u64* q, uint32_t sizeQl, const u64* p, uint32_t K,
                    u64* p_inv_mod_q, u64* phat_inv_mod_p, u64* phat_mod_q);

// Rescale constants for dropping limb sizeQl-1: qlql[i], qlinv[i] for i < sizeQl-1.
void rescale_tables(const u64* q, uint32_t sizeQl, u64* qlql, u64* qlinv);

}  // namespace afhe
