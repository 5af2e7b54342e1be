// modarith.cuh -- 64-bit RNS modular arithmetic for the CKKS evaluation core.
//
// Replaces the reference's Barrett mod_mul (hardware_fpga_model/hls/src/
// mod_arith.cpp:15-25, 128-bit m, 192-bit intermediate) with forms that map to
// the B200 integer pipe:
//   * Shoup multiplication by a constant w with companion w' = floor(w*2^64/q):
//     one __umul64hi + two 64-bit multiplies, result in [0, 2q) (lazy);
//   * a general 128-bit reduction (reduce128) for products of two variables,
//     built from two Shoup steps with the constants 2^64 mod q and 1.
// Every routine returns a value congruent to the exact product; callers
// canonicalise into [0, q) before any store that leaves the kernel, so results
// are bit-identical to the reference's exact residues.
//
// Valid for odd moduli q < 2^62 (so that 4q fits in 64 bits).
// All functions are __host__ __device__ so the CPU test suite exercises the
// same code the kernels run.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define AFHE_HD __host__ __device__ __forceinline__
#else
#define AFHE_HD inline
#endif

namespace afhe {

typedef uint64_t u64;

AFHE_HD u64 mulhi64(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

// floor(w * 2^64 / q) for w < q: the Shoup companion of w. Bitwise long
// division so it runs identically on host and device.
AFHE_HD u64 shoup_companion(u64 w, u64 q) {
    // numerator = w * 2^64; divide 128-bit (w, 0) by q, w < q so quotient < 2^64.
    u64 rem = w, quo = 0;
    for (int i = 0; i < 64; ++i) {
        // shift (rem, next bit 0) left by one; rem < q < 2^62 so no overflow
        rem <<= 1;
        quo <<= 1;
        if (rem >= q) { rem -= q; quo |= 1; }
    }
    return quo;
}

// a * w mod q, lazy: result in [0, 2q). Valid for any a < 2^64.
AFHE_HD u64 mul_shoup_lazy(u64 a, u64 w, u64 wsh, u64 q) {
    u64 t = mulhi64(a, wsh);
    return a * w - t * q;
}

AFHE_HD u64 csub(u64 x, u64 q) { return x >= q ? x - q : x; }

AFHE_HD u64 mul_shoup(u64 a, u64 w, u64 wsh, u64 q) { return csub(mul_shoup_lazy(a, w, wsh, q), q); }

AFHE_HD u64 add_mod(u64 a, u64 b, u64 q) { return csub(a + b, q); }
AFHE_HD u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }

// Per-modulus constants for reduce128: r64 = 2^64 mod q with its Shoup
// companion, and one_sh = floor(2^64 / q) (the companion of 1).
struct ModConst {
    u64 q;
    u64 r64;
    u64 r64_sh;
    u64 one_sh;
};

AFHE_HD ModConst make_modconst(u64 q) {
    ModConst m;
    m.q = q;
    // 2^64 mod q = (2^64 - q) mod q computed without overflow
    u64 t = (u64)0 - q;            // 2^64 - q
    m.r64 = t % q;
    m.r64_sh = shoup_companion(m.r64, q);
    m.one_sh = shoup_companion(1, q);
    return m;
}

// (hi * 2^64 + lo) mod q, exact, any 128-bit input, canonical output.
AFHE_HD u64 reduce128(u64 hi, u64 lo, const ModConst& m) {
    u64 a = mul_shoup_lazy(hi, m.r64, m.r64_sh, m.q);  // [0, 2q)
    u64 b = mul_shoup_lazy(lo, 1, m.one_sh, m.q);       // [0, 2q)
    u64 s = a + b;                                      // [0, 4q)
    u64 q2 = m.q << 1;
    s = s >= q2 ? s - q2 : s;
    return csub(s, m.q);
}

// a * b mod q for two variable operands, canonical.
AFHE_HD u64 mul_mod(u64 a, u64 b, const ModConst& m) {
    return reduce128(mulhi64(a, b), a * b, m);
}

// 128-bit accumulator for sums of products (key-switch inner product).
struct Acc128 {
    u64 lo, hi;
};
AFHE_HD void acc_init(Acc128& a) { a.lo = 0; a.hi = 0; }
AFHE_HD void acc_mad(Acc128& a, u64 x, u64 y) {
    u64 plo = x * y;
    u64 phi = mulhi64(x, y);
    u64 nlo = a.lo + plo;
    a.hi += phi + (nlo < plo ? 1 : 0);
    a.lo = nlo;
}
AFHE_HD u64 acc_reduce(const Acc128& a, const ModConst& m) { return reduce128(a.hi, a.lo, m); }

}  // namespace afhe
