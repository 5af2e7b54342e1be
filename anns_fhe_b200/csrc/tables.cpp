// tables.cpp -- host-side number theory (see tables.h).
#include "tables.h"

#include <algorithm>
#include <stdexcept>

namespace afhe {

typedef unsigned __int128 u128;

static inline u64 mulmod(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }

u64 pow_mod(u64 b, u64 e, u64 q) {
    u64 r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = mulmod(r, b, q);
        b = mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}

u64 inv_mod(u64 a, u64 q) { return pow_mod(a % q, q - 2, q); }

// Deterministic Miller-Rabin for 64-bit integers (first 12 prime bases).
bool is_prime64(u64 n) {
    if (n < 2) return false;
    static const u64 small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (u64 p : small) {
        if (n % p == 0) return n == p;
    }
    u64 d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    for (u64 a : small) {
        u64 x = pow_mod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = false; break; }
        }
        if (comp) return false;
    }
    return true;
}

uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

std::vector<u64> find_ntt_primes(uint32_t log_n, uint32_t bits, uint32_t count,
                                 const std::vector<u64>& exclude) {
    if (bits < log_n + 2 || bits > 61) throw std::invalid_argument("prime bit size out of range");
    const u64 m = 2ull << log_n;  // 2N
    // largest candidate < 2^bits with candidate == 1 mod 2N
    u64 c = ((1ull << bits) - 1) / m * m + 1;
    if (c >= (1ull << bits)) c -= m;
    std::vector<u64> out;
    while (out.size() < count) {
        if (c <= m) throw std::runtime_error("ran out of NTT-friendly primes");
        if (is_prime64(c) && std::find(exclude.begin(), exclude.end(), c) == exclude.end()) out.push_back(c);
        c -= m;
    }
    return out;
}

u64 min_primitive_root(uint32_t log_n, u64 q) {
    const u64 m = 2ull << log_n;
    if ((q - 1) % m != 0) throw std::invalid_argument("q != 1 mod 2N");
    u64 psi = 0;
    for (u64 g = 2; g < q; ++g) {
        u64 x = pow_mod(g, (q - 1) / m, q);
        if (pow_mod(x, m >> 1, q) == q - 1) { psi = x; break; }
    }
    // all primitive 2N-th roots are psi^(odd); take the smallest value
    u64 best = psi, cur = psi, psi2 = mulmod(psi, psi, q);
    for (u64 i = 1; i < (m >> 1); ++i) {
        cur = mulmod(cur, psi2, q);
        if (cur < best) best = cur;
    }
    return best;
}

void gen_twiddles(uint32_t log_n, u64 q, u64 psi, u64* tw, u64* itw) {
    const uint32_t n = 1u << log_n;
    u64 psi_inv = inv_mod(psi, q);
    std::vector<u64> pw(n), ipw(n);
    pw[0] = 1; ipw[0] = 1;
    for (uint32_t i = 1; i < n; ++i) { pw[i] = mulmod(pw[i - 1], psi, q); ipw[i] = mulmod(ipw[i - 1], psi_inv, q); }
    for (uint32_t j = 0; j < n; ++j) {
        uint32_t br = bitrev(j, (int)log_n);
        tw[j] = pw[br];
        itw[j] = ipw[br];
    }
}

void barrett_constant(u64 q, u64* m_lo, u64* m_hi, uint32_t* k) {
    uint32_t msb = 64 - __builtin_clzll(q);
    *k = 2 * msb + 3;
    u128 m = ((u128)1 << *k) / (u128)q;
    *m_lo = (u64)m;
    *m_hi = (u64)(m >> 64);
}

uint32_t galois_elt_for_step(uint32_t log_n, int32_t step) {
    const u64 m = 2ull << log_n;       // 2N
    const u64 order = m >> 2;          // multiplicative order of 5 mod 2N is N/2
    long long e = step % (long long)order;
    if (e < 0) e += (long long)order;
    u64 r = 1, b = 5 % m;
    u64 ee = (u64)e;
    while (ee) { if (ee & 1) r = r * b % m; b = b * b % m; ee >>= 1; }
    return (uint32_t)r;
}

// Slot i of the bit-reversed evaluation layout holds a(psi^(2*bitrev(i)+1)).
// sigma_k(a) evaluated there is a(psi^(k*(2*bitrev(i)+1))); that exponent is
// odd, 2*j'+1, and lives at index bitrev(j').
void automorphism_map(uint32_t log_n, uint32_t galois_elt, uint32_t* map) {
    const uint32_t n = 1u << log_n;
    const u64 m = 2ull * n;
    for (uint32_t i = 0; i < n; ++i) {
        u64 e = (u64)galois_elt * (2ull * bitrev(i, (int)log_n) + 1) % m;
        uint32_t jp = (uint32_t)((e - 1) >> 1);
        map[i] = bitrev(jp, (int)log_n);
    }
}

void part_qhat_tables(const u64* q, uint32_t sizeQl, uint32_t alpha, uint32_t part,
                      const u64* p, uint32_t K, u64* qhat_inv, u64* qhat_modp) {
    uint32_t num_parts = (sizeQl + alpha - 1) / alpha;
    uint32_t start = alpha * part;
    uint32_t size_part = (part == num_parts - 1) ? sizeQl - start : alpha;
    std::vector<u64> outp;
    for (uint32_t i = 0; i < sizeQl; ++i)
        if (i < start || i >= start + size_part) outp.push_back(q[i]);
    for (uint32_t k = 0; k < K; ++k) outp.push_back(p[k]);
    const uint32_t n_out = (uint32_t)outp.size();
    for (uint32_t i = 0; i < size_part; ++i) {
        u64 qi = q[start + i];
        // (Q_part / q_i)^-1 mod q_i
        u64 prod = 1;
        for (uint32_t t = 0; t < size_part; ++t)
            if (t != i) prod = mulmod(prod, q[start + t] % qi, qi);
        qhat_inv[i] = inv_mod(prod, qi);
        // (Q_part / q_i) mod p_j for each complementary prime
        for (uint32_t j = 0; j < n_out; ++j) {
            u64 pj = outp[j], r = 1;
            for (uint32_t t = 0; t < size_part; ++t)
                if (t != i) r = mulmod(r, q[start + t] % pj, pj);
            qhat_modp[(size_t)i * n_out + j] = r;
        }
    }
}

void moddown_tables(const u64* q, uint32_t sizeQl, const u64* p, uint32_t K,
                    u64* p_inv_mod_q, u64* phat_inv_mod_p, u64* phat_mod_q) {
    for (uint32_t i = 0; i < sizeQl; ++i) {
        u64 r = 1;
        for (uint32_t k = 0; k < K; ++k) r = mulmod(r, p[k] % q[i], q[i]);
        p_inv_mod_q[i] = inv_mod(r, q[i]);
    }
    for (uint32_t k = 0; k < K; ++k) {
        u64 r = 1;
        for (uint32_t t = 0; t < K; ++t)
            if (t != k) r = mulmod(r, p[t] % p[k], p[k]);
        phat_inv_mod_p[k] = inv_mod(r, p[k]);
        for (uint32_t i = 0; i < sizeQl; ++i) {
            u64 s = 1;
            for (uint32_t t = 0; t < K; ++t)
                if (t != k) s = mulmod(s, p[t] % q[i], q[i]);
            phat_mod_q[(size_t)k * sizeQl + i] = s;
        }
    }
}

// With Q' = prod_{i<l} q_i and t = floor(Q' * (Q'^-1 mod q_l) / q_l), the
// division is exact up to a remainder of 1, so q_l * t == -1 (mod q_i) and
// t mod q_i == -(q_l^-1) mod q_i: no big integers are needed.
void rescale_tables(const u64* q, uint32_t sizeQl, u64* qlql, u64* qlinv) {
    const u64 ql = q[sizeQl - 1];
    for (uint32_t i = 0; i + 1 < sizeQl; ++i) {
        u64 inv = inv_mod(ql % q[i], q[i]);
        qlinv[i] = inv;
        qlql[i] = inv == 0 ? 0 : q[i] - inv;
    }
}

}  // namespace afhe
