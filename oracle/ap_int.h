// ap_int.h -- project-written stand-in for the Xilinx arbitrary-precision header.
//
// TEST INFRASTRUCTURE ONLY (oracle). It exists so that the reference HLS
// C-simulation sources (hardware_fpga_model/hls/src/*.cpp and
// cpp_host_model/src/*.cpp in iheydardoost/ANNS_FHE) compile unmodified with
// g++ and can serve as the bit-exact checker for the CUDA path. Nothing in the
// product links against it.
//
// Semantics implemented (the subset the reference uses):
//   * ap_uint<W>: unsigned W-bit integer, stored as little-endian 64-bit words,
//     value always reduced mod 2^W (bits above W are kept zero);
//   * construction from integral values and from other widths (truncating /
//     zero-extending), implicit conversion to uint64_t (low 64 bits);
//   * a * b widens to W1 + W2 bits (as the Xilinx header does), so
//     `(ap_uint<128>)a * b` is an exact 192-bit product before assignment;
//   * <<, >>, |, &, +, -, comparisons;
//   * bit-range get/set: x(hi, lo) and x.range(hi, lo) for hi - lo < 64.
#pragma once
#include <cstdint>
#include <cstring>
#include <type_traits>

template <int W>
struct ap_uint {
    static_assert(W > 0, "width must be positive");
    static constexpr int NW = (W + 63) / 64;
    uint64_t w[NW];

    void clear_top() {
        constexpr int rem = W % 64;
        if (rem) w[NW - 1] &= (~0ull) >> (64 - rem);
    }

    ap_uint() { std::memset(w, 0, sizeof(w)); }

    template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    ap_uint(T v) {
        std::memset(w, 0, sizeof(w));
        // negative values sign-extend as in two's complement, then truncate
        uint64_t lo = (uint64_t)(long long)v;
        if (std::is_signed<T>::value && (long long)v < 0) {
            for (int i = 0; i < NW; ++i) w[i] = ~0ull;
        }
        w[0] = lo;
        clear_top();
    }

    ap_uint(unsigned __int128 v) {
        std::memset(w, 0, sizeof(w));
        w[0] = (uint64_t)v;
        if (NW > 1) w[1] = (uint64_t)(v >> 64);
        clear_top();
    }

    template <int W2>
    ap_uint(const ap_uint<W2>& o) {
        std::memset(w, 0, sizeof(w));
        const int n = NW < ap_uint<W2>::NW ? NW : ap_uint<W2>::NW;
        for (int i = 0; i < n; ++i) w[i] = o.w[i];
        clear_top();
    }

    operator uint64_t() const { return w[0]; }

    // ---- shifts -------------------------------------------------------------
    template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    ap_uint operator<<(T s) const {
        ap_uint r;
        int sh = (int)s;
        if (sh >= W) return r;
        int ws = sh / 64, bs = sh % 64;
        for (int i = NW - 1; i >= 0; --i) {
            uint64_t v = 0;
            int src = i - ws;
            if (src >= 0) {
                v = w[src] << bs;
                if (bs && src - 1 >= 0) v |= w[src - 1] >> (64 - bs);
            }
            r.w[i] = v;
        }
        r.clear_top();
        return r;
    }
    template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    ap_uint operator>>(T s) const {
        ap_uint r;
        int sh = (int)s;
        if (sh >= W) return r;
        int ws = sh / 64, bs = sh % 64;
        for (int i = 0; i < NW; ++i) {
            uint64_t v = 0;
            int src = i + ws;
            if (src < NW) {
                v = w[src] >> bs;
                if (bs && src + 1 < NW) v |= w[src + 1] << (64 - bs);
            }
            r.w[i] = v;
        }
        return r;
    }

    // ---- bitwise / additive ops (same width) -------------------------------
    ap_uint operator|(const ap_uint& o) const { ap_uint r; for (int i = 0; i < NW; ++i) r.w[i] = w[i] | o.w[i]; return r; }
    ap_uint operator&(const ap_uint& o) const { ap_uint r; for (int i = 0; i < NW; ++i) r.w[i] = w[i] & o.w[i]; return r; }
    ap_uint operator+(const ap_uint& o) const {
        ap_uint r; unsigned __int128 c = 0;
        for (int i = 0; i < NW; ++i) { c += (unsigned __int128)w[i] + o.w[i]; r.w[i] = (uint64_t)c; c >>= 64; }
        r.clear_top(); return r;
    }
    ap_uint operator-(const ap_uint& o) const {
        ap_uint r; uint64_t borrow = 0;
        for (int i = 0; i < NW; ++i) {
            uint64_t a = w[i], b = o.w[i];
            uint64_t d = a - b - borrow;
            borrow = (a < b) || (a - b < borrow);
            r.w[i] = d;
        }
        r.clear_top(); return r;
    }
    template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    ap_uint operator|(T v) const { return *this | ap_uint(v); }
    template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
    ap_uint operator&(T v) const { return *this & ap_uint(v); }

    ap_uint& operator|=(const ap_uint& o) { *this = *this | o; return *this; }
    ap_uint& operator+=(const ap_uint& o) { *this = *this + o; return *this; }

    // ---- comparisons ---------------------------------------------------------
    int cmp(const ap_uint& o) const {
        for (int i = NW - 1; i >= 0; --i) {
            if (w[i] != o.w[i]) return w[i] < o.w[i] ? -1 : 1;
        }
        return 0;
    }
    bool operator==(const ap_uint& o) const { return cmp(o) == 0; }
    bool operator!=(const ap_uint& o) const { return cmp(o) != 0; }
    bool operator<(const ap_uint& o) const { return cmp(o) < 0; }
    bool operator>(const ap_uint& o) const { return cmp(o) > 0; }
    bool operator<=(const ap_uint& o) const { return cmp(o) <= 0; }
    bool operator>=(const ap_uint& o) const { return cmp(o) >= 0; }

    // ---- bit ranges ----------------------------------------------------------
    uint64_t get_range(int hi, int lo) const {
        int width = hi - lo + 1;
        ap_uint t = *this >> lo;
        uint64_t v = t.w[0];
        if (width < 64) v &= (1ull << width) - 1;
        return v;
    }
    void set_range(int hi, int lo, uint64_t v) {
        int width = hi - lo + 1;
        uint64_t mask64 = width >= 64 ? ~0ull : ((1ull << width) - 1);
        v &= mask64;
        ap_uint m = ap_uint(mask64) << lo;
        ap_uint nv = ap_uint(v) << lo;
        for (int i = 0; i < NW; ++i) w[i] = (w[i] & ~m.w[i]) | nv.w[i];
        clear_top();
    }

    struct range_ref {
        ap_uint* p; int hi, lo;
        operator uint64_t() const { return p->get_range(hi, lo); }
        range_ref& operator=(uint64_t v) { p->set_range(hi, lo, v); return *this; }
        range_ref& operator=(const range_ref& o) { p->set_range(hi, lo, (uint64_t)o); return *this; }
        template <int W2>
        range_ref& operator=(const ap_uint<W2>& v) { p->set_range(hi, lo, v.w[0]); return *this; }
    };

    range_ref operator()(int hi, int lo) { return range_ref{this, hi, lo}; }
    uint64_t operator()(int hi, int lo) const { return get_range(hi, lo); }
    range_ref range(int hi, int lo) { return range_ref{this, hi, lo}; }
    uint64_t range(int hi, int lo) const { return get_range(hi, lo); }
};

// Widening multiply: W1 x W2 -> W1 + W2 bits (schoolbook over 64-bit words).
template <int W1, int W2>
ap_uint<W1 + W2> operator*(const ap_uint<W1>& a, const ap_uint<W2>& b) {
    ap_uint<W1 + W2> r;
    constexpr int NR = ap_uint<W1 + W2>::NW;
    for (int i = 0; i < ap_uint<W1>::NW; ++i) {
        unsigned __int128 carry = 0;
        for (int j = 0; j < ap_uint<W2>::NW && i + j < NR; ++j) {
            unsigned __int128 cur = (unsigned __int128)a.w[i] * b.w[j] + r.w[i + j] + carry;
            r.w[i + j] = (uint64_t)cur;
            carry = cur >> 64;
        }
        for (int k = i + ap_uint<W2>::NW; k < NR && carry; ++k) {
            unsigned __int128 cur = (unsigned __int128)r.w[k] + carry;
            r.w[k] = (uint64_t)cur;
            carry = cur >> 64;
        }
    }
    r.clear_top();
    return r;
}

template <int W1, typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
ap_uint<W1 + 64> operator*(const ap_uint<W1>& a, T b) { return a * ap_uint<64>((uint64_t)b); }

template <int W1, typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
ap_uint<W1 + 64> operator*(T b, const ap_uint<W1>& a) { return ap_uint<64>((uint64_t)b) * a; }

template <int W>
using ap_int = ap_uint<W>;  // signed variant is never used on the path
