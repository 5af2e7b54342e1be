"""Python access to the oracle: the C restatement (liborc.so) and, where it was
built, the reference's own HLS C-simulation (_ref/libref_hls.so at the
reference's N = 16384, and _ref/libref_hls_n<N>.so for the other ring degrees
the recipe builds from the same sources).

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker; the product never imports it.
Tables here are computed independently of the product with Python integers,
from their definitions (see tables_py below), so a product table bug cannot
hide inside the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_hls.so")
REF_N = 16384


def ref_lib_path(n: int = REF_N) -> str:
    """The reference build for ring degree n: verbatim at 16384, else the
    recipe's copy with the ring-degree literals rewritten."""
    return REF_LIB if n == REF_N else os.path.join(HERE, "_ref", f"libref_hls_n{n}.so")

P64 = C.POINTER(C.c_uint64)
P32 = C.POINTER(C.c_uint32)
u32, u64 = C.c_uint32, C.c_uint64
ORC_MAX_Q, ORC_MAX_P, ORC_MAX_PARTS = 64, 16, 16


def build_oracle(ref: bool = True) -> None:
    """make -C oracle (the reference part only where the reference tree exists)."""
    target = "all" if ref else "orc"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True, capture_output=True)


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(P64)


def _u(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------------------------------------------------------------------
# tables from their definitions (Python integers)
# ---------------------------------------------------------------------------
class tables_py:
    @staticmethod
    def bitrev(x: int, bits: int) -> int:
        return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0

    @staticmethod
    def min_root(log_n: int, q: int) -> int:
        m = 2 << log_n
        for g in range(2, q):
            x = pow(g, (q - 1) // m, q)
            if pow(x, m // 2, q) == q - 1:
                break
        best, cur, x2 = x, x, x * x % q
        for _ in range(m // 2 - 1):
            cur = cur * x2 % q
            best = min(best, cur)
        return best

    @staticmethod
    def twiddles(log_n: int, q: int, psi: int | None = None):
        n = 1 << log_n
        if psi is None:
            psi = tables_py.min_root(log_n, q)
        ipsi = pow(psi, -1, q)
        pw = [1] * n
        ipw = [1] * n
        for i in range(1, n):
            pw[i] = pw[i - 1] * psi % q
            ipw[i] = ipw[i - 1] * ipsi % q
        br = [tables_py.bitrev(j, log_n) for j in range(n)]
        return (np.array([pw[b] for b in br], dtype=np.uint64), np.array([ipw[b] for b in br], dtype=np.uint64))

    @staticmethod
    def is_prime(x: int) -> bool:
        """Deterministic Miller-Rabin for x < 2^64."""
        if x < 2:
            return False
        small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
        for b in small:
            if x % b == 0:
                return x == b
        d, r = x - 1, 0
        while d % 2 == 0:
            d //= 2
            r += 1
        for b in small:
            y = pow(b, d, x)
            if y in (1, x - 1):
                continue
            for _ in range(r - 1):
                y = y * y % x
                if y == x - 1:
                    break
            else:
                return False
        return True

    @staticmethod
    def ntt_primes(log_n: int, bits: int, count: int, exclude=()) -> list[int]:
        """The `count` largest primes below 2^bits that are 1 mod 2N, skipping
        `exclude`: the deterministic search the product's tables use
        (largest candidate first, step 2N)."""
        m = 2 << log_n
        c = ((1 << bits) - 1) // m * m + 1
        if c >= 1 << bits:
            c -= m
        out = []
        while len(out) < count:
            if c <= m:
                raise ValueError("ran out of NTT-friendly primes")
            if c not in exclude and tables_py.is_prime(c):
                out.append(c)
            c -= m
        return out

    @staticmethod
    def barrett(q: int):
        k = 2 * q.bit_length() + 3
        m = (1 << k) // q
        return m & (2**64 - 1), m >> 64, k

    @staticmethod
    def part_qhat(q, level, alpha, part, p):
        parts = (level + alpha - 1) // alpha
        start = alpha * part
        size = level - start if part == parts - 1 else alpha
        dig = q[start:start + size]
        Qj = 1
        for x in dig:
            Qj *= x
        outp = [q[i] for i in range(level) if not (start <= i < start + size)] + list(p)
        inv = [pow(Qj // qi % qi, -1, qi) for qi in dig]
        modp = [(Qj // qi) % pj for qi in dig for pj in outp]
        return np.array(inv, dtype=np.uint64), np.array(modp, dtype=np.uint64)

    @staticmethod
    def moddown(q, level, p):
        P = 1
        for x in p:
            P *= x
        pinv = [pow(P % q[i], -1, q[i]) for i in range(level)]
        phinv = [pow(P // pk % pk, -1, pk) for pk in p]
        phq = [(P // pk) % q[i] for pk in p for i in range(level)]
        return (np.array(pinv, dtype=np.uint64), np.array(phinv, dtype=np.uint64), np.array(phq, dtype=np.uint64))

    @staticmethod
    def rescale(q, level):
        """OpenFHE's definition: Q' = prod q_i (i < l), t = floor(Q' (Q'^-1 mod q_l) / q_l)."""
        ql = q[level - 1]
        Qp = 1
        for x in q[:level - 1]:
            Qp *= x
        t = Qp * pow(Qp % ql, -1, ql) // ql
        qlql = [t % q[i] for i in range(level - 1)]
        qlinv = [pow(ql % q[i], -1, q[i]) for i in range(level - 1)]
        return np.array(qlql, dtype=np.uint64), np.array(qlinv, dtype=np.uint64)

    @staticmethod
    def galois(log_n: int, step: int) -> int:
        m = 2 << log_n
        return pow(5, step % (m // 4), m)

    @staticmethod
    def auto_map(log_n: int, k: int) -> np.ndarray:
        """Evaluation-form permutation: slot i holds a(psi^(2 bitrev(i) + 1))."""
        n = 1 << log_n
        m = 2 * n
        idx = np.arange(n, dtype=np.int64)
        br = np.zeros(n, dtype=np.int64)
        for b in range(log_n):
            br |= ((idx >> b) & 1) << (log_n - 1 - b)
        e = (int(k) * (2 * br + 1)) % m
        return br[(e - 1) // 2].astype(np.uint32)


# ---------------------------------------------------------------------------
# C restatement
# ---------------------------------------------------------------------------
class OrcTopArgs(C.Structure):
    _fields_ = [
        ("op_code", u32), ("src_a_offset", u64), ("src_b_offset", u64), ("dst_offset", u64), ("evk_offset", u64),
        ("active_limbs", u32), ("prime_idx", u32), ("galois_elt", u32),
        ("sizeQl", u32), ("sizeP", u32), ("numPartQ", u32), ("alpha", u32),
        ("rns_primes", u64 * ORC_MAX_Q), ("p_primes", u64 * ORC_MAX_P),
        ("n_inv_q", u64 * ORC_MAX_Q), ("n_inv_p", u64 * ORC_MAX_P), ("n_inv_mod_q_last", u64),
        ("twiddles_q_offset", u64), ("inv_twiddles_q_offset", u64), ("twiddles_p_offset", u64),
        ("inv_twiddles_p_offset", u64),
        ("qhat_inv_offset", u64 * ORC_MAX_PARTS), ("qhat_modp_offset", u64 * ORC_MAX_PARTS),
        ("p_inv_mod_q_offset", u64), ("p_hat_inv_mod_p_offset", u64), ("p_hat_mod_q_offset", u64),
        ("qlql_offset", u64), ("qlinv_offset", u64),
    ]


def top_args_from(a) -> OrcTopArgs:
    """Copy an afhe_accel_args-shaped ctypes structure into the oracle's."""
    o = OrcTopArgs()
    for name, _ in OrcTopArgs._fields_:
        v = getattr(a, name)
        if hasattr(v, "__len__"):
            dst = getattr(o, name)
            for i in range(len(dst)):
                dst[i] = v[i]
        else:
            setattr(o, name, v)
    return o


class Orc:
    """liborc.so: the C restatement, any power-of-two N."""

    def __init__(self):
        if not os.path.exists(ORC_LIB):
            build_oracle(ref=False)
        lib = C.CDLL(ORC_LIB)
        sig = {
            "orc_mod_mul": (u64, [u64, u64, u64]),
            "orc_ntt_forward": (None, [P64, P64, u32, u64]),
            "orc_intt_inverse": (None, [P64, P64, u64, u32, u64]),
            "orc_poly_add": (None, [P64, P64, P64, u32, u64]),
            "orc_poly_sub": (None, [P64, P64, P64, u32, u64]),
            "orc_poly_mul": (None, [P64, P64, P64, u32, u64]),
            "orc_automorphism": (None, [P64, P64, P64, u32]),
            "orc_rescale": (None, [P64, P64, u32, P64, P64, P64, u64, P64, P64, u32]),
            "orc_fast_bases_conv": (None, [P64, P64, u32, u32, P64, P64, P64, P64, u32]),
            "orc_approx_mod_down": (None, [P64, P64, u32, u32, P64, P64, P64, P64, P64, P64, P64, P64, u32]),
            "orc_key_switch": (None, [P64, P64, P64, u32, u32, P64, P64, u32, u32, u32, u32, P64, P64, P64, P64,
                                      P64, P64, P64, P64, C.POINTER(P64), C.POINTER(P64), P64, P64, P64, u32]),
            "orc_ctx_create": (C.c_void_p, [u32]),
            "orc_ctx_destroy": (None, [C.c_void_p]),
            "orc_accel_top": (C.c_int, [C.c_void_p, P64, P64, C.POINTER(OrcTopArgs)]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype, f.argtypes = r, a
        self.lib = lib

    def ntt(self, a, tw, q):
        x = _u(a).copy()
        self.lib.orc_ntt_forward(_p(x), _p(_u(tw)), x.size, q)
        return x

    def intt(self, a, itw, q, n_inv=None):
        x = _u(a).copy()
        if n_inv is None:
            n_inv = pow(x.size, -1, q)
        self.lib.orc_intt_inverse(_p(x), _p(_u(itw)), n_inv, x.size, q)
        return x

    def poly(self, op, a, b, q):
        a, b = _u(a), _u(b)
        o = np.empty_like(a)
        getattr(self.lib, f"orc_poly_{op}")(_p(a), _p(b), _p(o), a.size, q)
        return o

    def automorphism(self, a, map64):
        a = _u(a)
        o = np.empty_like(a)
        self.lib.orc_automorphism(_p(a), _p(o), _p(_u(map64)), a.size)
        return o

    def rescale(self, a, q, itw_last, tw, qlql, qlinv, n):
        a = _u(a)
        L = a.size // n
        o = np.zeros((L - 1) * n, dtype=np.uint64)
        q = _u(q)
        self.lib.orc_rescale(_p(a), _p(o), L, _p(q), _p(_u(itw_last)), _p(_u(tw)), pow(n, -1, int(q[L - 1])),
                             _p(_u(qlql)), _p(_u(qlinv)), n)
        return o

    def key_switch(self, c_in, evk_a, evk_b, key_stride, key_pbase, sizeQl, sizeP, parts, alpha, q, p, tw_q, itw_q,
                   tw_p, itw_p, qhat_inv, qhat_modp, pinv, phinv, phq, n):
        c_in = _u(c_in)
        o0 = np.zeros(sizeQl * n, dtype=np.uint64)
        o1 = np.zeros(sizeQl * n, dtype=np.uint64)
        q, p = _u(q), _u(p)
        ninv_q = _u([pow(n, -1, int(x)) for x in q])
        ninv_p = _u([pow(n, -1, int(x)) for x in p])
        qi = [_u(x) for x in qhat_inv]
        qm = [_u(x) for x in qhat_modp]
        QI = (P64 * ORC_MAX_PARTS)(*[_p(x) for x in qi])
        QM = (P64 * ORC_MAX_PARTS)(*[_p(x) for x in qm])
        keep = (qi, qm, evk_a, evk_b)  # noqa: F841 - keep buffers alive during the call
        self.lib.orc_key_switch(_p(c_in), _p(_u(evk_a)), _p(_u(evk_b)), key_stride, key_pbase, _p(o0), _p(o1),
                                sizeQl, sizeP, parts, alpha, _p(q), _p(p), _p(_u(tw_q)), _p(_u(itw_q)),
                                _p(_u(tw_p)), _p(_u(itw_p)), _p(ninv_q), _p(ninv_p), QI, QM, _p(_u(pinv)),
                                _p(_u(phinv)), _p(_u(phq)), n)
        return o0, o1

    def accel_top(self, ctx_handle, poly: np.ndarray, key: np.ndarray, args) -> int:
        a = top_args_from(args)
        return self.lib.orc_accel_top(ctx_handle, _p(poly), _p(key), C.byref(a))

    def new_ctx(self, n: int):
        return self.lib.orc_ctx_create(n)

    def free_ctx(self, h) -> None:
        self.lib.orc_ctx_destroy(h)


class RefTopArgs(C.Structure):
    _fields_ = [
        ("op_code", u32), ("src_a_offset", u32), ("src_b_offset", u32), ("dst_offset", u32), ("evk_offset", u64),
        ("active_limbs", u32), ("prime_idx", u32), ("galois_elt", u32),
        ("sizeQl", u32), ("sizeP", u32), ("numPartQ", u32), ("alpha", u32),
        ("rns_primes", u64 * 15), ("p_primes", u64 * 4),
        ("barrett_m_q_lo", u64 * 15), ("barrett_m_q_hi", u64 * 15), ("barrett_k_q", u32 * 15),
        ("barrett_m_p_lo", u64 * 4), ("barrett_m_p_hi", u64 * 4), ("barrett_k_p", u32 * 4),
        ("n_inv_q", u64 * 15), ("n_inv_p", u64 * 4), ("n_inv_mod_q_last", u64),
        ("table_offsets", u32 * 15),
    ]


class Ref:
    """The reference's HLS functions at ring degree n (16384: the verbatim
    build; 8192 / 32768: the recipe's builds of the same sources)."""

    def __init__(self, n: int = REF_N):
        path = ref_lib_path(n)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        self.n = n
        sig = {
            "ref_mod_mul": (u64, [u64, u64, u64, u64, u64, u32]),
            "ref_ntt_forward": (None, [P64, P64, u64, u64, u64, u32]),
            "ref_intt_inverse": (None, [P64, P64, u64, u64, u64, u64, u32]),
            "ref_poly_add": (None, [P64, P64, P64, u64]),
            "ref_poly_sub": (None, [P64, P64, P64, u64]),
            "ref_poly_mul": (None, [P64, P64, P64, u64, u64, u64, u32]),
            "ref_automorphism": (None, [P64, P64, P64]),
            "ref_rescale": (None, [P64, P64, u32, P64, P64, P64, P32, P64, P64, u64, P64, P64]),
            "ref_key_switch": (None, [P64, P64, u64, u64, u64, P64, P64, u32, u32, u32, u32, P64, P64, P64, P64,
                                      P32, P64, P64, P32, P64, P64, P64, P64, P64, P64, P64, P64, P64, P64, P64,
                                      P64, P64, P64, P64]),
            "ref_fhe_accel_top": (None, [P64, u64, P64, u64, C.POINTER(RefTopArgs)]),
            "ref_ring_degree": (u32, []),
            "ref_bus_new": (C.c_void_p, [u64, u64]),
            "ref_bus_free": (None, [C.c_void_p]),
            "ref_bus_write_poly": (None, [C.c_void_p, u64, P64, u64]),
            "ref_bus_read_poly": (None, [C.c_void_p, u64, P64, u64]),
            "ref_bus_write_key": (None, [C.c_void_p, u64, P64, u64]),
            "ref_bus_accel_top": (None, [C.c_void_p, C.POINTER(RefTopArgs)]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype, f.argtypes = r, a
        self.lib = lib
        assert lib.ref_ring_degree() == n, "reference build has another ring degree"

    @staticmethod
    def available(n: int = REF_N) -> bool:
        return os.path.exists(ref_lib_path(n))

    def mod_mul(self, a, b, q):
        lo, hi, k = tables_py.barrett(q)
        return self.lib.ref_mod_mul(a, b, q, lo, hi, k)

    def ntt(self, a, tw, q):
        x = _u(a).copy()
        lo, hi, k = tables_py.barrett(q)
        self.lib.ref_ntt_forward(_p(x), _p(_u(tw)), q, lo, hi, k)
        return x

    def intt(self, a, itw, q):
        x = _u(a).copy()
        lo, hi, k = tables_py.barrett(q)
        self.lib.ref_intt_inverse(_p(x), _p(_u(itw)), pow(self.n, -1, q), q, lo, hi, k)
        return x

    def poly(self, op, a, b, q):
        a, b = _u(a), _u(b)
        o = np.empty_like(a)
        if op == "mul":
            lo, hi, k = tables_py.barrett(q)
            self.lib.ref_poly_mul(_p(a), _p(b), _p(o), q, lo, hi, k)
        else:
            getattr(self.lib, f"ref_poly_{op}")(_p(a), _p(b), _p(o), q)
        return o

    def automorphism(self, a, map64):
        a = _u(a)
        o = np.empty_like(a)
        self.lib.ref_automorphism(_p(a), _p(o), _p(_u(map64)))
        return o

    @staticmethod
    def _barrett_arrays(primes):
        b = [tables_py.barrett(int(x)) for x in primes]
        return (_u([x[0] for x in b]), _u([x[1] for x in b]), np.array([x[2] for x in b], dtype=np.uint32))

    def rescale(self, a, q, itw_last, tw, qlql, qlinv):
        a = _u(a)
        n = self.n
        L = a.size // n
        o = np.zeros((L - 1) * n, dtype=np.uint64)
        q = _u(q[:L])
        mlo, mhi, k = self._barrett_arrays(q)
        self.lib.ref_rescale(_p(a), _p(o), L, _p(q), _p(mlo), _p(mhi), k.ctypes.data_as(P32), _p(_u(itw_last)),
                             _p(_u(tw)), pow(n, -1, int(q[L - 1])), _p(_u(qlql)), _p(_u(qlinv)))
        return o

    def key_switch(self, c_in, key_words, evk_a_off, evk_b_off, sizeQl, sizeP, parts, alpha, q, p, tw_q, itw_q,
                   tw_p, itw_p, qhat_inv, qhat_modp, pinv, phinv, phq):
        n = self.n
        assert parts == 3, "the reference kernel takes exactly three digit tables"
        o0 = np.zeros(sizeQl * n, dtype=np.uint64)
        o1 = np.zeros(sizeQl * n, dtype=np.uint64)
        q, p = _u(q[:sizeQl]), _u(p[:sizeP])
        mql, mqh, kq = self._barrett_arrays(q)
        mpl, mph, kp = self._barrett_arrays(p)
        ninv_q = _u([pow(n, -1, int(x)) for x in q])
        ninv_p = _u([pow(n, -1, int(x)) for x in p])
        kw = _u(key_words)
        qi = [_u(x) for x in qhat_inv]
        qm = [_u(x) for x in qhat_modp]
        self.lib.ref_key_switch(_p(_u(c_in)), _p(kw), kw.size, evk_a_off, evk_b_off, _p(o0), _p(o1), sizeQl, sizeP,
                                parts, alpha, _p(q), _p(p), _p(mql), _p(mqh), kq.ctypes.data_as(P32), _p(mpl),
                                _p(mph), kp.ctypes.data_as(P32), _p(_u(tw_q)), _p(_u(itw_q)), _p(_u(tw_p)),
                                _p(_u(itw_p)), _p(ninv_q), _p(ninv_p), _p(qi[0]), _p(qm[0]), _p(qi[1]), _p(qm[1]),
                                _p(qi[2]), _p(qm[2]), _p(_u(pinv)), _p(_u(phinv)), _p(_u(phq)))
        return o0, o1

    def accel_top(self, poly: np.ndarray, key: np.ndarray, args) -> None:
        """One fhe_accel_top call; `args` is afhe_accel_args-shaped (offsets < 2^32)."""
        self.lib.ref_fhe_accel_top(_p(poly), poly.size, _p(key), key.size, C.byref(self.top_args(args)))

    @staticmethod
    def top_args(args) -> RefTopArgs:
        r = RefTopArgs()
        for f in ("op_code", "src_a_offset", "src_b_offset", "dst_offset", "evk_offset", "active_limbs",
                  "prime_idx", "galois_elt", "sizeQl", "sizeP", "numPartQ", "alpha", "n_inv_mod_q_last"):
            setattr(r, f, getattr(args, f))
        for i in range(15):
            r.rns_primes[i] = args.rns_primes[i]
            r.barrett_m_q_lo[i], r.barrett_m_q_hi[i] = args.barrett_m_q_lo[i], args.barrett_m_q_hi[i]
            r.barrett_k_q[i] = args.barrett_k_q[i]
            r.n_inv_q[i] = args.n_inv_q[i]
        for i in range(4):
            r.p_primes[i] = args.p_primes[i]
            r.barrett_m_p_lo[i], r.barrett_m_p_hi[i] = args.barrett_m_p_lo[i], args.barrett_m_p_hi[i]
            r.barrett_k_p[i] = args.barrett_k_p[i]
            r.n_inv_p[i] = args.n_inv_p[i]
        offs = [args.twiddles_q_offset, args.inv_twiddles_q_offset, args.twiddles_p_offset,
                args.inv_twiddles_p_offset, args.qhat_inv_offset[0], args.qhat_modp_offset[0],
                args.qhat_inv_offset[1], args.qhat_modp_offset[1], args.qhat_inv_offset[2],
                args.qhat_modp_offset[2], args.p_inv_mod_q_offset, args.p_hat_inv_mod_p_offset,
                args.p_hat_mod_q_offset, args.qlql_offset, args.qlinv_offset]
        for i, v in enumerate(offs):
            r.table_offsets[i] = v
        return r


class RefBus:
    """The reference's SimMemoryBus (cpp_host_model/src/sim_memory_bus.h:10-34)
    held across fhe_accel_top calls, as FHEHostDriver::dispatch drives it
    (fhe_host_driver.cpp:177-204): arenas stay resident between operators."""

    def __init__(self, ref: Ref, poly_words: int, key_words: int):
        self.ref, self.lib = ref, ref.lib
        self.h = self.lib.ref_bus_new(poly_words, key_words)

    def write_poly(self, off: int, x) -> None:
        x = _u(x)
        self.lib.ref_bus_write_poly(self.h, off, _p(x), x.size)

    def read_poly(self, off: int, count: int) -> np.ndarray:
        o = np.empty(count, dtype=np.uint64)
        self.lib.ref_bus_read_poly(self.h, off, _p(o), count)
        return o

    def write_key(self, off: int, x) -> None:
        x = _u(x)
        self.lib.ref_bus_write_key(self.h, off, _p(x), x.size)

    def top(self, r: RefTopArgs) -> None:
        self.lib.ref_bus_accel_top(self.h, C.byref(r))

    def close(self) -> None:
        if self.h:
            self.lib.ref_bus_free(self.h)
            self.h = None
