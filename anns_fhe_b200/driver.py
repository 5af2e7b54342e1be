"""Host-side mirror of the reference's FHEHostDriver over the C ABI.

``FheContext`` owns a device context (poly_gmem / key_gmem arenas in HBM plus
the per-prime and per-level tables) and replaces SimMemoryBus
(cpp_host_model/src/sim_memory_bus.h:10-34). ``FHEHostDriver`` keeps the
reference's method names and argument order
(cpp_host_model/src/fhe_host_driver.h:78-110); each method is one C-ABI call,
and errors come back as ``AfheError`` instead of ``std::runtime_error``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import check


def _p64(a: np.ndarray):
    return a.ctypes.data_as(L.P64)


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------------------------------------------------------------------
# host number theory (no GPU needed)
# ---------------------------------------------------------------------------
def find_ntt_primes(log_n: int, bits: int, count: int, exclude=()) -> list[int]:
    lib = L.load()
    ex = _u64(list(exclude) or [0])
    out = np.zeros(count, dtype=np.uint64)
    check(lib.afhe_find_ntt_primes(log_n, bits, count, _p64(ex), len(exclude), _p64(out)), "find_ntt_primes")
    return [int(x) for x in out]


def twiddles(log_n: int, q: int, psi: int | None = None):
    lib = L.load()
    if psi is None:
        psi = int(lib.afhe_min_primitive_root(log_n, q))
    n = 1 << log_n
    tw = np.zeros(n, dtype=np.uint64)
    itw = np.zeros(n, dtype=np.uint64)
    check(lib.afhe_gen_twiddles(log_n, q, psi, _p64(tw), _p64(itw)), "gen_twiddles")
    return tw, itw


def barrett_constant(q: int) -> tuple[int, int, int]:
    lib = L.load()
    lo, hi, k = C.c_uint64(), C.c_uint64(), C.c_uint32()
    lib.afhe_barrett_constant(q, C.byref(lo), C.byref(hi), C.byref(k))
    return lo.value, hi.value, k.value


def galois_elt(log_n: int, step: int) -> int:
    return int(L.load().afhe_galois_elt(log_n, step))


def automorphism_map(log_n: int, galois: int) -> np.ndarray:
    m = np.zeros(1 << log_n, dtype=np.uint32)
    check(L.load().afhe_automorphism_map(log_n, galois, m.ctypes.data_as(L.P32)), "automorphism_map")
    return m


def pack_map(m32: np.ndarray) -> np.ndarray:
    """Two u32 map entries per u64 word, low half first (fhe_host_driver.cpp:141-154)."""
    m = m32.astype(np.uint64)
    return m[0::2] | (m[1::2] << np.uint64(32))


def part_qhat_tables(q, level: int, alpha: int, part: int, p):
    lib = L.load()
    qa, pa = _u64(q), _u64(p)
    parts = (level + alpha - 1) // alpha
    size = level - alpha * part if part == parts - 1 else alpha
    inv = np.zeros(size, dtype=np.uint64)
    modp = np.zeros(size * (level - size + len(p)), dtype=np.uint64)
    check(lib.afhe_part_qhat_tables(_p64(qa), level, alpha, part, _p64(pa), len(p), _p64(inv), _p64(modp)),
          "part_qhat_tables")
    return inv, modp


def moddown_tables(q, level: int, p):
    lib = L.load()
    qa, pa = _u64(q), _u64(p)
    k = len(p)
    a = np.zeros(level, dtype=np.uint64)
    b = np.zeros(k, dtype=np.uint64)
    c = np.zeros(k * level, dtype=np.uint64)
    check(lib.afhe_moddown_tables(_p64(qa), level, _p64(pa), k, _p64(a), _p64(b), _p64(c)), "moddown_tables")
    return a, b, c


def rescale_tables(q, level: int):
    lib = L.load()
    qa = _u64(q)
    a = np.zeros(level - 1, dtype=np.uint64)
    b = np.zeros(level - 1, dtype=np.uint64)
    check(lib.afhe_rescale_tables(_p64(qa), level, _p64(a), _p64(b)), "rescale_tables")
    return a, b


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------
@dataclass
class CkksParams:
    """A parameter set: ring degree, Q / P chains and the digit size."""
    log_n: int
    q: list[int]
    p: list[int]
    alpha: int
    psi: tuple = ()     # primitive 2N-th roots behind the twiddles, Q then P (empty: the smallest)

    @property
    def n(self) -> int:
        return 1 << self.log_n

    @property
    def L(self) -> int:
        return len(self.q)

    @property
    def K(self) -> int:
        return len(self.p)

    @property
    def dnum(self) -> int:
        return (self.L + self.alpha - 1) // self.alpha

    @classmethod
    def generate(cls, log_n: int, num_q: int, q_bits: int, num_p: int, p_bits: int, alpha: int,
                 first_bits: int | None = None) -> "CkksParams":
        """Deterministic chain: the largest NTT-friendly primes below the sizes."""
        used: list[int] = []
        q: list[int] = []
        if first_bits and first_bits != q_bits:
            q += find_ntt_primes(log_n, first_bits, 1, used)
            used += q
            q += find_ntt_primes(log_n, q_bits, num_q - 1, used)
        else:
            q += find_ntt_primes(log_n, q_bits, num_q, used)
        used += q
        p = find_ntt_primes(log_n, p_bits, num_p, used)
        return cls(log_n, q, p, alpha)

    def key_words(self) -> int:
        """Words of one evaluation key at full level: 2 * dnum * (L + K) * N."""
        return 2 * self.dnum * (self.L + self.K) * self.n


class PinnedStaging:
    """Reusable page-locked host buffers by name (afhe_host_alloc), grown on
    demand; `get` returns a uint64 view whose contents the next `get` of the
    same name may reuse. A buffer replaced by a larger one is not freed until
    `close`: an asynchronous copy still in flight into it (a read enqueued
    without waiting) keeps a valid destination, and so does a view taken
    earlier."""

    def __init__(self):
        self.lib = L.load()
        self.bufs: dict[str, tuple[int, int, np.ndarray]] = {}     # name: (pointer, words, view)
        self.retired: list[int] = []

    def get(self, name: str, words: int) -> np.ndarray:
        ptr, cap, view = self.bufs.get(name, (0, 0, None))
        if cap < words:
            if ptr:
                self.retired.append(ptr)
            cap = max(words, 2 * cap)
            p = C.c_void_p()
            check(self.lib.afhe_host_alloc(cap * 8, C.byref(p)), "afhe_host_alloc")
            ptr = p.value
            view = np.frombuffer((C.c_uint64 * cap).from_address(ptr), dtype=np.uint64)
            self.bufs[name] = (ptr, cap, view)
        return view[:words]

    def close(self) -> None:
        for ptr in [b[0] for b in self.bufs.values()] + self.retired:
            if ptr:
                self.lib.afhe_host_free(C.c_void_p(ptr))
        self.bufs = {}
        self.retired = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FheContext:
    """Device context: arenas, tables, key directory (one CUDA stream)."""

    def __init__(self, params: CkksParams, poly_words: int, key_words: int, device: int = 0, max_batch: int = 0):
        self.lib = L.load()
        self.params = params
        pr = L.Params()
        pr.log_n, pr.num_q, pr.num_p, pr.alpha = params.log_n, params.L, params.K, params.alpha
        for i, x in enumerate(params.q):
            pr.q[i] = x
        for i, x in enumerate(params.p):
            pr.p[i] = x
        for i, x in enumerate(params.psi):
            if i < params.L:
                pr.psi_q[i] = x
            else:
                pr.psi_p[i - params.L] = x
        pr.poly_words, pr.key_words, pr.device = poly_words, key_words, device
        pr.max_batch = max_batch
        self.max_batch = max_batch or 64
        self.device = device
        h = L.CTX()
        check(self.lib.afhe_ctx_create(C.byref(pr), C.byref(h)), "afhe_ctx_create")
        self.h = h
        self.poly_words = poly_words
        self.key_words = key_words

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.afhe_ctx_destroy(self.h)
            self.h = None
        if getattr(self, "_staging", None) is not None:
            self._staging.close()
            self._staging = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- arenas ----
    def write_poly(self, off: int, data) -> None:
        a = _u64(data).ravel()
        check(self.lib.afhe_write_poly(self.h, off, _p64(a), a.size), "write_poly")

    def read_poly(self, off: int, count: int, out: np.ndarray | None = None) -> np.ndarray:
        """`count` words at `off`; into `out` (e.g. a pinned staging view) if given."""
        a = np.empty(count, dtype=np.uint64) if out is None else out[:count]
        check(self.lib.afhe_read_poly(self.h, off, _p64(a), count), "read_poly")
        return a

    @property
    def staging(self) -> "PinnedStaging":
        if getattr(self, "_staging", None) is None:
            self._staging = PinnedStaging()
        return self._staging

    def write_key(self, off: int, data) -> None:
        a = _u64(data).ravel()
        check(self.lib.afhe_write_key(self.h, off, _p64(a), a.size), "write_key")

    def read_key(self, off: int, count: int) -> np.ndarray:
        a = np.empty(count, dtype=np.uint64)
        check(self.lib.afhe_read_key(self.h, off, _p64(a), count), "read_key")
        return a

    def set_option(self, option: int, value: int) -> None:
        check(self.lib.afhe_ctx_set_option(self.h, option, int(value)), "afhe_ctx_set_option")

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        check(self.lib.afhe_ctx_get_option(self.h, option, C.byref(v)), "afhe_ctx_get_option")
        return int(v.value)

    def scratch_bytes(self) -> int:
        """Bytes of context-private device scratch (all lanes)."""
        return int(self.lib.afhe_scratch_words(self.h)) * 8

    def sync(self) -> None:
        check(self.lib.afhe_sync(self.h), "sync")

    def fence(self) -> int:
        """A fence after the work enqueued so far on the context's stream."""
        f = C.c_uint64()
        check(self.lib.afhe_fence(self.h, C.byref(f)), "fence")
        return int(f.value)

    def fence_wait(self, fence: int) -> None:
        """Block until the work before `fence` has finished."""
        check(self.lib.afhe_fence_wait(self.h, fence), "fence_wait")

    def write_context_tables(self, level: int) -> L.ContextLayout:
        lay = L.ContextLayout()
        check(self.lib.afhe_ctx_write_context_tables(self.h, level, C.byref(lay)), "write_context_tables")
        return lay

    def dispatch(self, args: L.AccelArgs) -> int:
        """fhe_accel_top: returns the status (does not raise)."""
        return self.lib.afhe_dispatch(self.h, C.byref(args))

    def accel_args(self, op: int, active_limbs: int, layout: L.ContextLayout | None = None, **kw) -> L.AccelArgs:
        """Registers for fhe_accel_top filled from this parameter set (as
        FHEHostDriver::dispatch does, fhe_host_driver.cpp:177-204)."""
        p = self.params
        a = L.AccelArgs()
        a.op_code = op
        a.active_limbs = active_limbs
        a.sizeQl = kw.pop("sizeQl", active_limbs)
        a.sizeP = kw.pop("sizeP", p.K)
        a.alpha = kw.pop("alpha", p.alpha)
        a.numPartQ = kw.pop("numPartQ", (a.sizeQl + a.alpha - 1) // a.alpha)
        n = p.n
        for i, q in enumerate(p.q):
            a.rns_primes[i] = q
            lo, hi, k = barrett_constant(q)
            a.barrett_m_q_lo[i], a.barrett_m_q_hi[i], a.barrett_k_q[i] = lo, hi, k
            a.n_inv_q[i] = pow(n, -1, q)
        for i, q in enumerate(p.p):
            a.p_primes[i] = q
            lo, hi, k = barrett_constant(q)
            a.barrett_m_p_lo[i], a.barrett_m_p_hi[i], a.barrett_k_p[i] = lo, hi, k
            a.n_inv_p[i] = pow(n, -1, q)
        if 0 < active_limbs <= p.L:
            a.n_inv_mod_q_last = a.n_inv_q[active_limbs - 1]
        if layout is not None:
            for f in ("twiddles_q_offset", "inv_twiddles_q_offset", "twiddles_p_offset", "inv_twiddles_p_offset",
                      "p_inv_mod_q_offset", "p_hat_inv_mod_p_offset", "p_hat_mod_q_offset", "qlql_offset",
                      "qlinv_offset"):
                setattr(a, f, getattr(layout, f))
            for j in range(L.MAX_PARTS):
                a.qhat_inv_offset[j] = layout.qhat_inv_offset[j]
                a.qhat_modp_offset[j] = layout.qhat_modp_offset[j]
        for k, v in kw.items():
            setattr(a, k, v)
        return a


class FHEHostDriver:
    """Composite operators with the reference's names and argument order."""

    def __init__(self, ctx: FheContext):
        self.ctx = ctx
        self.lib = ctx.lib
        self.h = ctx.h

    # key directory (m_cfg.relin_key_offset, m_rot_keys)
    def set_relin_key(self, evk_offset: int) -> None:
        check(self.lib.afhe_set_relin_key(self.h, evk_offset), "set_relin_key")

    def add_rotation_key(self, step: int, evk_offset: int) -> None:
        check(self.lib.afhe_add_rotation_key(self.h, step, evk_offset), "add_rotation_key")

    def has_rotation_key(self, step: int) -> bool:
        return bool(self.lib.afhe_has_rotation_key(self.h, step))

    # primitives (OP 1-8 with the context's own tables)
    def ntt(self, src, dst, limbs):
        check(self.lib.afhe_ntt(self.h, src, dst, limbs), "ntt")

    def intt(self, src, dst, limbs):
        check(self.lib.afhe_intt(self.h, src, dst, limbs), "intt")

    def poly_add(self, a, b, dst, limbs):
        check(self.lib.afhe_poly_add(self.h, a, b, dst, limbs), "poly_add")

    def poly_sub(self, a, b, dst, limbs):
        check(self.lib.afhe_poly_sub(self.h, a, b, dst, limbs), "poly_sub")

    def poly_mul_ntt(self, a, b, dst, limbs):
        check(self.lib.afhe_poly_mul_ntt(self.h, a, b, dst, limbs), "poly_mul_ntt")

    def automorphism(self, src, galois_elt, dst, limbs):
        check(self.lib.afhe_automorphism(self.h, src, galois_elt, dst, limbs), "automorphism")

    def rescale(self, c0_in, c1_in, c0_out, c1_out, limbs):
        check(self.lib.afhe_rescale(self.h, c0_in, c1_in, c0_out, c1_out, limbs), "rescale")

    def key_switch(self, src, evk_offset, dst_c0, dst_c1, limbs):
        check(self.lib.afhe_key_switch(self.h, src, evk_offset, dst_c0, dst_c1, limbs), "key_switch")

    # composite operators
    def eval_add(self, a0, a1, b0, b1, d0, d1, limbs):
        check(self.lib.afhe_eval_add(self.h, a0, a1, b0, b1, d0, d1, limbs), "eval_add")

    def eval_sub_plain(self, a0, a1, pt, d0, d1, limbs):
        check(self.lib.afhe_eval_sub_plain(self.h, a0, a1, pt, d0, d1, limbs), "eval_sub_plain")

    def eval_mult_relin_rescale(self, a0, a1, b0, b1, d0, d1, in_limbs):
        check(self.lib.afhe_eval_mult_relin_rescale(self.h, a0, a1, b0, b1, d0, d1, in_limbs),
              "eval_mult_relin_rescale")

    def eval_mult_plain_rescale(self, a0, a1, pt, d0, d1, in_limbs):
        check(self.lib.afhe_eval_mult_plain_rescale(self.h, a0, a1, pt, d0, d1, in_limbs), "eval_mult_plain_rescale")

    def eval_rotate_single_step(self, i0, i1, d0, d1, step, limbs):
        check(self.lib.afhe_eval_rotate_single_step(self.h, i0, i1, d0, d1, step, limbs), "eval_rotate_single_step")

    def eval_rotate(self, i0, i1, d0, d1, total_rot, limbs):
        check(self.lib.afhe_eval_rotate(self.h, i0, i1, d0, d1, total_rot, limbs), "eval_rotate")

    # batched
    @staticmethod
    def _refs(cts):
        arr = (L.CtRef * max(len(cts), 1))()
        for i, (c0, c1) in enumerate(cts):
            arr[i].c0_offset, arr[i].c1_offset = c0, c1
        return arr

    def eval_mult_relin_rescale_batch(self, a, b, d, in_limbs):
        check(self.lib.afhe_eval_mult_relin_rescale_batch(self.h, self._refs(a), self._refs(b), self._refs(d), len(a),
                                                          in_limbs), "eval_mult_relin_rescale_batch")

    def eval_rotate_batch(self, cts_in, cts_out, total_rot, limbs):
        check(self.lib.afhe_eval_rotate_batch(self.h, self._refs(cts_in), self._refs(cts_out), len(cts_in), total_rot,
                                              limbs), "eval_rotate_batch")
