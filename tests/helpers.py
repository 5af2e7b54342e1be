"""Test helpers: seeded inputs and reference-shaped arena images.

`AccelImage` lays out a key_gmem image the way
cpp_host_model/src/fhe_host_driver.cpp:46-117 does (twiddles Q then P from word
0, inverse twiddles after them, CRT tables in 64-word slots, an evaluation key
512-word aligned after the tables) using tables computed from their
definitions (oracle.tables_py), and fills the fhe_accel_top registers for it.
"""
from __future__ import annotations

import numpy as np

from anns_fhe_b200 import _lib as L
from oracle.oracle import tables_py as T


def primes_for(log_n: int, nq: int, q_bits: int, np_: int, p_bits: int, first_bits: int | None = None):
    from anns_fhe_b200.driver import find_ntt_primes
    used: list[int] = []
    q: list[int] = []
    if first_bits:
        q += find_ntt_primes(log_n, first_bits, 1, used)
        used += q
        q += find_ntt_primes(log_n, q_bits, nq - 1, used)
    else:
        q += find_ntt_primes(log_n, q_bits, nq, used)
    used += q
    p = find_ntt_primes(log_n, p_bits, np_, used)
    return q, p


def uniform_residues(rng: np.random.Generator, primes, n: int) -> np.ndarray:
    """One limb per prime, residues uniform in [0, q_i), limb-major."""
    return np.concatenate([rng.integers(0, int(q), size=n, dtype=np.uint64) for q in primes])


class AccelImage:
    def __init__(self, log_n: int, q: list[int], p: list[int], alpha: int, table_level: int,
                 numPartQ: int | None = None, key_level: int | None = None, seed: int = 7):
        self.log_n, self.n = log_n, 1 << log_n
        self.q, self.p, self.alpha = list(q), list(p), alpha
        n, Lq, K = self.n, len(q), len(p)
        self.L, self.K = Lq, K
        tw = [T.twiddles(log_n, x) for x in q + p]
        self.tw_q = np.concatenate([t[0] for t in tw[:Lq]])
        self.itw_q = np.concatenate([t[1] for t in tw[:Lq]])
        self.tw_p = np.concatenate([t[0] for t in tw[Lq:]])
        self.itw_p = np.concatenate([t[1] for t in tw[Lq:]])
        chunks: list[tuple[int, np.ndarray]] = []
        cur = 0
        self.off = {}
        self.off["twiddles_q"], cur = cur, cur
        chunks.append((cur, np.concatenate([self.tw_q, self.tw_p])))
        self.off["twiddles_p"] = cur + Lq * n
        cur += (Lq + K) * n
        self.off["inv_twiddles_q"] = cur
        chunks.append((cur, np.concatenate([self.itw_q, self.itw_p])))
        self.off["inv_twiddles_p"] = cur + Lq * n
        cur += (Lq + K) * n

        def slot(v):
            nonlocal cur
            at = cur
            chunks.append((at, np.asarray(v, dtype=np.uint64)))
            cur += max(64, -(-len(v) // 64) * 64)
            return at

        lvl = table_level
        self.table_level = lvl
        self.parts = numPartQ or -(-lvl // alpha)
        self.qhat_inv, self.qhat_modp = [], []
        self.off["qhat_inv"], self.off["qhat_modp"] = [], []
        for j in range(self.parts):
            a, b = T.part_qhat(q, lvl, alpha, j, p)
            self.qhat_inv.append(a)
            self.qhat_modp.append(b)
            self.off["qhat_inv"].append(slot(a))
            self.off["qhat_modp"].append(slot(b))
        self.pinv, self.phinv, self.phq = T.moddown(q, lvl, p)
        self.off["pinv"], self.off["phinv"], self.off["phq"] = slot(self.pinv), slot(self.phinv), slot(self.phq)
        self.qlql, self.qlinv = T.rescale(q, lvl) if lvl > 1 else (np.zeros(1, np.uint64), np.zeros(1, np.uint64))
        self.off["qlql"], self.off["qlinv"] = slot(self.qlql), slot(self.qlinv)
        cur = (cur + 511) & ~511
        # evaluation key laid out for OP_KEY_SWITCH at `key_level`:
        # [a_0..a_{d-1}][b_0..b_{d-1}], digit stride (key_level + K) * N
        kl = key_level or lvl
        self.key_level = kl
        rng = np.random.default_rng(seed)
        primes_k = q[:kl] + p
        self.evk_a = [uniform_residues(rng, primes_k, n) for _ in range(self.parts)]
        self.evk_b = [uniform_residues(rng, primes_k, n) for _ in range(self.parts)]
        self.off["evk"] = cur
        chunks.append((cur, np.concatenate(self.evk_a + self.evk_b)))
        cur += 2 * self.parts * (kl + K) * n
        self.key_words = cur + 512
        self.key = np.zeros(self.key_words, dtype=np.uint64)
        for at, v in chunks:
            self.key[at:at + v.size] = v

    def args(self, op: int, active_limbs: int, **kw) -> L.AccelArgs:
        a = L.AccelArgs()
        a.op_code = op
        a.active_limbs = active_limbs
        a.sizeQl = kw.pop("sizeQl", active_limbs)
        a.sizeP = kw.pop("sizeP", self.K)
        a.alpha = kw.pop("alpha", self.alpha)
        a.numPartQ = kw.pop("numPartQ", self.parts)
        n = self.n
        for i, q in enumerate(self.q):
            a.rns_primes[i] = q
            a.barrett_m_q_lo[i], a.barrett_m_q_hi[i], a.barrett_k_q[i] = T.barrett(q)
            a.n_inv_q[i] = pow(n, -1, q)
        for i, q in enumerate(self.p):
            a.p_primes[i] = q
            a.barrett_m_p_lo[i], a.barrett_m_p_hi[i], a.barrett_k_p[i] = T.barrett(q)
            a.n_inv_p[i] = pow(n, -1, q)
        a.n_inv_mod_q_last = a.n_inv_q[active_limbs - 1] if active_limbs >= 1 else 0
        a.twiddles_q_offset = self.off["twiddles_q"]
        a.inv_twiddles_q_offset = self.off["inv_twiddles_q"]
        a.twiddles_p_offset = self.off["twiddles_p"]
        a.inv_twiddles_p_offset = self.off["inv_twiddles_p"]
        for j in range(self.parts):
            a.qhat_inv_offset[j] = self.off["qhat_inv"][j]
            a.qhat_modp_offset[j] = self.off["qhat_modp"][j]
        a.p_inv_mod_q_offset = self.off["pinv"]
        a.p_hat_inv_mod_p_offset = self.off["phinv"]
        a.p_hat_mod_q_offset = self.off["phq"]
        a.qlql_offset = self.off["qlql"]
        a.qlinv_offset = self.off["qlinv"]
        a.evk_offset = self.off["evk"]
        for k, v in kw.items():
            setattr(a, k, v)
        return a
