"""FHEHostDriver composite operators restated on the CPU oracle.

TEST INFRASTRUCTURE ONLY. Follows cpp_host_model/src/fhe_host_driver.cpp:
  eval_add / eval_sub_plain           :248-270
  eval_mult_relin_rescale             :272-306
  eval_mult_plain_rescale             :308-329
  eval_rotate_single_step             :331-359
  eval_rotate (power-of-two steps)    :361-404
with the tables of the ciphertext's own level (the reference loads one
level's tables; at that level the two agree) and keys stored once at full
level: digit j, limb i of a key at level l is limb i (Q) or L + k (P) of the
full-level digit, i.e. orc_key_switch with key_digit_stride = L + K and
key_p_base = L. Ciphertext polys are limb-major uint64 arrays.
"""
from __future__ import annotations

import numpy as np

from .oracle import Orc, tables_py as T


class OracleCKKS:
    def __init__(self, log_n: int, q: list[int], p: list[int], alpha: int, orc: Orc | None = None):
        self.orc = orc or Orc()
        self.log_n, self.n = log_n, 1 << log_n
        self.q, self.p, self.alpha = list(q), list(p), alpha
        self.L, self.K = len(q), len(p)
        self.dnum = -(-self.L // alpha)
        tw = [T.twiddles(log_n, x) for x in self.q + self.p]
        self.tw = [t[0] for t in tw]
        self.itw = [t[1] for t in tw]
        self._lvl: dict[int, dict] = {}

    def tables(self, level: int) -> dict:
        if level not in self._lvl:
            parts = -(-level // self.alpha)
            qi, qm = zip(*[T.part_qhat(self.q, level, self.alpha, j, self.p) for j in range(parts)])
            pinv, phinv, phq = T.moddown(self.q, level, self.p)
            d = dict(parts=parts, qhat_inv=list(qi), qhat_modp=list(qm), pinv=pinv, phinv=phinv, phq=phq)
            if level > 1:
                d["qlql"], d["qlinv"] = T.rescale(self.q, level)
            self._lvl[level] = d
        return self._lvl[level]

    def limb(self, x: np.ndarray, i: int) -> np.ndarray:
        return x[i * self.n:(i + 1) * self.n]

    # ---- primitives ----
    def ntt(self, x, limbs):
        return np.concatenate([self.orc.ntt(self.limb(x, i), self.tw[i], self.q[i]) for i in range(limbs)])

    def intt(self, x, limbs):
        return np.concatenate([self.orc.intt(self.limb(x, i), self.itw[i], self.q[i]) for i in range(limbs)])

    def poly(self, op, a, b, limbs):
        return np.concatenate([self.orc.poly(op, self.limb(a, i), self.limb(b, i), self.q[i]) for i in range(limbs)])

    def automorphism(self, x, galois, limbs):
        m = T.auto_map(self.log_n, galois).astype(np.uint64)
        packed = m[0::2] | (m[1::2] << np.uint64(32))
        return np.concatenate([self.orc.automorphism(self.limb(x, i), packed) for i in range(limbs)])

    def rescale_poly(self, x, level):
        t = self.tables(level)
        tw = np.concatenate(self.tw[:level])
        return self.orc.rescale(x[:level * self.n], self.q[:level], self.itw[level - 1], tw, t["qlql"], t["qlinv"],
                                self.n)

    def key_switch(self, x, key_a, key_b, level):
        """key_a / key_b: full-level digits concatenated, dnum * (L + K) * N words."""
        t = self.tables(level)
        return self.orc.key_switch(x[:level * self.n], key_a, key_b, self.L + self.K, self.L, level, self.K,
                                   t["parts"], self.alpha, self.q[:level], self.p,
                                   np.concatenate(self.tw[:level]), np.concatenate(self.itw[:level]),
                                   np.concatenate(self.tw[self.L:]), np.concatenate(self.itw[self.L:]),
                                   t["qhat_inv"], t["qhat_modp"], t["pinv"], t["phinv"], t["phq"], self.n)

    # ---- composites ----
    def eval_add(self, a, b, limbs):
        return self.poly("add", a[0], b[0], limbs), self.poly("add", a[1], b[1], limbs)

    def eval_sub_plain(self, a, pt, limbs):
        return self.poly("sub", a[0], pt, limbs), a[1][:limbs * self.n].copy()

    def eval_mult_relin_rescale(self, a, b, relin, level):
        d0 = self.poly("mul", a[0], b[0], level)
        d2 = self.poly("mul", a[1], b[1], level)
        d1 = self.poly("add", self.poly("mul", a[0], b[1], level), self.poly("mul", a[1], b[0], level), level)
        k0, k1 = self.key_switch(d2, relin[0], relin[1], level)
        d0 = self.poly("add", d0, k0, level)
        d1 = self.poly("add", d1, k1, level)
        return self.rescale_poly(d0, level), self.rescale_poly(d1, level)

    def eval_mult_plain_rescale(self, a, pt, level):
        c0 = self.poly("mul", a[0], pt, level)
        c1 = self.poly("mul", a[1], pt, level)
        return self.rescale_poly(c0, level), self.rescale_poly(c1, level)

    def eval_rotate_single_step(self, c, step, rotkeys, limbs):
        k = T.galois(self.log_n, step)
        a0 = self.automorphism(c[0], k, limbs)
        a1 = self.automorphism(c[1], k, limbs)
        k0, k1 = self.key_switch(a1, rotkeys[step][0], rotkeys[step][1], limbs)
        return self.poly("add", a0, k0, limbs), k1

    def eval_rotate(self, c, total, rotkeys, limbs):
        if total == 0:
            return c[0][:limbs * self.n].copy(), c[1][:limbs * self.n].copy()
        rem, sign = abs(total), 1 if total > 0 else -1
        cur = c
        while rem > 0:
            s = 1
            while (s << 1) <= rem:
                s <<= 1
            cur = self.eval_rotate_single_step(cur, sign * s, rotkeys, limbs)
            rem -= s
        return cur
