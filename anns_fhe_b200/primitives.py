"""Batched primitive workloads at N = 2^16: the NTT microbenchmark and the
batched hybrid key switch with rotation.

* `NttBatch`. Forward and inverse negacyclic NTT (hls/src/ntt.cpp:4-80) on
  64 ciphertexts (2 polynomials each) of 24 limbs of 50-bit NTT-friendly
  primes at N = 2^16. Residues are uniform in [0, q_i) from a seed, stored as
  uint64, limb-major. One `afhe_ntt_batch` call transforms all 128
  polynomials in place.
* `KeySwitchBatch`. Hybrid key switching (hls/src/key_switch.cpp:167-439)
  inside rotations (fhe_host_driver.cpp:331-404). N = 2^16, 24 Q limbs of
  50-bit primes, 8 special 60-bit primes, dnum 3 (alpha 8). Evaluation keys
  are seeded uniform residues. There are 32 ciphertexts at seeded levels in
  [8, 24]. Each one is rotated and summed by 2^0 .. 2^14 (x += rot(x, 2^s),
  15 dependent key switches), then rescaled. One batched call runs each step
  for every ciphertext of a level. Ciphertexts of different levels are
  separate calls on the same stream. At N = 2^16 one ciphertext's key switch
  already spreads over many CTAs (a CTA per limb-job and pass).

Every input residue is a pure function of (seed, ciphertext or polynomial,
limb), so tests can regenerate any part of the inputs without keeping them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .driver import CkksParams, FheContext


def seeded_limb(seed: int, unit: int, limb: int, q: int, n: int) -> np.ndarray:
    """Uniform residues in [0, q) for (unit, limb), independent of everything else."""
    return np.random.default_rng([seed, unit, limb]).integers(0, q, n, dtype=np.uint64)


class NttBatch:
    def __init__(self, cts: int = 64, limbs: int = 24, log_n: int = 16, q_bits: int = 50, seed: int = 5,
                 device: int = 0):
        # the digit size only sizes key-switch tables, which this workload never uses
        self.params = CkksParams.generate(log_n, limbs, q_bits, 1, 60, 8)
        self.n, self.limbs, self.seed = 1 << log_n, limbs, seed
        self.polys = 2 * cts
        self.w = limbs * self.n
        self.ctx = FheContext(self.params, poly_words=self.polys * self.w, key_words=1024, device=device, max_batch=1)
        for z in range(self.polys):
            self.ctx.write_poly(z * self.w, self.input_poly(z))
        self.offs = (L.u64 * self.polys)(*[z * self.w for z in range(self.polys)])
        self.ctx.sync()

    def input_limb(self, z: int, i: int) -> np.ndarray:
        return seeded_limb(self.seed, z, i, self.params.q[i], self.n)

    def input_poly(self, z: int) -> np.ndarray:
        return np.concatenate([self.input_limb(z, i) for i in range(self.limbs)])

    def transform(self, inverse: bool) -> None:
        L.check(self.ctx.lib.afhe_ntt_batch(self.ctx.h, C_u64p(self.offs), self.polys, self.limbs, int(inverse)),
                "ntt_batch")

    def read_limb(self, z: int, i: int) -> np.ndarray:
        return self.ctx.read_poly(z * self.w + i * self.n, self.n)

    def algorithmic_bytes(self) -> int:
        """One direction: every limb read and written once."""
        return 2 * self.polys * self.w * 8

    def butterflies(self) -> int:
        return self.polys * self.limbs * (self.n // 2) * (self.n.bit_length() - 1)

    def close(self) -> None:
        self.ctx.close()


def C_u64p(arr):
    import ctypes as C
    return C.cast(arr, L.P64)


def pow2_rotations(log_max: int = 14) -> list[int]:
    return [1 << s for s in range(log_max + 1)]


class KeySwitchBatch:
    def __init__(self, cts: int = 32, log_n: int = 16, num_q: int = 24, num_p: int = 8, alpha: int = 8,
                 level_range: tuple[int, int] = (8, 24), steps: list[int] | None = None, seed: int = 9,
                 device: int = 0, lanes: int = 32):
        self.params = p = CkksParams.generate(log_n, num_q, 50, num_p, 60, alpha)
        self.n, self.seed = p.n, seed
        self.steps = steps or pow2_rotations()
        rng = np.random.default_rng([seed, 0xC0FFEE])
        self.levels = [int(x) for x in rng.integers(level_range[0], level_range[1] + 1, cts)]
        self.cts = cts
        self.w = p.L * p.n                       # one polynomial slot (full level)
        kw = p.key_words()
        # ciphertexts at [0, 2 cts w); rescaled outputs after them
        self.ctx = FheContext(p, poly_words=4 * cts * self.w, key_words=len(self.steps) * kw, device=device,
                              max_batch=lanes)
        self.key_off = {}
        for k, s in enumerate(self.steps):
            off = k * kw
            self.ctx.write_key(off, self.key_words(k))
            L.check(self.ctx.lib.afhe_add_rotation_key(self.ctx.h, s, off), "add_rotation_key")
            self.key_off[s] = off
        self.reset()

    # ---- seeded inputs ----
    def key_words(self, k: int) -> np.ndarray:
        """Rotation key k: dnum digits of a then of b, each over Q then P limbs."""
        p = self.params
        primes = p.q + p.p
        return np.concatenate([seeded_limb(self.seed + 1, 1000 * k + d, i, primes[i], self.n)
                               for d in range(2 * p.dnum) for i in range(len(primes))])

    def key_pair(self, step: int) -> tuple[np.ndarray, np.ndarray]:
        k = self.ctx.read_key(self.key_off[step], self.params.key_words())
        h = k.size // 2
        return k[:h], k[h:]

    def input_ct(self, z: int) -> tuple[np.ndarray, np.ndarray]:
        lv, q = self.levels[z], self.params.q
        return tuple(np.concatenate([seeded_limb(self.seed, 2 * z + c, i, q[i], self.n) for i in range(lv)])
                     for c in range(2))

    def ct(self, z: int) -> tuple[int, int]:
        return (2 * z * self.w, (2 * z + 1) * self.w)

    def out_ct(self, z: int) -> tuple[int, int]:
        return ((2 * self.cts + 2 * z) * self.w, (2 * self.cts + 2 * z + 1) * self.w)

    def reset(self, which=None) -> None:
        for z in (range(self.cts) if which is None else which):
            c0, c1 = self.input_ct(z)
            self.ctx.write_poly(self.ct(z)[0], c0)
            self.ctx.write_poly(self.ct(z)[1], c1)
        self.ctx.sync()

    # ---- the chain ----
    def groups(self, which=None) -> dict[int, list[int]]:
        g: dict[int, list[int]] = {}
        for z in (range(self.cts) if which is None else which):
            g.setdefault(self.levels[z], []).append(z)
        return g

    @staticmethod
    def _refs(cts):
        arr = (L.CtRef * max(len(cts), 1))()
        for i, (a, b) in enumerate(cts):
            arr[i].c0_offset, arr[i].c1_offset = a, b
        return arr

    def rotate_step(self, step: int, which=None, by_level: bool = False) -> int:
        """x += rot(x, step) for the ciphertexts `which` (default all), every
        level in one call (afhe_eval_rotate_accumulate_levels_batch), or with
        by_level one call per level group; returns calls made."""
        zs_all = list(range(self.cts) if which is None else which)
        if not by_level:
            refs = self._refs([self.ct(z) for z in zs_all])
            lv = (C.c_uint32 * len(zs_all))(*[self.levels[z] for z in zs_all])
            L.check(self.ctx.lib.afhe_eval_rotate_accumulate_levels_batch(self.ctx.h, refs, refs, lv, len(zs_all),
                                                                          step),
                    "eval_rotate_accumulate_levels_batch")
            return 1
        calls = 0
        for lv, zs in sorted(self.groups(which).items()):
            refs = self._refs([self.ct(z) for z in zs])
            L.check(self.ctx.lib.afhe_eval_rotate_accumulate_batch(self.ctx.h, refs, refs, len(zs), step, lv),
                    "eval_rotate_accumulate_batch")
            calls += 1
        return calls

    def rescale(self, which=None) -> int:
        calls = 0
        for lv, zs in sorted(self.groups(which).items()):
            L.check(self.ctx.lib.afhe_rescale_batch(self.ctx.h, self._refs([self.ct(z) for z in zs]),
                                                    self._refs([self.out_ct(z) for z in zs]), len(zs), lv),
                    "rescale_batch")
            calls += 1
        return calls

    def run(self, which=None, by_level: bool = False) -> None:
        for s in self.steps:
            self.rotate_step(s, which, by_level)
        self.rescale(which)

    def read_ct(self, z: int, out: bool = False) -> tuple[np.ndarray, np.ndarray]:
        lv = self.levels[z] - (1 if out else 0)
        c = self.out_ct(z) if out else self.ct(z)
        return self.ctx.read_poly(c[0], lv * self.n), self.ctx.read_poly(c[1], lv * self.n)

    def key_switch_count(self) -> int:
        return len(self.steps) * self.cts

    def algorithmic_bytes_per_step(self) -> int:
        """One rotate-and-sum step over all ciphertexts: per ciphertext c0, c1
        read and written at its level, plus each level group's key read once
        over that level's limbs (2 x ceil(level / alpha) digits of level + K
        limbs)."""
        p = self.params
        b = sum(4 * lv * self.n * 8 for lv in self.levels)
        for lv in self.groups():
            b += 2 * -(-lv // p.alpha) * (lv + p.K) * self.n * 8
        return b

    def close(self) -> None:
        self.ctx.close()
