"""Host CKKS layer: encoding, key generation, encryption and decryption.

Replaces the OpenFHE calls of the reference (integration_tools/
generate_interactive_test_vectors.cpp:161-224 KeyGen / EvalMultKeyGen /
EvalRotateKeyGen, :383-398 and :443-447 MakeCKKSPackedPlaintext / Encrypt,
software_golden_model/fhe_core/fhe_context_manager.cpp:81-128 and 460-512).
Conventions (documented choices; OpenFHE-level parity is not claimed):

* Encoding: slot j of m(X) is m(zeta^(5^j)), zeta = exp(i*pi/N), for
  j < N/2; the conjugate slots hold the conjugates, so coefficients are real.
  Rotation by r is the automorphism X -> X^(5^r mod 2N) (slot j <- j + r).
* Secret: uniform ternary. Errors: rounded Gaussian, sigma = 3.19.
* Switching key from s' to s (hybrid, dnum digits of alpha limbs), stored at
  full level as [a_0 .. a_{d-1}][b_0 .. b_{d-1}], each over the L + K primes:
      b_j = -a_j * s + e_j + [i in digit j] * (P mod q_i) * s'.
  A rotation key for step r uses s' = sigma_{5^r}(s), matching the reference's
  order "automorphism first, then key switch" (fhe_host_driver.cpp:331-359).
* Public-key encryption: (v * b + e0 + m, v * a + e1), v ternary.

All ring arithmetic runs on the device through the C ABI (NTT, products,
automorphisms); the host samples randomness, encodes and decodes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.fft as _sfft

from .driver import CkksParams, FheContext, FHEHostDriver

SIGMA = 3.19


class Encoder:
    """Canonical-embedding encoder for N/2 complex slots."""

    def __init__(self, log_n: int):
        n = 1 << log_n
        self.n, self.slots = n, n // 2
        m = 2 * n
        k = np.array([pow(5, j, m) for j in range(self.slots)], dtype=np.int64)
        self.t = (k - 1) // 2            # index of zeta^(5^j) among odd powers
        self.tc = (m - k - 1) // 2       # its conjugate
        self.zeta = np.exp(1j * np.pi * np.arange(n) / n)

    def encode(self, values, scale: float) -> np.ndarray:
        """Integer coefficients (int64) of round(scale * embedding^-1(values))."""
        z = np.zeros(self.slots, dtype=np.complex128)
        v = np.asarray(values, dtype=np.complex128)
        z[:v.size] = v
        M = np.zeros(self.n, dtype=np.complex128)
        M[self.t] = scale * z
        M[self.tc] = np.conj(scale * z)
        y = np.fft.fft(M) / self.n
        coef = np.rint((y * np.conj(self.zeta)).real)
        if np.max(np.abs(coef)) >= 2.0**62:
            raise OverflowError("encoded coefficients exceed 62 bits; lower the scale")
        return coef.astype(np.int64)

    def encode_batch(self, values: np.ndarray, scale: float) -> np.ndarray:
        """encode() for each row of a (count, <= N/2) real array; (count, N) int64."""
        v = np.asarray(values, dtype=np.complex128)
        M = np.zeros((v.shape[0], self.n), dtype=np.complex128)
        M[:, self.t[:v.shape[1]]] = scale * v
        M[:, self.tc[:v.shape[1]]] = np.conj(scale * v)
        y = _sfft.fft(M, axis=1, workers=-1) / self.n
        coef = np.rint((y * np.conj(self.zeta)[None, :]).real)
        if np.max(np.abs(coef)) >= 2.0**62:
            raise OverflowError("encoded coefficients exceed 62 bits; lower the scale")
        return coef.astype(np.int64)

    def decode(self, coeffs, scale: float) -> np.ndarray:
        y = np.asarray(coeffs, dtype=np.float64) * self.zeta
        M = self.n * np.fft.ifft(y)
        return M[self.t] / scale

    def decode_real_batch(self, coeffs: np.ndarray, scale, slots: int | None = None) -> np.ndarray:
        """Real parts of decode_batch: slot j of row r is Re m_r(zeta^(5^j)) /
        scale (scale: a number or one per row). One zero-padded real FFT of
        length 2N evaluates m at every 2N-th root of unity. Root zeta^e and
        its conjugate zeta^(2N-e) have equal real parts, so slot j reads bin
        min(e_j, 2N - e_j). There is no complex twist, and only the needed
        columns are gathered."""
        if not hasattr(self, "_rbin"):
            e = np.array([pow(5, j, 2 * self.n) for j in range(self.slots)], dtype=np.int64)
            self._rbin = np.minimum(e, 2 * self.n - e)
        c = np.asarray(coeffs, dtype=np.float64)
        if slots is not None and slots <= 64:
            # few slots: Re m(zeta^e) = sum_k c_k cos(pi k e / N), one matrix product
            out = c @ self._cos_matrix(slots)
        else:
            R = _sfft.rfft(c, n=2 * self.n, axis=1, workers=-1)
            idx = self._rbin if slots is None else self._rbin[:slots]
            out = np.take(R.real, idx, axis=1)
        sc = np.asarray(scale, dtype=np.float64)
        return out / (sc[:, None] if sc.ndim else sc)

    def _cos_matrix(self, slots: int) -> np.ndarray:
        """(N, slots): cos(pi k e_j / N), the exponent reduced exactly mod 2N."""
        if getattr(self, "_cos", None) is None or self._cos.shape[1] < slots:
            k = np.arange(self.n, dtype=np.int64)[:, None]
            m = (k * self._rbin[None, :slots]) % (2 * self.n)
            self._cos = np.cos(np.pi * m / self.n)
        return self._cos[:, :slots]

    def decode_batch(self, coeffs: np.ndarray, scale: float, slots: int | None = None) -> np.ndarray:
        """decode() for each row of a (count, N) coefficient array, the first
        `slots` slots (all by default); the transforms run on every host core."""
        y = np.asarray(coeffs, dtype=np.float64) * self.zeta[None, :]
        M = _sfft.ifft(y, axis=1, norm="forward", workers=-1)    # = N * ifft(y)
        t = self.t if slots is None else self.t[:slots]
        return M[:, t] / scale


def to_rns(coef: np.ndarray, primes) -> np.ndarray:
    """Signed integer coefficients -> limb-major residues (uint64)."""
    out = []
    for q in primes:
        out.append(np.mod(coef, np.int64(q)).astype(np.uint64) if coef.dtype == np.int64
                   else np.array([int(c) % q for c in coef], dtype=np.uint64))
    return np.concatenate(out)


def crt_centered(limbs: np.ndarray, primes) -> np.ndarray:
    """Limb-major residues -> centred integer coefficients (object array)."""
    n = limbs.size // len(primes)
    if len(primes) == 1:
        q = int(primes[0])
        v = limbs.astype(object)
        return np.where(v > q // 2, v - q, v)
    Q = 1
    for q in primes:
        Q *= int(q)
    acc = np.zeros(n, dtype=object)
    for i, q in enumerate(primes):
        q = int(q)
        Qi = Q // q
        inv = pow(Qi % q, -1, q)
        v = limbs[i * n:(i + 1) * n].astype(object)
        acc = acc + (v * inv % q) * Qi
    acc = acc % Q
    return np.where(acc > Q // 2, acc - Q, acc)


class Slots:
    """Bump allocator of polynomial slots ((L + K) * N words each) in poly_gmem."""

    def __init__(self, params: CkksParams, start: int, end: int):
        self.w = (params.L + params.K) * params.n
        self.cur, self.end = start, end

    def take(self, count: int = 1) -> list[int]:
        out = []
        for _ in range(count):
            if self.cur + self.w > self.end:
                raise MemoryError("poly_gmem slots exhausted")
            out.append(self.cur)
            self.cur += self.w
        return out


class CkksClient:
    """Secret-key holder: key generation, encryption, decryption."""

    def __init__(self, ctx: FheContext, slots: Slots, seed: int = 1):
        self.ctx = ctx
        self.drv = FHEHostDriver(ctx)
        self.p = ctx.params
        self.enc = Encoder(self.p.log_n)
        self.rng = np.random.default_rng(seed)
        self.slots = slots
        n, L, K = self.p.n, self.p.L, self.p.K
        self.qp = self.p.q + self.p.p
        (self.s_slot, self.t0, self.t1, self.t2, self.t3, self.pk_b, self.pk_a) = slots.take(7)
        s = self.rng.integers(-1, 2, n).astype(np.int64)
        self.s_coef = s
        self._put_ntt(self.s_slot, s, L + K)
        # public key over Q: b = -a * s + e, a uniform (evaluation form)
        a = self._uniform(L)
        self.ctx.write_poly(self.pk_a, a)
        self._put_ntt(self.t0, self._gauss(), L)
        self.drv.poly_mul_ntt(self.pk_a, self.s_slot, self.t1, L)
        self.drv.poly_sub(self.t0, self.t1, self.pk_b, L)

    # ---- sampling helpers ----
    def _uniform(self, limbs: int, primes=None) -> np.ndarray:
        primes = primes or self.qp[:limbs]
        n = self.p.n
        return np.concatenate([self.rng.integers(0, int(q), n, dtype=np.uint64) for q in primes])

    def _gauss(self) -> np.ndarray:
        return np.rint(self.rng.normal(0.0, SIGMA, self.p.n)).astype(np.int64)

    def _put_ntt(self, off: int, coef: np.ndarray, limbs: int) -> None:
        self.ctx.write_poly(off, to_rns(coef, self.qp[:limbs]))
        self.drv.ntt(off, off, limbs)

    # ---- keys ----
    def switch_key(self, sprime_slot: int) -> np.ndarray:
        """Key from s' (evaluation form over L + K limbs at sprime_slot) to s."""
        p = self.p
        n, L, K, d = p.n, p.L, p.K, p.dnum
        LK = L + K
        P = 1
        for x in p.p:
            P *= x
        A, B = [], []
        for j in range(d):
            a = self._uniform(LK)
            self.ctx.write_poly(self.t0, a)
            self._put_ntt(self.t1, self._gauss(), LK)                     # e_j
            self.drv.poly_mul_ntt(self.t0, self.s_slot, self.t2, LK)       # a_j * s
            self.drv.poly_sub(self.t1, self.t2, self.t1, LK)               # e_j - a_j s
            g = np.zeros(LK * n, dtype=np.uint64)
            for i in range(j * p.alpha, min((j + 1) * p.alpha, L)):
                g[i * n:(i + 1) * n] = P % p.q[i]
            self.ctx.write_poly(self.t3, g)
            self.drv.poly_mul_ntt(self.t3, sprime_slot, self.t2, LK)       # gadget * s'
            self.drv.poly_add(self.t1, self.t2, self.t1, LK)
            A.append(a)
            B.append(self.ctx.read_poly(self.t1, LK * n))
        return np.concatenate(A + B)

    def relin_key(self) -> np.ndarray:
        LK = self.p.L + self.p.K
        tmp = self.slots_tmp()
        self.drv.poly_mul_ntt(self.s_slot, self.s_slot, tmp, LK)   # s^2
        return self.switch_key(tmp)

    def slots_tmp(self) -> int:
        if not hasattr(self, "_tmp"):
            self._tmp = self.slots.take(1)[0]
        return self._tmp

    def rotation_key(self, step: int) -> np.ndarray:
        from .driver import galois_elt
        LK = self.p.L + self.p.K
        k = galois_elt(self.p.log_n, step)
        self.drv.automorphism(self.s_slot, k, self.slots_tmp(), LK)
        return self.switch_key(self._tmp)

    def install_keys(self, steps, key_base: int = 0) -> int:
        """Generate the relinearisation key and one rotation key per step,
        write them to key_gmem from key_base and register them. Returns the
        first free key word."""
        kw = self.p.key_words()
        off = key_base
        self.ctx.write_key(off, self.relin_key())
        self.drv.set_relin_key(off)
        off += kw
        for s in sorted(set(steps)):
            self.ctx.write_key(off, self.rotation_key(s))
            self.drv.add_rotation_key(s, off)
            off += kw
        return off

    # ---- encryption ----
    def encrypt_coef(self, coef: np.ndarray, c0: int, c1: int, level: int | None = None) -> None:
        """Public-key encryption of integer coefficients into (c0, c1)."""
        L = level or self.p.L
        self._put_ntt(self.t0, self.rng.integers(-1, 2, self.p.n).astype(np.int64), L)   # v
        self._put_ntt(self.t1, self._gauss(), L)                                          # e0
        self._put_ntt(self.t2, self._gauss(), L)                                          # e1
        self._put_ntt(self.t3, coef, L)                                                   # m
        self.drv.poly_mul_ntt(self.t0, self.pk_b, c0, L)
        self.drv.poly_add(c0, self.t1, c0, L)
        self.drv.poly_add(c0, self.t3, c0, L)
        self.drv.poly_mul_ntt(self.t0, self.pk_a, c1, L)
        self.drv.poly_add(c1, self.t2, c1, L)

    def encrypt(self, values, scale: float, c0: int, c1: int, level: int | None = None) -> None:
        self.encrypt_coef(self.enc.encode(values, scale), c0, c1, level)

    def decrypt_coef(self, c0: int, c1: int, level: int) -> np.ndarray:
        self.drv.poly_mul_ntt(c1, self.s_slot, self.t0, level)
        self.drv.poly_add(c0, self.t0, self.t0, level)
        self.drv.intt(self.t0, self.t0, level)
        limbs = self.ctx.read_poly(self.t0, level * self.p.n)
        return crt_centered(limbs, self.p.q[:level])

    def decrypt(self, c0: int, c1: int, level: int, scale: float) -> np.ndarray:
        coef = self.decrypt_coef(c0, c1, level).astype(np.float64)
        return self.enc.decode(coef, scale)

    def decrypt_host(self, c0_limbs: np.ndarray, c1_limbs: np.ndarray, level: int, scale: float) -> np.ndarray:
        """Decrypt a ciphertext the server returned as host arrays."""
        n = self.p.n
        off0, off1 = self.slots_pair()
        self.ctx.write_poly(off0, c0_limbs[:level * n])
        self.ctx.write_poly(off1, c1_limbs[:level * n])
        return self.decrypt(off0, off1, level, scale)

    def slots_pair(self) -> tuple[int, int]:
        if not hasattr(self, "_pair"):
            self._pair = tuple(self.slots.take(2))
        return self._pair

    def _region(self, name: str, words: int) -> int:
        """A contiguous client work region of at least `words` words (cached)."""
        have = getattr(self, "_regions", {})
        self._regions = have
        if name not in have or have[name][1] < words:
            # grow at least twofold, so that slowly rising batch sizes do not
            # leave a trail of outgrown regions behind
            k = max(-(-words // self.slots.w), 2 * (have[name][1] // self.slots.w if name in have else 0))
            have[name] = (self.slots.take(k)[0], k * self.slots.w)
        return have[name][0]

    def decrypt_batch(self, cts, level: int, scale: float, slots: int | None = None) -> np.ndarray:
        """Decrypt ciphertexts resident in poly_gmem; returns (count, slots) slot
        values (all N/2 slots by default)."""
        return self.enc.decode_batch(self.decrypt_batch_coef(cts, level), scale, slots)

    def decrypt_batch_coef(self, cts, level: int) -> np.ndarray:
        """The device part of decryption: m = c0 + c1 s, INTT, centred CRT
        lift on the host; returns (count, N) float64 coefficients (decode
        them with `enc.decode_batch`)."""
        from . import _lib as L
        n, count = self.p.n, len(cts)
        out = self._region("dec_out", count * level * n)
        arr = (L.CtRef * max(count, 1))()
        for i, (a, b) in enumerate(cts):
            arr[i].c0_offset, arr[i].c1_offset = a, b
        L.check(self.ctx.lib.afhe_decrypt_batch(self.ctx.h, arr, count, self.s_slot, out, level), "decrypt_batch")
        limbs = self.ctx.read_poly(out, count * level * n,
                                   self.ctx.staging.get("dec_coef", count * level * n)).reshape(count, level * n)
        return centred_coefficients(limbs, self.p.q, level)

    def decrypt_decode(self, cts, scales, slots: int) -> np.ndarray:
        """Decrypt ciphertexts resident in poly_gmem from limb 0 and decode
        them on the device (afhe_decrypt_batch, afhe_decode_batch): (count,
        slots) real slot values, row i at scales[i]."""
        return _decrypt_decode(self.ctx, cts, self.s_slot, self._region("dec_out", len(cts) * self.p.n), scales,
                               slots)

    def decryptor(self, max_count: int, max_level: int = 1) -> "CkksDecryptor":
        """This client's decryption on a device context of its own (see
        CkksDecryptor); closed with close_decryptors()."""
        d = CkksDecryptor(self, max_count, max_level)
        self._decryptors = getattr(self, "_decryptors", []) + [d]
        return d

    def close_decryptors(self) -> None:
        for d in getattr(self, "_decryptors", []):
            d.close()
        self._decryptors = []

    def decrypt_host_batch(self, cts: np.ndarray, level: int, scale: float, slots: int | None = None) -> np.ndarray:
        """Decrypt ciphertexts received as a host array (count, 2, level * N)."""
        return self.enc.decode_batch(self.decrypt_host_batch_coef(cts, level), scale, slots)

    def decrypt_host_batch_coef(self, cts: np.ndarray, level: int) -> np.ndarray:
        """The device part of `decrypt_host_batch`: (count, N) float64 coefficients."""
        n, count = self.p.n, cts.shape[0]
        w = level * n
        inp = self._region("dec_in", count * 2 * w)
        self.ctx.write_poly(inp, np.ascontiguousarray(cts).ravel())
        return self.decrypt_batch_coef([(inp + 2 * i * w, inp + (2 * i + 1) * w) for i in range(count)], level)

    def plaintext(self, values, scale: float, off: int, level: int) -> None:
        """Encode `values` into an evaluation-form plaintext at `off` (level limbs)."""
        self._put_ntt(off, self.enc.encode(values, scale), level)


def centred_coefficients(limbs: np.ndarray, q, level: int) -> np.ndarray:
    """(count, level * N) residues of decrypted polynomials -> (count, N)
    float64 coefficients, centred in (-Q/2, Q/2] for Q = q_0 ... q_(level-1)."""
    if level == 1 and q[0] < 2**53:
        # centre in 64-bit integers, then convert: values below 2^53 are exact
        s = limbs.view(np.int64)
        return (s - (s > q[0] // 2) * np.int64(q[0])).astype(np.float64)
    return np.stack([crt_centered(row, q[:level]).astype(np.float64) for row in limbs])


class CkksDecryptor:
    """The client's decryption on a device context of its own: its own stream
    and arenas, holding only the first limbs of the secret key's evaluation
    form. Its device work does not queue behind the server's work on the
    server's context, so the client can decrypt the results of one group of
    queries while the server computes the next group. Same arithmetic and
    results as CkksClient.decrypt_host_batch_coef."""

    def __init__(self, client: CkksClient, max_count: int, max_level: int = 1):
        p = client.p
        n = p.n
        self.p, self.enc = p, client.enc
        self.max_count, self.max_level = max_count, max_level
        self.s_off = 0
        self.in_off = max_level * n
        self.out_off = self.in_off + 2 * max_count * max_level * n
        self.ctx = FheContext(p, poly_words=self.out_off + max_count * max_level * n, key_words=n,
                              device=client.ctx.device, max_batch=1)
        self.ctx.write_poly(self.s_off, client.ctx.read_poly(client.s_slot, max_level * n))

    def decrypt_host_batch_coef(self, cts: np.ndarray, level: int) -> np.ndarray:
        """Ciphertexts received as a host array (count, 2, level * N) -> (count,
        N) float64 coefficients: m = c0 + c1 s and the INTT on the device,
        centring on the host."""
        from . import _lib as L
        n, count = self.p.n, cts.shape[0]
        if count > self.max_count or not 1 <= level <= self.max_level:
            raise ValueError(f"{count} ciphertexts at level {level}: the decryptor holds "
                             f"{self.max_count} at levels up to {self.max_level}")
        w = level * n
        self.ctx.write_poly(self.in_off, np.ascontiguousarray(cts).reshape(-1))
        arr = (L.CtRef * max(count, 1))()
        for i in range(count):
            arr[i].c0_offset, arr[i].c1_offset = self.in_off + 2 * i * w, self.in_off + (2 * i + 1) * w
        L.check(self.ctx.lib.afhe_decrypt_batch(self.ctx.h, arr, count, self.s_off, self.out_off, level),
                "decrypt_batch")
        limbs = self.ctx.read_poly(self.out_off, count * w, self.ctx.staging.get("dec_coef", count * w))
        return centred_coefficients(limbs.reshape(count, w), self.p.q, level)

    def decrypt_decode_host(self, cts: np.ndarray, scales, slots: int) -> np.ndarray:
        """Ciphertexts received as a host array (count, 2, N) (limb 0) ->
        (count, slots) real slot values, row i at scales[i]: decryption and
        decoding on the device (afhe_decode_batch)."""
        n, count = self.p.n, cts.shape[0]
        if count > self.max_count:
            raise ValueError(f"{count} ciphertexts: the decryptor holds {self.max_count}")
        self.ctx.write_poly(self.in_off, np.ascontiguousarray(cts).reshape(-1))
        refs = [(self.in_off + 2 * i * n, self.in_off + (2 * i + 1) * n) for i in range(count)]
        return _decrypt_decode(self.ctx, refs, self.s_off, self.out_off, scales, slots)

    def close(self) -> None:
        self.ctx.close()


def _decrypt_decode(ctx: FheContext, cts, s_off: int, out: int, scales, slots: int) -> np.ndarray:
    """m = c0 + c1 s of each ciphertext (limb 0) into out + i N, then its
    slots decoded on the device into page-locked staging."""
    from . import _lib as L
    n, count = ctx.params.n, len(cts)
    arr = (L.CtRef * max(count, 1))()
    for i, (a, b) in enumerate(cts):
        arr[i].c0_offset, arr[i].c1_offset = a, b
    L.check(ctx.lib.afhe_decrypt_batch(ctx.h, arr, count, s_off, out, 1), "decrypt_batch")
    coef = np.arange(count, dtype=np.uint64) * np.uint64(n) + np.uint64(out)
    sc = np.ascontiguousarray(np.broadcast_to(np.asarray(scales, dtype=np.float64), (count,)))
    res = ctx.staging.get("decoded", count * slots).view(np.float64).reshape(count, slots)
    L.check(ctx.lib.afhe_decode_batch(ctx.h, coef.ctypes.data_as(L.P64), sc.ctypes.data_as(C.POINTER(C.c_double)),
                                      count, slots, res.ctypes.data_as(C.POINTER(C.c_double))), "decode_batch")
    return res


def encode_plaintexts(ctx: FheContext, enc: Encoder, values: np.ndarray, scale: float, offs, level: int) -> None:
    """Server-side encoding of many real plaintexts on the device
    (afhe_encode_batch: special FFT, rounding, RNS, NTT): row i of `values`
    into the evaluation-form polynomial at offs[i] (level limbs). `enc` is the
    encoder whose slot order the device follows (the same canonical
    embedding)."""
    from . import _lib as L
    v = np.ascontiguousarray(values, dtype=np.float64)
    if v.ndim == 1:
        v = v[None, :]
    o = np.ascontiguousarray(offs, dtype=np.uint64)
    assert v.shape[0] == o.size and v.shape[1] <= enc.slots
    L.check(ctx.lib.afhe_encode_batch(ctx.h, v.ctypes.data_as(C.POINTER(C.c_double)), v.shape[0], v.shape[1],
                                      float(scale), level, o.ctypes.data_as(L.P64)), "encode_batch")


def encode_index_batches(ctx: FheContext, index, vids, first, counts, offs, scale: float, level: int,
                         norms: bool = False, layout: str = "batches", n1: int = 0, coef: float = 1.0) -> None:
    """The stage-3 candidate plaintexts built and encoded on the device
    (afhe_pq_*): batch b holds candidates vids[first[b] .. first[b] +
    counts[b]); slot d B + j = component d of candidate j's reconstruction
    (centroid of its list + its PQ codewords). With `norms`, the batches'
    squared norms instead: slot d B + j = ||x_j||^2 in every row d.
    layout "diagonals": the diagonal method's D plaintexts per unit (of up to
    N/2 candidates) into offs[u D + i] (afhe_pq_encode_diagonals, n1 baby
    steps, values times coef); "unit_norms": slot j = ||x_j||^2 per unit."""
    from . import _lib as L
    cent = np.ascontiguousarray(index.centroids, dtype=np.float32)
    books = np.ascontiguousarray(index.codebooks, dtype=np.float32)
    codes = np.ascontiguousarray(index.codes, dtype=np.uint8)
    assign = np.ascontiguousarray(index.assignments, dtype=np.uint32)
    M, K, sd = books.shape
    ix = L.PqIndex(cent.shape[0], cent.shape[1], M, K, codes.shape[0], cent.ctypes.data_as(C.POINTER(C.c_float)),
                   books.ctypes.data_as(C.POINTER(C.c_float)), codes.ctypes.data_as(C.POINTER(C.c_uint8)),
                   assign.ctypes.data_as(L.P32))
    h = C.c_void_p()
    L.check(ctx.lib.afhe_pq_create(ctx.h, C.byref(ix), C.byref(h)), "pq_create")
    try:
        v = np.ascontiguousarray(vids, dtype=np.uint32)
        f = np.ascontiguousarray(first, dtype=np.uint32)
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        o = np.ascontiguousarray(offs, dtype=np.uint64)
        args = (v.ctypes.data_as(L.P32), f.ctypes.data_as(L.P32), c.ctypes.data_as(L.P32))
        if layout == "diagonals":
            assert o.size == c.size * cent.shape[1]
            L.check(ctx.lib.afhe_pq_encode_diagonals(h, *args, c.size, n1, float(coef), float(scale), level,
                                                     o.ctypes.data_as(L.P64)), "pq_encode_diagonals")
        elif layout == "unit_norms":
            L.check(ctx.lib.afhe_pq_encode_unit_norms(h, *args, c.size, float(scale), level,
                                                      o.ctypes.data_as(L.P64)), "pq_encode_unit_norms")
        else:
            fn = ctx.lib.afhe_pq_encode_norms if norms else ctx.lib.afhe_pq_encode_batches
            L.check(fn(h, *args, o.size, float(scale), level, o.ctypes.data_as(L.P64)), "pq_encode")
    finally:
        ctx.lib.afhe_pq_destroy(h)


def encode_plaintexts_host(ctx: FheContext, enc: Encoder, values: np.ndarray, scale: float, offs, level: int,
                           chunk: int = 256) -> None:
    """encode_plaintexts with the host encoder (numpy FFT) and a device NTT:
    the exactly rounded coefficients, for comparison."""
    from . import _lib as L
    primes = [np.int64(q) for q in ctx.params.q[:level]]
    for c0 in range(0, len(offs), chunk):
        rows = enc.encode_batch(values[c0:c0 + chunk], scale)
        part = list(offs[c0:c0 + chunk])
        for coef, off in zip(rows, part):
            ctx.write_poly(off, np.concatenate([np.mod(coef, q).astype(np.uint64) for q in primes]))
        arr = (L.u64 * len(part))(*part)
        L.check(ctx.lib.afhe_ntt_batch(ctx.h, arr, len(part), level, 0), "ntt_batch")


def encode_plaintext(ctx: FheContext, enc: Encoder, values, scale: float, off: int, level: int) -> None:
    """Server-side plaintext encoding (no secret involved)."""
    coef = enc.encode(values, scale)
    ctx.write_poly(off, to_rns(coef, ctx.params.q[:level]))
    FHEHostDriver(ctx).ntt(off, off, level)
