"""Server-side encoding on the device (afhe_encode_batch, afhe_pq_*) against
the host encoder.

The host encoder (anns_fhe_b200.ckks.Encoder: the canonical embedding's
inverse by numpy FFT, rounded to nearest) gives the exactly rounded
coefficients up to its own rounding error. The device runs a different
double-precision transform (the special FFT), so a coefficient may come out
one away where the exact value lies within either transform's rounding error
of a half-integer: at most one in 1000 coefficients may differ, and by one
at most. The plaintexts then decode to the values within the encoding
precision. The candidate plaintexts built on the device from the IVF-PQ
index are identical word for word to afhe_encode_batch of the host's
reconstructions (the same doubles: float32 centroid + float32 codeword)."""
import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.ckks import Encoder, encode_index_batches, encode_plaintexts, encode_plaintexts_host
from anns_fhe_b200.driver import CkksParams, FheContext
from anns_fhe_b200.ivfpq import IvfPqIndex, gaussian_mixture

pytestmark = pytest.mark.gpu


def coefficients(ctx, off, limbs):
    """Coefficient form (INTT on the device) of the polynomial at off."""
    w = limbs * ctx.params.n
    tmp = ctx.params.L * ctx.params.n * 40
    ctx.write_poly(tmp, ctx.read_poly(off, w))
    L.check(ctx.lib.afhe_ntt_batch(ctx.h, (L.u64 * 1)(tmp), 1, limbs, 1), "ntt_batch")
    return ctx.read_poly(tmp, w).reshape(limbs, -1)


def centred(x, q):
    x = x.astype(np.int64) if q < 2 ** 62 else x
    return np.where(x > q // 2, x - np.int64(q), x)


@pytest.mark.parametrize("log_n", [10, 13, 15, 16])
def test_encode_batch_matches_host(log_n):
    prm = CkksParams.generate(log_n, 3, 50, 1, 60, 1)
    n, S = prm.n, prm.n // 2
    ctx = FheContext(prm, poly_words=48 * prm.L * n, key_words=1024)
    try:
        rng = np.random.default_rng(log_n)
        rows = [rng.standard_normal(S) * 3, rng.uniform(-1, 1, S // 3), np.zeros(7), np.eye(1, S // 2, 5)[0]]
        scales = [2.0 ** 40, 2.0 ** 30, 2.0 ** 40, float(prm.q[1])]
        enc = Encoder(log_n)
        for r, (vals, sc) in enumerate(zip(rows, scales)):
            dev, host = 8 * r * prm.L * n, (8 * r + 4) * prm.L * n
            encode_plaintexts(ctx, enc, vals[None, :], sc, [dev], prm.L)
            encode_plaintexts_host(ctx, enc, vals[None, :], sc, [host], prm.L)
            a, b = coefficients(ctx, dev, prm.L), coefficients(ctx, host, prm.L)
            for i, q in enumerate(prm.q):
                d = centred(a[i], q) - centred(b[i], q)
                assert np.all(np.abs(d) <= 1), f"row {r}: a coefficient differs by more than one"
                assert np.count_nonzero(d) <= max(1, n // 1000), f"row {r}: {np.count_nonzero(d)} coefficients differ"
            got = enc.decode(centred(a[0], prm.q[0]).astype(np.float64), sc)[:vals.size].real
            assert np.max(np.abs(got - vals)) < 1e-4
        with pytest.raises(L.AfheError):            # coefficients of 2^62 and more
            encode_plaintexts(ctx, enc, np.full((1, S), 1e6), 2.0 ** 50, [0], prm.L)
    finally:
        ctx.close()


def test_pq_batches_equal_encode_of_reconstructions():
    X = gaussian_mixture(1500, 32, 8, 0.1, 5)
    index = IvfPqIndex.train(X, 8, 4, 16, 5, iters=5)
    prm = CkksParams.generate(11, 3, 50, 1, 60, 1)
    n, S, D = prm.n, prm.n // 2, 32
    B = S // D
    ctx = FheContext(prm, poly_words=400 * prm.L * n, key_words=1024)
    try:
        vids, first, cnt, rows = [], [], [], []
        for c in range(index.n_list):
            vl = index.lists[c]
            for b0 in range(0, len(vl), B):
                ids = vl[b0:b0 + B]
                first.append(len(vids))
                cnt.append(len(ids))
                vids.extend(ids)
                packed = np.zeros((D, B))
                packed[:, :len(ids)] = index.reconstruct(ids).T
                rows.append(packed.ravel())
        m = len(rows)
        assert m > 8 and min(cnt) < B
        a = [i * prm.L * n for i in range(m)]
        b = [(m + i) * prm.L * n for i in range(m)]
        encode_index_batches(ctx, index, vids, first, cnt, a, 2.0 ** 40, prm.L)
        encode_plaintexts(ctx, Encoder(11), np.stack(rows), 2.0 ** 40, b, prm.L)
        for i in range(m):
            assert np.array_equal(ctx.read_poly(a[i], prm.L * n), ctx.read_poly(b[i], prm.L * n)), f"batch {i}"
    finally:
        ctx.close()


@pytest.mark.parametrize("log_n", [10, 13, 15])
def test_decode_batch_matches_host(log_n):
    """afhe_decode_batch (the client's decoding on the device) against the
    host decoder (Encoder.decode_real_batch) on random centred coefficients
    of up to 2^45 in limb 0: equal to 1e-9 relative to the largest slot, for
    every slot and for a prefix of slots; and the round trip through
    afhe_encode_batch returns the encoded values."""
    from anns_fhe_b200.driver import find_ntt_primes
    q = find_ntt_primes(log_n, 50, 2, [])
    p = find_ntt_primes(log_n, 60, 1, q)
    prm = CkksParams(log_n, q, p, 1)
    n = prm.n
    ctx = FheContext(prm, poly_words=128 * n, key_words=1024)
    try:
        rng = np.random.default_rng(log_n)
        enc = Encoder(log_n)
        c = rng.integers(-(1 << 45), 1 << 45, size=(6, n), dtype=np.int64)
        offs = np.arange(6, dtype=np.uint64) * np.uint64(2 * n)
        for i in range(6):
            ctx.write_poly(int(offs[i]), np.mod(c[i], q[0]).astype(np.uint64))
        scales = np.array([2.0 ** 30, 2.0 ** 40, 1.0, 3.5, 2.0 ** 20, 7.0])
        for slots in (n // 2, 37):
            out = np.zeros((6, slots))
            L.check(ctx.lib.afhe_decode_batch(ctx.h, offs.ctypes.data_as(L.P64),
                                              scales.ctypes.data_as(L.C.POINTER(L.C.c_double)), 6, slots,
                                              out.ctypes.data_as(L.C.POINTER(L.C.c_double))), "decode_batch")
            want = enc.decode_real_batch(c.astype(np.float64), scales, slots)
            assert np.max(np.abs(out - want) / np.max(np.abs(want), axis=1, keepdims=True)) < 1e-9
        # encode then decode (coefficient form via the INTT) returns the values
        vals = rng.normal(size=(3, n // 2)) * 100
        pts = [int(12 * 2 * n + 2 * i * n) for i in range(3)]
        encode_plaintexts(ctx, enc, vals, 2.0 ** 40, pts, 1)
        for i, off in enumerate(pts):
            ctx.write_poly(off, coefficients(ctx, off, 1)[0])
        out = np.zeros((3, n // 2))
        po = np.array(pts, dtype=np.uint64)
        sc = np.full(3, 2.0 ** 40)
        L.check(ctx.lib.afhe_decode_batch(ctx.h, po.ctypes.data_as(L.P64), sc.ctypes.data_as(L.C.POINTER(L.C.c_double)),
                                          3, n // 2, out.ctypes.data_as(L.C.POINTER(L.C.c_double))), "decode_batch")
        assert np.max(np.abs(out - vals)) < 1e-6
    finally:
        ctx.close()
