"""Host-side CKKS pieces that need no GPU: the encoder's round trip, the slot
rotation convention (X -> X^(5^r) rotates slots left by r), RNS conversion and
CRT reconstruction, the IVF-PQ index and the rotation-key set of the chain."""
import numpy as np

from anns_fhe_b200.ckks import Encoder, crt_centered, to_rns
from anns_fhe_b200.ivfpq import IvfPqIndex, gaussian_mixture, plaintext_search
from anns_fhe_b200.query import InteractiveQueryManager, pow2_steps


def coef_automorphism(coef: np.ndarray, k: int) -> np.ndarray:
    n = coef.size
    out = np.zeros(n, dtype=np.float64)
    for i, c in enumerate(coef):
        e = i * k % (2 * n)
        if e < n:
            out[e] += c
        else:
            out[e - n] -= c
    return out


def test_encoder_roundtrip_and_rotation():
    enc = Encoder(10)
    rng = np.random.default_rng(0)
    z = rng.normal(0, 10, enc.slots)
    scale = 2.0**30
    coef = enc.encode(z, scale)
    assert np.max(np.abs(enc.decode(coef, scale).real - z)) < 1e-6
    for r in (1, 3, -2):
        k = pow(5, r % (enc.n // 2), 2 * enc.n)
        rot = enc.decode(coef_automorphism(coef.astype(np.float64), k), scale).real
        assert np.max(np.abs(rot - np.roll(z, -r))) < 1e-6


def test_rns_crt_roundtrip():
    q = [1125899906826241, 1125899906629633, 1125899906596865]
    rng = np.random.default_rng(1)
    v = rng.integers(-(2**62), 2**62, 64, dtype=np.int64)
    for k in (1, 2, 3):
        back = crt_centered(to_rns(v, q[:k]), q[:k])
        if k >= 2:
            assert [int(x) for x in back] == [int(x) for x in v]
        else:
            assert all((int(a) - int(b)) % q[0] == 0 for a, b in zip(back, v))


def test_ivfpq_index_and_plaintext_search():
    X = gaussian_mixture(2048, 32, 16, 0.1, 5)
    idx = IvfPqIndex.train(X, n_list=16, M=4, K=32, seed=5, iters=10)
    assert sum(len(v) for v in idx.lists) == len(X)
    probes, cand, dist, top = plaintext_search(idx, X[0], nprobe=2, top_k=5)
    assert len(top) == 5 and idx.assignments[0] in probes


def test_pow2_steps():
    assert pow2_steps(63 * 5) == [256, 32, 16, 8, 2, 1]
    assert pow2_steps(-6) == [4, 2]
    assert sum(pow2_steps(12345)) == 12345


def test_query_layouts():
    """Client-side slot layouts: ct_query replicates q per centroid of a
    coarse ciphertext, ct_dimpack puts q[d] at every candidate slot d * B + j."""
    import numpy as np

    from anns_fhe_b200.query import QueryShape
    from anns_fhe_b200.workloads import dimpack_layout, query_layout
    q = np.arange(8, dtype=np.float32) + 1
    ref = QueryShape(D=8, n_list=4, slots=64, nprobe=1, top_k=1, scale=1.0)
    a = query_layout(q, ref)
    assert np.array_equal(a[:32], np.tile(q, 4)) and not a[32:].any()
    packed = QueryShape(D=8, n_list=20, slots=64, nprobe=1, top_k=1, scale=1.0, compaction="packed")
    assert packed.per_ct == 8 and packed.n_coarse == 3
    assert np.array_equal(query_layout(q, packed), np.tile(q, 8))
    d = dimpack_layout(q, packed)
    assert d.size == 64 and all(d[i * 8 + j] == q[i] for i in range(8) for j in range(8))
    # coarse slot map: list k * per_ct + c at slot c * D + k
    assert packed.coarse_slot(8 * 2 + 5) == 5 * 8 + 2
    assert sorted(packed.coarse_slot(c) for c in range(20)) == sorted({packed.coarse_slot(c) for c in range(20)})


def test_batch_offsets_never_straddle():
    """Candidate batches land whole in one result ciphertext, back to back
    otherwise, and fit the number of results `results_needed` reserves."""
    import numpy as np

    from anns_fhe_b200.query import InteractiveQueryManager, batch_offsets
    rng = np.random.default_rng(0)
    for S, B in ((512, 64), (16384, 128), (4096, 64)):
        counts = [int(x) for x in rng.integers(1, B + 1, 400)]
        offs = batch_offsets(counts, S)
        end = 0
        for off, cnt in zip(offs, counts):
            assert off // S == (off + cnt - 1) // S, "batch crosses a result boundary"
            assert off == end or (off % S == 0 and off > end), "gap other than a result start"
            end = off + cnt
        assert end <= InteractiveQueryManager.results_needed(sum(counts), S, B) * S
    assert batch_offsets([3, 3, 3], 8) == [0, 3, 8]


def test_decode_real_matches_decode():
    """The client's real decode (a zero-padded real FFT of length 2N, or a
    cosine-matrix product for a few slots) gives the real parts of the
    canonical-embedding decode, to float64 rounding, with per-row scales."""
    import numpy as np

    from anns_fhe_b200.ckks import Encoder
    e = Encoder(10)
    rng = np.random.default_rng(3)
    coef = np.rint(rng.normal(0, 1e9, (5, 1024)))
    want = np.stack([e.decode(c, 2.0**30).real for c in coef])
    for slots in (None, 100, 8):
        got = e.decode_real_batch(coef, 2.0**30, slots)
        assert got.shape == (5, slots or 512)
        assert np.max(np.abs(got - want[:, :got.shape[1]])) < 1e-12 * np.max(np.abs(want))
    sc = np.array([1.0, 2.0, 4.0, 8.0, 16.0]) * 2.0**30
    got = e.decode_real_batch(coef, sc, 8)
    assert np.allclose(got * sc[:, None] / 2.0**30, e.decode_real_batch(coef, 2.0**30, 8), rtol=0, atol=1e-9)


def test_norm_reserve_within_budget():
    """The candidate-norm plaintexts of the packed chain: levels lowest first,
    then the spare levels at L, while their slots fit the budget; the large
    configuration (7,813 batches, N = 2^15, L = 12, slots of 16 N words)."""
    from anns_fhe_b200.query import NORM_BUDGET_BYTES
    IQM = InteractiveQueryManager
    n, L, nb = 1 << 15, 12, 7813
    w = 16 * n
    per = {lv: IQM.norm_plaintext_slots(nb, lv, n, w) for lv in range(3, L + 1)}
    assert per[3] == -(-nb * 2 // 16) and per[12] == -(-nb * 11 // 16)
    # evaluation at 3 limbs, plus one spare level for the full-level leg
    assert IQM.norm_reserve_slots([3], 1, nb, L, n, w) == per[3] + per[12]
    # query levels 6..12 at their own level: 6 and 7 fit 32 GiB, 8 does not
    r = IQM.norm_reserve_slots(range(6, 13), 0, nb, L, n, w)
    assert r == per[6] + per[7] and (r + per[8]) * w * 8 > NORM_BUDGET_BYTES >= r * w * 8
    assert IQM.norm_reserve_slots([3], 0, nb, L, n, w, budget=0) == 0
    assert IQM.norm_reserve_slots([], 0, nb, L, n, w) == 0


def test_diagonal_method_algebra():
    """The diagonal chain's plaintexts and steps, on plaintext slot vectors:
    sum over g of rot(sum over b of pt_{g,b} * rot(q, b), n1 g) = -2 <q, x_j>
    in slot j, 0 elsewhere; a unit's plaintexts moved right by a multiple of
    D (its placement) move the result by the same amount."""
    from anns_fhe_b200.query import QueryShape
    rng = np.random.default_rng(0)
    for S, D, rows in ((512, 16, 70), (1024, 8, 1024), (2048, 64, 300)):
        sh = QueryShape(D=D, n_list=4, slots=S, nprobe=1, top_k=1, scale=1.0, compaction="diagonal")
        n1, n2 = sh.n1, sh.n2
        assert n1 * n2 == D and n1 >= n2
        X, q = rng.normal(size=(rows, D)), rng.normal(size=D)
        P = InteractiveQueryManager.diagonal_values(X, S, D, n1)
        rot = lambda v, r: np.roll(v, -r)      # noqa: E731  slot k <- slot k + r
        baby = [rot(np.tile(q, S // D), b) for b in range(n1)]
        for o in {o for o in (0, D, (S - rows) // D * D) if o + rows <= S}:
            out = sum(rot(sum(rot(P[g * n1 + b], -o) * baby[b] for b in range(n1)), n1 * g) for g in range(n2))
            assert np.allclose(out[o:o + rows], -2 * X @ q)
            assert np.allclose(np.delete(out, np.arange(o, o + rows)), 0)


def test_unit_offsets():
    from anns_fhe_b200.query import unit_offsets
    assert unit_offsets([5, 8, 9], 32, 8) == [0, 8, 16]
    assert unit_offsets([5, 8, 9, 1], 32, 8) == [0, 8, 16, 32]
    assert unit_offsets([32, 1, 32], 32, 8) == [0, 32, 64]
    assert unit_offsets([], 32, 8) == []
    rng = np.random.default_rng(1)
    counts = [int(x) for x in rng.integers(1, 513, 300)]
    offs = unit_offsets(counts, 512, 8)
    for off, cnt in zip(offs, counts):
        assert off % 8 == 0 and off // 512 == (off + cnt - 1) // 512


def test_diagonal_results_bound():
    """results_for (diagonal chain) covers every probe set of up to nprobe
    lists: random list sizes (some longer than the slots), random probes."""
    from types import SimpleNamespace

    from anns_fhe_b200.query import QueryShape, unit_offsets
    rng = np.random.default_rng(7)
    for S, D, nprobe in ((512, 8, 40), (16384, 128, 16), (4096, 64, 4)):
        sizes = [int(x) for x in rng.integers(0, 3 * S // 2, 200)]
        index = SimpleNamespace(lists=[list(range(k)) for k in sizes])
        sh = QueryShape(D=D, n_list=200, slots=S, nprobe=nprobe, top_k=1, scale=1.0, compaction="diagonal")
        bound = InteractiveQueryManager.results_for(index, sh, nprobe)
        for _ in range(300):
            probes = rng.choice(200, size=int(rng.integers(1, nprobe + 1)), replace=False)
            counts = [min(S, sizes[c] - u0) for c in probes for u0 in range(0, sizes[c], S)]
            offs = unit_offsets(counts, S, D)
            used = offs[-1] // S + 1 if offs else 1
            assert used <= bound
