"""End-to-end encrypted IVF-PQ on the GPU (small configuration: N = 2^13,
4,096 x 64 database, n_list 32, nprobe 4).

* decrypted coarse distances match the plaintext IVF coarse distances, and
  decrypted candidate distances match the plaintext ADC distances, within the
  CKKS tolerance of the scale. Results carry scale 2^80 / q_2 ~ 2^30. One key
  switch adds noise of rms ~ sqrt(2N/3) / sqrt(3) ~ 43 per coefficient (the
  approximate ModDown's floor rounding times the ternary secret), i.e.
  ~ sqrt(N) * 43 / 2^30 ~ 4e-6 per slot; a query runs ~100 key switches and
  64-slot tree sums, so errors stay below 1e-2 absolute (measured: ~1e-3 at
  distances of order 100-200);
* probed lists and top-k ids are identical to the plaintext search;
* the batched server (16 lanes) and the plain one-ciphertext-at-a-time server
  produce bit-identical result ciphertexts.
"""
import numpy as np
import pytest

from anns_fhe_b200.workloads import Workload

pytestmark = pytest.mark.gpu
TOL = 1e-2


@pytest.fixture(scope="module")
def wl():
    w = Workload(max_queries=8, lanes=16)
    yield w
    w.close()


def test_end_to_end_matches_plaintext(wl):
    Q = wl.queries(5, seed=3)
    res = wl.run(Q)
    for q, r in zip(Q, res):
        coarse, probes, cand, dist, top = wl.plaintext(q)
        assert np.max(np.abs(r["coarse"] - coarse)) < TOL
        assert list(r["probes"]) == list(probes)
        assert r["vids"] == list(cand)
        assert np.max(np.abs(r["dists"] - dist)) < TOL
        assert r["topk"] == list(top)


def test_batched_equals_plain(wl):
    Q = wl.queries(3, seed=5)
    recs = wl.records[:3]
    wl.run(Q, recs)
    batched = [(wl.iqm.read_ct(r.compact), wl.iqm.read_ct(r.dists)) for r in recs]
    # same ciphertexts in, one lane at a time
    lanes = wl.iqm.lanes
    try:
        wl.iqm.lanes = 1
        wl.iqm.stage1_coarse(recs)
        wl.iqm.stage3_fine(recs)
    finally:
        wl.iqm.lanes = lanes
    for r, (c, d) in zip(recs, batched):
        c2, d2 = wl.iqm.read_ct(r.compact), wl.iqm.read_ct(r.dists)
        assert all(np.array_equal(x, y) for x, y in zip(c, c2))
        assert all(np.array_equal(x, y) for x, y in zip(d, d2))


def test_pipelined_host_protocol(wl):
    """The host-buffer protocol with the queries split into groups whose
    client and server work overlap (asynchronous result reads, fences, the
    client decrypting on a context of its own) gives the same probes and
    top-k for 1, 2 and 4 groups, and the plaintext search's top-k. The
    decryptor's coefficients equal the client's own decryption."""
    Q = wl.queries(6, seed=11)
    recs = wl.records[:6]
    for r in recs:
        r.nprobe = 0
    wl.encrypt_queries(Q, recs)
    w = wl.params.L * wl.params.n
    host = [[wl.ctx.read_poly(o, w) for o in (*r.ct_query, *r.ct_dim)] for r in recs]
    dec = wl.client.decryptor(6 * max(1, wl.iqm.n_res))
    try:
        outs = []
        for groups in (1, 2, 4):
            top, h2d, d2h = wl.run_host_pipelined(recs, host, dec, groups)
            assert h2d == 6 * 4 * w * 8 and d2h > 0
            outs.append((top, [list(r.probes) for r in recs]))
        assert outs[0] == outs[1] == outs[2]
        for q, t, pr in zip(Q, *outs[1]):
            coarse, probes, cand, dist, want = wl.plaintext(q)
            assert pr == list(probes) and t == list(want)
        # streamed: 14 queries (the 6 in turn) in groups of 2 over 4 slices of the 8 records
        top, h2d, d2h = wl.run_host_stream(wl.records[:8], host, dec, total=14, group=2)
        assert top == [outs[0][0][i % 6] for i in range(14)]
        assert h2d == 14 * 4 * w * 8
        with pytest.raises(ValueError):
            wl.run_host_stream(wl.records[:5], host, dec, total=4, group=2)
        box = wl.iqm.read_results("compact", recs)[:, 0]
        assert np.array_equal(dec.decrypt_host_batch_coef(box, 1), wl.client.decrypt_host_batch_coef(box, 1))
        with pytest.raises(ValueError):
            dec.decrypt_host_batch_coef(np.zeros((6 * max(1, wl.iqm.n_res) + 1, 2, wl.params.n), np.uint64), 1)
    finally:
        dec.close()


def test_decryptor_at_every_level(wl):
    """The client's own decryption context gives the client's coefficients
    at level 1 (limb 0, the fast centring) and at the top level (CRT)."""
    recs = wl.records[:2]
    wl.encrypt_queries(wl.queries(2, seed=4), recs)
    n, L = wl.params.n, wl.params.L
    cts = np.stack([np.stack([wl.ctx.read_poly(r.ct_query[0], L * n), wl.ctx.read_poly(r.ct_query[1], L * n)])
                    for r in recs])
    dec = wl.client.decryptor(2, max_level=L)
    try:
        for lv in sorted({1, L}):
            part = np.ascontiguousarray(cts[:, :, :lv * n])
            assert np.array_equal(dec.decrypt_host_batch_coef(part, lv), wl.client.decrypt_host_batch_coef(part, lv))
        with pytest.raises(ValueError):
            dec.decrypt_host_batch_coef(cts[:, :, :n], L + 1)
    finally:
        dec.close()
