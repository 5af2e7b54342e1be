"""Encrypted IVF-PQ over the larger database on the GPU: 1,000,000 x 128
(1,024-component mixture), n_list 1024, PQ 16 x 256, nprobe 16; CKKS N = 2^15,
12 x 50-bit Q + 4 x 60-bit P, dnum 3, scale 2^40.

* Decrypted coarse distances (all 1,024, compacted the packed way from 8
  coarse ciphertexts) match the plaintext IVF-PQ ADC within 2e-2, and
  candidate distances (about 15,600 per query, in one or two result
  ciphertexts) within 0.25, absolute. The bound comes from the key switch's
  approximate ModDown (hls/src/key_switch.cpp:62-163, kept bit-exact). It
  floors, and its P -> Q base conversion has no overflow correction, so
  every key switch leaves a rounding error of mean about -(K + 1) / 2 in
  each coefficient of both output polynomials. A constant polynomial c
  decodes to c * 2 / (1 - zeta_k) in the slot of root zeta_k, which is up to
  2N / pi for the slots whose roots lie nearest +-1. At N = 2^15, K = 4 and
  scale 2^30 that is up to 4e-5 per key switch. A result ciphertext sums
  about 121 candidate batches of about 15 key switches, roughly 1,800 in
  all, so the biased slots reach about 0.07-0.11 (measured 0.11 at the slot
  of zeta^-3). All other slots stay near 1e-3. The coarse result sums 8
  coarse ciphertexts of 8 key switches, 64 in all, so it stays within 1e-2.
  The measured error is printed.
* Probed lists and top-k ids are the plaintext search's. The exception is a
  near-tie: two plaintext distances closer than twice the measured CKKS error
  at the rank boundary. It is reported, not hidden.
* The batched server (64 ciphertexts per launch) and the plain path (one per
  launch) give bit-identical result ciphertexts.
"""
import numpy as np
import pytest

from anns_fhe_b200.workloads import LARGE, Workload

pytestmark = pytest.mark.gpu
TOL_COARSE = 2e-2
TOL = 0.25


@pytest.fixture(scope="module")
def big():
    # ready for the serving trace's mixed traffic: query levels 6-12, up to 32 probes
    wl = Workload(LARGE, max_queries=4, lanes=64, levels=list(range(6, 13)), max_nprobe=32)
    yield wl
    wl.close()


def _same_up_to_ties(got, want_order, dist, margin):
    """got equals the first len(got) ids of want_order, except where the
    plaintext distances at the boundary are within `margin` of each other."""
    k = len(got)
    if list(got) == list(want_order[:k]):
        return True, []
    boundary = dist[k - 1]
    ties = [i for i in range(len(dist)) if abs(dist[i] - boundary) <= margin]
    ok = set(got) - set(want_order[:k]) <= set(want_order[i] for i in ties)
    return ok, ties


@pytest.mark.parametrize("mixed", [False, True], ids=["top_level", "mixed_levels_and_probes"])
def test_large_end_to_end_matches_plaintext(big, mixed):
    """mixed: the serving trace's shapes, queries at levels 6, 9, 12 with 4,
    32 and 16 probes in one batch."""
    Q = big.queries(3, seed=8 + mixed)
    levels, nprobes = ([6, 9, 12], [4, 32, 16]) if mixed else (None, None)
    res = big.run(Q, levels=levels, nprobes=nprobes)
    errs = []
    for i, (q, r) in enumerate(zip(Q, res)):
        npb = nprobes[i] if mixed else big.spec.nprobe
        coarse, probes, cand, dist, top = big.plaintext(q, npb)
        ec = float(np.max(np.abs(r["coarse"] - coarse)))
        assert ec < TOL_COARSE, f"coarse error {ec}"
        assert len(r["coarse"]) == 1024
        order = np.argsort(coarse, kind="stable")
        ok, ties = _same_up_to_ties(r["probes"], order, np.sort(coarse), 2 * ec)
        assert ok, f"probes differ beyond near-ties: {r['probes']} vs {list(order[:npb])}"
        if ties:
            print(f"near-tie at the probe boundary: lists {[int(order[i]) for i in ties]}")
        if list(r["probes"]) != list(probes):
            continue                         # a near-tie changed the probed lists
        assert r["vids"] == list(cand)
        ed = float(np.max(np.abs(r["dists"] - dist)))
        assert ed < TOL, f"candidate error {ed}"
        errs.append(max(ec, ed))
        dorder = np.argsort(dist, kind="stable")
        ok, ties = _same_up_to_ties(r["topk"], np.asarray(cand)[dorder], dist[dorder], 2 * ed)
        assert ok, "top-k differs beyond near-ties"
        if ties:
            print(f"near-tie at the top-k boundary ({len(ties)} candidates)")
    assert errs, "every query hit a near-tie at the probe boundary"
    print(f"max CKKS error {max(errs):.2e} over {len(errs)} queries, "
          f"{len(res[0]['vids'])} candidates in query 0")


def test_large_batched_equals_plain(big):
    Q = big.queries(1, seed=9)
    recs = big.records[:1]
    big.run(Q, recs)
    batched = [[big.iqm.read_ct(ct) for ct in [r.compact] + r.results] for r in recs]
    lanes = big.iqm.lanes
    try:
        big.iqm.lanes = 1
        big.iqm.stage1_coarse(recs)
        big.iqm.stage3_fine(recs)
    finally:
        big.iqm.lanes = lanes
    for r, b in zip(recs, batched):
        for ct, (c0, c1) in zip([r.compact] + r.results, b):
            g0, g1 = big.iqm.read_ct(ct)
            assert np.array_equal(g0, c0) and np.array_equal(g1, c1)
