"""The diagonal chain (baby-step giant-step inner products) on the GPU.

* residues: every compacted coarse ciphertext and every result ciphertext
  equals a one-ciphertext-at-a-time replay on the CPU oracle (the C
  restatement of the reference's HLS kernels) of the same chain: the baby
  steps as single-step rotations (eval_rotate_single_step), each inner product as
  poly_mul_ntt products of the plaintexts (moved by FHEHostDriver's
  automorphism) summed with eval_add, then rescale, the giant-step rotation
  and eval_add, + the client's ||q||^2 ciphertext + the placed norms; the
  keys, plaintexts and encrypted queries are read back from the device;
* decrypted coarse and candidate distances match the plaintext IVF-PQ
  search within the CKKS tolerance, probes and top-k ids are identical;
* the batched server and the one-lane server give identical ciphertexts.
"""
import dataclasses

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.workloads import SMALL, Workload, WorkloadSpec
from oracle.composite import OracleCKKS
from oracle.oracle import tables_py as T

pytestmark = pytest.mark.gpu
TOL = 1e-2

# 128 lists of 8 dimensions at N = 2^10 (512 slots), 40 probes: units padded
# to multiples of 8 slots spill into a second and third result ciphertext
TINY_DIAG = WorkloadSpec("ivfpq_2048x8_nlist128_N1024_L4_diag", n_vectors=2048, d=8, components=128, sigma=0.1,
                         n_list=128, M=2, K=16, nprobe=40, top_k=4, log_n=10, num_q=4, q_bits=50, num_p=2,
                         p_bits=60, alpha=2, log_scale=40, compaction="diagonal", init="farthest")
# two lists of about 1,000 vectors: each list is two or three units of up to
# 512 candidates, each unit a result ciphertext of its own
TINY_UNITS = dataclasses.replace(TINY_DIAG, name="ivfpq_2048x8_nlist2_N1024_L4_diag", n_list=2, components=2,
                                 nprobe=2)


def diagonal_replay(wl, ora, ct, nrm, probes, lv):
    """One query through the diagonal chain, one ciphertext at a time, on
    the oracle, at `lv` limbs (nrm: the client's ||q||^2 ciphertext at lv - 1
    limbs): (compact, [result ciphertexts used])."""
    iqm, p = wl.iqm, wl.params
    n, sh = p.n, iqm.sh
    D, S, n1, n2 = sh.D, sh.slots, sh.n1, sh.n2
    kw = p.key_words()
    half = kw // 2

    def key(off):
        k = wl.ctx.read_key(off, kw)
        return k[:half], k[half:]
    where = {s: kw * (1 + i) for i, s in enumerate(sorted(wl.steps))}

    class Keys(dict):
        def __missing__(self, step):
            self[step] = key(where[step])
            return self[step]
    rot = Keys()
    dg = iqm._diag[lv]

    def pt(off, limbs):
        return wl.ctx.read_poly(off, limbs * n)

    maps = {}

    def auto(x, gal, limbs):
        """FHEHostDriver::automorphism on each limb (maps cached by element)."""
        if gal not in maps:
            m = T.auto_map(p.log_n, gal).astype(np.uint64)
            maps[gal] = m[0::2] | (m[1::2] << np.uint64(32))
        return np.concatenate([ora.orc.automorphism(ora.limb(x, i), maps[gal]) for i in range(limbs)])

    def mac(terms, limbs):
        acc = None
        for src, off, gal in terms:
            x = pt(off, limbs)
            if gal != 1:
                x = auto(x, gal, limbs)
            m = (ora.poly("mul", src[0], x, limbs), ora.poly("mul", src[1], x, limbs))
            acc = m if acc is None else ora.eval_add(acc, m, limbs)
        if acc is None:
            z = np.zeros(limbs * n, dtype=np.uint64)
            acc = (z, z.copy())
        return acc

    def giant(per_g):
        total = None
        for g, terms in enumerate(per_g):
            c = mac(terms, lv)
            c = (ora.rescale_poly(c[0], lv), ora.rescale_poly(c[1], lv))
            if g:
                c = ora.eval_rotate_single_step(c, n1 * g, rot, lv - 1)
            total = c if total is None else ora.eval_add(total, c, lv - 1)
        return total

    babies = [ct] + [ora.eval_rotate_single_step(ct, b, rot, lv) for b in range(1, n1)]
    comp = giant([[(babies[b], dg["cent"][g * n1 + b], 1) for b in range(n1)] for g in range(n2)])
    comp = ora.eval_add(comp, nrm, lv - 1)
    comp = (ora.poly("add", comp[0], pt(dg["cnorm"], lv - 1), lv - 1), comp[1])
    layout = iqm.unit_offsets(probes)
    used = layout[-1][1] // S + 1 if layout else 1
    results = []
    for r in range(used):
        us = [(u, T.galois(p.log_n, -(off % S))) for u, off in layout if off // S == r]
        res = giant([[(babies[b], dg["pts"][u * D + g * n1 + b], gal) for u, gal in us for b in range(n1)]
                     for g in range(n2)])
        res = ora.eval_add(res, nrm, lv - 1)
        c0 = res[0]
        for u, gal in us:
            c0 = ora.poly("add", c0, auto(pt(dg["norms"][u], lv - 1), gal, lv - 1), lv - 1)
        results.append((c0, res[1]))
    return comp, results


def replay_and_compare(spec, nq, lanes, orc, levels=None):
    wl = Workload(spec, max_queries=nq, lanes=lanes, levels=sorted(set(levels)) if levels else None)
    try:
        p, n = wl.params, wl.params.n
        recs = wl.records[:nq]
        wl.encrypt_queries(wl.queries(nq, seed=21), recs, levels)
        ins = [(wl.ctx.read_poly(r.ct_query[0], r.level * n), wl.ctx.read_poly(r.ct_query[1], r.level * n))
               for r in recs]
        lvs = [wl.iqm.level_of(r) for r in recs]
        nrms = [(wl.ctx.read_poly(r.ct_dim[0], (lv - 1) * n), wl.ctx.read_poly(r.ct_dim[1], (lv - 1) * n))
                for r, lv in zip(recs, lvs)]
        wl.iqm.stage1_coarse(recs)
        wl.select(recs)
        wl.iqm.stage3_fine(recs)
        ora = OracleCKKS(p.log_n, p.q, p.p, p.alpha, orc)
        used = set()
        for r, ct, nrm in zip(recs, ins, nrms):
            lv = wl.iqm.level_of(r)
            comp, results = diagonal_replay(wl, ora, (ct[0][:lv * n], ct[1][:lv * n]), nrm, r.probes, lv)
            w = (lv - 1) * n
            got = [a[:w] for a in wl.iqm.read_ct(r.compact)]
            assert np.array_equal(got[0], comp[0]) and np.array_equal(got[1], comp[1]), "coarse ciphertext differs"
            used.add(len(results))
            for k, res in enumerate(results):
                got = [a[:w] for a in wl.iqm.read_ct(r.results[k])]
                assert np.array_equal(got[0], res[0]) and np.array_equal(got[1], res[1]), f"result {k} differs"
        return wl.iqm, used
    finally:
        wl.close()


def test_diagonal_chain_matches_oracle_replay(orc):
    iqm, used = replay_and_compare(TINY_DIAG, nq=2, lanes=16, orc=orc)
    assert iqm.sh.n1 == 4 and iqm.sh.n2 == 2 and iqm.n_res >= 2
    assert max(used) >= 2, "no query spilled into a second result ciphertext"


def test_diagonal_units_and_mixed_levels_match_oracle_replay(orc):
    """Lists longer than the slots (units of 512 candidates, one result
    each); queries at 4 and 3 limbs in the same batches."""
    iqm, used = replay_and_compare(TINY_UNITS, nq=3, lanes=8, orc=orc, levels=[4, 3, 3])
    assert iqm.levels == [3, 4] and max(len(u) for u in iqm.list_units) >= 2 and max(used) >= 3


def test_diagonal_eval_level_two_matches_oracle_replay(orc):
    """Depth 1: queries at 4 limbs evaluated at 2, results at 1 limb."""
    spec = dataclasses.replace(TINY_DIAG, name=TINY_DIAG.name + "_eval2", eval_level=2)
    iqm, _ = replay_and_compare(spec, nq=2, lanes=16, orc=orc, levels=[4, 3])
    assert iqm.levels == [2] and iqm.lvl_out == 1


CFG4_DIAG = WorkloadSpec("ivfpq_2048x128_nlist32_N32768_L12_diag_eval2", n_vectors=2048, d=128, components=32,
                         sigma=0.15, n_list=32, M=16, K=256, nprobe=2, top_k=8, log_n=15, num_q=12, q_bits=50,
                         num_p=4, p_bits=60, alpha=4, log_scale=40, compaction="diagonal", init="farthest",
                         eval_level=2)


def test_diagonal_large_parameters_match_oracle_replay(orc):
    """The large configuration's CKKS parameters and d = 128 (16 baby and 8
    giant steps) at evaluation level 2, one query replayed."""
    iqm, _ = replay_and_compare(CFG4_DIAG, nq=1, lanes=4, orc=orc)
    assert iqm.sh.n1 == 16 and iqm.sh.n2 == 8 and iqm.levels == [2]


@pytest.fixture(scope="module")
def small_diag():
    w = Workload(dataclasses.replace(SMALL, name=SMALL.name + "_diag", compaction="diagonal", eval_level=2),
                 max_queries=8, lanes=16)
    yield w
    w.close()


def test_diagonal_end_to_end_matches_plaintext(small_diag):
    wl = small_diag
    Q = wl.queries(6, seed=3)
    for q, r in zip(Q, wl.run(Q)):
        coarse, probes, cand, dist, top = wl.plaintext(q)
        assert np.max(np.abs(r["coarse"] - coarse)) < TOL
        assert list(r["probes"]) == list(probes)
        assert r["vids"] == list(cand)
        assert np.max(np.abs(r["dists"] - dist)) < TOL
        assert r["topk"] == list(top)


def test_diagonal_batched_equals_plain(small_diag):
    wl = small_diag
    Q = wl.queries(3, seed=5)
    recs = wl.records[:3]
    wl.run(Q, recs)
    batched = [[wl.iqm.read_ct(c) for c in [r.compact] + r.results] for r in recs]
    chunk = wl.ctx.get_option(L.OPT_CHUNK)      # ciphertexts per launch
    try:
        wl.ctx.set_option(L.OPT_CHUNK, 1)
        wl.iqm.stage1_coarse(recs)
        wl.iqm.stage3_fine(recs)
    finally:
        wl.ctx.set_option(L.OPT_CHUNK, chunk)
    for r, cts in zip(recs, batched):
        for c, (a, b) in zip([r.compact] + r.results, cts):
            a2, b2 = wl.iqm.read_ct(c)
            assert np.array_equal(a, a2) and np.array_equal(b, b2)
