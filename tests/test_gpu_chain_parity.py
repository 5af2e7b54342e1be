"""The GPU query chain equals the reference's chain, residue for residue.

The server chain (anns_fhe_b200/query.py) batches ciphertexts across queries,
lists and candidate batches. It runs the stage-1b rotations step by step across
all lists, and sums terms pairwise. The reference runs it one ciphertext at a
time: interactive_query_manager.cpp:85-303, with the semantics of
generate_interactive_test_vectors.cpp:383-541. For each list, mask, rescale,
eval_rotate by i (D - 1) and eval_add into a running sum; for each candidate
batch, the same with -offset.

For indexes whose centroids span several ciphertexts the chain compacts
them the "packed" way: mask every centroid slot, rotate coarse ciphertext k
right by k with one key, and sum. It places candidate batch t at slot t * B
with one key switch, continuing in a second result ciphertext past the slot
count. That chain is replayed the same way, one ciphertext at a time, on the
oracle.

This test replays that sequential chain on the CPU oracle (the C restatement
of the reference's HLS kernels) with the very keys, plaintexts and
encrypted queries the GPU used, read back from the device. It then requires
the compacted coarse ciphertext and the candidate-distance ciphertext of
every query to be identical word for word. A small ring (N = 2^10, 8 lists of
8 dimensions) keeps the oracle fast. The bench's configuration (N = 2^13) runs
for one query, through the one-kernel key switch.
"""
import numpy as np
import pytest

from anns_fhe_b200.workloads import SMALL, Workload, WorkloadSpec
from oracle.composite import OracleCKKS
from oracle.oracle import tables_py as T

pytestmark = pytest.mark.gpu

TINY = WorkloadSpec("ivfpq_512x8_nlist8_N1024_L3", n_vectors=512, d=8, components=8, sigma=0.1, n_list=8, M=2, K=16,
                    nprobe=2, top_k=4, log_n=10, num_q=3, q_bits=50, num_p=1, p_bits=60, alpha=1, log_scale=40)


def reference_chain(wl, ora, ct, ct_dim, probes, level=None):
    """One query through the reference's sequential chain on the oracle, at
    the query's level (default: the top level)."""
    iqm, p = wl.iqm, wl.params
    n, L = p.n, level or p.L
    D, B, nl = iqm.sh.D, iqm.sh.B, iqm.sh.n_list
    kw = p.key_words()
    half = kw // 2

    def key(off):
        k = wl.ctx.read_key(off, kw)
        return k[:half], k[half:]
    relin = key(0)
    where = {s: kw * (1 + i) for i, s in enumerate(sorted(wl.steps))}

    class Keys(dict):
        """Rotation keys read back from the device when first used (a
        configuration may hold more than a hundred keys of 25 MB)."""
        def __missing__(self, step):
            self[step] = key(where[step])
            return self[step]
    rot = Keys()

    def pt(off, limbs):
        return wl.ctx.read_poly(off, limbs * n)

    def tree(c, stride):
        s = stride
        while s < D * stride:
            c = ora.eval_add(c, ora.eval_rotate(c, s, rot, L - 1), L - 1)
            s <<= 1
        return c
    # stage 1 / 1b
    comp = None
    if iqm.sh.compaction == "reference":
        diff = ora.eval_sub_plain(ct, pt(iqm.pt_centroids, L), L)
        sq = tree(ora.eval_mult_relin_rescale(diff, diff, relin, L), 1)
        for i in range(nl):
            sel = ora.eval_mult_plain_rescale(sq, pt(iqm._onehot[L][i], L - 1), L - 1)
            if i:
                sel = ora.eval_rotate(sel, i * (D - 1), rot, L - 2)
            comp = sel if comp is None else ora.eval_add(comp, sel, L - 2)
    else:
        # packed: coarse ciphertext k masked at every centroid slot, rotated right by k
        for k, pk in enumerate(iqm.pt_centroid_cts):
            diff = ora.eval_sub_plain(ct, pt(pk, L), L)
            sq = tree(ora.eval_mult_relin_rescale(diff, diff, relin, L), 1)
            sel = ora.eval_mult_plain_rescale(sq, pt(iqm._stride[L], L - 1), L - 1)
            if k:
                sel = ora.eval_rotate_single_step(sel, -k, rot, L - 2)     # one key for step -k
            comp = sel if comp is None else ora.eval_add(comp, sel, L - 2)
    # stage 3: candidate p lands in result p // slots at slot p mod slots
    S = iqm.sh.slots
    packed = iqm.sh.compaction == "packed"
    if packed:      # expanded distances: the query's ||q||^2 once
        qnorm = ora.eval_mult_relin_rescale(ct_dim, ct_dim, relin, L)
    off, acc, t = 0, {}, 0
    for c in probes:
        for bi, (pt_off, cnt, _) in enumerate(iqm.batches[c]):
            if packed:                  # batch t starts at t * B, placed by its mask
                off = t * B
            elif off % S + cnt > S:     # a batch that does not fit starts the next result
                off = (off // S + 1) * S
            if packed:
                # ||q||^2 - 2 <q, x_j> in every row after the tree sum, then + ||x_j||^2
                cx = ora.eval_mult_plain_rescale(ct_dim, pt(pt_off, L), L)
                y = tuple(ora.poly("sub", ora.poly("sub", qn, ci, L - 1), ci, L - 1) for qn, ci in zip(qnorm, cx))
                sq = tree(y, B)
                nrm = pt(iqm._norms[L][iqm._first_batch[c] + bi], L - 1)
                sq = (ora.poly("add", sq[0], nrm, L - 1), sq[1])
            else:
                diff = ora.eval_sub_plain(ct_dim, pt(pt_off, L), L)
                sq = tree(ora.eval_mult_relin_rescale(diff, diff, relin, L), B)
            mask = pt(iqm._prefix_lv[(cnt, L)], L - 1)
            if packed:
                # the tree sum leaves the sums in every row; the prefix mask
                # moved to row t (a plaintext automorphism) selects them there
                mask = ora.automorphism(mask, T.galois(p.log_n, -(off % S)), L - 1)
                sel = ora.eval_mult_plain_rescale(sq, mask, L - 1)
            else:
                sel = ora.eval_mult_plain_rescale(sq, mask, L - 1)
                if off % S:
                    sel = ora.eval_rotate(sel, -(off % S), rot, L - 2)
            r = off // S
            acc[r] = sel if r not in acc else ora.eval_add(acc[r], sel, L - 2)
            off += cnt
            t += 1
    return comp, [acc[r] for r in sorted(acc)]


def run_and_compare(spec, nq, lanes, orc, levels=None):
    """levels: per-query encryption levels (mixed in the same batches)."""
    wl = Workload(spec, max_queries=nq, lanes=lanes, levels=sorted(set(levels)) if levels else None)
    try:
        p = wl.params
        n = p.n
        recs = wl.records[:nq]
        wl.encrypt_queries(wl.queries(nq, seed=21), recs, levels)
        ins = [((wl.ctx.read_poly(r.ct_query[0], r.level * n), wl.ctx.read_poly(r.ct_query[1], r.level * n)),
                (wl.ctx.read_poly(r.ct_dim[0], r.level * n), wl.ctx.read_poly(r.ct_dim[1], r.level * n)))
               for r in recs]
        wl.iqm.stage1_coarse(recs)
        wl.select(recs)
        wl.iqm.stage3_fine(recs)
        ora = OracleCKKS(p.log_n, p.q, p.p, p.alpha, orc)
        results_used = set()
        for r, (ct, ct_dim) in zip(recs, ins):
            lv = wl.iqm.level_of(r)          # the level the server evaluates this query at
            comp, accs = reference_chain(wl, ora, ct, ct_dim, r.probes, lv)
            got_c = [a[:(lv - 2) * n] for a in wl.iqm.read_ct(r.compact)]
            assert np.array_equal(got_c[0], comp[0]) and np.array_equal(got_c[1], comp[1]), "stage 1b differs"
            results_used.add(len(accs))
            for k, acc in enumerate(accs):
                got_d = [a[:(lv - 2) * n] for a in wl.iqm.read_ct(r.results[k])]
                assert np.array_equal(got_d[0], acc[0]) and np.array_equal(got_d[1], acc[1]), \
                    f"stage 3 result {k} differs"
        return wl.iqm, results_used
    finally:
        wl.close()


# the packed compaction and results spanning two ciphertexts: 128 lists of 8
# dimensions over 2 coarse ciphertexts (64 centroids each at N = 2^10), 40
# probes of about 16 vectors (> 512 candidates per query)
TINY_PACKED = WorkloadSpec("ivfpq_2048x8_nlist128_N1024_L4_packed", n_vectors=2048, d=8, components=128,
                           sigma=0.1, n_list=128, M=2, K=16, nprobe=40, top_k=4, log_n=10, num_q=4, q_bits=50,
                           num_p=2, p_bits=60, alpha=2, log_scale=40, compaction="packed", init="farthest")


def test_chain_matches_reference_small_ring(orc):
    run_and_compare(TINY, nq=3, lanes=4, orc=orc)


def test_packed_chain_matches_oracle_replay(orc):
    iqm, used = run_and_compare(TINY_PACKED, nq=2, lanes=16, orc=orc)
    assert iqm.sh.n_coarse == 2 and iqm.n_res >= 2
    assert max(used) >= 2, "no query spilled into a second result ciphertext"


def test_mixed_levels_match_oracle_replay(orc):
    """Queries at levels 4 and 3 in the same batches: each one's chain runs
    at its own level (masks per level) and equals the oracle replay there."""
    iqm, _ = run_and_compare(TINY_PACKED, nq=3, lanes=16, orc=orc, levels=[4, 3, 3])
    assert iqm.levels == [3, 4]


def test_eval_level_matches_oracle_replay(orc):
    """Queries encrypted at 5 and 4 limbs, evaluated at 3: the server drops
    the limbs the depth-2 chain does not need before its first operator; the
    chain at 3 limbs equals the oracle replay on the queries' first 3 limbs."""
    import dataclasses
    spec = dataclasses.replace(TINY_PACKED, name="ivfpq_2048x8_nlist128_N1024_L5_eval3", num_q=5, eval_level=3)
    iqm, _ = run_and_compare(spec, nq=2, lanes=16, orc=orc, levels=[5, 4])
    assert iqm.levels == [3]


def test_chain_matches_reference_bench_configuration(orc):
    run_and_compare(SMALL, nq=1, lanes=8, orc=orc)


# The large IVF-PQ configuration's CKKS parameters and query shape (N = 2^15,
# 12 x 50-bit Q + 4 x 60-bit P, alpha 4, d = 128, so B = 128 and 128
# centroids per coarse ciphertext; packed compaction; placement by one key
# per step) over a database small enough for the oracle to replay one query:
# 256 lists in 2 coarse ciphertexts, 2 probed lists.
CFG4_PARAMS = WorkloadSpec("ivfpq_2048x128_nlist256_N32768_L12", n_vectors=2048, d=128, components=256, sigma=0.15,
                           n_list=256, M=16, K=256, nprobe=2, top_k=8, log_n=15, num_q=12, q_bits=50, num_p=4,
                           p_bits=60, alpha=4, log_scale=40, compaction="packed", init="farthest")


def test_large_configuration_parameters_at_eval_level(orc):
    """One query at 12 limbs, evaluated at 3 (what the large configuration's
    bench runs): every key switch on 3 + 4 limbs, one digit."""
    import dataclasses
    spec = dataclasses.replace(CFG4_PARAMS, name=CFG4_PARAMS.name + "_eval3", eval_level=3)
    iqm, _ = run_and_compare(spec, nq=1, lanes=4, orc=orc)
    assert iqm.levels == [3] and iqm.sh.n_coarse == 2


def test_large_configuration_parameters_at_full_level(orc):
    """One query evaluated at its own 12 limbs: key switches at 12 and 11
    limbs (3 digits of 4 limbs, the last one 4 or 3), rescales to 10."""
    iqm, _ = run_and_compare(CFG4_PARAMS, nq=1, lanes=4, orc=orc)
    assert iqm.levels == [12] and iqm.sh.n_coarse == 2
