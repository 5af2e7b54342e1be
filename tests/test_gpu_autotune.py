"""The autotuner on the GPU: it measures every (path, tile) candidate and
returns one per level. Whatever it picks, the chain's residues do not
change. The query chain run with forced extreme choices (multi-kernel key
switch, two ciphertexts per launch) gives the same result ciphertexts as the
defaults (one-kernel key switch, all lanes per launch)."""
import numpy as np
import pytest

from anns_fhe_b200 import autotune as A
from anns_fhe_b200.driver import CkksParams
from anns_fhe_b200.workloads import Workload
from tests.test_gpu_chain_parity import TINY

pytestmark = pytest.mark.gpu


def test_tune_returns_a_choice_per_level():
    prm = CkksParams.generate(10, 3, 50, 1, 60, 1)
    ch = A.tune(prm, [3, 2, 1], lanes=16)
    assert sorted(ch) == [1, 2, 3]
    for c in ch.values():
        assert c.chunk in A.chunk_candidates(16, A.sm_count()) and c.us_per_ct > 0


def test_tuned_chain_is_bit_identical():
    wl = Workload(TINY, max_queries=3, lanes=8)
    try:
        Q = wl.queries(3, seed=4)
        recs = wl.records[:3]
        wl.run(Q, recs)
        base = [[wl.iqm.read_ct(ct) for ct in [r.compact] + r.results[:1]] for r in recs]
        wl.iqm.use_tuning({lv: A.KsChoice(False, 2, 0.0) for lv in (1, 2, 3)})
        wl.iqm.stage1_coarse(recs)
        wl.iqm.stage3_fine(recs)
        for r, b in zip(recs, base):
            for ct, (c0, c1) in zip([r.compact] + r.results[:1], b):
                g0, g1 = wl.iqm.read_ct(ct)
                assert np.array_equal(g0, c0) and np.array_equal(g1, c1)
    finally:
        wl.close()
