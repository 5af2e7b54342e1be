"""The native stage driver and the Python stage driver write the same residues.

InteractiveQueryManager runs stages 1/1b and 3 in C++ by default
(afhe_ivfpq_stage1 / afhe_ivfpq_stage3, csrc/ivfpq.cu); native=False runs
them from Python over the batched C ABI. For the reference, packed and
diagonal chains, mixed query levels and a reduced evaluation level, every
word of every compacted coarse ciphertext and result ciphertext must be
equal. (test_gpu_chain_parity.py checks the native path against the oracle's
one-ciphertext-at-a-time chain; test_ivfpq_native_trace.py checks the two
drivers' operator sequences on the CPU.)"""
import dataclasses

import numpy as np
import pytest

from anns_fhe_b200.workloads import SMALL, Workload
from tests.test_gpu_chain_parity import TINY, TINY_PACKED
from tests.test_gpu_diagonal_chain import TINY_DIAG, TINY_UNITS

pytestmark = pytest.mark.gpu


def results(wl, recs):
    return [wl.iqm.read_ct(ct) for r in recs for ct in [r.compact] + r.results]


def both_ways(wl, Q, levels=None, nprobes=None):
    """The protocol once through the native driver (encryption, stage 1,
    the client's selection, stage 3), then stages 1 and 3 again from Python
    on the same encrypted queries and selections."""
    recs = wl.records[:len(Q)]
    out = {}
    wl.run(Q, recs, levels=levels, nprobes=nprobes)
    out[True] = results(wl, recs)
    z = np.zeros(wl.iqm.lvl_out * wl.params.n, dtype=np.uint64)
    for r in recs:
        for ct in [r.compact] + r.results:       # nothing left from the native run
            wl.ctx.write_poly(ct[0], z)
            wl.ctx.write_poly(ct[1], z)
    wl.iqm.native = False
    try:
        wl.iqm.stage1_coarse(recs)
        wl.iqm.stage3_fine(recs)
        out[False] = results(wl, recs)
    finally:
        wl.iqm.native = True
    return out


@pytest.mark.parametrize("spec,levels,nprobes,lanes", [
    (TINY, None, None, 16),
    (TINY, [3, 3, 3, 3], [2, 4, 1, 8], 3),
    (TINY_PACKED, [4, 3, 4], None, 16),
    (dataclasses.replace(TINY_PACKED, name="ivfpq_2048x8_nlist128_N1024_L5_eval3", num_q=5, eval_level=3),
     [5, 4, 3], [2, 3, 4], 4),
    (SMALL, None, None, 64),
    (TINY_DIAG, [4, 3, 4], [30, 40, 12], 16),
    (dataclasses.replace(TINY_UNITS, eval_level=2), [4, 3], None, 3),
    (dataclasses.replace(SMALL, name=SMALL.name + "_diag", compaction="diagonal", eval_level=2), None, None, 64),
], ids=["tiny", "tiny_lanes3_probes", "tiny_packed_levels", "tiny_packed_eval3", "small", "tiny_diagonal_levels",
        "tiny_diagonal_units_eval2", "small_diagonal"])
def test_native_equals_python(spec, levels, nprobes, lanes):
    n = len(levels) if levels else 5
    wl = Workload(spec, max_queries=n, lanes=lanes, levels=sorted(set(levels or [])) or None,
                  max_nprobe=max(nprobes) if nprobes else None)
    try:
        Q = wl.queries(n, seed=31)
        out = both_ways(wl, Q, levels, nprobes)
        rn, rp = out[True], out[False]
        assert any(np.any(c0) for c0, _ in rn), "the native run wrote nothing"
        for i, ((a0, a1), (b0, b1)) in enumerate(zip(rn, rp)):
            assert np.array_equal(a0, b0) and np.array_equal(a1, b1), f"ciphertext {i} differs"
    finally:
        wl.close()
