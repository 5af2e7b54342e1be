"""Every NTT plan gives the same residues.

The tile shapes of the batched NTT (afhe_ntt_set_plan: values per thread for
N <= 2^13; columns per CTA and chunk-tile size for N >= 2^14) are the
autotuner's to pick. For every ring degree 2^10 .. 2^16 and every plan, the
forward transform of seeded limbs equals plan 0's word for word, plan 0's
equals the oracle's NTT (the reference's loop, hls/src/ntt.cpp:4-43) on a
sampled limb, and the inverse returns the input exactly. The key switch and
rescale paths, which run their transforms through the same launcher, are
checked under the fastest non-default plan at N = 2^14 against plan 0.
"""
import numpy as np
import pytest

from anns_fhe_b200.autotune import get_ntt_plan, ntt_plan_count, ntt_plan_describe, set_ntt_plan, time_ntt_plans
from anns_fhe_b200.primitives import NttBatch
from oracle.oracle import tables_py as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16])
def test_every_plan_same_residues(log_n, orc):
    assert ntt_plan_count(log_n) == (2 if log_n <= 13 else 6)
    keep = get_ntt_plan(log_n)
    wl = NttBatch(cts=2, limbs=3, log_n=log_n)
    try:
        p = wl.params
        outs = {}
        for plan in range(ntt_plan_count(log_n)):
            set_ntt_plan(log_n, plan)
            for z in range(wl.polys):
                wl.ctx.write_poly(z * wl.w, wl.input_poly(z))
            wl.transform(inverse=False)
            wl.ctx.sync()
            outs[plan] = [wl.ctx.read_poly(z * wl.w, wl.w) for z in range(wl.polys)]
            wl.transform(inverse=True)
            wl.ctx.sync()
            for z in range(wl.polys):
                assert np.array_equal(wl.ctx.read_poly(z * wl.w, wl.w), wl.input_poly(z)), \
                    f"plan {plan} ({ntt_plan_describe(log_n, plan)}): INTT(NTT(x)) != x"
        tw, _ = T.twiddles(log_n, p.q[1])
        assert np.array_equal(outs[0][1][wl.n:2 * wl.n], orc.ntt(wl.input_limb(1, 1), tw, p.q[1]))
        for plan, o in outs.items():
            for z in range(wl.polys):
                assert np.array_equal(o[z], outs[0][z]), f"plan {plan} ({ntt_plan_describe(log_n, plan)}) differs"
        set_ntt_plan(log_n, 0)
        t = time_ntt_plans(wl.ctx, wl.polys, wl.limbs, reps=1)
        assert set(t) == set(range(ntt_plan_count(log_n))) and get_ntt_plan(log_n) == 0   # restored
    finally:
        set_ntt_plan(log_n, keep)
        wl.close()


def test_key_switch_and_rescale_under_other_plans():
    """Rotation (multi-kernel key switch) and rescale at N = 2^14, 6 + 2
    limbs, under every two-pass plan: identical to plan 0."""
    from anns_fhe_b200.primitives import KeySwitchBatch
    from anns_fhe_b200 import _lib as L
    keep = get_ntt_plan(14)
    ksb = KeySwitchBatch(cts=4, log_n=14, num_q=6, num_p=2, alpha=3, level_range=(3, 6), steps=[1, 4], lanes=4)
    try:
        ksb.ctx.set_option(L.OPT_KS_FUSED, 0)
        base = None
        for plan in range(ntt_plan_count(14)):
            set_ntt_plan(14, plan)
            ksb.reset()
            ksb.run()
            ksb.ctx.sync()
            got = [x for z in range(ksb.cts) for out in (False, True) for x in ksb.read_ct(z, out)]
            if base is None:
                base = got
            else:
                for a, b in zip(got, base):
                    assert np.array_equal(a, b), f"plan {plan} ({ntt_plan_describe(14, plan)}) differs"
    finally:
        set_ntt_plan(14, keep)
        ksb.close()
