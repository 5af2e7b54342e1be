"""The one-kernel key switch gives the same residues at 8 and at 16 values
per thread (AFHE_OPT_KS_EPT), at every ring degree it runs at: one CTA per
ciphertext (N = 2^10, 2^13) and clusters of 2, 4 and 8 CTAs (N = 2^14, 2^15,
2^16); and with 2^12-value slices, clusters of 4 and 8 CTAs two to an SM
(AFHE_OPT_KS_SLICE 12, N = 2^14 and 2^15), at 8 values per thread (radix-8
rounds) and 16 (256 threads, radix-16 rounds). The workload is a rotate-and-sum chain over ciphertexts at mixed
levels in one launch per step (afhe_eval_rotate_accumulate_levels_batch),
then a rescale; the 8-value kernel is checked against the oracle by
test_gpu_ks_paths.py and test_gpu_primitives_n65536.py."""
import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.primitives import KeySwitchBatch

pytestmark = pytest.mark.gpu

# log_n, num_q, num_p, alpha, level range, ciphertexts
SHAPES = {
    "n1024": (10, 4, 2, 1, (2, 4), 6),
    "n8192": (13, 3, 1, 1, (2, 3), 6),
    "n16384_cl2": (14, 6, 2, 3, (2, 6), 5),
    "n32768_cl4": (15, 12, 4, 4, (3, 12), 4),
    "n65536_cl8": (16, 8, 4, 4, (3, 8), 3),
}


@pytest.mark.parametrize("shape", list(SHAPES))
def test_values_per_thread_same_residues(shape):
    log_n, nq, np_, alpha, lv, cts = SHAPES[shape]
    ksb = KeySwitchBatch(cts=cts, log_n=log_n, num_q=nq, num_p=np_, alpha=alpha, level_range=lv, steps=[1, 2, 8],
                         lanes=cts)
    try:
        if ksb.ctx.get_option(L.OPT_KS_FUSED) != 1:
            pytest.skip("the one-kernel key switch does not run on this GPU at this ring degree")
        ksb.ctx.set_option(L.OPT_FUSED_MIN, 1)
        out = {}
        variants = [(8, 13), (16, 13)] + ([(8, 12), (16, 12)] if log_n in (14, 15) else [])
        for ept, sl in variants:
            ksb.ctx.set_option(L.OPT_KS_EPT, ept)
            ksb.ctx.set_option(L.OPT_KS_SLICE, sl)
            assert ksb.ctx.get_option(L.OPT_KS_EPT) == ept and ksb.ctx.get_option(L.OPT_KS_SLICE) == sl
            assert ksb.ctx.get_option(L.OPT_KS_CAPACITY) > 0
            ksb.reset()
            ksb.run()
            ksb.ctx.sync()
            out[(ept, sl)] = [x for z in range(cts) for o in (False, True) for x in ksb.read_ct(z, o)]
        for v in variants[1:]:
            for i, (a, b) in enumerate(zip(out[(8, 13)], out[v])):
                assert np.array_equal(a, b), f"{shape}: polynomial {i} differs under {v} (values per thread, slice)"
        assert any(np.any(a) for a in out[(8, 13)])
        ksb.ctx.set_option(L.OPT_KS_SLICE, 13)
        with pytest.raises(L.AfheError):
            ksb.ctx.set_option(L.OPT_KS_EPT, 12)
        with pytest.raises(L.AfheError):
            ksb.ctx.set_option(L.OPT_KS_SLICE, 11)
    finally:
        ksb.close()
