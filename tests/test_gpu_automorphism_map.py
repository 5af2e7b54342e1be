"""afhe_automorphism_from_map: FHEHostDriver::automorphism with the
reference's own arguments (fhe_host_driver.h:82), the permutation read from
poly_gmem in the packed layout initialize_context_from_directory writes
(fhe_host_driver.cpp:141-154: two 32-bit indices per word, low half first).
It equals afhe_automorphism with the Galois element and the oracle's
automorphism, at the top level and below it, also in place."""
import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, automorphism_map, galois_elt
from tests.helpers import uniform_residues

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [10, 13, 15])
def test_from_map_equals_galois_form(log_n, orc):
    prm = CkksParams.generate(log_n, 3, 50, 1, 60, 1)
    n = prm.n
    ctx = FheContext(prm, poly_words=16 * prm.L * n, key_words=1024)
    try:
        rng = np.random.default_rng(log_n)
        x = uniform_residues(rng, prm.q, n)
        for step in (1, -3, 17):
            g = galois_elt(log_n, step)
            m = automorphism_map(log_n, g).astype(np.uint64)
            packed = m[0::2] | (m[1::2] << np.uint64(32))
            w = prm.L * n
            src, mp, d1, d2 = 0, w, 2 * w, 3 * w
            ctx.write_poly(src, x)
            ctx.write_poly(mp, packed)
            for limbs in (prm.L, 1):
                L.check(ctx.lib.afhe_automorphism_from_map(ctx.h, src, mp, d1, limbs, g), "automorphism_from_map")
                L.check(ctx.lib.afhe_automorphism(ctx.h, src, g, d2, limbs), "automorphism")
                a, b = ctx.read_poly(d1, limbs * n), ctx.read_poly(d2, limbs * n)
                assert np.array_equal(a, b)
                want = np.concatenate([orc.automorphism(x[i * n:(i + 1) * n], packed) for i in range(limbs)])
                assert np.array_equal(a, want)
            L.check(ctx.lib.afhe_automorphism_from_map(ctx.h, src, mp, src, prm.L, g), "in place")
            want = np.concatenate([orc.automorphism(x[i * n:(i + 1) * n], packed) for i in range(prm.L)])
            assert np.array_equal(ctx.read_poly(src, w), want)
        with pytest.raises(L.AfheError):
            L.check(ctx.lib.afhe_automorphism_from_map(ctx.h, 0, 16 * prm.L * n, 0, 1, 5), "map out of range")
    finally:
        ctx.close()
