"""A context loaded from a package in the reference's directory format
(formats.load_package / context_for) computes with the package's own roots
and keys. The package is built with roots other than the smallest (psi^3),
and its rotation keys are written one level down, as the reference writes
them. NTT, eval_mult_relin_rescale (full-level relinearisation key) and
eval_rotate (level L - 1 rotation keys) equal the oracle run with the
package's twiddles and keys, word for word."""
import numpy as np
import pytest

from anns_fhe_b200 import formats as F
from anns_fhe_b200.driver import FHEHostDriver
from oracle.composite import OracleCKKS
from tests.helpers import uniform_residues
from tests.test_formats import _key, _params

pytestmark = pytest.mark.gpu


def test_package_context_matches_oracle(tmp_path, orc):
    prm = _params(psi_power=3)
    rng = np.random.default_rng(5)
    relin = _key(prm, rng)
    rot = {1: _key(prm, rng), 2: _key(prm, rng)}
    d = str(tmp_path / "ctx")
    F.save_package(d, prm, relin=relin, rot=rot)
    pkg = F.load_package(d, prm.log_n, prm.alpha)
    F.check_package(pkg)
    n, Lq = prm.n, prm.L
    PW = (Lq + prm.K) * n
    ctx, offs = F.context_for(pkg, poly_words=8 * PW)
    try:
        drv = FHEHostDriver(ctx)
        ora = OracleCKKS(prm.log_n, prm.q, prm.p, prm.alpha, orc)
        ora.tw = [pkg.tw[i] for i in range(Lq + prm.K)]
        ora.itw = [pkg.itw[i] for i in range(Lq + prm.K)]
        # NTT with the package's roots
        x = uniform_residues(rng, prm.q, n)
        ctx.write_poly(0, x)
        drv.ntt(0, PW, Lq)
        assert np.array_equal(ctx.read_poly(PW, Lq * n), ora.ntt(x, Lq))
        # relinearisation with the package's key
        half = prm.key_words() // 2
        keys = {s: (F.full_level_key(prm, pkg.rot[s][2])[:half], F.full_level_key(prm, pkg.rot[s][2])[half:])
                for s in rot}
        A = (uniform_residues(rng, prm.q, n), uniform_residues(rng, prm.q, n))
        ctx.write_poly(0, A[0])
        ctx.write_poly(PW, A[1])
        drv.eval_mult_relin_rescale(0, PW, 0, PW, 2 * PW, 3 * PW, Lq)
        e0, e1 = ora.eval_mult_relin_rescale(A, A, (relin[:half], relin[half:]), Lq)
        assert np.array_equal(ctx.read_poly(2 * PW, (Lq - 1) * n), e0)
        assert np.array_equal(ctx.read_poly(3 * PW, (Lq - 1) * n), e1)
        # rotation by 3 = 2 + 1 with the level-(L - 1) rotation keys
        drv.eval_rotate(2 * PW, 3 * PW, 4 * PW, 5 * PW, 3, Lq - 1)
        r0, r1 = ora.eval_rotate((e0, e1), 3, keys, Lq - 1)
        assert np.array_equal(ctx.read_poly(4 * PW, (Lq - 1) * n), r0)
        assert np.array_equal(ctx.read_poly(5 * PW, (Lq - 1) * n), r1)
    finally:
        ctx.close()
