"""Batched primitives at N = 2^16 against the oracle.

* NTT microbenchmark: 64 ciphertexts x 2 polynomials x 24 limbs of 50-bit
  primes, one batched call per direction. Sampled (polynomial, limb) pairs of
  the forward transform equal the oracle's NTT (the reference's CT loop,
  hls/src/ntt.cpp:4-43) word for word. The inverse then returns every
  residue of the 1.6 GB batch exactly (INTT(NTT(x)) = x, the size-independent
  check).
* Batched key switching with rotation: N = 2^16, 24 + 8 limbs, dnum 3, 32
  ciphertexts at seeded levels in [8, 24]. One rotate-and-sum step
  (x += rot(x, s)) and one rescale, for ciphertexts at three levels, equal the
  oracle's eval_rotate_single_step + eval_add and rescale word for word. The
  whole chain (15 steps, then rescale), batched by level, equals the same
  chain run on a ciphertext alone.
"""
import numpy as np
import pytest

from anns_fhe_b200.primitives import KeySwitchBatch, NttBatch
from oracle.composite import OracleCKKS
from oracle.oracle import tables_py as T

pytestmark = pytest.mark.gpu


def test_ntt_batch_64ct_24limbs(orc):
    wl = NttBatch()
    try:
        p = wl.params
        wl.transform(inverse=False)
        wl.ctx.sync()
        rng = np.random.default_rng(0)
        picks = [(0, 0), (wl.polys - 1, wl.limbs - 1)] + [(int(rng.integers(wl.polys)), int(rng.integers(wl.limbs)))
                                                          for _ in range(4)]
        for z, i in picks:
            tw, _ = T.twiddles(p.log_n, p.q[i])
            want = orc.ntt(wl.input_limb(z, i), tw, p.q[i])
            assert np.array_equal(wl.read_limb(z, i), want), f"NTT of polynomial {z} limb {i} differs"
        wl.transform(inverse=True)
        wl.ctx.sync()
        for z in range(wl.polys):
            got = wl.ctx.read_poly(z * wl.w, wl.w)
            assert np.array_equal(got, wl.input_poly(z)), f"INTT(NTT(x)) != x for polynomial {z}"
    finally:
        wl.close()


@pytest.fixture(scope="module")
def ksb():
    wl = KeySwitchBatch()
    yield wl
    wl.close()


def _three_levels(wl):
    g = wl.groups()
    lv = sorted(g)
    return [g[lv[0]][0], g[lv[len(lv) // 2]][0], g[lv[-1]][0]]


def test_rotate_step_and_rescale_vs_oracle(ksb, orc):
    wl = ksb
    p = wl.params
    ora = OracleCKKS(p.log_n, p.q, p.p, p.alpha, orc)
    zs = _three_levels(wl)
    step = 1 << 14
    wl.reset(zs)
    wl.rotate_step(step, zs)
    wl.rescale(zs)
    keys = {step: wl.key_pair(step)}
    for z in zs:
        lv = wl.levels[z]
        c = wl.input_ct(z)
        r = ora.eval_add(c, ora.eval_rotate_single_step(c, step, keys, lv), lv)
        got = wl.read_ct(z)
        assert np.array_equal(got[0], r[0]) and np.array_equal(got[1], r[1]), f"rotation at level {lv} differs"
        out = wl.read_ct(z, out=True)
        assert np.array_equal(out[0], ora.rescale_poly(r[0], lv)), f"rescale at level {lv} differs"
        assert np.array_equal(out[1], ora.rescale_poly(r[1], lv)), f"rescale at level {lv} differs"


def test_chain_batched_equals_alone(ksb):
    """The chain over all 32 ciphertexts, every level in one launch per step,
    equals each ciphertext's chain run alone and the chain run one level
    group at a time."""
    wl = ksb
    wl.reset()
    wl.run()
    batched = {z: (wl.read_ct(z, out=True)) for z in range(wl.cts)}
    wl.reset()
    wl.run(by_level=True)
    for z in range(wl.cts):
        g = wl.read_ct(z, out=True)
        assert np.array_equal(g[0], batched[z][0]) and np.array_equal(g[1], batched[z][1]), f"level groups, {z}"
    for z in _three_levels(wl):
        wl.reset([z])
        wl.run([z])
        alone = wl.read_ct(z, out=True)
        assert np.array_equal(alone[0], batched[z][0]) and np.array_equal(alone[1], batched[z][1])
