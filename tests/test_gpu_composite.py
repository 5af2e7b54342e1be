"""The FHEHostDriver composite operators on the GPU (native per-level tables,
full-level keys) against the oracle's restatement, bit for bit; batched calls
equal one-at-a-time calls."""
import numpy as np
import pytest

from anns_fhe_b200.driver import CkksParams, FheContext, FHEHostDriver
from oracle.composite import OracleCKKS
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu

# name: log_n, nq, q_bits, np, p_bits, alpha
SHAPES = {
    "cfg1_n8192": (13, 3, 50, 1, 60, 1),
    "n16384_a2": (14, 6, 50, 2, 60, 2),
    "n65536_a3": (16, 5, 50, 3, 60, 3),
    "n1024_a4": (10, 7, 40, 2, 45, 4),
    # the large IVF-PQ configuration's exact parameter set: N = 2^15,
    # 12 x 50-bit Q + 4 x 60-bit P, alpha 4 (dnum 3)
    "cfg4_n32768": (15, 12, 50, 4, 60, 4),
}
STEPS = (1, 2, 4, -1, -2)
# levels at which every key-switching operator is checked: the top level, a
# middle one and the lowest the depth-2 query chain runs at
LEVELS = {"cfg4_n32768": (12, 6, 3)}


class Setup:
    def __init__(self, shape, orc):
        log_n, nq, qb, np_, pb, alpha = SHAPES[shape]
        q, p = primes_for(log_n, nq, qb, np_, pb)
        self.prm = CkksParams(log_n, q, p, alpha)
        self.n, self.L, self.K = 1 << log_n, nq, np_
        self.ora = OracleCKKS(log_n, q, p, alpha, orc)
        self.PW = (nq + np_) * self.n
        kw = self.prm.key_words()
        self.kw = kw
        self.ctx = FheContext(self.prm, poly_words=16 * self.PW, key_words=(2 + len(STEPS)) * kw)
        self.drv = FHEHostDriver(self.ctx)
        rng = np.random.default_rng(21)
        allp = q + p
        dig = self.prm.dnum
        self.keys = []
        for i in range(1 + len(STEPS)):
            a = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(dig)])
            b = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(dig)])
            self.ctx.write_key(i * kw, np.concatenate([a, b]))
            self.keys.append((a, b))
        self.drv.set_relin_key(0)
        self.rot = {}
        for i, s in enumerate(STEPS):
            self.drv.add_rotation_key(s, (i + 1) * kw)
            self.rot[s] = self.keys[i + 1]
        self.rng = rng

    def ct(self, level):
        qs = self.prm.q[:level]
        return uniform_residues(self.rng, qs, self.n), uniform_residues(self.rng, qs, self.n)

    def slot(self, i):
        return i * self.PW

    def put(self, i, x):
        self.ctx.write_poly(self.slot(i), x)

    def get(self, i, limbs):
        return self.ctx.read_poly(self.slot(i), limbs * self.n)


@pytest.fixture(scope="module", params=list(SHAPES))
def su(request, orc):
    s = Setup(request.param, orc)
    s.name = request.param
    yield s
    s.ctx.close()


def test_ntt_intt(su):
    x = su.ct(su.L)[0]
    su.put(0, x)
    su.drv.ntt(su.slot(0), su.slot(1), su.L)
    assert np.array_equal(su.get(1, su.L), su.ora.ntt(x, su.L))
    su.drv.intt(su.slot(1), su.slot(1), su.L)
    assert np.array_equal(su.get(1, su.L), x)


def test_rescale_every_level(su):
    for lvl in range(su.L, 1, -1):
        c0, c1 = su.ct(lvl)
        su.put(0, c0)
        su.put(1, c1)
        su.drv.rescale(su.slot(0), su.slot(1), su.slot(2), su.slot(3), lvl)
        assert np.array_equal(su.get(2, lvl - 1), su.ora.rescale_poly(c0, lvl))
        assert np.array_equal(su.get(3, lvl - 1), su.ora.rescale_poly(c1, lvl))


def test_key_switch_every_level(su):
    a, b = su.keys[0]
    for lvl in range(su.L, 0, -1):
        x = su.ct(lvl)[0]
        su.put(0, x)
        su.drv.key_switch(su.slot(0), 0, su.slot(1), su.slot(2), lvl)
        e0, e1 = su.ora.key_switch(x, a, b, lvl)
        assert np.array_equal(su.get(1, lvl), e0), lvl
        assert np.array_equal(su.get(2, lvl), e1), lvl


def test_eval_mult_relin_rescale(su):
    for lvl in (su.L, 2):
        A, B = su.ct(lvl), su.ct(lvl)
        for i, v in enumerate(A + B):
            su.put(i, v)
        su.drv.eval_mult_relin_rescale(su.slot(0), su.slot(1), su.slot(2), su.slot(3), su.slot(4), su.slot(5), lvl)
        e0, e1 = su.ora.eval_mult_relin_rescale(A, B, su.keys[0], lvl)
        assert np.array_equal(su.get(4, lvl - 1), e0)
        assert np.array_equal(su.get(5, lvl - 1), e1)
        # squaring in place (the query chain's ct_diff * ct_diff), output over input
        su.drv.eval_mult_relin_rescale(su.slot(0), su.slot(1), su.slot(0), su.slot(1), su.slot(0), su.slot(1), lvl)
        e0, e1 = su.ora.eval_mult_relin_rescale(A, A, su.keys[0], lvl)
        assert np.array_equal(su.get(0, lvl - 1), e0)
        assert np.array_equal(su.get(1, lvl - 1), e1)


def test_plain_ops(su):
    lvl = su.L
    A = su.ct(lvl)
    pt = su.ct(lvl)[0]
    su.put(0, A[0]); su.put(1, A[1]); su.put(2, pt)
    su.drv.eval_mult_plain_rescale(su.slot(0), su.slot(1), su.slot(2), su.slot(3), su.slot(4), lvl)
    e0, e1 = su.ora.eval_mult_plain_rescale(A, pt, lvl)
    assert np.array_equal(su.get(3, lvl - 1), e0) and np.array_equal(su.get(4, lvl - 1), e1)
    su.drv.eval_sub_plain(su.slot(0), su.slot(1), su.slot(2), su.slot(5), su.slot(6), lvl)
    e0, e1 = su.ora.eval_sub_plain(A, pt, lvl)
    assert np.array_equal(su.get(5, lvl), e0) and np.array_equal(su.get(6, lvl), e1)
    B = su.ct(lvl)
    su.put(7, B[0]); su.put(8, B[1])
    su.drv.eval_add(su.slot(0), su.slot(1), su.slot(7), su.slot(8), su.slot(0), su.slot(1), lvl)
    e0, e1 = su.ora.eval_add(A, B, lvl)
    assert np.array_equal(su.get(0, lvl), e0) and np.array_equal(su.get(1, lvl), e1)


def test_rotate(su):
    lvl = su.L - 1 if su.L > 2 else su.L
    A = su.ct(lvl)
    su.put(0, A[0]); su.put(1, A[1])
    for step in STEPS:
        su.drv.eval_rotate_single_step(su.slot(0), su.slot(1), su.slot(2), su.slot(3), step, lvl)
        e0, e1 = su.ora.eval_rotate_single_step(A, step, su.rot, lvl)
        assert np.array_equal(su.get(2, lvl), e0), step
        assert np.array_equal(su.get(3, lvl), e1), step
    for total in (3, 7, -3, 0):
        su.drv.eval_rotate(su.slot(0), su.slot(1), su.slot(2), su.slot(3), total, lvl)
        e0, e1 = su.ora.eval_rotate(A, total, su.rot, lvl)
        assert np.array_equal(su.get(2, lvl), e0), total
        assert np.array_equal(su.get(3, lvl), e1), total


def test_rotate_accumulate(su):
    from anns_fhe_b200 import _lib as L
    lvl = su.L
    A, B = su.ct(lvl), su.ct(lvl)
    su.put(0, A[0]); su.put(1, A[1]); su.put(2, B[0]); su.put(3, B[1])

    def refs(*cts):
        arr = (L.CtRef * len(cts))()
        for i, (a, b) in enumerate(cts):
            arr[i].c0_offset, arr[i].c1_offset = a, b
        return arr
    for total in (1, 3, -2, 0):
        su.put(2, B[0]); su.put(3, B[1])
        L.check(su.ctx.lib.afhe_eval_rotate_accumulate_batch(su.ctx.h, refs((su.slot(0), su.slot(1))),
                                                             refs((su.slot(2), su.slot(3))), 1, total, lvl), "racc")
        r0, r1 = su.ora.eval_rotate(A, total, su.rot, lvl)
        e0, e1 = su.ora.eval_add((r0, r1), B, lvl)
        assert np.array_equal(su.get(2, lvl), e0), total
        assert np.array_equal(su.get(3, lvl), e1), total
    # in place: x += rot(x, 2)
    L.check(su.ctx.lib.afhe_eval_rotate_accumulate_batch(su.ctx.h, refs((su.slot(0), su.slot(1))),
                                                         refs((su.slot(0), su.slot(1))), 1, 2, lvl), "racc")
    r0, r1 = su.ora.eval_rotate(A, 2, su.rot, lvl)
    e0, e1 = su.ora.eval_add(A, (r0, r1), lvl)
    assert np.array_equal(su.get(0, lvl), e0) and np.array_equal(su.get(1, lvl), e1)


def test_missing_rotation_key_is_an_error(su):
    from anns_fhe_b200 import AfheError
    with pytest.raises(AfheError) as ei:
        su.drv.eval_rotate(su.slot(0), su.slot(1), su.slot(2), su.slot(3), 8, su.L)
    assert ei.value.status == 3   # AFHE_E_NOKEY


def test_batched_equals_single(su):
    lvl = su.L
    cts = [su.ct(lvl) for _ in range(3)]
    for i, (c0, c1) in enumerate(cts):
        su.put(2 * i, c0)
        su.put(2 * i + 1, c1)
    ins = [(su.slot(2 * i), su.slot(2 * i + 1)) for i in range(3)]
    outs = [(su.slot(8 + 2 * i), su.slot(9 + 2 * i)) for i in range(3)]
    su.drv.eval_mult_relin_rescale_batch(ins, ins, outs, lvl)
    for i, c in enumerate(cts):
        e0, e1 = su.ora.eval_mult_relin_rescale(c, c, su.keys[0], lvl)
        assert np.array_equal(su.get(8 + 2 * i, lvl - 1), e0)
        assert np.array_equal(su.get(9 + 2 * i, lvl - 1), e1)
    su.drv.eval_rotate_batch(ins, outs, 3, lvl)
    for i, c in enumerate(cts):
        e0, e1 = su.ora.eval_rotate(c, 3, su.rot, lvl)
        assert np.array_equal(su.get(8 + 2 * i, lvl), e0)
        assert np.array_equal(su.get(9 + 2 * i, lvl), e1)


def test_key_switching_operators_at_levels(su):
    """Key switch, eval_mult_relin_rescale and eval_rotate (single steps and
    multi-step totals) at a high, a middle and a low level, each against the
    oracle (for the large configuration's parameters: levels 12, 6 and 3,
    where the last digit holds 4, 2 and 3 limbs)."""
    levels = LEVELS.get(su.name, tuple(sorted({su.L, max(2, su.L // 2), 2}, reverse=True)))
    a, b = su.keys[0]
    for lvl in levels:
        x = su.ct(lvl)[0]
        su.put(0, x)
        su.drv.key_switch(su.slot(0), 0, su.slot(1), su.slot(2), lvl)
        e0, e1 = su.ora.key_switch(x, a, b, lvl)
        assert np.array_equal(su.get(1, lvl), e0) and np.array_equal(su.get(2, lvl), e1), ("ks", lvl)
        A, B = su.ct(lvl), su.ct(lvl)
        for i, v in enumerate(A + B):
            su.put(i, v)
        su.drv.eval_mult_relin_rescale(su.slot(0), su.slot(1), su.slot(2), su.slot(3), su.slot(4), su.slot(5), lvl)
        e0, e1 = su.ora.eval_mult_relin_rescale(A, B, su.keys[0], lvl)
        assert np.array_equal(su.get(4, lvl - 1), e0) and np.array_equal(su.get(5, lvl - 1), e1), ("relin", lvl)
        for total in (1, -2, 7):
            su.drv.eval_rotate(su.slot(0), su.slot(1), su.slot(6), su.slot(7), total, lvl)
            e0, e1 = su.ora.eval_rotate(A, total, su.rot, lvl)
            assert np.array_equal(su.get(6, lvl), e0) and np.array_equal(su.get(7, lvl), e1), ("rot", lvl, total)
