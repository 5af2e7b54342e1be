"""The two key-switch implementations agree bit for bit: the one-kernel key
switch (N <= 2^13, the default there) and the multi-launch pipeline
(AFHE_KS_FUSED=0 at context creation), on every operator that key-switches,
against the oracle; and rotation batches whose entries alias each other still
produce the reference's results."""
import os

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, FHEHostDriver
from oracle.composite import OracleCKKS
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu

# name: log_n, nq, q_bits, np, p_bits, alpha
SHAPES = {
    "n8192_a1": (13, 3, 50, 1, 60, 1),
    "n4096_a2": (12, 5, 45, 2, 50, 2),
    "n2048_a3": (11, 7, 40, 3, 45, 3),
    "n1024_a1k2": (10, 4, 40, 2, 45, 1),
    # the large IVF-PQ configuration's parameter set (N = 2^15, 12 + 4 limbs,
    # alpha 4), checked at levels 12, 6 and 3 only
    "cfg4_n32768": (15, 12, 50, 4, 60, 4),
}
STEPS = (1, 2, -1, -2, 4)
LEVELS = {"cfg4_n32768": (12, 6, 3)}


def levels_of(pr):
    return LEVELS.get(pr.name, tuple(range(pr.L, 0, -1)))


def make_ctx(prm, fused, poly_words, key_words):
    old = os.environ.get("AFHE_KS_FUSED")
    os.environ["AFHE_KS_FUSED"] = "1" if fused else "0"
    try:
        return FheContext(prm, poly_words=poly_words, key_words=key_words)
    finally:
        if old is None:
            del os.environ["AFHE_KS_FUSED"]
        else:
            os.environ["AFHE_KS_FUSED"] = old


class Pair:
    """The same parameters and keys in a fused and a multi-launch context."""

    def __init__(self, shape, orc):
        log_n, nq, qb, np_, pb, alpha = SHAPES[shape]
        q, p = primes_for(log_n, nq, qb, np_, pb)
        self.prm = CkksParams(log_n, q, p, alpha)
        self.n, self.L, self.K = 1 << log_n, nq, np_
        self.ora = OracleCKKS(log_n, q, p, alpha, orc)
        self.PW = (nq + np_) * self.n
        kw = self.prm.key_words()
        rng = np.random.default_rng(77)
        allp = q + p
        self.keys = []
        for _ in range(1 + len(STEPS)):
            a = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(self.prm.dnum)])
            b = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(self.prm.dnum)])
            self.keys.append((a, b))
        self.rot = {s: self.keys[i + 1] for i, s in enumerate(STEPS)}
        self.ctxs = []
        for fused in (True, False):
            ctx = make_ctx(self.prm, fused, 16 * self.PW, (2 + len(STEPS)) * kw)
            drv = FHEHostDriver(ctx)
            for i, (a, b) in enumerate(self.keys):
                ctx.write_key(i * kw, np.concatenate([a, b]))
            drv.set_relin_key(0)
            for i, s in enumerate(STEPS):
                drv.add_rotation_key(s, (i + 1) * kw)
            self.ctxs.append((ctx, drv))
        self.rng = rng

    def ct(self, level):
        qs = self.prm.q[:level]
        return uniform_residues(self.rng, qs, self.n), uniform_residues(self.rng, qs, self.n)

    def slot(self, i):
        return i * self.PW


@pytest.fixture(scope="module", params=list(SHAPES))
def pr(request, orc):
    p = Pair(request.param, orc)
    p.name = request.param
    yield p
    for ctx, _ in p.ctxs:
        ctx.close()


def both(pr, fn):
    """Run fn(ctx, drv) on both contexts; return both results."""
    return [fn(ctx, drv) for ctx, drv in pr.ctxs]


def test_key_switch_every_level(pr):
    a, b = pr.keys[0]
    for lvl in levels_of(pr):
        x = pr.ct(lvl)[0]
        e0, e1 = pr.ora.key_switch(x, a, b, lvl)

        def run(ctx, drv):
            ctx.write_poly(pr.slot(0), x)
            drv.key_switch(pr.slot(0), 0, pr.slot(1), pr.slot(2), lvl)
            return ctx.read_poly(pr.slot(1), lvl * pr.n), ctx.read_poly(pr.slot(2), lvl * pr.n)
        for g0, g1 in both(pr, run):
            assert np.array_equal(g0, e0), lvl
            assert np.array_equal(g1, e1), lvl


def test_mult_relin_rescale(pr):
    for lvl in (pr.L, 2):
        A, B = pr.ct(lvl), pr.ct(lvl)
        e0, e1 = pr.ora.eval_mult_relin_rescale(A, B, pr.keys[0], lvl)

        def run(ctx, drv):
            for i, v in enumerate(A + B):
                ctx.write_poly(pr.slot(i), v)
            drv.eval_mult_relin_rescale(pr.slot(0), pr.slot(1), pr.slot(2), pr.slot(3), pr.slot(4), pr.slot(5), lvl)
            return ctx.read_poly(pr.slot(4), (lvl - 1) * pr.n), ctx.read_poly(pr.slot(5), (lvl - 1) * pr.n)
        for g0, g1 in both(pr, run):
            assert np.array_equal(g0, e0) and np.array_equal(g1, e1), lvl


@pytest.mark.parametrize("total", [1, -1, 3, 7, -3])
def test_rotate_every_level(pr, total):
    for lvl in levels_of(pr):
        A = pr.ct(lvl)
        e0, e1 = pr.ora.eval_rotate(A, total, pr.rot, lvl)

        def run(ctx, drv):
            ctx.write_poly(pr.slot(0), A[0])
            ctx.write_poly(pr.slot(1), A[1])
            drv.eval_rotate(pr.slot(0), pr.slot(1), pr.slot(2), pr.slot(3), total, lvl)
            return ctx.read_poly(pr.slot(2), lvl * pr.n), ctx.read_poly(pr.slot(3), lvl * pr.n)
        for g0, g1 in both(pr, run):
            assert np.array_equal(g0, e0) and np.array_equal(g1, e1), (lvl, total)


def refs(*cts):
    arr = (L.CtRef * len(cts))()
    for i, (a, b) in enumerate(cts):
        arr[i].c0_offset, arr[i].c1_offset = a, b
    return arr


def test_rotate_accumulate_batch(pr):
    lvl = pr.L
    cts = [pr.ct(lvl) for _ in range(3)]
    accs = [pr.ct(lvl) for _ in range(3)]
    exp = []
    for c, a in zip(cts, accs):
        r = pr.ora.eval_rotate(c, 3, pr.rot, lvl)
        exp.append(pr.ora.eval_add(r, a, lvl))

    def run(ctx, drv):
        for i, (c, a) in enumerate(zip(cts, accs)):
            for j, v in enumerate(c + a):
                ctx.write_poly(pr.slot(4 * i + j), v)
        L.check(ctx.lib.afhe_eval_rotate_accumulate_batch(
            ctx.h, refs(*[(pr.slot(4 * i), pr.slot(4 * i + 1)) for i in range(3)]),
            refs(*[(pr.slot(4 * i + 2), pr.slot(4 * i + 3)) for i in range(3)]), 3, 3, lvl), "racc")
        return [(ctx.read_poly(pr.slot(4 * i + 2), lvl * pr.n), ctx.read_poly(pr.slot(4 * i + 3), lvl * pr.n))
                for i in range(3)]
    for got in both(pr, run):
        for (g0, g1), (e0, e1) in zip(got, exp):
            assert np.array_equal(g0, e0) and np.array_equal(g1, e1)


def test_rotate_output_shifted_over_input(pr):
    """Output polynomials that overlap the input at a one-limb offset."""
    lvl = pr.L
    A = pr.ct(lvl)
    e0, e1 = pr.ora.eval_rotate_single_step(A, 1, pr.rot, lvl)
    d0, d1 = pr.slot(0) + pr.n, pr.slot(2) + pr.n

    def run(ctx, drv):
        ctx.write_poly(pr.slot(0), A[0])
        ctx.write_poly(pr.slot(2), A[1])
        drv.eval_rotate_single_step(pr.slot(0), pr.slot(2), d0, d1, 1, lvl)
        return ctx.read_poly(d0, lvl * pr.n), ctx.read_poly(d1, lvl * pr.n)
    for g0, g1 in both(pr, run):
        assert np.array_equal(g0, e0) and np.array_equal(g1, e1)


def test_rotate_batch_entries_chained(pr):
    """Entry 1 reads what entry 0 writes: every entry sees the inputs as they
    were when the call started."""
    lvl = pr.L
    X, Y = pr.ct(lvl), pr.ct(lvl)
    ex = pr.ora.eval_rotate(X, 2, pr.rot, lvl)
    ey = pr.ora.eval_rotate(Y, 2, pr.rot, lvl)

    def run(ctx, drv):
        for i, v in enumerate(X + Y):
            ctx.write_poly(pr.slot(i), v)
        L.check(ctx.lib.afhe_eval_rotate_batch(ctx.h, refs((pr.slot(0), pr.slot(1)), (pr.slot(2), pr.slot(3))),
                                               refs((pr.slot(2), pr.slot(3)), (pr.slot(4), pr.slot(5))), 2, 2, lvl),
                "rot")
        return [ctx.read_poly(pr.slot(i), lvl * pr.n) for i in (2, 3, 4, 5)]
    for g in both(pr, run):
        assert np.array_equal(g[0], ex[0]) and np.array_equal(g[1], ex[1])
        assert np.array_equal(g[2], ey[0]) and np.array_equal(g[3], ey[1])


def test_unregistered_key_and_rewritten_key(pr):
    """A key switch with a key offset that was never registered, and a
    registered key whose words are overwritten after registration: both use
    the key words as they are at call time."""
    lvl = pr.L
    x = pr.ct(lvl)[0]
    allp = pr.prm.q + pr.prm.p
    new_a = np.concatenate([uniform_residues(pr.rng, allp, pr.n) for _ in range(pr.prm.dnum)])
    new_b = np.concatenate([uniform_residues(pr.rng, allp, pr.n) for _ in range(pr.prm.dnum)])
    e0, e1 = pr.ora.key_switch(x, new_a, new_b, lvl)

    def run(ctx, drv):
        ctx.write_poly(pr.slot(0), x)
        # overwrite the registered relinearisation key (offset 0) ...
        ctx.write_key(0, np.concatenate([new_a, new_b]))
        drv.key_switch(pr.slot(0), 0, pr.slot(1), pr.slot(2), lvl)
        got = [ctx.read_poly(pr.slot(1), lvl * pr.n), ctx.read_poly(pr.slot(2), lvl * pr.n)]
        # ... and check the relinearisation itself picked the new key up
        A, B = pr.ct(lvl), pr.ct(lvl)
        for i, v in enumerate(A + B):
            ctx.write_poly(pr.slot(3 + i), v)
        drv.eval_mult_relin_rescale(pr.slot(3), pr.slot(4), pr.slot(5), pr.slot(6), pr.slot(7), pr.slot(8), lvl)
        m0, m1 = pr.ora.eval_mult_relin_rescale(A, B, (new_a, new_b), lvl)
        got.append(np.array_equal(ctx.read_poly(pr.slot(7), (lvl - 1) * pr.n), m0)
                   and np.array_equal(ctx.read_poly(pr.slot(8), (lvl - 1) * pr.n), m1))
        # restore the original relinearisation key for the other tests
        a, b = pr.keys[0]
        ctx.write_key(0, np.concatenate([a, b]))
        return got
    for g0, g1, mult_ok in both(pr, run):
        assert np.array_equal(g0, e0) and np.array_equal(g1, e1)
        assert mult_ok


def test_key_switch_with_unregistered_offset(pr):
    """Key words written past every registered key and never registered."""
    lvl = pr.L
    kw = pr.prm.key_words()
    off = (1 + len(STEPS)) * kw
    x = pr.ct(lvl)[0]
    allp = pr.prm.q + pr.prm.p
    ka = np.concatenate([uniform_residues(pr.rng, allp, pr.n) for _ in range(pr.prm.dnum)])
    kb = np.concatenate([uniform_residues(pr.rng, allp, pr.n) for _ in range(pr.prm.dnum)])
    e0, e1 = pr.ora.key_switch(x, ka, kb, lvl)

    def run(ctx, drv):
        ctx.write_key(off, np.concatenate([ka, kb]))
        ctx.write_poly(pr.slot(0), x)
        drv.key_switch(pr.slot(0), off, pr.slot(1), pr.slot(2), lvl)
        return ctx.read_poly(pr.slot(1), lvl * pr.n), ctx.read_poly(pr.slot(2), lvl * pr.n)
    for g0, g1 in both(pr, run):
        assert np.array_equal(g0, e0) and np.array_equal(g1, e1)
