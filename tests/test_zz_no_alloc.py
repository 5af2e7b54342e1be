"""The allocation-free key switch, afhe_key_switch_noalloc.

It exists for callers that cannot call cudaMalloc when they serve a request:
programs whose GPU memory already belongs to their own pool allocator, and
latency-bound threads that cannot absorb the device-wide synchronisation an
allocation can cause. Its working memory is a fixed array of static device
memory inside the library, shared by all calls on a device.

Checks, through the C ABI: calls in a row each give exactly the residues of
the ordinary afhe_key_switch on the same input and key. Between checked calls
the shared array is filled with other data: a call at a lower level first,
then one at the top level (which uses scratch words the first never wrote),
and before each checked call a call from a second context with other
parameters. A parameter set too big for the fixed array is refused with
AFHE_E_BUDGET. The file is named to run last; it also passes alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, FHEHostDriver
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu


class Shape:
    """A context with a random key at key word 0 and room for 8 polynomials."""

    def __init__(self, log_n, nq, qb, np_, pb, alpha, seed):
        q, p = primes_for(log_n, nq, qb, np_, pb)
        self.q = q
        self.prm = CkksParams(log_n, q, p, alpha)
        self.n = self.prm.n
        self.slot = (nq + np_) * self.n
        self.ctx = FheContext(self.prm, poly_words=8 * self.slot, key_words=self.prm.key_words())
        self.drv = FHEHostDriver(self.ctx)
        self.rng = np.random.default_rng(seed)
        allp = q + p
        a = np.concatenate([uniform_residues(self.rng, allp, self.n) for _ in range(self.prm.dnum)])
        b = np.concatenate([uniform_residues(self.rng, allp, self.n) for _ in range(self.prm.dnum)])
        self.ctx.write_key(0, np.concatenate([a, b]))
        self.base = self.ctx.lib.afhe_poly_gmem(self.ctx.h)

    def noalloc(self, x, lvl):
        """afhe_key_switch_noalloc of x: io = [input | ks0 | ks1] at slot 4."""
        ctx, w = self.ctx, lvl * self.n
        io_off = 4 * self.slot
        ctx.write_poly(io_off, x)
        ctx.write_poly(io_off + w, np.zeros(2 * w, dtype=np.uint64))
        rc = ctx.lib.afhe_key_switch_noalloc(ctx.h, C.c_void_p(self.base + io_off * 8), 0, lvl)
        assert rc == L.OK, ctx.lib.afhe_last_error()
        ctx.sync()
        assert np.array_equal(ctx.read_poly(io_off, w), x), "input must be left unchanged"
        return ctx.read_poly(io_off + w, w), ctx.read_poly(io_off + 2 * w, w)

    def reference(self, x, lvl):
        """The ordinary entry point: input at slot 0, outputs at slots 1 and 2."""
        ctx, w = self.ctx, lvl * self.n
        ctx.write_poly(0, x)
        self.drv.key_switch(0, 0, self.slot, 2 * self.slot, lvl)
        return ctx.read_poly(self.slot, w), ctx.read_poly(2 * self.slot, w)

    def close(self):
        self.ctx.close()


def run_shape(log_n, nq, qb, np_, pb, alpha):
    main = Shape(log_n, nq, qb, np_, pb, alpha, seed=log_n * 7 + nq)
    other = Shape(12, 2, 45, 2, 55, 1, seed=99)     # fills the shared array with its own data
    try:
        for call, lvl in enumerate((max(1, nq - 1), nq)):
            y = uniform_residues(other.rng, other.q, other.n)
            other.noalloc(y, 2)
            x = uniform_residues(main.rng, main.q[:lvl], main.n)
            want0, want1 = main.reference(x, lvl)
            got0, got1 = main.noalloc(x, lvl)
            assert np.array_equal(got0, want0), f"call {call}: ks0 differs"
            assert np.array_equal(got1, want1), f"call {call}: ks1 differs"
    finally:
        other.close()
        main.close()


def test_noalloc_matches_key_switch_small():
    run_shape(13, 3, 50, 1, 60, 1)


def test_noalloc_matches_key_switch_reference_shape():
    # N = 16384 with 11 Q + 4 P limbs, alpha 4: the reference's own shape
    run_shape(14, 11, 45, 4, 60, 4)


def test_noalloc_refuses_too_large():
    q, p = primes_for(16, 4, 50, 2, 60)
    prm = CkksParams(16, q, p, 2)
    ctx = FheContext(prm, poly_words=3 * 4 * prm.n, key_words=prm.key_words())
    try:
        base = ctx.lib.afhe_poly_gmem(ctx.h)
        rc = ctx.lib.afhe_key_switch_noalloc(ctx.h, C.c_void_p(base), 0, 4)
        assert rc == L.E_BUDGET
        assert b"scratch words" in ctx.lib.afhe_last_error()
    finally:
        ctx.close()
