"""The allocation-free key switch, afhe_key_switch_noalloc.

It exists for callers that cannot call cudaMalloc when they serve a request:
programs whose GPU memory already belongs to their own pool allocator, and
latency-bound threads that cannot absorb the device-wide synchronisation an
allocation can cause. Its working memory is a fixed array of static device
memory inside the library, shared by all calls on a device.

Checks, through the C ABI: two calls in a row (the second one sees whatever
the first left in the shared array) each give exactly the residues of the
ordinary afhe_key_switch on the same input and key, at every level; a
parameter set too big for the fixed array is refused with AFHE_E_BUDGET. The
file is named to run last; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, FHEHostDriver
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu


def run_shape(log_n, nq, qb, np_, pb, alpha):
    q, p = primes_for(log_n, nq, qb, np_, pb)
    prm = CkksParams(log_n, q, p, alpha)
    n = prm.n
    slot = (nq + np_) * n
    ctx = FheContext(prm, poly_words=8 * slot, key_words=prm.key_words())
    try:
        drv = FHEHostDriver(ctx)
        rng = np.random.default_rng(log_n * 7 + nq)
        allp = q + p
        a = np.concatenate([uniform_residues(rng, allp, n) for _ in range(prm.dnum)])
        b = np.concatenate([uniform_residues(rng, allp, n) for _ in range(prm.dnum)])
        ctx.write_key(0, np.concatenate([a, b]))
        base = ctx.lib.afhe_poly_gmem(ctx.h)
        for call, lvl in enumerate((nq, max(1, nq - 1))):
            x = uniform_residues(rng, q[:lvl], n)
            w = lvl * n
            # ordinary entry point: input at slot 0, outputs at slots 1 and 2
            ctx.write_poly(0, x)
            drv.key_switch(0, 0, slot, 2 * slot, lvl)
            want0, want1 = ctx.read_poly(slot, w), ctx.read_poly(2 * slot, w)
            # allocation-free entry point: io = [input | ks0 | ks1] at slot 4
            io_off = 4 * slot
            ctx.write_poly(io_off, x)
            ctx.write_poly(io_off + w, np.zeros(2 * w, dtype=np.uint64))
            rc = ctx.lib.afhe_key_switch_noalloc(ctx.h, C.c_void_p(base + io_off * 8), 0, lvl)
            assert rc == L.OK, ctx.lib.afhe_last_error()
            ctx.sync()
            got0, got1 = ctx.read_poly(io_off + w, w), ctx.read_poly(io_off + 2 * w, w)
            assert np.array_equal(got0, want0), f"call {call}: ks0 differs"
            assert np.array_equal(got1, want1), f"call {call}: ks1 differs"
            assert np.array_equal(ctx.read_poly(io_off, w), x), "input must be left unchanged"
    finally:
        ctx.close()


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
