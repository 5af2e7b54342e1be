"""afhe_dispatch (the fhe_accel_top drop-in) on the GPU against the oracle's
fhe_accel_top restatement: identical arenas in, identical poly_gmem out, for
every op code, bit for bit, at several ring degrees and RNS shapes."""
import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext
from oracle.oracle import tables_py as T
from tests.helpers import AccelImage, primes_for, uniform_residues

pytestmark = pytest.mark.gpu

# name: log_n, nq, q_bits, np, p_bits, first_bits, alpha, table_level
SHAPES = {
    "ref_n16384": (14, 11, 45, 4, 60, 60, 4, 10),
    "cfg1_n8192": (13, 3, 50, 1, 60, None, 1, 3),
    "n1024": (10, 4, 30, 2, 31, None, 2, 4),
    "n65536": (16, 5, 50, 2, 60, None, 2, 5),
    # the large IVF-PQ configuration's parameter set: N = 2^15, 12 x 50-bit Q
    # + 4 x 60-bit P, alpha 4, tables and key switch at all 12 limbs (dnum 3)
    "cfg4_n32768": (15, 12, 50, 4, 60, None, 4, 12),
}


def make(shape):
    log_n, nq, qb, np_, pb, fb, alpha, tl = SHAPES[shape]
    q, p = primes_for(log_n, nq, qb, np_, pb, first_bits=fb)
    img = AccelImage(log_n, q, p, alpha=alpha, table_level=tl)
    n = 1 << log_n
    pw = (nq + np_) * n
    ctx = FheContext(CkksParams(log_n, q, p, alpha), poly_words=6 * pw, key_words=img.key_words)
    ctx.write_key(0, img.key)
    return img, ctx, pw


@pytest.mark.parametrize("shape", list(SHAPES))
def test_every_op_matches_oracle(shape, orc):
    img, ctx, PW = make(shape)
    n, Lq = img.n, img.L
    rng = np.random.default_rng(11)
    poly = np.zeros(6 * PW, dtype=np.uint64)
    poly[:Lq * n] = uniform_residues(rng, img.q, n)
    poly[PW:PW + Lq * n] = uniform_residues(rng, img.q, n)
    m = T.auto_map(img.log_n, T.galois(img.log_n, 1)).astype(np.uint64)
    poly[5 * PW:5 * PW + n // 2] = m[0::2] | (m[1::2] << np.uint64(32))
    key = img.key.copy()
    ctx.write_poly(0, poly)
    tl = img.table_level
    ops = [
        (L.OP_LOAD_CONTEXT, Lq, dict(sizeQl=tl)),
        (L.OP_NTT, Lq, dict(src_a_offset=0, dst_offset=2 * PW)),
        (L.OP_INTT, Lq, dict(src_a_offset=2 * PW, dst_offset=3 * PW)),
        (L.OP_NTT, Lq, dict(src_a_offset=3 * PW, dst_offset=3 * PW)),             # in place
        (L.OP_INTT, Lq, dict(src_a_offset=3 * PW, dst_offset=3 * PW + n)),        # overlapping
        (L.OP_POLY_ADD, Lq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
        (L.OP_POLY_SUB, Lq, dict(src_a_offset=2 * PW, src_b_offset=PW, dst_offset=2 * PW)),
        (L.OP_POLY_MUL_NTT, Lq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
        (L.OP_AUTOMORPHISM, Lq, dict(src_a_offset=0, src_b_offset=5 * PW, dst_offset=4 * PW)),
        (L.OP_RESCALE, Lq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=3 * PW)),
        (L.OP_RESCALE, Lq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=0)),    # output over input
        (L.OP_KEY_SWITCH, tl, dict(src_a_offset=PW, dst_offset=2 * PW)),
        (L.OP_KEY_SWITCH, tl, dict(src_a_offset=2 * PW, dst_offset=2 * PW)),    # output over input
    ]
    h = orc.new_ctx(n)
    try:
        for op, limbs, kw in ops:
            a = img.args(op, limbs, **kw)
            assert orc.accel_top(h, poly, key, a) == 0
            rc = ctx.dispatch(a)
            assert rc == L.OK, (op, rc, L.load().afhe_last_error())
            got = ctx.read_poly(0, poly.size)
            assert np.array_equal(got, poly), f"op {op} {kw}"
    finally:
        orc.free_ctx(h)
        ctx.close()


def test_errors_are_statuses():
    img, ctx, PW = make("cfg1_n8192")
    try:
        a = img.args(L.OP_NTT, img.L, src_a_offset=0, dst_offset=PW)
        assert ctx.dispatch(a) == L.E_STATE            # before OP_LOAD_CONTEXT
        assert ctx.dispatch(img.args(L.OP_LOAD_CONTEXT, img.L)) == L.OK
        a = img.args(L.OP_NTT, img.L, src_a_offset=6 * PW, dst_offset=0)
        assert ctx.dispatch(a) == L.E_RANGE
        a = img.args(L.OP_NTT, img.L, src_a_offset=0, dst_offset=PW)
        a.rns_primes[0] += 2                            # primes differ from the loaded context
        assert ctx.dispatch(a) == L.E_ARG
        bad = img.args(L.OP_LOAD_CONTEXT, img.L)
        bad.barrett_k_q[0] += 1                         # inconsistent Barrett constant
        assert ctx.dispatch(bad) == L.E_ARG
        a = img.args(77, img.L)
        assert ctx.dispatch(a) == L.E_ARG
        a = img.args(L.OP_KEY_SWITCH, img.L, numPartQ=5)   # last digit would be empty
        assert ctx.dispatch(a) == L.E_ARG
        # the context is still usable after rejected calls
        a = img.args(L.OP_NTT, img.L, src_a_offset=0, dst_offset=PW)
        assert ctx.dispatch(a) == L.OK
    finally:
        ctx.close()
