"""afhe_eval_mac_plain_batch against exact integer arithmetic on the host.

Each output is the sum over its groups of the group's plaintexts, each moved
by its Galois automorphism (out[i] = pt[map[i]], the gather of
FHEHostDriver::automorphism), times the group's ciphertext, per limb mod
q_l; a group with AFHE_MAC_UNIT adds its plaintexts to c0. Checked with
60-bit primes and 300 terms in one output, so the 128-bit accumulators fold
(every 256 products at 60 bits); with accumulate; with an output that has
no groups; and the argument checks (overlap, bad Galois element).
"""
import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, automorphism_map, galois_elt
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu


def host_mac(q, n, jobs, poly, limbs, log_n, acc=None):
    out0 = [[0] * n for _ in range(limbs)] if acc is None else [list(map(int, acc[0][l * n:(l + 1) * n]))
                                                                 for l in range(limbs)]
    out1 = [[0] * n for _ in range(limbs)] if acc is None else [list(map(int, acc[1][l * n:(l + 1) * n]))
                                                                 for l in range(limbs)]
    o0 = [np.array(r, dtype=object) for r in out0]
    o1 = [np.array(r, dtype=object) for r in out1]
    for src, terms in jobs:
        for off, gal in terms:
            x = poly[off:off + limbs * n]
            m = automorphism_map(log_n, gal) if gal != 1 else np.arange(n)
            for l in range(limbs):
                pl = x[l * n:(l + 1) * n][m].astype(object)
                if src is None:
                    o0[l] = o0[l] + pl
                else:
                    o0[l] = o0[l] + pl * poly[src[0] + l * n:src[0] + (l + 1) * n].astype(object)
                    o1[l] = o1[l] + pl * poly[src[1] + l * n:src[1] + (l + 1) * n].astype(object)
    f = lambda o: np.concatenate([(o[l] % q[l]).astype(np.uint64) for l in range(limbs)])  # noqa: E731
    return f(o0), f(o1)


def call(ctx, outs, jobs_per_out, limbs, accumulate=False):
    first, groups, terms = [0], [], []
    for jobs in jobs_per_out:
        for src, ts in jobs:
            groups.append((src if src is not None else (L.MAC_UNIT, 0), len(terms), len(ts)))
            terms.extend(ts)
        first.append(len(groups))
    g = (L.MacGroup * max(1, len(groups)))()
    for k, (src, t0, nt) in enumerate(groups):
        g[k].src.c0_offset, g[k].src.c1_offset, g[k].first_term, g[k].n_terms = src[0], src[1], t0, nt
    t = (L.MacTerm * max(1, len(terms)))()
    for k, (off, gal) in enumerate(terms):
        t[k].pt, t[k].galois = off, gal
    o = (L.CtRef * len(outs))(*[L.CtRef(*c) for c in outs])
    fg = np.asarray(first, dtype=np.uint32)
    return ctx.lib.afhe_eval_mac_plain_batch(ctx.h, o, fg.ctypes.data_as(L.P32), len(outs), g, t, limbs,
                                             int(accumulate))


@pytest.mark.parametrize("q_bits", [50, 60])
def test_mac_plain_matches_host(q_bits):
    log_n, limbs = 11, 3
    q, p = primes_for(log_n, limbs, q_bits, 1, 61 if q_bits == 60 else 60)
    n = 1 << log_n
    w = limbs * n
    ctx = FheContext(CkksParams(log_n, q, p, 1), poly_words=400 * w, key_words=1024)
    try:
        rng = np.random.default_rng(q_bits)
        poly = np.concatenate([uniform_residues(rng, q, n) for _ in range(340)])
        ctx.write_poly(0, poly)
        src = [(2 * i * w, (2 * i + 1) * w) for i in range(8)]          # 8 ciphertexts
        pts = [(16 + i) * w for i in range(320)]                          # 320 plaintexts
        gals = [1, galois_elt(log_n, 1), galois_elt(log_n, -8), galois_elt(log_n, 64), 2 * n - 1]
        outs = [((336 + 2 * i) * w, (337 + 2 * i) * w) for i in range(2)] + [((350) * w, (351) * w)]
        jobs = [
            # 300 terms over 4 groups: the accumulators fold
            [(src[k], [(pts[75 * k + j], gals[j % len(gals)]) for j in range(75)]) for k in range(4)],
            # a unit group and a ciphertext group
            [(None, [(pts[300], gals[2]), (pts[301], 1)]), (src[5], [(pts[302], gals[3])])],
            [],
        ]
        assert call(ctx, outs, jobs, limbs) == L.OK, L.load().afhe_last_error()
        for o, job in zip(outs, jobs):
            e0, e1 = host_mac(q, n, job, poly, limbs, log_n)
            assert np.array_equal(ctx.read_poly(o[0], w), e0)
            assert np.array_equal(ctx.read_poly(o[1], w), e1)
        # accumulate adds the existing outputs
        before = [(ctx.read_poly(o[0], w), ctx.read_poly(o[1], w)) for o in outs[:2]]
        assert call(ctx, outs[:2], jobs[:2], limbs, accumulate=True) == L.OK
        for o, job, acc in zip(outs, jobs, before):
            e0, e1 = host_mac(q, n, job, poly, limbs, log_n, acc=acc)
            assert np.array_equal(ctx.read_poly(o[0], w), e0)
            assert np.array_equal(ctx.read_poly(o[1], w), e1)
        # an output may not overlap an operand, and Galois elements are odd and < 2N
        assert call(ctx, [src[6]], [[(src[6], [(pts[0], 1)])]], limbs) == L.E_ARG
        assert call(ctx, [src[6]], [[(src[7], [(src[6][0], 1)])]], limbs) == L.E_ARG
        assert call(ctx, [src[6]], [[(src[7], [(pts[0], 2)])]], limbs) == L.E_ARG
        assert call(ctx, [src[6], src[6]], [[], []], limbs) == L.E_ARG
    finally:
        ctx.close()


@pytest.mark.parametrize("nb,q_bits,local", [(1, 50, True), (4, 50, True), (16, 50, True), (16, 60, True),
                                              (16, 50, False), (4, 60, False)])
def test_diag_inner_equals_mac_plain(nb, q_bits, local):
    """afhe_eval_diag_inner_batch equals afhe_eval_mac_plain_batch with one
    group per baby step and one term per unit, units at pt + b * stride.
    With `local`, every placement is a rotation by a multiple of 64 slots,
    whose map keeps 256-word tiles in place (the shared-memory form of the
    kernel); otherwise a rotation by 5 is among them (the register form)."""
    log_n, limbs = 11, 2
    q, p = primes_for(log_n, limbs, q_bits, 1, 61 if q_bits == 60 else 60)
    n = 1 << log_n
    w = limbs * n
    ctx = FheContext(CkksParams(log_n, q, p, 1), poly_words=600 * w, key_words=1024)
    try:
        rng = np.random.default_rng(nb)
        ctx.write_poly(0, np.concatenate([uniform_residues(rng, q, n) for _ in range(500)]))
        stride = 3 * w                                   # a unit's plaintexts 3 polynomials apart
        srcs = [(2 * i * w, (2 * i + 1) * w) for i in range(32)]        # [0, 64 w)
        units = [64 * w + k * w for k in range(48)]                     # plaintexts in [64 w, 64 w + 48 w + 45 stride)
        gals = [1, galois_elt(log_n, -64), galois_elt(log_n, -256),
                galois_elt(log_n, 128) if local else galois_elt(log_n, 5)]
        jobs = [(list(range(0, 5)), 0), (list(range(7, 9)), 1), ([], 2)]    # (units, first source)
        outs_a = [((520 + 4 * j) * w, (521 + 4 * j) * w) for j in range(len(jobs))]
        outs_b = [((522 + 4 * j) * w, (523 + 4 * j) * w) for j in range(len(jobs))]
        src = (L.CtRef * (len(jobs) * nb))(*[L.CtRef(*srcs[(s + b) % 32]) for _, s in jobs for b in range(nb)])
        upt = np.array([units[k] for ks, _ in jobs for k in ks] or [0], dtype=np.uint64)
        ugal = np.array([gals[k % 4] for ks, _ in jobs for k in ks] or [1], dtype=np.uint32)
        first = np.concatenate([[0], np.cumsum([len(ks) for ks, _ in jobs])]).astype(np.uint32)
        oa = (L.CtRef * len(jobs))(*[L.CtRef(*c) for c in outs_a])
        rc = ctx.lib.afhe_eval_diag_inner_batch(ctx.h, oa, len(jobs), src, nb, upt.ctypes.data_as(L.P64),
                                                ugal.ctypes.data_as(L.P32), first.ctypes.data_as(L.P32), stride,
                                                limbs, 0)
        assert rc == L.OK, L.load().afhe_last_error()
        mac_jobs = [[(srcs[(s + b) % 32], [(units[k] + b * stride, gals[k % 4]) for k in ks]) for b in range(nb)]
                    for ks, s in jobs]
        assert call(ctx, outs_b, mac_jobs, limbs) == L.OK
        for a, b in zip(outs_a, outs_b):
            assert np.array_equal(ctx.read_poly(a[0], w), ctx.read_poly(b[0], w))
            assert np.array_equal(ctx.read_poly(a[1], w), ctx.read_poly(b[1], w))
        # nb must be a power of two up to 16
        assert ctx.lib.afhe_eval_diag_inner_batch(ctx.h, oa, 1, src, 3, upt.ctypes.data_as(L.P64),
                                                  ugal.ctypes.data_as(L.P32), first.ctypes.data_as(L.P32), stride,
                                                  limbs, 0) == L.E_ARG
    finally:
        ctx.close()
