"""Pins the oracle.

1. Known-answer properties of the C restatement that need no reference:
   INTT(NTT(x)) = x, the NTT diagonalises negacyclic convolution, the
   evaluation-form automorphism map equals the coefficient-form automorphism,
   rescale divides by q_l with the reference's centred rounding.
2. The C restatement (oracle/liborc.so) against the reference's own HLS
   C-simulation compiled verbatim (oracle/_ref/libref_hls.so) at the
   reference's ring degree N = 16384 and shapes (11 Q + 4 P limbs, dnum = 3,
   alpha = 4), word for word, including the full fhe_accel_top ABI.
"""
import numpy as np
import pytest

from oracle.oracle import tables_py as T
from tests.helpers import AccelImage, primes_for, uniform_residues

REF_N = 16384


def negacyclic(a, b, q):
    n = len(a)
    out = [0] * n
    for i in range(n):
        ai = int(a[i])
        if ai == 0:
            continue
        for j in range(n):
            k = i + j
            v = ai * int(b[j])
            if k < n:
                out[k] += v
            else:
                out[k - n] -= v
    return np.array([x % q for x in out], dtype=np.uint64)


def test_ntt_roundtrip_and_convolution(orc):
    log_n, n = 8, 256
    q = primes_for(log_n, 1, 40, 1, 41)[0][0]
    tw, itw = T.twiddles(log_n, q)
    rng = np.random.default_rng(1)
    a = rng.integers(0, q, n, dtype=np.uint64)
    b = rng.integers(0, q, n, dtype=np.uint64)
    A, B = orc.ntt(a, tw, q), orc.ntt(b, tw, q)
    assert np.array_equal(orc.intt(A, itw, q), a)
    prod = orc.poly("mul", A, B, q)
    assert np.array_equal(orc.intt(prod, itw, q), negacyclic(a, b, q))


def test_automorphism_map_is_coefficient_automorphism(orc):
    log_n, n = 8, 256
    q = primes_for(log_n, 1, 40, 1, 41)[0][0]
    tw, itw = T.twiddles(log_n, q)
    rng = np.random.default_rng(2)
    x = rng.integers(0, q, n, dtype=np.uint64)
    for step in (1, 3, -1, 17):
        k = T.galois(log_n, step)
        m = T.auto_map(log_n, k).astype(np.uint64)
        packed = m[0::2] | (m[1::2] << np.uint64(32))
        got = orc.automorphism(x, packed)
        coef = orc.intt(x, itw, q)
        sig = np.zeros(n, dtype=object)
        for i in range(n):
            e = i * k % (2 * n)
            if e < n:
                sig[e] = (sig[e] + int(coef[i])) % q
            else:
                sig[e - n] = (sig[e - n] - int(coef[i])) % q
        assert np.array_equal(got, orc.ntt(sig.astype(np.uint64), tw, q))


def test_rescale_divides_and_rounds(orc):
    log_n, n = 8, 256
    q, _ = primes_for(log_n, 3, 30, 1, 31)
    tws = [T.twiddles(log_n, x) for x in q]
    rng = np.random.default_rng(3)
    Q = q[0] * q[1] * q[2]
    vals = [int(v) for v in rng.integers(-(2**60), 2**60, n)]
    vals[0], vals[1] = q[2] // 2 + q[2] * 5, -(q[2] // 2) - q[2] * 7   # exact ties of the centred lift
    coef = [np.array([v % qi for v in vals], dtype=np.uint64) for qi in q]
    ev = np.concatenate([orc.ntt(c, tw, qi) for c, (tw, _), qi in zip(coef, tws, q)])
    qlql, qlinv = T.rescale(q, 3)
    out = orc.rescale(ev, q, tws[2][1], np.concatenate([t[0] for t in tws]), qlql, qlinv, n)
    for i in range(2):
        got = orc.intt(out[i * n:(i + 1) * n], tws[i][1], q[i])
        exp = []
        for v in vals:
            r = v % q[2]
            if r > q[2] >> 1:
                r -= q[2]
            exp.append(((v - r) // q[2]) % q[i])
        assert np.array_equal(got, np.array(exp, dtype=np.uint64))
    assert Q  # noqa


# ---------------------------------------------------------------------------
# against the reference compiled verbatim (N = 16384)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def refimg():
    q, p = primes_for(14, 11, 45, 4, 60, first_bits=60)
    return AccelImage(14, q, p, alpha=4, table_level=10, numPartQ=3, key_level=10)


def test_mod_mul_barrett_is_exact(ref, refimg):
    rng = np.random.default_rng(42)
    for q in refimg.q + refimg.p:
        a = rng.integers(0, q, 1000, dtype=np.uint64)
        b = rng.integers(0, q, 1000, dtype=np.uint64)
        for x, y in zip(a[:200], b[:200]):
            assert ref.mod_mul(int(x), int(y), q) == int(x) * int(y) % q
        # the call sites that pass a value >= q as "reduce by multiplying by 1"
        assert ref.mod_mul(q + 12345, 1, q) == 12345


def test_ntt_intt_poly_auto_vs_reference(ref, orc, refimg):
    img, n = refimg, REF_N
    rng = np.random.default_rng(5)
    for l in (0, 5, 10):
        q = img.q[l]
        tw, itw = img.tw_q[l * n:(l + 1) * n], img.itw_q[l * n:(l + 1) * n]
        a = rng.integers(0, q, n, dtype=np.uint64)
        b = rng.integers(0, q, n, dtype=np.uint64)
        assert np.array_equal(ref.ntt(a, tw, q), orc.ntt(a, tw, q))
        assert np.array_equal(ref.intt(a, itw, q), orc.intt(a, itw, q))
        for op in ("add", "sub", "mul"):
            assert np.array_equal(ref.poly(op, a, b, q), orc.poly(op, a, b, q))
    m = T.auto_map(14, 5).astype(np.uint64)
    packed = m[0::2] | (m[1::2] << np.uint64(32))
    a = rng.integers(0, img.q[0], n, dtype=np.uint64)
    assert np.array_equal(ref.automorphism(a, packed), orc.automorphism(a, packed))


def test_rescale_vs_reference(ref, orc):
    q, p = primes_for(14, 11, 45, 4, 60, first_bits=60)
    img = AccelImage(14, q, p, alpha=4, table_level=11)
    rng = np.random.default_rng(6)
    a = uniform_residues(rng, q, REF_N)
    itl = img.itw_q[10 * REF_N:11 * REF_N]
    r = ref.rescale(a, q, itl, img.tw_q, img.qlql, img.qlinv)
    o = orc.rescale(a, q, itl, img.tw_q, img.qlql, img.qlinv, REF_N)
    assert np.array_equal(r, o)


def test_key_switch_vs_reference(ref, orc, refimg):
    img, n = refimg, REF_N
    sq, K = 10, 4
    rng = np.random.default_rng(8)
    c = uniform_residues(rng, img.q[:sq], n)
    key = img.key[img.off["evk"]:img.off["evk"] + 2 * 3 * (sq + K) * n]
    r0, r1 = ref.key_switch(c, key, 0, 3 * (sq + K) * n, sq, K, 3, 4, img.q, img.p, img.tw_q, img.itw_q,
                            img.tw_p, img.itw_p, img.qhat_inv, img.qhat_modp, img.pinv, img.phinv, img.phq)
    ea = np.concatenate(img.evk_a)
    eb = np.concatenate(img.evk_b)
    o0, o1 = orc.key_switch(c, ea, eb, sq + K, sq, sq, K, 3, 4, img.q, img.p, img.tw_q, img.itw_q, img.tw_p,
                            img.itw_p, img.qhat_inv, img.qhat_modp, img.pinv, img.phinv, img.phq, n)
    assert np.array_equal(r0, o0)
    assert np.array_equal(r1, o1)


def test_accel_top_abi_vs_reference(ref, orc, refimg):
    """Every op code through fhe_accel_top, same arenas in, same arenas out
    (the shapes of hardware_fpga_model/hls/src/tb_fhe_accel.cpp:64-503)."""
    from anns_fhe_b200 import _lib as L
    img, n = refimg, REF_N
    PW = 15 * n
    poly = np.zeros(6 * PW, dtype=np.uint64)
    rng = np.random.default_rng(9)
    poly[:11 * n] = uniform_residues(rng, img.q, n)
    poly[PW:PW + 11 * n] = uniform_residues(rng, img.q, n)
    m = T.auto_map(14, 5).astype(np.uint64)
    poly[5 * PW:5 * PW + n // 2] = m[0::2] | (m[1::2] << np.uint64(32))
    key = img.key.copy()
    ctx = orc.new_ctx(n)
    try:
        rp, rk = poly.copy(), key.copy()
        op_list = [
            (L.OP_LOAD_CONTEXT, 11, {}),
            (L.OP_NTT, 11, dict(src_a_offset=0, dst_offset=2 * PW)),
            (L.OP_INTT, 11, dict(src_a_offset=2 * PW, dst_offset=3 * PW)),
            (L.OP_POLY_ADD, 11, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_POLY_SUB, 11, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_POLY_MUL_NTT, 11, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_AUTOMORPHISM, 11, dict(src_a_offset=0, src_b_offset=5 * PW, dst_offset=3 * PW)),
            (L.OP_RESCALE, 11, dict(src_a_offset=0, src_b_offset=PW, dst_offset=3 * PW)),
            (L.OP_KEY_SWITCH, 10, dict(src_a_offset=PW, dst_offset=2 * PW)),
        ]
        for op, limbs, kw in op_list:
            a = img.args(op, limbs, **kw)
            if op == L.OP_LOAD_CONTEXT:
                a.active_limbs = 11
                a.sizeQl = 10
            assert orc.accel_top(ctx, poly, key, a) == 0
            ref.accel_top(rp, rk, a)
            assert np.array_equal(poly, rp), f"op {op}"
    finally:
        orc.free_ctx(ctx)


@pytest.mark.parametrize("level", [2, 6])
def test_rescale_vs_reference_lower_levels(ref, orc, level):
    """Rescale from `level` limbs (tables for that level), as the reference
    does it below the top."""
    q, p = primes_for(14, 11, 45, 4, 60, first_bits=60)
    img = AccelImage(14, q, p, alpha=4, table_level=level)
    rng = np.random.default_rng(60 + level)
    a = uniform_residues(rng, q[:level], REF_N)
    itl = img.itw_q[(level - 1) * REF_N:level * REF_N]
    r = ref.rescale(a, q, itl, img.tw_q, img.qlql, img.qlinv)
    o = orc.rescale(a, q[:level], itl, img.tw_q, img.qlql, img.qlinv, REF_N)
    assert np.array_equal(r, o)


@pytest.mark.parametrize("sq", [9, 11])
def test_key_switch_vs_reference_partial_digits(ref, orc, sq):
    """The reference kernel takes three digits of alpha = 4 limbs; at 9 and 11
    limbs its last digit holds 1 and 3 limbs."""
    q, p = primes_for(14, 11, 45, 4, 60, first_bits=60)
    img = AccelImage(14, q, p, alpha=4, table_level=sq, numPartQ=3, key_level=sq, seed=sq)
    n, K = REF_N, 4
    rng = np.random.default_rng(80 + sq)
    c = uniform_residues(rng, q[:sq], n)
    key = img.key[img.off["evk"]:img.off["evk"] + 2 * 3 * (sq + K) * n]
    r0, r1 = ref.key_switch(c, key, 0, 3 * (sq + K) * n, sq, K, 3, 4, img.q, img.p, img.tw_q, img.itw_q,
                            img.tw_p, img.itw_p, img.qhat_inv, img.qhat_modp, img.pinv, img.phinv, img.phq)
    o0, o1 = orc.key_switch(c, np.concatenate(img.evk_a), np.concatenate(img.evk_b), sq + K, sq, sq, K, 3, 4,
                            img.q, img.p, img.tw_q, img.itw_q, img.tw_p, img.itw_p, img.qhat_inv, img.qhat_modp,
                            img.pinv, img.phinv, img.phq, n)
    assert np.array_equal(r0, o0)
    assert np.array_equal(r1, o1)


# ---------------------------------------------------------------------------
# the reference's sources built at other ring degrees (oracle/Makefile rewrites
# their N = 16384 literals): each build against the C restatement, which the
# tests above pin to the verbatim build
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("log_n,nq,qb,np_,pb,alpha", [(13, 3, 50, 1, 60, 1), (15, 9, 50, 4, 60, 4)],
                         ids=["n8192_3q1p_a1", "n32768_9q4p_a4"])
def test_reference_at_other_ring_degrees(orc, log_n, nq, qb, np_, pb, alpha):
    """Every op code through the rebuilt reference's fhe_accel_top, once over
    word arenas and once over its own SimMemoryBus held across the calls,
    equals the restatement: the small configuration's shape (N = 8192, 3 + 1
    limbs, alpha 1) and, at the large configuration's ring (N = 32768) and
    primes' sizes, 9 + 4 limbs with alpha 4. The reference's OP 99 loads
    tables for exactly three digits (fhe_accel_top.cpp:204-207 sizes the last
    one as active_limbs - 2 alpha), so its table load needs 2 alpha <
    active_limbs; 9 limbs give digits of 4, 4 and 1."""
    from anns_fhe_b200 import _lib as L
    from oracle.oracle import Ref, RefBus, build_oracle
    n = 1 << log_n
    if not Ref.available(n):
        try:
            build_oracle(ref=True)
        except Exception:
            pass
    if not Ref.available(n):
        pytest.skip(f"reference build for N = {n} absent (reference tree absent)")
    ref = Ref(n)
    q, p = primes_for(log_n, nq, qb, np_, pb)
    img = AccelImage(log_n, q, p, alpha=alpha, table_level=nq)
    PW = (nq + np_) * n
    poly = np.zeros(6 * PW, dtype=np.uint64)
    rng = np.random.default_rng(log_n)
    poly[:nq * n] = uniform_residues(rng, q, n)
    poly[PW:PW + nq * n] = uniform_residues(rng, q, n)
    m = T.auto_map(log_n, T.galois(log_n, 3)).astype(np.uint64)
    poly[5 * PW:5 * PW + n // 2] = m[0::2] | (m[1::2] << np.uint64(32))
    key = img.key.copy()
    rp, rk = poly.copy(), key.copy()
    bus = RefBus(ref, poly.size, key.size)
    bus.write_poly(0, poly)
    bus.write_key(0, key)
    ctx = orc.new_ctx(n)
    try:
        for op, limbs, kw in [
            (L.OP_LOAD_CONTEXT, nq, {}),
            (L.OP_NTT, nq, dict(src_a_offset=0, dst_offset=2 * PW)),
            (L.OP_INTT, nq, dict(src_a_offset=2 * PW, dst_offset=3 * PW)),
            (L.OP_POLY_ADD, nq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_POLY_SUB, nq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_POLY_MUL_NTT, nq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=2 * PW)),
            (L.OP_AUTOMORPHISM, nq, dict(src_a_offset=0, src_b_offset=5 * PW, dst_offset=3 * PW)),
            (L.OP_RESCALE, nq, dict(src_a_offset=0, src_b_offset=PW, dst_offset=3 * PW)),
            (L.OP_KEY_SWITCH, nq, dict(src_a_offset=PW, dst_offset=2 * PW)),
        ]:
            a = img.args(op, limbs, **kw)
            assert orc.accel_top(ctx, poly, key, a) == 0
            ref.accel_top(rp, rk, a)
            bus.top(Ref.top_args(a))
            assert np.array_equal(poly, rp), f"op {op}"
            assert np.array_equal(bus.read_poly(0, poly.size), poly), f"op {op} (bus)"
    finally:
        orc.free_ctx(ctx)
        bus.close()


def test_reference_host_sequence_matches_composites(orc):
    """The timed CPU baseline (oracle/refchain.py) drives the reference's
    fhe_accel_top in FHEHostDriver's operator sequence. At the level its
    tables are loaded for, eval_mult_relin_rescale, eval_rotate and
    eval_sub_plain / eval_add there equal the oracle's composites, so the
    sequence it times is the reference's chain (small configuration's shape:
    N = 8192, 3 + 1 limbs, alpha 1)."""
    from oracle.composite import OracleCKKS
    from oracle.oracle import Ref, build_oracle
    from oracle.refchain import HostDriver, RefBusBackend
    log_n, n, L, alpha = 13, 8192, 3, 1
    if not Ref.available(n):
        try:
            build_oracle(ref=True)
        except Exception:
            pass
    if not Ref.available(n):
        pytest.skip("reference build for N = 8192 absent (reference tree absent)")
    q = T.ntt_primes(log_n, 50, L)
    p = T.ntt_primes(log_n, 60, 1, q)
    ora = OracleCKKS(log_n, q, p, alpha, orc)
    t = ora.tables(L)
    rng = np.random.default_rng(33)
    allp = q + p
    ka = np.concatenate([uniform_residues(rng, allp, n) for _ in range(ora.dnum)])
    kb = np.concatenate([uniform_residues(rng, allp, n) for _ in range(ora.dnum)])
    tables = dict(tw=np.concatenate(ora.tw), itw=np.concatenate(ora.itw), qhat_inv=t["qhat_inv"],
                  qhat_modp=t["qhat_modp"], pinv=t["pinv"], phinv=t["phinv"], phq=t["phq"], qlql=t["qlql"],
                  qlinv=t["qlinv"], key=np.concatenate([ka, kb]))
    W = 8 * n
    steps = [1, 2, 4]
    bus = RefBusBackend(n, 20 * W, 2 * len(allp) * n + 2048 + 2 * ora.dnum * (L + 1) * n)
    try:
        drv = HostDriver(bus, log_n, q, p, alpha, L, 1, steps, W, 10 * W, 16 * W, 2 * len(allp) * n + 2048,
                         tables=tables)
        A = (uniform_residues(rng, q, n), uniform_residues(rng, q, n))
        pt = uniform_residues(rng, q, n)
        for i, v in enumerate(A + (pt,)):
            bus.write_poly(i * W, v)
        drv.eval_mult_relin_rescale(0, W, 0, W, 3 * W, 4 * W, L)
        e0, e1 = ora.eval_mult_relin_rescale(A, A, (ka, kb), L)
        assert np.array_equal(bus.read_poly(3 * W, (L - 1) * n), e0)
        assert np.array_equal(bus.read_poly(4 * W, (L - 1) * n), e1)
        rot = {s: (ka, kb) for s in steps}
        drv.eval_rotate(0, W, 5 * W, 6 * W, 7, L)
        e0, e1 = ora.eval_rotate(A, 7, rot, L)
        assert np.array_equal(bus.read_poly(5 * W, L * n), e0)
        assert np.array_equal(bus.read_poly(6 * W, L * n), e1)
        drv.eval_sub_plain(0, W, 2 * W, 7 * W, 8 * W, L)
        drv.eval_add(7 * W, 8 * W, 5 * W, 6 * W, 7 * W, 8 * W, L)
        e0, e1 = ora.eval_add(ora.eval_sub_plain(A, pt, L), (e0, e1), L)
        assert np.array_equal(bus.read_poly(7 * W, L * n), e0)
        assert np.array_equal(bus.read_poly(8 * W, L * n), e1)
    finally:
        bus.close()
