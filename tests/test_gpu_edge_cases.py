"""Edge cases of the batched C-ABI entry points on the GPU.

* Empty batches (count 0, null arrays) succeed and launch no kernel, on every
  batched entry point.
* Ragged batches: more ciphertexts than the context has lanes, and a chunk
  width that does not divide the batch, give every ciphertext exactly the
  oracle's result, with each entry's own rotation step, and with outputs
  that alias their inputs.
* Maximum sizes: operands that end on the last word of poly_gmem, the top
  level, and max_batch 4096 (one more is an error).
* Error statuses: out-of-range offsets (E_RANGE), a missing rotation key
  (E_NOKEY), limb counts outside the loaded levels (E_LEVEL), null arrays,
  bad options and bad row reads (E_ARG). A call that fails its checks
  launches no kernel and leaves the arena as it was, like the reference's
  memory bus, which rejects an out-of-range access before any word moves
  (cpp_host_model/src/sim_memory_bus.cpp:13-15), and its driver, which
  throws on a missing rotation key before it rotates
  (cpp_host_model/src/fhe_host_driver.cpp:337-339).
"""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.driver import CkksParams, FheContext, FHEHostDriver
from oracle.composite import OracleCKKS
from tests.helpers import primes_for, uniform_residues

pytestmark = pytest.mark.gpu

LOG_N, NQ, NP, ALPHA, LANES = 10, 4, 2, 2, 4
STEPS = (1, 2, -1, 5)
SLOTS = 64


class Edge:
    def __init__(self, orc):
        q, p = primes_for(LOG_N, NQ, 40, NP, 45)
        self.prm = CkksParams(LOG_N, q, p, ALPHA)
        self.n = 1 << LOG_N
        self.PW = (NQ + NP) * self.n
        self.ora = OracleCKKS(LOG_N, q, p, ALPHA, orc)
        kw = self.prm.key_words()
        self.ctx = FheContext(self.prm, poly_words=SLOTS * self.PW, key_words=(1 + len(STEPS)) * kw,
                              max_batch=LANES)
        self.lib, self.h = self.ctx.lib, self.ctx.h
        self.drv = FHEHostDriver(self.ctx)
        rng = np.random.default_rng(77)
        allp = q + p
        self.keys = []
        for i in range(1 + len(STEPS)):
            a = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(self.prm.dnum)])
            b = np.concatenate([uniform_residues(rng, allp, self.n) for _ in range(self.prm.dnum)])
            self.ctx.write_key(i * kw, np.concatenate([a, b]))
            self.keys.append((a, b))
        self.drv.set_relin_key(0)
        self.rot = {}
        for i, s in enumerate(STEPS):
            self.drv.add_rotation_key(s, (i + 1) * kw)
            self.rot[s] = self.keys[i + 1]
        self.rng = rng

    def slot(self, i):
        return i * self.PW

    def ct(self, level):
        qs = self.prm.q[:level]
        return uniform_residues(self.rng, qs, self.n), uniform_residues(self.rng, qs, self.n)

    def put_ct(self, i, c):
        self.ctx.write_poly(self.slot(2 * i), c[0])
        self.ctx.write_poly(self.slot(2 * i + 1), c[1])

    def get_ct(self, i, limbs):
        w = limbs * self.n
        return self.ctx.read_poly(self.slot(2 * i), w), self.ctx.read_poly(self.slot(2 * i + 1), w)

    def ref(self, i):
        return (self.slot(2 * i), self.slot(2 * i + 1))

    @staticmethod
    def refs(pairs):
        arr = (L.CtRef * max(len(pairs), 1))()
        for k, (c0, c1) in enumerate(pairs):
            arr[k].c0_offset, arr[k].c1_offset = c0, c1
        return arr

    def launches(self):
        self.ctx.sync()
        return self.lib.afhe_kernel_launches()

    def snapshot(self):
        self.ctx.sync()
        return self.ctx.read_poly(0, SLOTS * self.PW)


@pytest.fixture(scope="module")
def ed(orc):
    e = Edge(orc)
    yield e
    e.ctx.close()


def test_empty_batches_launch_nothing(ed):
    lib, h = ed.lib, ed.h
    nullref = C.POINTER(L.CtRef)()
    null64 = C.POINTER(C.c_uint64)()
    nulli32 = C.POINTER(C.c_int32)()
    before = ed.launches()
    calls = {
        "eval_add_batch": lib.afhe_eval_add_batch(h, nullref, nullref, nullref, 0, NQ),
        "eval_sub_plain_batch": lib.afhe_eval_sub_plain_batch(h, nullref, null64, nullref, 0, NQ),
        "eval_mult_relin_rescale_batch": lib.afhe_eval_mult_relin_rescale_batch(h, nullref, nullref, nullref, 0, NQ),
        "eval_mult_plain_rescale_batch": lib.afhe_eval_mult_plain_rescale_batch(h, nullref, null64, nullref, 0, NQ),
        "rescale_batch": lib.afhe_rescale_batch(h, nullref, nullref, 0, NQ),
        "eval_copy_batch": lib.afhe_eval_copy_batch(h, nullref, nullref, 0, NQ),
        "eval_rotate_batch": lib.afhe_eval_rotate_batch(h, nullref, nullref, 0, 3, NQ),
        "eval_rotate_accumulate_batch": lib.afhe_eval_rotate_accumulate_batch(h, nullref, nullref, 0, 3, NQ),
        "eval_rotate_steps_batch": lib.afhe_eval_rotate_steps_batch(h, nullref, nullref, nulli32, 0, NQ),
        "ntt_batch": lib.afhe_ntt_batch(h, null64, 0, NQ, 0),
        "decrypt_batch": lib.afhe_decrypt_batch(h, nullref, 0, ed.slot(0), ed.slot(1), NQ),
        "read_poly_rows": lib.afhe_read_poly_rows(h, 0, ed.n, 0, ed.n, null64),
        "read_poly": lib.afhe_read_poly(h, 0, null64, 0),
    }
    assert all(rc == L.OK for rc in calls.values()), calls
    assert ed.launches() == before
    # a null array with a non-zero count is an argument error
    assert lib.afhe_eval_rotate_steps_batch(h, nullref, nullref, nulli32, 1, NQ) == L.E_ARG
    assert lib.afhe_rescale_batch(h, nullref, nullref, 2, NQ) == L.E_ARG
    assert lib.afhe_read_poly_rows(h, 0, ed.n, 1, ed.n, null64) == L.E_ARG
    assert ed.launches() == before


@pytest.mark.parametrize("chunk", [0, 3], ids=["lanes", "chunk3"])
@pytest.mark.parametrize("fused", [1, 0], ids=["fused", "multi"])
def test_ragged_rotate_batches(ed, chunk, fused):
    """11 ciphertexts through a 4-lane context: chunks of 4, 4, 3 (or 3, 3,
    3, 2). Each entry has its own step; outputs overwrite the inputs."""
    ed.ctx.set_option(L.OPT_KS_FUSED, fused)
    ed.ctx.set_option(L.OPT_CHUNK, chunk)
    try:
        for lvl in (NQ, 2):
            cts = [ed.ct(lvl) for _ in range(11)]
            steps = [STEPS[i % len(STEPS)] for i in range(11)]
            for i, c in enumerate(cts):
                ed.put_ct(i, c)
            refs = ed.refs([ed.ref(i) for i in range(11)])
            st = (C.c_int32 * 11)(*steps)
            L.check(ed.lib.afhe_eval_rotate_steps_batch(ed.h, refs, refs, st, 11, lvl), "rotate_steps_batch")
            for i, (c, s) in enumerate(zip(cts, steps)):
                e0, e1 = ed.ora.eval_rotate_single_step(c, s, ed.rot, lvl)
                g0, g1 = ed.get_ct(i, lvl)
                assert np.array_equal(g0, e0) and np.array_equal(g1, e1), (lvl, i, s)
            # the same total rotation for all 11, written to separate outputs
            for i, c in enumerate(cts):
                ed.put_ct(i, c)
            ed.drv.eval_rotate_batch([ed.ref(i) for i in range(11)], [ed.ref(12 + i) for i in range(11)], 3, lvl)
            for i, c in enumerate(cts):
                e0, e1 = ed.ora.eval_rotate(c, 3, ed.rot, lvl)
                g0, g1 = ed.get_ct(12 + i, lvl)
                assert np.array_equal(g0, e0) and np.array_equal(g1, e1), (lvl, i)
    finally:
        ed.ctx.set_option(L.OPT_CHUNK, 0)
        ed.ctx.set_option(L.OPT_KS_FUSED, 1)


def test_ragged_rescale_and_copy_batches(ed):
    cts = [ed.ct(NQ) for _ in range(9)]
    for i, c in enumerate(cts):
        ed.put_ct(i, c)
    ed.ctx.set_option(L.OPT_CHUNK, 2)
    try:
        src = ed.refs([ed.ref(i) for i in range(9)])
        dst = ed.refs([ed.ref(12 + i) for i in range(9)])
        L.check(ed.lib.afhe_eval_copy_batch(ed.h, src, dst, 9, NQ), "copy_batch")
        for i, c in enumerate(cts):
            g0, g1 = ed.get_ct(12 + i, NQ)
            assert np.array_equal(g0, c[0]) and np.array_equal(g1, c[1])
        L.check(ed.lib.afhe_rescale_batch(ed.h, src, src, 9, NQ), "rescale_batch")   # in place
        for i, c in enumerate(cts):
            g0, g1 = ed.get_ct(i, NQ - 1)
            assert np.array_equal(g0, ed.ora.rescale_poly(c[0], NQ))
            assert np.array_equal(g1, ed.ora.rescale_poly(c[1], NQ))
    finally:
        ed.ctx.set_option(L.OPT_CHUNK, 0)


def test_operands_at_the_end_of_the_arena(ed):
    """An operand that ends exactly on the last word of poly_gmem is read and
    written like any other."""
    last = SLOTS * ed.PW - NQ * ed.n
    c = ed.ct(NQ)
    ed.ctx.write_poly(ed.slot(4), c[0])
    ed.ctx.write_poly(last, c[1])
    ed.drv.eval_rotate_single_step(ed.slot(4), last, ed.slot(0), ed.slot(1), 2, NQ)
    e0, e1 = ed.ora.eval_rotate_single_step(c, 2, ed.rot, NQ)
    assert np.array_equal(ed.ctx.read_poly(ed.slot(0), NQ * ed.n), e0)
    assert np.array_equal(ed.ctx.read_poly(ed.slot(1), NQ * ed.n), e1)
    L.check(ed.lib.afhe_eval_copy_batch(ed.h, ed.refs([(ed.slot(0), ed.slot(1))]), ed.refs([(ed.slot(2), last)]),
                                        1, NQ), "copy_batch")
    assert np.array_equal(ed.ctx.read_poly(last, NQ * ed.n), e1)
    # rows that end on the last word
    got = np.zeros(2 * ed.n, dtype=np.uint64)
    L.check(ed.lib.afhe_read_poly_rows(ed.h, last + ed.n, 2 * ed.n, 2, ed.n, got.ctypes.data_as(L.P64)), "rows")
    assert np.array_equal(got[:ed.n], e1[ed.n:2 * ed.n]) and np.array_equal(got[ed.n:], e1[3 * ed.n:])


def test_failed_checks_change_nothing(ed):
    lib, h = ed.lib, ed.h
    for i in range(4):
        ed.put_ct(i, ed.ct(NQ))
    before_mem = ed.snapshot()
    before = ed.launches()
    good = [ed.ref(0), ed.ref(1), ed.ref(2)]
    past_end = (SLOTS * ed.PW - NQ * ed.n + 1, ed.slot(7))
    # a missing key on the last entry: nothing of the batch runs
    st = (C.c_int32 * 3)(1, 2, 4)
    r = ed.refs(good)
    assert lib.afhe_eval_rotate_steps_batch(h, r, r, st, 3, NQ) == L.E_NOKEY
    assert b"4" in lib.afhe_last_error()
    # an operand one word past the end, on the last entry
    r2 = ed.refs(good[:2] + [past_end])
    st2 = (C.c_int32 * 3)(1, 2, 1)
    assert lib.afhe_eval_rotate_steps_batch(h, r2, r2, st2, 3, NQ) == L.E_RANGE
    assert lib.afhe_eval_copy_batch(h, ed.refs(good), r2, 3, NQ) == L.E_RANGE
    assert lib.afhe_rescale_batch(h, r2, r2, 3, NQ) == L.E_RANGE
    assert lib.afhe_eval_rotate_batch(h, r2, r2, 3, 3, NQ) == L.E_RANGE
    # limb counts outside the loaded levels
    r3 = ed.refs(good)
    assert lib.afhe_rescale_batch(h, r3, r3, 3, 1) == L.E_LEVEL
    assert lib.afhe_rescale_batch(h, r3, r3, 3, NQ + 1) == L.E_LEVEL
    assert lib.afhe_eval_copy_batch(h, r3, r3, 3, 0) == L.E_LEVEL
    assert lib.afhe_eval_rotate_steps_batch(h, r3, r3, (C.c_int32 * 3)(1, 1, 1), 3, NQ + 1) == L.E_LEVEL
    # a galois element that is even or >= 2N
    assert lib.afhe_automorphism(h, ed.slot(0), 4, ed.slot(1), NQ) == L.E_ARG
    assert lib.afhe_automorphism(h, ed.slot(0), 2 * ed.n + 1, ed.slot(1), NQ) == L.E_ARG
    # row reads: stride shorter than a row, rows past the end
    buf = np.zeros(4 * ed.n, dtype=np.uint64)
    p = buf.ctypes.data_as(L.P64)
    assert lib.afhe_read_poly_rows(h, 0, ed.n - 1, 2, ed.n, p) == L.E_ARG
    assert lib.afhe_read_poly_rows(h, SLOTS * ed.PW - ed.n, ed.n, 2, ed.n, p) == L.E_RANGE
    assert lib.afhe_read_poly_rows(h, 0, 2**62, 4, ed.n, p) == L.E_RANGE
    assert ed.launches() == before
    assert np.array_equal(ed.snapshot(), before_mem)


def test_options_and_limits(ed):
    lib, h = ed.lib, ed.h
    v = C.c_int64()
    assert lib.afhe_ctx_set_option(h, L.OPT_CHUNK, LANES + 1) == L.E_ARG
    assert lib.afhe_ctx_set_option(h, L.OPT_CHUNK, -1) == L.E_ARG
    assert lib.afhe_ctx_set_option(h, 99, 0) == L.E_ARG
    assert lib.afhe_ctx_get_option(h, 99, C.byref(v)) == L.E_ARG
    assert lib.afhe_ctx_get_option(h, L.OPT_CHUNK, C.byref(v)) == L.OK and v.value == LANES
    assert lib.afhe_ctx_set_option(h, L.OPT_CHUNK, LANES) == L.OK
    assert lib.afhe_ctx_set_option(h, L.OPT_CHUNK, 0) == L.OK
    # a null host buffer with a non-zero count
    assert lib.afhe_read_poly(h, 0, C.POINTER(C.c_uint64)(), 8) == L.E_ARG
    # above N = 2^13 the one-kernel key switch runs on thread-block clusters:
    # on by default where the GPU can place them, and it can be switched
    q, p = primes_for(14, 2, 40, 1, 45)
    with FheContext(CkksParams(14, q, p, 1), poly_words=1 << 16, key_words=1 << 16, max_batch=1) as big:
        assert big.get_option(L.OPT_KS_FUSED) == 1
        assert big.lib.afhe_ctx_set_option(big.h, L.OPT_KS_FUSED, 0) == L.OK
        assert big.lib.afhe_ctx_set_option(big.h, L.OPT_KS_FUSED, 1) == L.OK
        # smallest launch the one-kernel path takes
        assert big.lib.afhe_ctx_set_option(big.h, L.OPT_FUSED_MIN, 0) == L.E_ARG
        assert big.lib.afhe_ctx_set_option(big.h, L.OPT_FUSED_MIN, 5) == L.OK
        assert big.get_option(L.OPT_FUSED_MIN) == 5
    # max_batch: 4096 is the largest
    small = CkksParams(10, ed.prm.q[:2], ed.prm.p[:1], 1)
    with pytest.raises(L.AfheError) as ei:
        FheContext(small, poly_words=1 << 12, key_words=1 << 12, max_batch=4097)
    assert ei.value.status == L.E_ARG
    with FheContext(small, poly_words=1 << 12, key_words=1 << 12, max_batch=4096) as top:
        assert top.get_option(L.OPT_CHUNK) == 4096


def test_out_of_memory_leaves_later_calls_clean(ed):
    """An arena larger than the GPU's memory fails afhe_ctx_create with a CUDA
    status (cudaMalloc's out of memory, no fault); the next context's first
    launches do not report that stale error."""
    small = CkksParams(10, ed.prm.q[:2], ed.prm.p[:1], 1)
    with pytest.raises(L.AfheError) as ei:
        FheContext(small, poly_words=1 << 40, key_words=1 << 12)      # 8 TiB
    assert ei.value.status == L.E_CUDA and "out of memory" in str(ei.value)
    with FheContext(small, poly_words=1 << 14, key_words=1 << 12) as c:
        x = uniform_residues(np.random.default_rng(5), small.q[:2], small.n)
        c.write_poly(0, x)
        d = FHEHostDriver(c)
        d.ntt(0, 2 * small.n, 2)
        d.intt(2 * small.n, 4 * small.n, 2)
        assert np.array_equal(c.read_poly(4 * small.n, 2 * small.n), x)


def test_fences_and_asynchronous_rows(ed):
    lib, h, n = ed.lib, ed.h, ed.n
    c = ed.ct(NQ)
    ed.put_ct(0, c)
    buf = ed.ctx.staging.get("edge_rows", 2 * n)
    L.check(lib.afhe_read_poly_rows_async(h, ed.slot(0) + n, 2 * n, 2, n, buf.ctypes.data_as(L.P64)), "rows_async")
    f = ed.ctx.fence()
    ed.ctx.fence_wait(f)
    assert np.array_equal(buf[:n], c[0][n:2 * n]) and np.array_equal(buf[n:], c[0][3 * n:4 * n])
    # fence ids increase; a fence whose event was reused still waits and returns
    later = [ed.ctx.fence() for _ in range(70)]
    assert later == list(range(f + 1, f + 71))
    ed.ctx.fence_wait(f)
    ed.ctx.fence_wait(later[-1])
    assert lib.afhe_fence_wait(h, later[-1] + 1) == L.E_ARG
    assert lib.afhe_fence(h, C.POINTER(C.c_uint64)()) == L.E_ARG
    assert lib.afhe_read_poly_rows_async(h, SLOTS * ed.PW - n, n, 2, n, buf.ctypes.data_as(L.P64)) == L.E_RANGE
