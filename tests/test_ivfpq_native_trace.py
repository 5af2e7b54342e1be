"""The native stage driver issues the Python stage driver's operators.

anns_fhe_b200/csrc/ivfpq.cu (afhe_ivfpq_stage1 / afhe_ivfpq_stage3) restates
InteractiveQueryManager.stage1_coarse / stage3_fine (anns_fhe_b200/query.py,
native=False) in C++. Both are compared here without a GPU: ivfpq.cu is
linked with stubs of the batched operators that record every call
(tests/ivfpq_trace_stub.cu), and the Python manager runs against a fake
library that records the same calls in the same format. Each recorded line
holds the operator, its limb count, its ciphertext and plaintext offsets in
order, its rotation, and the key-switch options in force. The sequences must
be identical: same operators, same batches, same order, same tuning.

The GPU tests check the residues themselves (test_gpu_ivfpq_native.py)."""
import ctypes as C
import os
import shutil
import subprocess
import zlib

from types import SimpleNamespace

import numpy as np
import pytest

from anns_fhe_b200 import build as _build
from anns_fhe_b200 import _lib as L
from anns_fhe_b200.query import InteractiveQueryManager, QueryRecord, QueryShape

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def trace(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("trace") / "libivfpq_trace.so")
    cmd = [nvcc, "-O1", "-std=c++17", *_build.ARCH_FLAGS, "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", "-I", _build.INCLUDE, "-I", _build.CSRC, "-o", out,
           os.path.join(_build.CSRC, "ivfpq.cu"), os.path.join(HERE, "ivfpq_trace_stub.cu")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    lib = C.CDLL(out)
    lib.trace_ctx_new.restype, lib.trace_ctx_new.argtypes = C.c_void_p, [C.c_uint32, C.c_uint32, C.c_uint32]
    lib.trace_ctx_free.argtypes = [C.c_void_p]
    lib.trace_count.restype = C.c_uint32
    lib.trace_line.restype, lib.trace_line.argtypes = C.c_char_p, [C.c_uint32]
    for name in ("afhe_ivfpq_create", "afhe_ivfpq_destroy", "afhe_ivfpq_set_centroids", "afhe_ivfpq_set_level_masks",
                 "afhe_ivfpq_set_prefix_mask", "afhe_ivfpq_set_list", "afhe_ivfpq_set_lanes", "afhe_ivfpq_set_tuning",
                 "afhe_ivfpq_set_units", "afhe_ivfpq_set_diagonals", "afhe_ivfpq_set_scratch",
                 "afhe_ivfpq_stage1", "afhe_ivfpq_stage3"):
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = L.SIGNATURES[name]
    return lib


class FakeLib:
    """The batched operators the Python stage driver calls, recorded in the
    stub's format; key-switch options come from the fake context."""

    def __init__(self, ctx):
        self.ctx, self.log = ctx, []

    @staticmethod
    def _refs(r, n):
        return "".join(f" {r[i].c0_offset}:{r[i].c1_offset}" for i in range(n)) + " |"

    @staticmethod
    def _words(p, n):
        return "".join(f" {int(p[i])}" for i in range(n)) + " |"

    def _head(self, name, limbs, ks):
        s = f"{name} {limbs}"
        if ks:
            s += (f" fused={self.ctx.opts[L.OPT_KS_FUSED]} chunk={self.ctx.opts[L.OPT_CHUNK]}"
                  f" ept={self.ctx.opts[L.OPT_KS_EPT]} slice={self.ctx.opts[L.OPT_KS_SLICE]}"
                  f" fmin={self.ctx.opts[L.OPT_FUSED_MIN]}")
        return s + " |"

    def afhe_eval_add_batch(self, h, a, b, d, n, limbs):
        self.log.append(self._head("add", limbs, False) + self._refs(a, n) + self._refs(b, n) + self._refs(d, n))
        return 0

    def afhe_eval_sub_batch(self, h, a, b, d, n, limbs):
        self.log.append(self._head("sub", limbs, False) + self._refs(a, n) + self._refs(b, n) + self._refs(d, n))
        return 0

    def afhe_eval_add_plain_batch(self, h, a, pt, d, n, limbs):
        self.log.append(self._head("add_plain", limbs, False) + self._refs(a, n) + self._words(pt, n)
                        + self._refs(d, n))
        return 0

    def afhe_eval_copy_batch(self, h, a, d, n, limbs):
        self.log.append(self._head("copy", limbs, False) + self._refs(a, n) + self._refs(d, n))
        return 0

    def afhe_eval_sub_plain_batch(self, h, a, pt, d, n, limbs):
        self.log.append(self._head("sub_plain", limbs, False) + self._refs(a, n) + self._words(pt, n) + self._refs(d, n))
        return 0

    def afhe_eval_mult_plain_rescale_batch(self, h, a, pt, d, n, limbs):
        self.log.append(self._head("mult_plain", limbs, False) + self._refs(a, n) + self._words(pt, n)
                        + self._refs(d, n))
        return 0

    def afhe_eval_mult_relin_rescale_batch(self, h, a, b, d, n, limbs):
        self.log.append(self._head("square", limbs, True) + self._refs(a, n) + self._refs(b, n) + self._refs(d, n))
        return 0

    def afhe_eval_rotate_batch(self, h, a, d, n, rot, limbs):
        self.log.append(self._head("rotate", limbs, True) + f" {rot} |" + self._refs(a, n) + self._refs(d, n))
        return 0

    def afhe_eval_rotate_accumulate_batch(self, h, a, acc, n, rot, limbs):
        self.log.append(self._head("rot_acc", limbs, True) + f" {rot} |" + self._refs(a, n) + self._refs(acc, n))
        return 0

    def afhe_automorphism_batch(self, h, src, gal, dst, n, limbs):
        self.log.append(self._head("automorphism", limbs, False) + self._words(src, n) + self._words(gal, n)
                        + self._words(dst, n))
        return 0

    def afhe_eval_rotate_steps_batch(self, h, a, d, steps, n, limbs):
        self.log.append(self._head("rotate_steps", limbs, True) + self._words(steps, n) + self._refs(a, n)
                        + self._refs(d, n))
        return 0

    def afhe_rescale_batch(self, h, a, d, n, limbs):
        self.log.append(self._head("rescale", limbs, False) + self._refs(a, n) + self._refs(d, n))
        return 0

    def afhe_eval_diag_inner_batch(self, h, out, n, src, nb, upt, ugal, first, stride, limbs, acc):
        s = self._head("diag_inner", limbs, False) + f" nb={nb} stride={stride} acc={acc} |"
        s += self._refs(out, n) + self._refs(src, n * nb)
        for j in range(n):
            s += "".join(f" {int(upt[k])}@{int(ugal[k])}" for k in range(first[j], first[j + 1])) + " ;"
        self.log.append(s)
        return 0

    def afhe_eval_mac_plain_batch(self, h, out, first, n, g, t, limbs, acc):
        s = self._head("mac", limbs, False) + f" acc={acc} |" + self._refs(out, n)
        for j in range(n):
            for k in range(first[j], first[j + 1]):
                s += f" [{g[k].src.c0_offset}:{g[k].src.c1_offset}"
                s += "".join(f" {t[x].pt}@{t[x].galois}" for x in range(g[k].first_term, g[k].first_term + g[k].n_terms))
                s += "]"
            s += " ;"
        self.log.append(s)
        return 0


class FakeCtx:
    def __init__(self, lanes):
        self.h = None
        self.max_batch = lanes
        self.opts = {L.OPT_KS_FUSED: 1, L.OPT_CHUNK: 0, L.OPT_KS_EPT: 8, L.OPT_KS_SLICE: 13, L.OPT_FUSED_MIN: 18}

    def set_option(self, option, value):
        self.opts[option] = value

    def get_option(self, option):
        return self.opts[option]


class Choice:
    def __init__(self, fused, chunk, ept=8, slice=13, fused_min=0):
        self.fused, self.chunk, self.ept, self.slice, self.fused_min = fused, chunk, ept, slice, fused_min


def build_manager(rng, *, D, n_list, slots, L_top, lanes, compaction, eval_level, levels, tuning, ctx_lanes):
    """An InteractiveQueryManager with the state its stages read, placed at
    arbitrary distinct offsets (nothing is encoded)."""
    sh = QueryShape(D=D, n_list=n_list, slots=slots, nprobe=2, top_k=4, scale=2.0 ** 30, compaction=compaction,
                    eval_level=eval_level)
    m = object.__new__(InteractiveQueryManager)
    ctx = FakeCtx(ctx_lanes)
    m.ctx, m.sh, m.lanes, m.L, m.native = ctx, sh, lanes, L_top, False
    m.p = SimpleNamespace(log_n=(2 * slots).bit_length() - 1, n=2 * slots)
    m.lib = FakeLib(ctx)
    m._nh, m._nh_key, m._nh_ver = None, None, 0
    nxt = iter(range(1000, 10 ** 9, 7))
    m.pt_centroid_cts = [next(nxt) for _ in range(sh.n_coarse)]
    m.pt_centroids = m.pt_centroid_cts[0]
    m.levels = sorted({min(lv, eval_level or lv) for lv in levels})
    if compaction == "diagonal":
        return build_diagonal(m, rng, nxt, levels, tuning)
    m._onehot, m._stride, m._prefix_lv = {}, {}, {}
    B = sh.B
    for lv in m.levels:
        if compaction == "reference":
            m._onehot[lv] = [next(nxt) for _ in range(n_list)]
        else:
            m._stride[lv] = next(nxt)
        for cnt in range(1, B + 1):
            m._prefix_lv[(cnt, lv)] = next(nxt)
    m.batches = []
    vid = 0
    for c in range(n_list):
        out = []
        for _ in range(int(rng.integers(0, 4))):
            cnt = int(rng.integers(1, B + 1))
            out.append((next(nxt), cnt, list(range(vid, vid + cnt))))
            vid += cnt
        m.batches.append(out)
    m._first_batch = np.concatenate([[0], np.cumsum([len(b) for b in m.batches])]).astype(int).tolist()
    nb = m._first_batch[-1]
    # packed chain: the candidates' norm plaintexts per level (expanded distances)
    m._norms = {lv: [next(nxt) for _ in range(nb)] for lv in m.levels} if compaction == "packed" else {}
    m.work = [dict(diff=(next(nxt), next(nxt)), sq=(next(nxt), next(nxt)), tmp=(next(nxt), next(nxt)),
                   sel=(next(nxt), next(nxt))) for _ in range(lanes)]
    m.cmp = ([[(next(nxt), next(nxt)) for _ in range(n_list - 1)] for _ in range(lanes)]
             if compaction == "reference" and n_list > 1 else [])
    m.n_res = 8
    m._tuning = {lv: Choice(*t) for lv, t in tuning.items()}
    m._opt_now = None
    m._fused_ok = True
    recs = []
    for i in range(6):
        res = [(next(nxt), next(nxt)) for _ in range(m.n_res)]
        recs.append(QueryRecord((next(nxt), next(nxt)), (next(nxt), next(nxt)), (next(nxt), next(nxt)), res[0],
                                results=res, level=int(rng.choice([0] + list(levels))),
                                norm=(next(nxt), next(nxt)) if compaction == "packed" else None))
    for r in recs:
        r.probes = [int(c) for c in rng.choice(n_list, size=int(rng.integers(1, 4)), replace=False)]
    return m, recs


def build_diagonal(m, rng, nxt, levels, tuning):
    """The diagonal chain's state: units of up to `slots` candidates (at most
    two per list), per level the centroid and unit diagonals (D plaintexts
    `lv N` words apart) and norms, the inner-product pool, records with
    their baby-step ciphertexts."""
    sh = m.sh
    n = 2 * sh.slots
    m.units, m.list_units, m._ucnt, m._gal_cache = [], [], [], {}
    vid = 0
    for c in range(sh.n_list):
        us = []
        for _ in range(int(rng.integers(0, 3))):
            cnt = int(rng.integers(1, sh.slots + 1))
            us.append(len(m.units))
            m.units.append((c, list(range(vid, vid + cnt))))
            m._ucnt.append(cnt)
            vid += cnt
        m.list_units.append(us)
    m._diag = {}
    for lv in m.levels:
        base = next(nxt) * 1000
        cent = [base + i * lv * n for i in range(sh.D)]
        pts = np.array([base + (1 + u) * sh.D * lv * n + i * lv * n for u in range(len(m.units))
                        for i in range(sh.D)], dtype=np.uint64)
        m._diag[lv] = dict(cent=cent, cnorm=next(nxt), pts=pts,
                           norms=np.array([next(nxt) for _ in m.units], dtype=np.uint64))
    m._inner = [(next(nxt), next(nxt)) for _ in range(InteractiveQueryManager.inner_pool(m.lanes, sh.n2))]
    m._query_levels = set(levels)
    m._bcnt, m.batches, m.cmp, m.work = [], [], [], []
    m.n_res = 8
    m._tuning = {lv: Choice(*t) for lv, t in tuning.items()}
    m._opt_now = None
    m._fused_ok = True
    recs = []
    for i in range(6):
        res = [(next(nxt), next(nxt)) for _ in range(m.n_res)]
        recs.append(QueryRecord((next(nxt), next(nxt)), (next(nxt), next(nxt)), (next(nxt), next(nxt)), res[0],
                                results=res, level=int(rng.choice([0] + list(levels))),
                                norm=(next(nxt), next(nxt)), baby=[(next(nxt), next(nxt)) for _ in range(sh.n1 - 1)]))
    for r in recs:
        r.probes = [int(c) for c in rng.choice(sh.n_list, size=int(rng.integers(1, 4)), replace=False)]
    return m, recs


def run_native(trace, m, recs, L_top, n, ctx_lanes, stage):
    """Register the manager's state through its own code (what the product
    runs) with the stubbed library, then run the stage natively."""
    ctx = trace.trace_ctx_new(L_top, n, ctx_lanes)
    try:
        m.lib, m.ctx.h, m._nh = trace, ctx, None
        h = m._native_handle()
        arr, keep = m._native_queries(recs, probes=stage == 3)
        rc = (trace.afhe_ivfpq_stage1 if stage == 1 else trace.afhe_ivfpq_stage3)(h, arr, len(recs))
        log = [trace.trace_line(i).decode() for i in range(trace.trace_count())]
        assert rc == 0, log[-3:]
        m.close_native()
        return log
    finally:
        trace.trace_ctx_free(ctx)


CASES = {
    "reference_mixed_levels": dict(D=8, n_list=4, slots=64, L_top=6, lanes=3, compaction="reference",
                                   eval_level=None, levels=[6, 5, 4], tuning={6: (1, 2, 16, 13, 3), 5: (0, 3), 4: (1, 1),
                                                                             3: (0, 2), 2: (1, 3, 16)}),
    "reference_one_lane": dict(D=8, n_list=5, slots=64, L_top=5, lanes=1, compaction="reference", eval_level=None,
                               levels=[5], tuning={}),
    "packed_eval_level": dict(D=8, n_list=20, slots=64, L_top=7, lanes=4, compaction="packed", eval_level=4,
                              levels=[7, 6], tuning={4: (1, 4, 8, 12), 3: (0, 2), 2: (1, 4)}),
    "packed_mixed_levels": dict(D=4, n_list=30, slots=32, L_top=6, lanes=5, compaction="packed", eval_level=None,
                                levels=[6, 5, 3], tuning={5: (1, 5), 4: (1, 1)}),
    "diagonal_mixed_levels": dict(D=16, n_list=40, slots=64, L_top=5, lanes=9, compaction="diagonal",
                                  eval_level=None, levels=[5, 3, 2], tuning={}),
    "diagonal_eval_level": dict(D=64, n_list=50, slots=64, L_top=6, lanes=16, compaction="diagonal", eval_level=2,
                                levels=[6, 4], tuning={2: (1, 8, 8, 12), 1: (0, 4)}),
    # 32 baby steps: the generic sums of products
    "diagonal_generic": dict(D=1024, n_list=20, slots=1024, L_top=4, lanes=32, compaction="diagonal",
                             eval_level=3, levels=[4], tuning={}),
}


@pytest.mark.parametrize("stage", [1, 3])
@pytest.mark.parametrize("case", list(CASES))
def test_native_driver_issues_the_python_drivers_operators(trace, case, stage):
    kw = CASES[case]
    rng = np.random.default_rng(zlib.crc32(case.encode()))
    ctx_lanes = kw["lanes"] + 2
    m, recs = build_manager(rng, ctx_lanes=ctx_lanes, **kw)
    py = m.lib
    if stage == 1:
        m.stage1_coarse(recs)
    else:
        m.stage3_fine(recs)
    want = py.log
    assert want, "the Python driver issued nothing"
    m.ctx.opts = {L.OPT_KS_FUSED: 1, L.OPT_CHUNK: 0, L.OPT_KS_EPT: 8, L.OPT_KS_SLICE: 13, L.OPT_FUSED_MIN: 18}
    got = run_native(trace, m, recs, kw["L_top"], 2 * kw["slots"], ctx_lanes, stage)
    for i, (a, b) in enumerate(zip(got, want)):
        assert a == b, f"call {i} differs:\n native {a[:300]}\n python {b[:300]}"
    assert len(got) == len(want)


def test_native_driver_rejects_bad_arguments(trace):
    ctx = trace.trace_ctx_new(6, 128, 4)
    try:
        h = C.c_void_p()
        bad = [L.IvfpqShape(6, 4, 64, 2, 0, 0),        # D not a power of two
               L.IvfpqShape(8, 4, 32, 2, 0, 0),        # slots != N / 2
               L.IvfpqShape(8, 9, 64, 2, 0, 0),        # centroids do not fit one ciphertext
               L.IvfpqShape(8, 4, 64, 9, 0, 0),        # more lanes than the context
               L.IvfpqShape(4, 300, 64, 2, 1, 0),      # packed: n_coarse > D
               L.IvfpqShape(8, 4, 64, 2, 0, 7)]        # eval_level above L
        for s in bad:
            assert trace.afhe_ivfpq_create(ctx, C.byref(s), C.byref(h)) != 0
        s = L.IvfpqShape(8, 4, 64, 2, 0, 0)
        assert trace.afhe_ivfpq_create(ctx, C.byref(s), C.byref(h)) == 0
        q = (L.IvfpqQuery * 1)()
        assert trace.afhe_ivfpq_stage1(h, q, 1) != 0          # lanes and centroids not registered
        assert trace.afhe_ivfpq_set_list(h, 4, None, None, 0) != 0   # list out of range
        trace.afhe_ivfpq_destroy(h)
    finally:
        trace.trace_ctx_free(ctx)
