"""Host-side helpers of the query chain, on the CPU: the ctypes arrays the
batched entry points take, the grouping of rotations into power-of-two
steps, the centring of decrypted residues, and the schedules of the
end-to-end protocol in groups (pipelined and streamed)."""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.ckks import centred_coefficients, crt_centered
from anns_fhe_b200.query import InteractiveQueryManager as IQM


@pytest.mark.parametrize("m", [0, 1, 7, 296])
def test_ref_and_offset_arrays(m):
    rng = np.random.default_rng(m)
    pairs = [(int(a), int(b)) for a, b in rng.integers(0, 2**40, (m, 2))]
    for src in (pairs, np.array(pairs, dtype=np.uint64).reshape(m, 2)):
        p = IQM._refs(src)
        assert isinstance(p, C.POINTER(L.CtRef))
        assert [(p[i].c0_offset, p[i].c1_offset) for i in range(m)] == pairs
    offs = [int(x) for x in rng.integers(0, 2**50, m)]
    for src in (offs, np.array(offs, dtype=np.uint64)):
        p = IQM._offs(src)
        assert [p[i] for i in range(m)] == offs


class _Recorder:
    """Stands in for the query manager: records the batched rotations."""

    def __init__(self):
        self.calls = []

    def _rotate(self, cts, r, limbs):
        self.calls.append(([tuple(int(x) for x in c) for c in cts], r, limbs))


def _grouped_by_definition(items):
    """eval_rotate's steps (fhe_host_driver.cpp:361-404) for every item,
    grouped highest power first, positive shifts before negative ones."""
    items = [(ct, s) for ct, s in items if s]
    calls = []
    if not items:
        return calls
    top = max(abs(s) for _, s in items).bit_length()
    for b in range(top - 1, -1, -1):
        for sign in (1, -1):
            sub = [ct for ct, s in items if (s > 0) == (sign > 0) and (abs(s) >> b) & 1]
            if sub:
                calls.append((sub, sign * (1 << b), 3))
    return calls


def test_rotate_grouped_matches_its_definition():
    rng = np.random.default_rng(5)
    for trial in range(30):
        m = int(rng.integers(0, 60))
        items = [((int(rng.integers(0, 10**6)), int(rng.integers(0, 10**6))), int(rng.integers(-200, 201)))
                 for _ in range(m)]
        rec = _Recorder()
        IQM._rotate_grouped(rec, items, 3)
        assert rec.calls == _grouped_by_definition(items), trial


@pytest.mark.parametrize("level", [1, 2])
def test_centred_coefficients(level):
    from anns_fhe_b200.driver import find_ntt_primes
    q = find_ntt_primes(10, 50, 2)
    rng = np.random.default_rng(level)
    n = 1024
    limbs = np.concatenate([rng.integers(0, qi, (4, n), dtype=np.uint64) for qi in q[:level]], axis=1)
    limbs[0, 0] = q[0] // 2            # the largest value kept positive
    limbs[0, 1] = q[0] // 2 + 1        # the smallest one moved down
    got = centred_coefficients(limbs, q, level)
    want = np.stack([crt_centered(row, q[:level]).astype(np.float64) for row in limbs])
    assert np.array_equal(got, want)


class _FakeStreamWorkload:
    """Stands in for Workload in run_host_stream / run_host_pipelined: the
    group steps are recorded, and each record slice's use is checked."""

    def __init__(self):
        self.log = []
        self.in_use = set()

    def _group_stage1(self, part, hp, tag):
        ids = tuple(id(r) for r in part)
        assert not (set(ids) & self.in_use), "a record reused while its group is in flight"
        self.in_use |= set(ids)
        self.log.append(("stage1", [r.qid for r in part], tag))
        for r, h in zip(part, hp):
            r.payload = h
        return ("box", "fence", 10 * len(part))

    def _group_stage3(self, part, coarse, dec, tag):
        assert coarse[2] == 10 * len(part)
        self.log.append(("stage3", [r.qid for r in part], tag))
        return ("fbox", "ffence", 1)

    def _group_topk(self, part, fine, dec):
        self.log.append(("topk", [r.qid for r in part]))
        self.in_use -= {id(r) for r in part}
        return [[r.payload] for r in part], 2


class _Rec:
    def __init__(self, qid):
        self.qid = qid


@pytest.mark.parametrize("total,group,slices", [(14, 2, 4), (9, 4, 3), (1, 3, 3), (12, 3, 5)])
def test_stream_schedule(total, group, slices):
    """run_host_stream: group g's stage 1 is enqueued before the client
    selects for g - 1 and ranks g - 2; three groups at most are in flight,
    each on its own slice of the records; results come back in query order,
    query i being host entry i mod len(host)."""
    from anns_fhe_b200.workloads import Workload
    fake = _FakeStreamWorkload()
    recs = [_Rec(i) for i in range(slices * group)]
    host = [f"q{i}" for i in range(5)]
    tops, h2d, d2h = Workload.run_host_stream(fake, recs, host, None, total, group)
    G = -(-total // group)
    assert tops == [[host[i % len(host)]] for i in range(total)]
    assert h2d == 10 * total and d2h == G * (1 + 2)
    kinds = [e[0] for e in fake.log]
    assert kinds.count("stage1") == kinds.count("stage3") == kinds.count("topk") == G
    # the order of the software pipeline
    want = []
    for it in range(G + 2):
        if it < G:
            want.append("stage1")
        if 0 <= it - 1 < G:
            want.append("stage3")
        if 0 <= it - 2 < G:
            want.append("topk")
    assert kinds == want
    assert not fake.in_use
    with pytest.raises(ValueError):
        Workload.run_host_stream(fake, recs[:2 * group], host, None, total, group)


def test_pipelined_groups_schedule():
    """run_host_pipelined: every group's stage 1 first, then each group's
    selection and stage 3, then each group's ranking."""
    from anns_fhe_b200.workloads import Workload
    fake = _FakeStreamWorkload()
    recs = [_Rec(i) for i in range(7)]
    tops, h2d, d2h = Workload.run_host_pipelined(fake, recs, [f"q{i}" for i in range(7)], None, 3)
    assert tops == [[f"q{i}"] for i in range(7)]
    assert [e[0] for e in fake.log] == ["stage1"] * 3 + ["stage3"] * 3 + ["topk"] * 3
    assert [e[1] for e in fake.log[:3]] == [[0, 1, 2], [3, 4, 5], [6]]


def test_nearest_lists_is_the_stable_argsort_prefix():
    from anns_fhe_b200.workloads import nearest_lists
    rng = np.random.default_rng(3)
    for trial in range(20):
        rows, lists = int(rng.integers(1, 40)), int(rng.integers(1, 64))
        coarse = rng.integers(0, 5 if trial % 2 else 10**6, (rows, lists)).astype(np.float64)   # ties when small
        nprobes = [int(rng.integers(1, lists + 1)) for _ in range(rows)]
        got = nearest_lists(coarse, nprobes)
        for r in range(rows):
            assert got[r] == list(np.argsort(coarse[r], kind="stable")[:nprobes[r]])
    assert nearest_lists(np.zeros((0, 4)), []) == []
