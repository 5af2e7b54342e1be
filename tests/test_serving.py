"""Serving loop scheduling on the CPU, with a fake backend that records calls.

Checks the properties the GPU serving path relies on: every request
completes once; a query runs stage 1 in the tick that admits it and stage 3
in the next one; the HBM budget caps the queries in flight; arrivals are
admitted in order; requests that arrive while others are in flight share
their ticks (the mix); the Poisson trace has the requested rate.
"""
import numpy as np
import pytest

from anns_fhe_b200.serving import (Request, ServingLoop, make_trace, percentile, poisson_arrivals, summarize)


class Rec:
    def __init__(self, i):
        self.i = i
        self.probes = []
        self.vids = []


class FakeBackend:
    def __init__(self, records=8, lanes=4, bytes_per_query=100):
        self.records = [Rec(i) for i in range(records)]
        self.lanes = lanes
        self.bytes_per_query = bytes_per_query
        self.log = []
        self.payload = {}
        self.busy = set()      # records whose query's results are not yet on the host

    def upload(self, rec, req):
        assert rec.i not in self.busy, "record reused while its query is in flight"
        self.busy.add(rec.i)
        self.payload[rec.i] = req.payload

    def coarse(self, recs):
        self.log.append(("coarse", [r.i for r in recs]))

    def fine(self, recs):
        self.log.append(("fine", [r.i for r in recs]))
        assert all(r.probes for r in recs), "stage 3 before selection"

    def ticks(self):
        """The log grouped by tick: a tick runs stage 1 (if any) then stage 3 (if any)."""
        out = []
        for kind, ids in self.log:
            if kind.startswith("receive") or kind.startswith("request"):
                continue
            if kind == "fine" and out and "coarse" in out[-1] and "fine" not in out[-1]:
                out[-1]["fine"] = ids
            else:
                out.append({kind: ids})
        return out

    def request(self, kind, recs):
        # the copy is enqueued: the records may be reused from here on
        self.log.append(("request-" + kind, [r.i for r in recs]))
        if kind == "dists":
            self.busy -= {r.i for r in recs}
        return {"kind": kind, "ids": [r.i for r in recs], "payload": [self.payload[r.i] for r in recs],
                "taken": False}

    def receive(self, h):
        assert not h["taken"], "a handle received twice"
        h["taken"] = True
        self.log.append(("receive-" + h["kind"], h["ids"]))
        return {"box": np.zeros((len(h["ids"]), 2, 4), dtype=np.uint64), "ids": h["ids"], "payload": h["payload"]}

    def select(self, recs, got):
        assert got["ids"] == [r.i for r in recs]
        for r in recs:
            r.probes = [self.payload[r.i]]

    def topk(self, recs, got):
        assert got["ids"] == [r.i for r in recs]
        return [[p] for p in got["payload"]]


def test_every_request_completes_in_two_ticks():
    be = FakeBackend(records=6, lanes=3)
    loop = ServingLoop(be)
    trace = [Request(i, 0.0, 100 + i) for i in range(10)]
    done = loop.run(trace, realtime=False)
    assert sorted(c.qid for c in done) == list(range(10))
    # the result is the request's own (payload carried through the record)
    assert all(c.topk == [100 + c.qid] for c in done)
    # admission in arrival order, at most `lanes` per tick, in flight <= records
    admitted = [a for a, _ in loop.tick_log]
    assert all(a <= 3 for a in admitted) and sum(admitted) == 10
    assert all(a + f <= 6 for a, f in loop.tick_log)
    # a query admitted at tick t finishes at tick t + 1
    assert loop.tick_log[0] == (3, 0)
    assert all(f == a for (a, _), (_, f) in zip(loop.tick_log, loop.tick_log[1:]))


def test_budget_caps_inflight():
    be = FakeBackend(records=16, lanes=16, bytes_per_query=1000)
    loop = ServingLoop(be, budget_bytes=4500)
    assert loop.capacity == 4
    done = loop.run([Request(i, 0.0, i) for i in range(9)], realtime=False)
    assert len(done) == 9
    assert all(a + f <= 4 for a, f in loop.tick_log)
    with pytest.raises(ValueError):
        ServingLoop(be, budget_bytes=10)


def test_mix_stage1_and_stage3_share_ticks():
    be = FakeBackend(records=8, lanes=2)
    loop = ServingLoop(be)
    loop.run([Request(i, 0.0, i) for i in range(6)], realtime=False)
    ticks = be.ticks()
    assert len(ticks) == loop.ticks
    mixed = [k for k in ticks if "coarse" in k and "fine" in k]
    assert mixed, "no tick ran stage 1 of new queries beside stage 3 of earlier ones"
    for k in mixed:
        assert not set(k["coarse"]) & set(k["fine"])


def test_realtime_latency_and_order():
    be = FakeBackend(records=4, lanes=4)
    loop = ServingLoop(be)
    arr = np.array([0.0, 0.001, 0.002, 0.010, 0.011])
    done = loop.run(make_trace(arr, pool=3, seed=1), realtime=True)
    assert len(done) == 5
    for c in done:
        assert c.done >= c.arrival and c.admitted >= c.arrival - 1e-9
    s = summarize(done)
    assert s["completed"] == 5 and s["p99_ms"] >= s["p50_ms"] >= 0


def test_trace_mixed_probes():
    tr = make_trace(np.arange(200) * 0.01, pool=5, seed=3, nprobes=[4, 8, 16, 32])
    assert {r.nprobe for r in tr} == {4, 8, 16, 32}
    assert all(0 <= r.payload < 5 for r in tr)
    assert [r.nprobe for r in tr] == [r.nprobe for r in make_trace(np.arange(200) * 0.01, pool=5, seed=3,
                                                                   nprobes=[4, 8, 16, 32])]


def test_poisson_rate_and_percentile():
    t = poisson_arrivals(200.0, 20.0, seed=4)
    assert np.all(np.diff(t) > 0) and t[-1] < 20.0
    assert abs(len(t) / 20.0 - 200.0) < 15.0
    assert np.array_equal(t, poisson_arrivals(200.0, 20.0, seed=4))
    assert percentile([1, 2, 3, 4], 50) == 2 and percentile([1, 2, 3, 4], 99) == 4


def test_results_taken_next_tick_behind_its_stage1():
    """A tick's results are requested (copies enqueued) at its end and taken
    by the client in the next tick, after that tick's stage 1 is launched.
    Each kind's handle is taken before the next request of the same kind, so
    one staging buffer per kind suffices."""
    be = FakeBackend(records=8, lanes=2)
    loop = ServingLoop(be, defer_from=0)
    done = loop.run([Request(i, 0.0, i) for i in range(7)], realtime=False)
    assert len(done) == 7
    open_req = {}
    for kind, ids in be.log:
        if kind.startswith("request-"):
            k = kind[len("request-"):]
            assert k not in open_req, f"a second {k} request before the first was taken"
            open_req[k] = ids
        elif kind.startswith("receive-"):
            assert open_req.pop(kind[len("receive-"):]) == ids
    assert not open_req
    # a tick is [stage 1] [take the previous results] [stage 3] [requests]:
    # the stage 1 of a tick is launched before the client takes anything
    kinds = [k.split("-")[0] for k, _ in be.log]
    for a, b in zip(kinds, kinds[1:]):
        if b == "coarse":
            assert a == "request"
        if b == "receive":
            assert a in ("coarse", "request", "receive")


@pytest.mark.parametrize("defer_from", [None, 5])
def test_small_ticks_take_results_at_once(defer_from):
    """With defer_from=None every tick's results are taken at its end; with a
    threshold, ticks that ran fewer queries take them at once and larger ones
    during the next tick, after its stage 1 is launched. Every request still
    completes once."""
    be = FakeBackend(records=8, lanes=3)
    loop = ServingLoop(be, defer_from=defer_from)
    done = loop.run([Request(i, 0.0, i) for i in range(9)], realtime=False)
    assert sorted(c.qid for c in done) == list(range(9))
    assert len(loop.deferred) == len(loop.tick_log)
    for deferred, (a, f) in zip(loop.deferred, loop.tick_log):
        assert deferred == (defer_from is not None and a + f >= defer_from)
    if defer_from is not None:
        assert any(loop.deferred) and not all(loop.deferred)
    # a tick whose results were taken at once: its requests are followed by
    # their receives directly
    kinds = [k for k, _ in be.log]
    reqs = [i for i, k in enumerate(kinds) if k.startswith("request") and
            (i + 1 == len(kinds) or not kinds[i + 1].startswith("request"))]
    assert len(reqs) == len(loop.tick_log)
    for i, deferred in zip(reqs, loop.deferred):
        if not deferred:
            assert kinds[i + 1].startswith("receive")


def test_shedding_bounds_the_queue_under_overload():
    """Requests waiting longer than shed_after are refused, the rest complete
    once; without shedding every request completes."""
    import time as _t

    class SlowBackend(FakeBackend):
        def coarse(self, recs):
            _t.sleep(0.004)
            super().coarse(recs)

    arr = np.arange(120) * 0.0005            # 2,000 requests/s for 60 ms
    be = SlowBackend(records=4, lanes=2)
    loop = ServingLoop(be, shed_after=0.01)
    done = loop.run(make_trace(arr, pool=3, seed=2), realtime=True)
    ids = [c.qid for c in done] + [r.qid for r in loop.shed]
    assert sorted(ids) == list(range(120)), "a request was lost or served twice"
    assert loop.shed, "nothing shed at 2,000 requests/s on a server of about 250"
    assert all(c.admitted - c.arrival <= 0.01 + 0.05 for c in done)     # the deadline plus about a tick
    be2 = SlowBackend(records=4, lanes=2)
    assert len(ServingLoop(be2).run(make_trace(arr[:20], pool=3, seed=2), realtime=True)) == 20
