"""Serving loop for encrypted IVF-PQ queries: continuous batching on one GPU.

The reference runs one query at a time through InteractiveQueryManager::
execute_interactive_query (cpp_host_model/src/interactive_query_manager.cpp:
279-303): stage 1/1b on the server, stage 2 on the client, stage 3 on the
server, stage 4 on the client. Here many queries are in flight. The
protocol is the one in docs/interactive_search_protocol.md:13-55.

* Admission. A request that has arrived takes a free query record. A record
  holds the device-resident ciphertexts of one query: the two encrypted
  queries at the top level and the two result ciphertexts. The number of
  records in use is capped by an HBM budget (`budget_bytes` / bytes per
  query), so a request waits on the host while the budget is spent. Evaluation
  keys and the index's plaintexts are resident for the loop's whole life.
* Ticks. Each tick launches, as batched operators on the context stream:
  - stage 1/1b for the requests admitted since the last tick;
  - stage 3 for the queries whose lists the client selected from the
    previous tick's results.
  Both kinds of results are copied to the host behind the tick's launches,
  without waiting. At the next tick, once its stage 1 is launched, the
  client waits for those copies and does its work on them: decryption (on
  a device context of its own, so it does not queue behind the server),
  decoding, list selection, top-k. So the GPU has the next stage 1 while
  the client works. A query's record is freed once the copy of its
  candidate distances is enqueued. A request that arrives while a tick is
  on the GPU is admitted at the next tick. Its stage 1 then shares the GPU
  with other queries' stage 3.
* Results are independent of the mix. Each ciphertext's residues are those
  of the one-ciphertext-at-a-time chain, whatever else shares its launches,
  so a query's result ciphertexts are bit-identical alone and in any mix.
* The plain path is the same loop with one lane and one query in flight.
  That is one ciphertext per launch and one query at a time, as the
  reference runs it.

Latency is measured on the host from a request's arrival time to the moment
its top-k is known, with `time.perf_counter`.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    qid: int
    arrival: float          # seconds from the start of the trace
    payload: int            # index into the backend's encrypted-query pool
    nprobe: int = 0         # lists the client will probe (0: the workload's nprobe)


@dataclass
class Completion:
    qid: int
    arrival: float
    admitted: float
    done: float
    probes: list = field(default_factory=list)
    topk: list = field(default_factory=list)
    result: np.ndarray | None = None    # limb 0 of the candidate-distance ciphertexts, if kept

    @property
    def latency(self) -> float:
        return self.done - self.arrival

    @property
    def service(self) -> float:
        """Time from admission to the top-k (no queueing)."""
        return self.done - self.admitted


def poisson_arrivals(rate: float, duration: float, seed: int) -> np.ndarray:
    """Arrival times (seconds) of a seeded Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed)
    n = max(1, int(rate * duration * 1.2) + 16)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    while t[-1] < duration:
        t = np.concatenate([t, t[-1] + np.cumsum(rng.exponential(1.0 / rate, n))])
    return t[t < duration]


def make_trace(arrivals: np.ndarray, pool: int, seed: int = 0, nprobes=None) -> list[Request]:
    """Requests at the given arrival times, each drawing a pooled encrypted
    query (and, with `nprobes`, a probe count) uniformly from a seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i, t in enumerate(arrivals):
        payload = int(rng.integers(0, pool))
        nprobe = int(nprobes[rng.integers(0, len(nprobes))]) if nprobes is not None else 0
        out.append(Request(i, float(t), payload, nprobe))
    return out


def percentile(xs, p: float) -> float:
    """Nearest-rank percentile (p in [0, 100])."""
    if not len(xs):
        return float("nan")
    s = sorted(xs)
    k = max(0, min(len(s) - 1, int(math.ceil(p / 100.0 * len(s))) - 1))
    return float(s[k])


class WorkloadBackend:
    """The server and client of a `workloads.Workload`, driven through the C ABI.

    The encrypted-query pool is held on the host. The client encrypts each
    distinct query once, and a request's admission copies its four ciphertexts
    into the record on the context stream. Results come back to the host with
    one asynchronous copy per run of consecutive records (`request`), into
    page-locked staging. The client decrypts them with its secret key on a
    device context of its own (`receive`), as in the bench's end-to-end step.
    """

    def __init__(self, wl, Q: np.ndarray | None = None, lanes: int | None = None,
                 pool: list[list[np.ndarray]] | None = None, levels=None, pool_levels=None):
        """Q: query vectors the client encrypts into the pool (query i at
        levels[i] limbs, default the top level); or `pool`: ciphertexts
        already encrypted, the host arrays of iqm.input_polys (ct_query c0,
        c1, then ct_dim c0, c1 where the chain reads it) per query, at pool_levels[i] limbs (default the top level)."""
        self.wl = wl
        self.iqm = wl.iqm
        self.lib = wl.ctx.lib
        self.h = wl.ctx.h
        self.lanes = lanes or wl.iqm.lanes
        self.records = wl.records
        self.n = wl.params.n
        Lw = wl.params.L * self.n
        self.pool: list[list[np.ndarray]] = list(pool or [])
        self.pool_level = list(pool_levels) if pool_levels is not None else [wl.params.L] * len(self.pool)
        chunk = len(wl.records)
        for c0 in range(0, 0 if Q is None else len(Q), chunk):
            part = Q[c0:c0 + chunk]
            recs = wl.records[:len(part)]
            lv = None if levels is None else list(levels[c0:c0 + chunk])
            wl.encrypt_queries(part, recs, lv)
            for r in recs:
                self.pool.append([wl.ctx.read_poly(o, w) for o, w in zip(wl.iqm.input_polys(r), wl.iqm.input_words(r))])
                self.pool_level.append(r.level)
        w = self.iqm.lvl_out * self.n
        # device bytes one in-flight query holds: its encrypted polynomials at
        # L limbs, the compacted coarse result and n_res candidate results at
        # lvl_out limbs, and (diagonal chain) its baby steps
        r0 = wl.records[0]
        self.bytes_per_query = (len(self.iqm.input_polys(r0)) * Lw + 2 * w * (1 + self.iqm.n_res)
                                + 2 * len(r0.baby) * getattr(self.iqm, "_baby_limbs", 0) * self.n) * 8
        self._dec = {"dec": None}
        self._pool_ptrs: dict = {}

    def prepare(self) -> None:
        """Make, before serving, what the loop would otherwise allocate while
        requests wait: the client's decryption context at its full size and
        the page-locked staging of both kinds of results for every record."""
        n_res = max(1, self.iqm.n_res)
        dec = self._decryptor(len(self.records) * n_res)
        dec.ctx.staging.get("dec_coef", len(self.records) * n_res * self.n)
        for kind, per in (("compact", 1), ("dists", n_res)):
            self.wl.ctx.staging.get("res_" + kind, len(self.records) * per * 2 * self.n)

    def with_lanes(self, lanes: int) -> "WorkloadBackend":
        """The same server and encrypted-query pool, `lanes` ciphertexts per launch."""
        other = object.__new__(WorkloadBackend)
        other.__dict__.update(self.__dict__)
        other.lanes = lanes
        return other

    def upload(self, rec, req) -> None:
        from . import _lib as L
        rec.level = self.pool_level[req.payload]
        rec.nprobe = req.nprobe
        ptrs = self._pool_ptrs.get(req.payload)
        if ptrs is None:          # pointers made once per pool entry (each keeps its array alive)
            ptrs = self._pool_ptrs[req.payload] = [(a.ctypes.data_as(L.P64), a.size) for a in self.pool[req.payload]]
        for off, (p, size) in zip(self.iqm.input_polys(rec), ptrs):
            L.check(self.lib.afhe_write_poly_async(self.h, off, p, size), "write_poly_async")

    def coarse(self, recs) -> None:
        lanes = self.iqm.lanes
        try:
            self.iqm.lanes = self.lanes
            self.iqm.stage1_coarse(recs)
        finally:
            self.iqm.lanes = lanes

    def fine(self, recs) -> None:
        lanes = self.iqm.lanes
        try:
            self.iqm.lanes = self.lanes
            self.iqm.stage3_fine(recs)
        finally:
            self.iqm.lanes = lanes

    def request(self, kind: str, recs) -> dict:
        """Enqueue the copy of the records' results (limb 0) to the host
        behind the work already on the context stream, without waiting; the
        handle carries what `receive` needs. The records may be reused as
        soon as this returns: later work on them is ordered after the copy."""
        box, fence = self.iqm.read_results(kind, recs, staged=True, wait=False)
        h = {"kind": kind, "box": box, "fence": fence, "count": len(recs),
             "scale": np.array([self.iqm.out_scale_at(self.iqm.level_of(r)) for r in recs])}
        if kind == "dists":     # only the result ciphertexts that hold candidates
            h["need"] = max(1, -(-max((int(r.pos[-1]) + 1 if len(r.pos) else 1) for r in recs) // self.iqm.sh.slots))
            h["vids"] = [r.vids for r in recs]     # a record's next stage 3 builds new ones
            h["pos"] = [np.asarray(r.pos, dtype=np.int64) for r in recs]
        return h

    def _decryptor(self, count: int):
        """The client's decryption context (shared by with_lanes copies),
        grown to hold `count` ciphertexts."""
        d = self._dec.get("dec")
        if d is None or d.max_count < count:
            cap = max(count, 2 * d.max_count if d else 0, self.lanes * max(1, self.iqm.n_res))
            self._dec["dec"] = d = self.wl.client.decryptor(cap)
        return d

    def receive(self, h: dict) -> dict:
        """A request's results to the client: wait for its copy, then the
        client's decryption and decoding ("vals", the slots each query
        needs: its coarse distances, or up to its last candidate), on the
        client's own context, so they do not wait for the server's work
        enqueued since the request."""
        self.wl.ctx.fence_wait(h["fence"])
        need = h.get("need", 1)
        box = h["box"][:, :need]
        if h["kind"] == "compact":
            slots = self.iqm.coarse_slots_needed()
        else:
            last = max((int(p[-1]) + 1 if len(p) else 1) for p in h["pos"])
            slots = min(self.iqm.sh.slots, last) if need == 1 else self.iqm.sh.slots
        vals = self._decryptor(box.shape[0] * box.shape[1]).decrypt_decode_host(
            box.reshape(-1, 2, self.n), np.repeat(h["scale"], need), slots)
        return dict(h, box=box, vals=vals.reshape(h["count"], -1).copy())

    def select(self, recs, got: dict) -> None:
        """Stage 2 on the host: keep the nprobe nearest lists."""
        wl = self.wl
        vals = got["vals"]
        from .workloads import nearest_lists
        for r, pr in zip(recs, nearest_lists(self.iqm.coarse_from_slots(vals),
                                             [r.nprobe or wl.spec.nprobe for r in recs])):
            r.probes = pr

    def topk(self, recs, got: dict) -> list[list[int]]:
        """Stage 4 on the host: rank the candidate distances."""
        wl = self.wl
        vids = got["vids"]
        d = got["vals"]
        from .workloads import ranked_prefix
        return [[int(v[i]) for i in top] for v, top in zip(vids, ranked_prefix(d, got["pos"], wl.spec.top_k))]


class ServingLoop:
    """Continuous batching over a backend (see the module docstring).

    backend: an object with `records`, `bytes_per_query`, `upload(rec,
    request)`, `coarse(recs)`, `fine(recs)`, `request(kind, recs)` (enqueue
    the copy of results to the host, return a handle), `receive(handle)`,
    `select(recs, got)` and `topk(recs, got)`; `WorkloadBackend` drives the
    GPU.
    budget_bytes: HBM the in-flight queries may hold (None: every record).
    max_inflight: a further cap on queries in flight (None: no cap).
    max_admit: queries admitted per tick (None: the backend's lanes).
    keep_results: keep each query's candidate-distance ciphertext.

    A tick, in order: admit arrived requests and launch their stage 1; take
    the results the previous tick requested and do the client's work on
    them while that stage 1 runs on the GPU (decryption on the client's own
    context, selections, and the top-k of finished queries); launch stage 3
    for the queries just selected; request this tick's results (copies to
    the host enqueued behind its launches). A record is freed as soon as the
    copy of its query's candidate distances is enqueued: later work on the
    record is ordered after it on the stream.
    """

    def __init__(self, backend, budget_bytes: int | None = None, max_inflight: int | None = None,
                 max_admit: int | None = None, keep_results: bool = False, defer_from: int | None = 64,
                 shed_after: float | None = None):
        """defer_from: the client takes a tick's results during the next tick
        (behind that tick's stage 1) when the tick ran at least this many
        queries (stage 1 plus stage 3), and at the end of the tick otherwise.
        Deferring keeps the GPU busy while the client works, which pays
        when ticks are large; taking them at once puts no stage-1 launch
        ahead of them, which keeps latency down when ticks are small.
        0: always defer; None: never.
        shed_after: load shedding (real-time runs): a request still waiting
        for admission this many seconds after its arrival is refused (kept
        in `shed`) instead of served late. Above the server's capacity the
        queue then stays bounded, and the completed requests' latency stays
        near shed_after plus one query's service time. None: never shed."""
        self.b = backend
        self.defer_from = defer_from
        self.shed_after = shed_after
        self.shed: list[Request] = []
        cap = len(backend.records)
        if budget_bytes is not None:
            cap = min(cap, int(budget_bytes // backend.bytes_per_query))
        if max_inflight is not None:
            cap = min(cap, max_inflight)
        if cap < 1:
            raise ValueError("the HBM budget does not hold one query")
        self.capacity = cap
        self.max_admit = max_admit or getattr(backend, "lanes", cap)
        self.keep = keep_results
        self.ticks = 0
        self.tick_log: list[tuple[int, int]] = []      # (stage-1 queries, stage-3 queries) per tick
        self.deferred: list[bool] = []                 # per tick: results taken during the next tick

    def run(self, trace: list[Request], realtime: bool = True, clock=time.perf_counter) -> list[Completion]:
        """Serve `trace` (sorted by arrival). With realtime=False every request
        counts as arrived at once (the order and mixing of a saturated
        server, used by tests); latencies are then measured from the start."""
        free = deque(self.b.records[:self.capacity])
        place = {id(r): i for i, r in enumerate(self.b.records)}
        pending = deque(sorted(trace, key=lambda r: r.arrival))
        waiting: deque = deque()
        coarse_got = None      # (entries, request handle) of the last tick's stage 1
        fine_got = None        # (entries, request handle) of the last tick's stage 3
        done: list[Completion] = []
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        while pending or waiting or coarse_got or fine_got:
            t = now()
            while pending and (not realtime or pending[0].arrival <= t):
                waiting.append(pending.popleft())
            if realtime and self.shed_after is not None:
                while waiting and t - waiting[0].arrival > self.shed_after:
                    self.shed.append(waiting.popleft())
            admit = []
            while waiting and free and len(admit) < self.max_admit:
                req = waiting.popleft()
                admit.append((req, free.popleft(), now()))
            # records in allocation order, so results come back as runs of
            # consecutive records, copied in place without waiting
            admit.sort(key=lambda e: place[id(e[1])])
            if not admit and not coarse_got and not fine_got:
                if pending:                      # idle: wait for the next arrival
                    dt = pending[0].arrival - now()
                    if dt > 0:
                        time.sleep(min(dt, 0.005))
                continue
            arecs = [rec for _, rec, _ in admit]
            for req, rec, _ in admit:
                self.b.upload(rec, req)
            if arecs:
                self.b.coarse(arecs)
            # the previous tick's results, and the client's work on them,
            # overlapping the stage 1 just launched
            selected = []
            if coarse_got:
                entries, got, taken = coarse_got
                got = got if taken else self.b.receive(got)
                self.b.select([rec for _, rec, _ in entries], got)
                selected = [(req, rec, adm, list(rec.probes)) for req, rec, adm in entries]
            if fine_got:
                entries, got, taken = fine_got
                got = got if taken else self.b.receive(got)
                tops = self.b.topk([rec for _, rec, _, _ in entries], got)
                t_done = now()
                for k, ((req, rec, adm, probes), top) in enumerate(zip(entries, tops)):
                    done.append(Completion(req.qid, req.arrival if realtime else 0.0, adm, t_done,
                                           probes, top, got["box"][k].copy() if self.keep else None))
            srecs = [rec for _, rec, _, _ in selected]
            if srecs:
                self.b.fine(srecs)
            if arecs or srecs:
                self.ticks += 1
                self.tick_log.append((len(arecs), len(srecs)))
            # copies of this tick's results to the host, behind its launches;
            # the client takes them next tick
            now_ = self.defer_from is None or len(arecs) + len(srecs) < self.defer_from
            coarse_got = (admit, self.b.request("compact", arecs), False) if arecs else None
            fine_got = (selected, self.b.request("dists", srecs), False) if srecs else None
            if arecs or srecs:
                self.deferred.append(not now_)
            if now_:
                coarse_got = coarse_got and (admit, self.b.receive(coarse_got[1]), True)
                fine_got = fine_got and (selected, self.b.receive(fine_got[1]), True)
            for rec in srecs:                    # the copy is enqueued before any reuse: the record is free
                free.append(rec)
        return done


def summarize(done: list[Completion], duration: float | None = None) -> dict:
    """p50/p99 latency (ms) and throughput of a served trace."""
    if not done:
        return {"completed": 0}
    lat = [c.latency * 1e3 for c in done]
    first = min(c.arrival for c in done)
    last = max(c.done for c in done)
    span = duration if duration is not None else max(last - first, 1e-9)
    return {"completed": len(done), "qps": len(done) / max(last - first, 1e-9), "offered_span_s": span,
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "max_ms": max(lat)}
