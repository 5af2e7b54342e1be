"""Benchmark: encrypted IVF-PQ queries/s on the small interactive configuration.

Workload: 4,096 x 64 float32 database (32 Gaussian clusters), IVF n_list 32,
PQ 8 x 256, B 64, nprobe 4; CKKS N = 2^13, scale 2^40, 3 x 50-bit Q primes +
1 x 60-bit special prime (alpha 1). Seeded synthetic data and keys.

A step is one batch of `--batch` queries through the server's operator chain
(stages 1/1b, then stage 3 after the client's list selection).

* value: queries / device time of the server stages, inputs (encrypted
  queries) resident in HBM, CUDA events on the context stream.
* e2e: the same protocol through the C ABI with host buffers: host->device
  copy of the encrypted queries, stage 1/1b, device->host of the compacted
  coarse distances, client decrypt + selection, stage 3, device->host of the
  candidate distances, client decrypt + top-k, timed on the context stream.
  The K steps stream as groups of half a batch (--e2e-groups) whose client
  and server work overlap (Workload.run_host_stream): while the server runs
  one group's stage 1, the client selects for the group before it and ranks
  the one before that. The client decrypts on a device context of its own.
  Every step's queries are copied in and its results out.
* --impl reference: the oracle restatement of the same chain on the host's
  cores (one query per process), see oracle/chain.py.

Multi-GPU: replicas only (independent queries per rank, no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def clocks_sampler(stop: threading.Event, out: list, gpu: int):
    cmd = ["nvidia-smi", f"--id={gpu}", "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits"]
    while not stop.is_set():
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=5)
            if r.returncode == 0 and r.stdout.strip():
                out.append([x.strip() for x in r.stdout.strip().split(",")])
        except Exception:
            pass
        stop.wait(0.2)


def summarize_clocks(samples):
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = sorted(float(s[0]) for s in samples if s[0].replace(".", "").isdigit())
    mx = max((float(s[1]) for s in samples if s[1].replace(".", "").isdigit()), default=None)
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for s in samples for i in range(4) if len(s) > 3 + i and s[3 + i] == "Active"})
    return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons}


def run_ours(args, rank: int, world: int):
    import ctypes as C

    import numpy as np
    import torch

    from anns_fhe_b200._lib import P64
    from anns_fhe_b200.replicas import aggregate, query_seed
    from anns_fhe_b200.workloads import LARGE, SMALL, Workload

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    spec = LARGE if args.workload == "large" else SMALL
    if args.full_level:
        import dataclasses
        spec = dataclasses.replace(spec, eval_level=None)
    if args.batch <= 0:
        # small: the one-kernel key switch runs one CTA per ciphertext and one
        # CTA per SM at a time, so two full waves per launch; large: 256
        # queries per launch
        args.batch = 256 if spec is LARGE else 2 * torch.cuda.get_device_properties(dev).multi_processor_count
    if args.lanes <= 0:
        args.lanes = args.batch
    # twice the records of a step: the serving leg keeps one tick's queries
    # in flight while admitting the next
    wl = Workload(spec, max_queries=2 * args.batch, lanes=args.lanes, device=dev, tune=not args.no_tune)
    stream = torch.cuda.ExternalStream(wl.ctx.lib.afhe_stream(wl.ctx.h), device=dev)
    iqm = wl.iqm
    recs = wl.records[:args.batch]
    Q = wl.queries(args.batch, seed=query_seed(1000, rank))
    # client work done once: encrypted queries on the host (pinned) for e2e
    wl.encrypt_queries(Q, recs)
    n = wl.params.n
    Lw = wl.params.L * n
    host_cts = []
    for r in recs:
        host_cts.append([wl.ctx.read_poly(o, Lw) for o in (*r.ct_query, *r.ct_dim)])
    pinned = [[torch.from_numpy(a).pin_memory() for a in cts] for cts in host_cts]

    def select(rs):
        wl.select(rs)

    def device_step():
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        iqm.stage1_coarse(recs)
        e1.record(stream)
        select(recs)                      # client (outside the server time)
        e2.record(stream)
        iqm.stage3_fine(recs)
        e3.record(stream)
        e3.synchronize()
        return e0.elapsed_time(e1) + e2.elapsed_time(e3)

    # the client decrypts on a context of its own, so that its device work
    # does not queue behind the server's next group
    groups = max(1, args.e2e_groups)
    group = -(-args.batch // groups)
    dec = wl.client.decryptor(group * max(1, iqm.n_res))
    host_np = [[t.numpy() for t in cts] for cts in pinned]

    def e2e_stream(steps):
        """`steps` batches of queries streamed in groups (Workload.run_host_stream)
        over all records; one timed region. With one group per batch, batch
        after batch without overlap (Workload.run_host_pipelined)."""
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        if groups > 1:
            _, h2d, d2h = wl.run_host_stream(wl.records, host_np, dec, steps * args.batch, group)
        else:
            h2d = d2h = 0
            for _ in range(steps):
                _, a, b = wl.run_host_pipelined(recs, host_np, dec, 1)
                h2d, d2h = h2d + a, d2h + b
        eb.record(stream)
        eb.synchronize()
        return ea.elapsed_time(eb), h2d // steps, d2h // steps

    for _ in range(args.warmup):
        device_step()
    lib = wl.ctx.lib
    dist = world > 1
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    stop, samples = threading.Event(), []
    th = threading.Thread(target=clocks_sampler, args=(stop, samples, dev), daemon=True)
    th.start()
    launches0 = lib.afhe_kernel_launches()
    ms = [device_step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    launches = lib.afhe_kernel_launches() - launches0
    stop.set()
    th.join()
    total_ms = sum(ms)
    e2e_stream(max(1, args.warmup // 2) + 1)
    e2e = [e2e_stream(args.steps)]
    e2e_ms = e2e[0][0]
    # replicas: all ranks' queries over the slowest rank's time
    total_ms, queries = aggregate(total_ms, args.batch * args.steps)
    e2e_ms, _ = aggregate(e2e_ms, args.batch * args.steps)
    dec.close()
    line = {
        "metric": "encrypted IVF-PQ queries/s (batched server, interactive protocol)",
        "value": queries / (total_ms / 1e3),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded Gaussian mixture database, seeded keys)",
        "config": {"workload": wl.spec.name, "queries_per_step": args.batch, "lanes": args.lanes,
                   "eval_level": wl.spec.eval_level or wl.params.L,
                   "tuning": ({str(k): [int(v.fused), v.chunk] for k, v in wl.tuning.items()} if wl.tuning
                              else None),
                   "nprobe": wl.spec.nprobe, "n_list": wl.spec.n_list, "ring_degree": n,
                   "q_limbs": wl.params.L, "p_limbs": wl.params.K,
                   "l2": f"no flush; inputs larger than L2: {args.batch * 2 * Lw * 8 / 1e6:.0f} MB of query "
                         f"ciphertexts and {wl.ctx.scratch_bytes() / 1e9:.1f} GB of lane scratch per step "
                         f"(L2 126 MB)"},
        "e2e": {"value": queries / (e2e_ms / 1e3), "unit": "queries/s",
                "h2d_bytes_per_step": e2e[0][1], "d2h_bytes_per_step": e2e[0][2], "groups": groups,
                "streamed": groups > 1, "queries_per_group": group},
        "clocks": summarize_clocks(samples),
        "gpu_launches": int(launches),
    }
    if not args.skip_serving:
        line["serving"] = serve_leg(args, wl, [[t.numpy() for t in cts] for cts in pinned], rank)
    if spec is SMALL:
        line["roofline"] = ks_roofline(wl.params, args.lanes)
    else:
        line["config"]["setup_s"] = wl.setup_s
    wl.close()
    if world == 1 and rank == 0 and not args.skip_cpu and spec is SMALL:
        from oracle.chain import cpu_reference_rate
        ref = cpu_reference_rate(steps=1)
        line["cpu_baseline"] = ref["cpu_baseline"]
    return line


def serve_leg(args, wl, host_cts, rank: int):
    """Latency beside throughput: the plain path (one ciphertext per launch,
    one query at a time) and the continuous-batching server on a seeded
    Poisson trace, both from the same encrypted queries through the C ABI,
    host buffers in and out, client decryption included."""
    from anns_fhe_b200.serving import (Request, ServingLoop, WorkloadBackend, make_trace, percentile,
                                       poisson_arrivals, summarize)
    import gc
    be = WorkloadBackend(wl, pool=host_cts)
    be.prepare()
    plain = be.with_lanes(1)
    nplain = max(1, args.plain_queries)
    ServingLoop(plain, max_inflight=1, defer_from=None).run([Request(0, 0.0, 0)], realtime=False)     # warm-up
    svc = []
    for i in range(nplain):
        c = ServingLoop(plain, max_inflight=1, defer_from=None).run([Request(i, 0.0, i % len(host_cts))],
                                                                     realtime=False)[0]
        svc.append(c.service * 1e3)
    plain_qps = 1e3 * nplain / sum(svc)
    rate = args.serve_rate or 10.0 * plain_qps
    warm = make_trace(poisson_arrivals(rate, 0.3, seed=query_seed_base(rank) + 1), pool=len(host_cts), seed=1)
    defer = defer_arg(args.defer_from)
    ServingLoop(be, defer_from=defer).run(warm)
    trace = make_trace(poisson_arrivals(rate, args.serve_seconds, seed=query_seed_base(rank) + 2),
                       pool=len(host_cts), seed=2)
    gc.collect()
    loop = ServingLoop(be, defer_from=defer)
    done = loop.run(trace)
    s = summarize(done)
    return {"plain": {"queries_per_s": plain_qps, "p50_ms": percentile(svc, 50), "p99_ms": percentile(svc, 99),
                      "queries": nplain, "lanes": 1, "inflight": 1},
            "served": {"offered_qps": rate, "queries_per_s": s["qps"], "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"],
                       "completed": s["completed"], "offered": len(trace), "seconds": args.serve_seconds,
                       "ticks": loop.ticks, "lanes": be.lanes, "max_inflight": loop.capacity,
                       "defer_from": defer, "deferred_ticks": sum(loop.deferred),
                       "trace": f"seeded Poisson arrivals at {rate:.0f} queries/s (10x the plain path's rate "
                                f"unless --serve-rate is given)"}}


def serve_sweep(rates, seconds: float, batch: int, workload: str = "small", mixed: bool = False,
                plain_queries: int = 32, defer_from: int | None = 64):
    """Serving driver: the plain path's latency and rate, then the served loop
    at each offered rate for `seconds` (seeded Poisson arrivals); one JSON
    line per rate. `mixed` is the serving trace's query mix: levels drawn
    from 6..12 and nprobe from {4, 8, 16, 32}, on the large configuration,
    with a 120 GB admission budget."""
    import numpy as np
    import torch

    from anns_fhe_b200.serving import (Request, ServingLoop, WorkloadBackend, make_trace, percentile,
                                       poisson_arrivals, summarize)
    from anns_fhe_b200.workloads import LARGE, SMALL, Workload
    spec = LARGE if workload == "large" else SMALL
    levels = list(range(6, spec.num_q + 1)) if mixed else None
    nprobes = [4, 8, 16, 32] if mixed else None
    wl = Workload(spec, max_queries=2 * batch, lanes=batch, levels=levels, max_nprobe=32 if mixed else None)
    pool_levels = (np.random.default_rng(5).integers(6, spec.num_q + 1, batch).tolist() if mixed else None)
    enc = WorkloadBackend(wl, wl.queries(batch, seed=77), levels=pool_levels)
    be = WorkloadBackend(wl, pool=[[torch.from_numpy(a).pin_memory().numpy() for a in cts] for cts in enc.pool],
                         pool_levels=enc.pool_level)
    be.prepare()
    budget = 120e9 if mixed else None
    plain = be.with_lanes(1)
    ptrace = make_trace(np.zeros(plain_queries + 1), pool=batch, seed=9, nprobes=nprobes)
    ServingLoop(plain, max_inflight=1, defer_from=None).run([ptrace[0]], realtime=False)
    svc = [ServingLoop(plain, max_inflight=1, defer_from=None).run([r], realtime=False)[0].service * 1e3
           for r in ptrace[1:]]
    print(json.dumps({"path": "plain", "workload": spec.name, "mixed": mixed,
                      "queries_per_s": 1e3 * len(svc) / sum(svc), "p50_ms": percentile(svc, 50),
                      "p99_ms": percentile(svc, 99), "queries": len(svc)}), flush=True)
    ServingLoop(be, budget_bytes=budget, defer_from=defer_from).run(
        make_trace(poisson_arrivals(max(rates[0], 1.0), 2.0, seed=1), pool=batch, seed=1, nprobes=nprobes))
    for r in rates:
        trace = make_trace(poisson_arrivals(r, seconds, seed=int(r * 10)), pool=batch, seed=int(r * 10) + 1,
                           nprobes=nprobes)
        __import__("gc").collect()
        loop = ServingLoop(be, budget_bytes=budget, defer_from=defer_from)
        s = summarize(loop.run(trace))
        s.update(path="served", offered_qps=r, offered=len(trace), ticks=loop.ticks, seconds=seconds,
                 max_inflight=loop.capacity, defer_from=defer_from,
                 deferred_ticks=sum(loop.deferred))
        print(json.dumps(s), flush=True)
    wl.close()


def defer_arg(v: int) -> int | None:
    """--defer-from: a tick's results are taken during the next tick when it
    ran at least this many queries (-1: never)."""
    return None if v < 0 else v


def query_seed_base(rank: int) -> int:
    return 5000 + 1000 * rank


# ncu --set full of ks_fused_kernel, 148 ciphertexts of N = 8192, 3 + 1 limbs
# per launch (summary under profiles/)
KS_TRAFFIC_148 = 106.9e6 + 68.4e6
KS_FMAHEAVY_FRAC_148 = 0.580


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ks_roofline(params, lanes: int, reps: int = 20, level: int = 0):
    """The dominant kernel (ks_fused_kernel: the one-kernel key switch, ~88% of
    device time in the launch list) timed alone: one rotation step of `lanes`
    ciphertexts at the top level per launch (one launch per call), five batches
    cycled so the inputs (> L2 in total) stream from HBM.
    Algorithmic bytes per launch: per ciphertext c0 and c1 read and both
    outputs written (4 x L limbs of N words), plus the rotation key read once
    (2 x dnum x (L + K) limbs)."""
    import ctypes as C

    import numpy as np
    import torch

    from anns_fhe_b200._lib import CtRef
    from anns_fhe_b200.driver import FheContext
    p = params
    n, K = p.n, p.K
    L = level or p.L
    w = L * n
    nbuf = 5
    kw = p.key_words()
    ctx = FheContext(p, poly_words=(nbuf + 1) * lanes * 2 * w, key_words=kw, max_batch=lanes,
                     device=torch.cuda.current_device())
    rng = np.random.default_rng(3)
    allp = p.q + p.p
    key = np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for _ in range(2 * p.dnum) for q in allp])
    ctx.write_key(0, key)
    ctx.lib.afhe_add_rotation_key(ctx.h, 1, 0)
    limb = np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for q in p.q[:L]])
    for i in range((nbuf + 1) * lanes * 2):
        ctx.write_poly(i * w, limb)

    def refs(first):
        arr = (CtRef * lanes)()
        for i in range(lanes):
            arr[i].c0_offset, arr[i].c1_offset = (first + 2 * i) * w, (first + 2 * i + 1) * w
        return arr
    ins = [refs(b * lanes * 2) for b in range(nbuf)]
    out = refs(nbuf * lanes * 2)
    st = torch.cuda.ExternalStream(ctx.lib.afhe_stream(ctx.h), device=torch.cuda.current_device())
    for b in range(nbuf):
        ctx.lib.afhe_eval_rotate_batch(ctx.h, ins[b], out, lanes, 1, L)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.lib.afhe_kernel_launches()
    e0.record(st)
    for r in range(reps):
        ctx.lib.afhe_eval_rotate_batch(ctx.h, ins[r % nbuf], out, lanes, 1, L)
    e1.record(st)
    e1.synchronize()
    launches = ctx.lib.afhe_kernel_launches() - l0
    ms = e0.elapsed_time(e1) / launches
    ctx.close()
    key_bytes = 2 * p.dnum * (L + K) * n * 8
    bytes_per_launch = lanes * 4 * w * 8 + key_bytes
    achieved = bytes_per_launch / (ms * 1e-3) / 1e9
    peak, src = load_peaks()
    traffic = None
    if (n, L, K) == (8192, 3, 1):
        # DRAM read + write of one 148-ciphertext launch from the ncu capture
        # of this shape under profiles/: 175.3 MB, of which the key (read
        # once) is key_bytes; the rest grows with the ciphertexts.
        traffic = (KS_TRAFFIC_148 - key_bytes) * lanes / 148 + key_bytes
    return {"bound": "hbm", "kernel": f"ks_fused_kernel (rotation key switch, N={n}, {L} limbs, {lanes} ciphertexts/launch)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": src, "traffic": traffic, "ms_per_launch": ms,
            "algorithmic_bytes_per_launch": bytes_per_launch,
            # the kernel is bound by the integer multiply pipe, not HBM (same capture)
            "int_pipe": {"pipe": "fmaheavy (IMAD)", "frac": KS_FMAHEAVY_FRAC_148}}


def profile_ks(lanes: int, level: int = 0):
    """Profiling driver: the roofline measurement of the key-switch kernel alone
    (five warm-up launches, then 20 measured) at `level` limbs (default: all)."""
    from anns_fhe_b200.driver import CkksParams
    from anns_fhe_b200.workloads import SMALL as spec
    p = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
    print(json.dumps(ks_roofline(p, lanes, level=level)))


def profile_step(nq: int, workload: str = "small", lanes: int = 0):
    """Profiling driver: one warm step, then one measured step of `nq` queries.
    Prints the kernel-launch counts an ncu launch list needs (-s / -c)."""
    import numpy as np  # noqa: F401

    from anns_fhe_b200.workloads import LARGE, SMALL, Workload
    wl = Workload(LARGE if workload == "large" else SMALL, max_queries=nq, lanes=lanes or nq)
    lib = wl.ctx.lib
    recs = wl.records[:nq]
    wl.encrypt_queries(wl.queries(nq, seed=7), recs)

    def step():
        wl.iqm.stage1_coarse(recs)
        wl.select(recs)
        wl.iqm.stage3_fine(recs)
        wl.ctx.sync()
    step()
    a = lib.afhe_kernel_launches()
    t = time.time()
    step()
    print(f"WARM_LAUNCHES={a} STEP_LAUNCHES={lib.afhe_kernel_launches() - a} step_s={time.time() - t:.3f}")
    wl.close()


def profile_host(batch: int = 296, steps: int = 5):
    """Profiling driver for the end-to-end path on the host: (1) one batch
    through the protocol one phase at a time, each phase followed by a
    synchronisation, its wall time averaged over `steps` steps; (2) the
    streamed end-to-end run (Workload.run_host_stream) under cProfile, the
    host functions with the most own time. One JSON line each."""
    import cProfile
    import pstats

    import numpy as np
    import torch

    from anns_fhe_b200._lib import P64, check
    from anns_fhe_b200.workloads import SMALL, Workload
    wl = Workload(SMALL, max_queries=2 * batch, lanes=batch)
    iqm, n = wl.iqm, wl.params.n
    recs = wl.records[:batch]
    wl.encrypt_queries(wl.queries(batch, seed=1000), recs)
    Lw = wl.params.L * n
    host = [[torch.from_numpy(wl.ctx.read_poly(o, Lw)).pin_memory().numpy() for o in (*r.ct_query, *r.ct_dim)]
            for r in recs]
    dec = wl.client.decryptor(batch * max(1, iqm.n_res))
    phases: dict = {}

    def mark(name, t0):
        wl.ctx.sync()
        t = time.perf_counter()
        phases[name] = phases.get(name, 0.0) + (t - t0) * 1e3
        return t

    def phased_step():
        t = time.perf_counter()
        for r, cts in zip(recs, host):
            for off, a in zip((*r.ct_query, *r.ct_dim), cts):
                check(wl.ctx.lib.afhe_write_poly_async(wl.ctx.h, off, a.ctypes.data_as(P64), a.size), "write")
        t = mark("h2d", t)
        iqm.stage1_coarse(recs)
        t = mark("stage1", t)
        box = iqm.read_results("compact", recs, staged=True)[:, 0]
        t = mark("d2h_coarse", t)
        coef = dec.decrypt_host_batch_coef(box, 1)
        t = mark("client_decrypt_coarse", t)
        vals = dec.enc.decode_real_batch(coef, iqm.out_scale, iqm.coarse_slots_needed())
        for r, c in zip(recs, iqm.coarse_from_slots(vals)):
            r.probes = list(np.argsort(c, kind="stable")[:wl.spec.nprobe])
        t = mark("client_decode_select", t)
        iqm.stage3_fine(recs)
        t = mark("stage3", t)
        fbox = iqm.read_results("dists", recs, staged=True)
        t = mark("d2h_dists", t)
        wl._group_topk(recs, (fbox, wl.ctx.fence(), 0), dec)
        mark("client_decrypt_decode_topk", t)

    for _ in range(2):
        phased_step()
    phases.clear()
    for _ in range(steps):
        phased_step()
    total = sum(phases.values()) / steps
    print(json.dumps({"profile": "phases", "queries_per_step": batch, "ms": {k: round(v / steps, 2) for k, v in
                      phases.items()}, "total_ms": round(total, 2), "queries_per_s": round(batch / total * 1e3, 1)}),
          flush=True)
    wl.run_host_stream(wl.records, host, dec, 2 * batch, batch // 2)
    pr = cProfile.Profile()
    t = time.perf_counter()
    pr.enable()
    wl.run_host_stream(wl.records, host, dec, steps * batch, batch // 2)
    pr.disable()
    wall = time.perf_counter() - t
    st = pstats.Stats(pr)
    rows = sorted(st.stats.items(), key=lambda kv: -kv[1][2])[:15]
    print(json.dumps({"profile": "stream_cprofile", "queries": steps * batch, "wall_s": round(wall, 3),
                      "queries_per_s_under_profiler": round(steps * batch / wall, 1),
                      "top_own_time": [{"fn": f"{os.path.basename(k[0])}:{k[1]}({k[2]})", "calls": v[1],
                                        "own_ms": round(v[2] * 1e3, 1), "cum_ms": round(v[3] * 1e3, 1)}
                                       for k, v in rows]}), flush=True)
    wl.close()


def ref_shape(seconds: float = 10.0, cts: int = 128, reps: int = 10):
    """Reference-shape driver: key switches per second at the reference's own
    shape (N = 16384, 11 Q primes of which 10 in use, 4 P primes, alpha 4:
    three digits). CPU: the reference's HLS key switch compiled from its
    sources (oracle/_ref), one process per host core, timed first so the
    spawned pool never sits beside a CUDA context. GPU: this repository's
    batched key switch on the same primes, `cts` ciphertexts per launch, as
    afhe_eval_rotate_batch by one step (the automorphism is folded into the
    key switch's loads; c0's automorphism and add are the only extra work),
    CUDA events on the context stream. One JSON line."""
    import ctypes as C

    import numpy as np

    from anns_fhe_b200._lib import CtRef, check
    from anns_fhe_b200.driver import CkksParams, FheContext, find_ntt_primes
    q = find_ntt_primes(14, 60, 1)
    q += find_ntt_primes(14, 45, 10, q)
    p = find_ntt_primes(14, 60, 4, q)
    from oracle.refshape import PARTS, SIZE_QL, reference_key_switch_rate
    cpu = reference_key_switch_rate(q, p, seconds=seconds)

    import torch
    prm = CkksParams(14, q, p, 4)
    n, sq = prm.n, SIZE_QL
    assert prm.dnum == PARTS
    w = sq * n
    ctx = FheContext(prm, poly_words=4 * cts * w, key_words=prm.key_words(), max_batch=cts)
    rng = np.random.default_rng(5)
    allp = prm.q + prm.p
    ctx.write_key(0, np.concatenate([rng.integers(0, x, n, dtype=np.uint64) for _ in range(2 * prm.dnum)
                                     for x in allp]))
    check(ctx.lib.afhe_add_rotation_key(ctx.h, 1, 0), "add_rotation_key")
    for z in range(2 * cts):
        ctx.write_poly(z * w, np.concatenate([rng.integers(0, x, n, dtype=np.uint64) for x in prm.q[:sq]]))
    ins, outs = (CtRef * cts)(), (CtRef * cts)()
    for z in range(cts):
        ins[z].c0_offset, ins[z].c1_offset = 2 * z * w, (2 * z + 1) * w
        outs[z].c0_offset, outs[z].c1_offset = (2 * cts + 2 * z) * w, (2 * cts + 2 * z + 1) * w
    stream = torch.cuda.ExternalStream(ctx.lib.afhe_stream(ctx.h))

    def launch():
        check(ctx.lib.afhe_eval_rotate_batch(ctx.h, ins, outs, cts, 1, sq), "eval_rotate_batch")
    for _ in range(3):
        launch()
    ctx.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ctx.close()
    gpu = cts * reps / (ms / 1e3)
    print(json.dumps({"driver": "reference shape", "unit": "key switches/s",
                      "shape": f"N = 16384, {sq} of 11 Q limbs + 4 P limbs, {PARTS} digits of 4",
                      "gpu": {"value": gpu, "ciphertexts_per_launch": cts, "launches": reps,
                              "ms_per_launch": ms / reps},
                      "cpu_reference": cpu, "gpu_over_cpu": gpu / cpu["value"]}), flush=True)


def profile_ntt(polys: int, log_n: int = 13, reps: int = 10):
    """Profiling driver: batched in-place NTT / INTT over `polys` polynomials of
    4 limbs (the key switch's shape), forward then inverse, `reps` each."""
    import ctypes as C

    import numpy as np
    import torch

    from anns_fhe_b200._lib import P64
    from anns_fhe_b200.driver import CkksParams, FheContext
    prm = CkksParams.generate(log_n, 3, 50, 1, 60, 1)
    n, limbs = prm.n, 4
    ctx = FheContext(prm, poly_words=polys * limbs * n, key_words=1024)
    rng = np.random.default_rng(1)
    limb_data = np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for q in prm.q + prm.p])
    for b in range(polys):
        ctx.write_poly(b * limbs * n, limb_data)
    offs = (C.c_uint64 * polys)(*[b * limbs * n for b in range(polys)])
    lib = ctx.lib
    st = torch.cuda.ExternalStream(lib.afhe_stream(ctx.h))
    for inv in (0, 1):
        lib.afhe_ntt_batch(ctx.h, C.cast(offs, P64), polys, limbs, inv)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            lib.afhe_ntt_batch(ctx.h, C.cast(offs, P64), polys, limbs, inv)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gb = 2 * polys * limbs * n * 8 / 1e9
        print(f"log_n={log_n} inverse={inv} {polys}x{limbs} limbs: {ms * 1e3:.1f} us per launch, {gb / (ms * 1e-3):.0f} GB/s")
    ctx.close()


def ntt_config(reps: int = 5):
    """Primitive microbenchmark: forward and inverse NTT over 64 ciphertexts x
    2 polynomials x 24 limbs at N = 2^16 (one batched call each), CUDA events
    on the context stream; algorithmic bytes = every limb read and written once."""
    import torch

    from anns_fhe_b200.primitives import NttBatch
    wl = NttBatch()
    st = torch.cuda.ExternalStream(wl.ctx.lib.afhe_stream(wl.ctx.h))
    peak, src = load_peaks()
    out = {"workload": "ntt_64ct_x2_x24limbs_N65536", "algorithmic_bytes_per_call": wl.algorithmic_bytes(),
           "butterflies_per_call": wl.butterflies()}
    for inv in (False, True):
        for _ in range(2):
            wl.transform(inv)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = wl.ctx.lib.afhe_kernel_launches()
        e0.record(st)
        for _ in range(reps):
            wl.transform(inv)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = wl.algorithmic_bytes() / (ms * 1e-3) / 1e9
        out["inverse" if inv else "forward"] = {
            "ms_per_call": ms, "launches_per_call": (wl.ctx.lib.afhe_kernel_launches() - l0) / reps,
            "achieved_gbs": gbs, "frac_hbm": gbs / peak, "peak_gbs": peak, "peak_source": src,
            "gbutterflies_per_s": wl.butterflies() / (ms * 1e-3) / 1e9}
    wl.close()
    print(json.dumps(out))


def ks_config(reps: int = 3):
    """Batched hybrid key switching and rotation at N = 2^16 (24 + 8 limbs,
    dnum 3): 32 ciphertexts at seeded levels 8-24, rotate-and-sum by 2^0..2^14,
    then rescale; one batched call per level group and step."""
    import torch

    from anns_fhe_b200.primitives import KeySwitchBatch
    wl = KeySwitchBatch()
    st = torch.cuda.ExternalStream(wl.ctx.lib.afhe_stream(wl.ctx.h))
    wl.run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = wl.ctx.lib.afhe_kernel_launches()
    e0.record(st)
    for _ in range(reps):
        wl.run()
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    peak, src = load_peaks()
    byts = wl.algorithmic_bytes_per_step() * len(wl.steps)
    gbs = byts / (ms * 1e-3) / 1e9
    print(json.dumps({"workload": "ks_rotate_sum_32ct_N65536_L24_K8_dnum3", "levels": wl.levels,
                      "level_groups": len(wl.groups()), "ms_per_chain": ms,
                      "key_switches_per_chain": wl.key_switch_count(),
                      "key_switches_per_s": wl.key_switch_count() / (ms * 1e-3),
                      "launches_per_chain": (wl.ctx.lib.afhe_kernel_launches() - l0) / reps,
                      "algorithmic_bytes_per_chain": byts, "achieved_gbs": gbs, "frac_hbm": gbs / peak,
                      "peak_gbs": peak, "peak_source": src}))
    wl.close()


def run_reference(args, rank: int, world: int):
    from oracle.chain import cpu_reference_rate
    # one untimed query per worker at most: each takes seconds on a core
    return cpu_reference_rate(steps=args.steps, warmup=min(args.warmup, 1), n_gpus=args.gpus)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0, help="queries per step (default: 2 x the SM count)")
    ap.add_argument("--lanes", type=int, default=0, help="ciphertexts per launch (default: the batch)")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--skip-serving", action="store_true", help="omit the serving leg")
    ap.add_argument("--e2e-groups", type=int, default=2,
                    help="e2e: groups of queries whose client and server work overlap (1: one after the other)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner's key-switch choices")
    ap.add_argument("--workload", default="small", choices=["small", "large"],
                    help="small: 4,096 x 64, N=2^13 (default); large: 1M x 128, n_list 1024, N=2^15")
    ap.add_argument("--plain-queries", type=int, default=16, help="queries timed on the plain path")
    ap.add_argument("--serve-rate", type=float, default=0.0, help="served trace rate (default: 10x plain)")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="served trace length")
    ap.add_argument("--serve-sweep", default="", help="serving driver: comma-separated offered rates (queries/s)")
    ap.add_argument("--mixed", action="store_true", help="serving driver: mixed query levels 6-12 and nprobe")
    ap.add_argument("--defer-from", type=int, default=64,
                    help="serving: ticks of at least this many queries hand their results to the client "
                         "during the next tick (-1: never)")
    ap.add_argument("--full-level", action="store_true",
                    help="evaluate at the queries' own level instead of the workload's eval_level")
    ap.add_argument("--ntt-config", action="store_true", help="NTT microbenchmark driver (64 ct x 2 x 24 limbs, N=2^16)")
    ap.add_argument("--ks-config", action="store_true", help="batched key-switch driver (32 ct, N=2^16, dnum 3)")
    ap.add_argument("--profile-step", type=int, default=0, help="profiling driver: queries per step")
    ap.add_argument("--profile-host", action="store_true",
                    help="profiling driver: end-to-end phases and the streamed run's host hotspots")
    ap.add_argument("--ref-shape", action="store_true",
                    help="key switches/s at the reference's own shape: its compiled HLS code on the host "
                         "cores beside the batched GPU key switch")
    ap.add_argument("--ref-seconds", type=float, default=10.0, help="--ref-shape: seconds per host process")
    ap.add_argument("--profile-ntt", type=int, default=0, help="profiling driver: polynomials per NTT launch")
    ap.add_argument("--profile-ks", type=int, default=0, help="profiling driver: ciphertexts per key-switch launch")
    ap.add_argument("--level", type=int, default=0, help="limbs for --profile-ks (default: all)")
    ap.add_argument("--log-n", type=int, default=13, help="ring degree for --profile-ntt")
    args = ap.parse_args()
    if args.ntt_config:
        return ntt_config()
    if args.ks_config:
        return ks_config()
    if args.serve_sweep:
        return serve_sweep([float(x) for x in args.serve_sweep.split(",")], args.serve_seconds,
                           args.batch or (256 if args.workload == "large" else 296), args.workload, args.mixed,
                           args.plain_queries, defer_arg(args.defer_from))
    if args.profile_step:
        return profile_step(args.profile_step, args.workload, args.lanes)
    if args.profile_host:
        return profile_host()
    if args.ref_shape:
        return ref_shape(args.ref_seconds)
    if args.profile_ntt:
        return profile_ntt(args.profile_ntt, args.log_n)
    if args.profile_ks:
        return profile_ks(args.profile_ks, args.level)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)))
        return
    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    line = run_ours(args, rank, world)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
