"""Benchmark: encrypted IVF-PQ queries/s (batched server, interactive protocol).

Headline workload (default, --workload large): the largest single-GPU
configuration, 1,000,000 x 128 float32 vectors from a 1,024-component
Gaussian mixture (sigma 0.15), IVF n_list 1024, PQ 16 x 256, nprobe 16;
CKKS N = 2^15, scale 2^40, 12 x 50-bit Q primes + 4 x 60-bit special primes,
alpha 4 (dnum 3). Queries are encrypted at 12 limbs; the server runs the
diagonal chain (baby-step giant-step inner products, depth 1) on their first
2 limbs (`eval_level` 2), which is the same message at the same scale. A
step is 256 queries through the server's operator chain (stage 1, then
stage 3 after the client's list selection). `packed_chain` is the same
configuration through the packed chain (per-batch tree sums, depth 2, 3
limbs), with its `full_level` sample (--workload large_packed makes it the
headline).

* value: queries / device time of the server stages, inputs (encrypted
  queries) resident in HBM, CUDA events on the context stream.
* e2e: the same protocol through the C ABI with host buffers: host->device
  copy of the encrypted queries, stage 1/1b, device->host of the compacted
  coarse distances, client decrypt + selection, stage 3, device->host of the
  candidate distances, client decrypt + top-k. The K steps stream as groups
  (--e2e-groups per step) whose client and server work overlap
  (Workload.run_host_stream); the client decrypts on a device context of
  its own. Every step's queries are copied in and its results out.
* roofline: the step's largest operation, the rotation key switch at the
  chain's evaluation shape, timed alone (anns_fhe_b200/profiling.py);
  roofline_inner_products: the diagonal chain's inner-product kernel.
* cpu_baseline and --impl reference: the same chain on the host's cores,
  the reference's own HLS C-simulation rebuilt at this ring degree, driven in
  FHEHostDriver's operator sequence (oracle/refchain.py), in work units of a
  query.
* secondary keys: `packed_chain` (with `full_level`: the same queries
  evaluated at their 12 limbs, a sample of 64 queries), `small` (the small interactive
  configuration: 4,096 x 64, n_list 32, nprobe 4, N = 2^13, 3 + 1 limbs,
  296 queries per step), and `serving` (p50/p99 of the plain path and of
  the continuous-batching server on a Poisson trace).

--workload small makes the small configuration the headline. The config 2,
3 and 5 drivers are --ntt-config, --ks-config and --serve-sweep;
--ref-shape times the key switch at the reference's own shape (N = 2^14,
three digits) on the GPU beside the reference's HLS key switch on the host.

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

METRIC = "encrypted IVF-PQ queries/s (batched server, interactive protocol)"


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


def spec_of(workload: str):
    """large: config 4 through the diagonal chain (the headline); large_packed:
    the same configuration through the packed chain; small: config 1."""
    from anns_fhe_b200.workloads import LARGE, LARGE_DIAG, SMALL
    return {"large": LARGE_DIAG, "large_packed": LARGE, "small": SMALL}[workload]


def default_batch(spec) -> int:
    """Queries per step: 256 per launch on the large configuration; two
    waves of the one-kernel key switch (one CTA per ciphertext per SM) on
    the small one."""
    return 256 if spec.log_n >= 15 else 296


def config_of(spec, batch: int) -> dict:
    """The workload named by what it is; the same dict on both arms."""
    n = 1 << spec.log_n
    ev = spec.eval_level or spec.num_q
    # the encrypted queries the server reads (at the evaluated limbs) and the
    # resident plaintexts it streams per step
    q_bytes = batch * (2 * ev + (2 * (ev - 1) if spec.compaction == "diagonal" else 2 * ev)) * n * 8
    streamed = ("the units' diagonal plaintexts (64 GiB resident)" if spec.compaction == "diagonal"
                else "the candidate-batch plaintexts")
    return {"workload": spec.name, "queries_per_step": batch, "n_vectors": spec.n_vectors, "d": spec.d,
            "n_list": spec.n_list, "nprobe": spec.nprobe, "pq": f"{spec.M}x{spec.K}", "top_k": spec.top_k,
            "ring_degree": n, "q_limbs": spec.num_q, "p_limbs": spec.num_p, "alpha": spec.alpha,
            "scale_bits": spec.log_scale, "chain": spec.compaction, "eval_level": spec.eval_level or spec.num_q,
            "l2": f"no flush; inputs larger than L2: {q_bytes / 1e6:.0f} MB of encrypted queries per step and "
                  f"{streamed} (L2 126 MB)"}


def time_steps(wl, recs, stream, steps: int):
    """`steps` server steps on resident queries; device ms per step (stages 1
    and 3, CUDA events on the context stream; the client's selection between
    them is outside)."""
    import torch
    iqm = wl.iqm
    out = []
    for _ in range(steps):
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        iqm.stage1_coarse(recs)
        e1.record(stream)
        wl.select(recs)
        e2.record(stream)
        iqm.stage3_fine(recs)
        e3.record(stream)
        e3.synchronize()
        out.append(e0.elapsed_time(e1) + e2.elapsed_time(e3))
    return out


def measure(args, spec, rank: int, world: int, steps: int, warmup: int, batch: int, legs: bool,
            full_level: bool = False):
    """One workload: device-only steps, the streamed end-to-end run, and (with
    legs) serving and the roofline; with full_level, the full-level sample.
    Returns the line."""
    import torch

    from anns_fhe_b200 import _lib as L
    from anns_fhe_b200.autotune import get_ntt_plan
    from anns_fhe_b200.replicas import aggregate, query_seed
    from anns_fhe_b200.workloads import Workload

    dev = int(os.environ.get("LOCAL_RANK", 0))
    lanes = args.lanes or batch
    large = spec.log_n >= 15
    # twice the records of a step: the stream keeps three groups in flight
    wl = Workload(spec, max_queries=2 * batch, lanes=lanes, device=dev, tune=not args.no_tune,
                  spare_levels=1 if full_level else 0)
    try:
        stream = torch.cuda.ExternalStream(wl.ctx.lib.afhe_stream(wl.ctx.h), device=dev)
        recs = wl.records[:batch]
        Q = wl.queries(batch, seed=query_seed(1000, rank))
        wl.encrypt_queries(Q, recs)            # client work done once: encrypted queries on the host
        host = [[torch.from_numpy(wl.ctx.read_poly(o, w)).pin_memory()
                 for o, w in zip(wl.iqm.input_polys(r), wl.iqm.input_words(r))]
                for r in recs]
        host_np = [[t.numpy() for t in cts] for cts in host]
        groups = max(1, args.e2e_groups)
        group = -(-batch // groups)
        dec = wl.client.decryptor(group * max(1, wl.iqm.n_res))

        def e2e_stream(k):
            ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ea.record(stream)
            if groups > 1:
                _, h2d, d2h = wl.run_host_stream(wl.records, host_np, dec, k * batch, group)
            else:
                h2d = d2h = 0
                for _ in range(k):
                    _, a, b = wl.run_host_pipelined(recs, host_np, dec, 1)
                    h2d, d2h = h2d + a, d2h + b
            eb.record(stream)
            eb.synchronize()
            return ea.elapsed_time(eb), h2d // k, d2h // k

        time_steps(wl, recs, stream, warmup)
        lib = wl.ctx.lib
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        stop, samples = threading.Event(), []
        th = threading.Thread(target=clocks_sampler, args=(stop, samples, dev), daemon=True)
        th.start()
        l0 = lib.afhe_kernel_launches()
        ms = time_steps(wl, recs, stream, steps)
        torch.cuda.synchronize()
        launches = lib.afhe_kernel_launches() - l0
        e2e_stream(max(1, warmup // 2) + 1)
        e2e_ms, h2d, d2h = e2e_stream(steps)
        stop.set()
        th.join()
        total_ms, queries = aggregate(sum(ms), batch * steps)
        e2e_ms, _ = aggregate(e2e_ms, batch * steps)
        dec.close()
        line = {
            "metric": METRIC, "value": queries / (total_ms / 1e3), "unit": "queries/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded Gaussian mixture database, seeded keys)",
            "config": config_of(spec, batch),
            "e2e": {"value": queries / (e2e_ms / 1e3), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "groups_per_step": groups, "queries_per_group": group,
                    "streamed": groups > 1},
            "clocks": summarize_clocks(samples),
            "gpu_launches": int(launches),
            "run": {"lanes": lanes, "setup_s": round(wl.setup_s, 1),
                    "tuning": ({str(k): [int(v.fused), v.chunk, v.ept, v.slice, v.fused_min] for k, v in wl.tuning.items()} if wl.tuning
                               else None),
                    "lane_scratch_gb": round(wl.ctx.scratch_bytes() / 1e9, 1),
                    "ks_capacity": wl.ctx.get_option(L.OPT_KS_CAPACITY),
                    "ntt_plan": get_ntt_plan(spec.log_n), "stage_driver": "native" if wl.iqm.native else "python",
                    "chain": spec.compaction, "eval_level": spec.eval_level or spec.num_q},
        }
        if full_level and not args.skip_full_level:
            line["full_level"] = full_level_leg(wl, stream, rank)
        if legs and not args.skip_serving:
            line["serving"] = serve_leg(args, wl, host_np, rank, line["value"])
    finally:
        wl.close()
    if legs:
        from anns_fhe_b200.profiling import ks_roofline, mac_roofline
        ev = spec.eval_level or spec.num_q
        line["roofline"] = ks_roofline(wl.params, lanes, level=ev, choice=(wl.tuning or {}).get(ev))
        if spec.compaction == "diagonal" and large:
            line["roofline_inner_products"] = mac_roofline(64, 16, ev)
    return line


def full_level_leg(wl, stream, rank: int, queries: int = 64):
    """The same chain evaluated at the queries' own 12 limbs: every key switch
    on 12 + 4 limbs (3 digits) and below; one warm-up and one timed step of
    `queries` queries."""
    from anns_fhe_b200.replicas import query_seed
    iqm = wl.iqm
    ev = iqm.sh.eval_level
    recs = wl.records[:queries]
    wl.encrypt_queries(wl.queries(queries, seed=query_seed(3000, rank)), recs)
    try:
        iqm.set_eval_level(None)
        time_steps(wl, recs, stream, 1)
        ms = time_steps(wl, recs, stream, 1)[0]
    finally:
        iqm.set_eval_level(ev)
    return {"value": queries / (ms / 1e3), "unit": "queries/s", "eval_level": wl.params.L,
            "queries_per_step": queries, "steps": 1, "warmup": 1, "ms_per_step": ms}


def serve_leg(args, wl, host_cts, rank: int, device_qps: float = 0.0):
    """Latency beside throughput: the plain path (one ciphertext per launch,
    one query at a time) and the continuous-batching server on a seeded
    Poisson trace, both from the same encrypted queries through the C ABI,
    host buffers in and out, client decryption included. The trace runs at
    10x the plain path's rate, or at 60% of the device-only batched rate
    (`device_qps`) where that is lower: above the server's capacity a queue
    grows for as long as the trace lasts, and its latency says nothing about
    the server (the --serve-sweep driver covers rates up to 2,000/s with
    load shedding)."""
    import gc

    from anns_fhe_b200.serving import (Request, ServingLoop, WorkloadBackend, make_trace, percentile,
                                       poisson_arrivals, summarize)
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
    cap = 0.6 * device_qps if device_qps > 0 else float("inf")
    rate = args.serve_rate or min(10.0 * plain_qps, cap)
    why = ("--serve-rate" if args.serve_rate else
           "10x the plain path's rate" if 10.0 * plain_qps <= cap else "60% of the device-only batched rate")
    warm = make_trace(poisson_arrivals(rate, 0.3, seed=5000 + 1000 * rank + 1), pool=len(host_cts), seed=1)
    defer = None if args.defer_from < 0 else args.defer_from
    ServingLoop(be, defer_from=defer).run(warm)
    trace = make_trace(poisson_arrivals(rate, args.serve_seconds, seed=5000 + 1000 * rank + 2),
                       pool=len(host_cts), seed=2)
    gc.collect()
    loop = ServingLoop(be, defer_from=defer)
    s = summarize(loop.run(trace))
    return {"plain": {"queries_per_s": plain_qps, "p50_ms": percentile(svc, 50), "p99_ms": percentile(svc, 99),
                      "queries": nplain, "lanes": 1, "inflight": 1},
            "served": {"offered_qps": rate, "queries_per_s": s["qps"], "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"],
                       "completed": s["completed"], "offered": len(trace), "seconds": args.serve_seconds,
                       "ticks": loop.ticks, "lanes": be.lanes, "max_inflight": loop.capacity,
                       "defer_from": defer, "deferred_ticks": sum(loop.deferred),
                       "trace": f"seeded Poisson arrivals at {rate:.1f} queries/s ({why})",
                       "served_over_plain_qps": s["qps"] / plain_qps}}


def cpu_baseline(workload: str, steps: int = 5) -> dict:
    """The chain on the host's cores (the reference's own code; see
    oracle/refchain.py), a bounded sample: `steps` steps of one work unit per
    core after one warm-up step."""
    from oracle.refchain import reference_rate
    r = reference_rate(workload, steps=steps, warmup=1)
    return {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}


def run_ours(args, rank: int, world: int):
    spec = spec_of(args.workload)
    batch = args.batch or default_batch(spec)
    base = None
    if world == 1 and rank == 0 and not args.skip_cpu:
        # the host processes start (spawn) before this process touches the GPU
        base = cpu_baseline(args.workload)
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    line = measure(args, spec, rank, world, args.steps, args.warmup, batch, legs=True,
                   full_level=args.workload == "large_packed")
    if base:
        line["cpu_baseline"] = base
    if args.workload == "large" and not args.skip_packed:
        # the same configuration through the packed chain (tree sums per
        # candidate batch), with its full-level sample
        pk = measure(args, spec_of("large_packed"), rank, world, args.steps, args.warmup, batch, legs=False,
                     full_level=True)
        line["packed_chain"] = {k: pk[k] for k in ("value", "unit", "ms_per_step", "e2e", "gpu_launches", "run")
                                if k in pk}
        if "full_level" in pk:
            line["packed_chain"]["full_level"] = pk["full_level"]
    if args.workload == "large" and not args.skip_small:
        small = spec_of("small")
        s = measure(args, small, rank, world, max(3, args.steps // 4), 3, default_batch(small), legs=False)
        line["small"] = {k: s[k] for k in ("value", "unit", "steps", "warmup", "ms_per_step", "config", "e2e",
                                           "gpu_launches")}
    return line


def run_reference(args):
    """The reference's own CPU implementation of the chain on all host cores,
    on this arm's config, steps and warm-up (one work unit per core per step)."""
    from oracle.refchain import reference_rate
    spec = spec_of(args.workload)
    batch = args.batch or default_batch(spec)
    r = reference_rate(args.workload, steps=args.steps, warmup=args.warmup, units_per_step=1)
    return {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "queries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded uniform residues; the cost is independent of the values)",
            "config": config_of(spec, batch),
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
# drivers for the other configurations
# ---------------------------------------------------------------------------
def serve_sweep(rates, seconds: float, batch: int, workload: str = "small", mixed: bool = False,
                plain_queries: int = 32, defer_from: int | None = 64, shed_after: float | None = None,
                max_admit: int | None = None):
    """Config 5: the plain path's latency and rate, then the served loop at
    each offered rate for `seconds` (seeded Poisson arrivals); one JSON line
    per rate. `mixed`: levels drawn from 6..12 and nprobe from {4, 8, 16, 32},
    on the large configuration, with a 120 GB admission budget. shed_after:
    requests not admitted within this many seconds of arriving are refused
    (counted as shed), which bounds the queue above capacity; max_admit:
    queries admitted per tick (default: the lanes)."""
    import gc

    import numpy as np
    import torch

    from anns_fhe_b200.serving import (ServingLoop, WorkloadBackend, make_trace, percentile, poisson_arrivals,
                                       summarize)
    from anns_fhe_b200.workloads import Workload
    spec = spec_of(workload)
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
        gc.collect()
        loop = ServingLoop(be, budget_bytes=budget, defer_from=defer_from, shed_after=shed_after,
                           max_admit=max_admit)
        s = summarize(loop.run(trace))
        s.update(path="served", offered_qps=r, offered=len(trace), ticks=loop.ticks, seconds=seconds,
                 max_inflight=loop.capacity, defer_from=defer_from, deferred_ticks=sum(loop.deferred),
                 shed=len(loop.shed), shed_after_s=shed_after, max_admit=loop.max_admit,
                 goodput_qps=s["completed"] / seconds if s.get("completed") else 0.0)
        print(json.dumps(s), flush=True)
    wl.close()


def ntt_config(reps: int = 5):
    """Config 2: forward and inverse NTT over 64 ciphertexts x 2 polynomials x
    24 limbs at N = 2^16 (one batched call each), CUDA events on the context
    stream; algorithmic bytes = every limb read and written once."""
    import torch

    from anns_fhe_b200.primitives import NttBatch
    from anns_fhe_b200.profiling import load_peaks
    from anns_fhe_b200.autotune import ntt_plan_describe, set_ntt_plan, time_ntt_plans
    wl = NttBatch()
    st = torch.cuda.ExternalStream(wl.ctx.lib.afhe_stream(wl.ctx.h))
    peak, src = load_peaks()
    # every tile plan timed (autotuner), the fastest used below
    plans = time_ntt_plans(wl.ctx, wl.polys, wl.limbs)
    best = min(plans, key=plans.get)
    set_ntt_plan(wl.params.log_n, best)
    for z in range(wl.polys):
        wl.ctx.write_poly(z * wl.w, wl.input_poly(z))
    out = {"workload": "ntt_64ct_x2_x24limbs_N65536", "algorithmic_bytes_per_call": wl.algorithmic_bytes(),
           "butterflies_per_call": wl.butterflies(), "plan": best, "plan_shape": ntt_plan_describe(16, best),
           "plans_us_per_limb_fwd_plus_inv": {str(k): round(v, 3) for k, v in plans.items()}}
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


def ks_config(reps: int = 3):
    """Config 3: batched hybrid key switching and rotation at N = 2^16 (24 + 8
    limbs, dnum 3): 32 ciphertexts at seeded levels 8-24, rotate-and-sum by
    2^0..2^14, then rescale."""
    import torch

    from anns_fhe_b200.primitives import KeySwitchBatch
    from anns_fhe_b200.profiling import load_peaks
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "large_packed", "small"],
                    help="large: 1M x 128, n_list 1024, N=2^15, diagonal chain (default); large_packed: the same "
                         "through the packed chain; small: 4,096 x 64, N=2^13")
    ap.add_argument("--batch", type=int, default=0, help="queries per step (default: 256 large, 296 small)")
    ap.add_argument("--lanes", type=int, default=0, help="ciphertexts per launch (default: the batch)")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--skip-serving", action="store_true", help="omit the serving leg")
    ap.add_argument("--skip-small", action="store_true", help="omit the small configuration's secondary line")
    ap.add_argument("--skip-full-level", action="store_true", help="omit the full-level sample")
    ap.add_argument("--skip-packed", action="store_true", help="omit the packed chain's secondary line")
    ap.add_argument("--e2e-groups", type=int, default=2,
                    help="e2e: groups of queries per step whose client and server work overlap")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner's key-switch choices")
    ap.add_argument("--plain-queries", type=int, default=16, help="queries timed on the plain path")
    ap.add_argument("--serve-rate", type=float, default=0.0, help="served trace rate (default: 10x plain)")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="served trace length")
    ap.add_argument("--defer-from", type=int, default=64,
                    help="serving: ticks of at least this many queries hand their results to the client "
                         "during the next tick (-1: never)")
    ap.add_argument("--serve-sweep", default="", help="config 5 driver: comma-separated offered rates (queries/s)")
    ap.add_argument("--mixed", action="store_true", help="--serve-sweep: mixed query levels 6-12 and nprobe")
    ap.add_argument("--shed-after", type=float, default=0.0,
                    help="--serve-sweep: refuse requests not admitted within this many seconds (0: never)")
    ap.add_argument("--serve-admit", type=int, default=0, help="--serve-sweep: queries admitted per tick")
    ap.add_argument("--ntt-config", action="store_true", help="config 2 driver (64 ct x 2 x 24 limbs, N=2^16)")
    ap.add_argument("--ks-config", action="store_true", help="config 3 driver (32 ct, N=2^16, dnum 3)")
    ap.add_argument("--ref-shape", action="store_true",
                    help="key switches/s at the reference's own shape (N=2^14, 3 digits): its HLS key switch "
                         "on the host cores beside this one on the GPU")
    args = ap.parse_args()
    if args.ntt_config:
        return ntt_config()
    if args.ref_shape:
        return ref_shape()
    if args.ks_config:
        return ks_config()
    if args.serve_sweep:
        return serve_sweep([float(x) for x in args.serve_sweep.split(",")], args.serve_seconds,
                           args.batch or default_batch(spec_of(args.workload)), args.workload, args.mixed,
                           args.plain_queries, None if args.defer_from < 0 else args.defer_from,
                           args.shed_after or None, args.serve_admit or None)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    if world > 1:
        import datetime

        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_ours(args, rank, world)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
