"""Measurement helpers and profiling drivers (the commands `profiles/` quotes).

* `ks_roofline`: the dominant operation of a query step, a rotation key
  switch over a batch of ciphertexts at the chain's evaluation shape, timed
  alone with CUDA events on the context stream; its algorithmic bytes and
  the achieved fraction of the HBM peak.
* drivers for ncu captures, each a plain program whose launches are easy to
  count: `python -m anns_fhe_b200.profiling ks|ntt|step|host|dispatch ...`.

Algorithmic bytes of one rotation key switch per ciphertext: c0 and c1 read,
both outputs written (4 x l limbs of N words); the rotation key (2 x dnum x
(l + K) limbs, the digits this level reads) once per launch.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# DRAM traffic and integer-pipe use of the key switch from ncu captures of the
# current kernels (`--set full`, clocks not locked), per (N, l, K, slice): the
# traffic of one launch sequence per ciphertext (its scratch and I/O grow with
# the ciphertexts), the key's bytes read once, the kernel, and the busiest
# integer pipe's utilisation. The captures are summarised under profiles/.
KS_CAPTURES: dict = {
    (8192, 3, 1, 13): {"kernel": "ks_fused_kernel<13, 1>", "ciphertexts": 148, "dram_bytes": 175.3e6,
                       "pipe": "fmaheavy (IMAD)", "util": 0.580},
    # clusters of 4 CTAs of 2^13-value slices, one per SM; 37 clusters ran as
    # two waves (33 resident at once)
    (32768, 3, 4, 13): {"kernel": "ks_fused_kernel<13, 2, 1>", "ciphertexts": 37, "dram_bytes": 402.9e6,
                        "pipe": "alu", "util": 0.387},
    # clusters of 8 CTAs of 2^12-value slices, two per SM; 66 = two full waves
    (32768, 3, 4, 12): {"kernel": "ks_fused_kernel<12, 3, 1, 8>", "ciphertexts": 66, "dram_bytes": 715.8e6,
                        "pipe": "alu", "util": 0.370},
    # the diagonal chain's evaluation level (2 + 4 limbs), same shape
    (32768, 2, 4, 12): {"kernel": "ks_fused_kernel<12, 3, 1, 8>", "ciphertexts": 66, "dram_bytes": 522.2e6,
                        "pipe": "alu", "util": 0.371},
}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ks_roofline(params, lanes: int, reps: int = 20, level: int = 0, nbuf: int = 5, choice=None):
    """One rotation step (a key switch with the automorphism folded into its
    loads) of `lanes` ciphertexts at `level` limbs per call, `nbuf` input
    batches cycled so the inputs stream from HBM; `reps` calls timed with
    CUDA events on the context stream after `nbuf` warm-up calls. `choice`:
    the autotuner's key-switch options for this level (KsChoice), else the
    context's defaults."""
    import numpy as np
    import torch

    from ._lib import CtRef
    from .driver import FheContext
    p = params
    n, K = p.n, p.K
    L = level or p.L
    w = L * n
    kw = p.key_words()
    ctx = FheContext(p, poly_words=(nbuf + 1) * lanes * 2 * w, key_words=kw, max_batch=lanes,
                     device=torch.cuda.current_device())
    try:
        rng = np.random.default_rng(3)
        allp = p.q + p.p
        ctx.write_key(0, np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for _ in range(2 * p.dnum)
                                         for q in allp]))
        ctx.lib.afhe_add_rotation_key(ctx.h, 1, 0)
        if choice is not None:
            if not choice.fused or ctx.get_option(1) == 1:
                ctx.set_option(1, int(choice.fused))
            ctx.set_option(2, min(int(choice.chunk), lanes))
            ctx.set_option(5, int(getattr(choice, "ept", 8)))
            ctx.set_option(6, int(getattr(choice, "slice", 13)))
        ept, slc = ctx.get_option(5), ctx.get_option(6)
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
        launches = (ctx.lib.afhe_kernel_launches() - l0) / reps
        ms = e0.elapsed_time(e1) / reps
        fused = int(ctx.get_option(1))
    finally:
        ctx.close()
    parts = -(-L // p.alpha)
    key_bytes = 2 * parts * (L + K) * n * 8
    bytes_per_call = lanes * 4 * w * 8 + key_bytes
    achieved = bytes_per_call / (ms * 1e-3) / 1e9
    peak, src = load_peaks()
    cap = KS_CAPTURES.get((n, L, K, slc if n >= 1 << 14 else 13))
    traffic = int_pipe = None
    if cap and launches == 1 and fused and ept == cap.get("ept", 8):
        # the capture's per-ciphertext traffic scaled to this launch, the key once
        traffic = (cap["dram_bytes"] - key_bytes) * lanes / cap["ciphertexts"] + key_bytes
        int_pipe = {"pipe": cap["pipe"], "frac": cap["util"], "kernel": cap["kernel"],
                    "captured_ciphertexts": cap["ciphertexts"]}
    shape = f", 2^{slc}-value slices" if n >= 1 << 14 else ""
    kind = f"one-kernel, {ept} values per thread{shape}" if fused and launches == 1 else f"{launches:g}-launch"
    return {"bound": "hbm", "kernel": f"rotation key switch, {kind} (N={n}, {L} + {K} limbs, "
                                      f"{lanes} ciphertexts per call)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": src, "traffic": traffic, "ms_per_call": ms, "launches_per_call": launches,
            "algorithmic_bytes_per_call": bytes_per_call, "int_pipe": int_pipe}


# ---------------------------------------------------------------------------
# profiling drivers
# ---------------------------------------------------------------------------
def profile_ks(lanes: int, workload: str = "small", level: int = 0, ept: int = 8, slc: int = 13):
    """The roofline measurement of the key switch alone (five warm-up calls,
    then 20 measured) at `level` limbs (default: the workload's evaluation
    level), the one-kernel key switch at `ept` values per thread."""
    from .autotune import KsChoice
    from .driver import CkksParams
    from .workloads import WORKLOADS
    spec = WORKLOADS[workload]
    p = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
    print(json.dumps(ks_roofline(p, lanes, level=level or spec.eval_level or spec.num_q,
                                 choice=KsChoice(True, lanes, 0.0, ept, slc))))


def profile_step(nq: int, workload: str = "small", lanes: int = 0, tune: bool = False):
    """One warm step, then one measured step of `nq` queries (with `tune`,
    under the autotuner's options, as the benchmark runs). Prints the
    kernel-launch counts an ncu launch list needs (-s / -c)."""
    from .workloads import WORKLOADS, Workload
    wl = Workload(WORKLOADS[workload], max_queries=nq, lanes=lanes or nq, tune=tune)
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


def mac_roofline(outputs: int = 64, units: int = 16, limbs: int = 2, reps: int = 10, generic: bool = False) -> dict:
    """The diagonal chain's inner-product kernel (afhe_eval_mac_plain_batch)
    alone, shaped like its stage 3 on the large configuration (N = 2^15, d =
    128: n1 = 16 baby steps, n2 = 8 giant steps): `outputs` outputs (one per
    query and giant step), each 16 groups (baby-step ciphertexts) of `units`
    plaintexts placed at multiples of 1,024 slots; the plaintexts come from
    `units` units of 128 diagonals at `limbs` limbs (1 GiB at 16 units, more
    than L2). Timed with CUDA events on the context stream after 3 warm-up
    calls. Algorithmic bytes: every plaintext read once per output, the
    outputs written, the 16 sources (2 polynomials) read once. The kernel
    is the diagonal chain's (afhe_eval_diag_inner_batch), or with `generic`
    afhe_eval_mac_plain_batch on the same terms."""
    import numpy as np
    import torch

    from . import _lib as L
    from .driver import CkksParams, FheContext, galois_elt
    from .query import InteractiveQueryManager as IQM
    p = CkksParams.generate(15, 12, 50, 4, 60, 4)
    n, D, n1, n2 = p.n, 128, 16, 8
    torch.cuda.init()
    w = limbs * n
    n_pts = units * D
    srcs = [((n_pts + 2 * b) * w, (n_pts + 2 * b + 1) * w) for b in range(n1)]
    base = (n_pts + 2 * n1) * w
    outs = [(base + 2 * o * w, base + (2 * o + 1) * w) for o in range(outputs)]
    ctx = FheContext(p, poly_words=base + 2 * outputs * w + w, key_words=1024, device=torch.cuda.current_device())
    try:
        rng = np.random.default_rng(3)
        for off in range(0, base, w):       # residues below every prime of the limbs
            ctx.write_poly(off, rng.integers(0, min(p.q[:limbs]), size=w, dtype=np.uint64))
        gal = np.array([galois_elt(p.log_n, -1024 * i) for i in range(units)], dtype=np.uint32)
        ib = np.arange(n2)[:, None, None] * n1 + np.arange(n1)[None, :, None]
        first, G, T = [0], [], []
        for o in range(outputs):
            k, g = divmod(o, n2)
            u = (k + np.arange(units)) % units
            pts = (u[None, None, :] * D + ib)[g] * w                       # (n1, units)
            for b in range(n1):
                G.append((srcs[b][0], srcs[b][1], len(T), units))
                T.extend(zip(pts[b].tolist(), gal.tolist(), [0] * units))
            first.append(len(G))
        Ga = np.array(G, dtype=IQM.MAC_GROUP)
        Ta = np.array(T, dtype=IQM.MAC_TERM)
        fg = np.array(first, dtype=np.uint32)
        refs = (L.CtRef * outputs)(*[L.CtRef(*c) for c in outs])
        # the same terms in the structured form: per output its 16 sources and units
        dsrc = (L.CtRef * (outputs * n1))(*[L.CtRef(*srcs[b]) for _ in range(outputs) for b in range(n1)])
        upt = np.concatenate([Ta["pt"][o * n1 * units:o * n1 * units + units] for o in range(outputs)])
        ugal = np.concatenate([Ta["galois"][o * n1 * units:o * n1 * units + units] for o in range(outputs)])
        ufirst = np.arange(0, outputs * units + 1, units, dtype=np.uint32)

        def call():
            if generic:
                L.check(ctx.lib.afhe_eval_mac_plain_batch(ctx.h, refs, fg.ctypes.data_as(L.P32), outputs,
                                                          Ga.ctypes.data_as(ctypes.POINTER(L.MacGroup)),
                                                          Ta.ctypes.data_as(ctypes.POINTER(L.MacTerm)), limbs, 0),
                        "eval_mac_plain_batch")
            else:
                L.check(ctx.lib.afhe_eval_diag_inner_batch(ctx.h, refs, outputs, dsrc, n1, upt.ctypes.data_as(L.P64),
                                                           ugal.ctypes.data_as(L.P32), ufirst.ctypes.data_as(L.P32),
                                                           w, limbs, 0), "eval_diag_inner_batch")
        for _ in range(3):
            call()
        ctx.sync()
        st = torch.cuda.ExternalStream(ctx.lib.afhe_stream(ctx.h), device=torch.cuda.current_device())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            call()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        alg = (len(T) * w + outputs * 2 * w + n1 * 2 * w) * 8
        peak, src = load_peaks()
        return {"profile": "mac_plain" if generic else "diag_inner", "outputs": outputs, "terms": len(T),
                "limbs": limbs, "ms": round(ms, 4),
                "algorithmic_bytes": alg, "achieved_gbs": round(alg / ms / 1e6, 1), "peak_gbs": peak,
                "frac": round(alg / ms / 1e6 / peak, 3), "peak_source": src}
    finally:
        ctx.close()


def profile_ntt(polys: int, log_n: int = 13, reps: int = 10):
    """Batched in-place NTT / INTT over `polys` polynomials of 4 limbs (the
    key switch's shape), forward then inverse, `reps` each."""
    import ctypes as C

    import numpy as np
    import torch

    from ._lib import P64
    from .driver import CkksParams, FheContext
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
        print(f"log_n={log_n} inverse={inv} {polys}x{limbs} limbs: {ms * 1e3:.1f} us per launch, "
              f"{gb / (ms * 1e-3):.0f} GB/s")
    ctx.close()


def profile_host(batch: int = 296, steps: int = 5, workload: str = "small"):
    """The end-to-end path on the host: (1) one batch through the protocol one
    phase at a time, each phase followed by a synchronisation, its wall time
    averaged over `steps` steps; (2) the streamed end-to-end run under
    cProfile, the host functions with the most own time. One JSON line each."""
    import cProfile
    import pstats

    import numpy as np
    import torch

    from ._lib import P64, check
    from .workloads import WORKLOADS, Workload
    wl = Workload(WORKLOADS[workload], max_queries=2 * batch, lanes=batch, tune=workload != "small")
    iqm = wl.iqm
    recs = wl.records[:batch]
    wl.encrypt_queries(wl.queries(batch, seed=1000), recs)
    host = [[torch.from_numpy(wl.ctx.read_poly(o, w)).pin_memory().numpy()
             for o, w in zip(wl.iqm.input_polys(r), wl.iqm.input_words(r))]
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
            for off, a in zip(wl.iqm.input_polys(r), cts):
                check(wl.ctx.lib.afhe_write_poly_async(wl.ctx.h, off, a.ctypes.data_as(P64), a.size), "write")
        t = mark("h2d", t)
        iqm.stage1_coarse(recs)
        t = mark("stage1", t)
        box = iqm.read_results("compact", recs, staged=True)[:, 0]
        t = mark("d2h_coarse", t)
        scales = np.array([iqm.out_scale_at(iqm.level_of(r)) for r in recs])
        vals = dec.decrypt_decode_host(box, scales, iqm.coarse_slots_needed())
        t = mark("client_decrypt_decode_coarse", t)
        for r, c in zip(recs, iqm.coarse_from_slots(vals)):
            r.probes = list(np.argsort(c, kind="stable")[:wl.spec.nprobe])
        t = mark("client_select", t)
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
    print(json.dumps({"profile": "phases", "queries_per_step": batch,
                      "ms": {k: round(v / steps, 2) for k, v in phases.items()}, "total_ms": round(total, 2),
                      "queries_per_s": round(batch / total * 1e3, 1)}), flush=True)
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


def profile_dispatch(calls: int = 200, log_n: int = 13):
    """Host-to-completion cost of afhe_dispatch per op code, one polynomial
    per call, as a host driving the reference's kernel ABI issues them: the
    small configuration's shape (3 + 1 limbs, alpha 1). `calls` calls of each
    op back to back, then one wait: microseconds per call (wall clock, so the
    host's share and the device's are both in it)."""
    import numpy as np

    from . import _lib as L
    from .driver import CkksParams, FheContext
    prm = CkksParams.generate(log_n, 3, 50, 1, 60, 1)
    n, Lq = prm.n, prm.L
    pw = 16 * (Lq + prm.K) * n
    ctx = FheContext(prm, poly_words=pw, key_words=4 * prm.key_words() + 8 * (Lq + prm.K) * n)
    try:
        lay = ctx.write_context_tables(Lq)
        rng = np.random.default_rng(4)
        ctx.write_key(lay.first_free_offset, np.concatenate([rng.integers(0, q, n, dtype=np.uint64)
                                                             for _ in range(2 * prm.dnum) for q in prm.q + prm.p]))
        W = (Lq + prm.K) * n
        for i in range(4):
            ctx.write_poly(i * W, np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for q in prm.q]))
        L.check(ctx.dispatch(ctx.accel_args(L.OP_LOAD_CONTEXT, Lq, lay)), "OP 99")
        ops = {"ntt": (L.OP_NTT, dict(src_a_offset=0, dst_offset=4 * W)),
               "intt": (L.OP_INTT, dict(src_a_offset=0, dst_offset=4 * W)),
               "poly_add": (L.OP_POLY_ADD, dict(src_a_offset=0, src_b_offset=W, dst_offset=4 * W)),
               "poly_mul_ntt": (L.OP_POLY_MUL_NTT, dict(src_a_offset=0, src_b_offset=W, dst_offset=4 * W)),
               "rescale": (L.OP_RESCALE, dict(src_a_offset=0, src_b_offset=W, dst_offset=4 * W)),
               "key_switch": (L.OP_KEY_SWITCH, dict(src_a_offset=0, dst_offset=4 * W,
                                                    evk_offset=lay.first_free_offset))}
        out = {}
        for name, (op, kw) in ops.items():
            a = ctx.accel_args(op, Lq, lay, **kw)
            for _ in range(5):
                L.check(ctx.dispatch(a), name)
            ctx.sync()
            t = time.perf_counter()
            for _ in range(calls):
                ctx.dispatch(a)
            ctx.sync()
            out[name] = round((time.perf_counter() - t) / calls * 1e6, 1)
    finally:
        ctx.close()
    print(json.dumps({"profile": "afhe_dispatch", "ring_degree": n, "limbs": f"{Lq} + {prm.K}",
                      "us_per_call": out, "calls": calls}))


def main() -> None:
    ap = argparse.ArgumentParser(prog="python -m anns_fhe_b200.profiling")
    sub = ap.add_subparsers(dest="what", required=True)
    a = sub.add_parser("ks", help="rotation key switch alone: ciphertexts per call")
    a.add_argument("lanes", type=int)
    a.add_argument("--workload", default="small", choices=["small", "large", "large_diag"])
    a.add_argument("--level", type=int, default=0)
    a.add_argument("--ept", type=int, default=8, choices=[8, 16], help="values per thread (one-kernel path)")
    a.add_argument("--slice", type=int, default=13, choices=[12, 13], help="log2 of a cluster CTA's slice")
    a = sub.add_parser("ntt", help="batched NTT / INTT: polynomials per launch")
    a.add_argument("polys", type=int)
    a.add_argument("--log-n", type=int, default=13)
    a = sub.add_parser("step", help="one query step: queries per step")
    a.add_argument("queries", type=int)
    a.add_argument("--workload", default="small", choices=["small", "large", "large_diag"])
    a.add_argument("--lanes", type=int, default=0)
    a.add_argument("--tune", action="store_true", help="the autotuner's key-switch options (as the benchmark)")
    a = sub.add_parser("mac", help="the diagonal chain's inner-product kernel alone: outputs per call")
    a.add_argument("outputs", type=int)
    a.add_argument("--units", type=int, default=16)
    a.add_argument("--generic", action="store_true", help="afhe_eval_mac_plain_batch instead of the structured kernel")
    a = sub.add_parser("host", help="end-to-end phases and the streamed run's host hotspots")
    a.add_argument("--workload", default="small", choices=["small", "large", "large_diag"])
    a.add_argument("--batch", type=int, default=296)
    a = sub.add_parser("dispatch", help="afhe_dispatch cost per call and op code")
    a.add_argument("--calls", type=int, default=200)
    args = ap.parse_args()
    if args.what == "ks":
        profile_ks(args.lanes, args.workload, args.level, args.ept, args.slice)
    elif args.what == "ntt":
        profile_ntt(args.polys, args.log_n)
    elif args.what == "step":
        profile_step(args.queries, args.workload, args.lanes, args.tune)
    elif args.what == "mac":
        print(json.dumps(mac_roofline(args.outputs, args.units, generic=args.generic)))
    elif args.what == "dispatch":
        profile_dispatch(args.calls)
    else:
        profile_host(args.batch, workload=args.workload)


if __name__ == "__main__":
    main()
