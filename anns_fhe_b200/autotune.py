"""Autotuner for the batched key switch and the NTT's tile shapes.

For a parameter set on a given GPU it picks, per level, the key-switch
implementation (the one-kernel key switch, or the multi-kernel ModUp / inner
product / ModDown pipeline) and the number of ciphertexts per launch (a tile
of the batch: fewer per launch shortens the tail of the last wave, more
amortises launches and the key's L2 footprint). It times rotation batches on
the device. It also times every NTT plan of the ring degree (afhe_ntt_set_plan:
values per thread for one-pass transforms; columns per CTA and chunk-tile size
for two-pass ones) on batched forward and inverse transforms, and keeps the
fastest. The residues are the same for every choice, so the tuner only trades
speed. Results are cached per (GPU, N, L, K, alpha) as JSON under
anns_fhe_b200/tuning/, with every candidate's time.

    python -m anns_fhe_b200.autotune --workload small     # tune and write the cache
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time
from dataclasses import asdict, dataclass

import numpy as np

from . import _lib as L
from .driver import CkksParams, FheContext

CACHE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")


@dataclass
class KsChoice:
    fused: bool
    chunk: int
    us_per_ct: float
    ept: int = 8          # values per thread of the one-kernel key switch (AFHE_OPT_KS_EPT)
    slice: int = 13       # log2 of a cluster CTA's slice (AFHE_OPT_KS_SLICE; 12 at N = 2^14, 2^15)
    fused_min: int = 0    # launches of fewer ciphertexts take the multi-kernel path (0: context default)


def gpu_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "unknown"


def sm_count(device: int = 0) -> int:
    try:
        import torch
        return torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:
        return 148


def cache_path(params: CkksParams, name: str | None = None) -> str:
    gpu = (name or gpu_name()).replace(" ", "_")
    return os.path.join(CACHE_DIR, f"{gpu}_N{params.n}_L{params.L}_K{params.K}_a{params.alpha}.json")


def chunk_candidates(lanes: int, sms: int, capacity: int = 0) -> list[int]:
    """Ciphertexts per launch to try: fractions and multiples of one wave of
    SMs, multiples of the one-kernel key switch's capacity (ciphertexts it
    runs at once; full waves), up to the context's lanes."""
    c = {max(1, sms // 4), max(1, sms // 2), sms, 2 * sms, 3 * sms, 4 * sms, lanes}
    if capacity > 0:
        c |= {k * capacity for k in range(1, 9)}
    return sorted(x for x in c if 1 <= x <= lanes)


TIE = 0.10   # candidates within this fraction of the fastest count as ties
# Version of the key-switch kernels a cache was tuned against: a cache from
# other kernels (e.g. before the one-kernel path existed at this ring degree)
# is tuned again.
KERNELS = 8


def ntt_plan_count(log_n: int) -> int:
    n = C.c_uint32()
    L.check(L.load().afhe_ntt_plan_count(log_n, C.byref(n)), "ntt_plan_count")
    return n.value


def ntt_plan_describe(log_n: int, plan: int) -> str:
    buf = C.create_string_buffer(160)
    L.check(L.load().afhe_ntt_plan_describe(log_n, plan, buf, len(buf)), "ntt_plan_describe")
    return buf.value.decode()


def set_ntt_plan(log_n: int, plan: int) -> None:
    """Tile shapes of every NTT at ring degree 2^log_n, process-wide."""
    L.check(L.load().afhe_ntt_set_plan(log_n, plan), "ntt_set_plan")


def get_ntt_plan(log_n: int) -> int:
    p = C.c_uint32()
    L.check(L.load().afhe_ntt_get_plan(log_n, C.byref(p)), "ntt_get_plan")
    return p.value


def time_ntt_plans(ctx: FheContext, polys: int, limbs: int, reps: int = 3) -> dict:
    """{plan: microseconds per limb of a forward plus an inverse transform}
    over `polys` polynomials of `limbs` limbs at offsets 0, limbs N, ...
    (best of `reps` after a warm-up call each). Restores the plan in force."""
    n, log_n = ctx.params.n, ctx.params.log_n
    offs = (L.u64 * polys)(*[z * limbs * n for z in range(polys)])
    ptr = C.cast(offs, L.P64)
    lib = ctx.lib
    keep = get_ntt_plan(log_n)
    out = {}
    try:
        for plan in range(ntt_plan_count(log_n)):
            set_ntt_plan(log_n, plan)
            best = float("inf")
            for r in range(reps + 1):
                ctx.sync()
                t0 = time.perf_counter()
                L.check(lib.afhe_ntt_batch(ctx.h, ptr, polys, limbs, 0), "ntt_batch")
                L.check(lib.afhe_ntt_batch(ctx.h, ptr, polys, limbs, 1), "ntt_batch")
                ctx.sync()
                if r:
                    best = min(best, time.perf_counter() - t0)
            out[plan] = best / (polys * limbs) * 1e6
    finally:
        set_ntt_plan(log_n, keep)
    return out


SHAPE_TIE = 0.03   # 16 values per thread must beat 8 by more than this to be picked


def pick(timings: dict) -> tuple:
    """The key of {(fused, chunk[, ept, slice]): us_per_ct} to use: among the
    candidates within TIE of the fastest, the largest chunk (fewest
    launches; a chain's batches are rarely a multiple of the tile, and every
    extra launch costs its tail), then the one-kernel path, then the
    fastest. 16 values per thread counts SHAPE_TIE slower than measured: an
    isolated rotation batch favours it slightly more than the chain does."""
    def eff(k):
        return timings[k] * (1 + SHAPE_TIE) if len(k) > 2 and k[2] != 8 else timings[k]
    best = min(eff(k) for k in timings)
    near = [k for k in timings if eff(k) <= best * (1 + TIE)]
    return max(near, key=lambda k: (k[1], k[0], -eff(k)))


def time_rotations(ctx: FheContext, level: int, count: int, reps: int = 3) -> float:
    """Microseconds per ciphertext of a one-step rotation over `count`
    ciphertexts at `level` (best of `reps`, after a warm-up call)."""
    n = ctx.params.n
    w = level * n
    arr = (L.CtRef * count)()
    for i in range(count):
        arr[i].c0_offset, arr[i].c1_offset = 2 * i * w, (2 * i + 1) * w
    lib = ctx.lib
    L.check(lib.afhe_eval_rotate_batch(ctx.h, arr, arr, count, 1, level), "eval_rotate_batch")
    ctx.sync()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        L.check(lib.afhe_eval_rotate_batch(ctx.h, arr, arr, count, 1, level), "eval_rotate_batch")
        ctx.sync()
        best = min(best, time.perf_counter() - t0)
    return best / count * 1e6


def fused_crossover(ctx: FheContext, level: int, lanes: int, verbose: bool = False) -> int:
    """The fewest ciphertexts per launch from which the one-kernel key switch
    (one CTA or cluster per ciphertext) beats the multi-kernel pipeline (which
    spreads one ciphertext over many CTAs) at every larger count tried:
    AFHE_OPT_FUSED_MIN for this level. The context's options are restored."""
    keep = ctx.get_option(L.OPT_FUSED_MIN)
    counts = [c for c in (1, 2, 4, 8, 16, 32, 64, 128) if c <= lanes]
    wins = {}
    try:
        ctx.set_option(L.OPT_FUSED_MIN, 1)
        for c in counts:
            ctx.set_option(L.OPT_KS_FUSED, 1)
            t1 = time_rotations(ctx, level, c)
            ctx.set_option(L.OPT_KS_FUSED, 0)
            t0 = time_rotations(ctx, level, c)
            wins[c] = t1 <= t0
            if verbose:
                print(f"level {level}, {c} per launch: one-kernel {t1:.2f}, multi-kernel {t0:.2f} us/ct")
    finally:
        ctx.set_option(L.OPT_KS_FUSED, 1)
        ctx.set_option(L.OPT_FUSED_MIN, keep)
    fmin = min(4096, 2 * counts[-1]) if counts else 1
    for c in reversed(counts):
        if not wins[c]:
            break
        fmin = c
    return fmin


def tune(params: CkksParams, levels, lanes: int, device: int = 0, verbose: bool = False) -> dict:
    """{level: KsChoice} measured on `device`."""
    n = params.n
    count = lanes
    w_max = max(levels) * n
    ctx = FheContext(params, poly_words=2 * count * w_max, key_words=params.key_words() + 1024, device=device,
                     max_batch=lanes)
    try:
        rng = np.random.default_rng(7)
        key = np.concatenate([rng.integers(0, q, n, dtype=np.uint64)
                              for _ in range(2 * params.dnum) for q in params.q + params.p])
        ctx.write_key(0, key)
        L.check(ctx.lib.afhe_add_rotation_key(ctx.h, 1, 0), "add_rotation_key")
        for i in range(2 * count):
            ctx.write_poly(i * w_max, np.concatenate([rng.integers(0, q, n, dtype=np.uint64)
                                                      for q in params.q[:max(levels)]]))
        fused_ok = ctx.get_option(L.OPT_KS_FUSED) == 1    # the context enables it where the GPU can run it
        shapes = [(True, 8, 13), (True, 16, 13), (False, 8, 13)] if fused_ok else [(False, 8, 13)]
        if fused_ok and params.log_n in (14, 15):
            try:
                ctx.set_option(L.OPT_KS_SLICE, 12)
                shapes[2:2] = [(True, 8, 12), (True, 16, 12)]
            except L.AfheError:
                pass                     # two CTAs per SM cannot be placed in clusters here
            ctx.set_option(L.OPT_KS_SLICE, 13)
        out = {}
        for lv in sorted(set(levels)):
            timings = {}
            for fused, ept, sl in shapes:
                ctx.set_option(L.OPT_KS_FUSED, int(fused))
                ctx.set_option(L.OPT_KS_EPT, ept)
                ctx.set_option(L.OPT_KS_SLICE, sl)
                cap = ctx.get_option(L.OPT_KS_CAPACITY) if fused else 0
                for c in chunk_candidates(lanes, sm_count(device), cap):
                    ctx.set_option(L.OPT_CHUNK, c)
                    timings[(fused, c, ept, sl)] = time_rotations(ctx, lv, count)
                    if verbose:
                        print(f"level {lv} fused={fused} ept={ept} slice=2^{sl} chunk={c}: "
                              f"{timings[(fused, c, ept, sl)]:.2f} us/ct")
            f, c, e, sl = pick(timings)
            fmin = 0
            if f:
                ctx.set_option(L.OPT_KS_EPT, e)
                ctx.set_option(L.OPT_KS_SLICE, sl)
                fmin = fused_crossover(ctx, lv, lanes, verbose)
            out[lv] = KsChoice(f, c, timings[(f, c, e, sl)], e, sl, fmin)
        ctx.set_option(L.OPT_KS_EPT, 8)
        ctx.set_option(L.OPT_KS_SLICE, 13)
        ctx.set_option(L.OPT_KS_FUSED, 1 if fused_ok else 0)
        return out
    finally:
        ctx.close()


def tune_ntt(params: CkksParams, lanes: int, device: int = 0, verbose: bool = False) -> dict:
    """{"plan": fastest, "us_per_limb": {plan: time}, "describe": {plan: text}}
    for batched transforms of `lanes` ciphertexts (2 lanes polynomials) at
    the top level, capped at 2 GB of device memory."""
    n, log_n, limbs = params.n, params.log_n, params.L
    polys = max(1, min(2 * lanes, (2 << 30) // (limbs * n * 8)))
    ctx = FheContext(params, poly_words=polys * limbs * n, key_words=1024, device=device, max_batch=1)
    try:
        rng = np.random.default_rng(11)
        for z in range(polys):
            ctx.write_poly(z * limbs * n, np.concatenate([rng.integers(0, q, n, dtype=np.uint64)
                                                          for q in params.q[:limbs]]))
        t = time_ntt_plans(ctx, polys, limbs)
    finally:
        ctx.close()
    best = min(t, key=lambda p: (t[p] > min(t.values()) * (1 + TIE / 2), p))   # plan 0 unless another is clearly faster
    if verbose:
        for p, us in t.items():
            print(f"NTT plan {p} ({ntt_plan_describe(log_n, p)}): {us:.3f} us/limb")
    return {"plan": best, "us_per_limb": {str(p): v for p, v in t.items()},
            "describe": {str(p): ntt_plan_describe(log_n, p) for p in t}}


def save(path: str, params: CkksParams, choices: dict, lanes: int, ntt: dict | None = None) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"gpu": gpu_name(), "log_n": params.log_n, "L": params.L, "K": params.K,
                   "alpha": params.alpha, "lanes": lanes, "kernels": KERNELS,
                   "levels": {str(k): asdict(v) for k, v in sorted(choices.items())},
                   "ntt": ntt}, f, indent=1)


def load_full(path: str, lanes: int) -> tuple[dict, dict | None] | None:
    """(key-switch choices, NTT record) of a cache tuned for the same lanes
    and kernels, else None."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if d.get("lanes") != lanes or d.get("kernels") != KERNELS:
        return None
    return {int(k): KsChoice(**v) for k, v in d["levels"].items()}, d.get("ntt")


def load(path: str, lanes: int) -> dict | None:
    """Cached key-switch choices, if the cache exists and was tuned for the same lanes."""
    got = load_full(path, lanes)
    return got[0] if got else None


def load_or_tune(params: CkksParams, levels, lanes: int, device: int = 0) -> dict:
    """Key-switch choices per level (cached or measured now); the NTT plan of
    the cache (measured now when absent) is put in force."""
    path = cache_path(params)
    got = load_full(path, lanes)
    if got is not None and set(levels) <= set(got[0]) and got[1]:
        choices, ntt = got
    else:
        choices = tune(params, levels, lanes, device)
        ntt = tune_ntt(params, lanes, device)
        save(path, params, choices, lanes, ntt)
    set_ntt_plan(params.log_n, int(ntt["plan"]))
    return choices


def main() -> None:
    from .workloads import LARGE, SMALL
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="small", choices=["small", "large"])
    ap.add_argument("--lanes", type=int, default=0)
    a = ap.parse_args()
    spec = LARGE if a.workload == "large" else SMALL
    params = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
    lanes = a.lanes or (256 if spec is LARGE else 2 * sm_count())
    top = spec.eval_level or spec.num_q
    levels = [lv for lv in (top, top - 1, top - 2) if lv >= 1]
    choices = tune(params, levels, lanes, verbose=True)
    ntt = tune_ntt(params, lanes, verbose=True)
    path = cache_path(params)
    save(path, params, choices, lanes, ntt)
    print(json.dumps({"levels": {str(k): asdict(v) for k, v in choices.items()}, "ntt_plan": ntt["plan"]}), "->", path)


if __name__ == "__main__":
    main()
