"""Autotuner for the batched key switch.

For a parameter set on a given GPU it picks, per level, the key-switch
implementation (the one-kernel key switch for N <= 2^13, or the multi-kernel
ModUp / inner product / ModDown pipeline) and the number of ciphertexts per
launch (a tile of the batch: fewer per launch shortens the tail of the last
wave, more amortises launches and the key's L2 footprint). It times rotation
batches on the device. The residues are the same for every choice, so the
tuner only trades speed. Results are cached per (GPU, N, L, K, alpha) as JSON
under anns_fhe_b200/tuning/.

    python -m anns_fhe_b200.autotune --workload small     # tune and write the cache
"""
from __future__ import annotations

import argparse
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


def chunk_candidates(lanes: int, sms: int) -> list[int]:
    """Ciphertexts per launch to try: fractions and multiples of one wave of
    SMs, up to the context's lanes."""
    c = {max(1, sms // 4), max(1, sms // 2), sms, 2 * sms, 3 * sms, 4 * sms, lanes}
    return sorted(x for x in c if 1 <= x <= lanes)


TIE = 0.10   # candidates within this fraction of the fastest count as ties
# Version of the key-switch kernels a cache was tuned against: a cache from
# other kernels (e.g. before the one-kernel path existed at this ring degree)
# is tuned again.
KERNELS = 2


def pick(timings: dict) -> tuple:
    """The (fused, chunk) of {(fused, chunk): us_per_ct} to use: among the
    candidates within TIE of the fastest, the largest chunk (fewest
    launches; a chain's batches are rarely a multiple of the tile, and every
    extra launch costs its tail), then the one-kernel path."""
    best = min(timings.values())
    near = [k for k, v in timings.items() if v <= best * (1 + TIE)]
    return max(near, key=lambda k: (k[1], k[0], -timings[k]))


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
        out = {}
        for lv in sorted(set(levels)):
            timings = {}
            for fused in ([True, False] if fused_ok else [False]):
                ctx.set_option(L.OPT_KS_FUSED, int(fused))
                for c in chunk_candidates(lanes, sm_count(device)):
                    ctx.set_option(L.OPT_CHUNK, c)
                    timings[(fused, c)] = time_rotations(ctx, lv, count)
                    if verbose:
                        print(f"level {lv} fused={fused} chunk={c}: {timings[(fused, c)]:.2f} us/ct")
            f, c = pick(timings)
            out[lv] = KsChoice(f, c, timings[(f, c)])
        return out
    finally:
        ctx.close()


def save(path: str, params: CkksParams, choices: dict, lanes: int) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"gpu": gpu_name(), "log_n": params.log_n, "L": params.L, "K": params.K,
                   "alpha": params.alpha, "lanes": lanes, "kernels": KERNELS,
                   "levels": {str(k): asdict(v) for k, v in sorted(choices.items())}}, f, indent=1)


def load(path: str, lanes: int) -> dict | None:
    """Cached choices, if the cache exists and was tuned for the same lanes."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if d.get("lanes") != lanes or d.get("kernels") != KERNELS:
        return None
    return {int(k): KsChoice(**v) for k, v in d["levels"].items()}


def load_or_tune(params: CkksParams, levels, lanes: int, device: int = 0) -> dict:
    path = cache_path(params)
    got = load(path, lanes)
    if got is not None and set(levels) <= set(got):
        return got
    choices = tune(params, levels, lanes, device)
    save(path, params, choices, lanes)
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
    path = cache_path(params)
    save(path, params, choices, lanes)
    print(json.dumps({str(k): asdict(v) for k, v in choices.items()}), "->", path)


if __name__ == "__main__":
    main()
