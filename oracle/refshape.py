"""The reference's own key switch, compiled from its sources, timed on host cores.

TEST INFRASTRUCTURE ONLY: bench.py's reference-shape driver times this as
the CPU side of a kernel-level comparison; the product never runs it.

The reference's HLS C-simulation (hardware_fpga_model/hls/src/key_switch.cpp:
167-439, compiled verbatim into _ref/libref_hls.so) runs only at its own
shape: N = 16384, at most 11 Q + 4 P limbs, three digits. One key switch at
10 Q limbs (digits of 4, 4 and 2 limbs) is the unit. Inputs and keys are
seeded uniform residues: the cost does not depend on their values. Tables are
computed from their definitions (tables_py), as the reference's generator
lays them out.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

LOG_N = 14
SIZE_QL = 10
PARTS = 3
ALPHA = 4


def _worker(job):
    q, p, seconds, seed = job
    from oracle.oracle import Ref, tables_py as T
    n, K = 1 << LOG_N, len(p)
    tw = [T.twiddles(LOG_N, x) for x in q + p]
    tw_q = np.concatenate([t[0] for t in tw[:len(q)]])
    itw_q = np.concatenate([t[1] for t in tw[:len(q)]])
    tw_p = np.concatenate([t[0] for t in tw[len(q):]])
    itw_p = np.concatenate([t[1] for t in tw[len(q):]])
    qhat = [T.part_qhat(q, SIZE_QL, ALPHA, j, p) for j in range(PARTS)]
    pinv, phinv, phq = T.moddown(q, SIZE_QL, p)
    rng = np.random.default_rng(seed)
    primes_k = q[:SIZE_QL] + p
    key = np.concatenate([rng.integers(0, x, n, dtype=np.uint64) for _ in range(2 * PARTS) for x in primes_k])
    c = np.concatenate([rng.integers(0, x, n, dtype=np.uint64) for x in q[:SIZE_QL]])
    ref = Ref()
    count, t0 = 0, time.perf_counter()
    while True:
        ref.key_switch(c, key, 0, PARTS * (SIZE_QL + K) * n, SIZE_QL, K, PARTS, ALPHA, q, p, tw_q, itw_q, tw_p,
                       itw_p, [a for a, _ in qhat], [b for _, b in qhat], pinv, phinv, phq)
        count += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            return count, el


def reference_key_switch_rate(q, p, seconds: float = 10.0, procs: int | None = None) -> dict:
    """Key switches per second of the reference's HLS key switch, one process
    per host core (spawned: safe beside a CUDA context), each running for
    about `seconds` after building its tables."""
    procs = procs or os.cpu_count() or 1
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_worker, [(list(q), list(p), seconds, 100 + i) for i in range(procs)])
    count = sum(c for c, _ in res)
    wall = max(el for _, el in res)
    return {"value": count / wall, "unit": "key switches/s", "cores": procs, "kind": "reference",
            "sample": f"{count} key switches ({procs} processes, about {seconds:.0f} s each), N = 16384, "
                      f"{SIZE_QL} Q + {len(p)} P limbs, {PARTS} digits of {ALPHA}"}
