"""The encrypted IVF-PQ server chain on the CPU oracle (timed CPU baseline).

TEST INFRASTRUCTURE ONLY: bench.py's reference arm and its cpu_baseline
leg time this; the product never runs it.

Runs exactly the operator sequence of anns_fhe_b200/query.py (the reference's
InteractiveQueryManager chain, interactive_query_manager.cpp:85-303 with the
generator's semantics) for one query at a time on the C restatement of the
reference's HLS kernels (oracle/liborc.so). The reference's own compiled HLS
sources run only at N = 16384 with at most 15 limbs, so this workload
(N = 8192) is timed on the restatement ("port"). The cost of the chain does
not depend on residue values, so inputs, keys and plaintexts are seeded
uniform residues; the probed lists come from the plaintext index.
One worker process per host core, started with spawn.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np


def _config():
    from anns_fhe_b200.workloads import SMALL
    return SMALL


def _setup(seed: int):
    from oracle.composite import OracleCKKS
    from oracle.oracle import Orc
    spec = _config()
    # the same primes the GPU context uses (host-only helpers, no GPU needed)
    from anns_fhe_b200.driver import CkksParams
    prm = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
    ora = OracleCKKS(prm.log_n, prm.q, prm.p, prm.alpha, Orc())
    rng = np.random.default_rng(seed)
    n, L, K = prm.n, prm.L, prm.K

    def uni(primes):
        return np.concatenate([rng.integers(0, q, n, dtype=np.uint64) for q in primes])

    def key():
        return (np.concatenate([uni(prm.q + prm.p) for _ in range(prm.dnum)]),
                np.concatenate([uni(prm.q + prm.p) for _ in range(prm.dnum)]))

    slots = n // 2
    D, B = spec.d, slots // spec.d
    steps = set()
    s = 1
    while s < D:
        steps.update((s, B * s))
        s <<= 1
    for i in range(spec.n_list):
        r = i * (D - 1)
        while r:
            b = 1 << (r.bit_length() - 1)
            steps.add(b)
            r -= b
    s = 1
    while s < slots:
        steps.add(-s)
        s <<= 1
    rot = {st: key() for st in steps}
    relin = key()
    ct = (uni(prm.q), uni(prm.q))
    pt = uni(prm.q)
    masks = uni(prm.q[:L - 1])
    return dict(ora=ora, rot=rot, relin=relin, ct=ct, pt=pt, mask=masks, spec=spec, D=D, B=B, L=L, n=n)


def _items(spec, B):
    """Per-batch candidate counts of the 4 probed lists of a typical query."""
    from anns_fhe_b200.ivfpq import IvfPqIndex, gaussian_mixture, plaintext_search
    X = gaussian_mixture(spec.n_vectors, spec.d, spec.components, spec.sigma, spec.seed)
    idx = IvfPqIndex.train(X, spec.n_list, spec.M, spec.K, spec.seed)
    probes, _, _, _ = plaintext_search(idx, X[0], spec.nprobe, spec.top_k)
    counts = []
    for c in probes:
        m = len(idx.lists[c])
        counts += [min(B, m - b0) for b0 in range(0, m, B)]
    return counts


def one_query(st, counts) -> float:
    """Server chain for one query; returns seconds."""
    ora, rot, relin = st["ora"], st["rot"], st["relin"]
    D, B, L = st["D"], st["B"], st["L"]
    t0 = time.perf_counter()
    # stage 1 / 1b
    diff = ora.eval_sub_plain(st["ct"], st["pt"], L)
    sq = ora.eval_mult_relin_rescale(diff, diff, relin, L)
    s = 1
    while s < D:
        sq = ora.eval_add(sq, ora.eval_rotate(sq, s, rot, L - 1), L - 1)
        s <<= 1
    comp = None
    for i in range(st["spec"].n_list):
        sel = ora.eval_mult_plain_rescale(sq, st["mask"], L - 1)
        if i:
            sel = ora.eval_rotate(sel, i * (D - 1), rot, L - 2)
        comp = sel if comp is None else ora.eval_add(comp, sel, L - 2)
    # stage 3
    off, acc = 0, None
    for cnt in counts:
        diff = ora.eval_sub_plain(st["ct"], st["pt"], L)
        sq = ora.eval_mult_relin_rescale(diff, diff, relin, L)
        s = B
        while s < D * B:
            sq = ora.eval_add(sq, ora.eval_rotate(sq, s, rot, L - 1), L - 1)
            s <<= 1
        sel = ora.eval_mult_plain_rescale(sq, st["mask"], L - 1)
        if off:
            sel = ora.eval_rotate(sel, -off, rot, L - 2)
        acc = sel if acc is None else ora.eval_add(acc, sel, L - 2)
        off += cnt
    return time.perf_counter() - t0


def _worker(args):
    seed, counts, nq, warm = args
    st = _setup(seed)
    for _ in range(warm):
        one_query(st, counts)
    return [one_query(st, counts) for _ in range(nq)]


def cpu_reference_rate(steps: int = 1, warmup: int = 0, workers: int | None = None, queries_per_worker: int = 1,
                       n_gpus: int = 0):
    """Queries/s of the chain on all host cores: `warmup` untimed, then `steps`
    timed rounds of one query per worker process."""
    spec = _config()
    B = (1 << spec.log_n) // 2 // spec.d
    counts = _items(spec, B)
    workers = workers or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        t0 = time.perf_counter()
        per = pool.map(_worker, [(11 + w, counts, queries_per_worker * max(1, steps), warmup) for w in range(workers)])
        wall = time.perf_counter() - t0
    per_query = [x for p in per for x in p]
    done = len(per_query)
    chain_s = sum(per_query) / done
    # setup (tables, keys) is excluded: rate from the per-query chain times of
    # the concurrently running workers
    rate = workers / chain_s
    return {
        "impl": "reference",
        "metric": "encrypted IVF-PQ queries/s (batched server, interactive protocol)",
        "value": rate,
        "unit": "queries/s",
        "n_gpus": n_gpus,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": chain_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded uniform residues; cost is value-independent)",
        "config": {"workload": spec.name, "queries_per_step": workers, "nprobe": spec.nprobe,
                   "stage3_batches": len(counts)},
        "cpu_baseline": {"value": rate, "unit": "queries/s", "cores": workers, "kind": "port",
                         "sample": f"{done} queries ({workers} processes x {done // workers}), server chain only, "
                                   f"wall {wall:.1f}s"},
        "e2e": {"value": rate, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


if __name__ == "__main__":
    import json
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    st = _setup(1)
    B = (1 << st["spec"].log_n) // 2 // st["spec"].d
    c = _items(st["spec"], B)
    print("items", c)
    print("one query s", one_query(st, c))
