"""The encrypted IVF-PQ workload: seeded synthetic database, CKKS context,
keys, resident server plaintexts, and the full interactive protocol
(client encrypt -> server stages 1/1b -> client select -> server stage 3 ->
client top-k).

`small_ivfpq_workload()` is the plain single-query configuration the
reference's CPU path runs: 4,096 float32 vectors, d = 64, 32 Gaussian
clusters (centres N(0,1), sigma 0.1); IVF n_list 32, PQ M 8 x K 256, B 64,
nprobe 4; CKKS N = 2^13, scale 2^40, three 50-bit Q primes and one 60-bit
special prime, alpha 1 (dnum 3).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from .ckks import CkksClient, Slots
from .driver import CkksParams, FheContext
from .ivfpq import IvfPqIndex, gaussian_mixture, plaintext_coarse, plaintext_search
from .query import InteractiveQueryManager, QueryRecord, QueryShape


@dataclass
class WorkloadSpec:
    name: str
    n_vectors: int
    d: int
    components: int
    sigma: float
    n_list: int
    M: int
    K: int
    nprobe: int
    top_k: int
    log_n: int
    num_q: int
    q_bits: int
    num_p: int
    p_bits: int
    alpha: int
    log_scale: int
    seed: int = 2024


SMALL = WorkloadSpec("ivfpq_4096x64_nlist32_N8192_L3", n_vectors=4096, d=64, components=32, sigma=0.1, n_list=32,
                     M=8, K=256, nprobe=4, top_k=8, log_n=13, num_q=3, q_bits=50, num_p=1, p_bits=60, alpha=1,
                     log_scale=40)


class Workload:
    def __init__(self, spec: WorkloadSpec = SMALL, max_queries: int = 64, lanes: int = 64, device: int = 0,
                 index: IvfPqIndex | None = None):
        self.spec = spec
        t0 = time.time()
        self.X = gaussian_mixture(spec.n_vectors, spec.d, spec.components, spec.sigma, spec.seed)
        self.index = index or IvfPqIndex.train(self.X, spec.n_list, spec.M, spec.K, spec.seed)
        self.params = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
        n = self.params.n
        slots = n // 2
        shape = QueryShape(D=spec.d, n_list=spec.n_list, slots=slots, nprobe=spec.nprobe, top_k=spec.top_k,
                           scale=float(2 ** spec.log_scale))
        slot_w = (self.params.L + self.params.K) * n
        B = slots // spec.d
        n_batches = sum(-(-len(v) // B) for v in self.index.lists)
        w_out = (self.params.L - 2) * n
        most = max(max_queries, lanes)
        dec_slots = -(-most * 2 * w_out // slot_w) + -(-most * w_out // slot_w)
        n_slots = (16 + 1 + spec.n_list + 2 * n_batches + 8 * lanes + 8 * max_queries + 64 + max_queries
                   + InteractiveQueryManager.compaction_slots(spec.n_list, self.params.L, n, slot_w, lanes)
                   + dec_slots)
        self.ctx = FheContext(self.params, poly_words=n_slots * slot_w,
                              key_words=(2 + 2 * (spec.log_n + 1)) * self.params.key_words() + 4096, device=device,
                              max_batch=lanes)
        self.slots = Slots(self.params, 0, n_slots * slot_w)
        self.client = CkksClient(self.ctx, self.slots, seed=spec.seed + 7)
        self.iqm = InteractiveQueryManager(self.ctx, self.index, shape, self.slots, lanes=lanes)
        self.steps = self.iqm.rotation_steps()
        self.client.install_keys(self.steps)
        self.records = self.iqm.alloc_queries(max_queries)
        # the client's decryption staging, sized once for the largest batch
        self.client._region("dec_in", most * 2 * w_out)
        self.client._region("dec_out", most * w_out)
        self.ctx.sync()
        self.setup_s = time.time() - t0

    def queries(self, count: int, seed: int = 99) -> np.ndarray:
        """Query vectors: database vectors plus a little noise (seeded)."""
        rng = np.random.default_rng(seed)
        idx = rng.integers(0, len(self.X), count)
        return (self.X[idx] + rng.normal(0, self.spec.sigma / 2, (count, self.spec.d))).astype(np.float32)

    # ---- client side ----
    def encrypt_queries(self, Q: np.ndarray, recs: list[QueryRecord]) -> None:
        sh, D = self.iqm.sh, self.spec.d
        B = sh.B
        for q, r in zip(Q, recs):
            packed = np.zeros(sh.slots)
            for c in range(sh.n_list):
                packed[c * D:(c + 1) * D] = q
            self.client.encrypt(packed, sh.scale, r.ct_query[0], r.ct_query[1])
            dim = np.repeat(q.astype(np.float64), B)        # slot d*B + j = q[d]
            self.client.encrypt(dim, sh.scale, r.ct_dim[0], r.ct_dim[1])

    def decrypt_slots(self, ct) -> np.ndarray:
        return self.client.decrypt(ct[0], ct[1], self.iqm.lvl_out, self.iqm.out_scale).real

    def decrypt_many(self, cts) -> np.ndarray:
        return self.client.decrypt_batch(cts, self.iqm.lvl_out, self.iqm.out_scale).real

    def select(self, recs) -> None:
        """Stage 2 (client): decrypt the compacted coarse distances, keep nprobe lists."""
        coarse = self.decrypt_many([r.compact for r in recs])[:, :self.spec.n_list]
        for r, c in zip(recs, coarse):
            r.probes = list(np.argsort(c, kind="stable")[:self.spec.nprobe])

    # ---- protocol ----
    def run(self, Q: np.ndarray, recs: list[QueryRecord] | None = None):
        """Full protocol for a batch of queries; returns per-query dicts."""
        recs = recs or self.records[:len(Q)]
        self.encrypt_queries(Q, recs)
        self.iqm.stage1_coarse(recs)
        coarse = self.decrypt_many([r.compact for r in recs])[:, :self.spec.n_list]
        out = []
        for r, c in zip(recs, coarse):
            r.probes = list(np.argsort(c, kind="stable")[:self.spec.nprobe])
            out.append({"coarse": c, "probes": r.probes})
        self.iqm.stage3_fine(recs)
        dists = self.decrypt_many([r.dists for r in recs])
        for r, o, d in zip(recs, out, dists):
            d = d[:len(r.vids)]
            order = np.argsort(d, kind="stable")[:self.spec.top_k]
            o.update(dists=d, vids=list(r.vids), topk=[r.vids[i] for i in order])
        return out

    def plaintext(self, q: np.ndarray):
        coarse = plaintext_coarse(self.index, q)
        probes, cand, dist, top = plaintext_search(self.index, q, self.spec.nprobe, self.spec.top_k)
        return coarse, probes, cand, dist, top

    def close(self) -> None:
        self.ctx.close()
