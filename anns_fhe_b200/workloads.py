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
import dataclasses
from dataclasses import dataclass

import numpy as np

from .ckks import CkksClient, Slots
from .driver import CkksParams, FheContext
from .ivfpq import IvfPqIndex, gaussian_mixture, plaintext_coarse, plaintext_search
from .query import NORM_BUDGET_BYTES, InteractiveQueryManager, QueryRecord, QueryShape


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
    compaction: str = "reference"
    # index training (the reference's k-means by default)
    kmeans_iters: int = 25
    train_sample: int | None = None
    pq_sample: int | None = None
    init: str = "random"
    eval_level: int | None = None     # limbs the server evaluates at (None: the query's level)


SMALL = WorkloadSpec("ivfpq_4096x64_nlist32_N8192_L3", n_vectors=4096, d=64, components=32, sigma=0.1, n_list=32,
                     M=8, K=256, nprobe=4, top_k=8, log_n=13, num_q=3, q_bits=50, num_p=1, p_bits=60, alpha=1,
                     log_scale=40)

# Batched encrypted IVF-PQ ADC over a larger database: 1,000,000 x 128 from a
# 1,024-component mixture (sigma 0.15), n_list 1024, PQ 16 x 256, nprobe 16;
# CKKS N = 2^15, scale 2^40, 12 x 50-bit Q + 4 x 60-bit P, alpha 4 (dnum 3).
# The centroids span 8 ciphertexts, so the coarse distances use the packed
# compaction. The index trains on seeded samples (131,072 vectors for IVF,
# 32,768 for PQ) with farthest-point seeding, then assigns every vector.
# Queries arrive at 12 limbs; the depth-2 chain is evaluated on their first 3
# (eval_level), so every key switch runs on 3 + 4 limbs.
LARGE = WorkloadSpec("ivfpq_1Mx128_nlist1024_N32768_L12", n_vectors=1_000_000, d=128, components=1024, sigma=0.15,
                     n_list=1024, M=16, K=256, nprobe=16, top_k=8, log_n=15, num_q=12, q_bits=50, num_p=4,
                     p_bits=60, alpha=4, log_scale=40, compaction="packed", kmeans_iters=8, train_sample=131072,
                     pq_sample=32768, init="farthest", eval_level=3)

# The same database, index and CKKS parameters through the diagonal chain
# (baby-step giant-step inner products, depth 1): the queries' first 2 limbs
# suffice, and the 1,024 lists' diagonals (128 plaintexts of 2 limbs per list,
# 64 GiB) stay resident in HBM.
LARGE_DIAG = dataclasses.replace(LARGE, compaction="diagonal", eval_level=2)
WORKLOADS = {"small": SMALL, "large": LARGE, "large_diag": LARGE_DIAG}


def query_layout(q: np.ndarray, sh: QueryShape) -> np.ndarray:
    """Slots of ct_query: q replicated once per centroid of a coarse
    ciphertext (slot c * D + d = q[d]); the reference replicates it n_list
    times, one per centroid (generate_interactive_test_vectors.cpp:383-398)."""
    reps = sh.n_list if sh.compaction == "reference" else sh.per_ct
    out = np.zeros(sh.slots)
    out[:reps * sh.D] = np.tile(np.asarray(q, dtype=np.float64), reps)
    return out


def dimpack_layout(q: np.ndarray, sh: QueryShape) -> np.ndarray:
    """Slots of ct_query_dimpack: slot d * B + j = q[d] for every candidate j."""
    return np.repeat(np.asarray(q, dtype=np.float64), sh.B)


def nearest_lists(coarse: np.ndarray, nprobes) -> list[list[int]]:
    """Row r's first nprobes[r] entries of argsort(coarse[r], kind="stable"):
    the lists a client probes, ties to the lower list. One stable sort of all
    rows together."""
    if len(coarse) == 0:
        return []
    order = np.argsort(coarse, axis=1, kind="stable")[:, :max(nprobes)]
    return [row[:k].tolist() for row, k in zip(order, nprobes)]


def ranked_prefix(vals: np.ndarray, pos, k: int) -> list[np.ndarray]:
    """For each row r: the first k entries of argsort(vals[r, pos[r]],
    kind="stable"), i.e. the k smallest values in order, ties by position.
    The k-th smallest value of each row comes from one partition of a padded
    matrix; only the entries up to it are then sorted, all rows together."""
    rows = len(pos)
    lens = np.array([len(p) for p in pos], dtype=np.int64)
    width = int(lens.max()) if rows else 0
    if width == 0 or k <= 0:
        return [np.zeros(0, dtype=np.int64) for _ in range(rows)]
    M = np.full((rows, width), np.inf)
    r_idx = np.repeat(np.arange(rows), lens)
    c_idx = np.arange(int(lens.sum())) - np.repeat(np.cumsum(lens) - lens, lens)
    M[r_idx, c_idx] = vals[r_idx, np.concatenate([np.asarray(p, dtype=np.int64) for p in pos])]
    kk = min(k, width)
    kth = np.partition(M, kk - 1, axis=1)[:, kk - 1]
    rr, cc = np.nonzero(M <= kth[:, None])
    order = np.lexsort((cc, M[rr, cc], rr))          # by row, then value, then position
    rr, cc = rr[order], cc[order]
    starts = np.searchsorted(rr, np.arange(rows))
    return [cc[starts[i]:starts[i] + min(kk, int(lens[i]))] for i in range(rows)]


class Workload:
    def __init__(self, spec: WorkloadSpec = SMALL, max_queries: int = 64, lanes: int = 64, device: int = 0,
                 index: IvfPqIndex | None = None, levels=None, max_nprobe: int | None = None,
                 tune: bool = False, spare_levels: int = 0, norm_budget: int = NORM_BUDGET_BYTES):
        """levels: query levels to serve besides the top one (mixed-level
        traffic); max_nprobe: the most lists one query may probe; tune: apply
        the autotuner's key-switch choices (cached per GPU and parameter
        set, measured when absent); spare_levels: room for the masks of that
        many more evaluation levels (InteractiveQueryManager.set_eval_level);
        norm_budget: HBM bytes for the packed chain's candidate norms (levels
        beyond it evaluate the unexpanded distance)."""
        self.spec = spec
        t0 = time.time()
        self.X = gaussian_mixture(spec.n_vectors, spec.d, spec.components, spec.sigma, spec.seed)
        self.index = index or IvfPqIndex.train(self.X, spec.n_list, spec.M, spec.K, spec.seed, iters=spec.kmeans_iters,
                                               train_sample=spec.train_sample, pq_sample=spec.pq_sample,
                                               init=spec.init)
        self.params = CkksParams.generate(spec.log_n, spec.num_q, spec.q_bits, spec.num_p, spec.p_bits, spec.alpha)
        n = self.params.n
        slots = n // 2
        shape = QueryShape(D=spec.d, n_list=spec.n_list, slots=slots, nprobe=spec.nprobe, top_k=spec.top_k,
                           scale=float(2 ** spec.log_scale), compaction=spec.compaction, eval_level=spec.eval_level)
        slot_w = (self.params.L + self.params.K) * n
        B = slots // spec.d
        n_batches = sum(-(-len(v) // B) for v in self.index.lists)
        most_probes = max(max_nprobe or spec.nprobe, spec.nprobe)
        n_res = InteractiveQueryManager.results_for(self.index, shape, most_probes)
        n_keys = 1 + len(InteractiveQueryManager.steps_for(shape))
        lvls = sorted(set(levels or []) | {self.params.L})
        w_out = (self.params.L - 2) * n
        most = max(max_queries, lanes) * max(n_res, 1)
        # client staging: results arrive as limb 0 (N words per polynomial)
        dec_slots = -(-most * 2 * n // slot_w) + -(-most * n // slot_w)
        outbox_slots = -(-2 * max_queries * w_out // slot_w) + -(-2 * max_queries * n_res * w_out // slot_w)
        masks = InteractiveQueryManager.mask_slots(shape, len(lvls) + spare_levels, spec.compaction == "reference")
        norm_slots = norm_reserve = 0
        work_slots = 8 * lanes
        if spec.compaction == "diagonal":   # no batch plaintexts or masks: per-level diagonals, baby steps
            IQM = InteractiveQueryManager
            evl = sorted({min(x, spec.eval_level or x) for x in lvls})
            units = sum(-(-len(v) // slots) for v in self.index.lists)
            n_batches, masks, work_slots = 0, 0, 0
            w_out = (self.params.L - 1) * n
            outbox_slots = -(-2 * max_queries * w_out // slot_w) + -(-2 * max_queries * n_res * w_out // slot_w)
            norm_slots = (sum(IQM.diagonal_slots(units, spec.d, lv, n, slot_w) for lv in evl)
                          + IQM.diagonal_scratch_slots(max_queries, min(lanes, 4096), shape.n1, shape.n2, evl[-1], n,
                                                       slot_w))
        if spec.compaction == "packed":     # ||q||^2 scratch per query; the candidates' norms per level
            evl = sorted({min(x, spec.eval_level or x) for x in lvls})
            norm_reserve = InteractiveQueryManager.norm_reserve_slots(evl, spare_levels, n_batches, self.params.L,
                                                                      n, slot_w, norm_budget)
            norm_slots = InteractiveQueryManager.norm_slots(max_queries, self.params.L, n, slot_w) + norm_reserve
        n_slots = (16 + shape.n_coarse + masks + n_batches + work_slots + 4 * max_queries + outbox_slots + 64
                   + InteractiveQueryManager.compaction_slots(spec.n_list if spec.compaction == "reference" else 1,
                                                              self.params.L, n, slot_w, lanes)
                   + dec_slots + norm_slots)
        self.ctx = FheContext(self.params, poly_words=n_slots * slot_w,
                              key_words=n_keys * self.params.key_words() + 4096, device=device,
                              max_batch=lanes)
        self.slots = Slots(self.params, 0, n_slots * slot_w)
        self.client = CkksClient(self.ctx, self.slots, seed=spec.seed + 7)
        self.iqm = InteractiveQueryManager(self.ctx, self.index, shape, self.slots, lanes=lanes, levels=lvls,
                                           max_nprobe=most_probes, norm_budget=norm_reserve * slot_w * 8)
        self.tuning = None
        if tune:
            from .autotune import load_or_tune
            lv = sorted({x for ev in self.iqm.levels for x in (ev, ev - 1, ev - 2) if x >= 1})
            self.tuning = load_or_tune(self.params, lv, lanes, device)
            self.iqm.use_tuning(self.tuning)
        self.steps = self.iqm.rotation_steps()
        self.client.install_keys(self.steps)
        self.records = self.iqm.alloc_queries(max_queries)
        # the client's decryption staging, sized once for the largest batch
        self.client._region("dec_in", most * 2 * n)
        self.client._region("dec_out", most * n)
        self.ctx.sync()
        self.setup_s = time.time() - t0

    def queries(self, count: int, seed: int = 99) -> np.ndarray:
        """Query vectors: database vectors plus a little noise (seeded)."""
        rng = np.random.default_rng(seed)
        idx = rng.integers(0, len(self.X), count)
        return (self.X[idx] + rng.normal(0, self.spec.sigma / 2, (count, self.spec.d))).astype(np.float32)

    # ---- client side ----
    def encrypt_queries(self, Q: np.ndarray, recs: list[QueryRecord], levels=None) -> None:
        """Encrypt each query (both layouts; the diagonal chain: the query
        and its squared norm) into its record, at levels[i] limbs (default:
        the top level)."""
        sh = self.iqm.sh
        for i, (q, r) in enumerate(zip(Q, recs)):
            lv = levels[i] if levels is not None else self.params.L
            r.level = lv
            self.client.encrypt(query_layout(q, sh), sh.scale, r.ct_query[0], r.ct_query[1], level=lv)
            if sh.compaction == "diagonal":
                # ||q||^2 in every slot, at the scale and level the server's
                # inner products reach after their rescale
                ll = self.iqm.eval_at(lv)
                n2 = float(np.dot(np.asarray(q, dtype=np.float64), np.asarray(q, dtype=np.float64)))
                self.client.encrypt(np.full(sh.slots, n2), sh.scale * sh.scale / self.params.q[ll - 1],
                                    r.ct_dim[0], r.ct_dim[1], level=ll - 1)
            else:
                self.client.encrypt(dimpack_layout(q, sh), sh.scale, r.ct_dim[0], r.ct_dim[1], level=lv)

    def decrypt_many(self, cts, scales, slots: int | None = None) -> np.ndarray:
        """Decrypt result ciphertexts resident on the device from limb 0 (the
        messages are far below q_0 / 2; the query manager checks the bound);
        row i is decoded at scales[i]."""
        return self.client.decrypt_decode(cts, np.asarray(scales, dtype=np.float64),
                                          slots or self.iqm.sh.slots).copy()

    def coarse(self, recs) -> np.ndarray:
        """(count, n_list) decrypted coarse distances."""
        scales = [self.iqm.out_scale_at(self.iqm.level_of(r)) for r in recs]
        vals = self.decrypt_many([r.compact for r in recs], scales, self.iqm.coarse_slots_needed())
        return self.iqm.coarse_from_slots(vals)

    def candidates(self, recs) -> list[np.ndarray]:
        """Each query's decrypted candidate distances, in stage-3 order."""
        S = self.iqm.sh.slots
        need = [max(1, -(-(int(r.pos[-1]) + 1) // S)) if len(r.pos) else 1 for r in recs]
        scales = [self.iqm.out_scale_at(self.iqm.level_of(r)) for r, k in zip(recs, need) for _ in range(k)]
        vals = self.decrypt_many([ct for r, k in zip(recs, need) for ct in r.results[:k]], scales)
        out, i = [], 0
        for r, k in zip(recs, need):
            out.append(vals[i:i + k].ravel()[np.asarray(r.pos, dtype=np.int64)])
            i += k
        return out

    def select(self, recs) -> None:
        """Stage 2 (client): decrypt the compacted coarse distances, keep each
        query's nprobe nearest lists."""
        for r, c in zip(recs, self.coarse(recs)):
            r.probes = list(np.argsort(c, kind="stable")[:r.nprobe or self.spec.nprobe])

    # ---- protocol ----
    def run(self, Q: np.ndarray, recs: list[QueryRecord] | None = None, levels=None, nprobes=None):
        """Full protocol for a batch of queries; returns per-query dicts.
        levels / nprobes: per-query encryption level and probe count
        (default: the top level and the spec's nprobe)."""
        recs = recs or self.records[:len(Q)]
        for i, r in enumerate(recs):
            r.nprobe = nprobes[i] if nprobes is not None else 0
        self.encrypt_queries(Q, recs, levels)
        self.iqm.stage1_coarse(recs)
        out = []
        for r, c in zip(recs, self.coarse(recs)):
            r.probes = list(np.argsort(c, kind="stable")[:r.nprobe or self.spec.nprobe])
            out.append({"coarse": c, "probes": r.probes})
        self.iqm.stage3_fine(recs)
        for r, o, d in zip(recs, out, self.candidates(recs)):
            order = np.argsort(d, kind="stable")[:self.spec.top_k]
            o.update(dists=d, vids=[int(v) for v in r.vids], topk=[int(r.vids[i]) for i in order])
        return out

    # ---- protocol from host buffers, in groups of queries ----
    def _group_stage1(self, part, hp, tag: str):
        """Host->device copy of a group's encrypted queries (four page-locked
        arrays per query), stage 1/1b, and an asynchronous copy of limb 0 of
        the compacted coarse distances to the host. Returns (box, fence,
        bytes copied to the device)."""
        from . import _lib as L
        lib, h = self.ctx.lib, self.ctx.h
        h2d = 0
        for r, cts in zip(part, hp):
            for off, a in zip(self.iqm.input_polys(r), cts):
                L.check(lib.afhe_write_poly_async(h, off, a.ctypes.data_as(L.P64), a.size), "write_poly_async")
                h2d += a.nbytes
        self.iqm.stage1_coarse(part)
        box, fence = self.iqm.read_results("compact", part, staged=True, tag=tag, wait=False)
        return box, fence, h2d

    def _group_stage3(self, part, coarse, dec, tag: str):
        """The client takes a group's coarse distances (waits for their copy,
        decrypts on `dec`, keeps the nprobe nearest lists); the server runs
        stage 3 with an asynchronous copy back. Returns (box, fence, bytes
        copied to the host for the coarse distances)."""
        box, fence, _ = coarse
        iqm = self.iqm
        self.ctx.fence_wait(fence)
        scales = np.array([iqm.out_scale_at(iqm.level_of(r)) for r in part])
        vals = dec.decrypt_decode_host(box[:, 0], scales, iqm.coarse_slots_needed())
        for r, pr in zip(part, nearest_lists(iqm.coarse_from_slots(vals),
                                             [r.nprobe or self.spec.nprobe for r in part])):
            r.probes = pr
        iqm.stage3_fine(part)
        fbox, ffence = iqm.read_results("dists", part, staged=True, tag=tag, wait=False)
        return fbox, ffence, box.nbytes

    def _group_topk(self, part, fine, dec):
        """The client takes a group's candidate distances: waits for their
        copy, decrypts the result ciphertexts that hold candidates, decodes,
        ranks. Returns (top-k id lists, bytes copied to the host)."""
        box, fence, _ = fine
        iqm, n, S = self.iqm, self.params.n, self.iqm.sh.slots
        self.ctx.fence_wait(fence)
        pos = [np.asarray(r.pos, dtype=np.int64) for r in part]
        last = max((int(p[-1]) + 1 if len(p) else 1) for p in pos)
        need = -(-last // S)                      # result ciphertexts that hold candidates
        scales = np.repeat([iqm.out_scale_at(iqm.level_of(r)) for r in part], need)
        vals = dec.decrypt_decode_host(box[:, :need].reshape(-1, 2, n), scales,
                                       min(S, last) if need == 1 else S).reshape(len(part), -1)
        return [[int(r.vids[i]) for i in top] for r, top in zip(part, ranked_prefix(vals, pos, self.spec.top_k))], \
            box.nbytes

    def run_host_pipelined(self, recs: list[QueryRecord], host_cts, dec, groups: int = 2):
        """The interactive protocol for `recs` through the C ABI from host
        buffers, with the records split into `groups` runs of consecutive
        records whose client and server work overlap.

        Per group: host->device copy of the encrypted queries (host_cts[i]:
        record i's c0, c1 of both layouts, page-locked), stage 1/1b, and an
        asynchronous copy of limb 0 of the compacted coarse distances to the
        host. Then, group by group, the client waits for its group's copy,
        decrypts (on its own context, `dec`: a CkksDecryptor), keeps the
        nprobe nearest lists, and the server runs stage 3 with an
        asynchronous copy back. Last, group by group, the client decrypts
        and ranks the candidates. While the client works on one group the
        server computes the next one's stage. Each query's result is the one
        `run` gives. Returns (top-k id lists, host->device bytes,
        device->host bytes)."""
        size = -(-len(recs) // max(1, groups))
        parts = [(recs[i:i + size], host_cts[i:i + size]) for i in range(0, len(recs), size)]
        coarse = [self._group_stage1(part, hp, str(g)) for g, (part, hp) in enumerate(parts)]
        h2d = sum(c[2] for c in coarse)
        fine = [self._group_stage3(part, coarse[g], dec, str(g)) for g, (part, _) in enumerate(parts)]
        d2h = sum(f[2] for f in fine)
        out = []
        for g, (part, _) in enumerate(parts):
            top, nb = self._group_topk(part, fine[g], dec)
            out += top
            d2h += nb
        return out, h2d, d2h

    def run_host_stream(self, recs: list[QueryRecord], host_cts, dec, total: int, group: int):
        """`total` queries streamed through the protocol from host buffers:
        query i is host_cts[i % len(host_cts)], in groups of `group`
        consecutive queries. Group g runs on records slice g mod k of `recs`
        (k = len(recs) // group slices of `group` records, k >= 3).

        A software pipeline over the groups: while the server computes
        group g's stage 1, the client selects group g - 1's lists (and its
        stage 3 is enqueued) and ranks group g - 2's candidates. So the
        client's work and the copies overlap the GPU everywhere but at the
        two ends of the stream. Returns (top-k id lists, host->device bytes,
        device->host bytes)."""
        k = len(recs) // group
        if k < 3:
            raise ValueError("a stream keeps three groups in flight: len(recs) >= 3 * group")
        G = -(-total // group)

        def part_of(g):
            size = min(group, total - g * group)
            base = (g % k) * group
            return recs[base:base + size], [host_cts[(g * group + i) % len(host_cts)] for i in range(size)]

        coarse, fine, tops = {}, {}, [None] * G
        h2d = d2h = 0
        for it in range(G + 2):
            if it < G:
                part, hp = part_of(it)
                coarse[it] = self._group_stage1(part, hp, "s%d" % (it % k))
                h2d += coarse[it][2]
            g = it - 1
            if 0 <= g < G:
                fine[g] = self._group_stage3(part_of(g)[0], coarse.pop(g), dec, "s%d" % (g % k))
                d2h += fine[g][2]
            g = it - 2
            if 0 <= g < G:
                tops[g], nb = self._group_topk(part_of(g)[0], fine.pop(g), dec)
                d2h += nb
        return [t for grp in tops for t in grp], h2d, d2h

    def plaintext(self, q: np.ndarray, nprobe: int | None = None):
        coarse = plaintext_coarse(self.index, q)
        probes, cand, dist, top = plaintext_search(self.index, q, nprobe or self.spec.nprobe, self.spec.top_k)
        return coarse, probes, cand, dist, top

    def close(self) -> None:
        self.iqm.close_native()
        self.client.close_decryptors()
        self.ctx.close()
