"""Encrypted interactive IVF-PQ query: the server-side operator chain.

Mirrors InteractiveQueryManager (cpp_host_model/src/interactive_query_manager.cpp:85-303)
with the semantics fixed by integration_tools/generate_interactive_test_vectors.cpp:383-541:

  stage 1  (coarse)  ct_diff = ct_query - pt_centroids; ct_sq = rescale(ct_diff^2);
                     tree sum with rotations 1, 2, .., D/2
  stage 1b (compact) for i < n_list: mask slot i*D, rescale, rotate by i*(D-1), accumulate
  stage 2  (client)  decrypt, pick the nprobe nearest lists
  stage 3  (fine)    per batch of B = slots/D candidates: ct_dimpack - pt_batch, square,
                     rescale, tree sum with rotations B, 2B, .., B*D/2, mask the first
                     batch_count slots, rescale, rotate by -global_offset, accumulate
  stage 4  (client)  decrypt, sort, top-k

Every operator call processes a whole batch of independent ciphertexts (up to
the context's max_batch per launch; one lane of context scratch each): several queries in stage 1,
several (query, list, batch) items in stage 3. Each ciphertext's residues are
the ones the one-at-a-time chain produces. `lanes=1` is the plain path.

Phase-3 candidate plaintexts depend only on the index, so they are encoded
once and stay resident in HBM (poly_gmem), as do the masks.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .ckks import Encoder, Slots, encode_plaintext
from .driver import FheContext, FHEHostDriver
from .ivfpq import IvfPqIndex

MAX_LANES = 4096


@dataclass
class QueryShape:
    D: int
    n_list: int
    slots: int
    nprobe: int
    top_k: int
    scale: float

    @property
    def B(self) -> int:
        return self.slots // self.D


@dataclass
class QueryRecord:
    ct_query: tuple[int, int]
    ct_dim: tuple[int, int]
    compact: tuple[int, int]
    dists: tuple[int, int]
    probes: list = field(default_factory=list)
    vids: list = field(default_factory=list)       # slot -> vector id (stage 3 order)


def pow2_steps(x: int) -> list[int]:
    """Descending powers of two whose sum is |x| (fhe_host_driver.cpp:383-403)."""
    out, r = [], abs(x)
    while r:
        s = 1 << (r.bit_length() - 1)
        out.append(s)
        r -= s
    return out


class InteractiveQueryManager:
    def __init__(self, ctx: FheContext, index: IvfPqIndex, shape: QueryShape, slots: Slots, lanes: int = MAX_LANES):
        self.ctx, self.index, self.sh = ctx, index, shape
        self.drv = FHEHostDriver(ctx)
        self.lib = ctx.lib
        self.p = ctx.params
        self.L = self.p.L
        self.enc = Encoder(self.p.log_n)
        self.slots = slots
        self.lanes = max(1, min(lanes, MAX_LANES, ctx.max_batch))
        assert shape.n_list * shape.D <= shape.slots, "centroids do not fit one ciphertext"
        L, n = self.L, self.p.n
        self.lvl_sq = L - 1          # after the first rescale
        self.lvl_out = L - 2         # after the mask rescale
        # scale of the results: Delta^2 / q_{L-1}; masks carry q_{L-2} so the second rescale keeps it
        self.out_scale = shape.scale * shape.scale / self.p.q[L - 1]
        mask_scale = float(self.p.q[L - 2])
        D = shape.D
        # ---- resident plaintexts ----
        self.pt_centroids = slots.take(1)[0]
        vals = np.zeros(shape.slots)
        for c in range(index.n_list):
            vals[c * D:(c + 1) * D] = index.centroids[c]
        encode_plaintext(ctx, self.enc, vals, shape.scale, self.pt_centroids, L)
        self.mask_onehot = []
        for i in range(shape.n_list):
            off = slots.take(1)[0]
            m = np.zeros(shape.slots)
            m[i * D] = 1.0
            encode_plaintext(ctx, self.enc, m, mask_scale, off, self.lvl_sq)
            self.mask_onehot.append(off)
        self._mask_scale = mask_scale
        self.mask_prefix: dict[int, int] = {}
        self.batches: list[list[tuple[int, int, list]]] = []
        B = shape.B
        for c in range(index.n_list):
            vl = index.lists[c]
            out = []
            for b0 in range(0, len(vl), B):
                vids = vl[b0:b0 + B]
                rec = index.reconstruct(vids)
                packed = np.zeros(shape.slots)
                for j in range(len(vids)):
                    packed[np.arange(D) * B + j] = rec[j]
                off = slots.take(1)[0]
                encode_plaintext(ctx, self.enc, packed, shape.scale, off, L)
                out.append((off, len(vids), list(vids)))
                self._prefix(len(vids))
            self.batches.append(out)
        # ---- per-lane working ciphertexts ----
        self.work = []
        for _ in range(self.lanes):
            s = slots.take(8)
            self.work.append(dict(diff=(s[0], s[1]), sq=(s[2], s[3]), tmp=(s[4], s[5]), sel=(s[6], s[7])))
        # stage 1b: the n_list - 1 masked ciphertexts of each lane's query,
        # rotated side by side (lvl_out limbs each, packed)
        w = self.lvl_out * n
        per_lane = 2 * (shape.n_list - 1) * w
        base = slots.take(self.compaction_slots(shape.n_list, L, n, slots.w, self.lanes))[0] if per_lane else 0
        self.cmp = [[(base + k * per_lane + 2 * i * w, base + k * per_lane + (2 * i + 1) * w)
                     for i in range(shape.n_list - 1)] for k in range(self.lanes)]

    @staticmethod
    def compaction_slots(n_list: int, L: int, n: int, slot_w: int, lanes: int) -> int:
        """Slots of the stage-1b buffers: n_list - 1 ciphertexts at L - 2 limbs per lane."""
        return -(-lanes * 2 * (n_list - 1) * (L - 2) * n // slot_w)

    def _prefix(self, count: int) -> int:
        if count not in self.mask_prefix:
            off = self.slots.take(1)[0]
            m = np.zeros(self.sh.slots)
            m[:count] = 1.0
            encode_plaintext(self.ctx, self.enc, m, self._mask_scale, off, self.lvl_sq)
            self.mask_prefix[count] = off
        return self.mask_prefix[count]

    def rotation_steps(self, max_candidates: int | None = None) -> set[int]:
        D, B = self.sh.D, self.sh.B
        steps = set()
        s = 1
        while s < D:
            steps.add(s)            # coarse tree sum
            steps.add(B * s)        # fine tree sum
            s <<= 1
        for i in range(self.sh.n_list):
            steps.update(pow2_steps(i * (D - 1)))
        top = max_candidates or self.sh.slots
        s = 1
        while s < top:
            steps.add(-s)           # batch position shifts
            s <<= 1
        return steps

    def new_query(self) -> QueryRecord:
        s = self.slots.take(8)
        return QueryRecord((s[0], s[1]), (s[2], s[3]), (s[4], s[5]), (s[6], s[7]))

    def alloc_queries(self, count: int) -> list[QueryRecord]:
        """Records whose results (compacted coarse distances, candidate
        distances; level lvl_out) are packed back to back in two outboxes, so
        each reaches the host in one copy (read_outbox)."""
        w = self.lvl_out * self.p.n
        k = -(-2 * count * w // self.slots.w)
        comp = self.slots.take(k)[0]
        dist = self.slots.take(k)[0]
        recs = []
        for i in range(count):
            s = self.slots.take(4)
            recs.append(QueryRecord((s[0], s[1]), (s[2], s[3]),
                                    (comp + 2 * i * w, comp + (2 * i + 1) * w),
                                    (dist + 2 * i * w, dist + (2 * i + 1) * w)))
        self._outbox = {"compact": comp, "dists": dist}
        return recs

    def read_outbox(self, kind: str, count: int) -> np.ndarray:
        """(count, 2, lvl_out * N) result ciphertexts of the first `count`
        records from alloc_queries, in one device-to-host copy."""
        w = self.lvl_out * self.p.n
        return self.ctx.read_poly(self._outbox[kind], 2 * count * w).reshape(count, 2, w)

    # ---- batched C-ABI helpers ----
    @staticmethod
    def _refs(cts):
        arr = (L.CtRef * max(len(cts), 1))()
        for i, (a, b) in enumerate(cts):
            arr[i].c0_offset, arr[i].c1_offset = a, b
        return arr

    @staticmethod
    def _offs(v):
        return (L.u64 * max(len(v), 1))(*v)

    def _rotate(self, cts, r, limbs):
        L.check(self.lib.afhe_eval_rotate_batch(self.ctx.h, self._refs(cts), self._refs(cts), len(cts), r, limbs),
                "eval_rotate_batch")

    def _rot_acc(self, src, acc, r, limbs):
        L.check(self.lib.afhe_eval_rotate_accumulate_batch(self.ctx.h, self._refs(src), self._refs(acc), len(src), r,
                                                           limbs), "eval_rotate_accumulate_batch")

    def _add(self, a, b, d, limbs):
        L.check(self.lib.afhe_eval_add_batch(self.ctx.h, self._refs(a), self._refs(b), self._refs(d), len(a), limbs),
                "eval_add_batch")

    def _mult_plain(self, a, pts, d, limbs):
        L.check(self.lib.afhe_eval_mult_plain_rescale_batch(self.ctx.h, self._refs(a), self._offs(pts), self._refs(d),
                                                            len(a), limbs), "eval_mult_plain_rescale_batch")

    def _square(self, a, d, limbs):
        L.check(self.lib.afhe_eval_mult_relin_rescale_batch(self.ctx.h, self._refs(a), self._refs(a), self._refs(d),
                                                            len(a), limbs), "eval_mult_relin_rescale_batch")

    def _sub_plain(self, a, pts, d, limbs):
        L.check(self.lib.afhe_eval_sub_plain_batch(self.ctx.h, self._refs(a), self._offs(pts), self._refs(d), len(a),
                                                   limbs), "eval_sub_plain_batch")

    # ---- stages ----
    def stage1_coarse(self, queries: list[QueryRecord]) -> None:
        """Stages 1 and 1b for every query (lanes at a time)."""
        D, Ll = self.sh.D, self.L
        for c0 in range(0, len(queries), self.lanes):
            qs = queries[c0:c0 + self.lanes]
            w = self.work[:len(qs)]
            diff = [x["diff"] for x in w]
            sq = [x["sq"] for x in w]
            tmp = [x["tmp"] for x in w]
            sel = [x["sel"] for x in w]
            self._sub_plain([q.ct_query for q in qs], [self.pt_centroids] * len(qs), diff, Ll)
            self._square(diff, sq, Ll)
            s = 1
            while s < D:                     # sq += rot(sq, s)
                self._rot_acc(sq, sq, s, self.lvl_sq)
                s <<= 1
            self._compact(qs, sq)

    def _compact(self, qs: list[QueryRecord], sq) -> None:
        """Stage 1b for a chunk of queries: compact = sum over i of
        rot(rescale(sq * mask_i), i * (D - 1)).

        The reference runs the lists one after another, each rotation as
        eval_rotate's descending power-of-two steps, accumulating as it goes.
        Here every (query, list) term is masked in one batched operator. The
        rotations run step by step from the highest power of two down: each
        step rotates, in one batched launch, every term whose shift has that
        bit. So each term sees exactly its eval_rotate steps, in the same
        order, and its residues are the reference's. The terms are then
        summed pairwise. Modular addition is exact and commutative, so the
        sum equals the reference's running accumulation word for word. The
        depth is log2(max shift) rotations plus log2(n_list) additions,
        instead of one eval_rotate after another."""
        D, nl = self.sh.D, self.sh.n_list
        comp = [q.compact for q in qs]
        src, pts, dst = [], [], []
        for k in range(len(qs)):
            for i in range(nl):
                src.append(sq[k])
                pts.append(self.mask_onehot[i])
                dst.append(comp[k] if i == 0 else self.cmp[k][i - 1])
        self._mult_plain(src, pts, dst, self.lvl_sq)
        if nl == 1:
            return
        terms = [(self.cmp[k][i - 1], i * (D - 1)) for k in range(len(qs)) for i in range(1, nl)]
        top = max(s for _, s in terms).bit_length()
        for b in range(top - 1, -1, -1):
            sub = [ct for ct, s in terms if (s >> b) & 1]
            if sub:
                self._rotate(sub, 1 << b, self.lvl_out)
        # per query: comp += sum of its n_list - 1 rotated terms
        groups = [[comp[k]] + self.cmp[k] for k in range(len(qs))]
        self._sum_groups(groups, self.lvl_out)

    def _sum_groups(self, groups, limbs: int) -> None:
        """groups[g][0] += groups[g][1] + ... , all groups side by side, by
        pairwise batched additions (depth log2 of the largest group)."""
        live = [list(g) for g in groups]
        while any(len(g) > 1 for g in live):
            a, b = [], []
            for g in live:
                for j in range(0, len(g) - 1, 2):
                    a.append(g[j])
                    b.append(g[j + 1])
            self._add(a, b, a, limbs)
            live = [g[0::2] for g in live]

    def stage3_fine(self, queries: list[QueryRecord]) -> None:
        """Stage 3 for every (query, probed list, batch) item, lanes at a time.
        Each query's `probes` must be set (stage 2)."""
        D, B, Ll = self.sh.D, self.sh.B, self.L
        items = []
        for qi, q in enumerate(queries):
            off = 0
            q.vids = []
            for c in q.probes:
                for pt, cnt, vids in self.batches[c]:
                    items.append((qi, pt, cnt, off))
                    q.vids.extend(vids)
                    off += cnt
        for c0 in range(0, len(items), self.lanes):
            it = items[c0:c0 + self.lanes]
            w = self.work[:len(it)]
            diff = [x["diff"] for x in w]
            sq = [x["sq"] for x in w]
            tmp = [x["tmp"] for x in w]
            sel = [x["sel"] for x in w]
            self._sub_plain([queries[x[0]].ct_dim for x in it], [x[1] for x in it], diff, Ll)
            self._square(diff, sq, Ll)
            s = B
            while s < D * B:                 # sq += rot(sq, s)
                self._rot_acc(sq, sq, s, self.lvl_sq)
                s <<= 1
            self._mult_plain(sq, [self._prefix(x[2]) for x in it], sel, self.lvl_sq)
            # rotate each item by -offset: the same descending power-of-two steps
            # as eval_rotate, grouped across items step by step
            top = max((x[3] for x in it), default=0).bit_length()
            for b in range(top - 1, -1, -1):
                sub = [sel[k] for k, x in enumerate(it) if (x[3] >> b) & 1]
                if sub:
                    self._rotate(sub, -(1 << b), self.lvl_out)
            # accumulate: each query's items of this chunk are summed pairwise
            # (exact modular additions, so the order does not change a word);
            # the chunk holding the query's offset-0 item starts its sum.
            byq: dict[int, list[int]] = {}
            for k, x in enumerate(it):
                byq.setdefault(x[0], []).append(k)
            self._sum_groups([[sel[k] for k in ks] for ks in byq.values()], self.lvl_out)
            w_ = self.lvl_out * self.p.n
            adds = []
            for qi, ks in byq.items():
                dst, head = queries[qi].dists, sel[ks[0]]
                if any(it[k][3] == 0 for k in ks):
                    L.check(self.lib.afhe_copy_poly(self.ctx.h, dst[0], head[0], w_), "copy_poly")
                    L.check(self.lib.afhe_copy_poly(self.ctx.h, dst[1], head[1], w_), "copy_poly")
                else:
                    adds.append((dst, head))
            if adds:
                self._add([d for d, _ in adds], [h for _, h in adds], [d for d, _ in adds], self.lvl_out)

    # ---- result transfer ----
    def read_ct(self, ct: tuple[int, int]) -> tuple[np.ndarray, np.ndarray]:
        w = self.lvl_out * self.p.n
        return self.ctx.read_poly(ct[0], w), self.ctx.read_poly(ct[1], w)
