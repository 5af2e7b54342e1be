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
            comp = [q.compact for q in qs]
            for i in range(self.sh.n_list):
                shift = i * (D - 1)
                tgt = comp if i == 0 else sel
                self._mult_plain(sq, [self.mask_onehot[i]] * len(qs), tgt, self.lvl_sq)
                if shift:                    # comp += rot(sel, i * (D - 1))
                    self._rot_acc(sel, comp, shift, self.lvl_out)

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
            # accumulate: the item at offset 0 starts its query's sum
            pending = []
            n = self.p.n
            for k, x in enumerate(it):
                dst = queries[x[0]].dists
                if x[3] == 0:
                    w_ = self.lvl_out * n
                    L.check(self.lib.afhe_copy_poly(self.ctx.h, dst[0], sel[k][0], w_), "copy_poly")
                    L.check(self.lib.afhe_copy_poly(self.ctx.h, dst[1], sel[k][1], w_), "copy_poly")
                else:
                    pending.append((dst, sel[k]))
            while pending:
                seen, now, later = set(), [], []
                for dst, src in pending:
                    (later if dst in seen else now).append((dst, src))
                    seen.add(dst)
                self._add([d for d, _ in now], [s_ for _, s_ in now], [d for d, _ in now], self.lvl_out)
                pending = later

    # ---- result transfer ----
    def read_ct(self, ct: tuple[int, int]) -> tuple[np.ndarray, np.ndarray]:
        w = self.lvl_out * self.p.n
        return self.ctx.read_poly(ct[0], w), self.ctx.read_poly(ct[1], w)
