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

Three compactions:
  * "reference": the chain above, verbatim, for indexes whose centroids fit
    one ciphertext (n_list * D <= slots);
  * "packed", for larger indexes: the centroids span n_coarse = n_list /
    (slots / D) ciphertexts, centroid k * (slots / D) + c at slot c * D of
    coarse ciphertext k. Each coarse ciphertext's tree sum is masked at every
    slot c * D at once, rescaled, rotated right by k and summed, so one
    ciphertext returns all n_list distances (list k * (slots / D) + c at slot
    c * D + k). That takes n_coarse - 1 key switches per query instead of
    the reference's sum over lists of popcount(i * (D - 1)).
    The packed chain also places candidates without a key switch: candidate
    batch t of a query starts at slot (t mod (slots / B)) * B of result
    t // (slots / B). Its tree sum runs over all D rows of B slots, so every
    row already holds the batch's B sums; the prefix mask moved to row
    t mod (slots / B) (an automorphism of the plaintext) selects them there,
    instead of masking row 0 and rotating by the offset with
    popcount(offset) key switches.
  * "diagonal": the inner products by the diagonal method (baby-step
    giant-step). The query, repeated every D slots, is rotated by b = 1 ..
    n1 - 1 once per query (the baby steps, kept for stage 3). The distance
    of the candidate in slot j is ||q||^2 - 2 <q, x_j> + ||x_j||^2 with
    -2 <q, x_j> = sum over g < n2 of rot(sum over b < n1 of pt_{g,b} *
    rot(q, b), n1 g), pt_{g,b} the (pre-rotated) diagonal g n1 + b of the
    candidates x dims matrix: n2 - 1 giant-step key switches per output
    ciphertext instead of log2 D per candidate batch. Stage 1 treats the
    centroids as one such matrix (coarse distance of list c in slot c).
    Stage 3's plaintexts are built once per unit (a list, or N/2 candidates
    of it) and placed at the unit's output offset, a multiple of D, by an
    automorphism of the plaintext folded into the product's loads
    (afhe_eval_mac_plain_batch); ||q||^2 (the client's ciphertext, sent in
    place of ct_dim) and the placed unit norms are added. Depth 1: results
    at l - 1 limbs. Slots outside the probed units hold ||q||^2 alone.
In the reference chain, candidate distances past `slots` continue in further
result ciphertexts (position p at slot p mod slots of result p // slots). A
candidate batch never straddles two results: one that would not fit starts
the next result, so every batch lands whole in one ciphertext.

Phase-3 candidate plaintexts depend only on the index, so they are encoded
once and stay resident in HBM (poly_gmem), as do the masks.

By default the stages run in C++ (afhe_ivfpq_stage1 / afhe_ivfpq_stage3 in
libafhe.so, csrc/ivfpq.cu): this class encodes the plaintexts, registers their
offsets with the native driver and keeps the host bookkeeping (candidate ids,
slot positions). `native=False` runs the same stages from Python over the
batched C ABI; both issue the same operators and give identical residues.
"""
from __future__ import annotations

import ctypes as C
import itertools
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .ckks import Encoder, Slots, encode_index_batches, encode_plaintext, encode_plaintexts
from .driver import FheContext, FHEHostDriver, galois_elt
from .ivfpq import IvfPqIndex

MAX_LANES = 4096
# HBM for the packed chain's candidate-norm plaintexts (the expanded distance):
# (l - 1) N words per candidate batch and evaluation level l. Levels are
# prepared lowest first while they fit; the rest square the difference.
NORM_BUDGET_BYTES = 32 << 30


@dataclass
class QueryShape:
    D: int
    n_list: int
    slots: int
    nprobe: int
    top_k: int
    scale: float
    compaction: str = "reference"
    eval_level: int | None = None   # limbs the server evaluates at (None: the query's level)

    @property
    def B(self) -> int:
        return self.slots // self.D

    @property
    def per_ct(self) -> int:
        """Centroids per coarse ciphertext (one every D slots)."""
        return self.slots // self.D

    @property
    def n_coarse(self) -> int:
        if self.compaction == "diagonal":
            return 1
        return -(-self.n_list // self.per_ct)

    @property
    def n1(self) -> int:
        """Baby steps of the diagonal method: 2^ceil(log2(D) / 2)."""
        return 1 << ((self.D.bit_length() - 1 + 1) // 2)

    @property
    def n2(self) -> int:
        """Giant steps of the diagonal method: D / n1."""
        return self.D // self.n1

    @property
    def depth(self) -> int:
        """Rescales of the chain (limbs the results lose)."""
        return 1 if self.compaction == "diagonal" else 2

    def coarse_slot(self, lst: int) -> int:
        """Slot of list `lst`'s distance in the compacted coarse ciphertext."""
        if self.compaction in ("reference", "diagonal"):
            return lst
        return (lst % self.per_ct) * self.D + lst // self.per_ct


@dataclass
class QueryRecord:
    ct_query: tuple[int, int]
    ct_dim: tuple[int, int]        # diagonal chain: ||q||^2 in every slot (the client's), evaluation level - 1
    compact: tuple[int, int]
    dists: tuple[int, int]                          # the first result ciphertext
    probes: list = field(default_factory=list)
    vids: list = field(default_factory=list)       # candidate vector ids (stage 3 order)
    pos: list = field(default_factory=list)        # slot position of each candidate across the results
    results: list = field(default_factory=list)    # every result ciphertext (dists first)
    level: int = 0          # limbs of the encrypted query (0: the top level L)
    nprobe: int = 0         # lists the client selects (0: the shape's nprobe)
    norm: tuple | None = None   # packed chain: ||q||^2 (at the evaluation level - 1)
    baby: list = field(default_factory=list)       # diagonal chain: the query rotated by 1 .. n1 - 1
    layout: list = field(default_factory=list)     # diagonal chain: (unit, slot offset) per probed unit


def batch_offsets(counts, slots: int, align: int | None = None) -> list[int]:
    """Slot offsets of consecutive candidate batches across the result
    ciphertexts: back to back, except that a batch that would cross a
    result's end starts the next result (offset a multiple of `slots`).
    With `align` (a divisor of `slots`, at least every count), batch t starts
    at t * align instead."""
    if align:
        return [t * align for t in range(len(counts))]
    out, off = [], 0
    for cnt in counts:
        if off % slots + cnt > slots:
            off = (off // slots + 1) * slots
        out.append(off)
        off += cnt
    return out


def unit_offsets(counts, slots: int, D: int) -> list[int]:
    """Slot offsets of consecutive units of the diagonal chain (counts <=
    slots): each spans its count rounded up to a multiple of D, back to back,
    except that a unit that would cross a result's end starts the next
    result."""
    out, off = [], 0
    for cnt in counts:
        span = -(-cnt // D) * D
        if off % slots + span > slots:
            off = (off // slots + 1) * slots
        out.append(off)
        off += span
    return out


def pow2_steps(x: int) -> list[int]:
    """Descending powers of two whose sum is |x| (fhe_host_driver.cpp:383-403)."""
    out, r = [], abs(x)
    while r:
        s = 1 << (r.bit_length() - 1)
        out.append(s)
        r -= s
    return out


class InteractiveQueryManager:
    """The server chain over many queries. A query encrypted at level l runs
    the chain at l: results at l - 2 limbs with scale Delta^2 / q_{l-1}. The
    index's plaintexts are encoded once at the top level L. A plaintext at L
    restricted to its first l limbs is the same plaintext at level l. Masks
    are encoded per level, at scale q_{l-2}, the prime the mask rescale drops.
    `levels` lists the query levels to prepare masks for (default: L only).
    `max_nprobe` sizes the result ciphertexts (default: the shape's nprobe).
    `norm_budget`: bytes of candidate-norm plaintexts (packed chain) the
    slots hold room for (default NORM_BUDGET_BYTES)."""

    def __init__(self, ctx: FheContext, index: IvfPqIndex, shape: QueryShape, slots: Slots, lanes: int = MAX_LANES,
                 levels=None, max_nprobe: int | None = None, native: bool = True, norm_budget: int | None = None):
        self.ctx, self.index, self.sh = ctx, index, shape
        self.native = native
        self._nh, self._nh_key, self._nh_ver = None, None, 0
        self.drv = FHEHostDriver(ctx)
        self.lib = ctx.lib
        self.p = ctx.params
        self.L = self.p.L
        self.enc = Encoder(self.p.log_n)
        self.slots = slots
        self.lanes = max(1, min(lanes, MAX_LANES, ctx.max_batch))
        if shape.compaction == "reference":
            assert shape.n_list * shape.D <= shape.slots, "centroids do not fit one ciphertext"
        elif shape.compaction == "diagonal":
            assert shape.n_list <= shape.slots, "the centroids must fit one ciphertext"
            assert shape.D & (shape.D - 1) == 0 and shape.slots % shape.D == 0, "D: a power of two dividing slots"
        else:
            assert shape.compaction == "packed" and shape.n_coarse <= shape.D, "unsupported compaction"
        L, n = self.L, self.p.n
        self.lvl_sq = L - 1          # after the first rescale
        self.lvl_out = L - 2         # after the mask rescale
        # scale of the results: Delta^2 / q_{L-1}; masks carry q_{L-2} so the second rescale keeps it
        self.out_scale = shape.scale * shape.scale / self.p.q[L - 1]
        mask_scale = float(self.p.q[L - 2])
        self._mask_scale = mask_scale
        D, S = shape.D, shape.slots
        # the client decrypts results from limb 0 alone: every decrypted
        # coefficient (a distance times out_scale, plus noise) must stay well
        # inside +-q_0 / 2; distances are at most (|q| + |x|)^2 <= 4 max |x|^2
        bound = 4.0 * float(np.max((index.centroids.astype(np.float64) ** 2).sum(1))) * 4.0 + 64.0
        assert bound * self.out_scale * 4 < self.p.q[0] / 2, "results would not decrypt from limb 0"
        self._bound = bound
        if shape.compaction == "diagonal":
            self._init_diagonal(levels, max_nprobe)
            return
        # ---- resident plaintexts ----
        self.pt_centroid_cts = slots.take(shape.n_coarse)
        self.pt_centroids = self.pt_centroid_cts[0]
        vals = np.zeros((shape.n_coarse, S))
        for c in range(index.n_list):
            k, j = divmod(c, shape.per_ct)
            vals[k, j * D:(j + 1) * D] = index.centroids[c]
        encode_plaintexts(ctx, self.enc, vals, shape.scale, self.pt_centroid_cts, L)
        assert shape.eval_level is None or 3 <= shape.eval_level <= L, "eval_level must be in [3, L]"
        self._query_levels = set(levels or [L]) | {L}
        self._bound = bound
        self.levels = sorted({self.eval_at(lv) for lv in self._query_levels})
        assert all(3 <= lv <= L for lv in self.levels), "query levels must be in [3, L]"
        self._onehot: dict[int, list[int]] = {}      # level -> one-hot masks (reference compaction)
        self._stride: dict[int, int] = {}             # level -> centroid-slot mask (packed compaction)
        self._prefix_lv: dict[tuple[int, int], int] = {}
        self._counts: list[int] = []
        for lv in self.levels:
            self._level_masks(lv)
        top = self.levels[-1]                  # the level top-level queries are evaluated at
        self.mask_onehot = self._onehot.get(top, [])
        if shape.compaction == "packed":
            self.mask_stride = self._stride[top]
        self.mask_prefix: dict[int, int] = {}
        B = shape.B
        self.batches: list[list[tuple[int, int, list]]] = []
        counts, bvids, bfirst, bcnt, boffs = set(), [], [], [], []
        for c in range(index.n_list):
            vl = index.lists[c]
            out = []
            for b0 in range(0, len(vl), B):
                vids = vl[b0:b0 + B]
                off = slots.take(1)[0]
                bfirst.append(len(bvids))
                bcnt.append(len(vids))
                bvids.extend(vids)
                boffs.append(off)
                out.append((off, len(vids), list(vids)))
                counts.add(len(vids))
            self.batches.append(out)
        # built on the device from the index: slot d * B + j = x_j[d] (x_j the
        # reconstruction of candidate j: centroid + PQ codewords)
        if boffs:
            encode_index_batches(ctx, index, bvids, bfirst, bcnt, boffs, shape.scale, L)
        self._bvids, self._bfirst, self._bcnt = bvids, bfirst, bcnt
        self._first_batch = np.concatenate([[0], np.cumsum([len(b) for b in self.batches])]).astype(int).tolist()
        # packed chain: the candidates' squared norms per level, for the
        # expanded distance ||q||^2 - 2 <q, x_j> + ||x_j||^2
        self._norms: dict[int, list[int]] = {}
        self._norm_left = (NORM_BUDGET_BYTES if norm_budget is None else norm_budget) // 8
        if shape.compaction == "packed":
            for lv in self.levels:
                self._norm_plaintexts(lv)
        self._counts = sorted(counts)
        for lv in self.levels:
            self._prefix_masks(lv)
        self.mask_prefix = {cnt: self._prefix_lv[(cnt, top)] for cnt in counts}
        # result ciphertexts per query: enough for the largest lists a query may probe
        self.max_nprobe = max(max_nprobe or shape.nprobe, shape.nprobe)
        self.n_res = self.results_for(index, shape, self.max_nprobe)
        # ---- per-lane working ciphertexts ----
        self.work = []
        for _ in range(self.lanes):
            s = slots.take(8)
            self.work.append(dict(diff=(s[0], s[1]), sq=(s[2], s[3]), tmp=(s[4], s[5]), sel=(s[6], s[7])))
        # stage 1b (reference compaction): the n_list - 1 masked ciphertexts of
        # each lane's query, rotated side by side (lvl_out limbs each, packed)
        self.cmp = []
        if shape.compaction == "reference" and shape.n_list > 1:
            w = self.lvl_out * n
            per_lane = 2 * (shape.n_list - 1) * w
            base = slots.take(self.compaction_slots(shape.n_list, L, n, slots.w, self.lanes))[0]
            self.cmp = [[(base + k * per_lane + 2 * i * w, base + k * per_lane + (2 * i + 1) * w)
                         for i in range(shape.n_list - 1)] for k in range(self.lanes)]

    # ---- the diagonal chain: resident plaintexts ----
    def _init_diagonal(self, levels, max_nprobe) -> None:
        """Units (a list, or N/2 candidates of it), then per evaluation level
        lv the centroids' and every unit's D diagonals (lv limbs, scale Delta,
        times -2) and squared norms (lv - 1 limbs, scale Delta^2 / q_{lv-1}),
        all built and encoded on the device; n_res results per query; a pool
        of `lanes` working ciphertexts for the inner products."""
        sh, n, S = self.sh, self.p.n, self.sh.slots
        assert sh.eval_level is None or 2 <= sh.eval_level <= self.L, "eval_level must be in [2, L]"
        self._query_levels = set(levels or [self.L]) | {self.L}
        self.levels = sorted({self.eval_at(lv) for lv in self._query_levels})
        assert all(2 <= lv <= self.L for lv in self.levels), "evaluation levels must be in [2, L]"
        self._onehot, self._stride, self._prefix_lv, self._counts = {}, {}, {}, []
        self._norms, self.mask_prefix, self.cmp, self.batches = {}, {}, [], []
        self.pt_centroid_cts = []
        self.units: list[tuple[int, list]] = []       # (list, candidate ids)
        self.list_units: list[list[int]] = []
        uvids, ufirst, ucnt = [], [], []
        for c in range(self.index.n_list):
            vl = [int(v) for v in self.index.lists[c]]
            us = []
            for u0 in range(0, len(vl), S):
                part = vl[u0:u0 + S]
                us.append(len(self.units))
                self.units.append((c, part))
                ufirst.append(len(uvids))
                ucnt.append(len(part))
                uvids.extend(part)
            self.list_units.append(us)
        self._uvids, self._ufirst, self._ucnt = uvids, ufirst, ucnt
        self._gal_cache: dict[int, int] = {}
        self._diag: dict[int, dict] = {}
        for lv in self.levels:
            self._diag_plaintexts(lv)
        self.max_nprobe = max(max_nprobe or sh.nprobe, sh.nprobe)
        self.n_res = self.results_for(self.index, sh, self.max_nprobe)
        top = self.levels[-1]
        self.lvl_out = top - 1                 # results of the highest evaluation level
        self._baby_limbs = top
        w = top * n
        pool = self.inner_pool(self.lanes, sh.n2)
        base = self.slots.take(-(-2 * pool * w // self.slots.w))[0]
        self._inner = [(base + 2 * k * w, base + (2 * k + 1) * w) for k in range(pool)]
        self.work = []

    @staticmethod
    def diagonal_values(X: np.ndarray, S: int, D: int, n1: int, coef: float = -2.0) -> np.ndarray:
        """The D pre-rotated diagonals of the (rows x D) matrix X as slot
        vectors: row i = g n1 + b, slot k = coef X[j, (j + i) mod D] with
        j = (k - n1 g) mod S, 0 for j >= rows (afhe_pq_encode_diagonals'
        layout, for matrices given on the host)."""
        rows = X.shape[0]
        out = np.zeros((D, S))
        k = np.arange(S)
        for i in range(D):
            j = (k - (i // n1) * n1) % S
            ok = j < rows
            jj = j[ok]
            out[i, ok] = coef * X[jj, (jj + i) % D]
        return out

    def _diag_plaintexts(self, lv: int) -> None:
        sh, n, S, D, n1 = self.sh, self.p.n, self.sh.slots, self.sh.D, self.sh.n1
        sc = sh.scale * sh.scale / self.p.q[lv - 1]

        def region(count: int, limbs: int) -> list[int]:
            if count == 0:
                return []
            base = self.slots.take(-(-count * limbs * n // self.slots.w))[0]
            return [base + i * limbs * n for i in range(count)]

        cent = self.index.centroids.astype(np.float64)
        d = dict(cent=region(D, lv), cnorm=region(1, lv - 1)[0],
                 pts=np.asarray(region(len(self.units) * D, lv), dtype=np.uint64),
                 norms=np.asarray(region(len(self.units), lv - 1), dtype=np.uint64))
        encode_plaintexts(self.ctx, self.enc, self.diagonal_values(cent, S, D, n1), sh.scale, d["cent"], lv)
        cn = np.zeros((1, S))
        cn[0, :len(cent)] = (cent ** 2).sum(1)
        encode_plaintexts(self.ctx, self.enc, cn, sc, [d["cnorm"]], lv - 1)
        if self.units:
            args = (self.ctx, self.index, self._uvids, self._ufirst, self._ucnt)
            encode_index_batches(*args, d["pts"], sh.scale, lv, layout="diagonals", n1=n1, coef=-2.0)
            encode_index_batches(*args, d["norms"], sc, lv - 1, layout="unit_norms")
        self._diag[lv] = d
        self._nh_ver += 1

    @staticmethod
    def diagonal_slots(units: int, D: int, lv: int, n: int, slot_w: int) -> int:
        """Slots of one evaluation level's diagonal-chain plaintexts (the
        centroids' D diagonals and norms, the units' D diagonals and norms,
        each group packed back to back)."""
        return sum(-(-count * limbs * n // slot_w) for count, limbs in
                   ((D, lv), (1, lv - 1), (units * D, lv), (units, lv - 1)) if count)

    @staticmethod
    def inner_pool(lanes: int, n2: int) -> int:
        """Working ciphertexts of the inner products: n2 giant steps for each
        of up to 64 outputs per round (measured on the large configuration:
        32-128 outputs per round within 1% of each other; 256 was 4% slower
        on the device, its working set four times larger)."""
        return max(1, min(lanes, 64)) * n2

    @classmethod
    def diagonal_scratch_slots(cls, queries: int, lanes: int, n1: int, n2: int, top: int, n: int,
                               slot_w: int) -> int:
        """Slots of the queries' baby steps and the inner-product pool (top
        limbs each)."""
        return (-(-2 * queries * (n1 - 1) * top * n // slot_w)
                + -(-2 * cls.inner_pool(lanes, n2) * top * n // slot_w))

    def unit_offsets(self, probes) -> list[tuple[int, int]]:
        """(unit, slot offset across the results) for a query's probed lists,
        in probe order: each unit's slots start at a multiple of D (the
        plaintext placement keeps the diagonals aligned to the query's
        period), back to back, a unit that would cross a result's end
        starting the next result."""
        us = [u for c in probes for u in self.list_units[c]]
        return list(zip(us, unit_offsets([len(self.units[u][1]) for u in us], self.sh.slots, self.sh.D)))

    def _level_masks(self, lv: int) -> None:
        """The compaction masks of level lv, at scale q_{lv-2} (the prime the
        mask rescale drops)."""
        sh, S, D = self.sh, self.sh.slots, self.sh.D
        assert self._bound * self.out_scale_at(lv) * 4 < self.p.q[0] / 2, "results would not decrypt from limb 0"
        ms = float(self.p.q[lv - 2])
        if sh.compaction == "reference":
            m = np.zeros((sh.n_list, S))
            m[np.arange(sh.n_list), np.arange(sh.n_list) * D] = 1.0
            self._onehot[lv] = self.slots.take(sh.n_list)
            encode_plaintexts(self.ctx, self.enc, m, ms, self._onehot[lv], lv - 1)
        else:
            m = np.zeros((1, S))
            m[0, np.arange(sh.per_ct) * D] = 1.0
            self._stride[lv] = self.slots.take(1)[0]
            encode_plaintexts(self.ctx, self.enc, m, ms, [self._stride[lv]], lv - 1)

    def _norm_plaintexts(self, lv: int) -> None:
        """The candidate batches' squared norms at level lv - 1, scale
        Delta^2 / q_{lv-1} (the scale of <q, x_j> and ||q||^2 after their
        rescale), packed back to back. A level they do not fit the budget
        for keeps the unexpanded distance (the square of the difference)."""
        nb = len(self._bcnt)
        w1 = (lv - 1) * self.p.n
        k = self.norm_plaintext_slots(nb, lv, self.p.n, self.slots.w)
        if k * self.slots.w > self._norm_left:
            return
        self._norm_left -= k * self.slots.w
        base = self.slots.take(k)[0] if nb else 0
        offs = [base + b * w1 for b in range(nb)]
        if nb:
            encode_index_batches(self.ctx, self.index, self._bvids, self._bfirst, self._bcnt, offs,
                                 self.sh.scale * self.sh.scale / self.p.q[lv - 1], lv - 1, norms=True)
        self._norms[lv] = offs
        self._nh_ver += 1

    def _prefix_masks(self, lv: int) -> None:
        """Masks of the first `count` slots, for every candidate-batch size."""
        cs = self._counts
        m = np.zeros((len(cs), self.sh.slots))
        for r, cnt in enumerate(cs):
            m[r, :cnt] = 1.0
        offs = self.slots.take(len(cs))
        encode_plaintexts(self.ctx, self.enc, m, float(self.p.q[lv - 2]), offs, lv - 1)
        for cnt, off in zip(cs, offs):
            self._prefix_lv[(cnt, lv)] = off

    def set_eval_level(self, level: int | None) -> None:
        """Change the limbs the server evaluates queries at (None: each query's
        own level). Masks for levels not prepared yet are encoded now (the
        Workload reserves their slots). Call it between steps, with no query
        in flight. The diagonal chain only moves between levels prepared at
        construction (its plaintexts take D limbs per candidate slot and level)."""
        if self.sh.compaction == "diagonal":
            old = self.sh.eval_level
            self.sh.eval_level = level
            if any(self.eval_at(x) not in self._diag for x in self._query_levels):
                self.sh.eval_level = old
                raise ValueError("the diagonal chain has no plaintexts at that evaluation level")
            self._nh_ver += 1
            return
        assert level is None or 3 <= level <= self.L, "eval_level must be in [3, L]"
        self.sh.eval_level = level
        for lv in sorted({self.eval_at(x) for x in self._query_levels}):
            if lv not in self.levels:
                self._level_masks(lv)
                self._prefix_masks(lv)
                if self.sh.compaction == "packed":
                    self._norm_plaintexts(lv)
                self.levels = sorted(self.levels + [lv])
        self._nh_ver += 1

    @staticmethod
    def compaction_slots(n_list: int, L: int, n: int, slot_w: int, lanes: int) -> int:
        """Slots of the stage-1b buffers of the reference compaction: n_list - 1
        ciphertexts at L - 2 limbs per lane."""
        return -(-lanes * 2 * max(n_list - 1, 0) * (L - 2) * n // slot_w)

    @staticmethod
    def results_needed(candidates: int, slots: int, B: int) -> int:
        """Result ciphertexts for `candidates`: a result may end up to B - 1
        slots short, because batches do not straddle results."""
        return max(1, -(-candidates // (slots - B + 1)))

    @staticmethod
    def results_for(index: IvfPqIndex, shape: QueryShape, nprobe: int) -> int:
        """Result ciphertexts a query probing `nprobe` lists may need."""
        B, S = shape.B, shape.slots
        if shape.compaction == "diagonal":      # units of <= S candidates, each over a multiple of D slots
            spans = sorted((-(-min(len(v) - u0, S) // shape.D) * shape.D for v in index.lists
                            for u0 in range(0, len(v), S)), reverse=True)
            per_list = sorted((-(-len(v) // S) for v in index.lists), reverse=True)[:nprobe]
            total = sum(sorted((sum(-(-min(len(v) - u0, S) // shape.D) * shape.D for u0 in range(0, len(v), S))
                                for v in index.lists), reverse=True)[:nprobe])
            # a result closes only when the next unit does not fit: it holds
            # more than S - (largest span) + D slots, and at least one unit
            widest = spans[0] if spans else shape.D
            return max(1, min(sum(per_list), -(-total // (S - widest + shape.D))))
        if shape.compaction == "packed":        # aligned batches: S / B per result
            most = sum(sorted((-(-len(v) // B) for v in index.lists), reverse=True)[:nprobe])
            return max(1, -(-most // (S // B)))
        most = sum(sorted((len(v) for v in index.lists), reverse=True)[:nprobe])
        return InteractiveQueryManager.results_needed(most, S, B)

    @staticmethod
    def mask_slots(shape: QueryShape, levels: int, n_list_masks: bool) -> int:
        """Slots the per-level masks take: one-hot masks (reference compaction)
        or one stride mask, plus up to B prefix masks, per level."""
        return levels * ((shape.n_list if n_list_masks else 1) + shape.B)

    def eval_at(self, level: int) -> int:
        """Limbs the chain runs at for a query encrypted at `level`. The chain
        has multiplicative depth 2 (square, mask). A ciphertext's first l
        limbs are that ciphertext mod Q_l: same message, same scale. So with
        `eval_level` the server drops every limb it does not need before the
        first operator, and every key switch runs on eval_level limbs."""
        return min(level, self.sh.eval_level or level)

    def level_of(self, rec: QueryRecord) -> int:
        return self.eval_at(rec.level or self.L)

    def out_scale_at(self, lv: int) -> float:
        """Scale of the results of a query encrypted at level lv."""
        return self.sh.scale * self.sh.scale / self.p.q[lv - 1]

    def _prefix(self, count: int, lv: int | None = None) -> int:
        """Mask of the first `count` slots for a query at level lv (prepared
        for every candidate-batch size at construction)."""
        lv = lv or self.L
        key = (count, lv)
        if key not in self._prefix_lv:
            off = self.slots.take(1)[0]
            m = np.zeros(self.sh.slots)
            m[:count] = 1.0
            encode_plaintext(self.ctx, self.enc, m, float(self.p.q[lv - 2]), off, lv - 1)
            self._prefix_lv[key] = off
            self._nh_ver += 1
        return self._prefix_lv[key]

    @staticmethod
    def _by_level(recs, level_of):
        groups: dict[int, list[int]] = {}
        for i, r in enumerate(recs):
            groups.setdefault(level_of(r), []).append(i)
        return sorted(groups.items(), reverse=True)

    def rotation_steps(self) -> set[int]:
        return self.steps_for(self.sh)

    @staticmethod
    def steps_for(sh: QueryShape) -> set[int]:
        """Rotation keys the chain needs."""
        D, B = sh.D, sh.B
        if sh.compaction == "diagonal":
            return set(range(1, sh.n1)) | {sh.n1 * g for g in range(1, sh.n2)}     # baby and giant steps
        steps = set()
        s = 1
        while s < D:
            steps.add(s)            # coarse tree sum
            steps.add(B * s)        # fine tree sum
            s <<= 1
        if sh.compaction == "reference":
            for i in range(sh.n_list):
                steps.update(pow2_steps(i * (D - 1)))
            s = 1
            while s < sh.slots:
                steps.add(-s)       # batch position shifts, power-of-two steps
                s <<= 1
        else:
            steps.update(-k for k in range(1, sh.n_coarse))          # coarse packing, one step each
            # batch placement moves the plaintext mask instead: no key
        return steps

    def new_query(self) -> QueryRecord:
        if self.sh.compaction == "diagonal":
            return self.alloc_queries(1)[0]
        s = self.slots.take(10 if self.sh.compaction == "packed" else 8)
        return QueryRecord((s[0], s[1]), (s[2], s[3]), (s[4], s[5]), (s[6], s[7]), results=[(s[6], s[7])],
                           norm=(s[8], s[9]) if self.sh.compaction == "packed" else None)

    @staticmethod
    def norm_slots(count: int, L: int, n: int, slot_w: int) -> int:
        """Slots of the queries' ||q||^2 scratch (packed chain): 2 (L - 1) N
        words per query, packed back to back."""
        return -(-2 * count * (L - 1) * n // slot_w)

    @staticmethod
    def norm_plaintext_slots(batches: int, L: int, n: int, slot_w: int) -> int:
        """Slots of one level's candidate-norm plaintexts (at most L - 1 limbs
        each), packed back to back."""
        return -(-batches * (L - 1) * n // slot_w)

    @classmethod
    def norm_reserve_slots(cls, levels, spare: int, batches: int, L: int, n: int, slot_w: int,
                           budget: int = NORM_BUDGET_BYTES) -> int:
        """Slots to reserve for the candidate norms of the evaluation `levels`
        (lowest first) and `spare` more levels (any up to L), within `budget`
        bytes: what a manager given norm_budget = slots * slot_w * 8 takes."""
        cap, total = budget // 8 // slot_w, 0
        for lv in sorted(levels) + [L] * spare:
            k = cls.norm_plaintext_slots(batches, lv, n, slot_w)
            if total + k > cap:
                break
            total += k
        return total

    def alloc_queries(self, count: int) -> list[QueryRecord]:
        """Records whose results (compacted coarse distances; n_res candidate
        ciphertexts; level lvl_out) are packed back to back in two outboxes, so
        limb 0 of many reaches the host in one copy (read_results)."""
        w = self.lvl_out * self.p.n
        comp = self.slots.take(-(-2 * count * w // self.slots.w))[0]
        dist = self.slots.take(-(-2 * count * self.n_res * w // self.slots.w))[0]
        packed = self.sh.compaction == "packed"
        w1 = (self.L - 1) * self.p.n
        nbase = self.slots.take(self.norm_slots(count, self.L, self.p.n, self.slots.w))[0] if packed else 0
        nb = self.sh.n1 - 1 if self.sh.compaction == "diagonal" else 0
        wb = getattr(self, "_baby_limbs", 0) * self.p.n
        bbase = self.slots.take(-(-2 * count * nb * wb // self.slots.w))[0] if nb else 0
        recs = []
        for i in range(count):
            s = self.slots.take(4)
            res = [(dist + 2 * (i * self.n_res + k) * w, dist + (2 * (i * self.n_res + k) + 1) * w)
                   for k in range(self.n_res)]
            baby = [(bbase + 2 * (i * nb + b) * wb, bbase + (2 * (i * nb + b) + 1) * wb) for b in range(nb)]
            recs.append(QueryRecord((s[0], s[1]), (s[2], s[3]),
                                    (comp + 2 * i * w, comp + (2 * i + 1) * w), res[0], results=res,
                                    norm=(nbase + 2 * i * w1, nbase + (2 * i + 1) * w1) if packed else None,
                                    baby=baby))
        self._outbox = {"compact": (comp, 1), "dists": (dist, self.n_res)}
        return recs

    def record_index(self, kind: str, rec: QueryRecord) -> int:
        base, per = self._outbox[kind]
        first = rec.compact if kind == "compact" else rec.results[0]
        return (first[0] - base) // (2 * per * self.lvl_out * self.p.n)

    def read_results(self, kind: str, recs, staged: bool = False, tag: str = "", wait: bool = True):
        """Limb 0 of both polynomials of the records' result ciphertexts:
        (len(recs), per_record, 2, N); one copy per run of consecutive records.
        Limb 0 is what the client decrypts (see __init__). With `staged`, the
        array is a view of the context's page-locked staging, valid until the
        next staged read of the same kind and `tag`. With wait=False (staged
        only) the call returns (array, fence): the array holds the results
        once ctx.fence_wait(fence) has returned. The copies are only enqueued
        when the records are in ascending order of their outbox places (as
        allocated); otherwise they are made at once."""
        base, per = self._outbox[kind]
        n, w = self.p.n, self.lvl_out * self.p.n
        idx = [self.record_index(kind, r) for r in recs]
        size = len(recs) * per * 2 * n
        if staged:
            out = self.ctx.staging.get("res_" + kind + tag, size).reshape(len(recs), per, 2, n)
        else:
            if not wait:
                raise ValueError("an asynchronous read needs page-locked staging")
            out = np.empty((len(recs), per, 2, n), dtype=np.uint64)
        if all(a < b for a, b in zip(idx, idx[1:])):     # ascending: each run of records straight into place
            fn = self.lib.afhe_read_poly_rows if wait else self.lib.afhe_read_poly_rows_async
            i = 0
            while i < len(idx):
                j = i
                while j + 1 < len(idx) and idx[j + 1] == idx[j] + 1:
                    j += 1
                L.check(fn(self.ctx.h, base + idx[i] * per * 2 * w, w, (j - i + 1) * per * 2, n,
                           out[i:j + 1].ctypes.data_as(L.P64)), "read_poly_rows")
                i = j + 1
            return out if wait else (out, self.ctx.fence())
        order = np.argsort(idx, kind="stable")
        i = 0
        while i < len(order):
            j = i
            while j + 1 < len(order) and idx[order[j + 1]] == idx[order[j]] + 1:
                j += 1
            rows = (j - i + 1) * per * 2
            block = np.empty(rows * n, dtype=np.uint64)
            L.check(self.lib.afhe_read_poly_rows(self.ctx.h, base + idx[order[i]] * per * 2 * w, w, rows, n,
                                                 block.ctypes.data_as(L.P64)), "read_poly_rows")
            block = block.reshape(j - i + 1, per, 2, n)
            for k in range(i, j + 1):
                out[order[k]] = block[k - i]
            i = j + 1
        return out if wait else (out, self.ctx.fence())

    def coarse_from_slots(self, vals: np.ndarray) -> np.ndarray:
        """(count, n_list) coarse distances from the decoded slots of the
        compacted coarse ciphertexts."""
        idx = [self.sh.coarse_slot(c) for c in range(self.sh.n_list)]
        return vals[:, idx]

    def coarse_slots_needed(self) -> int:
        return max(self.sh.coarse_slot(c) for c in range(self.sh.n_list)) + 1

    # ---- tuning ----
    def use_tuning(self, choices: dict | None) -> None:
        """Per-level key-switch choices from the autotuner ({level: KsChoice});
        None restores the context's defaults."""
        self._tuning = choices or {}
        self._opt_now = None
        self._nh_ver += 1
        if not hasattr(self, "_fused_ok"):
            self._fused_ok = self.ctx.get_option(L.OPT_KS_FUSED) == 1

    def _at(self, level: int) -> None:
        """Apply the tuned options of the level an operator runs at."""
        ch = getattr(self, "_tuning", {}).get(level)
        if ch is None:
            return
        want = (int(ch.fused), int(ch.chunk), int(getattr(ch, "ept", 8)), int(getattr(ch, "slice", 13)),
                int(getattr(ch, "fused_min", 0)))
        if want != getattr(self, "_opt_now", None):
            if want[0] == 0 or self._fused_ok:
                self.ctx.set_option(L.OPT_KS_FUSED, want[0])
            if want[1]:
                self.ctx.set_option(L.OPT_CHUNK, min(want[1], self.ctx.max_batch))
            self.ctx.set_option(L.OPT_KS_EPT, want[2])
            self.ctx.set_option(L.OPT_KS_SLICE, want[3])
            if want[4]:
                self.ctx.set_option(L.OPT_FUSED_MIN, want[4])
            self._opt_now = want

    # ---- the native stage driver ----
    def _native_handle(self) -> C.c_void_p:
        """The afhe_ivfpq handle for the current lanes, eval_level, masks and
        tuning (re-registered when one of them changed)."""
        key = (self.lanes, self.sh.eval_level, self._nh_ver)
        if self._nh is not None and self._nh_key == key:
            return self._nh
        self.close_native()
        sh = self.sh
        kind = {"reference": 0, "packed": 1, "diagonal": 2}[sh.compaction]
        shape = L.IvfpqShape(sh.D, sh.n_list, sh.slots, self.lanes, kind, sh.eval_level or 0)
        h = C.c_void_p()
        L.check(self.lib.afhe_ivfpq_create(self.ctx.h, C.byref(shape), C.byref(h)), "ivfpq_create")
        self._nh = h
        lib = self.lib
        if kind == 2:
            first = np.concatenate([[0], np.cumsum([len(u) for u in self.list_units])]).astype(np.uint32)
            cnt = np.asarray(self._ucnt or [0], dtype=np.uint32)
            L.check(lib.afhe_ivfpq_set_units(h, first.ctypes.data_as(L.P32), cnt.ctypes.data_as(L.P32),
                                             len(self.units)), "ivfpq_set_units")
            for lv, d in self._diag.items():
                L.check(lib.afhe_ivfpq_set_diagonals(h, lv, int(d["cent"][0]), int(d["cnorm"]), self._offs(d["pts"][::sh.D]),
                                                     self._offs(d["norms"]), len(self.units)), "ivfpq_set_diagonals")
            L.check(lib.afhe_ivfpq_set_scratch(h, self._refs(self._inner), len(self._inner)), "ivfpq_set_scratch")
            self._native_tuning(h)
            self._nh_key = key
            return h
        L.check(lib.afhe_ivfpq_set_centroids(h, self._offs(self.pt_centroid_cts), len(self.pt_centroid_cts)),
                "ivfpq_set_centroids")
        for lv in self.levels:
            m = self._onehot[lv] if sh.compaction == "reference" else [self._stride[lv]]
            L.check(lib.afhe_ivfpq_set_level_masks(h, lv, self._offs(m), len(m)), "ivfpq_set_level_masks")
        for (cnt, lv), off in self._prefix_lv.items():
            L.check(lib.afhe_ivfpq_set_prefix_mask(h, lv, cnt, off), "ivfpq_set_prefix_mask")
        for lv, offs in getattr(self, "_norms", {}).items():
            L.check(lib.afhe_ivfpq_set_norms(h, lv, self._offs(offs), len(offs)), "ivfpq_set_norms")
        for c, bs in enumerate(self.batches):
            cnts = np.array([b[1] for b in bs] or [0], dtype=np.uint32)
            L.check(lib.afhe_ivfpq_set_list(h, c, self._offs([b[0] for b in bs]), cnts.ctypes.data_as(L.P32),
                                            len(bs)), "ivfpq_set_list")
        work = self._refs([w[k] for w in self.work[:self.lanes] for k in ("diff", "sq", "sel", "tmp")])
        cmp = self._refs([c for row in self.cmp[:self.lanes] for c in row]) if self.cmp else None
        L.check(lib.afhe_ivfpq_set_lanes(h, work, self.lanes, cmp), "ivfpq_set_lanes")
        self._native_tuning(h)
        self._nh_key = key
        return h

    def _native_tuning(self, h) -> None:
        for lv, ch in getattr(self, "_tuning", {}).items():
            o = L.KsOptions(int(ch.fused), int(ch.chunk), int(getattr(ch, "ept", 8)), int(getattr(ch, "slice", 13)),
                            int(getattr(ch, "fused_min", 0)))
            L.check(self.lib.afhe_ivfpq_set_tuning(h, lv, C.byref(o)), "ivfpq_set_tuning")

    def close_native(self) -> None:
        if self._nh is not None:
            self.lib.afhe_ivfpq_destroy(self._nh)
            self._nh, self._nh_key = None, None

    @staticmethod
    def _query_dtype() -> np.dtype:
        """afhe_ivfpq_query as a numpy record (offsets from the ctypes struct)."""
        f = L.IvfpqQuery
        names = [n for n, _ in f._fields_]
        kinds = {"ct_query": ("<u8", (2,)), "ct_dim": ("<u8", (2,)), "compact": ("<u8", (2,)),
                 "norm": ("<u8", (2,)), "results": ("<u8", ()), "probes": ("<u8", ()), "baby": ("<u8", ())}
        return np.dtype({"names": names,
                         "formats": [kinds[n] if n in kinds else "<u4" for n in names],
                         "offsets": [getattr(f, n).offset for n in names], "itemsize": C.sizeof(f)})

    @classmethod
    def _native_queries(cls, queries, probes: bool):
        """An afhe_ivfpq_query array for the records, built with numpy (the
        arrays it points to are kept alive by the returned list)."""
        m = len(queries)
        dt = getattr(cls, "_qdt", None)
        if dt is None:
            dt = cls._qdt = cls._query_dtype()
        a = np.zeros(max(1, m), dtype=dt)
        if m:
            a["ct_query"] = [r.ct_query for r in queries]
            a["ct_dim"] = [r.ct_dim for r in queries]
            a["compact"] = [r.compact for r in queries]
            a["norm"] = [r.norm if r.norm is not None else (0, 0) for r in queries]
            a["level"] = [r.level for r in queries]
        keep = [a]

        def pointers(field, count_field, rows, width):
            """rows: per query a list of (c0, c1) pairs or ints, all `width`
            long except where shorter; one contiguous array, one pointer each."""
            if not width:
                return
            flat = np.zeros((m, width) + ((2,) if field != "probes" else ()), dtype=np.uint64 if field != "probes"
                            else np.uint32)
            n = np.zeros(m, dtype=np.uint32)
            for i, row in enumerate(rows):
                if len(row):
                    flat[i, :len(row)] = row
                n[i] = len(row)
            keep.append(flat)
            a[field] = flat.ctypes.data + np.arange(m, dtype=np.uint64) * np.uint64(flat.strides[0])
            a[count_field] = n
        pointers("results", "n_results", [r.results for r in queries], max((len(r.results) for r in queries),
                                                                            default=0))
        if probes:
            pointers("probes", "nprobe", [[int(c) for c in r.probes] for r in queries],
                     max((len(r.probes) for r in queries), default=0))
        pointers("baby", "n_baby", [r.baby for r in queries], max((len(r.baby) for r in queries), default=0))
        return a.ctypes.data_as(C.POINTER(L.IvfpqQuery)), keep

    # ---- batched C-ABI helpers ----
    @staticmethod
    def _refs(cts):
        """An afhe_ct_ref array for the C ABI from (c0, c1) pairs: a list of
        pairs or an (m, 2) array. The pointer keeps its array alive."""
        if isinstance(cts, np.ndarray):
            a = np.ascontiguousarray(cts, dtype=np.uint64).reshape(-1)
        else:
            a = np.fromiter(itertools.chain.from_iterable(cts), dtype=np.uint64, count=2 * len(cts))
        if a.size == 0:
            a = np.zeros(2, dtype=np.uint64)
        return a.ctypes.data_as(C.POINTER(L.CtRef))

    @staticmethod
    def _offs(v):
        """A uint64 array for the C ABI from offsets (a list or an array)."""
        a = np.ascontiguousarray(v, dtype=np.uint64) if isinstance(v, np.ndarray) else \
            np.fromiter(v, dtype=np.uint64, count=len(v))
        if a.size == 0:
            a = np.zeros(1, dtype=np.uint64)
        return a.ctypes.data_as(L.P64)

    def _rotate(self, cts, r, limbs):
        self._at(limbs)
        refs = self._refs(cts)
        L.check(self.lib.afhe_eval_rotate_batch(self.ctx.h, refs, refs, len(cts), r, limbs), "eval_rotate_batch")

    def _rot_acc(self, src, acc, r, limbs):
        self._at(limbs)
        L.check(self.lib.afhe_eval_rotate_accumulate_batch(self.ctx.h, self._refs(src), self._refs(acc), len(src), r,
                                                           limbs), "eval_rotate_accumulate_batch")

    def _add(self, a, b, d, limbs):
        L.check(self.lib.afhe_eval_add_batch(self.ctx.h, self._refs(a), self._refs(b), self._refs(d), len(a), limbs),
                "eval_add_batch")

    def _copy(self, a, d, limbs):
        L.check(self.lib.afhe_eval_copy_batch(self.ctx.h, self._refs(a), self._refs(d), len(a), limbs),
                "eval_copy_batch")

    def _sub(self, a, b, d, limbs):
        L.check(self.lib.afhe_eval_sub_batch(self.ctx.h, self._refs(a), self._refs(b), self._refs(d), len(a), limbs),
                "eval_sub_batch")

    def _add_plain(self, a, pts, d, limbs):
        L.check(self.lib.afhe_eval_add_plain_batch(self.ctx.h, self._refs(a), self._offs(pts), self._refs(d), len(a),
                                                   limbs), "eval_add_plain_batch")

    def _mult_plain(self, a, pts, d, limbs):
        L.check(self.lib.afhe_eval_mult_plain_rescale_batch(self.ctx.h, self._refs(a), self._offs(pts), self._refs(d),
                                                            len(a), limbs), "eval_mult_plain_rescale_batch")

    def _square(self, a, d, limbs):
        self._at(limbs)
        L.check(self.lib.afhe_eval_mult_relin_rescale_batch(self.ctx.h, self._refs(a), self._refs(a), self._refs(d),
                                                            len(a), limbs), "eval_mult_relin_rescale_batch")

    def _sub_plain(self, a, pts, d, limbs):
        L.check(self.lib.afhe_eval_sub_plain_batch(self.ctx.h, self._refs(a), self._offs(pts), self._refs(d), len(a),
                                                   limbs), "eval_sub_plain_batch")

    def _rotate_direct(self, items, limbs: int) -> None:
        """Rotate each ciphertext of `items` ((ct, step) pairs) in place by
        its step in one key switch (every step has its own key)."""
        items = [(ct, s) for ct, s in items if s]
        if not items:
            return
        self._at(limbs)
        steps = (L.i32 * len(items))(*[s for _, s in items])
        refs = self._refs([ct for ct, _ in items])
        L.check(self.lib.afhe_eval_rotate_steps_batch(self.ctx.h, refs, refs, steps, len(items), limbs),
                "eval_rotate_steps_batch")

    def _rotate_grouped(self, items, limbs: int) -> None:
        """Rotate each ciphertext of `items` ((ct, shift) pairs) in place by its
        shift, as eval_rotate does it: |shift| in descending powers of two,
        sign kept (fhe_host_driver.cpp:361-404). The steps run highest power
        first, each as one batched launch over every item whose shift has
        that bit, so every item sees exactly its own eval_rotate steps in
        eval_rotate's order."""
        items = [(ct, s) for ct, s in items if s]
        if not items:
            return
        m = len(items)
        cts = np.fromiter(itertools.chain.from_iterable(ct for ct, _ in items), dtype=np.uint64,
                          count=2 * m).reshape(m, 2)
        shift = np.fromiter((s for _, s in items), dtype=np.int64, count=m)
        mag, up = np.abs(shift), shift > 0
        for b in range(int(mag.max()).bit_length() - 1, -1, -1):
            has = ((mag >> b) & 1).astype(bool)
            for sign, side in ((1, up), (-1, ~up)):
                sel = has & side
                if sel.any():
                    self._rotate(cts[sel], sign * (1 << b), limbs)

    def _accumulate(self, items, limbs: int) -> None:
        """items: (target, first, src). Per target, its sources of this call
        are summed pairwise, then copied into the target when one of them
        starts the target's sum (`first`), else added to it. Modular
        additions are exact, so any grouping gives the reference's running
        sum word for word."""
        by: dict = {}
        for tgt, first, src in items:
            e = by.setdefault(tgt, [False, []])
            e[0] = e[0] or first
            e[1].append(src)
        self._sum_groups([g for _, g in by.values()], limbs)
        copies = [(t, g[0]) for t, (f, g) in by.items() if f]
        adds = [(t, g[0]) for t, (f, g) in by.items() if not f]
        if copies:
            self._copy([s_ for _, s_ in copies], [t for t, _ in copies], limbs)
        if adds:
            self._add([t for t, _ in adds], [s_ for _, s_ in adds], [t for t, _ in adds], limbs)

    # ---- stages ----
    def stage1_coarse(self, queries: list[QueryRecord]) -> None:
        """Stages 1 and 1b for every query (lanes at a time, one level at a time)."""
        if self.sh.compaction == "diagonal" and not self._native_diagonal():
            for lv, idx in self._by_level(queries, self.level_of):
                self._stage1_diagonal([queries[i] for i in idx], lv)
            return
        if self.native:
            arr, keep = self._native_queries(queries, probes=False)
            L.check(self.lib.afhe_ivfpq_stage1(self._native_handle(), arr, len(queries)), "ivfpq_stage1")
            self._opt_now = None
            return
        for lv, idx in self._by_level(queries, self.level_of):
            qs = [queries[i] for i in idx]
            if self.sh.compaction == "packed":
                self._stage1_packed(qs, lv)
            else:
                self._stage1_reference(qs, lv)

    def _stage1_reference(self, queries: list[QueryRecord], Ll: int) -> None:
        D = self.sh.D
        for c0 in range(0, len(queries), self.lanes):
            qs = queries[c0:c0 + self.lanes]
            w = self.work[:len(qs)]
            diff = [x["diff"] for x in w]
            sq = [x["sq"] for x in w]
            self._sub_plain([q.ct_query for q in qs], [self.pt_centroids] * len(qs), diff, Ll)
            self._square(diff, sq, Ll)
            s = 1
            while s < D:                     # sq += rot(sq, s)
                self._rot_acc(sq, sq, s, Ll - 1)
                s <<= 1
            self._compact(qs, sq, Ll)

    def _stage1_packed(self, queries: list[QueryRecord], Ll: int) -> None:
        """Stage 1 and the packed compaction: items (query, coarse ciphertext k),
        lanes at a time, query-major."""
        D, nc = self.sh.D, self.sh.n_coarse
        items = [(qi, k) for qi in range(len(queries)) for k in range(nc)]
        for c0 in range(0, len(items), self.lanes):
            it = items[c0:c0 + self.lanes]
            w = self.work[:len(it)]
            diff = [x["diff"] for x in w]
            sq = [x["sq"] for x in w]
            sel = [x["sel"] for x in w]
            self._sub_plain([queries[qi].ct_query for qi, _ in it], [self.pt_centroid_cts[k] for _, k in it], diff,
                            Ll)
            self._square(diff, sq, Ll)
            s = 1
            while s < D:                     # sq += rot(sq, s)
                self._rot_acc(sq, sq, s, Ll - 1)
                s <<= 1
            self._mult_plain(sq, [self._stride[Ll]] * len(it), sel, Ll - 1)
            self._rotate_direct([(sel[j], -k) for j, (_, k) in enumerate(it)], Ll - 2)
            self._accumulate([(queries[qi].compact, k == 0, sel[j]) for j, (qi, k) in enumerate(it)], Ll - 2)

    def _compact(self, qs: list[QueryRecord], sq, Ll: int) -> None:
        """Stage 1b (reference compaction) for a chunk of queries: compact =
        sum over i of rot(rescale(sq * mask_i), i * (D - 1)).

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
        onehot = self._onehot[Ll]
        comp = [q.compact for q in qs]
        src, pts, dst = [], [], []
        for k in range(len(qs)):
            for i in range(nl):
                src.append(sq[k])
                pts.append(onehot[i])
                dst.append(comp[k] if i == 0 else self.cmp[k][i - 1])
        self._mult_plain(src, pts, dst, Ll - 1)
        if nl == 1:
            return
        self._rotate_grouped([(self.cmp[k][i - 1], i * (D - 1)) for k in range(len(qs)) for i in range(1, nl)],
                             Ll - 2)
        # per query: comp += sum of its n_list - 1 rotated terms
        self._sum_groups([[comp[k]] + self.cmp[k] for k in range(len(qs))], Ll - 2)

    # ---- the diagonal chain: stages ----
    def _native_diagonal(self) -> bool:
        return self.native

    MAC_GROUP = np.dtype([("c0", "<u8"), ("c1", "<u8"), ("first", "<u4"), ("n", "<u4")])
    MAC_TERM = np.dtype([("pt", "<u8"), ("galois", "<u4"), ("reserved", "<u4")])

    def _mac(self, outs, first, groups: np.ndarray, terms: np.ndarray, limbs: int, accumulate: bool = False) -> None:
        """afhe_eval_mac_plain_batch: outs[j] (+)= sum over groups [first[j],
        first[j + 1]) of the group's placed plaintexts times its ciphertext
        (c0 = MAC_UNIT: the constant ciphertext (1, 0)). groups / terms are
        MAC_GROUP / MAC_TERM arrays (the C ABI's afhe_mac_group / afhe_mac_term)."""
        fg = np.ascontiguousarray(first, dtype=np.uint32)
        assert fg.size == len(outs) + 1 and groups.dtype == self.MAC_GROUP and terms.dtype == self.MAC_TERM
        g = np.ascontiguousarray(groups if groups.size else np.zeros(1, self.MAC_GROUP))
        t = np.ascontiguousarray(terms if terms.size else np.zeros(1, self.MAC_TERM))
        L.check(self.lib.afhe_eval_mac_plain_batch(self.ctx.h, self._refs(outs), fg.ctypes.data_as(L.P32), len(outs),
                                                   g.ctypes.data_as(C.POINTER(L.MacGroup)),
                                                   t.ctypes.data_as(C.POINTER(L.MacTerm)), limbs, int(accumulate)),
                "eval_mac_plain_batch")

    def _diag_jobs(self, srcs, pts, gals):
        """Descriptors of inner-product outputs: output k, giant step g has
        n1 groups b (source srcs[k][b]) whose terms are pts[k][g, b, :] moved
        by gals[k][:]. pts[k]: (n2, n1, m_k) offsets; gals[k]: (m_k,)."""
        n1, n2 = self.sh.n1, self.sh.n2
        G = np.zeros(len(srcs) * n2 * n1, self.MAC_GROUP)
        sizes = np.repeat([p.shape[2] for p in pts], n2 * n1)
        G["n"] = sizes
        G["first"] = np.concatenate([[0], np.cumsum(sizes)[:-1]]) if sizes.size else []
        src = np.asarray(srcs, dtype=np.uint64).reshape(len(srcs), 1, n1, 2)
        src = np.broadcast_to(src, (len(srcs), n2, n1, 2)).reshape(-1, 2)
        G["c0"], G["c1"] = src[:, 0], src[:, 1]
        T = np.zeros(int(sizes.sum()), self.MAC_TERM)
        if T.size:
            T["pt"] = np.concatenate([p.reshape(-1) for p in pts])
            T["galois"] = np.concatenate([np.tile(np.asarray(g, dtype=np.uint32), n2 * n1) for g in gals])
        first = np.arange(0, len(srcs) * n2 * n1 + 1, n1)
        return first, G, T

    def _rescale(self, a, d, in_limbs: int) -> None:
        L.check(self.lib.afhe_rescale_batch(self.ctx.h, self._refs(a), self._refs(d), len(a), in_limbs),
                "rescale_batch")

    def _giant(self, inner, srcs, bases, gals, Ll: int) -> None:
        """Output k (of len(srcs)): giant step g's inner product into
        inner[k n2 + g] (Ll limbs): sum over units m and b < n1 of the unit's
        plaintext bases[k][g, m] + b Ll N moved by gals[k][m] times srcs[k][b];
        then rescaled, giant step g rotated by n1 g, summed into inner[k n2]
        (Ll - 1 limbs)."""
        n1, n2 = self.sh.n1, self.sh.n2
        stride = Ll * self.p.n
        if n1 in (1, 2, 4, 8, 16):
            sizes = np.repeat([b.shape[1] for b in bases], n2)
            first = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
            upt = np.ascontiguousarray(np.concatenate([b.reshape(-1) for b in bases]) if bases else
                                       np.zeros(1), dtype=np.uint64)
            ugal = np.ascontiguousarray(np.concatenate([np.tile(np.asarray(g, dtype=np.uint32), n2) for g in gals])
                                        if gals else np.zeros(1), dtype=np.uint32)
            src = [c for k in range(len(srcs)) for _ in range(n2) for c in srcs[k]]
            L.check(self.lib.afhe_eval_diag_inner_batch(self.ctx.h, self._refs(inner), len(inner), self._refs(src), n1,
                                                        upt.ctypes.data_as(L.P64) if upt.size else None,
                                                        ugal.ctypes.data_as(L.P32), first.ctypes.data_as(L.P32),
                                                        stride, Ll, 0), "eval_diag_inner_batch")
        else:
            pts = [bs[:, None, :] + np.arange(n1, dtype=np.uint64)[None, :, None] * np.uint64(stride) for bs in bases]
            self._mac(inner, *self._diag_jobs(srcs, pts, gals), Ll)
        self._rescale(inner, inner, Ll)
        self._rotate_direct([(inner[j], n1 * (j % n2)) for j in range(len(inner)) if j % n2], Ll - 1)
        self._sum_groups([inner[k:k + n2] for k in range(0, len(inner), n2)], Ll - 1)

    def _babies(self, q: QueryRecord) -> list:
        return [q.ct_query] + list(q.baby)

    def _stage1_diagonal(self, queries: list[QueryRecord], Ll: int) -> None:
        """Baby steps of every query, then the coarse distances ||q||^2 -
        2 <q, c> + ||c||^2 in slot c of `compact` (Ll - 1 limbs); ||q||^2 is
        the client's ciphertext in ct_dim."""
        D, n1, n2 = self.sh.D, self.sh.n1, self.sh.n2
        dg = self._diag[Ll]
        items = [(q, b) for q in queries for b in range(1, n1)]
        if items:
            steps = (L.i32 * len(items))(*[b for _, b in items])
            self._at(Ll)
            L.check(self.lib.afhe_eval_rotate_steps_batch(self.ctx.h, self._refs([q.ct_query for q, _ in items]),
                                                          self._refs([q.baby[b - 1] for q, b in items]), steps,
                                                          len(items), Ll), "eval_rotate_steps_batch")
        cent = np.asarray(dg["cent"], dtype=np.uint64)[np.arange(n2) * n1].reshape(n2, 1)
        per = len(self._inner) // n2
        for c0 in range(0, len(queries), per):
            qs = queries[c0:c0 + per]
            inner = self._inner[:len(qs) * n2]
            self._giant(inner, [self._babies(q) for q in qs], [cent] * len(qs), [np.ones(1, np.uint32)] * len(qs),
                        Ll)
            comp = [q.compact for q in qs]
            self._add(inner[0::n2], [q.ct_dim for q in qs], comp, Ll - 1)     # + ||q||^2 (the client's)
            self._add_plain(comp, [dg["cnorm"]] * len(qs), comp, Ll - 1)

    def _stage3_diagonal_layout(self, queries: list[QueryRecord]) -> None:
        """Each query's units, their offsets, candidate ids and slot positions."""
        S = self.sh.slots
        if getattr(self, "_unit_arrays", None) is None:
            self._unit_arrays = [np.asarray(v, dtype=np.int64) for _, v in self.units]
        ua, ar = self._unit_arrays, np.arange(S, dtype=np.int64)
        for q in queries:
            q.layout = self.unit_offsets(q.probes)
            if q.layout:
                q.vids = np.concatenate([ua[u] for u, _ in q.layout])
                q.pos = np.concatenate([ar[:len(ua[u])] + off for u, off in q.layout])
            else:
                q.vids, q.pos = [], np.zeros(0, dtype=np.int64)
            if q.layout and q.layout[-1][1] // S >= self.n_res:
                raise ValueError("more candidates than the result ciphertexts hold")

    def _placement_galois(self, off: int) -> int:
        """Galois element moving a unit's plaintext from slot 0 to `off` (mod slots)."""
        o = off % self.sh.slots
        if o not in self._gal_cache:
            self._gal_cache[o] = galois_elt(self.p.log_n, -o)
        return self._gal_cache[o]

    def _stage3_diagonal(self, queries: list[QueryRecord], Ll: int) -> None:
        """Per (query, result ciphertext): the placed units' inner products,
        the giant steps, + ||q||^2 + the placed unit norms."""
        D, S, n1, n2 = self.sh.D, self.sh.slots, self.sh.n1, self.sh.n2
        dg = self._diag[Ll]
        pts, norms = dg["pts"], dg["norms"]
        g0 = np.arange(n2)[:, None] * n1          # diagonal g n1 (b = 0) of each giant step
        items = []
        for q in queries:
            used = q.layout[-1][1] // S + 1 if q.layout else 1
            lay = np.asarray(q.layout, dtype=np.int64).reshape(-1, 2)
            for r in range(used):
                sel = lay[lay[:, 1] // S == r]
                gal = np.fromiter((self._placement_galois(int(o)) for o in sel[:, 1]), dtype=np.uint32,
                                  count=len(sel))
                items.append((q, r, sel[:, 0], gal))
        per = len(self._inner) // n2
        for c0 in range(0, len(items), per):
            it = items[c0:c0 + per]
            inner = self._inner[:len(it) * n2]
            self._giant(inner, [self._babies(q) for q, _, _, _ in it], [pts[u[None, :] * D + g0] for _, _, u, _ in it],
                        [g for _, _, _, g in it], Ll)
            outs = [q.results[r] for q, r, _, _ in it]
            self._add(inner[0::n2], [q.ct_dim for q, _, _, _ in it], outs, Ll - 1)
            sizes = np.array([len(u) for _, _, u, _ in it], dtype=np.int64)
            G = np.zeros(len(it), self.MAC_GROUP)
            G["c0"], G["n"] = L.MAC_UNIT, sizes
            G["first"] = np.concatenate([[0], np.cumsum(sizes)[:-1]])
            T = np.zeros(int(sizes.sum()), self.MAC_TERM)
            if T.size:
                T["pt"] = np.concatenate([norms[u] for _, _, u, _ in it])
                T["galois"] = np.concatenate([g for _, _, _, g in it])
            self._mac(outs, np.arange(len(it) + 1), G, T, Ll - 1, accumulate=True)

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
        S = self.sh.slots
        if self.sh.compaction == "diagonal":
            self._stage3_diagonal_layout(queries)
            if not self._native_diagonal():
                for lv, idx in self._by_level(queries, self.level_of):
                    self._stage3_diagonal([queries[i] for i in idx], lv)
                return
            arr, keep = self._native_queries(queries, probes=True)
            L.check(self.lib.afhe_ivfpq_stage3(self._native_handle(), arr, len(queries)), "ivfpq_stage3")
            self._opt_now = None
            return
        items: dict[int, list] = {}
        for qi, q in enumerate(queries):
            q.vids, q.pos = [], []
            lst = items.setdefault(self.level_of(q), [])
            bs = [b for c in q.probes for b in self.batches[c]]
            gbs = [self._first_batch[c] + i for c in q.probes for i in range(len(self.batches[c]))]
            align = self.sh.B if self.sh.compaction == "packed" else None
            offs = batch_offsets([b[1] for b in bs], S, align)
            for (pt, cnt, vids), off, gb in zip(bs, offs, gbs):
                lst.append((qi, pt, cnt, off, gb))
                q.vids.extend(vids)
            q.pos = (np.concatenate([np.arange(off, off + b[1]) for b, off in zip(bs, offs)]) if bs
                     else np.zeros(0, dtype=np.int64))
            if len(q.pos) and q.pos[-1] >= self.n_res * S:
                raise ValueError("more candidates than the result ciphertexts hold")
        if self.native:
            for lv, it in items.items():
                for x in it:
                    self._prefix(x[2], lv)          # every batch size's mask at this level exists
            arr, keep = self._native_queries(queries, probes=True)
            L.check(self.lib.afhe_ivfpq_stage3(self._native_handle(), arr, len(queries)), "ivfpq_stage3")
            self._opt_now = None
            return
        for lv in sorted(items, reverse=True):
            self._stage3_items(queries, items[lv], lv)

    def _stage3_items(self, queries: list[QueryRecord], items, Ll: int) -> None:
        D, B, S = self.sh.D, self.sh.B, self.sh.slots
        norms = getattr(self, "_norms", {}).get(Ll) if self.sh.compaction == "packed" else None
        if norms is not None:
            # expanded distances: ||q||^2 squared once per query
            seen, qs = set(), []
            for x in items:
                if x[0] not in seen:
                    seen.add(x[0])
                    qs.append(queries[x[0]])
            for c0 in range(0, len(qs), self.lanes):
                part = qs[c0:c0 + self.lanes]
                self._square([q.ct_dim for q in part], [q.norm for q in part], Ll)
        for c0 in range(0, len(items), self.lanes):
            it = items[c0:c0 + self.lanes]
            w = self.work[:len(it)]
            diff = [x["diff"] for x in w]
            sq = [x["sq"] for x in w]
            sel = [x["sel"] for x in w]
            if norms is not None:
                # ||q||^2 - 2 <q, x_j> in every row, then + ||x_j||^2
                self._mult_plain([queries[x[0]].ct_dim for x in it], [x[1] for x in it], diff, Ll)
                self._sub([queries[x[0]].norm for x in it], diff, sq, Ll - 1)
                self._sub(sq, diff, sq, Ll - 1)
            else:
                self._sub_plain([queries[x[0]].ct_dim for x in it], [x[1] for x in it], diff, Ll)
                self._square(diff, sq, Ll)
            s = B
            while s < D * B:                 # sq += rot(sq, s)
                self._rot_acc(sq, sq, s, Ll - 1)
                s <<= 1
            if norms is not None:
                self._add_plain(sq, [norms[x[4]] for x in it], sq, Ll - 1)
            prefix = [self._prefix(x[2], Ll) for x in it]
            if self.sh.compaction == "packed":
                # the tree sum leaves the batch's sums in every row: the prefix
                # mask moved to row offset / B (a plaintext automorphism, no
                # key switch) selects and places them at once
                masks = [x["tmp"][0] for x in w]
                gal = (L.u32 * len(it))(*[galois_elt(self.p.log_n, -(x[3] % S)) for x in it])
                L.check(self.lib.afhe_automorphism_batch(self.ctx.h, self._offs(prefix), gal, self._offs(masks),
                                                         len(it), Ll - 1), "automorphism_batch")
                self._mult_plain(sq, masks, sel, Ll - 1)
            else:
                # rotate each item by -(offset mod slots): eval_rotate's steps,
                # grouped across items step by step
                self._mult_plain(sq, prefix, sel, Ll - 1)
                self._rotate_grouped([(sel[k], -(x[3] % S)) for k, x in enumerate(it)], Ll - 2)
            # accumulate into result offset // slots; the item at slot 0 starts it
            self._accumulate([(queries[x[0]].results[x[3] // S], x[3] % S == 0, sel[k]) for k, x in enumerate(it)],
                             Ll - 2)

    # ---- result transfer ----
    def input_polys(self, rec: QueryRecord) -> tuple:
        """Offsets of the polynomials the server reads from a client: ct_query
        and ct_dim (the diagonal chain: ct_dim holds ||q||^2)."""
        return (*rec.ct_query, *rec.ct_dim)

    def input_words(self, rec: QueryRecord) -> tuple:
        """Words of each of input_polys a client sends: the limbs the server
        evaluates the query at (a ciphertext's first l limbs are the same
        message mod Q_l, so the client drops the rest before sending, as the
        server would on arrival); the diagonal chain's ||q||^2 ciphertext is
        at the evaluation level - 1."""
        lv, n = self.eval_at(rec.level or self.L), self.p.n
        wq = lv * n
        wd = (lv - 1) * n if self.sh.compaction == "diagonal" else wq
        return (wq, wq, wd, wd)

    def read_ct(self, ct: tuple[int, int]) -> tuple[np.ndarray, np.ndarray]:
        w = self.lvl_out * self.p.n
        return self.ctx.read_poly(ct[0], w), self.ctx.read_poly(ct[1], w)
