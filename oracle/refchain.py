"""The encrypted IVF-PQ server chain on the reference's own CPU code: the
timed CPU baseline.

TEST INFRASTRUCTURE ONLY: bench.py's reference arm and its cpu_baseline leg
time this, and tests/test_oracle.py checks its operator sequence; the
product never runs it.

What runs. The reference's HLS C-simulation (fhe_accel_top and its kernels,
hardware_fpga_model/hls/src/*.cpp) rebuilt at the workload's ring degree
(oracle/_ref/libref_hls_n<N>.so, oracle/Makefile) over the reference's own
SimMemoryBus (cpp_host_model/src/sim_memory_bus.cpp), driven operator by
operator in the sequence of FHEHostDriver (cpp_host_model/src/
fhe_host_driver.cpp:177-404): every composite expands into the op codes and
host-side copies the reference's driver issues, with its scratch slots.
`HostDriver` below restates that sequence. Where the reference's library is
absent, the same sequence runs on the C restatement (oracle/liborc.so) and
the result says kind "port".

Two registers follow the level of each call, as a host driving several
levels must set them: numPartQ = ceil(l / alpha) (FHEHostDriver passes its
fixed 3, fhe_host_driver.cpp:190-203, with which key_switch.cpp:226 reads
past the input below 2 alpha + 1 limbs), and n_inv_mod_q_last. The tables
are loaded once (OP 99) at the queries' top level, as
FHEHostDriver::load_context_to_hardware does (fhe_host_driver.cpp:206-208);
operators at lower levels then run on those tables, as with the reference's
own driver. The reference's OP 99 cannot load a level with fewer than three
key-switch digits (fhe_accel_top.cpp:204-207), which is another reason to
load the top level only.

The arithmetic cost of every operator is independent of the residues
(fixed-width Barrett products), so ciphertexts, plaintexts, keys and tables
are seeded uniform residues and all rotations share one key region; the
residues this chain produces are not checked here (the reference's results
are pinned by tests/test_oracle.py).

Work units. A query's server work splits into units of similar cost:
  * large configuration (packed compaction, evaluated at 3 limbs): coarse
    ciphertext k (8 per query): sub_plain, relinearised square, tree sum of
    7 rotations, centroid-slot mask and rescale, rotation by -k, add; and
    candidate batch t (128 per query: 16 probed lists of about 977
    vectors, 8 batches of B = 128 each): sub_plain, square, 7 tree
    rotations by 128 * 2^s, prefix mask and rescale, placement rotation by
    -128 (t mod 128) (one key switch), add;
  * small configuration (the reference chain): stage 1/1b (one unit:
    square, 6 tree rotations, and for each of the 32 lists a mask, rescale,
    eval_rotate by i * 63 in power-of-two steps, add) and each candidate
    batch of the query's 4 probed lists.
One worker process per host core (the reference kernel keeps static global
state, so threads cannot share it) runs units in turn; every step each
worker runs `units_per_step` units, and the rate is the query fractions
completed over the wall time of the timed steps.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

from .oracle import Orc, Ref, RefBus, RefTopArgs, tables_py as T

OP_NTT, OP_INTT, OP_ADD, OP_SUB, OP_MUL, OP_AUTO, OP_KS, OP_RESCALE, OP_LOAD = 1, 2, 3, 4, 5, 6, 7, 8, 99


# ---------------------------------------------------------------------------
# workload shapes (no GPU library: primes from the oracle's own search)
# ---------------------------------------------------------------------------
def shape(workload: str) -> dict:
    """The CKKS parameters, query shape and per-query work units of a workload."""
    from anns_fhe_b200.workloads import LARGE, SMALL
    spec = SMALL if workload == "small" else LARGE      # the reference's own chain on either large form
    log_n, n = spec.log_n, 1 << spec.log_n
    q = T.ntt_primes(log_n, spec.q_bits, spec.num_q)
    p = T.ntt_primes(log_n, spec.p_bits, spec.num_p, q)
    slots = n // 2
    D, B = spec.d, slots // spec.d
    L = spec.eval_level or spec.num_q
    sh = dict(spec=spec, name=spec.name, log_n=log_n, n=n, q=q, p=p, alpha=spec.alpha, D=D, B=B, slots=slots,
              L=L, L_top=spec.num_q, compaction=spec.compaction)
    if spec.compaction == "packed":
        n_coarse = -(-spec.n_list // (slots // D))
        per_list = -(-spec.n_vectors // spec.n_list // 1)            # vectors per list on average (rounded up)
        batches = spec.nprobe * -(-per_list // B)
        sh["units"] = [("c", k) for k in range(n_coarse)] + [("b", t) for t in range(batches)]
        sh["units_desc"] = (f"{n_coarse} coarse-ciphertext units + {batches} candidate-batch units per query "
                            f"({spec.nprobe} probes x ceil({per_list} / {B}))")
    else:
        counts = small_batches(spec, B)
        offs, off = [], 0
        for cnt in counts:
            if off % slots + cnt > slots:
                off = (off // slots + 1) * slots
            offs.append(off)
            off += cnt
        sh["units"] = [("s1", 0)] + [("b", (o, c)) for o, c in zip(offs, counts)]
        sh["units_desc"] = f"1 stage-1/1b unit + {len(counts)} candidate-batch units per query"
    return sh


def small_batches(spec, B: int) -> list[int]:
    """Candidate counts per batch of a typical query's probed lists (the
    index of the small database is quick to train)."""
    from anns_fhe_b200.ivfpq import IvfPqIndex, gaussian_mixture, plaintext_search
    X = gaussian_mixture(spec.n_vectors, spec.d, spec.components, spec.sigma, spec.seed)
    idx = IvfPqIndex.train(X, spec.n_list, spec.M, spec.K, spec.seed)
    probes, _, _, _ = plaintext_search(idx, X[0], spec.nprobe, spec.top_k)
    counts = []
    for c in probes:
        m = len(idx.lists[c])
        counts += [min(B, m - b0) for b0 in range(0, m, B)]
    return counts


def rotation_steps(sh: dict) -> list[int]:
    D, B, slots = sh["D"], sh["B"], sh["slots"]
    steps = set()
    s = 1
    while s < D:
        steps.update((s, B * s))
        s <<= 1
    if sh["compaction"] == "packed":
        steps.update(-k for k in range(1, -(-sh["spec"].n_list // (slots // D))))
        steps.update(-B * m for m in range(1, slots // B))
    else:
        for i in range(sh["spec"].n_list):
            r = i * (D - 1)
            while r:
                b = 1 << (r.bit_length() - 1)
                steps.add(b)
                r -= b
        s = 1
        while s < slots:
            steps.add(-s)
            s <<= 1
    return sorted(steps)


# ---------------------------------------------------------------------------
# backends: the reference's fhe_accel_top over its SimMemoryBus, or the port
# ---------------------------------------------------------------------------
class OrcBus:
    """The C restatement's fhe_accel_top over numpy arenas (kind "port")."""

    def __init__(self, n: int, poly_words: int, key_words: int):
        self.orc = Orc()
        self.h = self.orc.new_ctx(n)
        self.poly = np.zeros(poly_words, dtype=np.uint64)
        self.key = np.zeros(key_words, dtype=np.uint64)

    def write_poly(self, off, x):
        self.poly[off:off + len(x)] = x

    def read_poly(self, off, count):
        return self.poly[off:off + count].copy()

    def write_key(self, off, x):
        self.key[off:off + len(x)] = x

    def top_args(self, a):
        return a

    def top(self, a):
        rc = self.orc.accel_top(self.h, self.poly, self.key, a)
        assert rc == 0, f"orc_accel_top returned {rc}"

    def close(self):
        self.orc.free_ctx(self.h)


class RefBusBackend:
    def __init__(self, n: int, poly_words: int, key_words: int):
        self.bus = RefBus(Ref(n), poly_words, key_words)

    def write_poly(self, off, x):
        self.bus.write_poly(off, x)

    def read_poly(self, off, count):
        return self.bus.read_poly(off, count)

    def write_key(self, off, x):
        self.bus.write_key(off, x)

    def top_args(self, a):
        return Ref.top_args(a)

    def top(self, a):
        self.bus.top(a)

    def close(self):
        self.bus.close()


def backend_kind(n: int) -> str:
    return "reference" if Ref.available(n) else "port"


class Regs:
    """fhe_accel_top's registers (afhe_accel_args field names), set once per
    context and per call; the backends convert them to their own struct."""

    def __init__(self):
        self.qhat_inv_offset = [0] * 16
        self.qhat_modp_offset = [0] * 16
        self.rns_primes = [0] * 64
        self.p_primes = [0] * 16
        self.barrett_m_q_lo = [0] * 64
        self.barrett_m_q_hi = [0] * 64
        self.barrett_k_q = [0] * 64
        self.barrett_m_p_lo = [0] * 16
        self.barrett_m_p_hi = [0] * 16
        self.barrett_k_p = [0] * 16
        self.n_inv_q = [0] * 64
        self.n_inv_p = [0] * 16
        for f in ("op_code", "active_limbs", "src_a_offset", "src_b_offset", "dst_offset", "evk_offset",
                  "prime_idx", "galois_elt", "sizeQl", "sizeP", "numPartQ", "alpha", "n_inv_mod_q_last",
                  "twiddles_q_offset", "inv_twiddles_q_offset", "twiddles_p_offset", "inv_twiddles_p_offset",
                  "p_inv_mod_q_offset", "p_hat_inv_mod_p_offset", "p_hat_mod_q_offset", "qlql_offset",
                  "qlinv_offset"):
            setattr(self, f, 0)


# ---------------------------------------------------------------------------
# FHEHostDriver's operator sequence (fhe_host_driver.cpp:177-404)
# ---------------------------------------------------------------------------
class HostDriver:
    """Restates FHEHostDriver over fhe_accel_top: the same op codes, host
    copies and scratch slots per composite. Keys: one region laid out as the
    reference's OP 7 reads it (digit j limb i at evk + (j (l + K) + i) N,
    evk_b after numPartQ digits); rotation steps each have an automorphism
    map in poly_gmem, as initialize_context_from_directory installs them."""

    def __init__(self, bus, log_n: int, q: list[int], p: list[int], alpha: int, L_top: int, seed: int,
                 steps: list[int], slot_words: int, scratch_base: int, maps_base: int, key_base: int,
                 tables: dict | None = None):
        """tables: None fills tables and the key with seeded uniform residues
        (a timing run); else a dict with the real ones: "tw", "itw" (all
        primes, Q then P), "qhat_inv" / "qhat_modp" (per digit), "pinv",
        "phinv", "phq", "qlql", "qlinv" for level L_top, and "key" (the
        evaluation key region)."""
        self.bus, self.log_n, self.n = bus, log_n, 1 << log_n
        self.q, self.p, self.alpha, self.K = list(q), list(p), alpha, len(p)
        self.L_top = L_top
        n = self.n
        rng = np.random.default_rng(seed)
        r = Regs()
        for i, x in enumerate(self.q):
            r.rns_primes[i] = x
            r.barrett_m_q_lo[i], r.barrett_m_q_hi[i], r.barrett_k_q[i] = T.barrett(x)
            r.n_inv_q[i] = pow(n, -1, x)
        for i, x in enumerate(self.p):
            r.p_primes[i] = x
            r.barrett_m_p_lo[i], r.barrett_m_p_hi[i], r.barrett_k_p[i] = T.barrett(x)
            r.n_inv_p[i] = pow(n, -1, x)
        r.sizeP, r.alpha = self.K, alpha
        # key_gmem: twiddles Q then P, inverse twiddles, CRT tables in 64-word
        # slots, keys 512-word aligned (fhe_host_driver.cpp:63-117)
        allp = self.q + self.p
        Lq = len(self.q)
        cur = 0
        r.twiddles_q_offset, r.twiddles_p_offset = cur, cur + Lq * n
        cur += len(allp) * n
        r.inv_twiddles_q_offset, r.inv_twiddles_p_offset = cur, cur + Lq * n
        cur += len(allp) * n
        for j in range(3):
            r.qhat_inv_offset[j] = cur
            cur += 64
            r.qhat_modp_offset[j] = cur
            cur += 64
        r.p_inv_mod_q_offset, r.p_hat_inv_mod_p_offset, r.p_hat_mod_q_offset = cur, cur + 64, cur + 128
        cur += 256
        r.qlql_offset, r.qlinv_offset = cur, cur + 64
        cur += 128
        self.tables_end = cur
        self.regs = r
        self.key_base = key_base
        self.key_words = 2 * (-(-L_top // alpha)) * (L_top + self.K) * n
        if tables is None:
            uni = lambda primes: np.concatenate([rng.integers(0, x, n, dtype=np.uint64) for x in primes])
            bus.write_key(0, uni(allp))
            bus.write_key(len(allp) * n, uni(allp))
            for off in range(2 * len(allp) * n, cur, 64):
                bus.write_key(off, rng.integers(0, min(allp), 64, dtype=np.uint64))
            for off in range(0, self.key_words, 1 << 20):
                m = min(1 << 20, self.key_words - off)
                bus.write_key(key_base + off, rng.integers(0, min(allp), m, dtype=np.uint64))
        else:
            bus.write_key(r.twiddles_q_offset, tables["tw"])
            bus.write_key(r.inv_twiddles_q_offset, tables["itw"])
            for j, (a, b) in enumerate(zip(tables["qhat_inv"], tables["qhat_modp"])):
                bus.write_key(r.qhat_inv_offset[j], a)
                bus.write_key(r.qhat_modp_offset[j], b)
            for name, off in (("pinv", r.p_inv_mod_q_offset), ("phinv", r.p_hat_inv_mod_p_offset),
                              ("phq", r.p_hat_mod_q_offset), ("qlql", r.qlql_offset), ("qlinv", r.qlinv_offset)):
                bus.write_key(off, tables[name])
            bus.write_key(key_base, tables["key"])
        # rotation directory: one automorphism map per step, packed u32 pairs
        self.maps = {}
        for i, st in enumerate(steps):
            k = T.galois(log_n, st)
            m = T.auto_map(log_n, k).astype(np.uint64)
            off = maps_base + i * (n // 2)
            bus.write_poly(off, m[0::2] | (m[1::2] << np.uint64(32)))
            self.maps[st] = (off, k)
        self.W = slot_words
        s0 = scratch_base
        self.D0, self.D1, self.D2, self.KS_C0, self.TMP = (s0 + i * slot_words for i in range(5))
        self.load_context(L_top)

    # FHEHostDriver::dispatch (fhe_host_driver.cpp:177-204), level-aware numPartQ
    def dispatch(self, op, src_a, src_b, dst, evk, active_limbs, sizeQl, galois=0):
        r = self.regs
        r.op_code, r.src_a_offset, r.src_b_offset, r.dst_offset = op, src_a, src_b, dst
        r.evk_offset, r.active_limbs, r.galois_elt, r.sizeQl = evk, active_limbs, galois, sizeQl
        r.numPartQ = -(-sizeQl // self.alpha)
        r.n_inv_mod_q_last = r.n_inv_q[active_limbs - 1] if 0 < active_limbs <= len(self.q) else 0
        self.bus.top(self.bus.top_args(r))

    def load_context(self, level):
        self.dispatch(OP_LOAD, 0, 0, 0, 0, level, level)

    def poly_add(self, a, b, d, l):
        self.dispatch(OP_ADD, a, b, d, 0, l, l)

    def poly_sub(self, a, b, d, l):
        self.dispatch(OP_SUB, a, b, d, 0, l, l)

    def poly_mul(self, a, b, d, l):
        self.dispatch(OP_MUL, a, b, d, 0, l, l)

    def automorphism(self, src, map_off, dst, l, galois):
        self.dispatch(OP_AUTO, src, map_off, dst, 0, l, l, galois)

    def key_switch(self, src, evk, dst, l):
        self.dispatch(OP_KS, src, 0, dst, evk, l, l)

    def rescale(self, c0, c1, dst, l):
        self.dispatch(OP_RESCALE, c0, c1, dst, 0, l, l)

    def copy(self, src, dst, words):
        self.bus.write_poly(dst, self.bus.read_poly(src, words))

    # composites (fhe_host_driver.cpp:248-404)
    def eval_add(self, a0, a1, b0, b1, d0, d1, l):
        self.poly_add(a0, b0, d0, l)
        self.poly_add(a1, b1, d1, l)

    def eval_sub_plain(self, a0, a1, pt, d0, d1, l):
        self.poly_sub(a0, pt, d0, l)
        if a1 != d1:
            self.copy(a1, d1, l * self.n)

    def eval_mult_relin_rescale(self, a0, a1, b0, b1, d0, d1, l):
        self.poly_mul(a0, b0, self.D0, l)
        self.poly_mul(a1, b1, self.D2, l)
        self.poly_mul(a0, b1, self.D1, l)
        self.poly_mul(a1, b0, self.TMP, l)
        self.poly_add(self.D1, self.TMP, self.D1, l)
        self.key_switch(self.D2, self.key_base, self.KS_C0, l)
        self.poly_add(self.D0, self.KS_C0, self.D0, l)
        self.poly_add(self.D1, self.KS_C0 + l * self.n, self.D1, l)
        self.rescale(self.D0, self.D1, self.TMP, l)
        w = (l - 1) * self.n
        self.copy(self.TMP, d0, w)
        self.copy(self.TMP + w, d1, w)

    def eval_mult_plain_rescale(self, a0, a1, pt, d0, d1, l):
        self.poly_mul(a0, pt, self.D0, l)
        self.poly_mul(a1, pt, self.D1, l)
        self.rescale(self.D0, self.D1, self.TMP, l)
        w = (l - 1) * self.n
        self.copy(self.TMP, d0, w)
        self.copy(self.TMP + w, d1, w)

    def eval_rotate_single_step(self, i0, i1, d0, d1, step, l):
        map_off, galois = self.maps[step]
        self.automorphism(i0, map_off, self.D0, l, galois)
        self.automorphism(i1, map_off, self.D1, l, galois)
        self.key_switch(self.D1, self.key_base, self.KS_C0, l)
        self.poly_add(self.D0, self.KS_C0, d0, l)
        self.copy(self.KS_C0 + l * self.n, d1, l * self.n)

    def eval_rotate(self, i0, i1, d0, d1, total, l):
        if total == 0:
            if i0 != d0:
                self.copy(i0, d0, l * self.n)
            if i1 != d1:
                self.copy(i1, d1, l * self.n)
            return
        c0, c1 = i0, i1
        t0, t1 = self.TMP, self.TMP + l * self.n
        rem, sign = abs(total), 1 if total > 0 else -1
        while rem > 0:
            s = 1 << (rem.bit_length() - 1)
            n0, n1 = (d0, d1) if rem == s else (t0, t1)
            self.eval_rotate_single_step(c0, c1, n0, n1, sign * s, l)
            c0, c1 = n0, n1
            rem -= s


# ---------------------------------------------------------------------------
# one worker: arenas, keys and units of the chain
# ---------------------------------------------------------------------------
class ChainWorker:
    def __init__(self, sh: dict, seed: int, backend: str | None = None):
        self.sh = sh
        n, L = sh["n"], sh["L"]
        self.n, self.L = n, L
        steps = rotation_steps(sh)
        W = 8 * n                                   # words per poly_gmem slot (a KS output is 2 l N <= 6 N)
        self.W = W
        names = ["q0", "q1", "d0", "d1", "pt", "mask", "x0", "x1", "y0", "y1", "acc0", "acc1"]
        self.slot = {k: i * W for i, k in enumerate(names)}
        scratch = len(names) * W
        maps = scratch + 5 * W
        poly_words = maps + len(steps) * (n // 2)
        kind = backend or backend_kind(n)
        self.kind = kind
        kb = 2 * len(sh["q"] + sh["p"]) * n + 2048
        key_words = kb + 2 * (-(-sh["L_top"] // sh["alpha"])) * (sh["L_top"] + len(sh["p"])) * n
        self.bus = (RefBusBackend if kind == "reference" else OrcBus)(n, poly_words, key_words)
        self.drv = HostDriver(self.bus, sh["log_n"], sh["q"], sh["p"], sh["alpha"], sh["L_top"], seed, steps, W,
                              scratch, maps, kb)
        rng = np.random.default_rng(seed + 1)
        for k in names:
            self.bus.write_poly(self.slot[k], np.concatenate([rng.integers(0, x, n, dtype=np.uint64)
                                                              for x in sh["q"][:L]]))

    def tree(self, c0, c1, stride, l):
        """x += rot(x, s) for s = stride, 2 stride, .., (D / 2) stride."""
        d = self.drv
        s = stride
        while s < self.sh["D"] * stride:
            d.eval_rotate(c0, c1, self.slot["y0"], self.slot["y1"], s, l)
            d.eval_add(c0, c1, self.slot["y0"], self.slot["y1"], c0, c1, l)
            s <<= 1

    def square(self, src, l):
        """sub_plain then relinearised square into x (l -> l - 1 limbs)."""
        d, s = self.drv, self.slot
        d.eval_sub_plain(s[src + "0"], s[src + "1"], s["pt"], s["d0"], s["d1"], l)
        d.eval_mult_relin_rescale(s["d0"], s["d1"], s["d0"], s["d1"], s["x0"], s["x1"], l)

    def unit(self, u) -> None:
        kind, arg = u
        d, s, L, D, B = self.drv, self.slot, self.L, self.sh["D"], self.sh["B"]
        if kind == "c":             # large: coarse ciphertext k
            self.square("q", L)
            self.tree(s["x0"], s["x1"], 1, L - 1)
            d.eval_mult_plain_rescale(s["x0"], s["x1"], s["mask"], s["x0"], s["x1"], L - 1)
            if arg:
                d.eval_rotate_single_step(s["x0"], s["x1"], s["x0"], s["x1"], -arg, L - 2)
            d.eval_add(s["acc0"], s["acc1"], s["x0"], s["x1"], s["acc0"], s["acc1"], L - 2)
        elif kind == "b" and self.sh["compaction"] == "packed":     # large: candidate batch t
            self.square("d", L)
            self.tree(s["x0"], s["x1"], B, L - 1)
            d.eval_mult_plain_rescale(s["x0"], s["x1"], s["mask"], s["x0"], s["x1"], L - 1)
            m = arg % (self.sh["slots"] // B)
            if m:
                d.eval_rotate_single_step(s["x0"], s["x1"], s["x0"], s["x1"], -B * m, L - 2)
            d.eval_add(s["acc0"], s["acc1"], s["x0"], s["x1"], s["acc0"], s["acc1"], L - 2)
        elif kind == "s1":          # small: stage 1 / 1b of one query
            self.square("q", L)
            self.tree(s["x0"], s["x1"], 1, L - 1)
            for i in range(self.sh["spec"].n_list):
                d.eval_mult_plain_rescale(s["x0"], s["x1"], s["mask"], s["d0"], s["d1"], L - 1)
                if i:
                    d.eval_rotate(s["d0"], s["d1"], s["d0"], s["d1"], i * (D - 1), L - 2)
                d.eval_add(s["acc0"], s["acc1"], s["d0"], s["d1"], s["acc0"], s["acc1"], L - 2)
        else:                       # small: candidate batch at slot offset `off`
            off, _ = arg
            self.square("d", L)
            self.tree(s["x0"], s["x1"], B, L - 1)
            d.eval_mult_plain_rescale(s["x0"], s["x1"], s["mask"], s["x0"], s["x1"], L - 1)
            if off % self.sh["slots"]:
                d.eval_rotate(s["x0"], s["x1"], s["x0"], s["x1"], -(off % self.sh["slots"]), L - 2)
            d.eval_add(s["acc0"], s["acc1"], s["x0"], s["x1"], s["acc0"], s["acc1"], L - 2)

    def close(self):
        self.bus.close()


def _worker_main(conn, workload: str, wid: int, nworkers: int, units_per_step: int, backend):
    sh = shape(workload)
    w = ChainWorker(sh, seed=101 + wid, backend=backend)
    units = sh["units"]
    conn.send(("ready", w.kind))
    step = 0
    while True:
        msg = conn.recv()
        if msg == "stop":
            break
        t0 = time.perf_counter()
        # all workers together run consecutive units of the query's list
        first = (step * nworkers + wid) * units_per_step
        for j in range(units_per_step):
            w.unit(units[(first + j) % len(units)])
        step += 1
        conn.send(("done", time.perf_counter() - t0))
    w.close()


def reference_rate(workload: str = "large", steps: int = 3, warmup: int = 1, workers: int | None = None,
                   units_per_step: int = 1, backend: str | None = None) -> dict:
    """Queries/s of the server chain on the host's cores: `warmup` untimed
    steps, then `steps` timed ones; every step each worker process runs
    `units_per_step` work units. Setup (arenas, tables, keys) is outside the
    timed steps. Returns the rate and a description of the sample."""
    sh = shape(workload)
    U = len(sh["units"])
    workers = workers or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    pipes, procs = [], []
    for wid in range(workers):
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_worker_main, args=(b, workload, wid, workers, units_per_step, backend), daemon=True)
        pr.start()
        pipes.append(a)
        procs.append(pr)
    kinds = {c.recv()[1] for c in pipes}
    try:
        walls = []
        for it in range(warmup + steps):
            t0 = time.perf_counter()
            for c in pipes:
                c.send("go")
            for c in pipes:
                c.recv()
            if it >= warmup:
                walls.append(time.perf_counter() - t0)
    finally:
        for c in pipes:
            c.send("stop")
        for pr in procs:
            pr.join(timeout=30)
    wall = sum(walls)
    fractions = workers * units_per_step * steps / U        # queries' worth of units completed
    rate = fractions / wall
    kind = "reference" if kinds == {"reference"} else "port"
    what = ("the reference's HLS C-simulation rebuilt at N = %d over its SimMemoryBus, in FHEHostDriver's "
            "operator sequence of the reference's chain (%s compaction, depth 2, evaluated at %d limbs)"
            % (sh["n"], sh["compaction"], sh["L"])) if kind == "reference" else "the C restatement (oracle port)"
    return {"value": rate, "unit": "queries/s", "cores": workers, "kind": kind, "workload": sh["name"],
            "units_per_query": U, "seconds": wall, "ms_per_step": 1e3 * wall / max(1, steps),
            "sample": (f"{steps} timed steps after {warmup} warm-up; each step {workers} processes x "
                       f"{units_per_step} work unit(s) of the server chain ({sh['units_desc']}), "
                       f"{fractions:.2f} queries' worth in {wall:.1f}s; {what}; setup excluded")}


if __name__ == "__main__":
    import json
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    wl = sys.argv[1] if len(sys.argv) > 1 else "large"
    print(json.dumps(reference_rate(wl, steps=int(sys.argv[2]) if len(sys.argv) > 2 else 2,
                                    warmup=1, workers=int(sys.argv[3]) if len(sys.argv) > 3 else None)))
