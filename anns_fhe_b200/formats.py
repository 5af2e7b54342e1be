"""The reference's on-disk formats: the context directory its host driver
reads (cpp_host_model/src/fhe_host_driver.cpp:18-175) and SimMemoryBus's raw
word files (cpp_host_model/src/sim_memory_bus.cpp:64-102).

* Raw word files: little-endian uint64, polynomials limb-major, limb i at
  words [i N, (i + 1) N) (docs/data_format.md:46-103). A file's length gives
  its word count, and a wrong length is an error, as in load_*_file.
* rns_primes_Q.bin / rns_primes_P.bin: the Q / P chains, uint64 each.
* barrett_constants.bin: per prime, Q then P, m_lo (u64), m_hi (u64), k
  (u32): 20 bytes with no padding (fhe_host_driver.cpp:27-50).
* n_inv.bin: N^-1 mod each prime, Q then P.
* twiddles.bin / inv_twiddles.bin: (L + K) x N words, Q primes then P,
  tw[j] = psi^bitrev(j) (so psi = tw[N/2]).
* evalkey_mult_{a,b}_<d>.bin: digit d of the relinearisation key.
* rotation_keys_meta.txt: one line "step=<s> auto_idx=<k>" per rotation key.
* auto_map_step<s>.bin: N x uint32, the evaluation-form automorphism map.
* rotkey_step<s>_{a,b}_<d>.bin: digit d of the rotation key for step s.

A key digit file holds l + K limbs: its first l limbs are under q_0..q_{l-1}
and the last K under the special primes. The reference writes the
relinearisation key at the full level (l = L) and rotation keys one level
down (l = L - 1, "14 limbs per digit for Level 1", fhe_host_driver.cpp:156).
`install` lays every key out at the full level, the layout the composite
operators read. Q limbs a file does not have are zero, so such a key serves
ciphertexts of up to l limbs.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .driver import CkksParams, FheContext, FHEHostDriver, automorphism_map, barrett_constant, galois_elt, twiddles


# ---- raw files ----------------------------------------------------------------
def read_words(path: str, expected: int = 0) -> np.ndarray:
    """A raw little-endian uint64 file (SimMemoryBus::load_*_file)."""
    size = os.path.getsize(path)
    if size % 8:
        raise ValueError(f"{path}: {size} bytes is not a whole number of 64-bit words")
    if expected and size // 8 != expected:
        raise ValueError(f"{path}: size mismatch, {size // 8} words, expected {expected}")
    return np.fromfile(path, dtype="<u8").astype(np.uint64)


def write_words(path: str, words) -> None:
    """SimMemoryBus::save_poly_file: the words, little-endian uint64."""
    np.asarray(words, dtype=np.uint64).astype("<u8").tofile(path)


def read_barrett(path: str, count: int) -> list[tuple[int, int, int]]:
    """`count` Barrett records (m_lo, m_hi, k) of 20 bytes each."""
    rec = np.dtype([("lo", "<u8"), ("hi", "<u8"), ("k", "<u4")])
    a = np.fromfile(path, dtype=rec, count=count)
    if len(a) != count:
        raise ValueError(f"{path}: {len(a)} Barrett records, expected {count}")
    return [(int(r["lo"]), int(r["hi"]), int(r["k"])) for r in a]


def write_barrett(path: str, primes) -> None:
    rec = np.dtype([("lo", "<u8"), ("hi", "<u8"), ("k", "<u4")])
    a = np.zeros(len(primes), dtype=rec)
    for i, q in enumerate(primes):
        a[i] = barrett_constant(int(q))
    a.tofile(path)


_META = re.compile(r"step=(-?\d+)\s+auto_idx=(\d+)")


def read_rotation_meta(path: str) -> list[tuple[int, int]]:
    """(step, auto_idx) per non-empty line of rotation_keys_meta.txt."""
    out = []
    with open(path) as f:
        for line in f:
            if not line.strip():
                continue
            m = _META.search(line)
            if not m:
                raise ValueError(f"{path}: cannot parse {line.strip()!r}")
            out.append((int(m.group(1)), int(m.group(2))))
    return out


def write_rotation_meta(path: str, entries) -> None:
    with open(path, "w") as f:
        for step, idx in entries:
            f.write(f"step={step} auto_idx={idx}\n")


def read_auto_map(path: str, n: int) -> np.ndarray:
    a = np.fromfile(path, dtype="<u4")
    if a.size != n:
        raise ValueError(f"{path}: {a.size} map entries, expected {n}")
    return a.astype(np.uint32)


# ---- the context directory --------------------------------------------------------
@dataclass
class ContextPackage:
    params: CkksParams
    barrett_q: list
    barrett_p: list
    n_inv: np.ndarray                       # Q then P
    tw: np.ndarray                          # (L + K) x N
    itw: np.ndarray
    relin: tuple | None = None              # (a digits, b digits), each (dnum, l + K, N)
    rot: dict = field(default_factory=dict)  # step -> (auto_idx, map u32, a digits, b digits)


def _digits(vec_dir: str, stem: str, n: int, dnum: int):
    """(a, b) digit arrays of a key, or None if the files are absent."""
    out = []
    for ab in ("a", "b"):
        ds = []
        for d in range(dnum):
            path = os.path.join(vec_dir, f"{stem}_{ab}_{d}.bin")
            if not os.path.exists(path):
                return None
            w = read_words(path)
            if w.size % n:
                raise ValueError(f"{path}: not a whole number of limbs")
            ds.append(w.reshape(-1, n))
        out.append(np.stack(ds))
    return out[0], out[1]


def load_package(vec_dir: str, log_n: int, alpha: int) -> ContextPackage:
    """Read a context directory (initialize_context_from_directory's files).
    The ring degree and digit size are not in the directory (the reference
    fixes them at compile time), so the caller names them."""
    n = 1 << log_n
    q = [int(x) for x in read_words(os.path.join(vec_dir, "rns_primes_Q.bin"))]
    p = [int(x) for x in read_words(os.path.join(vec_dir, "rns_primes_P.bin"))]
    nq, np_ = len(q), len(p)
    bar = read_barrett(os.path.join(vec_dir, "barrett_constants.bin"), nq + np_)
    ninv = read_words(os.path.join(vec_dir, "n_inv.bin"), nq + np_)
    tw = read_words(os.path.join(vec_dir, "twiddles.bin"), (nq + np_) * n).reshape(nq + np_, n)
    itw = read_words(os.path.join(vec_dir, "inv_twiddles.bin"), (nq + np_) * n).reshape(nq + np_, n)
    psi = tuple(int(t[n // 2]) for t in tw)          # tw[j] = psi^bitrev(j), bitrev(N/2) = 1
    prm = CkksParams(log_n, q, p, alpha, psi)
    pkg = ContextPackage(prm, bar[:nq], bar[nq:], ninv, tw, itw)
    pkg.relin = _digits(vec_dir, "evalkey_mult", n, prm.dnum)
    meta = os.path.join(vec_dir, "rotation_keys_meta.txt")
    if os.path.exists(meta):
        for step, idx in read_rotation_meta(meta):
            m = read_auto_map(os.path.join(vec_dir, f"auto_map_step{step}.bin"), n)
            key = _digits(vec_dir, f"rotkey_step{step}", n, prm.dnum)
            pkg.rot[step] = (idx, m, key)
    return pkg


def check_package(pkg: ContextPackage) -> None:
    """The package's constants must be the ones its primes define: Barrett
    constants, N^-1, twiddles of its own roots, and each automorphism map
    the one for galois element 5^step. Raises ValueError naming the first
    mismatch (the reference would compute with it silently)."""
    prm = pkg.params
    n = prm.n
    primes = prm.q + prm.p
    for i, x in enumerate(primes):
        if tuple(pkg.barrett_q[i] if i < prm.L else pkg.barrett_p[i - prm.L]) != barrett_constant(x):
            raise ValueError(f"Barrett constant of prime {i} is not floor(2^k / q)")
        if int(pkg.n_inv[i]) * n % x != 1:
            raise ValueError(f"n_inv of prime {i} is not N^-1")
        tw, itw = twiddles(prm.log_n, x, prm.psi[i])
        if not (np.array_equal(tw, pkg.tw[i]) and np.array_equal(itw, pkg.itw[i])):
            raise ValueError(f"twiddles of prime {i} are not the powers of psi = tw[N/2]")
    for step, (_, m, _) in pkg.rot.items():
        if not np.array_equal(m, automorphism_map(prm.log_n, galois_elt(prm.log_n, step))):
            raise ValueError(f"auto_map_step{step} is not the evaluation-form map of 5^{step}")


def full_level_key(prm: CkksParams, digits) -> np.ndarray:
    """A key (a digits, b digits; each digit l + K limbs) in the full-level
    layout: digit j's Q limb i at (j (L + K) + i) N, P limb k at
    (j (L + K) + L + k) N, b after all a digits. Missing Q limbs are zero."""
    n, Lq, K, dnum = prm.n, prm.L, prm.K, prm.dnum
    out = np.zeros((2, dnum, Lq + K, n), dtype=np.uint64)
    for h, ds in enumerate(digits):
        lv = ds.shape[1] - K
        if lv < 1 or lv > Lq:
            raise ValueError(f"key digit has {ds.shape[1]} limbs; expected l + {K} with 1 <= l <= {Lq}")
        out[h, :, :lv] = ds[:, :lv]
        out[h, :, Lq:] = ds[:, lv:]
    return out.ravel()


def install(pkg: ContextPackage, ctx: FheContext, key_base: int | None = None) -> dict:
    """Load a package into a context the way initialize_context_from_directory
    fills key_gmem: twiddles (Q then P) from word 0, inverse twiddles after
    them. Then the keys, 512-word aligned after `key_base` (default: after the
    twiddles), each in the full-level layout, registered in the context's
    key directory. Returns {"relin": offset, step: offset, ...}."""
    prm = pkg.params
    n, S = prm.n, prm.L + prm.K
    ctx.write_key(0, pkg.tw.ravel())
    ctx.write_key(S * n, pkg.itw.ravel())
    cur = key_base if key_base is not None else 2 * S * n
    drv = FHEHostDriver(ctx)
    offs = {}

    def put(digits):
        nonlocal cur
        cur = (cur + 511) & ~511
        words = full_level_key(prm, digits)
        ctx.write_key(cur, words)
        at = cur
        cur += words.size
        return at
    if pkg.relin is not None:
        offs["relin"] = put(pkg.relin)
        drv.set_relin_key(offs["relin"])
    for step, (_, _, key) in sorted(pkg.rot.items()):
        if key is not None:
            offs[step] = put(key)
            drv.add_rotation_key(step, offs[step])
    offs["first_free"] = cur
    return offs


def package_key_words(pkg: ContextPackage) -> int:
    """key_gmem words `install` needs."""
    prm = pkg.params
    keys = (pkg.relin is not None) + sum(1 for v in pkg.rot.values() if v[2] is not None)
    return 2 * (prm.L + prm.K) * prm.n + keys * (prm.key_words() + 512)


def save_package(vec_dir: str, prm: CkksParams, relin=None, rot=None, rot_levels: int | None = None) -> None:
    """Write a context directory in the reference's format. relin / rot[step]:
    keys in the full-level layout (as `install` and the context use them);
    rotation keys are written with rot_levels Q limbs per digit (default
    L - 1, as the reference writes them)."""
    os.makedirs(vec_dir, exist_ok=True)
    n, Lq, K, dnum = prm.n, prm.L, prm.K, prm.dnum
    primes = prm.q + prm.p
    psi = prm.psi or tuple(int(L.load().afhe_min_primitive_root(prm.log_n, x)) for x in primes)
    write_words(os.path.join(vec_dir, "rns_primes_Q.bin"), prm.q)
    write_words(os.path.join(vec_dir, "rns_primes_P.bin"), prm.p)
    write_barrett(os.path.join(vec_dir, "barrett_constants.bin"), primes)
    write_words(os.path.join(vec_dir, "n_inv.bin"), [pow(n, -1, x) for x in primes])
    tws = [twiddles(prm.log_n, x, s) for x, s in zip(primes, psi)]
    write_words(os.path.join(vec_dir, "twiddles.bin"), np.concatenate([t[0] for t in tws]))
    write_words(os.path.join(vec_dir, "inv_twiddles.bin"), np.concatenate([t[1] for t in tws]))

    def digits(key, lv):
        k = np.asarray(key, dtype=np.uint64).reshape(2, dnum, Lq + K, n)
        return [np.concatenate([k[h, :, :lv], k[h, :, Lq:]], axis=1) for h in range(2)]

    def write_key(stem, key, lv):
        for ab, ds in zip("ab", digits(key, lv)):
            for d in range(dnum):
                write_words(os.path.join(vec_dir, f"{stem}_{ab}_{d}.bin"), ds[d].ravel())
    if relin is not None:
        write_key("evalkey_mult", relin, Lq)
    if rot:
        lv = rot_levels or max(1, Lq - 1)
        entries = []
        for step in sorted(rot):
            g = galois_elt(prm.log_n, step)
            entries.append((step, g))
            automorphism_map(prm.log_n, g).astype("<u4").tofile(os.path.join(vec_dir, f"auto_map_step{step}.bin"))
            write_key(f"rotkey_step{step}", rot[step], lv)
        write_rotation_meta(os.path.join(vec_dir, "rotation_keys_meta.txt"), entries)


def context_for(pkg: ContextPackage, poly_words: int, extra_key_words: int = 0, device: int = 0,
                max_batch: int = 0) -> tuple[FheContext, dict]:
    """A context on the package's primes and roots, with the package installed."""
    ctx = FheContext(pkg.params, poly_words=poly_words, key_words=package_key_words(pkg) + extra_key_words,
                     device=device, max_batch=max_batch)
    return ctx, install(pkg, ctx)
