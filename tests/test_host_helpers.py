"""Host-side helpers of the query chain, on the CPU: the ctypes arrays the
batched entry points take, the grouping of rotations into power-of-two
steps, and the centring of decrypted residues."""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib as L
from anns_fhe_b200.ckks import centred_coefficients, crt_centered
from anns_fhe_b200.query import InteractiveQueryManager as IQM


@pytest.mark.parametrize("m", [0, 1, 7, 296])
def test_ref_and_offset_arrays(m):
    rng = np.random.default_rng(m)
    pairs = [(int(a), int(b)) for a, b in rng.integers(0, 2**40, (m, 2))]
    for src in (pairs, np.array(pairs, dtype=np.uint64).reshape(m, 2)):
        p = IQM._refs(src)
        assert isinstance(p, C.POINTER(L.CtRef))
        assert [(p[i].c0_offset, p[i].c1_offset) for i in range(m)] == pairs
    offs = [int(x) for x in rng.integers(0, 2**50, m)]
    for src in (offs, np.array(offs, dtype=np.uint64)):
        p = IQM._offs(src)
        assert [p[i] for i in range(m)] == offs


class _Recorder:
    """Stands in for the query manager: records the batched rotations."""

    def __init__(self):
        self.calls = []

    def _rotate(self, cts, r, limbs):
        self.calls.append(([tuple(int(x) for x in c) for c in cts], r, limbs))


def _grouped_by_definition(items):
    """eval_rotate's steps (fhe_host_driver.cpp:361-404) for every item,
    grouped highest power first, positive shifts before negative ones."""
    items = [(ct, s) for ct, s in items if s]
    calls = []
    if not items:
        return calls
    top = max(abs(s) for _, s in items).bit_length()
    for b in range(top - 1, -1, -1):
        for sign in (1, -1):
            sub = [ct for ct, s in items if (s > 0) == (sign > 0) and (abs(s) >> b) & 1]
            if sub:
                calls.append((sub, sign * (1 << b), 3))
    return calls


def test_rotate_grouped_matches_its_definition():
    rng = np.random.default_rng(5)
    for trial in range(30):
        m = int(rng.integers(0, 60))
        items = [((int(rng.integers(0, 10**6)), int(rng.integers(0, 10**6))), int(rng.integers(-200, 201)))
                 for _ in range(m)]
        rec = _Recorder()
        IQM._rotate_grouped(rec, items, 3)
        assert rec.calls == _grouped_by_definition(items), trial


@pytest.mark.parametrize("level", [1, 2])
def test_centred_coefficients(level):
    from anns_fhe_b200.driver import find_ntt_primes
    q = find_ntt_primes(10, 50, 2)
    rng = np.random.default_rng(level)
    n = 1024
    limbs = np.concatenate([rng.integers(0, qi, (4, n), dtype=np.uint64) for qi in q[:level]], axis=1)
    limbs[0, 0] = q[0] // 2            # the largest value kept positive
    limbs[0, 1] = q[0] // 2 + 1        # the smallest one moved down
    got = centred_coefficients(limbs, q, level)
    want = np.stack([crt_centered(row, q[:level]).astype(np.float64) for row in limbs])
    assert np.array_equal(got, want)
