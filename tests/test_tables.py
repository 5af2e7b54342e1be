"""The library's host-side tables (primes, roots, twiddles, Barrett and CRT
constants, automorphism maps) equal their definitions computed independently
with Python integers (oracle.tables_py)."""
import numpy as np
import pytest

from anns_fhe_b200 import driver as D
from oracle.oracle import tables_py as T


@pytest.mark.parametrize("log_n,bits", [(10, 30), (13, 50), (14, 45), (16, 60)])
def test_root_and_twiddles(log_n, bits):
    q = D.find_ntt_primes(log_n, bits, 1)[0]
    n = 1 << log_n
    tw, itw = D.twiddles(log_n, q)
    psi = int(tw[T.bitrev(1, log_n)])  # tw[bitrev(1)] = psi^1
    assert pow(psi, n, q) == q - 1                      # primitive 2N-th root
    if log_n <= 13:
        assert psi == T.min_root(log_n, q)              # the smallest one
    rtw, ritw = T.twiddles(log_n, q, psi)
    assert np.array_equal(tw, rtw) and np.array_equal(itw, ritw)


def test_barrett_constant_matches_generator_formula():
    for q in D.find_ntt_primes(13, 50, 3) + D.find_ntt_primes(13, 60, 2):
        assert D.barrett_constant(q) == T.barrett(q)


@pytest.mark.parametrize("level,alpha,K", [(11, 4, 4), (10, 4, 4), (3, 1, 1), (12, 4, 4), (7, 3, 2)])
def test_crt_tables(level, alpha, K):
    q = D.find_ntt_primes(14, 45, level)
    p = D.find_ntt_primes(14, 60, K)
    parts = (level + alpha - 1) // alpha
    for j in range(parts):
        a, b = D.part_qhat_tables(q, level, alpha, j, p)
        ra, rb = T.part_qhat(q, level, alpha, j, p)
        assert np.array_equal(a, ra) and np.array_equal(b, rb)
    got = D.moddown_tables(q, level, p)
    exp = T.moddown(q, level, p)
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)
    if level > 1:
        got = D.rescale_tables(q, level)
        exp = T.rescale(q, level)
        for g, e in zip(got, exp):
            assert np.array_equal(g, e)


@pytest.mark.parametrize("log_n", [10, 13])
def test_galois_and_automorphism_map(log_n):
    for step in (1, 2, 5, -1, -4, 127):
        k = D.galois_elt(log_n, step)
        assert k == T.galois(log_n, step)
        m = D.automorphism_map(log_n, k)
        assert np.array_equal(m, T.auto_map(log_n, k))
        assert sorted(m.tolist()) == list(range(1 << log_n))   # a permutation
