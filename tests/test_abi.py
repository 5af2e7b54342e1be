"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every
entry point include/afhe.h declares; host-only helpers work on the CPU and
device calls fail with a status (never a crash) when no GPU is present."""
import ctypes as C

import numpy as np
import pytest

from anns_fhe_b200 import _lib


def test_every_header_symbol_is_exported(lib):
    names = _lib.header_symbols()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and every bound signature is declared in the header
    assert set(_lib.SIGNATURES) <= set(names)


def test_status_strings(lib):
    for s in range(9):
        assert lib.afhe_status_string(s)


def test_prime_search_is_ntt_friendly(lib):
    from anns_fhe_b200.driver import find_ntt_primes
    ps = find_ntt_primes(13, 50, 3)
    assert len(set(ps)) == 3
    for q in ps:
        assert q % (2 << 13) == 1 and q < 2**50 and q > 2**49
        assert pow(3, q - 1, q) == 1
    assert ps == sorted(ps, reverse=True)
    ex = find_ntt_primes(13, 50, 2, exclude=ps[:1])
    assert ex[0] == ps[1]


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU failure path")
def test_ctx_create_without_gpu_returns_status(lib):
    p = _lib.Params()
    p.log_n, p.num_q, p.num_p, p.alpha = 10, 1, 1, 1
    p.q[0] = 12289
    p.p[0] = 40961
    p.poly_words, p.key_words = 1024, 1024
    h = _lib.CTX()
    rc = lib.afhe_ctx_create(C.byref(p), C.byref(h))
    assert rc != _lib.OK
    assert not h.value


def test_ctx_create_rejects_bad_params(lib):
    p = _lib.Params()
    p.log_n, p.num_q, p.num_p, p.alpha = 9, 1, 1, 1   # log_n too small
    h = _lib.CTX()
    assert lib.afhe_ctx_create(C.byref(p), C.byref(h)) == _lib.E_ARG
    p.log_n = 10
    p.q[0] = 12289 + 2048                           # not prime
    p.p[0] = 40961
    assert lib.afhe_ctx_create(C.byref(p), C.byref(h)) == _lib.E_ARG


def test_ctx_create_rejects_bad_primes_and_roots(lib):
    """Parameter checks run before any device call, so they need no GPU."""
    from anns_fhe_b200.driver import find_ntt_primes
    q = find_ntt_primes(10, 40, 3)
    p = find_ntt_primes(10, 45, 1)

    def params(qs, ps, alpha=1, psi_q=()):
        pr = _lib.Params()
        pr.log_n, pr.num_q, pr.num_p, pr.alpha = 10, len(qs), len(ps), alpha
        for i, x in enumerate(qs):
            pr.q[i] = x
        for i, x in enumerate(ps):
            pr.p[i] = x
        for i, x in enumerate(psi_q):
            pr.psi_q[i] = x
        pr.poly_words, pr.key_words = 1 << 14, 1 << 14
        return pr

    h = _lib.CTX()

    def create(pr):
        return lib.afhe_ctx_create(C.byref(pr), C.byref(h))

    assert create(params([], p)) == _lib.E_ARG                      # no Q primes
    assert create(params(q, [])) == _lib.E_ARG                      # no P primes
    assert create(params(q, [q[0]])) == _lib.E_ARG                  # a prime twice
    assert create(params(q, p, alpha=0)) == _lib.E_ARG
    assert create(params(q[:2] + [10007], p)) == _lib.E_ARG          # prime, but not 1 mod 2N
    # psi must be a primitive 2N-th root: psi^N = -1 mod q
    assert create(params(q, p, psi_q=[1])) == _lib.E_ARG
    assert create(params(q, p, psi_q=[q[0]])) == _lib.E_ARG          # not reduced
    psi = lib.afhe_min_primitive_root(10, q[0])
    assert pow(psi, 1 << 10, q[0]) == q[0] - 1
    assert not h.value


def test_null_context_is_an_error(lib):
    assert lib.afhe_sync(None) == _lib.E_ARG
    a = _lib.AccelArgs()
    assert lib.afhe_dispatch(None, C.byref(a)) == _lib.E_ARG
    buf = np.zeros(4, dtype=np.uint64)
    assert lib.afhe_write_poly(None, 0, buf.ctypes.data_as(_lib.P64), 4) == _lib.E_ARG


def test_plain_c_caller_compiles_links_and_runs(lib):
    """tests/c/abi_host_calls.c includes include/afhe.h, links libafhe.so
    with gcc and makes the host-only calls and parameter checks from C."""
    import os
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc absent")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "anns_fhe_b200", "lib")
    out_dir = os.path.join(root, "tests", "c", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "abi_host_calls")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "c", "abi_host_calls.c"), "-L", libdir, "-lafhe",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.splitlines() == ["primes ok", "root ok", "galois ok", "checks ok: bad argument"]
