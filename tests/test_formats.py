"""The reference's on-disk formats (cpp_host_model/src/fhe_host_driver.cpp:18-175,
sim_memory_bus.cpp:64-102), host side: a context directory written by
`save_package` reads back field for field, its constants pass the
consistency check, a corrupted constant is caught, and keys written at
fewer Q limbs (the reference's level-1 rotation keys) come back in the
full-level layout with the missing limbs zero."""
import os

import numpy as np
import pytest

from anns_fhe_b200 import formats as F
from anns_fhe_b200.driver import CkksParams, automorphism_map, galois_elt


def _params(psi_power=1):
    prm = CkksParams.generate(10, 3, 40, 2, 45, 2)
    if psi_power != 1:
        from anns_fhe_b200 import _lib as L
        lib = L.load()
        prm.psi = tuple(pow(int(lib.afhe_min_primitive_root(10, x)), psi_power, x) for x in prm.q + prm.p)
    return prm


def _key(prm, rng):
    return np.concatenate([rng.integers(0, x, prm.n, dtype=np.uint64)
                           for _ in range(2 * prm.dnum) for x in prm.q + prm.p])


def test_raw_words_and_size_check(tmp_path):
    a = np.arange(12, dtype=np.uint64) * np.uint64(2**61 - 1)
    p = str(tmp_path / "w.bin")
    F.write_words(p, a)
    assert os.path.getsize(p) == 96
    assert np.array_equal(F.read_words(p), a)
    assert np.array_equal(F.read_words(p, 12), a)
    with pytest.raises(ValueError):
        F.read_words(p, 13)


def test_barrett_records_are_20_bytes(tmp_path):
    prm = _params()
    p = str(tmp_path / "barrett_constants.bin")
    F.write_barrett(p, prm.q + prm.p)
    assert os.path.getsize(p) == 20 * 5
    recs = F.read_barrett(p, 5)
    for (lo, hi, k), q in zip(recs, prm.q + prm.p):
        m = (hi << 64) | lo
        assert k == 2 * q.bit_length() + 3 and m == (1 << k) // q


def test_rotation_meta_lines(tmp_path):
    p = str(tmp_path / "rotation_keys_meta.txt")
    F.write_rotation_meta(p, [(1, 5), (-4, 1234)])
    assert open(p).read() == "step=1 auto_idx=5\nstep=-4 auto_idx=1234\n"
    assert F.read_rotation_meta(p) == [(1, 5), (-4, 1234)]


@pytest.mark.parametrize("psi_power", [1, 3])
def test_package_round_trip(tmp_path, psi_power):
    prm = _params(psi_power)
    rng = np.random.default_rng(2)
    relin = _key(prm, rng)
    rot = {1: _key(prm, rng), -2: _key(prm, rng)}
    d = str(tmp_path / "ctx")
    F.save_package(d, prm, relin=relin, rot=rot)
    pkg = F.load_package(d, prm.log_n, prm.alpha)
    assert pkg.params.q == prm.q and pkg.params.p == prm.p
    if psi_power != 1:
        assert pkg.params.psi == prm.psi
    F.check_package(pkg)
    assert np.array_equal(F.full_level_key(prm, pkg.relin), relin)
    for step, key in rot.items():
        idx, m, digits = pkg.rot[step]
        assert idx == galois_elt(prm.log_n, step)
        assert np.array_equal(m, automorphism_map(prm.log_n, idx))
        got = F.full_level_key(prm, digits).reshape(2, prm.dnum, prm.L + prm.K, prm.n)
        want = key.reshape(2, prm.dnum, prm.L + prm.K, prm.n).copy()
        assert not got[:, :, prm.L - 1].any()          # written one level down: limb L-1 absent
        want[:, :, prm.L - 1] = 0
        assert np.array_equal(got, want)


def test_check_catches_a_bad_constant(tmp_path):
    prm = _params()
    d = str(tmp_path / "ctx")
    F.save_package(d, prm)
    ninv = F.read_words(os.path.join(d, "n_inv.bin"))
    ninv[1] ^= np.uint64(1)
    F.write_words(os.path.join(d, "n_inv.bin"), ninv)
    with pytest.raises(ValueError, match="n_inv"):
        F.check_package(F.load_package(d, prm.log_n, prm.alpha))


def test_ranked_prefix_is_the_stable_argsort_prefix():
    """The client's vectorised top-k equals np.argsort(kind="stable")[:k] row
    by row: ragged rows, rows shorter than k, empty rows, and ties (including
    ties at the k-th value)."""
    from anns_fhe_b200.workloads import ranked_prefix
    rng = np.random.default_rng(12)
    for trial in range(40):
        rows = int(rng.integers(1, 12))
        width = int(rng.integers(1, 300))
        vals = rng.integers(0, 6 if trial % 2 else 10**6, (rows, width)).astype(np.float64)
        pos = []
        for _ in range(rows):
            m = int(rng.integers(0, width + 1))
            sel = rng.choice(width, m, replace=False)      # any order: ties go by index in pos
            pos.append(np.sort(sel) if trial % 3 else sel)
        k = int(rng.integers(1, 12))
        got = ranked_prefix(vals, pos, k)
        for r in range(rows):
            want = np.argsort(vals[r, pos[r]], kind="stable")[:k]
            assert list(got[r]) == list(want), (trial, r)
    assert ranked_prefix(np.zeros((2, 4)), [np.zeros(0, np.int64)] * 2, 3)[1].size == 0
