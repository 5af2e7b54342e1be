"""Shared test setup: the `gpu` marker, import paths and common fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Contexts made by the tests take the one-kernel key switch for launches of
# any size (the library's default sends launches smaller than half a wave of
# SMs to the multi-kernel path), so single-ciphertext checks exercise it; the
# multi-kernel path has its own contexts (AFHE_KS_FUSED=0) in the tests that
# compare the two.
os.environ.setdefault("AFHE_FUSED_MIN", "1")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    # temporary files stay inside the tree (git-ignored), not in the system's temp folder
    if not config.option.basetemp:
        os.makedirs(os.path.join(ROOT, "tests", "_build"), exist_ok=True)
        config.option.basetemp = os.path.join(ROOT, "tests", "_build", "pytest-tmp")


@pytest.fixture(scope="session")
def lib():
    from anns_fhe_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Orc
    return Orc()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref
    if not Ref.available():
        try:
            from oracle.oracle import build_oracle
            build_oracle(ref=True)
        except Exception:
            pass
    if not Ref.available():
        pytest.skip("reference HLS library not built (reference tree absent)")
    return Ref()
