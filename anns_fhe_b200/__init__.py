"""B200-native CKKS evaluation core for encrypted IVF-PQ search.

The compute path is the CUDA C-ABI library ``lib/libafhe.so`` (sources in
``csrc/``, declared in ``include/afhe.h``); this package is its host-side
mirror of the reference's FHEHostDriver / InteractiveQueryManager.
"""
from ._lib import AfheError, load  # noqa: F401
from .driver import CkksParams, FheContext, FHEHostDriver  # noqa: F401
