"""The device encoder's transform plan (anns_fhe_b200/csrc/encode.cu) restated
on the CPU with the kernels' own index arithmetic: global stages for blocks
longer than a tile, then every shorter stage inside tiles, then the
bit-reversed read, / (N/2), * scale and rounding. At small rings it must give
the host encoder's coefficients (anns_fhe_b200.ckks.Encoder) up to a
rounding difference of one, and every index must stay inside the buffers.
(The GPU tests compare the device itself, test_gpu_encode.py.)"""
import numpy as np
import pytest

from anns_fhe_b200.ckks import Encoder


def stage(v, ln, ksi, rot, m, base=0, width=None):
    width = width or v.size
    lenh, lenq = ln >> 1, ln << 2
    b = np.arange(width // 2)
    i0 = base + (b // lenh) * ln + b % lenh
    assert i0.max() + lenh < base + width
    idx = (lenq - (rot[b % lenh] & (lenq - 1))) * (m // lenq)
    assert idx.min() >= 0 and idx.max() <= m
    a, c = v[i0].copy(), v[i0 + lenh].copy()
    v[i0], v[i0 + lenh] = a + c, (a - c) * ksi[idx]


def plan(vals, tile):
    s = vals.size
    m = 4 * s
    ksi = np.exp(2j * np.pi * np.arange(m + 1) / m)
    rot = np.array([pow(5, j, m) for j in range(s)], dtype=np.int64)
    v = vals.astype(np.complex128)
    tile = min(s, tile)
    ln = s
    while ln > tile:                       # fft_global_stage
        stage(v, ln, ksi, rot, m)
        ln >>= 1
    for t0 in range(0, s, tile):           # fft_tile_stages, one CTA per tile
        ln = tile
        while ln >= 2:
            stage(v, ln, ksi, rot, m, t0, tile)
            ln >>= 1
    log_s = s.bit_length() - 1
    rev = np.array([int(format(i, f"0{log_s}b")[::-1], 2) for i in range(s)])   # __brev(i) >> (32 - log_s)
    return v[rev] / s                      # fft_finish


@pytest.mark.parametrize("log_n,tile", [(10, 4096), (11, 64), (12, 256), (13, 4096)])
def test_plan_matches_host_encoder(log_n, tile):
    n = 1 << log_n
    s = n // 2
    rng = np.random.default_rng(log_n)
    z = rng.standard_normal(s) * 3
    x = plan(z, tile)
    scale = 2.0 ** 40
    coef = np.concatenate([np.rint(x.real * scale), np.rint(x.imag * scale)]).astype(np.int64)
    host = Encoder(log_n).encode(z, scale)
    d = coef - host
    assert np.all(np.abs(d) <= 1) and np.count_nonzero(d) <= max(1, n // 1000)
