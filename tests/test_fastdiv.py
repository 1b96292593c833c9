"""The multiply-high division used by the kernels' index arithmetic
(FastDiv in openqg_b200/csrc/oqg_dev.cuh), restated in integer arithmetic:
exact for every divisor the kernels use and numerators below 2^31."""
import numpy as np
import pytest


def magic(d):
    s = 0
    while (1 << s) < d:
        s += 1
    m = ((1 << 32) * ((1 << s) - d)) // d + 1
    return m & 0xFFFFFFFF, s


def fastdiv(n, d):
    m, s = magic(d)
    t = (m * n) >> 32
    return (t + n) >> s


@pytest.mark.parametrize("d", list(range(1, 70)) + [96, 127, 128, 192, 193, 320, 384, 513, 1025, 2049, 4097])
def test_fastdiv_exact(d):
    rng = np.random.default_rng(d)
    ns = list(range(0, 5000)) + [int(x) for x in rng.integers(0, 2**31, size=2000)] + [2**31 - 1]
    for n in ns:
        assert fastdiv(n, d) == n // d, (n, d)
