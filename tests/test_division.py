"""The exact division by a lattice extent the kernels use: n / d as the high
64 bits of n * m with m = ceil(2^64 / d) (div_magic / div_by in
csrc/lattice.cuh), checked here in exact integer arithmetic for every
32-bit numerator class the kernels meet (no GPU)."""
import numpy as np
import pytest


def div_magic(d):
    return (2 ** 64 - 1) // d + 1  # wraps to 2^64 for d = 1: the device treats that case apart


@pytest.mark.parametrize("d", [2, 3, 4, 6, 7, 12, 64, 96, 192, 255, 256, 257, 1000, 4096, 73728, 147456,
                               2 ** 20 + 3, 2 ** 31 - 1, 2 ** 32 - 5])
def test_multiply_high_division_is_exact(d):
    m = div_magic(d)
    rng = np.random.default_rng(d)
    ns = [0, 1, d - 1, d, d + 1, 2 ** 32 - 1, 2 ** 31 - 1] + [int(v) for v in rng.integers(0, 2 ** 32, 2000)]
    ns += [k * d + r for k in (1, 7, 1000) for r in (0, d - 1) if k * d + r < 2 ** 32]
    for n in ns:
        assert (n * m) >> 64 == n // d, (n, d)
