"""Division by invariant integers as the hopping kernels use it for site
coordinates (fields.cuh: geom_div; runtime.cpp: make_geom).

For a divisor d >= 2 the host stores m = ceil(2^32 / d) when (Vh + 64) d < 2^32,
and the kernels take n / d = umulhi(n, m) = (n m) >> 32 for every site index
n < Vh + 64 (padding included).  The bound makes it exact: with m d = 2^32 + e,
0 <= e < d, the error term n e / (d 2^32) stays below 1/d.  Here the formula
is checked exhaustively against integer division for every divisor a lattice
extent can take (Lx/2, Ly, Lz up to 256) and every index the bound admits,
capped at 2^22 indices per divisor, plus the largest indices near the bound."""
import numpy as np
import pytest


def magic(vh, d):
    """The host's multiplier (0: the kernels divide normally)."""
    if d < 2 or (vh + 64) * d >= 1 << 32:
        return 0
    return ((1 << 32) + d - 1) // d


def umulhi(n, m):
    return (n.astype(np.uint64) * np.uint64(m)) >> np.uint64(32)


@pytest.mark.parametrize("d", list(range(2, 257)))
def test_umulhi_division_exact_for_admitted_indices(d):
    vh = min((1 << 32) // d - 65, (1 << 22) - 64)  # the largest Vh the bound admits, capped
    m = magic(vh, d)
    assert m != 0
    n = np.arange(vh + 64, dtype=np.uint64)
    assert np.array_equal(umulhi(n, m), n // np.uint64(d))


@pytest.mark.parametrize("d", [3, 7, 16, 48, 100, 255, 256, 1000, 4096])
def test_umulhi_division_exact_near_the_bound(d):
    vh = (1 << 32) // d - 65  # (vh + 64) d < 2^32 holds, barely
    m = magic(vh, d)
    assert m != 0
    n = np.arange(max(0, vh + 64 - (1 << 20)), vh + 64, dtype=np.uint64)
    assert np.array_equal(umulhi(n, m), n // np.uint64(d))


def test_multiplier_refused_past_the_bound():
    assert magic((1 << 32) // 3, 3) == 0
    assert magic(1000, 1) == 0
