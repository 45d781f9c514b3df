"""The oracle pinned against qcu's own outputs (tests/golden/qcu_ref_golden.npz,
made by tests/golden/make_golden.py from qcu compiled from its sources)."""
import os

import numpy as np
import pytest

import oracle as O
from util import rel

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qcu_ref_golden.npz")


@pytest.fixture(scope="module")
def g():
    if not os.path.exists(PATH):
        pytest.fail(f"golden fixture missing: {PATH}")
    return np.load(PATH)


@pytest.mark.parametrize("tag", ["w4", "w8"])
@pytest.mark.parametrize("api", ["dslashQcu", "ncclDslashQcu"])
def test_oracle_dslash_matches_qcu(g, tag, api):
    latt = list(g[f"{tag}_latt"])
    U, psi = g[f"{tag}_U"], g[f"{tag}_psi"]
    for p in (0, 1):
        assert rel(O.dslash(psi[1 - p], U, latt, p), g[f"{tag}_{api}_p{p}"]) <= 1e-14


def _gj_growth(A):
    """max |A| / min |pivot| of the unpivoted Gauss-Jordan qcu runs per site
    (include/define.h:334-365): the factor by which it amplifies rounding."""
    worst = 1.0
    for M in A:
        M = M.copy()
        piv = []
        for i in range(12):
            piv.append(abs(M[i, i]))
            M[i] /= M[i, i]
            for j in range(12):
                if j != i:
                    M[j] -= M[j, i] * M[i]
        worst = max(worst, np.abs(A).max() / min(piv))
    return worst


@pytest.mark.parametrize("tag", ["c4s", "c4h"])
def test_oracle_clover_matches_qcu(g, tag):
    latt = list(g[f"{tag}_latt"])
    U, psi = g[f"{tag}_U"], g[f"{tag}_psi"]
    for p in (0, 1):
        A = O.clover_build(U, latt, p, 1.0)
        expect = O.clover_apply(O.clover_invert(A), O.dslash(psi[1 - p], U, latt, p))
        got = g[f"{tag}_dslashCloverQcu_p{p}"]
        # both sides run an unpivoted elimination; on hot links some sites have
        # tiny intermediate pivots, so the bound scales with the growth squared
        tol = 1e-15 * max(_gj_growth(A), 10.0) ** 2
        assert rel(expect, got) <= tol
        # and where the elimination is benign the agreement is at rounding level
        if tag == "c4s":
            assert rel(expect, got) <= 1e-11


def test_qcu_solver_output_solves_the_oracle_system(g):
    latt = list(g["s_latt"])
    U, b, x = g["s_U"], g["s_b"], g["s_x"]
    r = b - O.mfull(x, U, latt, 0.125)
    # qcu stops on the iterated ||r_o||^2 < 1e-9 and computes x_e from the
    # previous iterate (include/lattice_bistabcg.h:301-332)
    assert np.linalg.norm(r) ** 2 < 1e-7
    xo, it, _ = O.solve_full(b, U, latt, 0.125, tol=1e-12, maxiter=1000)
    assert rel(x, xo) < 1e-5
