"""Two-level multigrid (qcuMG) on the GPU, checked against the CPU oracle.

Set-up: P^dag P = 1 on every aggregate and chirality, and the coarse
operator equal to P^dag M P (both to FP32 rounding, bar 1e-5).  Solve: the
FP64 true residual ||b - M x|| / ||b|| of the returned x, recomputed by the
oracle's full operator on the host, at most 1e-10 (tol 1e-10 requested),
for Wilson and clover, periodic and antiperiodic time boundaries and
aggregates that wrap onto themselves (one aggregate across a direction)."""
import numpy as np
import pytest

import oracle as O
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _true_residual(x, b, U, latt, kappa, t_bc, A=(None, None)):
    return rel(O.mfull(x, U, latt, kappa, t_bc, True, A[0], A[1]), b)


@pytest.mark.parametrize("latt,block", [([8, 8, 8, 8], [4, 4, 4, 4]), ([8, 4, 4, 12], [4, 4, 2, 4]),
                                        ([4, 4, 8, 8], [4, 2, 4, 4])])
@pytest.mark.parametrize("clover", [False, True])
def test_mg_setup_orthonormal_and_galerkin(q, latt, block, clover):
    U = O.gauge_smooth(latt, 0.3, 11)
    kappa = 0.12
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=kappa if clover else 0.0) as G:
        mg = q.Multigrid(G, kappa, geo_block_size=block, n_vec=6, setup_maxiter=20)
        orth, gal = mg.check()
        mg.close()
    assert orth <= 1e-5, orth
    assert gal <= 1e-5, gal


@pytest.mark.parametrize("clover,t_bc", [(False, -1.0), (False, 1.0), (True, -1.0)])
def test_mg_solve_matches_oracle_operator(q, clover, t_bc):
    latt = [8, 8, 8, 16]
    U = O.gauge_smooth(latt, 0.3, 5)
    b = O.fermion_gauss(O.full_shape(latt), 105)
    kappa = 0.124
    c = kappa if clover else 0.0
    A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
    with q.Gauge(dev(U), latt, t_boundary=t_bc, clover_coeff=c) as G:
        mg = q.Multigrid(G, kappa, geo_block_size=[4, 4, 4, 4], n_vec=8, setup_maxiter=32)
        x = empty_like_dev(O.full_shape(latt))
        info = mg.invert(x, dev(b), tol=1e-10, maxiter=300)
        mg.close()
    assert info["status"] == 1, info
    res = _true_residual(host(x), b, U, latt, kappa, t_bc, A)
    assert res <= 1e-10, (res, info)
    assert abs(res - info["true_residual"]) <= 1e-11 + 0.05 * res, (res, info)
    assert info["coarse_iters"] > 0


def test_mg_coarse_correction_reduces_outer_steps(q):
    """The coarse space does the work: with the same smoother, the two-level
    cycle needs fewer outer steps than the cycle with the coarse solve capped at one iteration."""
    latt = [8, 8, 8, 8]
    U = O.gauge_smooth(latt, 0.3, 9)
    b = O.fermion_gauss(O.full_shape(latt), 109)
    kappa = 0.124
    steps = {}
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        for cm in (1, 50):
            mg = q.Multigrid(G, kappa, n_vec=8, setup_maxiter=32, coarse_maxiter=cm, coarse_tol=0.05, nu_post=4)
            x = empty_like_dev(O.full_shape(latt))
            info = mg.invert(x, dev(b), tol=1e-8, maxiter=400)
            mg.close()
            assert info["status"] == 1, info
            steps[cm] = info["outer"]
    assert steps[50] < steps[1], steps


def test_mg_zero_source_and_bad_parameters(q):
    latt = [8, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.3, 3)
    with q.Gauge(dev(U), latt) as G:
        mg = q.Multigrid(G, 0.12, geo_block_size=[4, 4, 4, 4], n_vec=4, setup_maxiter=8)
        import torch

        x = empty_like_dev(O.full_shape(latt))
        info = mg.invert(x, torch.zeros(O.full_shape(latt), dtype=torch.complex128, device="cuda"))
        assert info["status"] == 1 and info["outer"] == 0
        assert np.count_nonzero(host(x)) == 0
        mg.close()
        for bad in ({"geo_block_size": [3, 4, 4, 4]}, {"geo_block_size": [4, 4, 4, 3]},
                    {"geo_block_size": [2, 2, 2, 2]}, {"n_vec": 17}, {"gcr_k": 0}):
            with pytest.raises(q.QcuError):
                q.Multigrid(G, 0.12, **bad)


@pytest.mark.parametrize("clover", [False, True])
def test_gcr_with_coarse_grid_correction(q, clover):
    """solve()'s precond 3: the coarse-grid correction of the multigrid, then
    the inner 16-bit BiCGSTAB, inside the FP64 flexible GCR on M_pc."""
    latt = [8, 8, 8, 16]
    U = O.gauge_smooth(latt, 0.3, 21)
    b = O.fermion_gauss(O.full_shape(latt), 121)
    kappa = 0.124
    c = kappa if clover else 0.0
    A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=c) as G:
        mg = q.Multigrid(G, kappa, n_vec=8, setup_maxiter=32, coarse_tol=0.05, coarse_maxiter=50)
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(b), kappa, tol=1e-10, maxiter=20000, precision=16, solver="gcr", inner_iters=32,
                        inner_tol=0.1, gcr_k=4, clover=clover, precond=3, mg=mg)
        assert info["status"] == 1 and not info["fallback"], info
        assert _true_residual(host(x), b, U, latt, kappa, -1.0, A) <= 1e-10
        # the multigrid belongs to this handle and kappa: anything else is refused
        with pytest.raises(q.QcuError):
            G.invert(x, dev(b), kappa * 0.99, tol=1e-10, solver="gcr", clover=clover, precond=3, mg=mg)
        with pytest.raises(q.QcuError):
            G.invert(x, dev(b), kappa, tol=1e-10, solver="gcr", clover=clover, precond=3)
        mg.close()
