"""GPU checks of the batched solver (qcuInvertBatch): several right-hand
sides on lattices of different volume, with and without clover, solved
together; every solution is checked against the CPU oracle's full operator
(true residual recomputed on the host) and against single-rhs solves."""
import numpy as np
import pytest

import oracle as O
from util import dev, host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _system(q, latt, seed, kappa, nrhs, clover, eps=0.25):
    U = O.gauge_smooth(latt, eps, seed)
    c = kappa * 1.0 if clover else 0.0
    A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
    b = np.stack([O.fermion_gauss(O.full_shape(latt), seed * 100 + j) for j in range(nrhs)])
    G = q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=c)
    x = dev(np.full(b.shape, np.nan + 0j))
    return dict(latt=latt, U=U, A=A, b=b, G=G, x=x, db=dev(b), kappa=kappa, clover=clover)


def _check(sysd, xs, tol):
    for j in range(sysd["b"].shape[0]):
        b = sysd["b"][j]
        r = b - O.mfull(xs[j], sysd["U"], sysd["latt"], sysd["kappa"], -1.0, True, sysd["A"][0], sysd["A"][1])
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05 * tol


@pytest.mark.parametrize("prec,gprec", [(64, 0), (32, 0), (32, 16), (16, 0)])
def test_batch_uneven_lattices(q, prec, gprec):
    systems = [_system(q, [8, 8, 8, 8], 3, 0.124, 3, False),
               _system(q, [4, 4, 8, 8], 4, 0.125, 2, True),
               _system(q, [6, 4, 4, 8], 5, 0.12, 1, False)]
    try:
        res, tune = q.invert_batch([(s["G"], s["x"], s["db"], s["kappa"], s["clover"]) for s in systems],
                                   tol=1e-10, maxiter=4000, precision=prec, gauge_precision=gprec, inner_iters=16,
                                   inner_tol=0.1, gcr_k=6)
        assert len(res) == 6
        for r in res:
            assert r["status"] == 1, res
            assert r["true_residual"] <= 1e-10
        assert tune["dslash_threads"] in (64, 128, 256) and tune["blas_sites"] in (128, 256, 512)
        for s in systems:
            _check(s, host(s["x"]), 1e-10)
    finally:
        for s in systems:
            s["G"].close()


@pytest.mark.parametrize("prec,gprec", [(32, 16), (16, 0)])
def test_batch_matches_single_solves(q, prec, gprec):
    """Each rhs of a batch reaches the same solution as its own single solve."""
    s = _system(q, [8, 8, 8, 16], 7, 0.126, 4, True)
    try:
        res, _ = q.invert_batch([(s["G"], s["x"], s["db"], s["kappa"], True)], tol=1e-11, maxiter=4000,
                                precision=prec, gauge_precision=gprec, inner_iters=24, inner_tol=0.05, gcr_k=4)
        xb = host(s["x"])
        for j in range(4):
            xs = dev(np.zeros(O.full_shape(s["latt"]), complex))
            info = s["G"].invert(xs, s["db"][j].contiguous(), s["kappa"], tol=1e-11, maxiter=4000, precision=prec,
                                 gauge_precision=gprec, clover=True, solver="gcr", inner_iters=24, inner_tol=0.05,
                                 gcr_k=4)
            assert info["status"] == 1 and res[j]["status"] == 1
            d = np.linalg.norm(xb[j] - host(xs)) / np.linalg.norm(host(xs))
            assert d < 1e-8, (j, d)
            # the same method on the same data: the inner iteration counts agree closely
            assert abs(res[j]["iterations"] - info["iterations"]) <= 0.2 * info["iterations"] + 8
    finally:
        s["G"].close()


def test_batch_zero_and_repeated_sources(q):
    """A zero rhs gives x = 0 at once; identical rhs give identical solutions."""
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 9)
    b1 = O.fermion_gauss(O.full_shape(latt), 91)
    b = np.stack([b1, np.zeros_like(b1), b1])
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        x = dev(np.full(b.shape, np.nan + 0j))
        res, _ = q.invert_batch([(G, x, dev(b), 0.12, False)], tol=1e-10, maxiter=2000, precision=32,
                                gauge_precision=16, inner_iters=16, gcr_k=4)
    xs = host(x)
    assert res[1]["status"] == 1 and res[1]["iterations"] == 0
    assert np.all(xs[1] == 0)
    assert np.array_equal(xs[0], xs[2])
    assert res[0]["status"] == 1 and res[0]["true_residual"] <= 1e-10


def test_batch_maxiter(q):
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 12)
    b = np.stack([O.fermion_gauss(O.full_shape(latt), 120 + j) for j in range(2)])
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        x = dev(np.full(b.shape, np.nan + 0j))
        res, _ = q.invert_batch([(G, x, dev(b), 0.124, False)], tol=1e-14, maxiter=10, precision=32,
                                gauge_precision=0, inner_iters=4, gcr_k=2)
    for r in res:
        assert r["status"] == 2 and r["iterations"] >= 10
    assert np.isfinite(host(x)).all()


def test_batch_rejects_bad_input(q):
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 13)
    b = dev(np.zeros((1,) + O.full_shape(latt), complex))
    with q.Gauge(dev(U), latt) as G:
        with pytest.raises(q.QcuError):
            q.invert_batch([(G, b.clone(), b, 0.12, True)])  # no clover loaded
        with pytest.raises(q.QcuError):
            q.invert_batch([(G, b.clone(), b, 0.12, False)], precision=16, gauge_precision=16)
        bb = dev(np.zeros((65,) + O.full_shape(latt), complex))
        with pytest.raises(q.QcuError):
            q.invert_batch([(G, bb.clone(), bb, 0.12, False)])  # more than 64 rhs


def test_invert12_point_propagator(q):
    """The 12 point-source solves of a propagator in one batch, against the
    CPU oracle's full-system solve of each source."""
    latt = [4, 4, 4, 8]
    kappa = 0.124
    U = O.gauge_smooth(latt, 0.25, 14)
    origin = [1, 2, 3, 5]
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        prop, res, _ = q.invert12(G, kappa, origin, tol=1e-11, maxiter=4000, precision=32, gauge_precision=16,
                                  inner_iters=16, gcr_k=4)
    P = host(prop)  # [2, Lt, Lz, Ly, Lxh, s_sink, s_src, c_sink, c_src]
    assert P.shape == (2, 8, 4, 4, 2, 4, 4, 3, 3)
    x, y, z, t = origin
    for s in range(4):
        for c in range(3):
            b = np.zeros(O.full_shape(latt), complex)
            b[(x + y + z + t) % 2, t, z, y, x // 2, s, c] = 1.0
            xo, _, _ = O.solve_full(b, U, latt, kappa, t_bc=-1.0, tol=1e-13, maxiter=4000)
            got = P[..., :, s, :, c]
            assert np.linalg.norm(got - xo) / np.linalg.norm(xo) < 1e-8
    assert all(r["status"] == 1 for r in res)


@pytest.mark.parametrize("tune", ["64,1,128,0", "128,1,256,0", "256,1,512,0", "64,2,256,0", "128,2,128,0",
                                  "64,4,256,0", "128,4,512,0", "32,8,256,1", "32,8,128,2"])
def test_batch_every_dslash_shape(q, tune, monkeypatch):
    """Every block shape the autotuner can pick (sites per tile, rhs per
    group, BLAS tile, tensor-core path) gives a converged, correct batch:
    two lattices, a clover system, groups with partly filled slots."""
    monkeypatch.setenv("QCU_BATCH_TUNE", tune)
    systems = [_system(q, [8, 8, 8, 8], 21, 0.124, 5, False),
               _system(q, [4, 4, 8, 8], 22, 0.125, 3, True)]
    try:
        res, got = q.invert_batch([(s["G"], s["x"], s["db"], s["kappa"], s["clover"]) for s in systems],
                                  tol=1e-10, maxiter=4000, precision=32, gauge_precision=16, inner_iters=16,
                                  inner_tol=0.1, gcr_k=4)
        th, nr, bs, mma = [int(v) for v in tune.split(",")]
        assert (got["dslash_threads"], got["dslash_rhs"], got["blas_sites"], got["mma"]) == (th, nr, bs, mma)
        for r in res:
            assert r["status"] == 1 and r["true_residual"] <= 1e-10, res
        for s in systems:
            _check(s, host(s["x"]), 1e-10)
    finally:
        for s in systems:
            s["G"].close()
