"""CPU checks of the learned-preconditioner oracle (oracle/nn_ref.py): the
analytic gradient against finite differences, gauge equivariance, and the
identity start."""
import numpy as np

import oracle as O
from oracle import nn_ref as R


def _setup(latt=(4, 2, 2, 4), seed=3, t_bc=-1.0):
    U = O.gauge_haar(list(latt), seed)
    lat = R.Lattice(U, list(latt), t_bc)
    rng = np.random.default_rng(seed)
    w = rng.normal(0, 0.3, R.N_W1 * 2 + R.N_W2 * 2)
    r = O.fermion_gauss((2, lat.Vh, 4, 3), seed + 1)
    e = O.fermion_gauss((2, lat.Vh, 4, 3), seed + 2)
    return lat, w, r, e


def test_gradient_matches_finite_differences():
    lat, w, r, e = _setup()
    g, L = R.gradient(lat, w, r, e)
    assert abs(L - R.loss(lat, w, r, e)) < 1e-12
    rng = np.random.default_rng(0)
    eps = 1e-6
    for k in rng.choice(w.size, 24, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[k] += eps
        wm[k] -= eps
        fd = (R.loss(lat, wp, r, e) - R.loss(lat, wm, r, e)) / (2 * eps)
        # real-parameter derivative = 2 x conjugate Wirtinger derivative
        assert abs(fd - 2 * g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, 2 * g[k])


def test_gauge_equivariance():
    latt = [4, 2, 2, 4]
    lat, w, r, _ = _setup(tuple(latt))
    U = lat.U.reshape(4, 2, lat.Vh, 3, 3)
    gtr = O.gauge_haar(latt, 99).reshape(4, 2, lat.Vh, 3, 3)[0]  # one SU(3) per site: [2, Vh, 3, 3]
    Ug = np.empty_like(U)
    for mu in range(4):
        for p in (0, 1):
            n = lat.fwd[mu, p]
            Ug[mu, p] = np.einsum("sij,sjk,slk->sil", gtr[p], U[mu, p], gtr[1 - p][n].conj())
    latg = R.Lattice(Ug.reshape(4, 2, *([1] * 0), lat.Vh, 3, 3), latt, -1.0)
    rg = np.einsum("sij,bscj->bsci", gtr[1], r)
    o, _, _ = R.forward(lat, w, r)
    og, _, _ = R.forward(latg, w, rg)
    assert np.abs(og - np.einsum("sij,bscj->bsci", gtr[1], o)).max() < 1e-10


def test_identity_start_is_identity():
    lat, _, r, _ = _setup()
    w1 = np.zeros((R.HOPS, R.C_HID, R.C_IN), complex)
    w2 = np.zeros((R.HOPS, R.C_OUT, R.C_HID), complex)
    for a in range(4):
        w1[0, a, a] = 1
        w2[0, a, a] = 1
    o, _, _ = R.forward(lat, R.join_weights(w1, w2), r)
    assert np.abs(o - r).max() < 1e-14
