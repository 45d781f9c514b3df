"""CPU tests of the oracle itself (no GPU): the C restatement of qcu's path is
checked against an independent numpy formulation (explicit gamma matrices on
the lexicographic lattice, tests/npref.py), against algebraic identities the
reference's operator must satisfy, and against the golden vectors produced by
qcu's own library (tests/golden/, see tests/golden/make_golden.py)."""
import numpy as np
import pytest

import npref
import oracle as O
from util import rel

LATTS = [[4, 4, 4, 4], [4, 2, 6, 8], [2, 4, 4, 6], [6, 4, 2, 10]]


@pytest.mark.parametrize("latt", LATTS)
@pytest.mark.parametrize("t_bc", [1.0, -1.0])
def test_dslash_matches_lexicographic_numpy(latt, t_bc):
    U = O.gauge_haar(latt, 7)
    psi = O.fermion_gauss(O.full_shape(latt), 3)
    D = npref.dslash_lexico(npref.cb2_to_lexico(psi, latt), npref.gauge_lexico(U, latt), latt, t_bc)
    Dcb = npref.lexico_to_cb2(D, latt)
    for p in (0, 1):
        assert rel(O.dslash(psi[1 - p], U, latt, p, t_bc), Dcb[p]) < 1e-14


def test_recon12_is_exact_on_su3_and_differs_on_sign_flipped_links():
    latt = [4, 4, 4, 4]
    U = O.gauge_smooth(latt, 0.25, 1)
    psi = O.fermion_gauss(O.half_shape(latt), 2)
    assert rel(O.dslash(psi, U, latt, 0, 1.0, True), O.dslash(psi, U, latt, 0, 1.0, False)) < 1e-14
    # PyQuda's antiperiodic trick flips the sign of t links at Lt-1 (field.py:160-164);
    # reconstruct-12 cannot represent it, the in-kernel phase can.
    Uf = U.copy()
    Uf[3, :, -1] *= -1
    full18 = O.dslash(psi, Uf, latt, 0, 1.0, False)
    assert rel(O.dslash(psi, U, latt, 0, -1.0, True), full18) < 1e-14
    assert rel(O.dslash(psi, Uf, latt, 0, 1.0, True), full18) > 1e-3


def test_generators():
    latt = [4, 4, 4, 4]
    for U in (O.gauge_haar(latt, 5), O.gauge_smooth(latt, 0.25, 5)):
        m = U.reshape(-1, 3, 3)
        assert np.abs(np.einsum("nab,ncb->nac", m, m.conj()) - np.eye(3)).max() < 1e-14
        assert np.abs(np.linalg.det(m) - 1).max() < 1e-14
    # smooth links are close to 1, Haar links are not
    assert np.abs(O.gauge_smooth(latt, 0.25, 5).reshape(-1, 3, 3) - np.eye(3)).mean() < 0.2
    assert np.abs(O.gauge_haar(latt, 5).reshape(-1, 3, 3) - np.eye(3)).mean() > 0.4
    z = O.fermion_gauss((200000,), 9)
    assert abs(z.real.mean()) < 0.01 and abs(z.real.std() - 1) < 0.01 and abs(z.imag.std() - 1) < 0.01
    u = O.fermion_uniform((100000,), 9)
    assert u.real.min() > 0 and u.real.max() <= 1 and abs(u.imag.mean() - 0.5) < 0.01
    # counter-based: a prefix of a longer stream is the shorter stream
    assert np.array_equal(O.fermion_gauss((1000,), 4), O.fermion_gauss((2000,), 4)[:1000])
    assert O.rng_u64(1, 0) != O.rng_u64(2, 0)


def test_su3_exponential_matches_scipy():
    from scipy.linalg import expm

    h8 = np.array([0.3, -1.2, 0.5, 0.9, -0.4, 1.1, 0.2, -0.7])
    lam = np.zeros((8, 3, 3), complex)
    lam[0][0, 1] = lam[0][1, 0] = 1
    lam[1][0, 1], lam[1][1, 0] = -1j, 1j
    lam[2][0, 0], lam[2][1, 1] = 1, -1
    lam[3][0, 2] = lam[3][2, 0] = 1
    lam[4][0, 2], lam[4][2, 0] = -1j, 1j
    lam[5][1, 2] = lam[5][2, 1] = 1
    lam[6][1, 2], lam[6][2, 1] = -1j, 1j
    lam[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    H = np.einsum("a,aij->ij", h8, lam) / 2
    assert np.abs(O.su3_from_coeffs(h8, 0.25) - expm(1j * 0.25 * H)).max() < 1e-13


def test_gamma5_hermiticity():
    """gamma5 D is Hermitian for the Wilson hopping term: <a, g5 D b> = <g5 D a, b>."""
    latt = [4, 4, 4, 4]
    U = O.gauge_haar(latt, 11)
    g5 = np.diag([1, 1, -1, -1]).astype(complex)
    a = O.fermion_gauss(O.full_shape(latt), 1)
    b = O.fermion_gauss(O.full_shape(latt), 2)

    def g5D(psi):
        out = np.empty_like(psi)
        for p in (0, 1):
            out[p] = np.einsum("st,...tc->...sc", g5, O.dslash(psi[1 - p], U, latt, p))
        return out

    lhs = np.vdot(a, g5D(b))
    rhs = np.vdot(g5D(a), b)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
    # gamma5 = gamma1 gamma2 gamma3 gamma4 in this basis
    G = [O.gamma(m) for m in range(4)]
    assert np.allclose(G[0] @ G[1] @ G[2] @ G[3], g5)
    for m in range(4):
        assert np.allclose(G[m] @ G[m], np.eye(4)) and np.allclose(G[m], G[m].conj().T)


@pytest.mark.parametrize("latt", [[4, 4, 4, 4], [4, 2, 2, 6]])
def test_clover_matches_lexicographic_numpy(latt):
    U = O.gauge_haar(latt, 3)
    A = npref.lexico_to_cb2(npref.clover_lexico(npref.gauge_lexico(U, latt), latt, 1.0), latt)
    for p in (0, 1):
        Ao = O.clover_build(U, latt, p, 1.0)
        assert rel(Ao, A[p].reshape(-1, 12, 12)) < 1e-14
        # Hermitian, block diagonal in the chiral basis (spins {0,1} x {2,3})
        assert np.abs(Ao - np.swapaxes(Ao, 1, 2).conj()).max() < 1e-14
        assert np.abs(Ao[:, :6, 6:]).max() == 0 and np.abs(Ao[:, 6:, :6]).max() == 0


def test_clover_inverse_and_coefficient():
    latt = [4, 4, 4, 4]
    U = O.gauge_smooth(latt, 0.3, 2)
    A1 = O.clover_build(U, latt, 0, 1.0)
    A2 = O.clover_build(U, latt, 0, 0.5)
    # linear in the coefficient: A(c) - 1 = c (A(1) - 1)
    assert rel(A2 - np.eye(12), 0.5 * (A1 - np.eye(12))) < 1e-14
    Ai = O.clover_invert(A1)
    assert np.abs(np.einsum("nab,nbc->nac", Ai, A1) - np.eye(12)).max() < 1e-12
    # the clover term vanishes on a unit gauge
    Uu = np.zeros_like(U)
    Uu[...] = np.eye(3)
    assert np.abs(O.clover_build(Uu, latt, 1, 1.0) - np.eye(12)).max() == 0


def test_mpc_is_the_schur_complement():
    """M_pc x_o = b'_o  <=>  the full M x = b with x_e = b_e + kappa D_eo x_o."""
    latt = [4, 4, 4, 6]
    U = O.gauge_smooth(latt, 0.25, 4)
    kappa = 0.12
    x = O.fermion_gauss(O.full_shape(latt), 5)
    b = O.mfull(x, U, latt, kappa)
    bp = b[1] + kappa * O.dslash(b[0], U, latt, 1)
    assert rel(O.mpc(x[1], U, latt, kappa), bp) < 1e-13
    xe = b[0] + kappa * O.dslash(x[1], U, latt, 0)
    assert rel(xe, x[0]) < 1e-13


@pytest.mark.parametrize("clover", [False, True])
def test_solver_converges_to_true_residual(clover):
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 8)
    kappa = 0.12
    b = O.fermion_gauss(O.full_shape(latt), 6)
    kw = {}
    Afull = {}
    if clover:
        c = kappa * 1.0
        for p in (0, 1):
            Afull[p] = O.clover_build(U, latt, p, c)
        kw = dict(Ainv_e=O.clover_invert(Afull[0]), Ainv_o=O.clover_invert(Afull[1]))
    x, it, _ = O.solve_full(b, U, latt, kappa, tol=1e-10, maxiter=500, **kw)
    r = b - O.mfull(x, U, latt, kappa, A_e=Afull.get(0), A_o=Afull.get(1))
    assert 0 < it < 500
    assert np.linalg.norm(r) / np.linalg.norm(b) < 3e-10


def test_solver_qcu_legacy_mode():
    """qcu's ncclBistabCgQcu criterion: kappa 0.125, random start, ||r||^2 < 1e-9."""
    latt = [4, 4, 4, 4]
    U = O.gauge_haar(latt, 1)
    b = np.ones(O.full_shape(latt), complex)
    x0 = np.zeros_like(b)
    x0[1] = O.fermion_uniform(O.half_shape(latt), 23333)
    x, it, res2 = O.solve_full(b, U, latt, 0.125, x0=x0, tol=1e-9, abs_tol=True, maxiter=1000)
    assert res2 < 1e-9 and it < 1000
    r = b - O.mfull(x, U, latt, 0.125)
    assert np.linalg.norm(r) ** 2 < 1e-8
