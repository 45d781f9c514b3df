"""Independent numpy formulation of the Wilson/clover operator on the full
lexicographic lattice (explicit 4x4 gamma matrices, np.roll shifts).

Used only by the tests, to cross-check the C oracle's even-odd indexing,
spin projection and clover leaves against a second, structurally different
implementation.  Layout conversions follow PyQuda's cb2/lexico
(python/PyQuda/pyquda/field.py:22-63).
"""
import numpy as np

# DeGrand-Rossi gamma matrices (x, y, z, t), the basis hard-coded in qcu's
# spin projections (src/wilson_dslash.cu:56-243).
GAMMA = np.zeros((4, 4, 4), np.complex128)
GAMMA[0][0, 3] = 1j; GAMMA[0][1, 2] = 1j; GAMMA[0][2, 1] = -1j; GAMMA[0][3, 0] = -1j
GAMMA[1][0, 3] = -1; GAMMA[1][1, 2] = 1; GAMMA[1][2, 1] = 1; GAMMA[1][3, 0] = -1
GAMMA[2][0, 2] = 1j; GAMMA[2][1, 3] = -1j; GAMMA[2][2, 0] = -1j; GAMMA[2][3, 1] = 1j
GAMMA[3][0, 2] = 1; GAMMA[3][1, 3] = 1; GAMMA[3][2, 0] = 1; GAMMA[3][3, 1] = 1


def cb2_to_lexico(a, latt):
    """[2, Lt, Lz, Ly, Lxh, ...] -> [Lt, Lz, Ly, Lx, ...]"""
    Lx, Ly, Lz, Lt = latt
    out = np.zeros((Lt, Lz, Ly, Lx) + a.shape[5:], a.dtype)
    for t in range(Lt):
        for z in range(Lz):
            for y in range(Ly):
                eo = (t + z + y) % 2
                out[t, z, y, eo::2] = a[0, t, z, y]
                out[t, z, y, 1 - eo::2] = a[1, t, z, y]
    return out


def lexico_to_cb2(a, latt):
    Lx, Ly, Lz, Lt = latt
    out = np.zeros((2, Lt, Lz, Ly, Lx // 2) + a.shape[4:], a.dtype)
    for t in range(Lt):
        for z in range(Lz):
            for y in range(Ly):
                eo = (t + z + y) % 2
                out[0, t, z, y] = a[t, z, y, eo::2]
                out[1, t, z, y] = a[t, z, y, 1 - eo::2]
    return out


def gauge_lexico(gauge, latt):
    """[4, 2, Lt, Lz, Ly, Lxh, 3, 3] -> [4, Lt, Lz, Ly, Lx, 3, 3]"""
    return np.stack([cb2_to_lexico(gauge[mu], latt) for mu in range(4)])


_AXIS = {0: 3, 1: 2, 2: 1, 3: 0}  # direction -> array axis in [t, z, y, x]


def _shift(f, mu, step):
    """f(x + step*mu)"""
    return np.roll(f, -step, axis=_AXIS[mu])


def _tphase(latt, step, t_bc):
    """factor applied to hops crossing the t boundary"""
    Lt = latt[3]
    ph = np.ones(Lt)
    if step > 0:
        ph[Lt - 1] = t_bc
    else:
        ph[0] = t_bc
    return ph[:, None, None, None, None, None]


def dslash_lexico(psi, U, latt, t_bc=1.0):
    """D psi on the full lattice: psi [Lt,Lz,Ly,Lx,4,3], U [4,Lt,Lz,Ly,Lx,3,3]."""
    out = np.zeros_like(psi)
    one = np.eye(4)
    for mu in range(4):
        fwd = _shift(psi, mu, +1)
        proj = np.einsum("st,...tc->...sc", one - GAMMA[mu], fwd)
        h = np.einsum("...ab,...sb->...sa", U[mu], proj)
        if mu == 3:
            h = h * _tphase(latt, +1, t_bc)
        out += h
        Ub = _shift(U[mu], mu, -1)
        bwd = _shift(psi, mu, -1)
        proj = np.einsum("st,...tc->...sc", one + GAMMA[mu], bwd)
        h = np.einsum("...ba,...sb->...sa", Ub.conj(), proj)
        if mu == 3:
            h = h * _tphase(latt, -1, t_bc)
        out += h
    return out


def clover_lexico(U, latt, coeff=1.0):
    """A = 1 - coeff/8 sum_{mu<nu} g_mu g_nu (Q - Q^+) as [Lt,Lz,Ly,Lx,12,12]."""
    def dag(m):
        return np.swapaxes(m, -1, -2).conj()

    def mm(*ms):
        r = ms[0]
        for m in ms[1:]:
            r = np.einsum("...ab,...bc->...ac", r, m)
        return r

    shape = U.shape[1:5]
    A = np.zeros(shape + (4, 3, 4, 3), np.complex128)
    for mu in range(4):
        for nu in range(mu + 1, 4):
            S = lambda f, a, s: _shift(f, a, s)
            Umu, Unu = U[mu], U[nu]
            q = mm(Umu, S(Unu, mu, 1), dag(S(Umu, nu, 1)), dag(Unu))
            q = q + mm(Unu, dag(S(S(Umu, mu, -1), nu, 1)), dag(S(Unu, mu, -1)), S(Umu, mu, -1))
            q = q + mm(dag(S(Umu, mu, -1)), dag(S(S(Unu, mu, -1), nu, -1)), S(S(Umu, mu, -1), nu, -1),
                       S(Unu, nu, -1))
            q = q + mm(dag(S(Unu, nu, -1)), S(Umu, nu, -1), S(S(Unu, mu, 1), nu, -1), dag(Umu))
            F = q - dag(q)
            sig = GAMMA[mu] @ GAMMA[nu]
            A += np.einsum("st,...ab->...satb", sig, F)
    A *= -coeff / 8.0
    A = A.reshape(shape + (12, 12))
    A += np.eye(12)
    return A
