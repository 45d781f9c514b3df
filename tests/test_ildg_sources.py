"""Gauge I/O (ILDG/LIME) and the source constructors, on CPU."""
import os

import numpy as np
import pytest

import oracle as O

# PyQuda's own test configuration (python/PyQuda/tests/weak_field.lime), copied
# beside the other fixtures by tests/golden/make_golden.py
WEAK = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "weak_field.lime")


def _su3_error(U):
    M = np.asarray(U).reshape(-1, 3, 3)
    return max(np.abs(np.einsum("sij,skj->sik", M, M.conj()) - np.eye(3)).max(),
               np.abs(np.linalg.det(M) - 1).max())


@pytest.mark.parametrize("prec", [64, 32])
def test_ildg_round_trip(tmp_path, prec):
    from qcu_b200 import ildg

    latt = [4, 2, 2, 6]
    U = O.gauge_haar(latt, 5)
    f = tmp_path / "u.lime"
    ildg.write_ildg(str(f), U, latt, precision=prec)
    V, latt2, info = ildg.read_ildg(str(f))
    assert latt2 == latt and info["checksum"] == "ok" and info["precision"] == prec
    if prec == 64:
        assert np.array_equal(V, U)
    else:
        assert np.abs(V - U).max() < 1e-7
    # the records are well-formed LIME
    recs = ildg.read_lime(str(f))
    assert [r[0] for r in recs] == ["ildg-format", "ildg-binary-data", "scidac-checksum"]
    assert recs[0][2] & 0x8000 and recs[-1][2] & 0x4000


def test_ildg_lexicographic_order():
    """binary data is [t][z][y][x][mu][3][3]: site (x,y,z,t) lands at parity
    (x+y+z+t)%2, half index x/2 (python/PyQuda/pyquda/field.py cb2)."""
    from qcu_b200 import ildg

    latt = [4, 2, 2, 2]
    Lx, Ly, Lz, Lt = latt
    lex = np.zeros((Lt, Lz, Ly, Lx, 4, 3, 3), complex)
    for t in range(Lt):
        for z in range(Lz):
            for y in range(Ly):
                for x in range(Lx):
                    lex[t, z, y, x, :, 0, 0] = 1000 * t + 100 * z + 10 * y + x
    eo = ildg.lexico_to_eo(lex, latt)
    for t in range(Lt):
        for z in range(Lz):
            for y in range(Ly):
                for x in range(Lx):
                    p = (x + y + z + t) % 2
                    assert eo[2, p, t, z, y, x // 2, 0, 0] == 1000 * t + 100 * z + 10 * y + x
    assert np.array_equal(ildg.eo_to_lexico(eo, latt), lex)


def test_ildg_rejects_corruption(tmp_path):
    from qcu_b200 import ildg

    latt = [2, 2, 2, 2]
    f = tmp_path / "u.lime"
    ildg.write_ildg(str(f), O.gauge_haar(latt, 6), latt)
    raw = bytearray(f.read_bytes())
    raw[600] ^= 0x01  # one bit inside the binary record
    f.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        ildg.read_ildg(str(f))
    with pytest.raises(ValueError, match="LIME"):
        g = tmp_path / "junk.lime"
        g.write_bytes(b"\0" * 200)
        ildg.read_ildg(str(g))


@pytest.mark.skipif(not os.path.exists(WEAK), reason="PyQuda's weak_field.lime test configuration not present")
def test_reads_pyquda_weak_field():
    """PyQuda's own test configuration (python/PyQuda/tests/weak_field.lime):
    the file's SciDAC checksum holds, the links are SU(3), and the hopping
    term of the oracle on it is gamma5-hermitian."""
    from qcu_b200 import ildg

    U, latt, info = ildg.read_ildg(WEAK)
    assert latt == [4, 4, 4, 8] and info["checksum"] == "ok" and info["field"] == "su3gauge"
    assert _su3_error(U) < 1e-13
    psi = O.fermion_gauss(O.full_shape(latt), 3)
    chi = O.fermion_gauss(O.full_shape(latt), 4)
    g5 = np.diag([1, 1, -1, -1]).astype(complex)
    D = lambda v: np.stack([O.dslash(v[1], U, latt, 0), O.dslash(v[0], U, latt, 1)])  # noqa: E731
    lhs = np.vdot(chi, np.einsum("ab,...bc->...ac", g5, D(psi)))
    rhs = np.vdot(np.einsum("ab,...bc->...ac", g5, D(chi)), psi)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_sources():
    import torch

    import qcu_b200 as q

    latt = [4, 4, 2, 6]
    b = q.point_sources(latt, [3, 1, 0, 4], device="cpu")
    assert b.shape == (12, 2, 6, 2, 4, 2, 4, 3)
    assert float(b.abs().sum()) == 12.0
    assert b[1 * 3 + 2, (3 + 1 + 0 + 4) % 2, 4, 0, 1, 1, 1, 2] == 1
    w = q.wall_source(latt, 2, 3, 1, device="cpu")
    assert float(w.abs().sum()) == latt[0] * latt[1] * latt[2]
    assert torch.all(w[:, 2, ..., 3, 1] == 1)
    ph = q.momentum_phase(latt, [1, 0, 0], device="cpu")
    # x-momentum 1: phase exp(2 pi i x / Lx) at the site's full x coordinate
    for p in (0, 1):
        for xh in range(2):
            x = 2 * xh + ((5 + 1 + 1 + p) % 2)  # t=5, z=1, y=1
            assert abs(complex(ph[p, 5, 1, 1, xh]) - np.exp(2j * np.pi * x / 4)) < 1e-12
    m = q.momentum_source(latt, 5, ph, 0, 0, device="cpu")
    assert torch.allclose(m[:, 5, ..., 0, 0], ph[:, 5])
