"""Drop-in check through qcu's own Python binding: PyQuda's pyquda.pyqcu and
pyquda.pointer Cython modules (python/PyQuda/pyquda/src/pyqcu.pyx,
pointer.pyx), built unchanged from the reference sources against this
repository's include/qcu.h and libqcu.so by oracle/pyqcu_build.py, drive the
hot path exactly as PyQuda's qcu tests do (test/test.nccl.dslash.qcu-np1.py:
Pointer objects from ndarrayDataPointer, QcuParam.lattice_size, the output
parity).  Skipped when that build is absent."""
import os
import sys

import numpy as np
import pytest

import oracle as O
from test_golden import _gj_growth
from util import dev, host, rel

pytestmark = pytest.mark.gpu
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.fixture(scope="module")
def pyqcu():
    if not os.path.isdir(os.path.join(REF, "pyquda")):
        pytest.skip("PyQuda's qcu binding not built (python oracle/pyqcu_build.py)")
    sys.path.insert(0, REF)
    try:
        from pyquda import pointer, pyqcu
    finally:
        sys.path.remove(REF)
    import qcu_b200  # noqa: F401  (libqcu.so built and loadable)

    return pyqcu, pointer


def _param(pyqcu, latt):
    p = pyqcu.QcuParam()
    p.lattice_size = list(latt)
    return p


@pytest.mark.parametrize("latt", [[4, 4, 4, 8], [8, 8, 8, 8]])
def test_dslash_through_pyqcu(pyqcu, latt):
    mod, ptr = pyqcu
    U = O.gauge_haar(latt, 31)
    psi = O.fermion_gauss(O.full_shape(latt), 32)
    dU = dev(U)
    for p in (0, 1):
        din = dev(psi[1 - p])
        out = dev(np.zeros(O.half_shape(latt), complex))
        mod.dslashQcu(ptr.ndarrayDataPointer(out.reshape(-1), True), ptr.ndarrayDataPointer(din.reshape(-1), True),
                      ptr.ndarrayDataPointer(dU.reshape(-1), True), _param(mod, latt), p)
        ref = O.dslash(psi[1 - p], U, latt, p, 1.0)
        assert rel(host(out), ref) <= 1e-13
        # ncclDslashQcu with the one-GPU grid: same result
        out2 = dev(np.zeros(O.half_shape(latt), complex))
        mod.ncclDslashQcu(ptr.ndarrayDataPointer(out2.reshape(-1), True),
                          ptr.ndarrayDataPointer(din.reshape(-1), True), ptr.ndarrayDataPointer(dU.reshape(-1), True),
                          _param(mod, latt), p, _param(mod, [1, 1, 1, 1]))
        assert np.array_equal(host(out2), host(out))
    assert np.array_equal(host(dU), U)  # the binding's caller keeps its gauge untouched


def test_clover_dslash_through_pyqcu(pyqcu):
    mod, ptr = pyqcu
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.3, 33)
    psi = O.fermion_gauss(O.full_shape(latt), 34)
    dU = dev(U)
    for p in (0, 1):
        din = dev(psi[1 - p])
        out = dev(np.zeros(O.half_shape(latt), complex))
        mod.dslashCloverQcu(ptr.ndarrayDataPointer(out.reshape(-1), True),
                            ptr.ndarrayDataPointer(din.reshape(-1), True), ptr.ndarrayDataPointer(dU.reshape(-1), True),
                            _param(mod, latt), p)
        A = O.clover_build(U, latt, p, 1.0)
        ref = O.clover_apply(O.clover_invert(A), O.dslash(psi[1 - p], U, latt, p, 1.0))
        # the oracle inverts with qcu's unpivoted Gauss-Jordan, this library with LDL^H:
        # both amplify rounding by the elimination growth
        assert rel(host(out), ref) <= 1e-15 * max(_gj_growth(A), 10.0) ** 2


def test_bistabcg_through_pyqcu(pyqcu):
    """ncclBistabCgQcu through the binding: qcu's contract (kappa 0.125,
    absolute ||r||^2 < 1e-9); the solution satisfies the oracle's system."""
    mod, ptr = pyqcu
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 35)
    b = O.fermion_gauss(O.full_shape(latt), 36)
    dU, db = dev(U), dev(b)
    x = dev(np.zeros(O.full_shape(latt), complex))
    mod.ncclBistabCgQcu(ptr.ndarrayDataPointer(x.reshape(-1), True), ptr.ndarrayDataPointer(db.reshape(-1), True),
                        ptr.ndarrayDataPointer(dU.reshape(-1), True), _param(mod, latt), _param(mod, [1, 1, 1, 1]))
    xs = host(x)
    r = b - O.mfull(xs, U, latt, 0.125, 1.0)
    # qcu's criterion: ||r_o||^2 < 1e-9, absolute (include/define.h:68, lattice_bistabcg.h:301); x_e is
    # rebuilt exactly from x_o, so the even residual vanishes and the full residual obeys the same bound
    assert np.linalg.norm(r) ** 2 < 1e-9
    assert np.linalg.norm(r[0]) ** 2 < 1e-20
