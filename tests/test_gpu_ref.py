"""Direct parity with qcu itself on the GPU: qcu compiled from its own sources
(oracle/_ref/libqcu_ref.so) and this library, same seeded inputs, same calls.
Skipped when the reference build is absent."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from test_golden import _gj_growth
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libqcu_ref.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("qcu reference build not present (make -C oracle ref)")
    import qcu_b200

    lib = ctypes.CDLL(REF)
    P = ctypes.POINTER(qcu_b200.QcuParam)
    vp = ctypes.c_void_p
    lib.dslashQcu.argtypes = [vp, vp, vp, P, ctypes.c_int]
    lib.dslashCloverQcu.argtypes = [vp, vp, vp, P, ctypes.c_int]
    return lib


@pytest.mark.parametrize("latt", [[8, 8, 8, 8], [16, 8, 8, 16]])
def test_dslash_matches_qcu_kernel(ref, latt):
    import qcu_b200 as q

    U = O.gauge_haar(latt, 21)
    psi = O.fermion_gauss(O.full_shape(latt), 22)
    for p in (0, 1):
        a, b = empty_like_dev(O.half_shape(latt)), dev(np.zeros(O.half_shape(latt), complex))
        din, dU = dev(psi[1 - p]), dev(U)  # tensors stay alive across the raw-pointer call
        q.dslashQcu(a, din, dU, q.QcuParam(latt), p)
        ref.dslashQcu(b.data_ptr(), din.data_ptr(), dU.data_ptr(), ctypes.byref(q.QcuParam(latt)), p)
        assert rel(host(a), host(b)) <= 1e-13


def test_clover_matches_qcu_kernel(ref):
    import qcu_b200 as q

    latt = [8, 8, 8, 8]
    U = O.gauge_smooth(latt, 0.3, 23)
    psi = O.fermion_gauss(O.full_shape(latt), 24)
    for p in (0, 1):
        a, b = empty_like_dev(O.half_shape(latt)), dev(np.zeros(O.half_shape(latt), complex))
        din, dU = dev(psi[1 - p]), dev(U)
        q.dslashCloverQcu(a, din, dU, q.QcuParam(latt), p)
        ref.dslashCloverQcu(b.data_ptr(), din.data_ptr(), dU.data_ptr(), ctypes.byref(q.QcuParam(latt)), p)
        # qcu inverts with an unpivoted 12x12 Gauss-Jordan, this library with a
        # 6x6 LDL^H: both amplify rounding by the elimination growth
        growth = _gj_growth(O.clover_build(U, latt, p, 1.0))
        assert rel(host(a), host(b)) <= 1e-15 * max(growth, 10.0) ** 2
