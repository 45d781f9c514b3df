"""The domain-decomposed hopping term on the GPU.  One GPU per run here, so
all ranks of a grid run in one process (qcuDslashDDEmulate): the pack and
dslash kernels of every rank, the faces exchanged by device copies in each
rank's own schedule -- the kernels and the exchange of ncclDslashQcu, with
device copies in place of NCCL.  The ranks' outputs, gathered, must equal
the single-GPU dslash of the global lattice (and the oracle's) to rounding:
every hop does the single-GPU kernel's arithmetic, so they normally agree
bit for bit.  The NCCL path itself needs two GPUs; here its set-up and its
argument checks run."""
import numpy as np
import pytest

import oracle as O
from ddref import gather_half, scatter_gauge, scatter_spinor
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu

CASES = [([2, 1, 1, 1], [4, 4, 4, 4]), ([1, 2, 1, 1], [4, 4, 4, 4]), ([1, 1, 2, 1], [4, 4, 4, 4]),
         ([1, 1, 1, 2], [4, 4, 4, 4]), ([2, 2, 1, 1], [4, 6, 4, 2]), ([1, 1, 2, 2], [6, 4, 2, 4]),
         ([2, 2, 2, 2], [4, 4, 4, 4]), ([1, 1, 3, 1], [4, 4, 4, 6]), ([4, 1, 1, 1], [2, 4, 4, 4]),
         ([1, 1, 1, 4], [4, 2, 2, 2])]


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


@pytest.mark.parametrize("grid,loc", CASES, ids=lambda v: "x".join(map(str, v)))
def test_dd_dslash_equals_global(q, grid, loc):
    glatt = [loc[d] * grid[d] for d in range(4)]
    n = int(np.prod(grid))
    U = O.gauge_haar(glatt, 61)
    psi = O.fermion_gauss(O.full_shape(glatt), 62)
    Ul = scatter_gauge(U, glatt, loc, grid)       # [n, 4, 2, ...]
    pl = scatter_spinor(psi, glatt, loc, grid)    # [n, 2, ...]
    dUl = dev(Ul)
    for parity in (0, 1):
        inl = dev(np.ascontiguousarray(pl[:, 1 - parity]))
        outl = empty_like_dev(inl.shape)
        q.dslash_dd_emulate(outl, inl, dUl, loc, parity, grid)
        got = gather_half(host(outl), parity, glatt, loc, grid)
        ref = O.dslash(psi[1 - parity], U, glatt, parity)
        assert rel(got, ref) <= 1e-14, (grid, parity)
        # against the single-GPU kernel on the global lattice
        out1 = empty_like_dev(O.half_shape(glatt))
        q.dslashQcu(out1, dev(psi[1 - parity]), dev(U), q.QcuParam(glatt), parity)
        assert rel(got, host(out1)) <= 1e-15
    assert np.array_equal(host(dUl), Ul)  # inputs untouched


def test_dd_rejects_odd_extents_and_bad_ranks(q):
    loc, grid = [4, 3, 4, 4], [1, 2, 1, 1]
    poison = empty_like_dev((16,))
    with pytest.raises(q.QcuError, match="even"):
        q.dslash_dd_emulate(poison, poison, poison, loc, 0, grid)
    assert np.isnan(host(poison)).all()


def test_nccl_path_setup_and_checks(q):
    """The NCCL side on one GPU: a one-rank communicator is made and freed;
    ncclDslashQcu with a grid of several ranks refuses a missing or
    mismatched communicator and writes nothing."""
    loc = [4, 4, 4, 4]
    U = dev(O.gauge_haar(loc, 3))
    psi = dev(O.fermion_gauss(O.half_shape(loc), 4))
    out = empty_like_dev(O.half_shape(loc))
    q.ncclDslashQcu(out, psi, U, q.QcuParam(loc), 0, q.QcuParam([2, 1, 1, 1]))
    code, msg = q.last_error()
    assert code != 0 and "communicator" in msg and np.isnan(host(out)).all()
    uid = q.comm_unique_id()
    assert len(uid) == 128
    import ctypes

    buf = (ctypes.c_ubyte * 128)(*uid)
    assert q._lib.qcuCommInit(buf, 1, 0) == 0, q.last_error()
    try:
        q.ncclDslashQcu(out, psi, U, q.QcuParam(loc), 0, q.QcuParam([2, 1, 1, 1]))
        code, msg = q.last_error()
        assert code != 0 and "rank count" in msg and np.isnan(host(out)).all()
    finally:
        q.comm_free()
    # grid {1,1,1,1} stays the single-GPU call
    q.ncclDslashQcu(out, psi, U, q.QcuParam(loc), 0, q.QcuParam([1, 1, 1, 1]))
    assert q.last_error()[0] == 0
    assert rel(host(out), O.dslash(host(psi), host(U), loc, 0)) <= 1e-13


@pytest.mark.parametrize("grid,loc", [([2, 1, 1, 1], [4, 4, 4, 4]), ([1, 1, 2, 2], [4, 4, 4, 4]),
                                      ([1, 2, 1, 1], [4, 4, 4, 8])], ids=lambda v: "x".join(map(str, v)))
def test_dd_bistabcg_equals_global(q, grid, loc):
    """ncclBistabCgQcu over a grid (every rank emulated in this process):
    qcu's contract (kappa 0.125, random start, grid-wide ||r_o||^2 < 1e-9);
    the gathered solution solves the oracle's global system to that bound
    and agrees with the single-GPU solve of the global lattice, which starts
    from the same field."""
    glatt = [loc[d] * grid[d] for d in range(4)]
    U = O.gauge_smooth(glatt, 0.25, 71)
    b = O.fermion_gauss(O.full_shape(glatt), 72)
    xl = empty_like_dev((int(np.prod(grid)), 2) + tuple(O.half_shape(loc)))
    it, r2 = q.bistabcg_dd_emulate(xl, dev(scatter_spinor(b, glatt, loc, grid)),
                                   dev(scatter_gauge(U, glatt, loc, grid)), loc, grid)
    assert 0 < it < 1000 and r2 < 1e-9
    xh = host(xl)
    x = np.stack([gather_half(np.ascontiguousarray(xh[:, p]), p, glatt, loc, grid) for p in (0, 1)])
    r = b - O.mfull(x, U, glatt, 0.125)
    assert np.linalg.norm(r) ** 2 < 1.1e-9
    x1 = empty_like_dev(O.full_shape(glatt))
    q.ncclBistabCgQcu(x1, dev(b), dev(U), q.QcuParam(glatt), q.QcuParam([1, 1, 1, 1]))
    assert q.last_error()[0] == 0
    assert rel(x, host(x1)) < 1e-6
