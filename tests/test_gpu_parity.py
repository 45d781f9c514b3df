"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs.  Tolerances: FP64 <= 1e-13 relative (legacy dslash),
FP32 <= 1e-6, 16-bit fixed-point storage <= 2e-4; solves to a 1e-10 FP64 true residual."""
import numpy as np
import pytest

import oracle as O
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu

LATTS = [[4, 4, 4, 4], [8, 8, 8, 8], [6, 4, 2, 10], [2, 2, 2, 2], [4, 6, 8, 12]]


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _fields(latt, kind="haar", seed=1):
    U = O.gauge_haar(latt, seed) if kind == "haar" else O.gauge_smooth(latt, 0.3, seed)
    psi = O.fermion_gauss(O.full_shape(latt), seed + 100)
    return U, psi


@pytest.mark.parametrize("latt", LATTS)
@pytest.mark.parametrize("kind", ["haar", "smooth"])
def test_dslashQcu_fp64(q, latt, kind):
    U, psi = _fields(latt, kind)
    dU, dpsi = dev(U), dev(psi)
    for p in (0, 1):
        out = empty_like_dev(O.half_shape(latt))
        q.dslashQcu(out, dpsi[1 - p], dU, q.QcuParam(latt), p)
        assert q.last_error()[0] == 0
        assert rel(host(out), O.dslash(psi[1 - p], U, latt, p)) <= 1e-13
    # inputs untouched (qcu permuted them in place and restored them)
    assert np.array_equal(host(dU), U) and np.array_equal(host(dpsi), psi)


def test_ncclDslashQcu_and_grid_check(q):
    latt = [8, 4, 4, 8]
    U, psi = _fields(latt)
    dU, dpsi = dev(U), dev(psi)
    out = empty_like_dev(O.half_shape(latt))
    q.ncclDslashQcu(out, dpsi[0], dU, q.QcuParam(latt), 1, q.QcuParam([1, 1, 1, 1]))
    assert rel(host(out), O.dslash(psi[0], U, latt, 1)) <= 1e-13
    out2 = empty_like_dev(O.half_shape(latt))
    q.ncclDslashQcu(out2, dpsi[0], dU, q.QcuParam(latt), 1, q.QcuParam([2, 1, 1, 1]))
    code, msg = q.last_error()
    assert code != 0 and "grid" in msg
    assert np.isnan(host(out2)).all()  # nothing written
    q.mpiDslashQcu(out2, dpsi[0], dU, q.QcuParam(latt), 1, q.QcuParam([1, 1, 1, 1]))  # no-op, as in qcu
    assert np.isnan(host(out2)).all()


def test_bad_arguments_do_not_crash(q):
    latt = [5, 4, 4, 4]  # odd Lx
    out = empty_like_dev((10,))
    q.dslashQcu(out, out, out, q.QcuParam(latt), 0)
    assert q.last_error()[0] == 1
    q.dslashQcu(out, out, out, q.QcuParam([4, 4, 4, 4]), 2)
    assert q.last_error()[0] == 1
    q.dslashQcu(None, out, out, q.QcuParam([4, 4, 4, 4]), 0)
    assert q.last_error()[0] == 1


@pytest.mark.parametrize("latt,kind", [([4, 4, 4, 4], "smooth"), ([4, 4, 2, 8], "smooth"), ([4, 4, 4, 4], "haar")])
def test_dslashCloverQcu(q, latt, kind):
    U, psi = _fields(latt, kind, seed=3)
    dU, dpsi = dev(U), dev(psi)
    for p in (0, 1):
        A = O.clover_build(U, latt, p, 1.0)
        cond = np.linalg.cond(A).max()
        expect = O.clover_apply(O.clover_invert(A), O.dslash(psi[1 - p], U, latt, p))
        out = empty_like_dev(O.half_shape(latt))
        q.dslashCloverQcu(out, dpsi[1 - p], dU, q.QcuParam(latt), p)
        assert q.last_error()[0] == 0
        assert rel(host(out), expect) <= 1e-14 * max(cond, 10)


@pytest.mark.parametrize("latt", [[8, 4, 6, 8], [6, 2, 2, 6]])  # Vh = 768 and 72 (not a multiple of 32)
@pytest.mark.parametrize("t_bc", [1.0, -1.0])
@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-6), (16, 2e-4), (3216, 2e-4)])
def test_ext_dslash_precisions(q, latt, t_bc, prec, tol):
    """Every storage precision of the hopping term against the FP64 oracle
    (3216: FP32 spinors with 16-bit links)."""
    U, psi = _fields(latt, "smooth", 5)
    with q.Gauge(dev(U), latt, t_boundary=t_bc) as G:
        for p in (0, 1):
            out = empty_like_dev(O.half_shape(latt))
            G.dslash(out, dev(psi[1 - p]), p, precision=prec)
            assert rel(host(out), O.dslash(psi[1 - p], U, latt, p, t_bc)) <= tol


@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-6), (16, 2e-4), (3216, 2e-4)])
def test_ext_clover_dslash_csw(q, prec, tol):
    latt = [4, 4, 6, 8]
    U, psi = _fields(latt, "smooth", 6)
    kappa, csw = 0.12, 1.0
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=kappa * csw) as G:
        for p in (0, 1):
            Ainv = O.clover_invert(O.clover_build(U, latt, p, kappa * csw))
            expect = O.clover_apply(Ainv, O.dslash(psi[1 - p], U, latt, p, -1.0))
            out = empty_like_dev(O.half_shape(latt))
            G.dslash(out, dev(psi[1 - p]), p, clover=True, precision=prec)
            assert rel(host(out), expect) <= tol


@pytest.mark.parametrize("clover", [False, True])
def test_ext_matpc_and_mat(q, clover):
    latt = [4, 6, 4, 8]
    U, psi = _fields(latt, "smooth", 7)
    kappa = 0.11
    c = kappa * 1.0
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=c if clover else 0.0) as G:
        A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
        Ai = [O.clover_invert(a) for a in A] if clover else [None, None]
        out = empty_like_dev(O.half_shape(latt))
        G.matpc(out, dev(psi[1]), kappa, clover=clover)
        assert rel(host(out), O.mpc(psi[1], U, latt, kappa, 1, -1.0, True, Ai[1], Ai[0])) <= 1e-13
        full = empty_like_dev(O.full_shape(latt))
        G.mat(full, dev(psi), kappa, clover=clover)
        assert rel(host(full), O.mfull(psi, U, latt, kappa, -1.0, True, A[0], A[1])) <= 1e-13


def test_generators_match_oracle(q):
    import torch

    latt = [4, 4, 6, 8]
    for kind, ref in ((0, O.gauge_haar(latt, 77)), (1, O.gauge_smooth(latt, 0.25, 77))):
        g = torch.empty(O.gauge_shape(latt), dtype=torch.complex128, device="cuda")
        q.gauge_random(g, latt, kind, 0.25, 77)
        assert rel(host(g), ref) < 1e-13
    f = torch.empty(O.full_shape(latt), dtype=torch.complex128, device="cuda")
    q.fermion_random(f, f.numel(), 0, 5)
    assert rel(host(f), O.fermion_gauss(O.full_shape(latt), 5)) < 1e-14
    q.fermion_random(f, f.numel(), 1, 5)
    assert np.array_equal(host(f), O.fermion_uniform(O.full_shape(latt), 5))


def test_ncclBistabCgQcu(q):
    """qcu's solver semantics: kappa = 0.125, random start, ||r_o||^2 < 1e-9."""
    latt = [8, 8, 8, 8]
    U = O.gauge_haar(latt, 2)
    b = np.ones(O.full_shape(latt), complex)  # the reference test's source (test.nccl.bistabcg.qcu-np1.py:30)
    x = empty_like_dev(O.full_shape(latt))
    q.ncclBistabCgQcu(x, dev(b), dev(U), q.QcuParam(latt), q.QcuParam([1, 1, 1, 1]))
    assert q.last_error()[0] == 0
    xg = host(x)
    x0 = np.zeros_like(b)
    x0[1] = O.fermion_uniform(O.half_shape(latt), 23333)
    xo, it, res2 = O.solve_full(b, U, latt, 0.125, x0=x0, tol=1e-9, abs_tol=True, maxiter=1000)
    r = b - O.mfull(xg, U, latt, 0.125)
    assert np.linalg.norm(r) ** 2 < 1e-9
    assert rel(xg, xo) < 1e-6


@pytest.mark.parametrize("prec", [64, 32, 16])
@pytest.mark.parametrize("clover", [False, True])
def test_invert_true_residual(q, prec, clover):
    latt = [8, 8, 8, 16]
    U = O.gauge_smooth(latt, 0.25, 9)
    b = O.fermion_gauss(O.full_shape(latt), 19)
    kappa = 0.125
    c = kappa * 1.0
    A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=c if clover else 0.0) as G:
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(b), kappa, tol=1e-10, maxiter=5000, precision=prec, delta=0.1, clover=clover)
    assert info["status"] == 1, info
    assert info["true_residual"] <= 1e-10
    xg = host(x)
    r = b - O.mfull(xg, U, latt, kappa, -1.0, True, A[0], A[1])
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-10
    # same solution as the FP64 oracle solve (error bounded by the condition number)
    kw = dict(Ainv_e=O.clover_invert(A[0]), Ainv_o=O.clover_invert(A[1])) if clover else {}
    xo, _, _ = O.solve_full(b, U, latt, kappa, t_bc=-1.0, tol=1e-12, maxiter=5000, **kw)
    assert rel(xg, xo) < 1e-7
    if prec == 64 and not clover:
        # same algorithm, same stopping point: the library stops on
        # ||r_o|| <= tol ||b|| (full source), the oracle on ||r_o|| <= tol' ||b'_o||
        bp = b[1] + kappa * O.dslash(b[0], U, latt, 1, -1.0)
        tol_o = 1e-10 * np.linalg.norm(b) / np.linalg.norm(bp)
        _, it, _ = O.solve_full(b, U, latt, kappa, t_bc=-1.0, tol=tol_o, maxiter=5000)
        assert abs(info["iterations"] - it) <= 2


def test_invert_zero_source_and_initial_guess(q):
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 3)
    with q.Gauge(dev(U), latt) as G:
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(np.zeros(O.full_shape(latt), complex)), 0.12)
        assert info["status"] == 1 and np.abs(host(x)).max() == 0
        b = O.fermion_gauss(O.full_shape(latt), 1)
        x = dev(np.zeros(O.full_shape(latt), complex))
        i1 = G.invert(x, dev(b), 0.12, tol=1e-10)
        i2 = G.invert(x, dev(b), 0.12, tol=1e-10, x0_mode=1)  # restart from the solution
        assert i2["iterations"] <= 2 and i2["true_residual"] <= 1e-10 and i1["iterations"] > 10


def test_invert_maxiter_reports_status(q):
    latt = [4, 4, 4, 8]
    U = O.gauge_smooth(latt, 0.25, 3)
    b = O.fermion_gauss(O.full_shape(latt), 2)
    with q.Gauge(dev(U), latt) as G:
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(b), 0.124, tol=1e-12, maxiter=3)
    assert info["status"] == 2 and info["iterations"] == 3
    assert np.isfinite(host(x)).all()


@pytest.mark.parametrize("prec", [32, 16, 3216])
@pytest.mark.parametrize("clover", [False, True])
def test_invert_gcr_true_residual(q, prec, clover):
    """Flexible GCR (FP64) preconditioned by a low-precision inner BiCGSTAB."""
    latt = [8, 8, 8, 16]
    U = O.gauge_smooth(latt, 0.25, 10)
    b = O.fermion_gauss(O.full_shape(latt), 20)
    kappa = 0.126
    c = kappa * 1.0
    A = [O.clover_build(U, latt, p, c) for p in (0, 1)] if clover else [None, None]
    with q.Gauge(dev(U), latt, t_boundary=-1.0, clover_coeff=c if clover else 0.0) as G:
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(b), kappa, tol=1e-10, maxiter=5000, precision=32 if prec == 3216 else prec,
                        gauge_precision=16 if prec == 3216 else 0, clover=clover, solver="gcr", inner_iters=12,
                        gcr_k=6)
    assert info["status"] == 1, info
    assert info["true_residual"] <= 1e-10
    r = b - O.mfull(host(x), U, latt, kappa, -1.0, True, A[0], A[1])
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-10
    assert info["reliable_updates"] >= 2  # outer steps


def test_gauge_load_waits_for_inflight_copy(q):
    """A gauge field still being copied host->device on another stream when
    the handle is loaded: the load must see the finished field."""
    import torch

    latt = [16, 16, 16, 32]
    U = O.gauge_smooth(latt, 0.25, 41)
    psi = O.fermion_gauss(O.half_shape(latt), 42)
    hU = torch.from_numpy(U).pin_memory()
    dU = torch.zeros(U.shape, dtype=torch.complex128, device="cuda")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        dU.copy_(hU, non_blocking=True)  # no synchronisation before the load
        G = q.Gauge(dU, latt, t_boundary=-1.0)
    try:
        out = empty_like_dev(O.half_shape(latt))
        G.dslash(out, dev(psi), 0)
    finally:
        G.close()
    assert rel(host(out), O.dslash(psi, U, latt, 0, -1.0)) <= 1e-13


def test_gcr_stall_falls_back_to_plain_fp64(q, monkeypatch):
    """A GCR solve that stalls hands over to plain FP64 BiCGSTAB, which
    finishes from the last FP64 iterate; the FP64 true residual decides as
    always.  The stall is declared on the host: QCU_GCR_STALL_CYCLES=0 ends the
    GCR solve after its first cycle."""
    latt, kappa = [8, 8, 8, 8], 0.124
    U, _ = _fields(latt, "smooth", 41)
    b = O.fermion_gauss(O.full_shape(latt), 42)
    kw = dict(tol=1e-10, maxiter=4000, solver="gcr", precision=16, inner_iters=4, inner_tol=0.5, gcr_k=2)
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        x = empty_like_dev(O.full_shape(latt))
        ref = G.invert(x, dev(b), kappa, **kw)
        assert ref["status"] == 1 and ref["fallback"] == 0, ref
        monkeypatch.setenv("QCU_GCR_STALL_CYCLES", "0")
        x = empty_like_dev(O.full_shape(latt))
        info = G.invert(x, dev(b), kappa, **kw)
        assert info["status"] == 1 and info["fallback"] == 1, info
        assert info["true_residual"] <= 1e-10
        r = b - O.mfull(host(x), U, latt, kappa, -1.0)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-10


def test_repeated_gcr_solves_reuse_nothing_stale(q):
    """Workspace, graphs and solver state carry nothing from one solve to the
    next: a solve repeated after one with another kappa is bit-identical, and a
    solve on a second gauge field of the same size (a new handle, possibly at
    the same addresses) solves its own system."""
    latt = [8, 8, 8, 8]
    kw = dict(tol=1e-10, maxiter=4000, solver="gcr", precision=16, inner_iters=16, inner_tol=0.1, gcr_k=4)
    U1, _ = _fields(latt, "smooth", 51)
    U2, _ = _fields(latt, "smooth", 52)
    b = O.fermion_gauss(O.full_shape(latt), 53)
    with q.Gauge(dev(U1), latt, t_boundary=-1.0) as G:
        xa = empty_like_dev(O.full_shape(latt))
        ia = G.invert(xa, dev(b), 0.124, **kw)
        xb = empty_like_dev(O.full_shape(latt))
        ib = G.invert(xb, dev(b), 0.12, **kw)
        xc = empty_like_dev(O.full_shape(latt))
        ic = G.invert(xc, dev(b), 0.124, **kw)
    assert ia["status"] == ib["status"] == ic["status"] == 1
    assert ia["iterations"] == ic["iterations"]
    assert np.array_equal(host(xa), host(xc))
    for x, kappa in ((xa, 0.124), (xb, 0.12)):
        r = b - O.mfull(host(x), U1, latt, kappa, -1.0)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-10
    with q.Gauge(dev(U2), latt, t_boundary=-1.0) as G2:  # a new handle, possibly at the same addresses
        xd = empty_like_dev(O.full_shape(latt))
        idd = G2.invert(xd, dev(b), 0.124, **kw)
    assert idd["status"] == 1
    r = b - O.mfull(host(xd), U2, latt, 0.124, -1.0)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-10


def test_dslashCloverQcu_threads_share_one_device(q):
    """dslashCloverQcu keeps its clover scratch in the calling device's
    context, under that context's lock: calls from two host threads on one
    device give, call after call, exactly the results of serial calls."""
    import threading

    cases = [([8, 8, 8, 8], 41, 0), ([4, 4, 8, 8], 42, 1)]
    inputs, refs = [], []
    for latt, seed, par in cases:
        U, psi = _fields(latt, "smooth", seed)
        dU, dpsi = dev(U), dev(psi[1 - par])
        out = empty_like_dev(O.half_shape(latt))
        q.dslashCloverQcu(out, dpsi, dU, q.QcuParam(latt), par)
        assert q.last_error()[0] == 0
        A = O.clover_build(U, latt, par, 1.0)
        ref = O.clover_apply(O.clover_invert(A), O.dslash(psi[1 - par], U, latt, par, 1.0))
        assert rel(host(out), ref) <= 1e-11  # smooth links: the inverse is well conditioned
        inputs.append((latt, dU, dpsi, par))
        refs.append(host(out))
    errors = []

    def worker(k):
        import torch

        torch.cuda.set_device(0)
        latt, dU, dpsi, par = inputs[k]
        for _ in range(6):
            out = empty_like_dev(O.half_shape(latt))
            q.dslashCloverQcu(out, dpsi, dU, q.QcuParam(latt), par)
            code, msg = q.last_error()
            if code != 0 or not np.array_equal(host(out), refs[k]):
                errors.append((k, code, msg))

    th = [threading.Thread(target=worker, args=(k,)) for k in range(len(cases))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors


def test_dslashQcu_on_pyquda_weak_field_lime(q):
    """A gauge file this project did not write: PyQuda's own test
    configuration (python/PyQuda/tests/weak_field.lime, 4^3 x 8), read by
    qcu_b200.ildg, through dslashQcu, dslashCloverQcu and a solve, against
    the oracle."""
    import os

    from qcu_b200 import ildg

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "weak_field.lime")
    U, latt, info = ildg.read_ildg(path)
    assert latt == [4, 4, 4, 8] and info["checksum"] == "ok"
    psi = O.fermion_gauss(O.full_shape(latt), 77)
    dU, dpsi = dev(U), dev(psi)
    for p in (0, 1):
        out = empty_like_dev(O.half_shape(latt))
        q.dslashQcu(out, dpsi[1 - p], dU, q.QcuParam(latt), p)
        assert q.last_error()[0] == 0
        assert rel(host(out), O.dslash(psi[1 - p], U, latt, p)) <= 1e-13
        out = empty_like_dev(O.half_shape(latt))
        q.dslashCloverQcu(out, dpsi[1 - p], dU, q.QcuParam(latt), p)
        assert q.last_error()[0] == 0
        A = O.clover_build(U, latt, p, 1.0)
        ref = O.clover_apply(O.clover_invert(A), O.dslash(psi[1 - p], U, latt, p))
        assert rel(host(out), ref) <= 1e-12
    # a clover solve on the file's field (antiperiodic t, csw = 1), checked with the oracle's operator
    kappa = 0.12
    A = [O.clover_build(U, latt, p, kappa) for p in (0, 1)]
    x = empty_like_dev(O.full_shape(latt))
    with q.Gauge(dU, latt, t_boundary=-1.0, clover_coeff=kappa) as G:
        res = G.invert(x, dpsi, kappa, tol=1e-10, precision=16, solver="gcr", clover=True)
    assert res["status"] == 1
    r = psi - O.mfull(host(x), U, latt, kappa, -1.0, True, A[0], A[1])
    assert np.linalg.norm(r) / np.linalg.norm(psi) <= 1.05e-10


def test_dslashQcu_16_byte_aligned_buffers(q):
    """dslashQcu reads 32-byte aligned PyQuda buffers with 32-byte accesses;
    buffers that are only 16-byte aligned (a complex128 view one element into
    an allocation) take the 16-byte path and give the same result."""
    import torch

    latt = [8, 4, 4, 8]
    U, psi = _fields(latt, "haar", 21)
    ref = O.dslash(psi[0], U, latt, 1)
    n = int(np.prod(O.half_shape(latt)))
    for shift in (0, 1):  # elements of 16 bytes
        src = torch.zeros(n + 1, dtype=torch.complex128, device="cuda")
        src[shift:shift + n] = torch.from_numpy(np.ascontiguousarray(psi[0]).reshape(-1)).cuda()
        dst = torch.full((n + 1,), float("nan"), dtype=torch.complex128, device="cuda")
        pin, pout = src[shift:shift + n], dst[shift:shift + n]
        assert (pin.data_ptr() % 32 == 0) == (shift == 0)
        q.dslashQcu(pout, pin, dev(U), q.QcuParam(latt), 1)
        assert q.last_error()[0] == 0
        assert rel(host(pout).reshape(ref.shape), ref) <= 1e-13
        assert np.isnan(host(dst)[shift + n:]).all() and np.isnan(host(dst)[:shift]).all()
