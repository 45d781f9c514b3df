"""The workloads at their full sizes, checked against the CPU oracle (OpenMP;
one FP64 hopping term at 32^3 x 64 takes tens of milliseconds on the host):

- 24^3 x 48, smooth links eps 0.3, clover csw 1 (the clover dslash and solve
  workload): the FP64 clover hopping term against the oracle's, the FP32,
  FP32-with-16-bit-links and 16-bit ones against the oracle within their
  storage bars, the FP64 one linear to rounding; solves at every inner
  precision reaching a true relative residual <= 1e-10 of the oracle's full
  clover operator;
- 32^3 x 64, smooth links eps 0.25, kappa 0.1303 (the benchmark system): the
  FP64 hopping term (legacy PyQuda-layout path and packed path) against the
  oracle's, and the chosen solver (16-bit inner solve) and plain FP64
  BiCGSTAB both reaching a true relative residual <= 1e-10 of the oracle's
  full operator, and agreeing with each other."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _nrel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _system(q, latt, eps, gauge_seed, src_seed):
    L = q.Layout(tuple(latt))
    U = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(U, latt, 1, eps, gauge_seed)
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, src_seed)
    return L, U, b


def _oracle_residual(x, b, Uh, latt, kappa, A=(None, None)):
    """|b - M x| / |b| with the oracle's FP64 full operator, on the host."""
    bh = b.cpu().numpy()
    r = bh - O.mfull(x.cpu().numpy(), Uh, latt, kappa, -1.0, True, A[0], A[1])
    return float(np.linalg.norm(r) / np.linalg.norm(bh))


LATT_CLOVER = [24, 24, 24, 48]
KAPPA_CLOVER, CSW = 0.125, 1.0


@pytest.fixture(scope="module")
def clover_system(q):
    L, U, b = _system(q, LATT_CLOVER, 0.3, 2401, 2402)
    G = q.Gauge(U, LATT_CLOVER, t_boundary=-1.0, clover_coeff=KAPPA_CLOVER * CSW)
    Uh = U.cpu().numpy()
    A = [O.clover_build(Uh, LATT_CLOVER, p, KAPPA_CLOVER * CSW) for p in (0, 1)]
    del U
    yield L, G, b, Uh, A
    G.close()


def _oracle_clover_dslash(Uh, A, inp, parity):
    return O.clover_apply(O.clover_invert(A[parity]), O.dslash(inp, Uh, LATT_CLOVER, parity, -1.0))


@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-6), (3216, 2e-4), (16, 2e-4)])
def test_clover_dslash_precisions_full_size(q, clover_system, prec, tol):
    L, G, b, Uh, A = clover_system
    for parity in (0, 1):
        inp = b[1 - parity].contiguous()
        out = torch.full(L.half, float("nan"), dtype=torch.complex128, device="cuda")
        G.dslash(out, inp, parity, clover=True, precision=prec)
        assert _nrel(out.cpu().numpy(), _oracle_clover_dslash(Uh, A, inp.cpu().numpy(), parity)) <= tol


def test_clover_dslash_linear_full_size(q, clover_system):
    L, G, b, _, _ = clover_system
    x, y = b[0].contiguous(), b[1].contiguous()
    a, c = 0.7 - 0.2j, -1.3 + 0.4j
    dx, dy, dz = (torch.empty(L.half, dtype=torch.complex128, device="cuda") for _ in range(3))
    G.dslash(dx, x, 1, clover=True, precision=64)
    G.dslash(dy, y, 1, clover=True, precision=64)
    G.dslash(dz, (a * x + c * y).contiguous(), 1, clover=True, precision=64)
    assert _rel(dz, a * dx + c * dy) <= 1e-14


@pytest.mark.parametrize("prec,gprec", [(16, 0), (32, 16), (32, 0), (64, 0)])
def test_clover_solve_full_size(q, clover_system, prec, gprec):
    L, G, b, Uh, A = clover_system
    x = torch.zeros_like(b)
    info = G.invert(x, b, KAPPA_CLOVER, tol=1e-10, maxiter=20000, clover=True, precision=prec,
                    gauge_precision=gprec, solver="gcr", inner_iters=96, inner_tol=0.05, gcr_k=4)
    assert info["status"] == 1, info
    assert _oracle_residual(x, b, Uh, LATT_CLOVER, KAPPA_CLOVER, A) <= 1.05e-10


@pytest.fixture(scope="module")
def bench_system(q):
    import bench  # the benchmark's own system: its seeds, eps and kappa

    latt, kappa = list(bench.LATT), bench.KAPPA
    L, U, b = _system(q, latt, bench.EPS, bench.GAUGE_SEED, bench.SRC_SEED)
    yield latt, kappa, L, U, b


def test_benchmark_dslash_fp64_vs_oracle(q, bench_system):
    latt, _, L, U, b = bench_system
    Uh = U.cpu().numpy()
    inp = b[0].contiguous()
    ref = O.dslash(inp.cpu().numpy(), Uh, latt, 1, 1.0)
    out = torch.full(L.half, float("nan"), dtype=torch.complex128, device="cuda")
    q.dslashQcu(out, inp, U, q.QcuParam(latt), 1)  # legacy path: PyQuda layout, periodic
    assert q.last_error()[0] == 0
    assert _nrel(out.cpu().numpy(), ref) <= 1e-13
    with q.Gauge(U, latt, t_boundary=-1.0) as G:  # packed path, antiperiodic t
        out.fill_(float("nan"))
        G.dslash(out, inp, 1, precision=64)
        assert _nrel(out.cpu().numpy(), O.dslash(inp.cpu().numpy(), Uh, latt, 1, -1.0)) <= 1e-13


def test_benchmark_system_chosen_vs_plain(q, bench_system):
    latt, kappa, L, U, b = bench_system
    Uh = U.cpu().numpy()
    with q.Gauge(U, latt, t_boundary=-1.0) as G:
        x64 = torch.zeros_like(b)
        info = G.invert(x64, b, kappa, tol=1e-10, maxiter=20000, precision=64, delta=0.0)
        assert info["status"] == 1, info
        assert _oracle_residual(x64, b, Uh, latt, kappa) <= 1.05e-10
        x = torch.zeros_like(b)
        info = G.invert(x, b, kappa, tol=1e-10, maxiter=20000, precision=16, solver="gcr", inner_iters=96,
                        inner_tol=0.05, gcr_k=4)
        assert info["status"] == 1, info
        assert _oracle_residual(x, b, Uh, latt, kappa) <= 1.05e-10
        # two solutions of the same system to 1e-10 residual: they differ by at
        # most the condition-number-amplified residual
        assert _rel(x, x64) <= 1e-6
