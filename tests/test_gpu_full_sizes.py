"""The workloads at their full sizes, through properties that need no CPU
oracle at that size (the oracle pins every kernel on small lattices):

- 24^3 x 48, smooth links eps 0.3, clover csw 1 (the clover dslash and solve
  workload): the FP32, FP32-with-16-bit-links and 16-bit clover hopping terms
  against the FP64 one; the FP64 one linear to rounding; solves at every inner
  precision reaching a true relative residual <= 1e-10, recomputed here with
  the FP64 operator on the full system;
- 32^3 x 64, smooth links eps 0.25, kappa 0.1303 (the benchmark system): the
  chosen solver (16-bit inner solve) against plain FP64 BiCGSTAB, both checked
  the same way, and their solutions against each other."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _system(q, latt, eps, gauge_seed, src_seed):
    L = q.Layout(tuple(latt))
    U = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(U, latt, 1, eps, gauge_seed)
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, src_seed)
    return L, U, b


def _true_residual(G, x, b, kappa, clover):
    r = torch.empty_like(b)
    G.mat(r, x, kappa, clover=clover)
    return _rel(r, b)  # |M x - b| / |b|


LATT_CLOVER = [24, 24, 24, 48]
KAPPA_CLOVER, CSW = 0.125, 1.0


@pytest.fixture(scope="module")
def clover_system(q):
    L, U, b = _system(q, LATT_CLOVER, 0.3, 2401, 2402)
    G = q.Gauge(U, LATT_CLOVER, t_boundary=-1.0, clover_coeff=KAPPA_CLOVER * CSW)
    yield L, G, b
    G.close()


@pytest.mark.parametrize("prec,tol", [(32, 1e-6), (3216, 2e-4), (16, 2e-4)])
def test_clover_dslash_precisions_full_size(q, clover_system, prec, tol):
    L, G, b = clover_system
    for parity in (0, 1):
        inp = b[1 - parity].contiguous()
        ref = torch.empty(L.half, dtype=torch.complex128, device="cuda")
        out = torch.full(L.half, float("nan"), dtype=torch.complex128, device="cuda")
        G.dslash(ref, inp, parity, clover=True, precision=64)
        G.dslash(out, inp, parity, clover=True, precision=prec)
        assert _rel(out, ref) <= tol


def test_clover_dslash_linear_full_size(q, clover_system):
    L, G, b = clover_system
    x, y = b[0].contiguous(), b[1].contiguous()
    a, c = 0.7 - 0.2j, -1.3 + 0.4j
    dx, dy, dz = (torch.empty(L.half, dtype=torch.complex128, device="cuda") for _ in range(3))
    G.dslash(dx, x, 1, clover=True, precision=64)
    G.dslash(dy, y, 1, clover=True, precision=64)
    G.dslash(dz, (a * x + c * y).contiguous(), 1, clover=True, precision=64)
    assert _rel(dz, a * dx + c * dy) <= 1e-14


@pytest.mark.parametrize("prec,gprec", [(16, 0), (32, 16), (32, 0), (64, 0)])
def test_clover_solve_full_size(q, clover_system, prec, gprec):
    L, G, b = clover_system
    x = torch.zeros_like(b)
    info = G.invert(x, b, KAPPA_CLOVER, tol=1e-10, maxiter=20000, clover=True, precision=prec,
                    gauge_precision=gprec, solver="gcr", inner_iters=96, inner_tol=0.05, gcr_k=4)
    assert info["status"] == 1, info
    assert _true_residual(G, x, b, KAPPA_CLOVER, True) <= 1.05e-10


def test_benchmark_system_chosen_vs_plain(q):
    import bench  # the benchmark's own system: its seeds, eps and kappa

    latt, kappa = list(bench.LATT), bench.KAPPA
    L, U, b = _system(q, latt, bench.EPS, bench.GAUGE_SEED, bench.SRC_SEED)
    with q.Gauge(U, latt, t_boundary=-1.0) as G:
        x64 = torch.zeros_like(b)
        info = G.invert(x64, b, kappa, tol=1e-10, maxiter=20000, precision=64, delta=0.0)
        assert info["status"] == 1, info
        assert _true_residual(G, x64, b, kappa, False) <= 1.05e-10
        x = torch.zeros_like(b)
        info = G.invert(x, b, kappa, tol=1e-10, maxiter=20000, precision=16, solver="gcr", inner_iters=96,
                        inner_tol=0.05, gcr_k=4)
        assert info["status"] == 1, info
        assert _true_residual(G, x, b, kappa, False) <= 1.05e-10
        # two solutions of the same system to 1e-10 residual: they differ by at
        # most the condition-number-amplified residual
        assert _rel(x, x64) <= 1e-6
