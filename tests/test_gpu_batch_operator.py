"""Operator-level parity of the batched solver's inner kernels.

A flexible outer Krylov method converges even with a wrong inner operator
(only more slowly), so a converged batched solve does not show that the
batched hopping kernels compute D.  Here qcuBatchApplyMatPC runs those
kernels once, with the launch shapes the autotuner chooses from (sites per
block x right-hand sides per thread, and the tensor-core kernel in both
modes), on right-hand sides of three lattices of uneven volume (one with a
ragged last block, one with clover) at every inner storage, and each
right-hand side's result is compared with the CPU oracle:
    even half  [A_e^-1] D_eo b_o       odd half  M_pc b_o
together with the two fused reductions of the inner iteration.
Bars (relative, per right-hand side): FP64 1e-12; FP32 spinors and links,
and the 3xTF32 tensor-core mode, 1e-6; 16-bit links or spinors 2e-4 (the
15-bit fixed point of the stored input and links); one-pass TF32 2e-3
(operands rounded to 11 significant bits, 4 x 2^-11)."""
import numpy as np
import pytest

import oracle as O
from util import dev, host, rel

pytestmark = pytest.mark.gpu

T_BC = -1.0
# (lattice, kappa, nrhs, clover): uneven volumes; Vh = 2048, 512 and 72 (72: no block size divides it)
SYSTEMS = [([8, 8, 8, 8], 0.124, 3, False), ([4, 4, 8, 8], 0.125, 2, True), ([6, 2, 2, 6], 0.12, 1, False)]
# (sites per block, rhs per thread, tensor-core mode): every shape the autotuner tries
SHAPES = [(64, 1, 0), (128, 1, 0), (256, 1, 0), (64, 2, 0), (128, 2, 0), (64, 4, 0), (128, 4, 0), (32, 8, 1),
          (32, 8, 2)]
# (spinor precision, link precision, bar)
PRECS = [(32, 0, 1e-6), (32, 16, 2e-4), (16, 0, 2e-4)]


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


@pytest.fixture(scope="module")
def systems(q):
    out = []
    for i, (latt, kappa, nrhs, clover) in enumerate(SYSTEMS):
        U = O.gauge_smooth(latt, 0.25, 50 + i)
        c = kappa if clover else 0.0
        Ainv = [O.clover_invert(O.clover_build(U, latt, p, c)) for p in (0, 1)] if clover else [None, None]
        b = np.stack([O.fermion_gauss(O.full_shape(latt), 500 + 10 * i + j) for j in range(nrhs)])
        exp_e, exp_o = [], []
        for j in range(nrhs):
            bo = b[j, 1]
            e = O.dslash(bo, U, latt, 0, T_BC)
            if clover:
                e = O.clover_apply(Ainv[0], e)
            exp_e.append(e)
            exp_o.append(O.mpc(bo, U, latt, kappa, 1, T_BC, True, Ainv[1], Ainv[0]))
        G = q.Gauge(dev(U), latt, t_boundary=T_BC, clover_coeff=c)
        out.append(dict(latt=latt, kappa=kappa, clover=clover, b=b, db=dev(b), G=G, exp_e=exp_e, exp_o=exp_o))
    yield out
    for s in out:
        s["G"].close()


def _run(q, systems, prec, gprec, shape):
    import torch

    xs = [torch.full(s["b"].shape, float("nan"), dtype=torch.complex128, device="cuda") for s in systems]
    dots = q.batch_apply_matpc([(s["G"], x, s["db"], s["kappa"], s["clover"]) for s, x in zip(systems, xs)],
                               precision=prec, gauge_precision=gprec, dslash_threads=shape[0], dslash_rhs=shape[1],
                               mma=shape[2])
    return [host(x) for x in xs], dots


def _check(systems, xs, dots, bar):
    k = 0
    for s, x in zip(systems, xs):
        for j in range(s["b"].shape[0]):
            assert rel(x[j, 0], s["exp_e"][j]) <= bar, ("even", s["latt"], j)
            assert rel(x[j, 1], s["exp_o"][j]) <= bar, ("odd", s["latt"], j)
            bo, v = s["b"][j, 1], s["exp_o"][j]
            scale = np.linalg.norm(bo) * np.linalg.norm(v)
            d_rt = np.vdot(bo, v)  # <b_o, M_pc b_o>
            assert abs(complex(dots[k, 0], dots[k, 1]) - d_rt) <= 2 * bar * scale, ("<rt,v>", s["latt"], j)
            assert abs(complex(dots[k, 2], dots[k, 3]) - np.conj(d_rt)) <= 2 * bar * scale, ("<t,s>", s["latt"], j)
            assert abs(dots[k, 4] - np.vdot(v, v).real) <= 3 * bar * np.vdot(v, v).real, ("|t|^2", s["latt"], j)
            k += 1


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}mma{s[2]}")
@pytest.mark.parametrize("prec,gprec,bar", PRECS, ids=["fp32", "fp32-links16", "16bit"])
def test_batched_inner_operator(q, systems, prec, gprec, bar, shape):
    if shape[2] and prec != 32:
        with pytest.raises(q.QcuError, match="tensor-core"):
            _run(q, systems, prec, gprec, shape)
        return
    if shape[2] == 2:
        bar = 2e-3  # one TF32 pass
    xs, dots = _run(q, systems, prec, gprec, shape)
    _check(systems, xs, dots, bar)


def test_batched_fp64_operator(q, systems):
    """The batched FP64 kernels (precision 64 runs the inner solve in FP64)."""
    xs, dots = _run(q, systems, 64, 0, (128, 1, 0))
    _check(systems, xs, dots, 1e-12)


def test_batched_operator_rejects_unknown_shape(q, systems):
    with pytest.raises(q.QcuError, match="shape"):
        _run(q, systems, 32, 0, (96, 1, 0))
