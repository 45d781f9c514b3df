"""The multi-right-hand-side hopping term on the tcgen05 tensor cores
(qcuDslashMultiTC) against the CPU oracle, right-hand side by right-hand side.

Per site and hop one tensor-core product serves every right-hand side:
A = the neighbours' spinors (rows = right-hand sides), B = the real form of
(1 -+ gamma_mu) x U.  Operands are FP16: each input spinor component is
rounded once to 11 significant bits, each entry of B likewise (from the
16-bit links), the products accumulate in FP32 and the result is rounded to
FP16.  Every rounding is at most 2^-11 relative, and the 96 products of an
output component average theirs, so the bar per right-hand side is 2e-3
relative.  Covered: 1, 12, 64 (rows padded to 64), 65 and 128 (padded to 128)
right-hand sides; both output parities; periodic and antiperiodic time
boundaries; a lattice whose site count is not a multiple of the CTA count
and whose Lz takes z-slabs of 2 planes, and one with many sites per CTA (both
pipeline slots cycling); repeated application bit-identical; a right-hand
side that is twice another gives twice its output (to 1e-8: FP16 rounding
commutes with the factor 2 except for subnormal values) and a zero
right-hand side gives zero."""
import numpy as np
import pytest

import oracle as O
from util import dev, host, rel

pytestmark = pytest.mark.gpu

# (lattice, t boundary): Vh = 2048, 288 (Lz = 6: slabs of 2 planes), 8192 (27-28 sites per CTA)
LATTS = [([8, 8, 8, 8], -1.0), ([6, 4, 6, 4], 1.0), ([16, 8, 8, 16], -1.0)]
NRHS = [1, 12, 64, 65, 128]
BAR = 2e-3


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


@pytest.fixture(scope="module")
def fields(q):
    out = {}
    for i, (latt, tbc) in enumerate(LATTS):
        U = O.gauge_smooth(latt, 0.25, 70 + i)
        G = q.Gauge(dev(U), latt, t_boundary=tbc)
        psi = np.stack([O.fermion_gauss(O.half_shape(latt), 900 + 37 * i + j) for j in range(max(NRHS))])
        out[i] = dict(latt=latt, tbc=tbc, U=U, G=G, psi=psi, ref={})
    yield out
    for f in out.values():
        f["G"].close()


def _expected(f, j, par):
    key = (j, par)
    if key not in f["ref"]:
        f["ref"][key] = O.dslash(f["psi"][j], f["U"], f["latt"], par, f["tbc"])
    return f["ref"][key]


@pytest.mark.parametrize("li", range(len(LATTS)))
@pytest.mark.parametrize("nrhs", NRHS)
def test_multi_rhs_tensor_core_dslash_matches_oracle(q, fields, li, nrhs):
    import torch

    f = fields[li]
    inp = dev(f["psi"][:nrhs])
    out = torch.full_like(inp, float("nan"))
    for par in (0, 1):
        f["G"].dslash_multi_tc(out, inp, nrhs, par)
        got = host(out)
        errs = [rel(got[j], _expected(f, j, par)) for j in range(nrhs)]
        assert max(errs) < BAR, (f["latt"], nrhs, par, max(errs))
    # the same application again: bit for bit
    again = torch.full_like(inp, float("nan"))
    f["G"].dslash_multi_tc(again, inp, nrhs, 1)
    assert torch.equal(again, out)


def test_multi_rhs_linearity_and_zero_rhs(q, fields):
    import torch

    f = fields[0]
    psi = f["psi"][:12].copy()
    psi[5] = 2.0 * psi[3]  # a power of two: FP16 rounding commutes with it except in the subnormal range
    psi[7] = 0.0
    inp = dev(psi)
    out = torch.full_like(inp, float("nan"))
    f["G"].dslash_multi_tc(out, inp, 12, 0)
    got = host(out)
    assert np.array_equal(got[7], np.zeros_like(got[7]))
    assert rel(got[5], 2.0 * got[3]) < 1e-8
    assert rel(got[3], _expected(f, 3, 0)) < BAR


def test_multi_rhs_argument_checks(q, fields):
    import torch

    f = fields[0]
    inp = dev(f["psi"][:2])
    out = torch.empty_like(inp)
    with pytest.raises(RuntimeError):
        f["G"].dslash_multi_tc(out, inp, 129, 0)
    with pytest.raises(RuntimeError):
        f["G"].dslash_multi_tc(out, inp, 2, 2)
    with pytest.raises(RuntimeError):
        f["G"].dslash_multi_tc(out, inp, 0, 0)


def test_multi_rhs_timing_entry_points(q, fields):
    f = fields[2]
    ms = f["G"].dslash_multi_tc_time(64, 0, iters=3)
    assert 0.0 < ms < 1e3
    b = dev(np.stack([O.fermion_gauss(O.full_shape(f["latt"]), 5 + j) for j in range(4)]))
    x = dev(np.zeros((4,) + tuple(O.full_shape(f["latt"])), dtype=np.complex128))
    ms2, tune = q.batch_dslash_time([(f["G"], x, b, 0.12, False)], precision=32, gauge_precision=16, iters=3)
    assert 0.0 < ms2 < 1e3 and tune["dslash_threads"] in (32, 64, 128, 256)
