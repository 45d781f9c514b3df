"""GPU checks of the learned preconditioner: the CUDA forward and backward
kernels against the CPU oracle (oracle/nn_ref.py), training, and what the
trained network gains inside flexible GCR over the same method without it."""
import numpy as np
import pytest

import oracle as O
from oracle import nn_ref as R
from util import dev, empty_like_dev, host, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


def _random_weights(seed, scale=0.3):
    return np.random.default_rng(seed).normal(0, scale, R.N_W1 * 2 + R.N_W2 * 2).astype(np.float32)


@pytest.mark.parametrize("latt,t_bc", [([4, 4, 4, 8], -1.0), ([6, 4, 2, 4], 1.0)])
def test_forward_fma_matches_oracle(q, latt, t_bc):
    U = O.gauge_haar(latt, 5)
    r = O.fermion_gauss(O.half_shape(latt), 6)
    w = _random_weights(7)
    net = q.Network()
    net.set_weights(w)
    net.set_tensor_cores(False)
    with q.Gauge(dev(U), latt, t_boundary=t_bc) as G:
        out = empty_like_dev(O.half_shape(latt))
        net.apply(G, out, dev(r))
    lat = R.Lattice(U, latt, t_bc)
    ref, _, _ = R.forward(lat, R.bf16_round(w).astype(np.float64), r.reshape(1, lat.Vh, 4, 3))
    # the FMA layers: bf16 weights (rounded identically), FP32 links and FP32 arithmetic
    assert rel(host(out).reshape(ref.shape), ref) < 2e-5


@pytest.mark.parametrize("latt,t_bc", [([4, 4, 4, 8], -1.0), ([6, 4, 2, 4], 1.0), ([16, 16, 16, 32], -1.0)])
def test_forward_tensor_cores_match_oracle(q, latt, t_bc):
    """The tcgen05 layers (the default for inference): transported inputs
    rounded to bf16 as the MMA's A operand, bf16 weights, FP32 accumulation,
    the hidden field stored as bf16, 16-bit links.  Against the oracle that
    rounds the same operands: within 3e-3 (a value computed in FP32 from
    16-bit links here and in FP64 there can round to the neighbouring bf16
    value, one unit of 2^-8 relative, at each of the two roundings: the
    stored hidden field and the transported operand); against the unrounded
    network within the bf16 resolution.  16^3 x 32 has more 128-site tiles than resident CTAs, so
    the CTAs loop over tiles; 6x4x2x4 ends in a partial tile."""
    U = O.gauge_haar(latt, 5)
    r = O.fermion_gauss(O.half_shape(latt), 6)
    w = _random_weights(7)
    net = q.Network()
    net.set_weights(w)
    with q.Gauge(dev(U), latt, t_boundary=t_bc) as G:
        out = empty_like_dev(O.half_shape(latt))
        net.apply(G, out, dev(r))
        out2 = empty_like_dev(O.half_shape(latt))
        net.apply(G, out2, dev(r))
    got = host(out)
    assert np.array_equal(got, host(out2))  # deterministic
    lat = R.Lattice(U, latt, t_bc)
    wb = R.bf16_round(w).astype(np.float64)
    ref, _, _ = R.forward(lat, wb, r.reshape(1, lat.Vh, 4, 3), round_act=True)
    assert rel(got.reshape(ref.shape), ref) < 3e-3
    exact, _, _ = R.forward(lat, wb, r.reshape(1, lat.Vh, 4, 3))
    assert rel(got.reshape(exact.shape), exact) < 1e-2


def test_gradient_matches_oracle(q):
    latt = [4, 4, 2, 4]
    U = O.gauge_haar(latt, 8)
    B = 3
    r = O.fermion_gauss((B,) + O.half_shape(latt), 9)
    e = O.fermion_gauss((B,) + O.half_shape(latt), 10)
    w = _random_weights(11)
    net = q.Network()
    net.set_weights(w)
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        loss, grad = net.train_step(G, dev(r), dev(e), B, 0.0, want_grad=True)
    lat = R.Lattice(U, latt, -1.0)
    gref, lref = R.gradient(lat, w.astype(np.float64), r.reshape(B, lat.Vh, 4, 3), e.reshape(B, lat.Vh, 4, 3))
    assert abs(loss - lref) <= 1e-5 * lref
    assert rel(grad, gref) < 1e-4
    # lr = 0 leaves the weights untouched
    assert np.array_equal(net.get_weights(), w)


def test_training_helps_gcr(q):
    """Train on (residual, error) pairs from plain solves; the trained network
    as GCR preconditioner needs fewer outer steps than the untrained one."""
    import torch

    from qcu_b200 import learn

    latt = [8, 8, 8, 8]
    kappa = 0.124
    U = O.gauge_smooth(latt, 0.25, 12)
    with q.Gauge(dev(U), latt, t_boundary=-1.0) as G:
        r, e = learn.make_pairs(G, kappa, n_src=4, checkpoints=[2, 4, 8, 16, 32], seed=3)
        net = q.Network(seed=2, init_scale=0.01)
        losses = learn.train(net, G, r, e, steps=300, batch=8, lr=3e-3)
        assert np.mean(losses[-20:]) < 0.7 * np.mean(losses[:5])
        b = torch.from_numpy(O.fermion_gauss(O.full_shape(latt), 77)).cuda()
        x = empty_like_dev(O.full_shape(latt))
        plain = q.Network(seed=2, init_scale=0.0)  # exactly the identity: GCR without preconditioning
        i0 = G.invert(x, b, kappa, tol=1e-10, maxiter=4000, solver="gcr", precond=1, nn=plain, gcr_k=16)
        i1 = G.invert(x, b, kappa, tol=1e-10, maxiter=4000, solver="gcr", precond=1, nn=net, gcr_k=16)
        assert i0["status"] == 1 and i1["status"] == 1
        assert i1["true_residual"] <= 1e-10
        assert i1["reliable_updates"] < i0["reliable_updates"], (i0, i1)
        # and combined with the inner solver (precond 2) it converges as well
        i2 = G.invert(x, b, kappa, tol=1e-10, maxiter=4000, solver="gcr", precond=2, nn=net, precision=32,
                      inner_iters=16, gcr_k=8)
        assert i2["status"] == 1 and i2["true_residual"] <= 1e-10
