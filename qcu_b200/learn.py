"""Training the learned preconditioner on (residual, error) pairs.

Pairs come from the plain FP64 BiCGSTAB solver itself: for a seeded smooth
gauge field and Gaussian sources, the solution x* is computed to 1e-12, the
solver is re-run from zero for k iterations, and the odd-site error
e_k = x*_o - x_k,o together with its residual r_k = M_pc e_k form a pair.
Iterates of a Krylov solver concentrate their error in the slowly
converging (low) modes, which is what a preconditioner has to capture.
The network (qcu_b200.Network) is trained on these pairs with the
library's own forward/backward CUDA kernels and Adam.

    python -m qcu_b200.learn --latt 16 16 16 16 --kappa 0.1303 --out net.npy

Torch is used only to hold device buffers.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def make_pairs(G, kappa: float, n_src: int, checkpoints, seed: int = 1, n_random: int = -1, clover: bool = False):
    """Returns (r, e): complex64 tensors [pairs, Vh, 4, 3] on the GPU.

    Solver-iterate errors concentrate on the low modes; on their own they
    teach the network to amplify, which hurts on the rough part of a
    residual.  n_random pairs with white-noise errors (default: as many as
    the solver pairs) make the loss also cover |N M - 1| on every mode.
    clover: pairs of the clover operator (G must carry a clover term)."""
    import torch

    import qcu_b200 as q

    L = q.Layout(tuple(G.latt))
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    xs = torch.empty_like(b)
    xk = torch.empty_like(b)
    e = torch.empty(L.half, dtype=torch.complex128, device="cuda")
    r = torch.empty_like(e)
    rs, es = [], []
    for i in range(n_src):
        q.fermion_random(b, b.numel(), 0, seed + i)
        info = G.invert(xs, b, kappa, tol=1e-12, maxiter=20000, precision=64, delta=0.0, clover=clover)
        if info["status"] != 1:
            raise RuntimeError(f"training solve failed: {info}")
        for k in checkpoints:
            G.invert(xk, b, kappa, tol=1e-30, maxiter=int(k), precision=64, delta=0.0, clover=clover)
            e.copy_(xs[1] - xk[1])
            if float(torch.linalg.vector_norm(e)) == 0.0:
                continue  # the iterate is already the solution to the last bit
            G.matpc(r, e, kappa, clover=clover)
            rs.append(r.to(torch.complex64).clone())
            es.append(e.to(torch.complex64).clone())
    n_random = len(rs) if n_random < 0 else n_random
    for i in range(n_random):
        q.fermion_random(e, e.numel(), 0, seed + 100000 + i)
        G.matpc(r, e, kappa, clover=clover)
        rs.append(r.to(torch.complex64).clone())
        es.append(e.to(torch.complex64).clone())
    return torch.stack(rs), torch.stack(es)


def train(net, G, r, e, steps: int, batch: int = 16, lr: float = 3e-3, seed: int = 0, log_every: int = 0):
    """Adam on random mini-batches; returns the list of losses."""
    import torch

    gen = torch.Generator(device="cpu").manual_seed(seed)
    n = r.shape[0]
    losses = []
    for it in range(steps):
        idx = torch.randint(0, n, (batch,), generator=gen).cuda()
        rb = r[idx].to(torch.complex128).contiguous()
        eb = e[idx].to(torch.complex128).contiguous()
        loss, _ = net.train_step(G, rb, eb, batch, lr)
        losses.append(loss)
        if log_every and (it % log_every == 0 or it == steps - 1):
            print(f"step {it:5d}  loss {loss:.5f}", flush=True)
    return losses


def main():
    import torch

    import qcu_b200 as q

    ap = argparse.ArgumentParser()
    ap.add_argument("--latt", type=int, nargs=4, default=[16, 16, 16, 16])
    ap.add_argument("--eps", type=float, default=0.25)
    ap.add_argument("--kappa", type=float, default=0.1303)
    ap.add_argument("--csw", type=float, default=0.0, help="clover coefficient (0: Wilson)")
    ap.add_argument("--gauge-seed", type=int, default=4242)
    ap.add_argument("--sources", type=int, default=100)
    ap.add_argument("--checkpoints", type=int, nargs="+", default=[2, 4, 6, 8, 10, 12, 16, 20, 24, 28,
                                                                  32, 40, 48, 56, 64, 80, 96, 112, 128, 160])
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default="net.npy")
    args = ap.parse_args()
    L = q.Layout(tuple(args.latt))
    gauge = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(gauge, args.latt, 1, args.eps, args.gauge_seed)
    G = q.Gauge(gauge, args.latt, t_boundary=-1.0, clover_coeff=args.kappa * args.csw)
    t0 = time.time()
    r, e = make_pairs(G, args.kappa, args.sources, args.checkpoints, clover=args.csw != 0.0)
    print(f"{r.shape[0]} pairs in {time.time() - t0:.1f} s", flush=True)
    net = q.Network(seed=1, init_scale=0.01)
    t0 = time.time()
    losses = train(net, G, r, e, args.steps, args.batch, args.lr, log_every=100)
    print(f"trained {args.steps} steps in {time.time() - t0:.1f} s, final loss {np.mean(losses[-50:]):.5f}")
    np.save(args.out, net.get_weights())


if __name__ == "__main__":
    main()
