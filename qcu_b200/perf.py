"""Micro-benchmarks of the library's hot path, for timing and profiling.

    python -m qcu_b200.perf dslash --precision 32 --gauge-precision 16 --iters 5
    python -m qcu_b200.perf solve  --precision 32 --gauge-precision 16
    python -m qcu_b200.perf batch  --csw 1.0 --kappa 0.128
    python -m qcu_b200.perf precisions
    python -m qcu_b200.perf legacy --iters 20
    python -m qcu_b200.perf nn --iters 20
    python -m qcu_b200.perf mg --n-vec 12 --setup-maxiter 200

`dslash` applies the even-odd hopping term `iters` times (after 3 warm-up
launches) on a seeded smooth gauge field and prints the time per launch and
the bandwidth of the algorithmic bytes (input spinor, 8 reconstruct-12 links,
output spinor per site).  `solve` runs one solve of M x = b with the given
solver settings (--repeat N: N solves, the median of all but the first,
which includes graph capture) and prints the solver report and its wall time.  `batch`
solves, in one batched call, the 12 point sources of a propagator on the
main lattice together with 4 Gaussian right-hand sides on each of
16^3 x 32, 24^3 x 48 and a second gauge field of the main lattice, and
prints the batched wall time next to the same 24 systems solved one at a
time.  `legacy` calls dslashQcu (qcu's ABI: PyQuda-layout complex128
fields, one kernel per call) `iters` times and prints the wall time per
synchronous call.  `nn` applies the learned preconditioner's network
(random weights, scale 0.3) `iters` times on an odd half spinor and prints
the time per application with the tensor-core layers and with the FP32 FMA
layers.  `mg` sets up the two-level multigrid (--n-vec near-null vectors from
--setup-maxiter iterations, 4^4 aggregates, nu_post 4, coarse tolerance 0.05
with at most 50 iterations) and solves M x = b once with it, printing the
set-up time and the solver report.  `mrhs` times the multi-right-hand-side
tensor-core hopping kernel (tcgen05, FP16 operands) against the batched FMA
kernel (autotuned, FP32 spinors with 16-bit links and 16-bit spinors) on the
same --nrhs right-hand sides of one system (the FMA one up to 64).  `precisions` solves one system (default: the benchmark's) with plain
FP64 BiCGSTAB, BiCGSTAB with FP64 reliable updates at 32 and 16 bits, and
the FP64 GCR around 32- and 16-bit inner solves, and states each solution's
difference from the FP64 one.  Inputs are
generated on the GPU by the library's own generators; the working set of the
default 32^3 x 64 lattice is larger than L2.
"""
from __future__ import annotations

import argparse
import json
import time

# algorithmic bytes per output site of the hopping term, keyed by spinor/link precision
DSLASH_BYTES = {(64, 64): 1152, (32, 32): 576, (16, 16): 296, (32, 16): 384}


def _gauge(latt, eps, seed, t_bc, csw=0.0, kappa=0.0):
    import torch

    import qcu_b200 as q

    L = q.Layout(tuple(latt))
    u = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(u, latt, 1, eps, seed)
    G = q.Gauge(u, latt, t_boundary=t_bc, clover_coeff=kappa * csw)
    return G, u, L


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["dslash", "solve", "batch", "precisions", "legacy", "nn", "mg", "mrhs"])
    ap.add_argument("--nrhs", type=int, nargs="+", default=[12, 48, 64, 128], help="mrhs: right-hand-side counts")
    ap.add_argument("--no-fma", action="store_true", help="mrhs: only the tensor-core kernel")
    ap.add_argument("--n-vec", type=int, default=12)
    ap.add_argument("--setup-maxiter", type=int, default=200)
    ap.add_argument("--latt", type=int, nargs=4, default=[32, 32, 32, 64])
    ap.add_argument("--eps", type=float, default=0.25)
    ap.add_argument("--seed", type=int, default=20251203)
    ap.add_argument("--t-bc", type=float, default=-1.0)
    ap.add_argument("--precision", type=int, default=32, choices=[16, 32, 64])
    ap.add_argument("--gauge-precision", type=int, default=16, choices=[0, 16])
    ap.add_argument("--clover", action="store_true", help="dslash: apply the inverse clover term too")
    ap.add_argument("--csw", type=float, default=0.0)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--repeat", type=int, default=1, help="solve: solves to time (median of all but the first)")
    ap.add_argument("--src-seed", type=int, default=7, help="solve: seed of the Gaussian source")
    ap.add_argument("--kappa", type=float, default=0.1303)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--solver", default="gcr", choices=["gcr", "bicgstab"])
    ap.add_argument("--inner-iters", type=int, default=96)
    ap.add_argument("--inner-tol", type=float, default=0.03)
    ap.add_argument("--gcr-k", type=int, default=4)
    ap.add_argument("--single", action="store_true", help="batch: also time the 24 systems one at a time")
    ap.add_argument("--only-point", action="store_true", help="batch: only the 12 point sources on --latt")
    a = ap.parse_args(argv)
    import torch

    import qcu_b200 as q

    gp = a.gauge_precision if a.gauge_precision else a.precision
    if a.what == "dslash":
        G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw if a.clover else 0.0, a.kappa)
        del u
        torch.cuda.empty_cache()
        ms = G.bench_dslash(a.precision, a.clover, a.iters, gauge_precision=a.gauge_precision)
        nb = DSLASH_BYTES[(a.precision, gp)] * L.vh
        print(json.dumps({"kernel": "dslash", "latt": a.latt, "precision": a.precision, "gauge_precision": gp,
                          "clover": a.clover, "ms": round(ms, 5), "bytes": nb,
                          "GBps": round(nb / (ms * 1e-3) / 1e9, 1)}))
        G.close()
        return
    if a.what == "batch":
        _batch(a)
        return
    if a.what == "nn":
        import numpy as np

        G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw, a.kappa)
        del u
        r = torch.empty(L.half, dtype=torch.complex128, device="cuda")
        q.fermion_random(r, r.numel(), 0, 7)
        out = torch.empty_like(r)
        net = q.Network(seed=1)
        w = np.random.default_rng(3).normal(0, 0.3, q.Network.num_params()).astype(np.float32)
        net.set_weights(w)
        stream = torch.cuda.ExternalStream(q.stream_handle())
        res = {"kernel": "nn", "latt": a.latt}
        for name, on in (("tensor_cores", True), ("fma", False)):
            net.set_tensor_cores(on)
            for _ in range(2):
                net.apply(G, out, r)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(a.iters):
                net.apply(G, out, r)
            e1.record(stream)
            e1.synchronize()
            res[name + "_ms_per_apply"] = round(e0.elapsed_time(e1) / a.iters, 4)
        print(json.dumps(res))
        net.close()
        G.close()
        return
    if a.what == "mrhs":
        _mrhs(a)
        return
    if a.what == "mg":
        G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw, a.kappa)
        del u
        b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
        q.fermion_random(b, b.numel(), 0, 7)
        x = torch.empty_like(b)
        mg = q.Multigrid(G, a.kappa, n_vec=a.n_vec, setup_maxiter=a.setup_maxiter, nu_post=4, coarse_tol=0.05,
                         coarse_maxiter=50)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = mg.invert(x, b, tol=a.tol, maxiter=1000)
        torch.cuda.synchronize()
        print(json.dumps({"kernel": "mg", "latt": a.latt, "kappa": a.kappa, "setup_s": round(mg.setup_seconds, 3),
                          "solve_s": round(time.perf_counter() - t0, 4), **info}))
        mg.close()
        G.close()
        return
    if a.what == "legacy":
        L = q.Layout(tuple(a.latt))
        u = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
        q.gauge_random(u, a.latt, 1, a.eps, a.seed)
        psi = torch.empty(L.half, dtype=torch.complex128, device="cuda")
        q.fermion_random(psi, psi.numel(), 0, 7)
        out = torch.empty_like(psi)
        par = q.QcuParam(a.latt)
        for i in range(3):
            q.dslashQcu(out, psi, u, par, i & 1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(a.iters):
            q.dslashQcu(out, psi, u, par, i & 1)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / a.iters
        print(json.dumps({"call": "dslashQcu", "latt": a.latt, "ms_per_call": round(ms, 4),
                          "GBps_at_1152B_per_site": round(1152 * L.vh / (ms * 1e-3) / 1e9, 1)}))
        return
    if a.what == "precisions":
        _precisions(a)
        return
    G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw, a.kappa)
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, a.src_seed)
    x = torch.empty_like(b)
    times = []
    for _ in range(max(1, a.repeat)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = G.invert(x, b, a.kappa, tol=a.tol, maxiter=20000, precision=a.precision,
                        gauge_precision=a.gauge_precision, solver=a.solver, inner_iters=a.inner_iters,
                        inner_tol=a.inner_tol, gcr_k=a.gcr_k, clover=a.csw != 0.0)
        torch.cuda.synchronize()
        times.append(round(time.perf_counter() - t0, 4))
    info["seconds"] = times[0] if len(times) == 1 else sorted(times[1:])[(len(times) - 1) // 2]
    if len(times) > 1:
        info["seconds_each"] = times  # the first includes graph capture; the median is of the others
    print(json.dumps(info))
    G.close()


def _mrhs(a):
    """The multi-rhs hopping term: the tcgen05 kernel against the batched FMA
    kernel (autotuned: sites per block, rhs per thread, the mma.sync path) on
    the same right-hand sides of one system, per application and per
    right-hand-side site."""
    import torch

    import qcu_b200 as q

    G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc)
    del u
    res = {"kernel": "mrhs", "latt": a.latt, "vh": L.vh, "rows": []}
    for n in a.nrhs:
        row = {"nrhs": n}
        ms = G.dslash_multi_tc_time(n, 0, iters=a.iters)
        # algorithmic bytes: FP16 in and out (48 B each per rhs-site) + 8 16-bit links per site
        byts = L.vh * (96 * n + 8 * 24)
        row["tc"] = {"ms": round(ms, 4), "ps_per_rhs_site": round(ms * 1e9 / (L.vh * n), 2),
                     "GBps": round(byts / (ms * 1e-3) / 1e9, 1)}
        if n <= 64 and not a.no_fma:
            b = torch.empty((n,) + tuple(L.full), dtype=torch.complex128, device="cuda")
            q.fermion_random(b, b.numel(), 0, 11)
            x = torch.zeros_like(b)
            for name, prec, gp in (("fma_fp32_links16", 32, 16), ("fma_16bit", 16, 0)):
                ms2, tune = q.batch_dslash_time([(G, x, b, 0.12, False)], precision=prec, gauge_precision=gp,
                                                iters=a.iters)
                row[name] = {"ms": round(ms2, 4), "ps_per_rhs_site": round(ms2 * 1e9 / (L.vh * n), 2), "tune": tune}
            del b, x
            torch.cuda.empty_cache()
        res["rows"].append(row)
    print(json.dumps(res))
    G.close()


def _precisions(a):
    """The storage precisions on one system: plain FP64 BiCGSTAB, BiCGSTAB
    with FP64 reliable updates at 32 and 16 bits, and the FP64 GCR around
    32- and 16-bit inner solves; per method the time of one solve after a
    warm-up one (CUDA events on the library stream), the iterations, the FP64
    true residual and the solution's relative difference from the FP64 one."""
    import torch

    import qcu_b200 as q

    G, u, L = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw, a.kappa)
    del u
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, 7)
    stream = torch.cuda.ExternalStream(q.stream_handle())
    gcr = dict(solver="gcr", inner_iters=a.inner_iters, inner_tol=a.inner_tol, gcr_k=a.gcr_k)
    methods = [("plain FP64 BiCGSTAB", dict(precision=64, delta=0.0)),
               ("BiCGSTAB FP32, FP64 reliable updates", dict(precision=32, delta=0.1)),
               ("BiCGSTAB 16-bit, FP64 reliable updates", dict(precision=16, delta=0.1)),
               ("FP64 GCR, inner FP32 / 16-bit links", dict(precision=32, gauge_precision=16, **gcr)),
               ("FP64 GCR, inner 16-bit", dict(precision=16, **gcr))]
    x64 = None
    for name, kw in methods:
        x = torch.empty_like(b)
        G.invert(x, b, a.kappa, tol=a.tol, maxiter=20000, clover=a.csw != 0.0, **kw)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = G.invert(x, b, a.kappa, tol=a.tol, maxiter=20000, clover=a.csw != 0.0, **kw)
        e1.record(stream)
        e1.synchronize()
        if x64 is None:
            x64 = x.clone()
        diff = float(torch.linalg.vector_norm(x - x64) / torch.linalg.vector_norm(x64))
        print(json.dumps({"method": name, "seconds": round(e0.elapsed_time(e1) / 1e3, 4),
                          "iterations": info["iterations"], "status": info["status"],
                          "true_residual": info["true_residual"], "rel_diff_vs_fp64": diff}))
    G.close()


def _batch(a):
    import torch

    import qcu_b200 as q

    kw = dict(tol=a.tol, maxiter=20000, precision=a.precision, gauge_precision=a.gauge_precision,
              inner_iters=a.inner_iters, inner_tol=a.inner_tol, gcr_k=a.gcr_k)
    clov = a.csw != 0.0
    systems, handles = [], []
    G0, u, L0 = _gauge(a.latt, a.eps, a.seed, a.t_bc, a.csw, a.kappa)
    del u
    handles.append(G0)
    b0 = q.point_sources(a.latt, [0, 0, 0, 0])
    systems.append((G0, torch.empty_like(b0), b0, a.kappa, clov))
    for i, latt in enumerate([] if a.only_point else [[16, 16, 16, 32], [24, 24, 24, 48], list(a.latt)]):
        G, u, L = _gauge(latt, a.eps, a.seed + 1 + i, a.t_bc, a.csw, a.kappa)
        del u
        handles.append(G)
        b = torch.empty((4,) + L.full, dtype=torch.complex128, device="cuda")
        q.fermion_random(b, b.numel(), 0, 100 + i)
        systems.append((G, torch.empty_like(b), b, a.kappa, clov))
    torch.cuda.empty_cache()
    q.invert_batch(systems, **kw)  # first call of this shape: autotune, allocation
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res, tune = q.invert_batch(systems, **kw)
    torch.cuda.synchronize()
    tb = time.perf_counter() - t0
    out = {"kernel": "batch", "rhs": len(res), "seconds": round(tb, 4), "tune": tune,
           "iterations": [r["iterations"] for r in res], "status": sorted(set(r["status"] for r in res)),
           "max_true_residual": max(r["true_residual"] for r in res)}
    if a.single:
        ts, it = 0.0, []
        for G, x, b, kappa, cl in systems:
            for j in range(b.shape[0]):
                xj = torch.empty_like(b[j])
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                info = G.invert(xj, b[j].contiguous(), kappa, clover=cl, solver="gcr", **kw)
                torch.cuda.synchronize()
                ts += time.perf_counter() - t0
                it.append(info["iterations"])
        out["single_seconds"] = round(ts, 4)
        out["single_iterations"] = it
    print(json.dumps(out))
    for G in handles:
        G.close()


if __name__ == "__main__":
    main()
