#!/usr/bin/env python
"""Benchmark of qcu's hot path on B200: even-odd preconditioned solves of the
Wilson (and clover) operator on a 32^3 x 64 lattice.

Workload (one "step" = one full solve):
  * lattice 32x32x32x64, antiperiodic in t, smooth SU(3) links
    U = exp(i eps H), eps = 0.25, reunitarised (seeded, generated on the GPU
    by the library's own generator);
  * source: complex normal N(0,1) per component (seeded);
  * kappa = 0.1303, as close to the critical point as plain FP64 BiCGSTAB
    still converges on this field (865-870 iterations; at 0.1304 it does not
    converge within 4000);
  * stop at a true relative residual ||b - M x|| / ||b|| <= 1e-10, recomputed
    in FP64 on the full two-parity system at the end of every solve.
Timed (`value`): the chosen solver -- FP64 flexible GCR(4) around an inner
BiCGSTAB on 16-bit fixed-point spinors and 16-bit links with FP32
arithmetic, run as one CUDA graph with a device-side WHILE loop per outer
step.  Reported beside it: plain FP64 BiCGSTAB on the same GPU (this source
and four more), the hopping-term bandwidth per storage and its roofline, the
end-to-end time through the C ABI from host buffers, the clover target
(32^3 x 64, csw 1, near-critical kappa), the 24^3 x 48 clover workload at
every storage precision with errors against the CPU oracle's FP64 solve, the
learned preconditioner, the batched multi-RHS solve, the two-level
multigrid (set-up, its own solve, and the chosen solver with its coarse-grid
correction), the multi-right-hand-side hopping term on the tcgen05 tensor
cores against the batched FMA kernel, and a CPU baseline (the FP64 CPU oracle on all host cores,
bounded sample).

`--impl reference` times one complete FP64 solve of the CPU restatement of
qcu's algorithm on the same system, measured, beside qcu's own GPU kernels
rebuilt for sm_100a (its wilson_dslash kernel time, a full dslashQcu call,
ncclBistabCgQcu).

Multi-GPU: the path does not shard in this implementation (replicas only):
every rank solves its own seeded system; the time is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LATT = [32, 32, 32, 64]
EPS = 0.25
T_BC = -1.0
GAUGE_SEED = 20251203
SRC_SEED = 7
KAPPA = 0.1303            # plain FP64 BiCGSTAB: 865-870 iterations on this ensemble (0.1304: no convergence in 4000)
TOL = 1e-10
CSW = 1.0
KAPPA_CLOVER = 0.1291     # clover csw = 1 on the same field: near-critical (plain FP64 ~1000 iterations)
METRIC = "solve s to 1e-10 true residual, chosen vs plain FP64, 1 B200; dslash HBM GB/s"
# algorithmic bytes per output site of the hopping term (in-spinor + 8 recon-12 links + out-spinor)
DSLASH_BYTES = {"64": 192 + 8 * 96 + 192, "32": 96 + 8 * 48 + 96, "16": 52 + 8 * 24 + 52, "32/16": 96 + 8 * 24 + 96}
DSLASH_FLOPS = 1320
# DRAM bytes (read + write) per launch of each dslash storage at 32^3 x 64 from
# one ncu capture each (profiles/k_dslash_*_32x32x32x64.txt)
DSLASH_TRAFFIC = {"16": {"bytes": 298_198_016, "profile": "profiles/k_dslash_soa16_gsoa16_32x32x32x64.txt"},
                  "32/16": {"bytes": 387_940_000, "profile": "profiles/k_dslash_soa32_gsoa16_32x32x32x64.txt"},
                  "64": {"bytes": 1_208_100_000, "profile": "profiles/k_dslash_soa64_32x32x32x64.txt"}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", type=int, default=16, choices=[16, 32, 64],
                    help="inner spinor precision of the chosen solver (16: 16-bit spinors and links)")
    ap.add_argument("--solver", default="gcr", choices=["gcr", "bicgstab"], help="chosen solver")
    ap.add_argument("--gauge-precision", type=int, default=None, choices=[0, 16],
                    help="16: FP32 spinors with 16-bit links (default 16 with --precision 32, else 0)")
    ap.add_argument("--inner-iters", type=int, default=96)
    ap.add_argument("--inner-tol", type=float, default=0.03)
    ap.add_argument("--gcr-k", type=int, default=4)
    ap.add_argument("--kappa", type=float, default=KAPPA)
    ap.add_argument("--latt", type=int, nargs=4, default=LATT)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the clover and batched measurements")
    args = ap.parse_args()
    if args.gauge_precision is None:
        args.gauge_precision = 16 if args.precision == 32 else 0
    return args


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            ident = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            ident = str(self.dev)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={ident}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(latt, kappa, gauge_np, b_np, plain_iters, budget_s=12.0):
    """FP64 CPU oracle (OpenMP, all host threads) on a bounded number of
    BiCGSTAB iterations of the same system, extrapolated to plain_iters."""
    import numpy as np

    import oracle as O

    threads = O.get_threads()
    bo = np.ascontiguousarray(b_np[1])
    t0 = time.perf_counter()
    O.bicgstab(bo, gauge_np, latt, kappa, t_bc=T_BC, tol=1e-30, maxiter=1)
    t1 = time.perf_counter() - t0
    n = max(2, min(50, int(budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    _, it, _ = O.bicgstab(bo, gauge_np, latt, kappa, t_bc=T_BC, tol=1e-30, maxiter=n)
    dt = time.perf_counter() - t0
    per_iter = dt / max(it, 1)
    return {"value": per_iter * plain_iters, "unit": "s", "cores": threads, "kind": "port",
            "sample": f"{it} FP64 BiCGSTAB iterations of the CPU oracle on {'x'.join(map(str, latt))} "
                      f"({dt:.1f} s, {per_iter:.3f} s/iteration), extrapolated to {plain_iters} iterations",
            "seconds_per_iteration": per_iter}


def cpu_dslash_medians(latt):
    """Median time of one FP64 hopping-term application of the CPU oracle on
    8^4 and on `latt`, with 1 host thread and with all of them."""
    import numpy as np

    import oracle as O

    out = {}
    nthreads = O.get_threads()
    for lt in ([8, 8, 8, 8], list(latt)):
        U = O.gauge_smooth(lt, EPS, GAUGE_SEED)
        psi = O.fermion_gauss(O.half_shape(lt), SRC_SEED)
        rec = {}
        for th in (1, nthreads):
            O.set_threads(th)
            O.dslash(psi, U, lt, 0, T_BC)
            ts = []
            for _ in range(3 if lt[3] >= 32 else 9):
                t0 = time.perf_counter()
                O.dslash(psi, U, lt, 0, T_BC)
                ts.append(time.perf_counter() - t0)
            rec[f"threads_{th}"] = round(1e3 * float(np.median(ts)), 3)
        out["x".join(map(str, lt))] = rec
    O.set_threads(nthreads)
    return {"unit": "ms per application (FP64, one parity)", **out}


def reference_gpu(latt, U, psi):
    """qcu's own CUDA code, built from its sources for sm_100a
    (oracle/_ref/libqcu_ref.so), on this GPU, fed with the oracle's seeded
    fields through torch (this library is not loaded):
      * its hopping kernel wilson_dslash (src/wilson_dslash.cu:9-245) at
        `latt`, launched as qcu launches it and timed with CUDA events by
        oracle/ref_timer.cu, with its output checked against the oracle;
      * the full dslashQcu call (qcu's per-call set-up and in-place layout
        permutations included) at `latt`;
      * ncclBistabCgQcu (its fixed kappa 0.125 and absolute 1e-9 criterion) on
        16^3 x 32.
    qcu prints a line per dslash; its output is kept off this process's
    stdout.  None when the build or a GPU is absent."""
    import ctypes

    import numpy as np

    import oracle as O

    path = os.path.join(ROOT, "oracle", "_ref", "libqcu_ref.so")
    try:
        import torch

        if not (os.path.exists(path) and torch.cuda.is_available()):
            return None

        class Param(ctypes.Structure):
            _fields_ = [("lattice_size", ctypes.c_int * 4)]

        def param(v):
            p = Param()
            for i in range(4):
                p.lattice_size[i] = v[i]
            return p

        ref = ctypes.CDLL(path)
        Pp, vp = ctypes.POINTER(Param), ctypes.c_void_p
        ref.dslashQcu.argtypes = [vp, vp, vp, Pp, ctypes.c_int]
        ref.dslashQcu.restype = None
        ref.ncclBistabCgQcu.argtypes = [vp, vp, vp, Pp, Pp]
        ref.ncclBistabCgQcu.restype = None
        sys.stdout.flush()
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        try:
            out = {}
            tag = "x".join(map(str, latt))
            dU = torch.from_numpy(U).cuda()
            dpsi = torch.from_numpy(psi).cuda()
            o = torch.empty_like(dpsi)
            if hasattr(ref, "qcu_ref_wilson_dslash_timed"):  # the event-timing harness linked into the build
                tim = ref
                tim.qcu_ref_wilson_dslash_timed.argtypes = [vp, vp, vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                                            ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
                ms = ctypes.c_double(0)
                lat = (ctypes.c_int * 4)(*latt)
                rc = tim.qcu_ref_wilson_dslash_timed(o.data_ptr(), dpsi.data_ptr(), dU.data_ptr(), lat, 0, 20,
                                                     ctypes.byref(ms))
                if rc == 0:
                    oref = O.dslash(psi, U, latt, 0, 1.0)
                    err = float(np.linalg.norm(o.cpu().numpy() - oref) / np.linalg.norm(oref))
                    vh = O.vh(latt)
                    out["wilson_dslash_kernel"] = {
                        "lattice": tag, "ms": round(ms.value, 4), "launch": "qcu's own: blocks of 32, one site per thread",
                        "GBps_at_1152B_per_site": round(DSLASH_BYTES["64"] * vh / (ms.value * 1e-3) / 1e9, 1),
                        "rel_err_vs_oracle": err}
            par = param(latt)
            ref.dslashQcu(o.data_ptr(), dpsi.data_ptr(), dU.data_ptr(), ctypes.byref(par), 0)
            ts = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ref.dslashQcu(o.data_ptr(), dpsi.data_ptr(), dU.data_ptr(), ctypes.byref(par), 0)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            out["dslashQcu_call_ms_" + tag] = round(1e3 * min(ts), 2)
            del dU, dpsi, o
            small = [16, 16, 16, 32]
            dU = torch.from_numpy(O.gauge_smooth(small, EPS, GAUGE_SEED)).cuda()
            db = torch.from_numpy(O.fermion_gauss(O.full_shape(small), SRC_SEED)).cuda()
            x = torch.zeros_like(db)
            par, grid = param(small), param([1, 1, 1, 1])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ref.ncclBistabCgQcu(x.data_ptr(), db.data_ptr(), dU.data_ptr(), ctypes.byref(par), ctypes.byref(grid))
            torch.cuda.synchronize()
            out["ncclBistabCgQcu_s_16x16x16x32_kappa0.125"] = round(time.perf_counter() - t0, 4)
            return out
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)
    except Exception as e:  # the timing is informative; the arm's value is the CPU one
        return {"error": str(e)[:200]}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v, device=None):
    if pg is None:
        return v
    import torch

    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_full_solve(latt, kappa, U, b, tol=TOL):
    """One complete FP64 even-odd BiCGSTAB solve of the CPU oracle (qcu's
    algorithm, include/lattice_bistabcg.h:101-132,221-340; OpenMP on every
    host thread) to a true relative residual <= tol of the full system,
    recomputed with the oracle's FP64 operator; restarted from its own
    iterate with a tighter target if the iterated residual met the target
    but the true one did not.  Returns (seconds, iterations, true residual)."""
    import numpy as np

    import oracle as O

    t0 = time.perf_counter()
    nb = np.linalg.norm(b)
    x, its, t_in = None, 0, tol
    for _ in range(4):
        x, it, _ = O.solve_full(b, U, latt, kappa, x0=x, t_bc=T_BC, tol=t_in, maxiter=20000)
        its += it
        res = float(np.linalg.norm(b - O.mfull(x, U, latt, kappa, T_BC)) / nb)
        if res <= tol:
            break
        t_in *= 0.5 * tol / res
    return time.perf_counter() - t0, its, res


def run_reference(args, world, rank, pg):
    """Reference arm.  qcu's code for this path is GPU code only, with no CPU
    implementation, and its solver is fixed to kappa 0.125 and an absolute
    tolerance (include/define.h:67-69), so it cannot run this workload.  The
    arm therefore times the CPU restatement of qcu's algorithm (FP64 even-odd
    BiCGSTAB, OpenMP, all host threads) on the same system: ONE complete
    solve to a 1e-10 true residual, measured, not extrapolated.  A complete
    solve takes minutes, so it runs once whatever --steps says
    (cpu_solves_run).  Beside it: qcu's own GPU kernels rebuilt for sm_100a
    (reference_gpu), and the CPU oracle's hopping term."""
    if rank != 0:
        return
    import oracle as O

    latt = list(args.latt)
    U = O.gauge_smooth(latt, EPS, GAUGE_SEED)
    b = O.fermion_gauss(O.full_shape(latt), SRC_SEED)
    threads = O.get_threads()
    extra = {} if args.no_cpu else {"cpu_dslash": cpu_dslash_medians(latt)}
    rg = reference_gpu(latt, U, b[1]) if latt == LATT else None
    if rg is not None:
        extra["reference_gpu"] = rg
    if args.no_cpu:  # qcu's GPU timings only (profiling runs)
        print(json.dumps({"impl": "reference", "reference_gpu": rg}), flush=True)
        return
    secs, its, res = cpu_full_solve(latt, args.kappa, U, b)
    sample = (f"one complete FP64 BiCGSTAB solve of the CPU oracle on {'x'.join(map(str, latt))}, kappa {args.kappa}: "
              f"{its} iterations, true residual {res:.2e}, {secs:.1f} s on {threads} host threads (measured)")
    line = {"metric": METRIC, "value": round(secs, 3), "unit": "s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs * 1e3, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded smooth SU(3) gauge, Gaussian source)",
            "config": {"workload": "wilson-bicgstab-32^3x64-smooth-eps0.25", "latt": latt, "kappa": args.kappa,
                       "tol": TOL, "t_boundary": T_BC},
            "cpu_solves_run": 1,
            "note": ("value = one complete CPU solve, measured; it runs once (about 2.5 min), not --steps times, so "
                     "the arm ends within minutes"),
            "cpu_solve": {"seconds": round(secs, 3), "iterations": its, "true_residual": res},
            "cpu_baseline": {"value": round(secs, 3), "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": round(secs, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            **extra}
    print(json.dumps(line), flush=True)


def event_time(stream, fn):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


def clover_target(args, q, gauge, b, x, latt, stream, chosen_kw):
    """Clover csw = 1 at near-critical kappa on the same field: plain FP64
    BiCGSTAB vs the chosen solver (one timed solve each after a warm-up)."""
    with q.Gauge(gauge, latt, t_boundary=T_BC, clover_coeff=KAPPA_CLOVER * CSW) as G:
        def solve(**kw):
            info = G.invert(x, b, KAPPA_CLOVER, tol=TOL, maxiter=20000, clover=True, **kw)
            if info["status"] != 1 or info["true_residual"] > TOL:
                raise RuntimeError(f"clover solve failed: {info}")
            return info
        solve(**chosen_kw)
        tp, ip = event_time(stream, lambda: solve(precision=64, delta=0.0))
        tc, ic = event_time(stream, lambda: solve(**chosen_kw))
    return {"workload": f"wilson-clover-csw{CSW}-32^3x64-smooth-eps0.25", "kappa": KAPPA_CLOVER,
            "plain_fp64": {"seconds": round(tp, 4), "iterations": ip["iterations"],
                           "true_residual": ip["true_residual"]},
            "chosen": {"seconds": round(tc, 4), "iterations": ic["iterations"], "outer_steps": ic["reliable_updates"],
                       "true_residual": ic["true_residual"]},
            "speedup_vs_plain_fp64": round(tp / tc, 3)}


def multigrid_block(args, q, G, b, x, stream, chosen_kw):
    """Two-level multigrid on the benchmark system (Wilson, kappa 0.1303):
    set-up (12 near-null vectors from 200 FP32 BiCGSTAB iterations each, 4^4
    aggregates), then one timed solve to the same 1e-10 true residual with
    the multigrid alone (FP64 flexible GCR around the two-level cycle) and
    one with the chosen solver whose GCR step first applies the coarse-grid
    correction (precond 3); each after a warm-up solve."""
    mg = q.Multigrid(G, args.kappa, n_vec=12, setup_maxiter=200, nu_post=4, coarse_tol=0.05, coarse_maxiter=50)
    try:
        def mg_solve():
            info = mg.invert(x, b, tol=TOL, maxiter=1000)
            if info["status"] != 1 or info["true_residual"] > TOL:
                raise RuntimeError(f"multigrid solve failed: {info}")
            return info
        def pc_solve():
            info = G.invert(x, b, args.kappa, tol=TOL, maxiter=20000, **{**chosen_kw, "solver": "gcr"}, precond=3, mg=mg)
            if info["status"] != 1 or info["true_residual"] > TOL:
                raise RuntimeError(f"coarse-corrected solve failed: {info}")
            return info
        mg_solve()
        tm, im = event_time(stream, mg_solve)
        pc_solve()
        tp, ip = event_time(stream, pc_solve)
        orth, gal = mg.check()
        return {"workload": "wilson-bicgstab-32^3x64-smooth-eps0.25", "kappa": args.kappa,
                "params": {"geo_block_size": [4, 4, 4, 4], "n_vec": 12, "setup_maxiter": 200, "nu_pre": 0,
                           "nu_post": 4, "coarse_tol": 0.05, "coarse_maxiter": 50, "gcr_k": 8},
                "setup_seconds": round(mg.setup_seconds, 3), "orthonormality_err": orth, "galerkin_err": gal,
                "mg_solve": {"seconds": round(tm, 4), "outer_steps": im["outer"], "coarse_iterations": im["coarse_iters"],
                             "true_residual": im["true_residual"]},
                "chosen_with_coarse_correction": {"seconds": round(tp, 4), "iterations": ip["iterations"],
                                                  "outer_steps": ip["reliable_updates"],
                                                  "true_residual": ip["true_residual"]}}
    finally:
        mg.close()


def multi_rhs_tc_block(q, G, latt):
    """The multi-right-hand-side hopping term on the tcgen05 tensor cores
    (FP16 operands, FP32 accumulation) on the benchmark gauge field, 64 and 128
    right-hand sides, against the batched FMA kernel (autotuned shape, FP32
    spinors with 16-bit links and 16-bit spinors) on the same 64 right-hand
    sides of a 16^3 x 32 system, where the FMA batch fits in memory; device
    time per application with CUDA events, and per right-hand-side site."""
    import torch

    vh = latt[0] * latt[1] * latt[2] * latt[3] // 2
    out = {"operator": "D_{0<-1} on nrhs half spinors", "lattice": "x".join(map(str, latt)), "rows": []}
    for n in (64, 128):
        ms = G.dslash_multi_tc_time(n, 0, iters=10)
        out["rows"].append({"nrhs": n, "tc_ms": round(ms, 4), "tc_ps_per_rhs_site": round(ms * 1e9 / (vh * n), 2)})
    small = [16, 16, 16, 32]
    Ls = q.Layout(tuple(small))
    us = torch.empty(Ls.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(us, small, 1, 0.25, 5)
    with q.Gauge(us, small, t_boundary=-1.0) as Gs:
        cmp = {"lattice": "16x16x16x32", "nrhs": 64}
        ms = Gs.dslash_multi_tc_time(64, 0, iters=10)
        cmp["tc_ps_per_rhs_site"] = round(ms * 1e9 / (Ls.vh * 64), 2)
        ms = Gs.dslash_multi_tc_time(128, 0, iters=10)
        cmp["tc_128rhs_ps_per_rhs_site"] = round(ms * 1e9 / (Ls.vh * 128), 2)
        bb = torch.empty((64,) + tuple(Ls.full), dtype=torch.complex128, device="cuda")
        q.fermion_random(bb, bb.numel(), 0, 11)
        xx = torch.zeros_like(bb)
        for name, prec, gp in (("fma_fp32_links16", 32, 16), ("fma_16bit", 16, 0)):
            ms, tune = q.batch_dslash_time([(Gs, xx, bb, 0.12, False)], precision=prec, gauge_precision=gp, iters=10)
            cmp[name + "_ps_per_rhs_site"] = round(ms * 1e9 / (Ls.vh * 64), 2)
            cmp[name + "_tune"] = tune
        del bb, xx
    del us
    torch.cuda.empty_cache()
    out["vs_batched_fma"] = cmp
    return out


def batch_config(args, q, stream, chosen_kw):
    """Batched multi-RHS workload: the 12 point sources of a propagator on
    32^3 x 64 clover (csw = 1) together with 4 Gaussian right-hand sides on
    each of 16^3 x 32, 24^3 x 48 and 32^3 x 64 (clover), one batched solve;
    against the same 24 systems solved one at a time by the chosen solver and
    by plain FP64 BiCGSTAB (one solve per system, times nrhs)."""
    import torch

    # both arms run the chosen solver's inner precision
    kw = {k: chosen_kw[k] for k in ("precision", "gauge_precision", "inner_iters", "inner_tol", "gcr_k")}
    systems, handles, plain, single = [], [], 0.0, 0.0
    shapes = [(LATT, "point12"), ([16, 16, 16, 32], 4), ([24, 24, 24, 48], 4), (LATT, 4)]
    try:
        for i, (lt, what) in enumerate(shapes):
            L = q.Layout(tuple(lt))
            u = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
            q.gauge_random(u, lt, 1, EPS, GAUGE_SEED + 11 * i)
            G = q.Gauge(u, lt, t_boundary=T_BC, clover_coeff=KAPPA_CLOVER * CSW)
            del u
            handles.append(G)
            if what == "point12":
                bb = q.point_sources(lt, [0, 0, 0, 0])
            else:
                bb = torch.empty((what,) + L.full, dtype=torch.complex128, device="cuda")
                q.fermion_random(bb, bb.numel(), 0, SRC_SEED + 100 + i)
            systems.append((G, torch.empty_like(bb), bb, KAPPA_CLOVER, True))
        torch.cuda.empty_cache()
        res, tune = q.invert_batch(systems, tol=TOL, maxiter=20000, **kw)  # autotune + allocation
        tb, (res, tune) = event_time(stream, lambda: q.invert_batch(systems, tol=TOL, maxiter=20000, **kw))
        for r in res:
            if r["status"] != 1 or r["true_residual"] > TOL:
                raise RuntimeError(f"batched solve failed: {r}")
        for G, x, bb, kappa, cl in systems:
            xs = torch.empty_like(bb[0])
            b0 = bb[0].contiguous()
            tp, ip = event_time(stream, lambda: G.invert(xs, b0, kappa, tol=TOL, maxiter=20000, precision=64,
                                                         delta=0.0, clover=True))
            plain += tp * bb.shape[0]
            for j in range(bb.shape[0]):
                bj = bb[j].contiguous()
                tj, _ = event_time(stream, lambda: G.invert(xs, bj, kappa, tol=TOL, maxiter=20000, clover=True,
                                                            solver="gcr", **kw))
                single += tj
    finally:
        for G in handles:
            G.close()
    return {"workload": "propagator (12 point sources) 32^3x64 + 4 rhs each on 16^3x32, 24^3x48, 32^3x64; "
                        f"clover csw {CSW}, kappa {KAPPA_CLOVER}",
            "inner": ({16: "16-bit spinors and links", 32: "FP32 spinors", 64: "FP64"}[kw["precision"]]
                      + (" / 16-bit links" if kw["gauge_precision"] == 16 else "") + " (both arms)"),
            "rhs": len(res), "seconds": round(tb, 4), "tune": tune,
            "iterations_max": max(r["iterations"] for r in res),
            "max_true_residual": max(r["true_residual"] for r in res),
            "one_at_a_time_seconds": round(single, 4),
            "plain_fp64_seconds_estimate": round(plain, 4),
            "speedup_vs_one_at_a_time": round(single / tb, 3),
            "speedup_vs_plain_fp64": round(plain / tb, 3)}


def legacy_calls(q, latt):
    """This library through qcu's own ABI, on the inputs reference_gpu gives
    qcu (same generators and seeds): a dslashQcu call at `latt` and
    ncclBistabCgQcu (kappa 0.125, absolute 1e-9) on 16^3 x 32, wall time of
    each synchronous call."""
    import torch

    out = {}
    L = q.Layout(tuple(latt))
    U = torch.empty(L.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(U, latt, 1, EPS, GAUGE_SEED)
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, SRC_SEED)
    psi = b[1].contiguous()
    o = torch.empty_like(psi)
    par = q.QcuParam(latt)
    q.dslashQcu(o, psi, U, par, 0)
    ts = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q.dslashQcu(o, psi, U, par, 0)
        ts.append(time.perf_counter() - t0)
    out["dslashQcu_call_ms_" + "x".join(map(str, latt))] = round(1e3 * min(ts), 3)
    del U, b, psi, o
    small = [16, 16, 16, 32]
    Ls = q.Layout(tuple(small))
    U = torch.empty(Ls.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(U, small, 1, EPS, GAUGE_SEED)
    b = torch.empty(Ls.full, dtype=torch.complex128, device="cuda")
    q.fermion_random(b, b.numel(), 0, SRC_SEED)
    x = torch.zeros_like(b)
    grid = q.QcuParam([1, 1, 1, 1])
    q.ncclBistabCgQcu(x, b, U, q.QcuParam(small), grid)
    ts = []
    for _ in range(3):  # the fastest of three calls, as for dslashQcu above
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q.ncclBistabCgQcu(x, b, U, q.QcuParam(small), grid)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    out["ncclBistabCgQcu_s_16x16x16x32_kappa0.125"] = round(min(ts), 4)
    return out


def sources_block(q, G, latt, kappa, stream, chosen_kw, n_src=4):
    """Plain FP64 BiCGSTAB and the chosen solver on n_src more Gaussian
    sources of the benchmark system (same field): one timed solve each (CUDA
    events), with the iteration counts, so the speed-up rests on more than
    one right-hand side of a near-critical system."""
    import statistics

    import torch

    L = q.Layout(tuple(latt))
    b = torch.empty(L.full, dtype=torch.complex128, device="cuda")
    x = torch.empty_like(b)
    rows = []
    for i in range(n_src):
        seed = SRC_SEED + 1000 + i
        q.fermion_random(b, b.numel(), 0, seed)
        tp, ip = event_time(stream, lambda: G.invert(x, b, kappa, tol=TOL, maxiter=20000, precision=64, delta=0.0))
        tc, ic = event_time(stream, lambda: G.invert(x, b, kappa, tol=TOL, maxiter=20000, **chosen_kw))
        rows.append({"source_seed": seed, "plain_fp64_s": round(tp, 4), "plain_iterations": ip["iterations"],
                     "plain_status": ip["status"], "chosen_s": round(tc, 4), "chosen_iterations": ic["iterations"],
                     "chosen_status": ic["status"], "chosen_true_residual": ic["true_residual"],
                     "speedup": round(tp / tc, 3)})
    sp = [r["speedup"] for r in rows]
    return {"sources": rows, "speedup_median": round(statistics.median(sp), 3),
            "speedup_min": round(min(sp), 3), "speedup_max": round(max(sp), 3),
            "plain_fp64_s_median": round(statistics.median(r["plain_fp64_s"] for r in rows), 4),
            "chosen_s_median": round(statistics.median(r["chosen_s"] for r in rows), 4)}


def clover_c3_block(q, stream):
    """The clover workload: 24^3 x 48, smooth links eps 0.3, csw 1, kappa
    0.125, Gaussian source.  Each storage precision's solve (one timed solve
    after a warm-up) with its solution's error against the FP64 CPU oracle's
    solve of the same system (OpenMP, to a 1e-11 true residual)."""
    import numpy as np
    import torch

    import oracle as O

    latt, eps, kappa = [24, 24, 24, 48], 0.3, 0.125
    U = O.gauge_smooth(latt, eps, GAUGE_SEED + 3)
    b = O.fermion_gauss(O.full_shape(latt), SRC_SEED + 3)
    A = [O.clover_build(U, latt, p, kappa * CSW) for p in (0, 1)]
    Ainv = [O.clover_invert(a) for a in A]
    t0 = time.perf_counter()
    xo, it_o, _ = O.solve_full(b, U, latt, kappa, t_bc=T_BC, Ainv_e=Ainv[0], Ainv_o=Ainv[1], tol=1e-11,
                               maxiter=20000)
    t_oracle = time.perf_counter() - t0
    res_o = float(np.linalg.norm(b - O.mfull(xo, U, latt, kappa, T_BC, True, A[0], A[1])) / np.linalg.norm(b))
    del A, Ainv
    gcr = dict(solver="gcr", inner_iters=96, inner_tol=0.03, gcr_k=4)
    methods = [("plain FP64 BiCGSTAB", dict(precision=64, delta=0.0)),
               ("BiCGSTAB FP32 storage, FP64 reliable updates", dict(precision=32, delta=0.1)),
               ("BiCGSTAB 16-bit storage, FP64 reliable updates", dict(precision=16, delta=0.1)),
               ("FP64 GCR, inner FP32 spinors / 16-bit links", dict(precision=32, gauge_precision=16, **gcr)),
               ("FP64 GCR, inner 16-bit spinors and links", dict(precision=16, **gcr))]
    dU, db = torch.from_numpy(U).cuda(), torch.from_numpy(b).cuda()
    x = torch.empty_like(db)
    xo_t = torch.from_numpy(xo).cuda()
    rows = []
    with q.Gauge(dU, latt, t_boundary=T_BC, clover_coeff=kappa * CSW) as G:
        del dU
        for name, kw in methods:
            G.invert(x, db, kappa, tol=TOL, maxiter=20000, clover=True, **kw)
            t, info = event_time(stream, lambda: G.invert(x, db, kappa, tol=TOL, maxiter=20000, clover=True, **kw))
            err = float(torch.linalg.vector_norm(x - xo_t) / torch.linalg.vector_norm(xo_t))
            rows.append({"method": name, "seconds": round(t, 4), "iterations": info["iterations"],
                         "status": info["status"], "true_residual": info["true_residual"],
                         "rel_err_vs_fp64_oracle_solve": err})
    return {"workload": f"wilson-clover-csw{CSW}-24^3x48-smooth-eps{eps}", "kappa": kappa,
            "oracle_solve": {"iterations": it_o, "true_residual": res_o, "seconds_cpu": round(t_oracle, 2),
                             "cores": O.get_threads()},
            "methods": rows}


def learned_block(q, stream, chosen_kw, gauge, b, latt):
    """The learned preconditioner: the network trained (by the library's own
    forward/backward kernels and Adam) on ~2000 (residual, error) pairs from
    plain FP64 clover solves on seeded 16^4 smooth fields (eps 0.25), then
    applied inside the FP64 flexible GCR on the 32^3 x 64 clover target at
    near-critical kappa (precond=2: network, then the inner BiCGSTAB on what
    it leaves); the chosen solver without it beside it, same system, on the
    benchmark source and three more seeded Gaussian sources (near the
    critical point one source's iteration count moves by ~10 % with any
    change of rounding, so the gain is reported per source and as the
    median)."""
    import torch

    from qcu_b200 import learn

    small = [16, 16, 16, 16]
    Ls = q.Layout(tuple(small))
    us = torch.empty(Ls.gauge, dtype=torch.complex128, device="cuda")
    q.gauge_random(us, small, 1, EPS, 4242)
    t0 = time.perf_counter()
    with q.Gauge(us, small, t_boundary=T_BC, clover_coeff=KAPPA_CLOVER * CSW) as Gs:
        r, e = learn.make_pairs(Gs, KAPPA_CLOVER, 48, [2, 4, 6, 8, 10, 12, 16, 20, 24, 28, 32, 40, 48, 56, 64, 80,
                                                     96, 112, 128, 160], clover=True)
        t_pairs = time.perf_counter() - t0
        net = q.Network(seed=1, init_scale=0.01)
        t0 = time.perf_counter()
        losses = learn.train(net, Gs, r, e, 1500, 16, 3e-3)
        t_train = time.perf_counter() - t0
    npairs = int(r.shape[0])
    del r, e, us
    x = torch.empty_like(b)
    per_source = []
    with q.Gauge(gauge, latt, t_boundary=T_BC, clover_coeff=KAPPA_CLOVER * CSW) as G:
        kw = dict(chosen_kw)
        kw["solver"] = "gcr"
        for seed in (None, 2001, 2002, 2003):
            src = b
            if seed is not None:
                src = torch.empty_like(b)
                q.fermion_random(src, src.numel(), 0, seed)
            G.invert(x, src, KAPPA_CLOVER, tol=TOL, maxiter=20000, clover=True, **kw)
            t_no, i_no = event_time(stream, lambda: G.invert(x, src, KAPPA_CLOVER, tol=TOL, maxiter=20000,
                                                               clover=True, **kw))
            G.invert(x, src, KAPPA_CLOVER, tol=TOL, maxiter=20000, clover=True, precond=2, nn=net, **kw)
            t_nn, i_nn = event_time(stream, lambda: G.invert(x, src, KAPPA_CLOVER, tol=TOL, maxiter=20000,
                                                               clover=True, precond=2, nn=net, **kw))
            if i_nn["true_residual"] > TOL or i_no["true_residual"] > TOL:
                raise RuntimeError(f"learned block: a solve missed the tolerance: {i_no}, {i_nn}")
            per_source.append({"source_seed": seed if seed is not None else "benchmark",
                               "without_s": round(t_no, 4), "without_iterations": i_no["iterations"],
                               "with_s": round(t_nn, 4), "with_iterations": i_nn["iterations"],
                               "fallback": i_nn["fallback"], "gain": round(t_no / t_nn, 3)})
            if seed is None:
                first = (t_no, i_no, t_nn, i_nn)
    net.close()
    t_no, i_no, t_nn, i_nn = first
    gains = sorted(p["gain"] for p in per_source)
    return {"training": {"lattice": "16^4 clover csw 1, eps 0.25", "pairs": npairs, "pair_seconds": round(t_pairs, 2),
                         "steps": 1500, "train_seconds": round(t_train, 2),
                         "loss_first": round(float(sum(losses[:50]) / 50), 5),
                         "loss_last": round(float(sum(losses[-50:]) / 50), 5)},
            "target": f"32^3x64 clover csw {CSW}, kappa {KAPPA_CLOVER}",
            "without_network": {"seconds": round(t_no, 4), "inner_iterations": i_no["iterations"],
                                "outer_steps": i_no["reliable_updates"], "true_residual": i_no["true_residual"]},
            "with_network": {"seconds": round(t_nn, 4), "inner_iterations": i_nn["iterations"],
                             "outer_steps": i_nn["reliable_updates"], "true_residual": i_nn["true_residual"],
                             "status": i_nn["status"], "fallback": i_nn["fallback"]},
            "gain": round(t_no / t_nn, 3),
            "sources": per_source,
            "gain_median": round((gains[1] + gains[2]) / 2, 3),
            "gain_total": round(sum(p["without_s"] for p in per_source) / sum(p["with_s"] for p in per_source), 3)}


def run_ours(args, world, rank, local, pg):
    import numpy as np
    import torch

    import qcu_b200 as q

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    latt = list(args.latt)
    L = q.Layout(tuple(latt))
    gauge = torch.empty(L.gauge, dtype=torch.complex128, device=dev)
    q.gauge_random(gauge, latt, 1, EPS, GAUGE_SEED + rank)
    b = torch.empty(L.full, dtype=torch.complex128, device=dev)
    q.fermion_random(b, b.numel(), 0, SRC_SEED + rank)
    x = torch.empty_like(b)
    G = q.Gauge(gauge, latt, t_boundary=T_BC)
    lib_stream = torch.cuda.ExternalStream(q.stream_handle(), device=dev)

    chosen_kw = dict(precision=args.precision, delta=0.1, solver=args.solver, inner_iters=args.inner_iters,
                     inner_tol=args.inner_tol, gcr_k=args.gcr_k, gauge_precision=args.gauge_precision)

    def timed_solve(**kw):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        info = G.invert(x, b, args.kappa, tol=TOL, maxiter=20000, **kw)
        e1.record(lib_stream)
        e1.synchronize()
        if info["status"] != 1 or info["true_residual"] > TOL:
            raise RuntimeError(f"solve failed: {info}")
        return e0.elapsed_time(e1) / 1e3, info

    # plain FP64 BiCGSTAB (reliable update only at the end = true-residual check)
    plain_t, plain_info = timed_solve(precision=64, delta=0.0)
    plain_t = min(plain_t, timed_solve(precision=64, delta=0.0)[0])
    x_plain = x.clone()  # the FP64 solution, to state the chosen solver's error against it
    # chosen solver: warm-up then K timed solves
    for _ in range(args.warmup):
        timed_solve(**chosen_kw)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = q.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    infos = []
    for _ in range(args.steps):
        infos.append(G.invert(x, b, args.kappa, tol=TOL, maxiter=20000, **chosen_kw))
    e1.record(lib_stream)
    e1.synchronize()
    torch.cuda.synchronize()
    launches = q.kernel_launches() - launches0
    clk = clocks.stop()
    total = e0.elapsed_time(e1) / 1e3
    for info in infos:
        if info["status"] != 1 or info["true_residual"] > TOL:
            raise RuntimeError(f"chosen solve failed: {info}")
    total = max_over_ranks(pg, total, dev)
    per_solve = total / args.steps
    x_err = float(torch.linalg.vector_norm(x - x_plain) / torch.linalg.vector_norm(x_plain))
    del x_plain

    # dslash bandwidth (CUDA events on the library stream)
    pk, pk_kind = peaks()
    vh = L.vh
    dsl = {}
    for key, (prec, gprec) in {"64": (64, 0), "32": (32, 0), "16": (16, 0), "32/16": (32, 16)}.items():
        ms = G.bench_dslash(prec, False, 50, gauge_precision=gprec)
        dsl[key] = {"ms": ms, "GBps": DSLASH_BYTES[key] * vh / (ms * 1e-3) / 1e9,
                    "TFLOPs": DSLASH_FLOPS * vh / (ms * 1e-3) / 1e12}
    key = f"{args.precision}/16" if args.gauge_precision == 16 else str(args.precision)
    dom = dsl[key]
    kname = {"64": "SOA64,GSOA64", "32": "SOA32,GSOA32", "16": "SOA16,GSOA16", "32/16": "SOA32,GSOA16"}[key]
    tr = DSLASH_TRAFFIC.get(key) if latt == LATT else None
    roofline = {"bound": "hbm", "achieved": round(dom["GBps"], 1), "peak": pk, "unit": "GB/s",
                "frac": round(dom["GBps"] / pk, 4), "traffic": tr["bytes"] if tr else None,
                "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                "traffic_source": tr["profile"] if tr else None,
                "algorithmic_bytes": DSLASH_BYTES[key] * vh,
                "kernel": f"k_dslash<{kname}> ({DSLASH_BYTES[key]} B/site x {vh} sites per launch)",
                "peak_kind": pk_kind}

    # end to end through the C ABI with host buffers: H2D gauge + b, load, solve, D2H x
    e2e = None
    if not args.no_e2e:
        hg = gauge.cpu().pin_memory()
        hb = b.cpu().pin_memory()
        hx = torch.empty(L.full, dtype=torch.complex128).pin_memory()
        dg = torch.empty_like(gauge)
        db = torch.empty_like(b)
        dx = torch.empty_like(b)
        times, phases, all_phases = [], None, []
        for i in range(3):
            torch.cuda.synchronize()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            s0.record()
            dg.copy_(hg, non_blocking=True)
            db.copy_(hb, non_blocking=True)
            ev[0].record()
            with q.Gauge(dg, latt, t_boundary=T_BC) as G2:
                ev[1].record()
                info = G2.invert(dx, db, args.kappa, tol=TOL, maxiter=20000, **chosen_kw)
                ev[2].record()
            hx.copy_(dx, non_blocking=True)
            s1.record()
            s1.synchronize()
            if info["status"] != 1:
                raise RuntimeError(f"e2e solve failed: {info}")
            if i > 0:
                t = s0.elapsed_time(s1) / 1e3
                ph = {"total": round(t, 4), "h2d": round(s0.elapsed_time(ev[0]) / 1e3, 4),
                      "gauge_load": round(ev[0].elapsed_time(ev[1]) / 1e3, 4),
                      "solve": round(ev[1].elapsed_time(ev[2]) / 1e3, 4),
                      "free_and_d2h": round(ev[2].elapsed_time(s1) / 1e3, 4), "iterations": info["iterations"]}
                phases = ph if not times or t < min(times) else phases
                all_phases.append(ph)
                times.append(t)
        e2e_t = max_over_ranks(pg, min(times), dev)
        e2e = {"value": round(e2e_t, 4), "unit": "s", "h2d_bytes_per_step": hg.numel() * 16 + hb.numel() * 16,
               "d2h_bytes_per_step": hx.numel() * 16, "samples_s": [round(t, 4) for t in times],
               "phases": phases, "all_phases": all_phases}

    extra = {}
    if not args.no_extra and latt == LATT:
        extra["legacy_abi"] = legacy_calls(q, latt)
        extra["more_sources"] = sources_block(q, G, latt, args.kappa, lib_stream, chosen_kw)
        extra["clover_target"] = clover_target(args, q, gauge, b, x, latt, lib_stream, chosen_kw)
        extra["clover_24x24x24x48"] = clover_c3_block(q, lib_stream)
        extra["learned"] = learned_block(q, lib_stream, chosen_kw, gauge, b, latt)
        extra["batch"] = batch_config(args, q, lib_stream, chosen_kw)
        extra["multigrid"] = multigrid_block(args, q, G, b, x, lib_stream, chosen_kw)
        extra["multi_rhs_tc"] = multi_rhs_tc_block(q, G, latt)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_sample(latt, args.kappa, gauge.cpu().numpy(), b.cpu().numpy(), plain_info["iterations"])
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu["dslash"] = cpu_dslash_medians(latt)

    if rank == 0:
        chosen = infos[-1]
        line = {
            "metric": METRIC, "value": round(per_solve, 4), "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(per_solve * 1e3, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ({64: "f64", 32: "f32 storage / f64 reductions",
                       16: "int16+norm spinor storage / int16 links / f32 math / f64 reductions"}[
                args.precision] + (" / int16 links" if args.gauge_precision == 16 else "") + " (outer FP64)"),
            "data": "synthetic (seeded smooth SU(3) gauge, Gaussian source)",
            "config": {"workload": "wilson-bicgstab-32^3x64-smooth-eps0.25", "latt": latt, "kappa": args.kappa,
                       "tol": TOL, "t_boundary": T_BC,
                       "solver": (f"FP64 flexible GCR({args.gcr_k}), inner BiCGSTAB {args.precision}-bit"
                                  f"{'/16-bit links' if args.gauge_precision == 16 or args.precision == 16 else ''} "
                                  f"x{args.inner_iters} "
                                  f"(inner tol {args.inner_tol})") if args.solver == "gcr" else
                                 f"BiCGSTAB {args.precision}-bit, FP64 reliable updates (delta 0.1)",
                       "parallelism": "replicas" if world > 1 else "single", "l2": "working set (GBs) larger than L2"},
            "chosen": {"iterations": chosen["iterations"], "outer_steps_or_updates": chosen["reliable_updates"],
                       "true_residual": chosen["true_residual"],
                       "solution_rel_diff_vs_plain_fp64": x_err},
            "plain_fp64": {"seconds": round(plain_t, 4), "iterations": plain_info["iterations"],
                           "true_residual": plain_info["true_residual"]},
            "speedup_vs_plain_fp64": round(plain_t / per_solve, 3),
            "dslash": {k: {"ms": round(v["ms"], 4), "GBps": round(v["GBps"], 1), "frac_of_peak": round(v["GBps"] / pk, 4),
                           "TFLOPs": round(v["TFLOPs"], 2)} for k, v in dsl.items()},
            "roofline": roofline,
            **extra,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    G.close()


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
