"""qcu_b200 -- B200-native implementation of qcu's fermion-matrix hot path.

The product is the shared library ``libqcu.so`` next to this file: sm_100a
CUDA kernels and C++ host code behind qcu's own C ABI (``include/qcu.h``) and
an additive extension ABI (``include/qcu_ext.h``).  This module is the Python
host side.  Its legacy half mirrors PyQuda's ``pyquda.pyqcu`` binding
(python/PyQuda/pyquda/src/pyqcu.pyx:1-34): a ``QcuParam`` with a
``lattice_size`` attribute and the six ``*Qcu`` functions taking device
pointers (anything with a ``.ptr`` attribute, an ``int`` address, or a CUDA
torch tensor).  The extension half wraps ``qcu_ext.h``.

There is no CPU fallback: importing this module raises if the library is
missing, and every call goes to the GPU.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqcu.so")


def build(jobs: int = 8) -> str:
    """Compile libqcu.so for sm_100a (nvcc cross-compiles; no GPU needed)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE, f"-j{jobs}"], check=True)
    return LIB_PATH


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}` (no CPU fallback exists)")

_lib = ctypes.CDLL(LIB_PATH)
_vp = ctypes.c_void_p


class QcuParam(ctypes.Structure):
    """``QcuParam`` of include/qcu.h:17-19: ``lattice_size`` is [Lx, Ly, Lz, Lt]."""

    _fields_ = [("_size", ctypes.c_int * 4)]

    def __init__(self, lattice_size=None):
        super().__init__()
        if lattice_size is not None:
            self.lattice_size = lattice_size

    @property
    def lattice_size(self):
        return list(self._size)

    @lattice_size.setter
    def lattice_size(self, value):
        v = [int(x) for x in value]
        if len(v) != 4:
            raise ValueError("lattice_size needs 4 entries")
        for i in range(4):
            self._size[i] = v[i]


class QcuInvertParam(ctypes.Structure):
    _fields_ = [
        ("kappa", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("maxiter", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("delta", ctypes.c_double),
        ("abs_tol", ctypes.c_int),
        ("x0_mode", ctypes.c_int),
        ("x0_seed", ctypes.c_ulonglong),
        ("use_clover", ctypes.c_int),
        ("chunk", ctypes.c_int),
        ("solver", ctypes.c_int),
        ("inner_iters", ctypes.c_int),
        ("inner_tol", ctypes.c_double),
        ("gcr_k", ctypes.c_int),
        ("gauge_precision", ctypes.c_int),
        ("precond", ctypes.c_int),
        ("nn", ctypes.c_void_p),
        ("mg", ctypes.c_void_p),
    ]


class QcuInvertResult(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("reliable_updates", ctypes.c_int),
        ("status", ctypes.c_int),
        ("restarts", ctypes.c_int),
        ("true_residual", ctypes.c_double),
        ("iter_residual2", ctypes.c_double),
        ("seconds", ctypes.c_double),
        ("fallback", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class QcuBatchSystem(ctypes.Structure):
    _fields_ = [
        ("gauge", ctypes.c_void_p),
        ("nrhs", ctypes.c_int),
        ("kappa", ctypes.c_double),
        ("use_clover", ctypes.c_int),
        ("x", ctypes.c_void_p),
        ("b", ctypes.c_void_p),
    ]


class QcuMGParam(ctypes.Structure):
    _fields_ = [
        ("geo_block_size", ctypes.c_int * 4),
        ("n_vec", ctypes.c_int),
        ("setup_maxiter", ctypes.c_int),
        ("coarse_tol", ctypes.c_double),
        ("coarse_maxiter", ctypes.c_int),
        ("nu_pre", ctypes.c_int),
        ("nu_post", ctypes.c_int),
        ("gcr_k", ctypes.c_int),
    ]


class QcuMGResult(ctypes.Structure):
    _fields_ = [
        ("outer", ctypes.c_int),
        ("coarse_iters", ctypes.c_int),
        ("status", ctypes.c_int),
        ("true_residual", ctypes.c_double),
        ("seconds", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class QcuBatchTune(ctypes.Structure):
    _fields_ = [("dslash_threads", ctypes.c_int), ("dslash_rhs", ctypes.c_int), ("blas_sites", ctypes.c_int),
                ("mma", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.POINTER(QcuParam)
for _name in ("dslashQcu", "dslashCloverQcu"):
    getattr(_lib, _name).argtypes = [_vp, _vp, _vp, _P, ctypes.c_int]
    getattr(_lib, _name).restype = None
_lib.mpiDslashQcu.argtypes = [_vp, _vp, _vp, _P, ctypes.c_int, _P]
_lib.mpiBistabCgQcu.argtypes = [_vp, _P, _P]
_lib.ncclDslashQcu.argtypes = [_vp, _vp, _vp, _P, ctypes.c_int, _P]
_lib.ncclBistabCgQcu.argtypes = [_vp, _vp, _vp, _P, _P]
for _name in ("mpiDslashQcu", "mpiBistabCgQcu", "ncclDslashQcu", "ncclBistabCgQcu"):
    getattr(_lib, _name).restype = None
_lib.qcuGetLastError.argtypes = [ctypes.c_char_p, ctypes.c_int]
_lib.qcuGetLastError.restype = ctypes.c_int
_lib.qcuGaugeLoad.argtypes = [ctypes.POINTER(_vp), _vp, ctypes.POINTER(ctypes.c_int), ctypes.c_double, ctypes.c_double]
_lib.qcuGaugeFree.argtypes = [_vp]
_lib.qcuDslash.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
_lib.qcuMatPC.argtypes = [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int]
_lib.qcuMat.argtypes = [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int]
_lib.qcuInvertParamDefault.argtypes = [ctypes.POINTER(QcuInvertParam)]
_lib.qcuInvertParamDefault.restype = None
_lib.qcuInvert.argtypes = [_vp, _vp, _vp, ctypes.POINTER(QcuInvertParam), ctypes.POINTER(QcuInvertResult)]
_lib.qcuInvertBatch.argtypes = [ctypes.POINTER(QcuBatchSystem), ctypes.c_int, ctypes.POINTER(QcuInvertParam),
                                ctypes.POINTER(QcuInvertResult), ctypes.POINTER(QcuBatchTune)]
_lib.qcuBatchDslashTime.argtypes = [ctypes.POINTER(QcuBatchSystem), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
_lib.qcuDslashMultiTC.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
_lib.qcuDslashMultiTCTime.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
_lib.qcuBatchApplyMatPC.argtypes = [ctypes.POINTER(QcuBatchSystem), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(QcuBatchTune), ctypes.c_void_p]
_ip = ctypes.POINTER(ctypes.c_int)
_lib.qcuCommUniqueId.argtypes = [ctypes.c_void_p]
_lib.qcuCommInit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
_lib.qcuDDPlan.argtypes = [_ip, _ip, ctypes.c_int, _ip]
_lib.qcuDDSchedule.argtypes = [_ip, _ip, ctypes.c_int, _ip, _ip]
_lib.qcuDslashDDEmulate.argtypes = [_vp, _vp, _vp, _ip, ctypes.c_int, _ip]
_lib.qcuBistabCgDDEmulate.argtypes = [_vp, _vp, _vp, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_double)]
_lib.qcuGaugeRandom.argtypes = [_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong]
_lib.qcuFermionRandom.argtypes = [_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_ulonglong]
_lib.qcuGetStream.restype = _vp
_lib.dslashCloverQcuNoAlloc.argtypes = [_vp, _vp, _vp, _P, ctypes.c_int]
_lib.dslashCloverQcuNoAlloc.restype = ctypes.c_int
_lib.qcuNoAllocMaxSites.restype = ctypes.c_int
_lib.qcuKernelLaunches.restype = ctypes.c_longlong
_lib.qcuNNCreate.argtypes = [ctypes.POINTER(_vp), ctypes.c_ulonglong, ctypes.c_double]
_lib.qcuNNFree.argtypes = [_vp]
_lib.qcuNNNumParams.restype = ctypes.c_int
_lib.qcuNNGetWeights.argtypes = [_vp, ctypes.c_void_p]
_lib.qcuNNSetWeights.argtypes = [_vp, ctypes.c_void_p]
_lib.qcuNNApply.argtypes = [_vp, _vp, _vp, _vp]
_lib.qcuNNSetTensorCores.argtypes = [_vp, ctypes.c_int]
_lib.qcuNNTrainStep.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                ctypes.c_void_p]
_lib.qcuMGParamDefault.argtypes = [ctypes.POINTER(QcuMGParam)]
_lib.qcuMGParamDefault.restype = None
_lib.qcuMGCreate.argtypes = [ctypes.POINTER(_vp), _vp, ctypes.c_double, ctypes.POINTER(QcuMGParam),
                             ctypes.POINTER(ctypes.c_double)]
_lib.qcuMGFree.argtypes = [_vp]
_lib.qcuMGInvert.argtypes = [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(QcuMGResult)]
_lib.qcuMGCheck.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
_lib.qcuBenchDslash.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double)]


class QcuError(RuntimeError):
    pass


def last_error():
    buf = ctypes.create_string_buffer(1024)
    code = _lib.qcuGetLastError(buf, 1024)
    return code, buf.value.decode(errors="replace")


def _check(rc: int):
    if rc != 0:
        raise QcuError(last_error()[1] or f"qcu error {rc}")


def _ptr(x) -> int:
    """Device address of a Pointer-like (``.ptr``), an int, or a CUDA tensor."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "ptr"):
        return int(x.ptr)
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("tensor must live on the GPU")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return int(x.data_ptr())
    raise TypeError(f"cannot take a device pointer of {type(x)!r}")


def _param(p) -> QcuParam:
    return p if isinstance(p, QcuParam) else QcuParam(p)


# ------------------------------------------------------------------ qcu.h (pyqcu mirror)
def dslashQcu(fermion_out, fermion_in, gauge, param, parity: int) -> None:
    _lib.dslashQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(_param(param)), int(parity))


def dslashCloverQcu(fermion_out, fermion_in, gauge, param, parity: int) -> None:
    _lib.dslashCloverQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(_param(param)), int(parity))


def mpiDslashQcu(fermion_out, fermion_in, gauge, param, parity: int, grid) -> None:
    _lib.mpiDslashQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(_param(param)), int(parity),
                      ctypes.byref(_param(grid)))


def mpiBistabCgQcu(gauge, param, grid) -> None:
    _lib.mpiBistabCgQcu(_ptr(gauge), ctypes.byref(_param(param)), ctypes.byref(_param(grid)))


def ncclDslashQcu(fermion_out, fermion_in, gauge, param, parity: int, grid) -> None:
    _lib.ncclDslashQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(_param(param)), int(parity),
                       ctypes.byref(_param(grid)))


def ncclBistabCgQcu(fermion_out, fermion_in, gauge, param, grid) -> None:
    _lib.ncclBistabCgQcu(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge), ctypes.byref(_param(param)),
                         ctypes.byref(_param(grid)))


# ------------------------------------------------------------------ qcu_ext.h
def dslashCloverQcuNoAlloc(fermion_out, fermion_in, gauge, param, parity: int) -> int:
    """dslashCloverQcu without device allocation: the inverse clover scratch
    lives in a static device array, so lattices are limited to
    ``noalloc_max_sites()`` sites per parity; returns the status code."""
    return int(_lib.dslashCloverQcuNoAlloc(_ptr(fermion_out), _ptr(fermion_in), _ptr(gauge),
                                           ctypes.byref(_param(param)), int(parity)))


def noalloc_max_sites() -> int:
    return int(_lib.qcuNoAllocMaxSites())


def _latt(latt):
    return (ctypes.c_int * 4)(*[int(v) for v in latt])


class Gauge:
    """A gauge field (and optional clover term) resident on the device."""

    def __init__(self, gauge, latt, t_boundary: float = 1.0, clover_coeff: float = 0.0):
        self.latt = [int(v) for v in latt]
        self._h = _vp()
        _check(_lib.qcuGaugeLoad(ctypes.byref(self._h), _ptr(gauge), _latt(self.latt), float(t_boundary),
                                 float(clover_coeff)))
        self.t_boundary = t_boundary
        self.clover_coeff = clover_coeff

    def close(self):
        if self._h:
            _lib.qcuGaugeFree(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def dslash(self, out, inp, parity: int, clover: bool = False, precision: int = 64):
        """out = [A^-1] D in on PyQuda-layout half spinors, computed with the
        spinors stored in `precision` bits (64, 32, 16) or as FP32 spinors
        with 16-bit links (3216)."""
        _check(_lib.qcuDslash(self._h, _ptr(out), _ptr(inp), int(parity), int(clover), int(precision)))

    def dslash_multi_tc(self, out, inp, nrhs: int, parity: int):
        """out_j = D in_j for nrhs half spinors back to back ([nrhs][Vh][4][3]
        complex128), on the tcgen05 tensor cores (FP16 operands, FP32
        accumulation; qcuDslashMultiTC)."""
        _check(_lib.qcuDslashMultiTC(self._h, _ptr(out), _ptr(inp), int(nrhs), int(parity)))

    def dslash_multi_tc_time(self, nrhs: int, parity: int = 0, iters: int = 20) -> float:
        """ms per application of the tensor-core multi-rhs kernel on resident fields."""
        ms = ctypes.c_double()
        _check(_lib.qcuDslashMultiTCTime(self._h, int(nrhs), int(parity), int(iters), ctypes.byref(ms)))
        return ms.value

    def matpc(self, out, inp, kappa: float, clover: bool = False):
        _check(_lib.qcuMatPC(self._h, _ptr(out), _ptr(inp), float(kappa), int(clover)))

    def mat(self, out, inp, kappa: float, clover: bool = False):
        _check(_lib.qcuMat(self._h, _ptr(out), _ptr(inp), float(kappa), int(clover)))

    def invert(self, x, b, kappa: float, tol: float = 1e-10, maxiter: int = 10000, precision: int = 64,
               delta: float = 0.1, clover: bool = False, x0_mode: int = 0, x0_seed: int = 0, abs_tol: bool = False,
               chunk: int = 0, solver: str = "bicgstab", inner_iters: int = 16, inner_tol: float = 0.1,
               gcr_k: int = 8, gauge_precision: int = 0, precond: int = 0, nn: "Network" = None,
               mg: "Multigrid" = None) -> dict:
        """Solve M x = b (full spinors).  solver="bicgstab": BiCGSTAB in
        `precision` with FP64 reliable updates; solver="gcr": FP64 flexible
        GCR(gcr_k) preconditioned by `inner_iters` BiCGSTAB iterations in
        `precision` (or until the inner residual drops by inner_tol).
        precond: 1 the network nn, 2 nn then the inner solve, 3 the coarse-grid
        correction of the Multigrid mg (built on this gauge and kappa) then the
        inner solve."""
        p = QcuInvertParam()
        _lib.qcuInvertParamDefault(ctypes.byref(p))
        p.kappa, p.tol, p.maxiter, p.precision, p.delta = kappa, tol, maxiter, precision, delta
        p.abs_tol, p.x0_mode, p.x0_seed, p.use_clover, p.chunk = int(abs_tol), x0_mode, x0_seed, int(clover), chunk
        p.solver = {"bicgstab": 0, "gcr": 1}[solver]
        p.inner_iters, p.inner_tol, p.gcr_k = inner_iters, inner_tol, gcr_k
        p.gauge_precision = gauge_precision
        p.precond = precond
        p.nn = nn._h.value if nn is not None else None
        p.mg = mg._h.value if mg is not None else None
        r = QcuInvertResult()
        _check(_lib.qcuInvert(self._h, _ptr(x), _ptr(b), ctypes.byref(p), ctypes.byref(r)))
        return r.as_dict()

    def bench_dslash(self, precision: int = 64, clover: bool = False, iters: int = 20, gauge_precision: int = 0) -> float:
        ms = ctypes.c_double(0)
        _check(_lib.qcuBenchDslash(self._h, int(precision), int(gauge_precision), int(clover), int(iters),
                                   ctypes.byref(ms)))
        return ms.value


def invert_batch(systems, tol: float = 1e-10, maxiter: int = 10000, precision: int = 16, gauge_precision: int = 0,
                 inner_iters: int = 96, inner_tol: float = 0.05, gcr_k: int = 4):
    """Solve every right-hand side of every system together (qcuInvertBatch).

    systems: sequence of (gauge, x, b, kappa, clover) with `gauge` a Gauge and
    x, b contiguous complex128 CUDA tensors of nrhs full spinors
    ([nrhs, 2, Lt, Lz, Ly, Lx/2, 4, 3]).  Lattices may differ between
    systems.  The inner solve runs on 16-bit spinors and links by default
    (precision=32 with gauge_precision=16 or 0, or 64, for the others).
    Returns (one result dict per right-hand side in system order, the
    tunables the autotuner chose)."""
    sys_arr, nrhs_total = _batch_systems(systems)
    p = QcuInvertParam()
    _lib.qcuInvertParamDefault(ctypes.byref(p))
    p.tol, p.maxiter, p.precision, p.gauge_precision = tol, maxiter, precision, gauge_precision
    p.solver, p.inner_iters, p.inner_tol, p.gcr_k = 1, inner_iters, inner_tol, gcr_k
    res = (QcuInvertResult * max(nrhs_total, 1))()
    tune = QcuBatchTune()
    _check(_lib.qcuInvertBatch(sys_arr, len(systems), ctypes.byref(p), res, ctypes.byref(tune)))
    return [res[i].as_dict() for i in range(nrhs_total)], tune.as_dict()


def _batch_systems(systems):
    sys_arr = (QcuBatchSystem * len(systems))()
    nrhs_total = 0
    for i, (G, x, b, kappa, clover) in enumerate(systems):
        L = Layout(tuple(G.latt))
        n = x.numel() // (2 * L.vh * 12)
        if n * 2 * L.vh * 12 != x.numel() or b.numel() != x.numel():
            raise ValueError("x and b must hold whole full spinors of the same count")
        sys_arr[i].gauge = G._h.value
        sys_arr[i].nrhs = n
        sys_arr[i].kappa = float(kappa)
        sys_arr[i].use_clover = int(bool(clover))
        sys_arr[i].x = _ptr(x)
        sys_arr[i].b = _ptr(b)
        nrhs_total += n
    return sys_arr, nrhs_total


def batch_apply_matpc(systems, precision: int = 16, gauge_precision: int = 0, dslash_threads: int = 128,
                      dslash_rhs: int = 1, mma: int = 0, blas_sites: int = 256):
    """The batched solver's inner operator, applied once (qcuBatchApplyMatPC).

    systems as for invert_batch.  For every right-hand side j, the kernels of
    the batched inner solve, with the given tunables, write to x[j]: the even
    half [A_e^-1] D_eo b_o and the odd half M_pc b_o, both computed from b[j]'s
    odd half stored in the inner precision.  Returns an [nrhs, 5] numpy array
    of the fused reductions: Re/Im <b_o, M_pc b_o>, Re/Im <M_pc b_o, b_o>,
    |M_pc b_o|^2."""
    import numpy as np

    sys_arr, nrhs = _batch_systems(systems)
    tune = QcuBatchTune()
    tune.dslash_threads, tune.dslash_rhs, tune.blas_sites, tune.mma = dslash_threads, dslash_rhs, blas_sites, mma
    dots = np.zeros((max(nrhs, 1), 5))
    _check(_lib.qcuBatchApplyMatPC(sys_arr, len(systems), int(precision), int(gauge_precision), ctypes.byref(tune),
                                   dots.ctypes.data))
    return dots[:nrhs]


def batch_dslash_time(systems, precision: int = 16, gauge_precision: int = 0, iters: int = 20, tune=None):
    """ms per launch of the batched solver's inner hopping kernel (first half
    of M_pc on the odd halves of every b), timed with CUDA events
    (qcuBatchDslashTime).  tune: None = the autotuner's choice, else a dict
    with dslash_threads, dslash_rhs, mma (and blas_sites).  Returns (ms, the
    tunables used as a dict)."""
    sys_arr, _ = _batch_systems(systems)
    t = QcuBatchTune()
    if tune is not None:
        t.dslash_threads = int(tune["dslash_threads"])
        t.dslash_rhs = int(tune["dslash_rhs"])
        t.mma = int(tune.get("mma", 0))
        t.blas_sites = int(tune.get("blas_sites", 256))
    ms = ctypes.c_double()
    _check(_lib.qcuBatchDslashTime(sys_arr, len(systems), int(precision), int(gauge_precision), ctypes.byref(t),
                                   int(iters), ctypes.byref(ms)))
    return ms.value, {"dslash_threads": t.dslash_threads, "dslash_rhs": t.dslash_rhs, "mma": t.mma,
                      "blas_sites": t.blas_sites}


# ---------------------------------------------------------------- several GPUs
def _ivec(v, n=4):
    if len(v) != n:
        raise ValueError(f"expected {n} integers")
    return (ctypes.c_int * n)(*[int(x) for x in v])


def dd_plan(latt, grid, rank: int) -> dict:
    """This rank's place in the grid (qcuDDPlan): coordinates, the
    neighbouring ranks in each direction, and the face sizes (sites of one
    parity) of the partitioned directions.  Needs no GPU."""
    out = (ctypes.c_int * 22)()
    _check(_lib.qcuDDPlan(_ivec(latt), _ivec(grid), int(rank), out))
    v = list(out)
    return {"nranks": v[0], "rank": v[1], "coord": v[2:6], "fwd": v[6:10], "bwd": v[10:14], "face": v[14:18]}


def dd_schedule(latt, grid, rank: int):
    """The face exchange this rank carries out, in order (qcuDDSchedule): a
    list of (kind, direction, slot, peer, count) with kind "send" or "recv"
    and count in complex numbers.  Needs no GPU."""
    ops = (ctypes.c_int * 80)()
    n = ctypes.c_int(0)
    _check(_lib.qcuDDSchedule(_ivec(latt), _ivec(grid), int(rank), ops, ctypes.byref(n)))
    v = list(ops)
    return [(("send", "recv")[v[5 * i]], v[5 * i + 1], v[5 * i + 2], v[5 * i + 3], v[5 * i + 4])
            for i in range(n.value)]


def dslash_dd_emulate(out_all, in_all, gauge_all, latt, parity: int, grid) -> None:
    """Every rank of `grid` in this process on the current GPU
    (qcuDslashDDEmulate): *_all hold the ranks' local PyQuda-layout fields
    back to back in rank order; latt is the local lattice."""
    _check(_lib.qcuDslashDDEmulate(_ptr(out_all), _ptr(in_all), _ptr(gauge_all), _ivec(latt), int(parity),
                                   _ivec(grid)))


def bistabcg_dd_emulate(x_all, b_all, gauge_all, latt, grid):
    """ncclBistabCgQcu's solve over `grid` for every rank at once in this
    process (qcuBistabCgDDEmulate); returns (iterations, final ||r_o||^2)."""
    it = ctypes.c_int(0)
    r2 = ctypes.c_double(0)
    _check(_lib.qcuBistabCgDDEmulate(_ptr(x_all), _ptr(b_all), _ptr(gauge_all), _ivec(latt), _ivec(grid),
                                     ctypes.byref(it), ctypes.byref(r2)))
    return it.value, r2.value


def comm_init(group=None) -> None:
    """Set up this device's communicator for ncclDslashQcu with a grid of
    ranks, from an initialised torch.distributed process group (any backend):
    rank 0 makes the NCCL id, the group broadcasts it, every rank calls
    qcuCommInit with its rank."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    buf = (ctypes.c_ubyte * 128)()
    if rank == 0:
        _check(_lib.qcuCommUniqueId(buf))
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(list(buf), dtype=torch.uint8, device=dev)
    dist.broadcast(t, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
    ids = (ctypes.c_ubyte * 128)(*t.cpu().tolist())
    _check(_lib.qcuCommInit(ids, world, rank))


def comm_unique_id() -> bytes:
    """A fresh NCCL unique id (qcuCommUniqueId), 128 bytes."""
    buf = (ctypes.c_ubyte * 128)()
    _check(_lib.qcuCommUniqueId(buf))
    return bytes(buf)


def comm_free() -> None:
    _check(_lib.qcuCommFree())


def point_sources(latt, origin, device="cuda"):
    """The 12 point sources (source spin s, colour c at `origin` = [x, y, z, t])
    of a propagator, PyQuda layout, [12 = s*3+c, 2, Lt, Lz, Ly, Lx/2, 4, 3]
    (python/PyQuda/pyquda/utils/source.py:7-22)."""
    import torch

    L = Layout(tuple(latt))
    x, y, z, t = [int(v) for v in origin]
    b = torch.zeros((12,) + L.full, dtype=torch.complex128, device=device)
    eo = (x + y + z + t) % 2
    for s in range(4):
        for c in range(3):
            b[s * 3 + c, eo, t, z, y, x // 2, s, c] = 1.0
    return b


def wall_source(latt, t: int, spin: int, color: int, device="cuda"):
    """Wall source at time slice t: 1 on every site of the slice for (spin,
    color), PyQuda layout [2, Lt, Lz, Ly, Lx/2, 4, 3]
    (python/PyQuda/pyquda/utils/source.py:25-34)."""
    import torch

    L = Layout(tuple(latt))
    b = torch.zeros(L.full, dtype=torch.complex128, device=device)
    b[:, t, :, :, :, spin, color] = 1.0
    return b


def momentum_phase(latt, mom, device="cuda"):
    """exp(i 2 pi sum_k p_k x_k / L_k) on the spatial coordinates, PyQuda
    even-odd layout [2, Lt, Lz, Ly, Lx/2]."""
    import math

    import torch

    Lx, Ly, Lz, Lt = [int(v) for v in latt]
    t, z, y, xh = torch.meshgrid(torch.arange(Lt), torch.arange(Lz), torch.arange(Ly), torch.arange(Lx // 2),
                                 indexing="ij")
    out = torch.empty((2, Lt, Lz, Ly, Lx // 2), dtype=torch.complex128)
    px, py, pz = [float(v) for v in mom]
    for p in (0, 1):
        x = (2 * xh + ((t + z + y + p) % 2)).to(torch.float64)
        arg = 2 * math.pi * (px * x / Lx + py * y.to(torch.float64) / Ly + pz * z.to(torch.float64) / Lz)
        out[p] = torch.polar(torch.ones_like(arg), arg)
    return out.to(device)


def momentum_source(latt, t: int, phase, spin: int, color: int, device="cuda"):
    """Momentum (wall) source: the phase on time slice t for (spin, color)
    (python/PyQuda/pyquda/utils/source.py:37-46)."""
    import torch

    L = Layout(tuple(latt))
    b = torch.zeros(L.full, dtype=torch.complex128, device=device)
    b[:, t, :, :, :, spin, color] = phase.to(device)[:, t]
    return b


def invert12(G: "Gauge", kappa: float, origin, clover: bool = False, **kw):
    """Propagator from a point source at `origin`: the 12 spin-colour solves in
    one batched solve.  Returns (propagator [2, Lt, Lz, Ly, Lx/2, 4, 4, 3, 3] =
    [.., sink spin, source spin, sink colour, source colour] -- PyQuda's
    LatticePropagator layout, python/PyQuda/pyquda/core.py:44-57 --, the
    per-source result dicts, the tunables)."""
    import torch

    b = point_sources(G.latt, origin, device="cuda")
    x = torch.empty_like(b)
    res, tune = invert_batch([(G, x, b, kappa, clover)], **kw)
    L = Layout(tuple(G.latt))
    prop = x.view((4, 3) + L.full).permute(2, 3, 4, 5, 6, 7, 0, 8, 1).contiguous()
    return prop, res, tune


class Network:
    """Learned preconditioner (qcuNN): a gauge-equivariant parallel-transport
    network approximating M_pc^{-1}; see include/qcu_ext.h."""

    def __init__(self, seed: int = 0, init_scale: float = 0.01):
        self._h = _vp()
        _check(_lib.qcuNNCreate(ctypes.byref(self._h), int(seed), float(init_scale)))

    @staticmethod
    def num_params() -> int:
        return int(_lib.qcuNNNumParams())

    def get_weights(self):
        import numpy as np

        w = np.empty(self.num_params(), np.float32)
        _check(_lib.qcuNNGetWeights(self._h, w.ctypes.data))
        return w

    def set_weights(self, w):
        import numpy as np

        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.num_params()
        _check(_lib.qcuNNSetWeights(self._h, w.ctypes.data))

    def apply(self, gauge: "Gauge", out, inp):
        _check(_lib.qcuNNApply(self._h, gauge._h, _ptr(out), _ptr(inp)))

    def set_tensor_cores(self, on: bool):
        """Inference on the tcgen05 tensor-core layers (default) or the FP32 FMA ones."""
        _check(_lib.qcuNNSetTensorCores(self._h, int(bool(on))))

    def train_step(self, gauge: "Gauge", r, e, batch: int, lr: float, want_grad: bool = False):
        """Returns (loss, grad or None); r, e: [batch][Vh][4][3] complex128 device buffers."""
        import numpy as np

        loss = ctypes.c_double(0)
        g = np.empty(self.num_params(), np.float32) if want_grad else None
        _check(_lib.qcuNNTrainStep(self._h, gauge._h, _ptr(r), _ptr(e), int(batch), float(lr), ctypes.byref(loss),
                                   g.ctypes.data if g is not None else None))
        return loss.value, g

    def close(self):
        if self._h:
            _lib.qcuNNFree(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Multigrid:
    """Two-level adaptive aggregation multigrid (qcuMG) for the full operator
    M = A - kappa D of a Gauge; parameters as PyQuda's multigrid set-up
    (geo_block_size, n_vec, setup_maxiter, coarse_tol, coarse_maxiter,
    nu_pre, nu_post) plus gcr_k, the outer GCR restart length.  The gauge
    must stay open while the multigrid is used."""

    def __init__(self, gauge: "Gauge", kappa: float, **params):
        p = QcuMGParam()
        _lib.qcuMGParamDefault(ctypes.byref(p))
        for k, v in params.items():
            if k == "geo_block_size":
                p.geo_block_size = (ctypes.c_int * 4)(*[int(x) for x in v])
            elif k in dict(QcuMGParam._fields_):
                setattr(p, k, v)
            else:
                raise TypeError(f"unknown multigrid parameter {k!r}")
        self.gauge = gauge
        self.kappa = kappa
        self._h = _vp()
        secs = ctypes.c_double(0)
        _check(_lib.qcuMGCreate(ctypes.byref(self._h), gauge._h, float(kappa), ctypes.byref(p), ctypes.byref(secs)))
        self.setup_seconds = secs.value

    def invert(self, x, b, tol: float = 1e-10, maxiter: int = 1000) -> dict:
        """x = M^-1 b on full PyQuda-layout spinors (complex128, device)."""
        r = QcuMGResult()
        _check(_lib.qcuMGInvert(self._h, _ptr(x), _ptr(b), float(tol), int(maxiter), ctypes.byref(r)))
        return r.as_dict()

    def check(self):
        """(|P^dag P c - c| / |c|, |A_c c - P^dag M P c| / |P^dag M P c|) for a seeded coarse c."""
        o, g = ctypes.c_double(0), ctypes.c_double(0)
        _check(_lib.qcuMGCheck(self._h, ctypes.byref(o), ctypes.byref(g)))
        return o.value, g.value

    def close(self):
        if self._h:
            _lib.qcuMGFree(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gauge_random(gauge, latt, kind: int = 0, eps: float = 0.25, seed: int = 0):
    """Fill a PyQuda-layout complex128 gauge buffer: kind 0 Haar, 1 exp(i eps H), 2 unit."""
    _check(_lib.qcuGaugeRandom(_ptr(gauge), _latt(latt), int(kind), float(eps), int(seed)))


def fermion_random(psi, n_complex: int, kind: int = 0, seed: int = 0):
    """Fill n complex128 values: kind 0 complex normal N(0,1), 1 uniform (0,1]."""
    _check(_lib.qcuFermionRandom(_ptr(psi), int(n_complex), int(kind), int(seed)))


def kernel_launches() -> int:
    """Kernels launched by libqcu so far in this process (graph replays count every node)."""
    return int(_lib.qcuKernelLaunches())


def stream_handle() -> int:
    return int(_lib.qcuGetStream() or 0)


@dataclass(frozen=True)
class Layout:
    """PyQuda field shapes for a lattice [Lx, Ly, Lz, Lt] (field.py:72,78)."""

    latt: tuple

    @property
    def half(self):
        Lx, Ly, Lz, Lt = self.latt
        return (Lt, Lz, Ly, Lx // 2, 4, 3)

    @property
    def full(self):
        return (2,) + self.half

    @property
    def gauge(self):
        Lx, Ly, Lz, Lt = self.latt
        return (4, 2, Lt, Lz, Ly, Lx // 2, 3, 3)

    @property
    def vh(self):
        Lx, Ly, Lz, Lt = self.latt
        return Lx * Ly * Lz * Lt // 2
