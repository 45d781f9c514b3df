"""CPU oracle for qcu's fermion-matrix hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker.  Only the test-suite, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it; the product library
``qcu_b200`` never does.  Every function works on numpy complex128 arrays in
PyQuda's field layouts (python/PyQuda/pyquda/field.py:72,78,152,230):

* half spinor ``[Lt, Lz, Ly, Lx/2, 4, 3]``
* full spinor ``[2, Lt, Lz, Ly, Lx/2, 4, 3]`` (even half first)
* gauge       ``[4, 2, Lt, Lz, Ly, Lx/2, 3, 3]``

``latt`` is always ``[Lx, Ly, Lz, Lt]`` (QcuParam order, include/qcu.h:17-19).
The C code in ``qcu_oracle.c`` cites the reference lines each routine restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def reference_root() -> str:
    """Root of qcu's source tree, read only by the recipes that rebuild qcu
    and PyQuda's binding and by the scripts that make fixtures: the
    ``QCU_REFERENCE`` environment variable, else ``reference/`` beside this
    repository's own directory.  Nothing that runs on a GPU needs it."""
    env = os.environ.get("QCU_REFERENCE")
    if env:
        return os.path.abspath(env)
    return os.path.normpath(os.path.join(_HERE, "..", "..", "reference"))
_lib = None

_c128p = ctypes.c_void_p
_i32p = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile ``liboracle.so`` with gcc/OpenMP (no GPU needed)."""
    src = os.path.join(_HERE, "qcu_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_rng_u64.restype = ctypes.c_uint64
        L.orc_rng_u64.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_fermion_gauss.argtypes = [_c128p, ctypes.c_int64, ctypes.c_uint64]
        L.orc_fermion_uniform.argtypes = [_c128p, ctypes.c_int64, ctypes.c_uint64]
        L.orc_gauge_haar.argtypes = [_c128p, _i32p, ctypes.c_uint64]
        L.orc_gauge_smooth.argtypes = [_c128p, _i32p, ctypes.c_double, ctypes.c_uint64]
        L.orc_su3_from_coeffs.argtypes = [ctypes.c_void_p, ctypes.c_double, _c128p]
        L.orc_gamma.argtypes = [ctypes.c_int, _c128p]
        L.orc_dslash.argtypes = [_c128p, _c128p, _c128p, _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_cdot2.argtypes = [_c128p, _c128p, ctypes.c_int64, ctypes.c_void_p]
        L.orc_norm2.restype = ctypes.c_double
        L.orc_norm2.argtypes = [_c128p, ctypes.c_int64]
        L.orc_clover_leaves.argtypes = [_c128p, _i32p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, _c128p]
        L.orc_clover_build.argtypes = [_c128p, _c128p, _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_clover_invert.restype = ctypes.c_int64
        L.orc_clover_invert.argtypes = [_c128p, _c128p, ctypes.c_int64]
        L.orc_clover_apply.argtypes = [_c128p, _c128p, _c128p, ctypes.c_int64]
        L.orc_mpc.argtypes = [_c128p, _c128p, _c128p, _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int, _c128p, _c128p]
        L.orc_mfull.argtypes = [_c128p, _c128p, _c128p, _i32p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                _c128p, _c128p]
        L.orc_bicgstab.restype = ctypes.c_int
        L.orc_bicgstab.argtypes = [_c128p, _c128p, _c128p, _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, _c128p, _c128p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double)]
        L.orc_solve_full.restype = ctypes.c_int
        L.orc_solve_full.argtypes = [_c128p, _c128p, _c128p, _i32p, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, _c128p, _c128p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


# --------------------------------------------------------------------------- helpers
def _latt(latt):
    latt = [int(v) for v in latt]
    if len(latt) != 4 or latt[0] % 2:
        raise ValueError("latt must be [Lx, Ly, Lz, Lt] with Lx even")
    return (ctypes.c_int * 4)(*latt)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.complex128 and a.flags.c_contiguous
    return a.ctypes.data


def vh(latt) -> int:
    Lx, Ly, Lz, Lt = latt
    return Lx * Ly * Lz * Lt // 2


def half_shape(latt):
    Lx, Ly, Lz, Lt = latt
    return (Lt, Lz, Ly, Lx // 2, 4, 3)


def full_shape(latt):
    return (2,) + half_shape(latt)


def gauge_shape(latt):
    Lx, Ly, Lz, Lt = latt
    return (4, 2, Lt, Lz, Ly, Lx // 2, 3, 3)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


# --------------------------------------------------------------------------- generators
def rng_u64(seed: int, ctr: int) -> int:
    return int(lib().orc_rng_u64(seed, ctr))


def fermion_gauss(shape, seed: int) -> np.ndarray:
    out = np.empty(shape, np.complex128)
    lib().orc_fermion_gauss(_p(out), out.size, seed)
    return out


def fermion_uniform(shape, seed: int) -> np.ndarray:
    out = np.empty(shape, np.complex128)
    lib().orc_fermion_uniform(_p(out), out.size, seed)
    return out


def gauge_haar(latt, seed: int) -> np.ndarray:
    out = np.empty(gauge_shape(latt), np.complex128)
    lib().orc_gauge_haar(_p(out), _latt(latt), seed)
    return out


def gauge_smooth(latt, eps: float, seed: int) -> np.ndarray:
    out = np.empty(gauge_shape(latt), np.complex128)
    lib().orc_gauge_smooth(_p(out), _latt(latt), eps, seed)
    return out


def su3_from_coeffs(h8, eps: float) -> np.ndarray:
    h = np.ascontiguousarray(h8, np.float64)
    out = np.empty((3, 3), np.complex128)
    lib().orc_su3_from_coeffs(h.ctypes.data, eps, _p(out))
    return out


def gamma(mu: int) -> np.ndarray:
    out = np.empty((4, 4), np.complex128)
    lib().orc_gamma(mu, _p(out))
    return out


# --------------------------------------------------------------------------- operators
def dslash(inp, gauge, latt, parity: int, t_bc: float = 1.0, recon12: bool = True) -> np.ndarray:
    """Wilson hopping term onto ``parity`` from the opposite-parity half spinor."""
    inp = np.ascontiguousarray(inp, np.complex128)
    gauge = np.ascontiguousarray(gauge, np.complex128)
    out = np.empty(half_shape(latt), np.complex128)
    lib().orc_dslash(_p(out), _p(inp), _p(gauge), _latt(latt), parity, t_bc, int(recon12))
    return out


def cdot(a, b) -> complex:
    a = np.ascontiguousarray(a, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    r = np.zeros(2)
    lib().orc_cdot2(_p(a), _p(b), a.size, r.ctypes.data)
    return complex(r[0], r[1])


def norm2(a) -> float:
    a = np.ascontiguousarray(a, np.complex128)
    return float(lib().orc_norm2(_p(a), a.size))


def clover_leaves(gauge, latt, parity: int, site: int, mu: int, nu: int, recon12: bool = True):
    out = np.empty((3, 3), np.complex128)
    lib().orc_clover_leaves(_p(np.ascontiguousarray(gauge)), _latt(latt), parity, site, mu, nu,
                            int(recon12), _p(out))
    return out


def clover_build(gauge, latt, parity: int, coeff: float = 1.0, recon12: bool = True) -> np.ndarray:
    """Clover matrix A = 1 - coeff/8 sum_{mu<nu} g_mu g_nu (Q - Q^+), [Vh, 12, 12]."""
    gauge = np.ascontiguousarray(gauge, np.complex128)
    out = np.empty((vh(latt), 12, 12), np.complex128)
    lib().orc_clover_build(_p(out), _p(gauge), _latt(latt), parity, coeff, int(recon12))
    return out


def clover_invert(A) -> np.ndarray:
    A = np.ascontiguousarray(A, np.complex128)
    out = np.empty_like(A)
    bad = lib().orc_clover_invert(_p(out), _p(A), A.shape[0])
    if bad:
        raise ZeroDivisionError(f"{bad} sites with a zero pivot")
    return out


def clover_apply(A, inp) -> np.ndarray:
    A = np.ascontiguousarray(A, np.complex128)
    inp = np.ascontiguousarray(inp, np.complex128)
    out = np.empty_like(inp)
    lib().orc_clover_apply(_p(out), _p(A), _p(inp), A.shape[0])
    return out


def mpc(inp, gauge, latt, kappa: float, parity: int = 1, t_bc: float = 1.0, recon12: bool = True,
        Ainv_p=None, Ainv_np=None) -> np.ndarray:
    inp = np.ascontiguousarray(inp, np.complex128)
    out = np.empty_like(inp)
    lib().orc_mpc(_p(out), _p(inp), _p(np.ascontiguousarray(gauge)), _latt(latt), parity, kappa, t_bc,
                  int(recon12), _p(Ainv_p), _p(Ainv_np))
    return out


def mfull(inp, gauge, latt, kappa: float, t_bc: float = 1.0, recon12: bool = True, A_e=None, A_o=None):
    inp = np.ascontiguousarray(inp, np.complex128)
    out = np.empty_like(inp)
    lib().orc_mfull(_p(out), _p(inp), _p(np.ascontiguousarray(gauge)), _latt(latt), kappa, t_bc,
                    int(recon12), _p(A_e), _p(A_o))
    return out


def bicgstab(b, gauge, latt, kappa: float, x0=None, parity: int = 1, t_bc: float = 1.0, recon12: bool = True,
             Ainv_p=None, Ainv_np=None, tol: float = 1e-10, abs_tol: bool = False, maxiter: int = 1000):
    """BiCGSTAB on M_pc; returns (x, iterations, final iterated ||r||^2)."""
    b = np.ascontiguousarray(b, np.complex128)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.complex128, copy=True, order="C")
    res = ctypes.c_double(0)
    it = lib().orc_bicgstab(_p(x), _p(b), _p(np.ascontiguousarray(gauge)), _latt(latt), parity, kappa, t_bc,
                            int(recon12), _p(Ainv_p), _p(Ainv_np), tol, int(abs_tol), maxiter,
                            ctypes.byref(res))
    return x, int(it), float(res.value)


def solve_full(b, gauge, latt, kappa: float, x0=None, t_bc: float = 1.0, recon12: bool = True, Ainv_e=None,
               Ainv_o=None, tol: float = 1e-10, abs_tol: bool = False, maxiter: int = 1000):
    """Full two-parity solve M x = b via the odd Schur complement; returns (x, iterations, res2)."""
    b = np.ascontiguousarray(b, np.complex128)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.complex128, copy=True, order="C")
    res = ctypes.c_double(0)
    it = lib().orc_solve_full(_p(x), _p(b), _p(np.ascontiguousarray(gauge)), _latt(latt), kappa, t_bc,
                              int(recon12), _p(Ainv_e), _p(Ainv_o), tol, int(abs_tol), maxiter,
                              ctypes.byref(res))
    return x, int(it), float(res.value)
