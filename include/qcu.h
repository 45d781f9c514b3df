/*
 * qcu.h -- the drop-in C ABI of qcu's fermion-matrix path.
 *
 * Same struct and the same six entry points, with the same argument meaning,
 * as the reference header (include/qcu.h:17-30 of ZhangXin8069/qcu; the copy
 * PyQuda's Cython binding compiles against is
 * python/PyQuda/pyquda/include/qcu/qcu.h:1-20, bound in
 * python/PyQuda/pyquda/src/qcu.pxd:1-8 and pyqcu.pyx:15-34), so pyqcu links
 * against libqcu.so from this project unchanged.
 *
 * Conventions (unchanged from qcu):
 *  - every pointer is a DEVICE pointer to complex128 data in PyQuda layout
 *    (python/PyQuda/pyquda/field.py:72,78,152,230):
 *      half spinor  [Lt][Lz][Ly][Lx/2][4][3]
 *      full spinor  [2][Lt][Lz][Ly][Lx/2][4][3]   (even half first)
 *      gauge        [4][2][Lt][Lz][Ly][Lx/2][3][3]
 *  - lattice_size is {Lx, Ly, Lz, Lt}; `parity` is the OUTPUT parity.
 *  - links are SU(3): row 2 of every link is rebuilt from rows 0 and 1
 *    (reconstruct-12, as qcu does), boundaries are periodic.
 *  - calls are synchronous: they wait for all prior device work, and return
 *    after their own work has completed.
 *
 * Differences, all on the safe side:
 *  - inputs are never modified (qcu permuted gauge and spinors in place and
 *    restored them afterwards);
 *  - no NCCL/MPI setup per call; nothing is printed;
 *  - errors do not exit the process: the call does nothing more, and the
 *    reason is available from qcuGetLastError() (qcu_ext.h);
 *  - Vh does not need to be a multiple of 32.
 */
#ifndef QCU_B200_QCU_H
#define QCU_B200_QCU_H

#ifdef __cplusplus
extern "C" {
#endif

/* include/qcu.h:17-19 */
typedef struct QcuParam_s {
  int lattice_size[4];
} QcuParam;

/* out(parity) = D_{parity <- 1-parity} in, the Wilson hopping term without kappa
 * (replaces src/draft.cu:3-28, kernel src/wilson_dslash.cu:9-245) */
void dslashQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity);

/* out(parity) = A_parity^{-1} D_{parity <- 1-parity} in, with qcu's clover
 * A = 1 - 1/8 sum_{mu<nu} gamma_mu gamma_nu (Q_munu - Q_munu^dag) of the output
 * parity (replaces src/nccl_clover_dslash.cu:3-79, src/clover_dslash.cu:5-882) */
void dslashCloverQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity);

/* empty in the reference (src/draft.cu:29-31); kept as no-ops */
void mpiDslashQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity, QcuParam *grid);
void mpiBistabCgQcu(void *gauge, QcuParam *param, QcuParam *grid);

/* as dslashQcu on one GPU when `grid` is {1,1,1,1} (periodic wrap in-kernel);
 * otherwise this rank's part of the dslash of the global lattice split over
 * `grid` ranks, `param` being the local lattice (see qcuCommInit in
 * qcu_ext.h).  Replaces src/nccl_wilson_dslash.cu:3-19. */
void ncclDslashQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity, QcuParam *grid);

/* Solves M x = b, M = 1 - kappa D, kappa = 0.125 (include/define.h:69), by
 * even-odd preconditioned BiCGSTAB from a uniform random initial guess, until
 * the iterated ||r_o||^2 < 1e-9 or 1000 iterations (include/define.h:67-68,
 * include/lattice_bistabcg.h:221-340).  fermion_out = x, fermion_in = b, both
 * full spinors; with `grid` != {1,1,1,1}, this rank's part of the solve on the
 * global lattice split over the grid (param = the local lattice; see
 * qcuCommInit in qcu_ext.h).  Replaces src/nccl_wilson_bistabcg.cu:7-27. */
void ncclBistabCgQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, QcuParam *grid);

#ifdef __cplusplus
}
#endif

#endif
