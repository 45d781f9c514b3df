/*
 * qcu_oracle.c -- CPU restatement of qcu's fermion-matrix hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it to produce
 * the expected answer.  Nothing in the product library (qcu_b200/) links,
 * loads or calls it.
 *
 * Everything here works directly in PyQuda's field layouts, which is the
 * layout the qcu C ABI receives (python/PyQuda/pyquda/field.py:72,78,152,230):
 *   half spinor  : complex128 [Lt][Lz][Ly][Lx/2][Ns=4][Nc=3]
 *   full spinor  : complex128 [2][Lt][Lz][Ly][Lx/2][4][3]   (even half first)
 *   gauge        : complex128 [Nd=4][2][Lt][Lz][Ly][Lx/2][3][3]
 * The half-lattice site index is i = ((t*Lz + z)*Ly + y)*(Lx/2) + xh and the
 * site (x,y,z,t) of parity p has x = 2*xh + ((y+z+t+p) & 1)
 * (field.py:22-63, cb2/lexico; qcu's move_*_x macros, include/define.h:127-134).
 *
 * Parity conventions are qcu's: `parity` is the OUTPUT parity, the input lives
 * on 1-parity (src/wilson_dslash.cu:9-245, src/draft.cu:14-15).
 *
 * Build: `make -C oracle` (gcc, OpenMP).  Compiled without -march=native so
 * the shared object runs on any x86-64 host.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
  int L[4];    /* x, y, z, t (QcuParam order, include/qcu.h:17-19) */
  int Lxh;     /* Lx / 2 */
  int64_t Vh;  /* Lx*Ly*Lz*Lt / 2 */
} geo_t;

static geo_t mkgeo(const int *L) {
  geo_t g;
  for (int d = 0; d < 4; d++) g.L[d] = L[d];
  g.Lxh = L[0] / 2;
  g.Vh = (int64_t)g.Lxh * L[1] * L[2] * L[3];
  return g;
}

/* full coordinates (x,y,z,t) of half-lattice site i with parity p */
static inline void site_coords(const geo_t *g, int64_t i, int p, int c[4]) {
  int xh = (int)(i % g->Lxh);
  int64_t r = i / g->Lxh;
  int y = (int)(r % g->L[1]);
  r /= g->L[1];
  int z = (int)(r % g->L[2]);
  int t = (int)(r / g->L[2]);
  c[0] = 2 * xh + ((y + z + t + p) & 1);
  c[1] = y;
  c[2] = z;
  c[3] = t;
}

/* half index and parity of the (already wrapped) full coordinate c */
static inline int64_t half_index(const geo_t *g, const int c[4], int *par) {
  *par = (c[0] + c[1] + c[2] + c[3]) & 1;
  return (((int64_t)c[3] * g->L[2] + c[2]) * g->L[1] + c[1]) * g->Lxh + c[0] / 2;
}

static inline void shift(const geo_t *g, const int c[4], int mu, int step, int out[4]) {
  for (int d = 0; d < 4; d++) out[d] = c[d];
  out[mu] = (c[mu] + step + g->L[mu]) % g->L[mu];
}

/* ------------------------------------------------------------------------ */
/* counter-based random numbers                                              */
/*                                                                           */
/* SplitMix64's output function (Steele, Lea & Flood, OOPSLA 2014) applied   */
/* to (hashed seed + counter * golden gamma).  Each field element owns fixed */
/* counters, so any implementation of the same arithmetic (the CUDA one in   */
/* qcu_b200/csrc/fields.cu) produces bit-identical integers.                 */
/* ------------------------------------------------------------------------ */
static inline uint64_t sm64_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

uint64_t orc_rng_u64(uint64_t seed, uint64_t ctr) {
  uint64_t s = sm64_mix(seed + 0x9E3779B97F4A7C15ULL);
  return sm64_mix(s + (ctr + 1) * 0x9E3779B97F4A7C15ULL);
}

/* uniform on (0, 1] with 53 random bits */
static inline double rng_uniform(uint64_t seed, uint64_t ctr) {
  return (double)((orc_rng_u64(seed, ctr) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

/* complex normal variate, real and imaginary parts ~ N(0,1) (Box-Muller) */
static inline cplx rng_cgauss(uint64_t seed, uint64_t k) {
  double u1 = rng_uniform(seed, 2 * k);
  double u2 = rng_uniform(seed, 2 * k + 1);
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  return r * cos(th) + I * (r * sin(th));
}

/* ------------------------------------------------------------------------ */
/* 3x3 complex helpers (row-major, m[r*3+c])                                 */
/* ------------------------------------------------------------------------ */
static inline void su3_third_row(cplx *m) {
  /* row2 = conj(row0 x row1): qcu's reconstruct-12 (include/define.h:198-206) */
  m[6] = conj(m[1] * m[5] - m[2] * m[4]);
  m[7] = conj(m[2] * m[3] - m[0] * m[5]);
  m[8] = conj(m[0] * m[4] - m[1] * m[3]);
}

static void mat_mul(const cplx *a, const cplx *b, cplx *c) {
  cplx t[9];
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 3; k++) {
      cplx s = 0;
      for (int j = 0; j < 3; j++) s += a[r * 3 + j] * b[j * 3 + k];
      t[r * 3 + k] = s;
    }
  memcpy(c, t, sizeof t);
}

static void mat_dag(const cplx *a, cplx *c) {
  cplx t[9];
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 3; k++) t[r * 3 + k] = conj(a[k * 3 + r]);
  memcpy(c, t, sizeof t);
}

/* Gram-Schmidt on rows 0 and 1, row 2 from the cross product (det = 1) */
static void reunitarise(cplx *m) {
  double n0 = 0;
  for (int c = 0; c < 3; c++) n0 += creal(m[c] * conj(m[c]));
  n0 = 1.0 / sqrt(n0);
  for (int c = 0; c < 3; c++) m[c] *= n0;
  cplx pr = 0;
  for (int c = 0; c < 3; c++) pr += conj(m[c]) * m[3 + c];
  for (int c = 0; c < 3; c++) m[3 + c] -= pr * m[c];
  double n1 = 0;
  for (int c = 0; c < 3; c++) n1 += creal(m[3 + c] * conj(m[3 + c]));
  n1 = 1.0 / sqrt(n1);
  for (int c = 0; c < 3; c++) m[3 + c] *= n1;
  su3_third_row(m);
}

/* exp(i*eps*H) for Hermitian H: Taylor series after scaling by 2^-s,
 * then s squarings (Moler & Van Loan, "Nineteen dubious ways", method 3). */
static void expi_herm(const cplx *h, double eps, cplx *out) {
  cplx a[9];
  double nrm = 0;
  for (int k = 0; k < 9; k++) {
    a[k] = I * eps * h[k];
    nrm += creal(a[k] * conj(a[k]));
  }
  nrm = sqrt(nrm);
  int s = 0;
  while (nrm > 0.25) {
    nrm *= 0.5;
    s++;
  }
  double sc = ldexp(1.0, -s);
  for (int k = 0; k < 9; k++) a[k] *= sc;
  cplx res[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  cplx term[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int n = 1; n <= 16; n++) {
    mat_mul(term, a, term);
    for (int k = 0; k < 9; k++) {
      term[k] *= 1.0 / n;
      res[k] += term[k];
    }
  }
  for (int q = 0; q < s; q++) mat_mul(res, res, res);
  memcpy(out, res, sizeof res);
}

/* ------------------------------------------------------------------------ */
/* seeded field generators                                                   */
/* ------------------------------------------------------------------------ */

/* Complex normal N(0,1) per component: n complex numbers, element k uses
 * counters 2k and 2k+1.  Matches the reference tests' source, re and im drawn
 * from randn (test/test.nccl.dslash.qcu-np1.py:23). */
void orc_fermion_gauss(cplx *psi, int64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) psi[k] = rng_cgauss(seed, (uint64_t)k);
}

/* Haar-random SU(3) per link (hot start): rows of a complex Gaussian matrix,
 * Gram-Schmidt orthonormalised (Mezzadri, Notices AMS 54 (2007) 592), the
 * third row fixed by det = 1.  Link l = (d*2+p)*Vh + i draws elements 9l..9l+8. */
void orc_gauge_haar(cplx *gauge, const int *L, uint64_t seed) {
  geo_t g = mkgeo(L);
  int64_t nlink = 8 * g.Vh;
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < nlink; l++) {
    cplx m[9];
    for (int k = 0; k < 9; k++) m[k] = rng_cgauss(seed, (uint64_t)(9 * l + k));
    reunitarise(m);
    memcpy(gauge + 9 * l, m, sizeof m);
  }
}

/* Smooth links U = exp(i eps H), H = sum_a h_a lambda_a / 2 with h_a ~ N(0,1)
 * and lambda_a the Gell-Mann matrices, then reunitarised.  Link l draws the
 * 8 real coefficients from complex variates 4l..4l+3 (re, im pairs). */
void orc_su3_from_coeffs(const double *h8, double eps, cplx *u) {
  const double s3 = 0.57735026918962576450914878050196; /* 1/sqrt(3) */
  cplx H[9];
  /* lambda_1..lambda_8 / 2 */
  H[0] = 0.5 * (h8[2] + s3 * h8[7]);
  H[4] = 0.5 * (-h8[2] + s3 * h8[7]);
  H[8] = 0.5 * (-2.0 * s3 * h8[7]);
  H[1] = 0.5 * (h8[0] - I * h8[1]);
  H[3] = conj(H[1]);
  H[2] = 0.5 * (h8[3] - I * h8[4]);
  H[6] = conj(H[2]);
  H[5] = 0.5 * (h8[5] - I * h8[6]);
  H[7] = conj(H[5]);
  expi_herm(H, eps, u);
  reunitarise(u);
}

void orc_gauge_smooth(cplx *gauge, const int *L, double eps, uint64_t seed) {
  geo_t g = mkgeo(L);
  int64_t nlink = 8 * g.Vh;
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < nlink; l++) {
    double h8[8];
    for (int k = 0; k < 4; k++) {
      cplx z = rng_cgauss(seed, (uint64_t)(4 * l + k));
      h8[2 * k] = creal(z);
      h8[2 * k + 1] = cimag(z);
    }
    orc_su3_from_coeffs(h8, eps, gauge + 9 * l);
  }
}

/* uniform (0,1] real and imaginary parts, counters 2k / 2k+1 (the role of
 * qcu's curand initial guess, src/lattice_cuda.cu:3-14, with this project's
 * own generator) */
void orc_fermion_uniform(cplx *psi, int64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++)
    psi[k] = rng_uniform(seed, 2 * (uint64_t)k) + I * rng_uniform(seed, 2 * (uint64_t)k + 1);
}

/* ------------------------------------------------------------------------ */
/* gamma matrices (DeGrand-Rossi basis), as hard-coded in qcu's spin         */
/* projections (src/wilson_dslash.cu:56-91 x, :110-143 y, :160-196 z,       */
/* :212-243 t).  Each row has one non-zero entry: gam_col[mu][r] is its       */
/* column and gam_val[mu][r] its value.                                      */
/* ------------------------------------------------------------------------ */
static const int gam_col[4][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}, {2, 3, 0, 1}};
static cplx gam_val[4][4];
static int gam_ready = 0;

static void gam_init(void) {
  if (gam_ready) return;
  gam_val[0][0] = I;  gam_val[0][1] = I;  gam_val[0][2] = -I; gam_val[0][3] = -I;
  gam_val[1][0] = -1; gam_val[1][1] = 1;  gam_val[1][2] = 1;  gam_val[1][3] = -1;
  gam_val[2][0] = I;  gam_val[2][1] = -I; gam_val[2][2] = -I; gam_val[2][3] = I;
  gam_val[3][0] = 1;  gam_val[3][1] = 1;  gam_val[3][2] = 1;  gam_val[3][3] = 1;
  gam_ready = 1;
}

void orc_gamma(int mu, cplx *m16) {
  gam_init();
  for (int k = 0; k < 16; k++) m16[k] = 0;
  for (int r = 0; r < 4; r++) m16[r * 4 + gam_col[mu][r]] = gam_val[mu][r];
}

/* ------------------------------------------------------------------------ */
/* link access                                                               */
/* ------------------------------------------------------------------------ */
static inline void load_link(const cplx *gauge, const geo_t *g, int mu, int par, int64_t i,
                             int recon12, cplx *u) {
  const cplx *src = gauge + ((int64_t)(mu * 2 + par) * g->Vh + i) * 9;
  if (recon12) {
    for (int k = 0; k < 6; k++) u[k] = src[k];
    su3_third_row(u);
  } else {
    for (int k = 0; k < 9; k++) u[k] = src[k];
  }
}

static inline void link_at(const cplx *gauge, const geo_t *g, const int c[4], int mu, int recon12,
                           cplx *u) {
  int par;
  int64_t i = half_index(g, c, &par);
  load_link(gauge, g, mu, par, i, recon12, u);
}

/* ------------------------------------------------------------------------ */
/* Wilson hopping term                                                       */
/*                                                                           */
/* out(x) = sum_mu [ U_mu(x) (1 - gamma_mu) in(x+mu)                         */
/*                 + U_mu(x-mu)^dag (1 + gamma_mu) in(x-mu) ]                */
/* on the output parity, periodic in x,y,z and multiplied by t_bc on hops    */
/* that cross the t boundary (t_bc = -1: antiperiodic).  No kappa and no      */
/* diagonal term, as in qcu's wilson_dslash (src/wilson_dslash.cu:9-245).    */
/* recon12 != 0 rebuilds row 2 of each link from rows 0-1                    */
/* (include/define.h:198-206), which is what qcu always does.                */
/*                                                                           */
/* The projector (1 + sigma*gamma) has rank 2: the upper two spin rows       */
/* h_k = psi_k + sigma*g[k] psi_col[k] determine the lower ones through       */
/* row_m = sigma*g[m] h_col[m], so only two colour vectors are multiplied by  */
/* the link, as in qcu's kernel.                                             */
/* ------------------------------------------------------------------------ */
static inline void hop_accum(cplx *acc, const cplx *psi, const cplx *u, int dag, int mu, double sigma,
                             double phase) {
  cplx h[2][3], uh[2][3];
  for (int k = 0; k < 2; k++)
    for (int c = 0; c < 3; c++)
      h[k][c] = psi[k * 3 + c] + sigma * gam_val[mu][k] * psi[gam_col[mu][k] * 3 + c];
  for (int k = 0; k < 2; k++)
    for (int r = 0; r < 3; r++) {
      cplx s = 0;
      if (dag)
        for (int c = 0; c < 3; c++) s += conj(u[c * 3 + r]) * h[k][c];
      else
        for (int c = 0; c < 3; c++) s += u[r * 3 + c] * h[k][c];
      uh[k][r] = phase * s;
    }
  for (int c = 0; c < 3; c++) {
    acc[0 * 3 + c] += uh[0][c];
    acc[1 * 3 + c] += uh[1][c];
    acc[2 * 3 + c] += sigma * gam_val[mu][2] * uh[gam_col[mu][2]][c];
    acc[3 * 3 + c] += sigma * gam_val[mu][3] * uh[gam_col[mu][3]][c];
  }
}

void orc_dslash(cplx *out, const cplx *in, const cplx *gauge, const int *L, int parity, double t_bc,
                int recon12) {
  gam_init();
  geo_t g = mkgeo(L);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < g.Vh; i++) {
    int c[4], n[4], par;
    cplx acc[12] = {0};
    cplx u[9];
    site_coords(&g, i, parity, c);
    for (int mu = 0; mu < 4; mu++) {
      /* forward: U_mu(x) (1 - gamma_mu) psi(x + mu) */
      shift(&g, c, mu, +1, n);
      int64_t j = half_index(&g, n, &par);
      double ph = (mu == 3 && c[3] == g.L[3] - 1) ? t_bc : 1.0;
      load_link(gauge, &g, mu, parity, i, recon12, u);
      hop_accum(acc, in + j * 12, u, 0, mu, -1.0, ph);
      /* backward: U_mu(x - mu)^dag (1 + gamma_mu) psi(x - mu) */
      shift(&g, c, mu, -1, n);
      j = half_index(&g, n, &par);
      ph = (mu == 3 && c[3] == 0) ? t_bc : 1.0;
      load_link(gauge, &g, mu, 1 - parity, j, recon12, u);
      hop_accum(acc, in + j * 12, u, 1, mu, +1.0, ph);
    }
    memcpy(out + i * 12, acc, sizeof acc);
  }
}

/* ------------------------------------------------------------------------ */
/* level-1 helpers on n complex numbers                                      */
/* ------------------------------------------------------------------------ */
cplx orc_cdot(const cplx *a, const cplx *b, int64_t n) { /* sum conj(a)*b */
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
  for (int64_t k = 0; k < n; k++) {
    cplx z = conj(a[k]) * b[k];
    re += creal(z);
    im += cimag(z);
  }
  return re + I * im;
}

double orc_norm2(const cplx *a, int64_t n) {
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t k = 0; k < n; k++) s += creal(a[k]) * creal(a[k]) + cimag(a[k]) * cimag(a[k]);
  return s;
}

/* wrapper used from Python (complex returns are awkward through ctypes) */
void orc_cdot2(const cplx *a, const cplx *b, int64_t n, double *re_im) {
  cplx z = orc_cdot(a, b, n);
  re_im[0] = creal(z);
  re_im[1] = cimag(z);
}

/* ------------------------------------------------------------------------ */
/* clover term                                                               */
/*                                                                           */
/* qcu's make_clover (src/clover_dslash.cu:5-837): for each plane mu<nu the  */
/* four plaquette leaves around x are summed into Q_munu (same leaf order     */
/* and product order as :46-159), F = Q - Q^dag, and the spin structure of   */
/* plane munu is gamma_mu*gamma_nu (the +-1/+-i block pattern written at     */
/* :161-172, :289-299, ...).  Then A = 1 - coeff/8 * sum (:826-835).  qcu has */
/* coeff fixed to 1; coeff = kappa*csw gives the Sheikholeslami-Wohlert term  */
/* 1 - kappa*csw/2 * sigma_munu F_munu with F = (Q - Q^dag)/(8i).             */
/* Output: full 12x12 matrix per site, A[i][(s0*3+c0)*12 + s1*3+c1].         */
/* ------------------------------------------------------------------------ */
void orc_clover_leaves(const cplx *gauge, const int *L, int parity, int64_t i, int mu, int nu,
                       int recon12, cplx *Q) {
  geo_t g = mkgeo(L);
  int c[4], a[4], b[4];
  cplx u1[9], u2[9], u3[9], u4[9], t[9];
  site_coords(&g, i, parity, c);
  for (int k = 0; k < 9; k++) Q[k] = 0;
  /* leaf 1: U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag */
  link_at(gauge, &g, c, mu, recon12, u1);
  shift(&g, c, mu, +1, a);
  link_at(gauge, &g, a, nu, recon12, u2);
  shift(&g, c, nu, +1, a);
  link_at(gauge, &g, a, mu, recon12, u3);
  link_at(gauge, &g, c, nu, recon12, u4);
  mat_mul(u1, u2, t);
  mat_dag(u3, u3);
  mat_mul(t, u3, t);
  mat_dag(u4, u4);
  mat_mul(t, u4, t);
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  /* leaf 2: U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu) */
  link_at(gauge, &g, c, nu, recon12, u1);
  shift(&g, c, mu, -1, a);
  shift(&g, a, nu, +1, b);
  link_at(gauge, &g, b, mu, recon12, u2);
  link_at(gauge, &g, a, nu, recon12, u3);
  link_at(gauge, &g, a, mu, recon12, u4);
  mat_dag(u2, u2);
  mat_mul(u1, u2, t);
  mat_dag(u3, u3);
  mat_mul(t, u3, t);
  mat_mul(t, u4, t);
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  /* leaf 3: U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu) */
  shift(&g, c, mu, -1, a);
  link_at(gauge, &g, a, mu, recon12, u1);
  shift(&g, a, nu, -1, b);
  link_at(gauge, &g, b, nu, recon12, u2);
  link_at(gauge, &g, b, mu, recon12, u3);
  shift(&g, c, nu, -1, a);
  link_at(gauge, &g, a, nu, recon12, u4);
  mat_dag(u1, u1);
  mat_dag(u2, u2);
  mat_mul(u1, u2, t);
  mat_mul(t, u3, t);
  mat_mul(t, u4, t);
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  /* leaf 4: U_nu(x-nu)^dag U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^dag */
  shift(&g, c, nu, -1, a);
  link_at(gauge, &g, a, nu, recon12, u1);
  link_at(gauge, &g, a, mu, recon12, u2);
  shift(&g, a, mu, +1, b);
  link_at(gauge, &g, b, nu, recon12, u3);
  link_at(gauge, &g, c, mu, recon12, u4);
  mat_dag(u1, u1);
  mat_mul(u1, u2, t);
  mat_mul(t, u3, t);
  mat_dag(u4, u4);
  mat_mul(t, u4, t);
  for (int k = 0; k < 9; k++) Q[k] += t[k];
}

void orc_clover_build(cplx *A, const cplx *gauge, const int *L, int parity, double coeff,
                      int recon12) {
  gam_init();
  geo_t g = mkgeo(L);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < g.Vh; i++) {
    cplx acc[144] = {0};
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        cplx Q[9], F[9];
        orc_clover_leaves(gauge, L, parity, i, mu, nu, recon12, Q);
        for (int r = 0; r < 3; r++)
          for (int k = 0; k < 3; k++) F[r * 3 + k] = Q[r * 3 + k] - conj(Q[k * 3 + r]);
        /* spin matrix gamma_mu gamma_nu: row s0 has its entry in column
           gam_col[nu][gam_col[mu][s0]] */
        for (int s0 = 0; s0 < 4; s0++) {
          int j = gam_col[mu][s0];
          int s1 = gam_col[nu][j];
          cplx sv = gam_val[mu][s0] * gam_val[nu][j];
          for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++) acc[(s0 * 3 + r) * 12 + s1 * 3 + k] += sv * F[r * 3 + k];
        }
      }
    for (int k = 0; k < 144; k++) acc[k] *= -0.125 * coeff;
    for (int k = 0; k < 12; k++) acc[k * 13] += 1.0;
    memcpy(A + i * 144, acc, sizeof acc);
  }
}

/* Gauss-Jordan inverse without pivoting on each 12x12, the algorithm of
 * qcu's inverse_clover (src/clover_dslash.cu:839-855, include/define.h:334-365),
 * with a correct complex division.  Returns the number of sites whose pivot
 * was exactly zero. */
int64_t orc_clover_invert(cplx *Ainv, const cplx *A, int64_t Vh) {
  int64_t bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
  for (int64_t i = 0; i < Vh; i++) {
    cplx aug[12 * 24];
    const cplx *a = A + i * 144;
    for (int r = 0; r < 12; r++) {
      for (int c = 0; c < 12; c++) {
        aug[r * 24 + c] = a[r * 12 + c];
        aug[r * 24 + 12 + c] = (r == c) ? 1.0 : 0.0;
      }
    }
    for (int r = 0; r < 12; r++) {
      cplx piv = aug[r * 24 + r];
      if (piv == 0) {
        bad++;
        piv = 1;
      }
      for (int c = 0; c < 24; c++) aug[r * 24 + c] /= piv;
      for (int j = 0; j < 12; j++) {
        if (j == r) continue;
        cplx f = aug[j * 24 + r];
        for (int c = 0; c < 24; c++) aug[j * 24 + c] -= f * aug[r * 24 + c];
      }
    }
    for (int r = 0; r < 12; r++)
      for (int c = 0; c < 12; c++) Ainv[i * 144 + r * 12 + c] = aug[r * 24 + 12 + c];
  }
  return bad;
}

/* out = A * in per site (qcu's give_clover, src/clover_dslash.cu:857-882);
 * out may alias in */
void orc_clover_apply(cplx *out, const cplx *A, const cplx *in, int64_t Vh) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < Vh; i++) {
    cplx t[12];
    for (int r = 0; r < 12; r++) {
      cplx s = 0;
      for (int c = 0; c < 12; c++) s += A[i * 144 + r * 12 + c] * in[i * 12 + c];
      t[r] = s;
    }
    memcpy(out + i * 12, t, sizeof t);
  }
}

/* ------------------------------------------------------------------------ */
/* even-odd preconditioned operator                                          */
/*                                                                           */
/* Wilson (qcu's _dslash, include/lattice_bistabcg.h:125-132 with            */
/* bistabcg_give_dest_o, src/bistabcg.cu:85-96):                              */
/*   M_pc in = in - kappa^2 D_{p,1-p} D_{1-p,p} in                            */
/* clover (Ainv_* != NULL):                                                  */
/*   M_pc in = in - kappa^2 A_p^-1 D_{p,1-p} A_{1-p}^-1 D_{1-p,p} in          */
/* tmp must hold 2 half spinors.                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
  const cplx *gauge;
  int L[4];
  int parity;  /* parity the preconditioned system lives on */
  double kappa;
  double t_bc;
  int recon12;
  const cplx *Ainv_p;    /* [Vh][144] on parity `parity`, or NULL */
  const cplx *Ainv_np;   /* on 1-parity, or NULL */
  cplx *tmp;
} mpc_t;

static void mpc_apply(const mpc_t *m, cplx *out, const cplx *in) {
  geo_t g = mkgeo(m->L);
  int64_t n = g.Vh * 12;
  cplx *t1 = m->tmp, *t2 = m->tmp + n;
  orc_dslash(t1, in, m->gauge, m->L, 1 - m->parity, m->t_bc, m->recon12);
  if (m->Ainv_np) orc_clover_apply(t1, m->Ainv_np, t1, g.Vh);
  orc_dslash(t2, t1, m->gauge, m->L, m->parity, m->t_bc, m->recon12);
  if (m->Ainv_p) orc_clover_apply(t2, m->Ainv_p, t2, g.Vh);
  double k2 = m->kappa * m->kappa;
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) out[k] = in[k] - k2 * t2[k];
}

void orc_mpc(cplx *out, const cplx *in, const cplx *gauge, const int *L, int parity, double kappa,
             double t_bc, int recon12, const cplx *Ainv_p, const cplx *Ainv_np) {
  geo_t g = mkgeo(L);
  mpc_t m = {gauge, {L[0], L[1], L[2], L[3]}, parity, kappa, t_bc, recon12, Ainv_p, Ainv_np, NULL};
  m.tmp = (cplx *)malloc(sizeof(cplx) * 24 * g.Vh);
  mpc_apply(&m, out, in);
  free(m.tmp);
}

/* full unpreconditioned operator on a two-parity spinor:
 *   Wilson: M psi = psi - kappa D psi          (QUDA/PyQuda kappa normalisation)
 *   clover: M psi = A psi - kappa D psi        (A passed per parity, not inverted) */
void orc_mfull(cplx *out, const cplx *in, const cplx *gauge, const int *L, double kappa, double t_bc,
               int recon12, const cplx *A_e, const cplx *A_o) {
  geo_t g = mkgeo(L);
  int64_t n = g.Vh * 12;
  cplx *t = (cplx *)malloc(sizeof(cplx) * n);
  for (int p = 0; p < 2; p++) {
    orc_dslash(t, in + (1 - p) * n, gauge, L, p, t_bc, recon12);
    const cplx *A = p ? A_o : A_e;
    cplx *o = out + p * n;
    if (A) orc_clover_apply(o, A, in + p * n, g.Vh);
    else memcpy(o, in + p * n, sizeof(cplx) * n);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) o[k] -= kappa * t[k];
  }
  free(t);
}

/* ------------------------------------------------------------------------ */
/* BiCGSTAB on M_pc, restating qcu's LatticeBistabcg::run_nccl               */
/* (include/lattice_bistabcg.h:221-340, kernels src/bistabcg.cu:4-169):      */
/*   rho = <r~,r>; beta = (rho/rho_prev)(alpha/omega); rho_prev = rho;       */
/*   p = r + beta (p - omega v); v = M p; alpha = rho/<r~,v>;                */
/*   s = r - alpha v; t = M s; omega = <t,s>/<t,t>;                           */
/*   r = s - omega t; x = x + alpha p + omega s.                             */
/* Initial rho_prev = alpha = omega = 1 and p = v = 0 (qcu seeds the scalars */
/* at lattice_bistabcg.h:52-57; p, v are taken as zero, the textbook start).  */
/* Stopping: abs_tol != 0 -> qcu's test ||r||^2 < tol, checked on the        */
/* residual at the top of the iteration (lattice_bistabcg.h:268-301);        */
/* abs_tol == 0 -> ||r||/||b|| <= tol on the iterated residual.               */
/* Returns iterations; *res_out = final iterated ||r||^2.                    */
/* ------------------------------------------------------------------------ */
int orc_bicgstab(cplx *x, const cplx *b, const cplx *gauge, const int *L, int parity, double kappa,
                 double t_bc, int recon12, const cplx *Ainv_p, const cplx *Ainv_np, double tol,
                 int abs_tol, int maxiter, double *res_out) {
  geo_t g = mkgeo(L);
  int64_t n = g.Vh * 12;
  cplx *w = (cplx *)calloc((size_t)(8 * n), sizeof(cplx));
  cplx *r = w, *rt = w + n, *p = w + 2 * n, *v = w + 3 * n, *s = w + 4 * n, *t = w + 5 * n;
  mpc_t m = {gauge, {L[0], L[1], L[2], L[3]}, parity, kappa, t_bc, recon12, Ainv_p, Ainv_np, w + 6 * n};
  mpc_apply(&m, r, x);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) {
    r[k] = b[k] - r[k];
    rt[k] = r[k];
  }
  double bn2 = orc_norm2(b, n);
  cplx rho_prev = 1, alpha = 1, omega = 1;
  double rn2 = orc_norm2(r, n);
  int it = 0;
  for (it = 0; it < maxiter; it++) {
    if (abs_tol) {
      if (rn2 < tol) break;
    } else if (sqrt(rn2) <= tol * sqrt(bn2)) {
      break;
    }
    cplx rho = orc_cdot(rt, r, n);
    cplx beta = (rho / rho_prev) * (alpha / omega);
    rho_prev = rho;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) p[k] = r[k] + (p[k] - v[k] * omega) * beta;
    mpc_apply(&m, v, p);
    alpha = rho / orc_cdot(rt, v, n);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) s[k] = r[k] - v[k] * alpha;
    mpc_apply(&m, t, s);
    omega = orc_cdot(t, s, n) / orc_cdot(t, t, n);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) {
      r[k] = s[k] - t[k] * omega;
      x[k] = x[k] + p[k] * alpha + s[k] * omega;
    }
    rn2 = orc_norm2(r, n);
  }
  if (res_out) *res_out = rn2;
  free(w);
  return it;
}

/* Full two-parity solve M x = b through the odd-parity Schur complement,
 * restating qcu's ncclBistabCgQcu flow (src/nccl_wilson_bistabcg.cu:7-27,
 * include/lattice_bistabcg.h:101-132,313-332) for Wilson, and its clover
 * analogue when A_e/A_o (and their inverses) are given:
 *   b'_o = A_o^-1 (b_o + kappa D_oe A_e^-1 b_e)
 *   solve (1 - kappa^2 A_o^-1 D_oe A_e^-1 D_eo) x_o = b'_o
 *   x_e  = A_e^-1 (b_e + kappa D_eo x_o)
 * x holds the initial guess on entry (its odd half is used). */
int orc_solve_full(cplx *x, const cplx *b, const cplx *gauge, const int *L, double kappa,
                   double t_bc, int recon12, const cplx *Ainv_e, const cplx *Ainv_o, double tol,
                   int abs_tol, int maxiter, double *res_out) {
  geo_t g = mkgeo(L);
  int64_t n = g.Vh * 12;
  cplx *bo = (cplx *)malloc(sizeof(cplx) * 2 * n);
  cplx *t = bo + n;
  const cplx *be = b, *bodd = b + n;
  cplx *xe = x, *xo = x + n;
  /* b'_o */
  if (Ainv_e) orc_clover_apply(t, Ainv_e, be, g.Vh);
  else memcpy(t, be, sizeof(cplx) * n);
  orc_dslash(bo, t, gauge, L, 1, t_bc, recon12);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) bo[k] = bodd[k] + kappa * bo[k];
  if (Ainv_o) orc_clover_apply(bo, Ainv_o, bo, g.Vh);
  int it = orc_bicgstab(xo, bo, gauge, L, 1, kappa, t_bc, recon12, Ainv_o, Ainv_e, tol, abs_tol,
                        maxiter, res_out);
  /* x_e */
  orc_dslash(t, xo, gauge, L, 0, t_bc, recon12);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) xe[k] = be[k] + kappa * t[k];
  if (Ainv_e) orc_clover_apply(xe, Ainv_e, xe, g.Vh);
  free(bo);
  return it;
}

/* ------------------------------------------------------------------------ */
/* misc                                                                      */
/* ------------------------------------------------------------------------ */
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
