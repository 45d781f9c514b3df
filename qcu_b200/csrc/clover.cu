// Clover term: build, pack, invert, apply.
//
// qcu's make_clover (src/clover_dslash.cu:5-837) forms, for each plane mu<nu,
// the four plaquette leaves Q_munu around x, F = Q - Q^dag, adds F into the
// 12x12 site matrix with the spin pattern of gamma_mu gamma_nu, and returns
// A = 1 - 1/8 sum (:826-835); inverse_clover (:839-855) then runs an
// unpivoted 12x12 Gauss-Jordan per site with a 288-entry local array, and
// give_clover (:857-882) multiplies densely.
//
// Here A is kept as what it is in the DeGrand-Rossi (chiral) basis: two
// Hermitian 6x6 blocks (spins {0,1} and {2,3}), 36 reals each -- 72 reals per
// site instead of 144 complex.  The inverse is an LDL^H factorisation per
// block (real pivots, no square roots, valid whenever the leading minors are
// non-zero, which is also what the unpivoted Gauss-Jordan requires), written
// back in the same packed form, and the apply is fused into the dslash
// epilogue (fields.cuh: clover_apply_site).  `coeff` scales the field-strength
// term: 1 reproduces qcu, kappa*csw gives the Sheikholeslami-Wohlert term.
#include "internal.h"

namespace qcu {

using C = Cpx<double>;

__device__ __forceinline__ void m3_mul(const C *a, const C *b, C *c) {
  C t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 3; k++) t[r * 3 + k] = a[r * 3] * b[k] + a[r * 3 + 1] * b[3 + k] + a[r * 3 + 2] * b[6 + k];
#pragma unroll
  for (int i = 0; i < 9; i++) c[i] = t[i];
}
__device__ __forceinline__ void m3_dag(C *a) {
  C t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 3; k++) t[r * 3 + k] = a[k * 3 + r].conj();
#pragma unroll
  for (int i = 0; i < 9; i++) a[i] = t[i];
}

// link U_mu at full coordinate (x,y,z,t) (wrapped), from the PyQuda gauge
__device__ __forceinline__ void link_at(const GaugeView<GAOS64> &U, const Geom &g, int x, int y, int z, int t, int mu,
                                        C *u) {
  const int Lx = 2 * g.Lxh;
  x = (x + Lx) % Lx;
  y = (y + g.Ly) % g.Ly;
  z = (z + g.Lz) % g.Lz;
  t = (t + g.Lt) % g.Lt;
  const int par = (x + y + z + t) & 1;
  const int s = ((t * g.Lz + z) * g.Ly + y) * g.Lxh + (x >> 1);
  link_load<GAOS64, double>(U, mu, par, s, u);
}

// sum of the four leaves in plane (mu, nu) at c[] (same products as qcu, in the
// same left-to-right order)
__device__ __noinline__ void clover_leaves(const GaugeView<GAOS64> &U, const Geom &g, const int c[4], int mu, int nu,
                                           C *Q) {
  int a[4], b[4];
  C u1[9], u2[9], u3[9], u4[9], t[9];
#define SH(dst, src, d, st)                 \
  {                                         \
    for (int q = 0; q < 4; q++) dst[q] = src[q]; \
    dst[d] += st;                           \
  }
#define LK(p, d, u) link_at(U, g, p[0], p[1], p[2], p[3], d, u)
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] = C(0, 0);
  // U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
  LK(c, mu, u1);
  SH(a, c, mu, 1);
  LK(a, nu, u2);
  SH(a, c, nu, 1);
  LK(a, mu, u3);
  LK(c, nu, u4);
  m3_mul(u1, u2, t);
  m3_dag(u3);
  m3_mul(t, u3, t);
  m3_dag(u4);
  m3_mul(t, u4, t);
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  // U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
  LK(c, nu, u1);
  SH(a, c, mu, -1);
  SH(b, a, nu, 1);
  LK(b, mu, u2);
  LK(a, nu, u3);
  LK(a, mu, u4);
  m3_dag(u2);
  m3_mul(u1, u2, t);
  m3_dag(u3);
  m3_mul(t, u3, t);
  m3_mul(t, u4, t);
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  // U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
  SH(a, c, mu, -1);
  LK(a, mu, u1);
  SH(b, a, nu, -1);
  LK(b, nu, u2);
  LK(b, mu, u3);
  SH(a, c, nu, -1);
  LK(a, nu, u4);
  m3_dag(u1);
  m3_dag(u2);
  m3_mul(u1, u2, t);
  m3_mul(t, u3, t);
  m3_mul(t, u4, t);
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] += t[k];
  // U_nu(x-nu)^+ U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^+
  SH(a, c, nu, -1);
  LK(a, nu, u1);
  LK(a, mu, u2);
  SH(b, a, mu, 1);
  LK(b, nu, u3);
  LK(c, mu, u4);
  m3_dag(u1);
  m3_mul(u1, u2, t);
  m3_mul(t, u3, t);
  m3_dag(u4);
  m3_mul(t, u4, t);
#pragma unroll
  for (int k = 0; k < 9; k++) Q[k] += t[k];
#undef SH
#undef LK
}

__device__ __forceinline__ C unit(int re, int im) { return C((double)re, (double)im); }

// packed block store (site-blocked CSOA64): d[0..5] then lower triangle
__device__ __forceinline__ void block_store(void *out, int blk, int s, const C M[36]) {
  double2 *p = static_cast<double2 *>(out) + blk_base<36>(s) + blk * 18 * SB;
  p[0] = make_double2(M[0].re, M[7].re);
  p[SB] = make_double2(M[14].re, M[21].re);
  p[2 * SB] = make_double2(M[28].re, M[35].re);
  int k = 3;
  for (int i = 1; i < 6; i++)
    for (int j = 0; j < i; j++, k++) p[k * SB] = make_double2(M[i * 6 + j].re, M[i * 6 + j].im);
}

// Hermitian inverse of a 6x6 block by LDL^H; returns false on a zero pivot
__device__ bool herm6_inverse(const C A[36], C Ai[36]) {
  C L[36];
  double D[6];
#pragma unroll
  for (int j = 0; j < 6; j++) {
    double dj = A[j * 6 + j].re;
#pragma unroll
    for (int k = 0; k < j; k++) dj -= L[j * 6 + k].norm2() * D[k];
    if (dj == 0.0 || !(dj == dj)) return false;
    D[j] = dj;
#pragma unroll
    for (int i = j + 1; i < 6; i++) {
      C v = A[i * 6 + j];
#pragma unroll
      for (int k = 0; k < j; k++) v -= L[i * 6 + k] * L[j * 6 + k].conj() * D[k];
      L[i * 6 + j] = v * (1.0 / dj);
    }
  }
  // M = L^-1 (unit lower triangular)
  C M[36];
#pragma unroll
  for (int j = 0; j < 6; j++) {
#pragma unroll
    for (int i = 0; i < 6; i++) M[i * 6 + j] = C(i == j ? 1.0 : 0.0, 0.0);
#pragma unroll
    for (int i = j + 1; i < 6; i++) {
      C v(0, 0);
#pragma unroll
      for (int k = j; k < i; k++) v += L[i * 6 + k] * M[k * 6 + j];
      M[i * 6 + j] = -v;
    }
  }
  // A^-1 = M^H D^-1 M
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j <= i; j++) {
      C v(0, 0);
#pragma unroll
      for (int k = i; k < 6; k++) v += M[k * 6 + i].conj() * M[k * 6 + j] * (1.0 / D[k]);
      Ai[i * 6 + j] = v;
      Ai[j * 6 + i] = v.conj();
    }
  return true;
}

__global__ void k_clover_build(Geom g, GaugeView<GAOS64> U, int par, double coeff, void *A64, void *Ainv64,
                               int *bad) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.Vh) return;
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int c[4] = {2 * xh + ((y + z + t + par) & 1), y, z, t};
  // every loop below is unrolled, so blk is indexed at compile time and
  // stays in registers (a runtime index would place it in local memory)
  C blk[2][36];
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int k = 0; k < 36; k++) blk[b][k] = C(0, 0);
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int nu = mu + 1; nu < 4; nu++) {
      C Q[9], F[9];
      clover_leaves(U, g, c, mu, nu, Q);
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) F[i * 3 + k] = Q[i * 3 + k] - Q[k * 3 + i].conj();
#pragma unroll
      for (int s0 = 0; s0 < 4; s0++) {
        const int j = gcol(mu, s0), s1 = gcol(nu, j);
        const C sv = unit(gre(mu, s0), gim(mu, s0)) * unit(gre(nu, j), gim(nu, j));
        const int b = s0 >> 1, r0 = (s0 & 1) * 3, c0 = (s1 & 1) * 3;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int k = 0; k < 3; k++) blk[b][(r0 + i) * 6 + c0 + k] += sv * F[i * 3 + k];
      }
    }
#pragma unroll
  for (int b = 0; b < 2; b++) {
#pragma unroll
    for (int k = 0; k < 36; k++) blk[b][k] = blk[b][k] * (-0.125 * coeff);
#pragma unroll
    for (int k = 0; k < 6; k++) blk[b][k * 7] += C(1.0, 0.0);
    if (A64) block_store(A64, b, s, blk[b]);
    if (Ainv64) {
      C inv[36];
      if (!herm6_inverse(blk[b], inv)) {
        atomicAdd(bad, 1);
        for (int k = 0; k < 36; k++) inv[k] = C(0, 0);
      }
      block_store(Ainv64, b, s, inv);
    }
  }
}

__global__ void k_clover_to32(int Vh, const double2 *in, float4 *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < Vh; s += gridDim.x * blockDim.x) {
    const double2 *pi = in + blk_base<36>(s);
    float4 *po = out + blk_base<18>(s);
    for (int b = 0; b < 2; b++)
      for (int k = 0; k < 9; k++) {
        const double2 u = pi[(b * 18 + 2 * k) * SB], w = pi[(b * 18 + 2 * k + 1) * SB];
        po[(b * 9 + k) * SB] = make_float4((float)u.x, (float)u.y, (float)w.x, (float)w.y);
      }
  }
}

template <int K>
__global__ void k_clover_apply(int Vh, CloverView<CSOA64> cv, const void *in, void *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < Vh; s += gridDim.x * blockDim.x) {
    Cpx<double> v[12];
    spinor_load<K, double>(SpinorView<K>{const_cast<void *>(in), nullptr, Vh}, s, v);
    clover_apply_site<CSOA64, double>(cv, s, v);
    spinor_store<K, double>(SpinorView<K>{out, nullptr, Vh}, s, v);
  }
}

size_t clover_bytes(int ckind, int Vh) { return (size_t)2 * (ckind == CSOA64 ? 18 * 16 : 9 * 16) * pad_sites(Vh); }

void launch_clover_build(const Geom &g, const void *gauge_pyq, int par, double coeff, void *A64, void *Ainv64, int *bad,
                         cudaStream_t s) {
  k_clover_build<<<(g.Vh + 63) / 64, 64, 0, s>>>(g, GaugeView<GAOS64>{gauge_pyq, g.Vh}, par, coeff, A64, Ainv64, bad);
  QCU_CHECK_LAUNCH();
}

void launch_clover_to32(int Vh, const void *c64, void *c32, cudaStream_t s) {
  k_clover_to32<<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, static_cast<const double2 *>(c64), static_cast<float4 *>(c32));
  QCU_CHECK_LAUNCH();
}

void launch_clover_apply(int kind, int Vh, const void *c64, const void *in, void *out, cudaStream_t s) {
  const CloverView<CSOA64> cv{c64, Vh};
  if (kind == AOS64) k_clover_apply<AOS64><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, cv, in, out);
  else if (kind == SOA64) k_clover_apply<SOA64><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, cv, in, out);
  else throw Error(1, "clover apply: unsupported spinor kind");
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
