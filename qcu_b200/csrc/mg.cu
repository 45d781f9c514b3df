// Two-level adaptive aggregation multigrid for the full Wilson or clover
// operator M = A - kappa D (A = 1 without clover).  qcu's own multigrid file
// is empty (src/multgrid.cu); the method is the aggregation multigrid that
// PyQuda configures for QUDA in python/PyQuda/pyquda/dslash/general.py:121-230
// (aggregates of geo_block_size sites, n_vec near-null vectors, chirality
// kept, MR smoother, loosely solved coarse system, flexible GCR outside).
//
// Set-up
//   * near-null vectors: for k = 1..n_vec, a Gaussian v0 and the error left
//     by a short solve of M y = M v0 (FP32 BiCGSTAB on the even-odd system,
//     setup_maxiter iterations), v = v0 - y: the slowly converging, low modes;
//   * aggregates: blocks of geo_block_size sites (both parities), each split
//     by chirality (spins 0,1 and 2,3: gamma_5 is diagonal in the DeGrand-Rossi
//     basis), so the coarse space keeps gamma_5's block structure;
//   * P: the vectors orthonormalised on every aggregate and chirality
//     (modified Gram-Schmidt with FP64 sums), stored in FP32;
//   * the Galerkin operator A_c = P^dag M P, built directly from the fine
//     hops: per aggregate a self block X (the local term A and the hops that
//     stay inside the aggregate) and one block Y_d per direction (the hops
//     that leave it), each 2 n_vec x 2 n_vec complex, FP32.
// Solve: flexible GCR in FP64 on the full system, preconditioned by one
// two-level cycle: nu_pre MR steps, the coarse correction P A_c^-1 P^dag r
// (FP32 BiCGSTAB on A_c to coarse_tol, at most coarse_maxiter iterations),
// nu_post MR steps.  The FP64 true residual decides convergence.
#include <chrono>
#include <cmath>
#include <memory>
#include <vector>

#include "mg.h"

namespace qcu {

namespace {

constexpr int MG_MAXVEC = 16;
constexpr int MG_MAXBLOCK = 512;  // sites per aggregate, at most
constexpr int MG_RED = 256;
constexpr int MG_RED_GRID = 148 * 4;

struct MGGeom {
  int L[4];    // fine full extents (x, y, z, t)
  int b[4];    // aggregate extents
  int nb[4];   // aggregates per direction
  int nblocks;
  int bsites;  // sites per aggregate (both parities)
  int Vh, Vp;  // sites per parity, and padded to the site blocks of 32
  int nvec;
  int nc;      // coarse degrees of freedom per aggregate (2 nvec)
};

struct SiteC {
  int x[4];  // full coordinates
  int par, s;
};

// site t (< bsites) of aggregate B: full coordinates, parity, half-lattice
// index i = ((t Lz + z) Ly + y) Lx/2 + x/2 (the PyQuda/qcu ordering)
__device__ __forceinline__ SiteC mg_site(const MGGeom &m, int B, int t) {
  SiteC c;
  int r = B, q = t;
#pragma unroll
  for (int d = 0; d < 4; d++) {
    c.x[d] = (r % m.nb[d]) * m.b[d] + q % m.b[d];
    r /= m.nb[d];
    q /= m.b[d];
  }
  c.par = (c.x[0] + c.x[1] + c.x[2] + c.x[3]) & 1;
  c.s = ((c.x[3] * m.L[2] + c.x[2]) * m.L[1] + c.x[1]) * (m.L[0] / 2) + (c.x[0] >> 1);
  return c;
}
__device__ __forceinline__ int mg_block_of(const MGGeom &m, const int x[4]) {
  return ((x[3] / m.b[3] * m.nb[2] + x[2] / m.b[2]) * m.nb[1] + x[1] / m.b[1]) * m.nb[0] + x[0] / m.b[0];
}
// the aggregate next to B in direction d = 2 mu + (0 forward, 1 backward); d = 8: B itself
__device__ __forceinline__ int mg_cnbr(const MGGeom &m, int B, int d) {
  if (d == 8) return B;
  const int mu = d >> 1;
  int stride = 1, n = m.nb[0];  // selects, not an indexed array: no local memory
  if (mu >= 1) stride *= m.nb[0], n = m.nb[1];
  if (mu >= 2) stride *= m.nb[1], n = m.nb[2];
  if (mu >= 3) stride *= m.nb[2], n = m.nb[3];
  const int c = (B / stride) % n;
  const int cn = (d & 1) ? (c == 0 ? n - 1 : c - 1) : (c == n - 1 ? 0 : c + 1);
  return B + (cn - c) * stride;
}

// a full fine vector: two site-blocked parity slabs in the SOA64 element
// order, parity p at p * Vp * 12
__device__ __forceinline__ size_t fidx(const MGGeom &m, int par, int s, int comp) {
  return (size_t)par * m.Vp * 12 + blk_base<12>(s) + (size_t)comp * SB;
}
// near-null vector k, FP32, aggregate-major: component comp of site t of
// aggregate B at ((k nblocks + B) 12 + comp) bsites + t, so the threads of
// an aggregate (one per site) read each component as one contiguous run
__device__ __forceinline__ size_t nidx(const MGGeom &m, int k, int B, int t, int comp) {
  return (((size_t)k * m.nblocks + B) * 12 + comp) * m.bsites + t;
}
// the index within its aggregate of the site with full coordinates x (inverse of mg_site)
__device__ __forceinline__ int mg_local(const MGGeom &m, const int x[4]) {
  return ((x[3] % m.b[3] * m.b[2] + x[2] % m.b[2]) * m.b[1] + x[1] % m.b[1]) * m.b[0] + x[0] % m.b[0];
}

// the coarse operator of aggregate B as a 9 nc x nc complex matrix
// (column j = d nc + col: d = 0..7 the directions Y_d, d = 8 the self block
// X), stored with the columns in pairs: element (j, row) at float2 index
// ((B * 9 nc / 2 + j / 2) * nc + row) * 2 + j % 2, so a lane reading its row
// takes the entries of two columns in one 16-byte load
__host__ __device__ __forceinline__ size_t yidx(const MGGeom &m, int B, int j, int row) {
  return (((size_t)B * (9 * m.nc / 2) + j / 2) * m.nc + row) * 2 + (j & 1);
}

// sum of N doubles over the thread block, every thread gets the totals
// (sh: blockDim / 32 * N doubles)
template <int N>
__device__ __forceinline__ void mg_block_sum(double (&v)[N], double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  __syncthreads();  // sh may still be read by an earlier call
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; k++) sh[w * N + k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; k++) {
    double t = 0;
    for (int q = 0; q < nw; q++) t += sh[q * N + k];
    v[k] = t;
  }
}

// ---------------------------------------------------------------- P and P^dag
// modified Gram-Schmidt of the near-null vectors on every aggregate and
// chirality (one thread block per aggregate, one thread per site)
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_orth(MGGeom m, float2 *nv) {
  __shared__ double sh[(MG_MAXBLOCK / 32) * 4];
  const int B = blockIdx.x, t = threadIdx.x;
  for (int k = 0; k < m.nvec; k++) {
    for (int j = 0; j <= k; j++) {
      double v[4] = {0, 0, 0, 0};  // per chirality: Re, Im of <v_j, v_k> (j == k: |v_k|^2)
      for (int comp = 0; comp < 12; comp++) {
        const int ch = comp / 6;
        const float2 a = nv[nidx(m, j, B, t, comp)], b = nv[nidx(m, k, B, t, comp)];
        v[2 * ch] += (double)a.x * b.x + (double)a.y * b.y;
        v[2 * ch + 1] += (double)a.x * b.y - (double)a.y * b.x;
      }
      mg_block_sum<4>(v, sh);
      for (int comp = 0; comp < 12; comp++) {
        const int ch = comp / 6;
        float2 &b = nv[nidx(m, k, B, t, comp)];
        if (j < k) {  // v_k -= <v_j, v_k> v_j
          const float2 a = nv[nidx(m, j, B, t, comp)];
          const double dr = v[2 * ch], di = v[2 * ch + 1];
          b = make_float2((float)(b.x - (dr * a.x - di * a.y)), (float)(b.y - (dr * a.y + di * a.x)));
        } else {
          const double inv = v[2 * ch] > 0 ? 1.0 / sqrt(v[2 * ch]) : 0.0;
          b = make_float2((float)(b.x * inv), (float)(b.y * inv));
        }
      }
    }
  }
}

// A fine FP64 vector as two parity slabs (SOA64 element order); a null
// slab reads as zero and is not written.
struct FineVec {
  double2 *p[2];
};
__device__ __forceinline__ size_t hidx(int s, int comp) { return blk_base<12>(s) + (size_t)comp * SB; }

// coarse c[B][ch nvec + k] = <v_k^ch, r>_B: per k a warp sum, then one pass
// over the warps
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_restrict(MGGeom m, const float2 *nv, FineVec r, float2 *cv) {
  __shared__ double red[MG_MAXBLOCK / 32][MG_MAXVEC][4];
  const int B = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  const SiteC c = mg_site(m, B, t);
  const double2 *rp = c.par ? r.p[1] : r.p[0];  // a select: no local copy of r
  double2 rv[12];
#pragma unroll
  for (int comp = 0; comp < 12; comp++) rv[comp] = rp ? rp[hidx(c.s, comp)] : make_double2(0, 0);
  for (int k = 0; k < m.nvec; k++) {
    double v[4] = {0, 0, 0, 0};
    if (rp) {
#pragma unroll
      for (int comp = 0; comp < 12; comp++) {
        const int ch = comp / 6;
        const float2 a = nv[nidx(m, k, B, t, comp)];
        v[2 * ch] += (double)a.x * rv[comp].x + (double)a.y * rv[comp].y;
        v[2 * ch + 1] += (double)a.x * rv[comp].y - (double)a.y * rv[comp].x;
      }
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < 4; i++) red[w][k][i] = v[i];
  }
  __syncthreads();
  for (int i = t; i < 2 * m.nvec; i += blockDim.x) {  // i = ch nvec + k
    const int ch = i / m.nvec, k = i % m.nvec;
    double re = 0, im = 0;
    for (int q = 0; q < nw; q++) {
      re += red[q][k][2 * ch];
      im += red[q][k][2 * ch + 1];
    }
    cv[(size_t)B * m.nc + i] = make_float2((float)re, (float)im);
  }
}

// e = P c (e += P c when add)
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_prolong(MGGeom m, const float2 *nv, const float2 *cv, FineVec e,
                                                          int add) {
  const int B = blockIdx.x, t = threadIdx.x;
  const SiteC c = mg_site(m, B, t);
  double2 *ep = c.par ? e.p[1] : e.p[0];
  if (!ep) return;
  const float2 *cb = cv + (size_t)B * m.nc;
#pragma unroll
  for (int comp = 0; comp < 12; comp++) {
    const int ch = comp / 6;
    double re = 0, im = 0;
    for (int k = 0; k < m.nvec; k++) {
      const float2 a = nv[nidx(m, k, B, t, comp)];
      const float2 q = cb[ch * m.nvec + k];
      re += (double)a.x * q.x - (double)a.y * q.y;
      im += (double)a.x * q.y + (double)a.y * q.x;
    }
    double2 &o = ep[hidx(c.s, comp)];
    if (add) o = make_double2(o.x + re, o.y + im);
    else o = make_double2(re, im);
  }
}

// ---------------------------------------------------------------- coarse operator
// h = the hop of direction MU (forward or backward) at site (par, s) applied
// to near-null vector k2 restricted to chirality ch2, taken at the neighbour
// n (site tn of aggregate Bn): U (1 - gamma_mu) forward, U^dag (1 + gamma_mu)
// backward, the stencil core of the dslash kernels
template <int MU, bool FWD>
__device__ __forceinline__ void mg_hop(const MGGeom &m, const GaugeView<GSOA64> &U, const float2 *nv, int par, int s,
                                       int n, int Bn, int tn, int k2, int ch2, double ph, Cpx<double> h[12]) {
  Cpx<double> psi[12], u[9];
#pragma unroll
  for (int comp = 0; comp < 12; comp++) {
    if (comp / 6 == ch2) {
      const float2 a = nv[nidx(m, k2, Bn, tn, comp)];
      psi[comp] = Cpx<double>(a.x, a.y);
    } else {
      psi[comp] = Cpx<double>(0, 0);
    }
  }
  link_load<GSOA64, double>(U, MU, FWD ? par : 1 - par, FWD ? s : n, u);
#pragma unroll
  for (int q = 0; q < 12; q++) h[q] = Cpx<double>(0, 0);
  hop<MU, FWD, MU == 3, double>(h, psi, u, ph);
}

// The coarse operator (yidx), column j = d nc + col, d = 0..7 the directions
// (Y_d), d = 8 the self block X; col = ch2 nvec + k2 (the vector acted on),
// row = ch nvec + k:
//   Y_d = -kappa sum_{x in B, x +- mu outside B} v_row(x)^dag [D_d v_col](x)
//   X   = sum_{x in B} v_row^dag A v_col - kappa sum_{x, x +- mu in B} v_row^dag [D_d v_col](x)
// One thread block per aggregate, one thread per site; sums by warp shuffles,
// then over the warps in shared memory.
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_build(MGGeom m, GaugeView<GSOA64> U, CloverView<CSOA64> A0,
                                                        CloverView<CSOA64> A1, int clover, double t_bc,
                                                        double kappa, const float2 *nv, float2 *Y) {
  __shared__ double red[MG_MAXBLOCK / 32][MG_MAXVEC][8];
  __shared__ double2 xs[2 * MG_MAXVEC][2 * MG_MAXVEC];
  const int B = blockIdx.x;
  const int nc = m.nc, nvec = m.nvec;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int t = threadIdx.x;
  const SiteC c = mg_site(m, B, t);
  for (int i = threadIdx.x; i < nc * nc; i += blockDim.x) xs[i / nc][i % nc] = make_double2(0, 0);
  __syncthreads();
  for (int d = 0; d < 9; d++) {
    int n = 0, inblock = 1, Bn = B, tn = t;
    double ph = 1.0;
    if (d < 8) {
      const int mu = d >> 1;
      const bool fwd = !(d & 1);
      int y[4] = {c.x[0], c.x[1], c.x[2], c.x[3]};
      y[mu] = fwd ? (y[mu] + 1) % m.L[mu] : (y[mu] + m.L[mu] - 1) % m.L[mu];
      n = ((y[3] * m.L[2] + y[2]) * m.L[1] + y[1]) * (m.L[0] / 2) + (y[0] >> 1);
      Bn = mg_block_of(m, y);
      tn = mg_local(m, y);
      inblock = Bn == B;
      if (mu == 3 && ((fwd && c.x[3] == m.L[3] - 1) || (!fwd && c.x[3] == 0))) ph = t_bc;
    }
    for (int col = 0; col < nc; col++) {
      const int ch2 = col / nvec, k2 = col % nvec;
      Cpx<double> h[12];
      switch (d) {
        case 0: mg_hop<0, true>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 1: mg_hop<0, false>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 2: mg_hop<1, true>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 3: mg_hop<1, false>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 4: mg_hop<2, true>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 5: mg_hop<2, false>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 6: mg_hop<3, true>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        case 7: mg_hop<3, false>(m, U, nv, c.par, c.s, n, Bn, tn, k2, ch2, ph, h); break;
        default:  // the local term A v_col (v_col itself without clover)
#pragma unroll
          for (int comp = 0; comp < 12; comp++) {
            if (comp / 6 == ch2) {
              const float2 a = nv[nidx(m, k2, B, t, comp)];
              h[comp] = Cpx<double>(a.x, a.y);
            } else {
              h[comp] = Cpx<double>(0, 0);
            }
          }
          if (clover) clover_apply_site<CSOA64, double>(c.par ? A1 : A0, c.s, h);
          break;
      }
      for (int k = 0; k < nvec; k++) {
        double p[4] = {0, 0, 0, 0};  // Re, Im of v_k^dag h on chirality 0, then 1
#pragma unroll
        for (int comp = 0; comp < 12; comp++) {
          const int ch = comp / 6;
          const float2 a = nv[nidx(m, k, B, t, comp)];
          p[2 * ch] += (double)a.x * h[comp].re + (double)a.y * h[comp].im;
          p[2 * ch + 1] += (double)a.x * h[comp].im - (double)a.y * h[comp].re;
        }
        double q[8];  // [0..3]: hops that stay in B (and the local term), [4..7]: hops that leave it
#pragma unroll
        for (int i = 0; i < 4; i++) {
          q[i] = inblock ? p[i] : 0.0;
          q[4 + i] = inblock ? 0.0 : p[i];
        }
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) q[i] += __shfl_xor_sync(0xffffffffu, q[i], o);
        if (lane == 0)
#pragma unroll
          for (int i = 0; i < 8; i++) red[w][k][i] = q[i];
      }
      __syncthreads();
      for (int i = threadIdx.x; i < 8 * nvec; i += blockDim.x) {
        const int k = i >> 3, j = i & 7;
        double tot = 0;
        for (int q = 0; q < nw; q++) tot += red[q][k][j];
        const int leaves = j >> 2, ch = (j >> 1) & 1, im = j & 1;
        const int row = ch * nvec + k;
        const double val = d == 8 ? tot : -kappa * tot;
        if (!leaves) {
          double *x = im ? &xs[col][row].y : &xs[col][row].x;
          *x += val;  // one writer per (row, Re/Im)
        } else if (d < 8) {
          float *y = reinterpret_cast<float *>(Y + yidx(m, B, d * nc + col, row));
          y[im] = (float)val;
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < nc * nc; i += blockDim.x) {
    const double2 v = xs[i / nc][i % nc];
    Y[yidx(m, B, 8 * nc + i / nc, i % nc)] = make_float2((float)v.x, (float)v.y);
  }
}

// ---------------------------------------------------------------- coarse solve on the device
// BiCGSTAB on A_c with its scalars on the device: every kernel of an
// iteration reads them from CState, one-block finalize kernels update them,
// and a conditional WHILE node of a CUDA graph repeats the iteration until
// `done` (converged, iteration cap, breakdown) -- no host round trip.
struct CState {
  double2 rho_prev, rho, alpha, omega;
  double bb, rr;
  int it, done, status;
  unsigned guard;
  long long total_it;      // iterations summed over the solves since the last reset
  long long total_passes;  // passes of the WHILE body, likewise
};
enum CFin { CFIN_INIT = 0, CFIN_ALPHA = 1, CFIN_OMEGA = 2, CFIN_ITER = 3 };

__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cdiv2(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

constexpr int CAPPLY_WARPS = 8;

// out = A_c in, one warp per aggregate, lane = row; the neighbours' inputs
// staged in shared memory.  MODE 1: block partials of <w, out>; MODE 2: of
// <out, w> and |out|^2 (into part[block * 3 + k]).  Skipped when st says done.
template <int MODE>
__global__ void __launch_bounds__(32 * CAPPLY_WARPS) k_mg_capply(MGGeom m, const float4 *Y, const float2 *in,
                                                               float2 *out, const float2 *w, double *part,
                                                               const CState *st) {
  if (st != nullptr && st->done) return;
  __shared__ float2 xin[CAPPLY_WARPS][9 * 2 * MG_MAXVEC];
  __shared__ double sh[CAPPLY_WARPS * 3];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int B = blockIdx.x * CAPPLY_WARPS + wib;
  const int nc = m.nc, J = 9 * nc;
  double v[3] = {0, 0, 0};
  if (B < m.nblocks) {
    for (int i = lane; i < J; i += 32) {
      const int d = i / nc;
      xin[wib][i] = in[(size_t)mg_cnbr(m, B, d) * nc + (i - d * nc)];
    }
    __syncwarp();
    if (lane < nc) {
      const float4 *Yb = Y + (size_t)B * (J / 2) * nc + lane;
      float re0 = 0.f, im0 = 0.f, re1 = 0.f, im1 = 0.f;
#pragma unroll 4
      for (int jp = 0; jp < J / 2; jp++) {
        const float4 a = __ldg(Yb + (size_t)jp * nc);  // (A[2 jp][row], A[2 jp + 1][row])
        const float2 x0 = xin[wib][2 * jp], x1 = xin[wib][2 * jp + 1];
        re0 = fmaf(a.x, x0.x, fmaf(-a.y, x0.y, re0));
        im0 = fmaf(a.x, x0.y, fmaf(a.y, x0.x, im0));
        re1 = fmaf(a.z, x1.x, fmaf(-a.w, x1.y, re1));
        im1 = fmaf(a.z, x1.y, fmaf(a.w, x1.x, im1));
      }
      const float2 o = make_float2(re0 + re1, im0 + im1);
      out[(size_t)B * nc + lane] = o;
      if (MODE == 1) {
        const float2 a = w[(size_t)B * nc + lane];
        v[0] = (double)a.x * o.x + (double)a.y * o.y;
        v[1] = (double)a.x * o.y - (double)a.y * o.x;
      } else if (MODE == 2) {
        const float2 a = w[(size_t)B * nc + lane];
        v[0] = (double)o.x * a.x + (double)o.y * a.y;
        v[1] = (double)o.x * a.y - (double)o.y * a.x;
        v[2] = (double)o.x * o.x + (double)o.y * o.y;
      }
    }
  }
  if (MODE != 0) {
    mg_block_sum<3>(v, sh);
    if (threadIdx.x == 0)
      for (int k = 0; k < 3; k++) part[(size_t)blockIdx.x * 3 + k] = v[k];
  }
}

// x = 0, p = v = 0, r = rt = b; block partials of |b|^2 (slot 2)
__global__ void __launch_bounds__(MG_RED) k_c_init(int64_t n, const float2 *b, float2 *x, float2 *r, float2 *rt,
                                                 float2 *p, float2 *v, double *part) {
  __shared__ double sh[(MG_RED / 32) * 3];
  double a[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 q = b[i];
    x[i] = p[i] = v[i] = make_float2(0.f, 0.f);
    r[i] = rt[i] = q;
    a[2] += (double)q.x * q.x + (double)q.y * q.y;
  }
  mg_block_sum<3>(a, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[(size_t)blockIdx.x * 3 + k] = a[k];
}

// the scalar steps: sums nparts partials, then updates the state (one block)
__global__ void __launch_bounds__(MG_RED) k_c_fin(CState *st, const double *part, int nparts, int op, double tol2,
                                                int maxit) {
  if (op != CFIN_INIT && st->done) return;
  __shared__ double sh[(MG_RED / 32) * 3];
  double a[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
    for (int k = 0; k < 3; k++) a[k] += part[(size_t)i * 3 + k];
  mg_block_sum<3>(a, sh);
  if (threadIdx.x != 0) return;
  const double2 one = make_double2(1, 0);
  if (op == CFIN_INIT) {
    st->bb = a[2];
    st->rr = a[2];
    st->rho = make_double2(a[2], 0);  // <rt, r> with rt = r = b
    st->rho_prev = st->alpha = st->omega = one;
    st->it = 0;
    st->guard = 0;
    st->done = !(a[2] > 0);
    st->status = st->done ? ST_CONVERGED : ST_RUNNING;
  } else if (op == CFIN_ALPHA) {  // a = <rt, v>
    const double2 rtv = make_double2(a[0], a[1]);
    if (!(rtv.x * rtv.x + rtv.y * rtv.y > 0)) {
      st->done = 1;
      st->status = ST_BREAKDOWN;
    } else {
      st->alpha = cdiv2(st->rho, rtv);
    }
  } else if (op == CFIN_OMEGA) {  // a = <t, s>, |t|^2; omega = 0 when t = 0 (then s = 0 too)
    st->omega = a[2] > 0 ? make_double2(a[0] / a[2], a[1] / a[2]) : make_double2(0, 0);
  } else {  // CFIN_ITER: a = <rt, r>, |r|^2 of the new residual
    st->it++;
    st->total_it++;
    st->rr = a[2];
    st->rho_prev = st->rho;
    st->rho = make_double2(a[0], a[1]);
    if (!(a[2] == a[2])) {
      st->done = 1;
      st->status = ST_NAN;
    } else if (a[2] <= tol2 * st->bb) {
      st->done = 1;
      st->status = ST_CONVERGED;
    } else if (st->it >= maxit) {
      st->done = 1;
      st->status = ST_MAXITER;
    } else if (!(st->rho.x * st->rho.x + st->rho.y * st->rho.y > 0) ||
               !(st->omega.x * st->omega.x + st->omega.y * st->omega.y > 0)) {
      st->done = 1;
      st->status = ST_BREAKDOWN;
    }
  }
}

// p = r + beta (p - omega v), beta = (rho / rho_prev) (alpha / omega)
__global__ void k_c_pupdate(int64_t n, float2 *p, const float2 *r, const float2 *v, const CState *st) {
  if (st->done) return;
  const double2 beta = cmul2(cdiv2(st->rho, st->rho_prev), cdiv2(st->alpha, st->omega));
  const double2 bw = cmul2(beta, st->omega);
  const float br = (float)beta.x, bi = (float)beta.y, wr = (float)bw.x, wi = (float)bw.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 pp = p[i], rr = r[i], vv = v[i];
    p[i] = make_float2(rr.x + br * pp.x - bi * pp.y - wr * vv.x + wi * vv.y,
                       rr.y + br * pp.y + bi * pp.x - wr * vv.y - wi * vv.x);
  }
}

// s = r - alpha v (in r)
__global__ void k_c_supdate(int64_t n, float2 *r, const float2 *v, const CState *st) {
  if (st->done) return;
  const float ar = (float)st->alpha.x, ai = (float)st->alpha.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 rr = r[i], vv = v[i];
    r[i] = make_float2(rr.x - ar * vv.x + ai * vv.y, rr.y - ar * vv.y - ai * vv.x);
  }
}

// x += alpha p + omega s; r = s - omega t; block partials of <rt, r>, |r|^2
__global__ void __launch_bounds__(MG_RED) k_c_xrupdate(int64_t n, float2 *x, const float2 *p, float2 *r,
                                                     const float2 *t, const float2 *rt, const CState *st,
                                                     double *part) {
  if (st->done) return;
  __shared__ double sh[(MG_RED / 32) * 3];
  const float ar = (float)st->alpha.x, ai = (float)st->alpha.y, wr = (float)st->omega.x, wi = (float)st->omega.y;
  double a[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 pp = p[i], ss = r[i], tt = t[i], xx = x[i], q = rt[i];
    x[i] = make_float2(xx.x + ar * pp.x - ai * pp.y + wr * ss.x - wi * ss.y,
                       xx.y + ar * pp.y + ai * pp.x + wr * ss.y + wi * ss.x);
    const float2 rn = make_float2(ss.x - wr * tt.x + wi * tt.y, ss.y - wr * tt.y - wi * tt.x);
    r[i] = rn;
    a[0] += (double)q.x * rn.x + (double)q.y * rn.y;
    a[1] += (double)q.x * rn.y - (double)q.y * rn.x;
    a[2] += (double)rn.x * rn.x + (double)rn.y * rn.y;
  }
  mg_block_sum<3>(a, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[(size_t)blockIdx.x * 3 + k] = a[k];
}

// the WHILE node's condition: another pass while not done (at most cap passes)
__global__ void k_c_cond(CState *st, cudaGraphConditionalHandle h, unsigned cap) {
  const unsigned g = ++st->guard;
  st->total_passes++;
  bool go = st->done == 0;
  if (go && g >= cap) {
    st->done = 1;
    st->status = ST_MAXITER;
    go = false;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ---------------------------------------------------------------- vector kernels
// out = a x + b y + c z (complex scalars; y, z may be null), n complex numbers
template <typename V>
__global__ void k_mg_lin3(int64_t n, V *out, double2 a, const V *x, double2 b, const V *y, double2 c, const V *z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double xr = x[i].x, xi = x[i].y;
    double re = a.x * xr - a.y * xi, im = a.x * xi + a.y * xr;
    if (y) {
      const double yr = y[i].x, yi = y[i].y;
      re += b.x * yr - b.y * yi;
      im += b.x * yi + b.y * yr;
    }
    if (z) {
      const double zr = z[i].x, zi = z[i].y;
      re += c.x * zr - c.y * zi;
      im += c.x * zi + c.y * zr;
    }
    out[i].x = re;
    out[i].y = im;
  }
}
// per-block partials of Re<a,b>, Im<a,b>, |a|^2 (<a,b> = sum conj(a) b)
template <typename V>
__global__ void __launch_bounds__(MG_RED) k_mg_dots(int64_t n, const V *a, const V *b, double *part) {
  __shared__ double sh[(MG_RED / 32) * 3];
  double v[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ax = a[i].x, ay = a[i].y, bx = b[i].x, by = b[i].y;
    v[0] += ax * bx + ay * by;
    v[1] += ax * by - ay * bx;
    v[2] += ax * ax + ay * ay;
  }
  mg_block_sum<3>(v, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[blockIdx.x * 3 + k] = v[k];
}
// x += a y; r -= a w (the MR and GCR updates in one pass)
__global__ void k_mg_axpy2(int64_t n, double2 *x, const double2 *y, double2 *r, const double2 *w, double2 a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 yy = y[i], ww = w[i], xx = x[i], rr = r[i];
    x[i] = make_double2(xx.x + a.x * yy.x - a.y * yy.y, xx.y + a.x * yy.y + a.y * yy.x);
    r[i] = make_double2(rr.x - a.x * ww.x + a.y * ww.y, rr.y - a.x * ww.y - a.y * ww.x);
  }
}
// flexible GCR orthogonalisation, up to MG_CHUNK earlier directions per pass
constexpr int MG_CHUNK = 8;
struct Dirs {
  const double2 *p[MG_CHUNK];
  double2 c[MG_CHUNK];
};
// block partials of <W_i, w>, i < cnt: part[block * 2 MG_CHUNK + 2 i + (0 Re, 1 Im)]
__global__ void __launch_bounds__(MG_RED) k_mg_multidot(int64_t n, Dirs W, int cnt, const double2 *w, double *part) {
  __shared__ double sh[(MG_RED / 32) * 2 * MG_CHUNK];
  double v[2 * MG_CHUNK];
#pragma unroll
  for (int i = 0; i < 2 * MG_CHUNK; i++) v[i] = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double2 b = w[e];
#pragma unroll
    for (int i = 0; i < MG_CHUNK; i++) {
      if (i < cnt) {
        const double2 a = W.p[i][e];
        v[2 * i] += a.x * b.x + a.y * b.y;
        v[2 * i + 1] += a.x * b.y - a.y * b.x;
      }
    }
  }
  mg_block_sum<2 * MG_CHUNK>(v, sh);
  if (threadIdx.x == 0)
    for (int i = 0; i < 2 * MG_CHUNK; i++) part[(size_t)blockIdx.x * 2 * MG_CHUNK + i] = v[i];
}
// out -= sum_{i < cnt} c_i W_i
__global__ void k_mg_multiaxpy(int64_t n, double2 *out, Dirs W, int cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double2 o = out[e];
#pragma unroll
    for (int i = 0; i < MG_CHUNK; i++) {
      if (i < cnt) {
        const double2 a = W.p[i][e], c = W.c[i];
        o.x -= c.x * a.x - c.y * a.y;
        o.y -= c.x * a.y + c.y * a.x;
      }
    }
    out[e] = o;
  }
}

// one parity (SOA64 half spinors, the Vh real sites only): block partials of <a, b>, |a|^2
__global__ void __launch_bounds__(MG_RED) k_mg_half_dots(int Vh, const double2 *a, const double2 *b, double *part) {
  __shared__ double sh[(MG_RED / 32) * 3];
  double v[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)Vh * 12;
       i += (int64_t)gridDim.x * blockDim.x) {
    const size_t k = hidx((int)(i / 12), (int)(i % 12));
    const double2 x = a[k], y = b[k];
    v[0] += x.x * y.x + x.y * y.y;
    v[1] += x.x * y.y - x.y * y.x;
    v[2] += x.x * x.x + x.y * x.y;
  }
  mg_block_sum<3>(v, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[blockIdx.x * 3 + k] = v[k];
}
// z *= alpha; q = r - alpha q (one parity)
__global__ void k_mg_half_mr(int Vh, double2 *z, double2 *q, const double2 *r, double2 al) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)Vh * 12;
       i += (int64_t)gridDim.x * blockDim.x) {
    const size_t k = hidx((int)(i / 12), (int)(i % 12));
    const double2 zz = z[k], qq = q[k], rr = r[k];
    z[k] = make_double2(al.x * zz.x - al.y * zz.y, al.x * zz.y + al.y * zz.x);
    q[k] = make_double2(rr.x - (al.x * qq.x - al.y * qq.y), rr.y - (al.x * qq.y + al.y * qq.x));
  }
}
// near-null vector k (FP32, aggregate-major) from a full FP64 vector
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_store_nv(MGGeom m, int k, const double2 *v, float2 *nv) {
  const int B = blockIdx.x, t = threadIdx.x;
  const SiteC c = mg_site(m, B, t);
#pragma unroll
  for (int comp = 0; comp < 12; comp++) {
    const double2 a = v[fidx(m, c.par, c.s, comp)];
    nv[nidx(m, k, B, t, comp)] = make_float2((float)a.x, (float)a.y);
  }
}

int mg_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + MG_RED - 1) / MG_RED, MG_RED_GRID));
}

}  // namespace

// ---------------------------------------------------------------- host
struct MG {
  GaugeHandle *G = nullptr;
  double kappa = 0;
  MGParams p;
  MGGeom m;
  int device = 0;
  DevBuf nv, Y;  // near-null vectors (FP32 full vectors), coarse operator (FP32)
  DevBuf part;   // reduction partials
  std::vector<double> part_h;
  // FP64 full vectors: b, x, r; s, q (the smoother); e1 (scratch of mg_check); tmp (one parity, A in)
  DevBuf b, x, r, e1, s, q, tmp;
  std::vector<std::unique_ptr<DevBuf>> Z, W;  // flexible GCR directions
  // coarse FP32 vectors
  DevBuf cb, cx, cr, crt, cp, cv, ct;
  DevBuf cstate;                        // CState of the coarse solve
  cudaGraphExec_t coarse = nullptr;     // the coarse solve cb -> cx as one graph
  long long coarse_cycles = 0;          // coarse solves launched since the last reset
  double setup_seconds = 0;

  int64_t nfull() const { return (int64_t)2 * m.Vp * 12; }
  int64_t ncoarse() const { return (int64_t)m.nblocks * m.nc; }
  ~MG() {
    if (coarse) cudaGraphExecDestroy(coarse);
  }
};

namespace {

using C = Cpx<double>;
double2 *f64(DevBuf &d) { return d.as<double2>(); }
float2 *f32(DevBuf &d) { return d.as<float2>(); }
// the parity slabs of a full vector
FineVec slabs(const MG &mg, const double2 *v) {
  double2 *p = const_cast<double2 *>(v);
  return FineVec{{p, p + (size_t)mg.m.Vp * 12}};
}

template <typename V>
void dots(MG &mg, cudaStream_t st, int64_t n, const V *a, const V *b, double out[3]) {
  const int gr = mg_grid(n);
  k_mg_dots<V><<<gr, MG_RED, 0, st>>>(n, a, b, mg.part.as<double>());
  QCU_CHECK_LAUNCH();
  QCU_CUDA(cudaMemcpyAsync(mg.part_h.data(), mg.part.p, (size_t)gr * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QCU_CUDA(cudaStreamSynchronize(st));
  out[0] = out[1] = out[2] = 0;
  for (int i = 0; i < gr; i++)
    for (int k = 0; k < 3; k++) out[k] += mg.part_h[(size_t)i * 3 + k];
}

template <typename V>
void lin3(cudaStream_t st, int64_t n, V *out, C a, const V *x, C b = C(0, 0), const V *y = nullptr, C c = C(0, 0),
          const V *z = nullptr) {
  k_mg_lin3<V><<<mg_grid(n), MG_RED, 0, st>>>(n, out, make_double2(a.re, a.im), x, make_double2(b.re, b.im), y,
                                             make_double2(c.re, c.im), z);
  QCU_CHECK_LAUNCH();
}

// out = M in on full FP64 vectors: out_p = A_p in_p - kappa D_{p <- 1-p} in_{1-p}
void mat(MG &mg, Context &ctx, const double2 *in, double2 *out) {
  const GaugeHandle &G = *mg.G;
  const size_t half = (size_t)mg.m.Vp * 12;
  for (int p = 0; p < 2; p++) {
    DslashArgs d;
    d.gauge = G.g64.p;
    d.t_bc = G.t_bc;
    d.a = -mg.kappa;
    d.b1 = 1.0;
    d.in = in + (1 - p) * half;
    d.out = out + p * half;
    d.parity = p;
    if (G.has_clover) {
      launch_clover_apply(SOA64, G.g.Vh, G.A64[p].p, in + p * half, mg.tmp.p, ctx.stream);
      d.x1 = mg.tmp.p;
    } else {
      d.x1 = in + p * half;
    }
    launch_dslash(SOA64, GSOA64, CSOA64, G.g, d, ctx, ctx.stream);
  }
}

int capply_grid(const MG &mg) { return (mg.m.nblocks + CAPPLY_WARPS - 1) / CAPPLY_WARPS; }

// out = A_c in (no reduction)
// out = b - M e on full FP64 vectors in one dslash pass per parity:
// out_p = kappa D_{p <- 1-p} e_{1-p} + b_p - A_p e_p
void residual(MG &mg, Context &ctx, const double2 *e, const double2 *b, double2 *out) {
  const GaugeHandle &G = *mg.G;
  const size_t half = (size_t)mg.m.Vp * 12;
  for (int p = 0; p < 2; p++) {
    DslashArgs d;
    d.gauge = G.g64.p;
    d.t_bc = G.t_bc;
    d.a = mg.kappa;
    d.in = e + (1 - p) * half;
    d.out = out + p * half;
    d.parity = p;
    d.x1 = b + p * half;
    d.b1 = 1.0;
    if (G.has_clover) {
      launch_clover_apply(SOA64, G.g.Vh, G.A64[p].p, e + p * half, mg.tmp.p, ctx.stream);
      d.x2 = mg.tmp.p;
    } else {
      d.x2 = e + p * half;
    }
    d.b2 = -1.0;
    launch_dslash(SOA64, GSOA64, CSOA64, G.g, d, ctx, ctx.stream);
  }
}

void capply(MG &mg, cudaStream_t st, const float2 *in, float2 *out) {
  k_mg_capply<0><<<capply_grid(mg), 32 * CAPPLY_WARPS, 0, st>>>(mg.m, mg.Y.as<float4>(), in, out, nullptr, nullptr,
                                                                nullptr);
  QCU_CHECK_LAUNCH();
}

constexpr int COARSE_KERNELS_PER_PASS = 9;

// The coarse solve cx ~ A_c^-1 cb as a graph: init, then a WHILE node whose
// body is one BiCGSTAB iteration (FP32 vectors, FP64 scalars in CState) to
// |r| <= coarse_tol |b| or coarse_maxiter iterations.
void capture_coarse(MG &mg, Context &ctx) {
  cudaStream_t st = ctx.stream;
  const int64_t n = mg.ncoarse();
  const int gv = mg_grid(n), ga = capply_grid(mg);
  CState *cs = mg.cstate.as<CState>();
  double *part = mg.part.as<double>();
  const double tol2 = mg.p.coarse_tol * mg.p.coarse_tol;
  const int maxit = mg.p.coarse_maxiter;
  float2 *b = f32(mg.cb), *x = f32(mg.cx), *r = f32(mg.cr), *rt = f32(mg.crt), *p = f32(mg.cp), *v = f32(mg.cv),
         *t = f32(mg.ct);
  const float4 *Y = mg.Y.as<float4>();
  const auto mode = cudaStreamCaptureModeThreadLocal;
  const long long before = launch_count();
  cudaGraph_t g = nullptr;
  QCU_CUDA(cudaGraphCreate(&g, 0));
  try {
    QCU_CUDA(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode));
    k_c_init<<<gv, MG_RED, 0, st>>>(n, b, x, r, rt, p, v, part);
    QCU_CHECK_LAUNCH();
    k_c_fin<<<1, MG_RED, 0, st>>>(cs, part, gv, CFIN_INIT, tol2, maxit);
    QCU_CHECK_LAUNCH();
    QCU_CUDA(cudaStreamEndCapture(st, &g));
    size_t nn = 0;
    QCU_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    require(nn == 2, "mg: unexpected coarse-solve init capture");
    std::vector<cudaGraphNode_t> nodes(nn);
    QCU_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    cudaGraphNode_t last = nodes[0];  // the node without dependents (the finalize)
    for (cudaGraphNode_t nd : nodes) {
      size_t nd_out = 0;
      QCU_CUDA(cudaGraphNodeGetDependentNodes(nd, nullptr, &nd_out));
      if (nd_out == 0) last = nd;
    }
    cudaGraphConditionalHandle h;
    QCU_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop;
    QCU_CUDA(cudaGraphAddNode(&loop, g, &last, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    QCU_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode));
    k_c_pupdate<<<gv, MG_RED, 0, st>>>(n, p, r, v, cs);
    QCU_CHECK_LAUNCH();
    k_mg_capply<1><<<ga, 32 * CAPPLY_WARPS, 0, st>>>(mg.m, Y, p, v, rt, part, cs);
    QCU_CHECK_LAUNCH();
    k_c_fin<<<1, MG_RED, 0, st>>>(cs, part, ga, CFIN_ALPHA, tol2, maxit);
    QCU_CHECK_LAUNCH();
    k_c_supdate<<<gv, MG_RED, 0, st>>>(n, r, v, cs);
    QCU_CHECK_LAUNCH();
    k_mg_capply<2><<<ga, 32 * CAPPLY_WARPS, 0, st>>>(mg.m, Y, r, t, r, part, cs);
    QCU_CHECK_LAUNCH();
    k_c_fin<<<1, MG_RED, 0, st>>>(cs, part, ga, CFIN_OMEGA, tol2, maxit);
    QCU_CHECK_LAUNCH();
    k_c_xrupdate<<<gv, MG_RED, 0, st>>>(n, x, p, r, t, rt, cs, part);
    QCU_CHECK_LAUNCH();
    k_c_fin<<<1, MG_RED, 0, st>>>(cs, part, gv, CFIN_ITER, tol2, maxit);
    QCU_CHECK_LAUNCH();
    k_c_cond<<<1, 1, 0, st>>>(cs, h, (unsigned)maxit + 2u);
    QCU_CHECK_LAUNCH();
    QCU_CUDA(cudaStreamEndCapture(st, &body));
    QCU_CUDA(cudaGraphInstantiate(&mg.coarse, g, 0));
  } catch (...) {
    cudaStreamCaptureStatus csx;
    if (cudaStreamIsCapturing(st, &csx) == cudaSuccess && csx != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk;
      cudaStreamEndCapture(st, &junk);
    }
    cudaGetLastError();
    cudaGraphDestroy(g);
    set_launch_count(before);
    throw;
  }
  cudaGraphDestroy(g);
  set_launch_count(before);  // replays are counted from the passes the state records
}

// cx ~ A_c^-1 cb on the device
void coarse_solve(MG &mg, cudaStream_t st) {
  QCU_CUDA(cudaGraphLaunch(mg.coarse, st));
  mg.coarse_cycles++;
}

void axpy2(cudaStream_t st, int64_t n, double2 *x, const double2 *y, double2 *r, const double2 *w, C a) {
  k_mg_axpy2<<<mg_grid(n), MG_RED, 0, st>>>(n, x, y, r, w, make_double2(a.re, a.im));
  QCU_CHECK_LAUNCH();
}

// steps MR iterations on M e = r from e (start: s = r - M e, or s = r when
// e = 0); s = r - M e on return
void smooth(MG &mg, Context &ctx, const double2 *r, double2 *e, int steps, bool e_zero) {
  cudaStream_t st = ctx.stream;
  const int64_t n = mg.nfull();
  double2 *s = f64(mg.s), *q = f64(mg.q);
  if (e_zero) {
    QCU_CUDA(cudaMemsetAsync(e, 0, (size_t)n * sizeof(double2), st));
    QCU_CUDA(cudaMemcpyAsync(s, r, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  } else {
    residual(mg, ctx, e, r, s);
  }
  for (int k = 0; k < steps; k++) {
    mat(mg, ctx, s, q);
    double d[3];
    dots(mg, st, n, q, s, d);  // <M s, s>, |M s|^2
    if (!(d[2] > 0)) break;
    axpy2(st, n, e, s, s, q, C(d[0] / d[2], d[1] / d[2]));
  }
}

// e = K r: nu_pre MR steps, the coarse correction, nu_post MR steps
void cycle(MG &mg, Context &ctx, const double2 *r, double2 *e) {
  cudaStream_t st = ctx.stream;
  const MGGeom &m = mg.m;
  const int64_t n = mg.nfull();
  const float2 *nv = mg.nv.as<float2>();
  const double2 *rc = r;  // the residual the coarse grid sees
  if (mg.p.nu_pre > 0) {
    smooth(mg, ctx, r, e, mg.p.nu_pre, true);
    rc = f64(mg.s);  // r - M e
  }
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, slabs(mg, rc), f32(mg.cb));
  QCU_CHECK_LAUNCH();
  coarse_solve(mg, st);
  k_mg_prolong<<<m.nblocks, m.bsites, 0, st>>>(m, nv, f32(mg.cx), slabs(mg, e), mg.p.nu_pre > 0 ? 1 : 0);
  QCU_CHECK_LAUNCH();
  if (mg.p.nu_post > 0) smooth(mg, ctx, r, e, mg.p.nu_post, false);
}

}  // namespace

MG *mg_create(GaugeHandle &G, double kappa, const MGParams &p) {
  const auto t0 = std::chrono::steady_clock::now();
  require(kappa > 0, "mg: kappa must be positive");
  require(p.n_vec >= 1 && p.n_vec <= MG_MAXVEC, "mg: n_vec must be 1.." + std::to_string(MG_MAXVEC));
  require(p.gcr_k >= 1 && p.gcr_k <= 32, "mg: gcr_k must be 1..32");
  require(p.nu_pre >= 0 && p.nu_post >= 0 && p.coarse_maxiter >= 1 && p.setup_maxiter >= 1 && p.coarse_tol > 0,
          "mg: nu_pre, nu_post >= 0, coarse_maxiter, setup_maxiter >= 1 and coarse_tol > 0 are required");
  auto mg = std::make_unique<MG>();
  mg->G = &G;
  mg->kappa = kappa;
  mg->p = p;
  MGGeom &m = mg->m;
  for (int d = 0; d < 4; d++) {
    m.L[d] = G.latt[d];
    m.b[d] = p.geo_block_size[d];
    require(m.b[d] >= 1 && m.L[d] % m.b[d] == 0, "mg: every block extent must divide the lattice extent");
    m.nb[d] = m.L[d] / m.b[d];
  }
  require(m.b[0] % 2 == 0, "mg: the x block extent must be even");
  m.nblocks = m.nb[0] * m.nb[1] * m.nb[2] * m.nb[3];
  m.bsites = m.b[0] * m.b[1] * m.b[2] * m.b[3];
  require(m.bsites % 32 == 0 && m.bsites <= MG_MAXBLOCK,
          "mg: sites per block must be a multiple of 32 and at most " + std::to_string(MG_MAXBLOCK));
  m.Vh = G.g.Vh;
  m.Vp = pad_sites(G.g.Vh);
  m.nvec = p.n_vec;
  m.nc = 2 * p.n_vec;
  const int Vh = m.Vh;
  const int clov = G.has_clover ? 1 : 0;
  Context &ctx = context();
  mg->device = ctx.device;
  {
    std::lock_guard<std::mutex> lk(ctx.mu);
    const size_t full = (size_t)mg->nfull() * sizeof(double2);
    const size_t cfull = (size_t)mg->ncoarse() * sizeof(float2);
    mg->nv.ensure((size_t)m.nvec * mg->nfull() * sizeof(float2));
    mg->Y.ensure((size_t)m.nblocks * 9 * m.nc * m.nc * sizeof(float2));
    mg->part.ensure((size_t)std::max(MG_RED_GRID * 2 * MG_CHUNK, capply_grid(*mg) * 3) * sizeof(double));
    mg->cstate.ensure(sizeof(CState));
    QCU_CUDA(cudaMemsetAsync(mg->cstate.p, 0, sizeof(CState), ctx.stream));
    mg->part_h.resize((size_t)MG_RED_GRID * 2 * MG_CHUNK);
    for (DevBuf *d : {&mg->b, &mg->x, &mg->r, &mg->e1, &mg->s, &mg->q}) d->ensure(full);
    mg->tmp.ensure(full / 2);
    for (int k = 0; k < p.gcr_k; k++) {
      mg->Z.emplace_back(new DevBuf);
      mg->W.emplace_back(new DevBuf);
      mg->Z.back()->ensure(full);
      mg->W.back()->ensure(full);
    }
    for (DevBuf *d : {&mg->cb, &mg->cx, &mg->cr, &mg->crt, &mg->cp, &mg->cv, &mg->ct}) d->ensure(cfull);
    // the padding sites of the full vectors stay zero throughout
    for (DevBuf *d : {&mg->b, &mg->x, &mg->r, &mg->e1, &mg->s, &mg->q}) QCU_CUDA(cudaMemsetAsync(d->p, 0, full, ctx.stream));
    for (int k = 0; k < p.gcr_k; k++) {
      QCU_CUDA(cudaMemsetAsync(mg->Z[k]->p, 0, full, ctx.stream));
      QCU_CUDA(cudaMemsetAsync(mg->W[k]->p, 0, full, ctx.stream));
    }
    QCU_CUDA(cudaMemsetAsync(mg->nv.p, 0, mg->nv.n, ctx.stream));
    QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  }
  // near-null vectors: v = v0 - y, y a short solve of M y = M v0 (PyQuda-layout buffers)
  {
    const size_t half_pyq = spinor_bytes(AOS64, Vh);
    DevBuf v0, bq, yq;
    {
      std::lock_guard<std::mutex> lk(ctx.mu);
      v0.ensure(2 * half_pyq);
      bq.ensure(2 * half_pyq);
      yq.ensure(2 * half_pyq);
    }
    SolveParams sp;
    sp.kappa = kappa;
    sp.tol = 1e-30;  // never met: the solve stops after setup_maxiter iterations
    sp.maxiter = p.setup_maxiter;
    sp.precision = 32;
    sp.solver = 0;
    sp.use_clover = clov;
    for (int k = 0; k < m.nvec; k++) {
      {
        std::lock_guard<std::mutex> lk(ctx.mu);
        launch_fermion_random(v0.p, (int64_t)Vh * 24, 0, 0x6d670000ULL + 7919ULL * (k + 1), ctx.stream);
        QCU_CUDA(cudaStreamSynchronize(ctx.stream));
      }
      handle_mat(G, bq.p, v0.p, kappa, clov);
      solve(G, yq.p, bq.p, sp);
      std::lock_guard<std::mutex> lk(ctx.mu);
      cudaStream_t st = ctx.stream;
      double2 *vf = f64(mg->b), *yf = f64(mg->x);
      const size_t half = (size_t)m.Vp * 12;
      for (int par = 0; par < 2; par++) {
        launch_convert(AOS64, SOA64, Vh, static_cast<char *>(v0.p) + par * half_pyq, nullptr, vf + par * half,
                       nullptr, st);
        launch_convert(AOS64, SOA64, Vh, static_cast<char *>(yq.p) + par * half_pyq, nullptr, yf + par * half,
                       nullptr, st);
      }
      const int64_t n = mg->nfull();
      lin3(st, n, vf, C(1, 0), vf, C(-1, 0), yf);
      k_mg_store_nv<<<m.nblocks, m.bsites, 0, st>>>(m, k, vf, mg->nv.as<float2>());
      QCU_CHECK_LAUNCH();
      QCU_CUDA(cudaStreamSynchronize(st));
    }
  }
  std::lock_guard<std::mutex> lk(ctx.mu);
  cudaStream_t st = ctx.stream;
  k_mg_orth<<<m.nblocks, m.bsites, 0, st>>>(m, mg->nv.as<float2>());
  QCU_CHECK_LAUNCH();
  const CloverView<CSOA64> A0{clov ? G.A64[0].p : nullptr, Vh}, A1{clov ? G.A64[1].p : nullptr, Vh};
  k_mg_build<<<m.nblocks, m.bsites, 0, st>>>(m, GaugeView<GSOA64>{G.g64.p, m.Vp}, A0, A1, clov, G.t_bc, kappa,
                                             mg->nv.as<float2>(), mg->Y.as<float2>());
  QCU_CHECK_LAUNCH();
  QCU_CUDA(cudaStreamSynchronize(st));
  capture_coarse(*mg, ctx);
  mg->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return mg.release();
}

void mg_free(MG *mg) { delete mg; }

void mg_require_compatible(const MG &mg, const GaugeHandle &G, double kappa, int use_clover) {
  require(mg.G == &G, "mg: the multigrid was built on another gauge handle");
  require(mg.kappa == kappa, "mg: the multigrid was built for another kappa");
  require((use_clover != 0) == G.has_clover,
          "mg: the multigrid's operator includes the handle's clover term exactly when it has one");
  require(context().device == mg.device, "mg: the multigrid was set up on another device");
}

void mg_coarse_odd(MG &mg, Context &ctx, const void *r_odd, void *z_odd) {
  cudaStream_t st = ctx.stream;
  const MGGeom &m = mg.m;
  const GaugeHandle &G = *mg.G;
  const double2 *src = static_cast<const double2 *>(r_odd);
  if (G.has_clover) {  // M_pc = A_o^-1 S: S^-1 acts on A_o r
    launch_clover_apply(SOA64, G.g.Vh, G.A64[1].p, r_odd, mg.tmp.p, st);
    src = mg.tmp.as<double2>();
  }
  const float2 *nv = mg.nv.as<float2>();
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, FineVec{{nullptr, const_cast<double2 *>(src)}},
                                                f32(mg.cb));
  QCU_CHECK_LAUNCH();
  coarse_solve(mg, st);
  k_mg_prolong<<<m.nblocks, m.bsites, 0, st>>>(m, nv, f32(mg.cx), FineVec{{nullptr, static_cast<double2 *>(z_odd)}},
                                               0);
  QCU_CHECK_LAUNCH();
}

double2 mg_minres_scale(MG &mg, Context &ctx, void *z, void *q, const void *r) {
  cudaStream_t st = ctx.stream;
  const int Vh = mg.m.Vh;
  const int gr = mg_grid((int64_t)Vh * 12);
  k_mg_half_dots<<<gr, MG_RED, 0, st>>>(Vh, static_cast<const double2 *>(q), static_cast<const double2 *>(r),
                                        mg.part.as<double>());
  QCU_CHECK_LAUNCH();
  QCU_CUDA(cudaMemcpyAsync(mg.part_h.data(), mg.part.p, (size_t)gr * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QCU_CUDA(cudaStreamSynchronize(st));
  double d[3] = {0, 0, 0};
  for (int i = 0; i < gr; i++)
    for (int k = 0; k < 3; k++) d[k] += mg.part_h[(size_t)i * 3 + k];
  const double2 al = d[2] > 0 ? make_double2(d[0] / d[2], d[1] / d[2]) : make_double2(0, 0);
  k_mg_half_mr<<<gr, MG_RED, 0, st>>>(Vh, static_cast<double2 *>(z), static_cast<double2 *>(q),
                                      static_cast<const double2 *>(r), al);
  QCU_CHECK_LAUNCH();
  return al;
}

long long mg_take_launches(MG &mg, Context &ctx) {
  CState cs;
  QCU_CUDA(cudaMemcpyAsync(&cs, mg.cstate.p, sizeof(CState), cudaMemcpyDeviceToHost, ctx.stream));
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  const long long n = 2 * mg.coarse_cycles + COARSE_KERNELS_PER_PASS * cs.total_passes;
  QCU_CUDA(cudaMemsetAsync(mg.cstate.p, 0, sizeof(CState), ctx.stream));
  mg.coarse_cycles = 0;
  return n;
}

double mg_setup_seconds(const MG &mg) { return mg.setup_seconds; }

MGInfo mg_solve(MG &mg, void *x_pyq, const void *b_pyq, double tol, int maxiter) {
  require(x_pyq != nullptr && b_pyq != nullptr, "mg: null spinor pointer");
  require(tol > 0 && maxiter > 0, "mg: tol and maxiter must be positive");
  const auto t0 = std::chrono::steady_clock::now();
  Context &ctx = context();
  require(ctx.device == mg.device, "mg: the multigrid was set up on another device");
  std::lock_guard<std::mutex> lk(ctx.mu);
  QCU_CUDA(cudaDeviceSynchronize());  // inputs written on any stream are complete
  cudaStream_t st = ctx.stream;
  const MGGeom &m = mg.m;
  const int Vh = m.Vh;
  const size_t half = (size_t)m.Vp * 12, half_pyq = spinor_bytes(AOS64, Vh);
  const int64_t n = mg.nfull();
  double2 *b = f64(mg.b), *x = f64(mg.x), *r = f64(mg.r);
  for (int par = 0; par < 2; par++)
    launch_convert(AOS64, SOA64, Vh, static_cast<const char *>(b_pyq) + par * half_pyq, nullptr, b + par * half,
                   nullptr, st);
  QCU_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double2), st));
  QCU_CUDA(cudaMemcpyAsync(r, b, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  MGInfo info;
  mg.coarse_cycles = 0;
  QCU_CUDA(cudaMemsetAsync(mg.cstate.p, 0, sizeof(CState), st));
  double d[3];
  dots(mg, st, n, b, b, d);
  const double bb = d[2];
  if (bb == 0.0) {
    QCU_CUDA(cudaMemsetAsync(x_pyq, 0, 2 * half_pyq, st));
    QCU_CUDA(cudaStreamSynchronize(st));
    info.status = ST_CONVERGED;
    return info;
  }
  const double target = tol * tol * bb;
  double rr = bb;
  std::vector<double> nw(mg.p.gcr_k);  // |w_j|^2
  info.status = ST_MAXITER;
  while (info.outer < maxiter) {
    for (int j = 0; j < mg.p.gcr_k && info.outer < maxiter; j++) {
      double2 *z = f64(*mg.Z[j]), *w = f64(*mg.W[j]);
      cycle(mg, ctx, r, z);
      mat(mg, ctx, z, w);
      // w_j -= sum_i <w_i, w_j> / |w_i|^2 w_i, z_j likewise; in chunks of
      // MG_CHUNK directions (Gram-Schmidt by blocks)
      for (int i0 = 0; i0 < j; i0 += MG_CHUNK) {
        const int cnt = std::min(MG_CHUNK, j - i0);
        Dirs Wd{}, Zd{};
        for (int i = 0; i < cnt; i++) {
          Wd.p[i] = f64(*mg.W[i0 + i]);
          Zd.p[i] = f64(*mg.Z[i0 + i]);
        }
        const int gr = mg_grid(n);
        k_mg_multidot<<<gr, MG_RED, 0, st>>>(n, Wd, cnt, w, mg.part.as<double>());
        QCU_CHECK_LAUNCH();
        QCU_CUDA(cudaMemcpyAsync(mg.part_h.data(), mg.part.p, (size_t)gr * 2 * MG_CHUNK * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
        QCU_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < cnt; i++) {
          double re = 0, im = 0;
          for (int b = 0; b < gr; b++) {
            re += mg.part_h[(size_t)b * 2 * MG_CHUNK + 2 * i];
            im += mg.part_h[(size_t)b * 2 * MG_CHUNK + 2 * i + 1];
          }
          Wd.c[i] = Zd.c[i] = make_double2(re / nw[i0 + i], im / nw[i0 + i]);
        }
        k_mg_multiaxpy<<<mg_grid(n), MG_RED, 0, st>>>(n, w, Wd, cnt);
        QCU_CHECK_LAUNCH();
        k_mg_multiaxpy<<<mg_grid(n), MG_RED, 0, st>>>(n, z, Zd, cnt);
        QCU_CHECK_LAUNCH();
      }
      dots(mg, st, n, w, r, d);  // <w, r>, |w|^2
      if (!(d[2] > 0) || !(d[0] == d[0]) || !(d[1] == d[1])) {
        info.status = d[2] == d[2] ? ST_BREAKDOWN : ST_NAN;
        break;
      }
      nw[j] = d[2];
      axpy2(st, n, x, z, r, w, C(d[0] / d[2], d[1] / d[2]));  // alpha = <w, r> / |w|^2
      info.outer++;
      rr = std::max(0.0, rr - (d[0] * d[0] + d[1] * d[1]) / d[2]);  // |r - alpha w|^2; the restart recomputes it
      if (rr <= target) break;
    }
    if (info.status == ST_BREAKDOWN || info.status == ST_NAN) break;
    // restart from the FP64 true residual
    residual(mg, ctx, x, b, r);
    dots(mg, st, n, r, r, d);
    rr = d[2];
    if (rr <= target) {
      info.status = ST_CONVERGED;
      break;
    }
  }
  if (info.status == ST_BREAKDOWN || info.status == ST_NAN) {
    residual(mg, ctx, x, b, r);
    dots(mg, st, n, r, r, d);
    rr = d[2];
  }
  info.true_residual = std::sqrt(rr / bb);
  CState cs;
  QCU_CUDA(cudaMemcpyAsync(&cs, mg.cstate.p, sizeof(CState), cudaMemcpyDeviceToHost, st));
  QCU_CUDA(cudaStreamSynchronize(st));
  info.coarse_iters = (int)std::min<long long>(cs.total_it, 0x7fffffff);
  note_launch(2 * mg.coarse_cycles + COARSE_KERNELS_PER_PASS * cs.total_passes);
  for (int par = 0; par < 2; par++)
    launch_convert(SOA64, AOS64, Vh, x + par * half, nullptr, static_cast<char *>(x_pyq) + par * half_pyq, nullptr,
                   st);
  QCU_CUDA(cudaStreamSynchronize(st));
  info.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return info;
}

void mg_check(MG &mg, double *orth_err, double *galerkin_err) {
  Context &ctx = context();
  require(ctx.device == mg.device, "mg: the multigrid was set up on another device");
  std::lock_guard<std::mutex> lk(ctx.mu);
  cudaStream_t st = ctx.stream;
  const MGGeom &m = mg.m;
  const int64_t nc = mg.ncoarse();
  // a seeded coarse vector, uniform in [-1, 1) (xorshift64)
  std::vector<float2> hc((size_t)nc);
  uint64_t z = 0x9e3779b97f4a7c15ULL;
  auto next = [&z]() {
    z ^= z << 13;
    z ^= z >> 7;
    z ^= z << 17;
    return (float)((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
  };
  for (auto &v : hc) {
    v.x = next();
    v.y = next();
  }
  float2 *c0 = f32(mg.cb), *c1 = f32(mg.cx), *c2 = f32(mg.cr);
  QCU_CUDA(cudaMemcpyAsync(c0, hc.data(), (size_t)nc * sizeof(float2), cudaMemcpyHostToDevice, st));
  double2 *e = f64(mg.e1), *q = f64(mg.q);
  const float2 *nv = mg.nv.as<float2>();
  double d[3], d0[3];
  // P^dag P c against c
  k_mg_prolong<<<m.nblocks, m.bsites, 0, st>>>(m, nv, c0, slabs(mg, e), 0);
  QCU_CHECK_LAUNCH();
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, slabs(mg, e), c1);
  QCU_CHECK_LAUNCH();
  lin3(st, nc, c1, C(1, 0), c1, C(-1, 0), c0);
  dots(mg, st, nc, c1, c1, d);
  dots(mg, st, nc, c0, c0, d0);
  *orth_err = std::sqrt(d[2] / d0[2]);
  // A_c c against P^dag M P c
  mat(mg, ctx, e, q);
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, slabs(mg, q), c1);
  QCU_CHECK_LAUNCH();
  capply(mg, st, c0, c2);
  dots(mg, st, nc, c1, c1, d0);
  lin3(st, nc, c2, C(1, 0), c2, C(-1, 0), c1);
  dots(mg, st, nc, c2, c2, d);
  *galerkin_err = std::sqrt(d[2] / d0[2]);
}

}  // namespace qcu
