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
// near-null vector k: full FP32 vectors one after the other
__device__ __forceinline__ size_t nidx(const MGGeom &m, int k, int par, int s, int comp) {
  return (size_t)k * 2 * m.Vp * 12 + fidx(m, par, s, comp);
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
  const SiteC c = mg_site(m, blockIdx.x, threadIdx.x);
  for (int k = 0; k < m.nvec; k++) {
    for (int j = 0; j <= k; j++) {
      double v[4] = {0, 0, 0, 0};  // per chirality: Re, Im of <v_j, v_k> (j == k: |v_k|^2)
      for (int comp = 0; comp < 12; comp++) {
        const int ch = comp / 6;
        const float2 a = nv[nidx(m, j, c.par, c.s, comp)], b = nv[nidx(m, k, c.par, c.s, comp)];
        v[2 * ch] += (double)a.x * b.x + (double)a.y * b.y;
        v[2 * ch + 1] += (double)a.x * b.y - (double)a.y * b.x;
      }
      mg_block_sum<4>(v, sh);
      for (int comp = 0; comp < 12; comp++) {
        const int ch = comp / 6;
        float2 &b = nv[nidx(m, k, c.par, c.s, comp)];
        if (j < k) {  // v_k -= <v_j, v_k> v_j
          const float2 a = nv[nidx(m, j, c.par, c.s, comp)];
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

// coarse c[B][ch nvec + k] = <v_k^ch, r>_B for a full FP64 vector r
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_restrict(MGGeom m, const float2 *nv, const double2 *r,
                                                           float2 *cv) {
  __shared__ double sh[(MG_MAXBLOCK / 32) * 4];
  const int B = blockIdx.x;
  const SiteC c = mg_site(m, B, threadIdx.x);
  double2 rv[12];
#pragma unroll
  for (int comp = 0; comp < 12; comp++) rv[comp] = r[fidx(m, c.par, c.s, comp)];
  for (int k = 0; k < m.nvec; k++) {
    double v[4] = {0, 0, 0, 0};
#pragma unroll
    for (int comp = 0; comp < 12; comp++) {
      const int ch = comp / 6;
      const float2 a = nv[nidx(m, k, c.par, c.s, comp)];
      v[2 * ch] += (double)a.x * rv[comp].x + (double)a.y * rv[comp].y;
      v[2 * ch + 1] += (double)a.x * rv[comp].y - (double)a.y * rv[comp].x;
    }
    mg_block_sum<4>(v, sh);
    if (threadIdx.x == 0) {
      cv[(size_t)B * m.nc + k] = make_float2((float)v[0], (float)v[1]);
      cv[(size_t)B * m.nc + m.nvec + k] = make_float2((float)v[2], (float)v[3]);
    }
  }
}

// e = P c (FP64 full vector; e += P c when add)
__global__ void __launch_bounds__(MG_MAXBLOCK) k_mg_prolong(MGGeom m, const float2 *nv, const float2 *cv,
                                                          double2 *e, int add) {
  const int B = blockIdx.x;
  const SiteC c = mg_site(m, B, threadIdx.x);
  const float2 *cb = cv + (size_t)B * m.nc;
#pragma unroll
  for (int comp = 0; comp < 12; comp++) {
    const int ch = comp / 6;
    double re = 0, im = 0;
    for (int k = 0; k < m.nvec; k++) {
      const float2 a = nv[nidx(m, k, c.par, c.s, comp)];
      const float2 q = cb[ch * m.nvec + k];
      re += (double)a.x * q.x - (double)a.y * q.y;
      im += (double)a.x * q.y + (double)a.y * q.x;
    }
    double2 &o = e[fidx(m, c.par, c.s, comp)];
    if (add) o = make_double2(o.x + re, o.y + im);
    else o = make_double2(re, im);
  }
}

// ---------------------------------------------------------------- coarse operator
// h = the hop of direction MU (forward or backward) at site (par, s) applied
// to near-null vector k2 restricted to chirality ch2, taken at the neighbour
// n: U (1 - gamma_mu) forward, U^dag (1 + gamma_mu) backward, the stencil core
// of the dslash kernels
template <int MU, bool FWD>
__device__ __forceinline__ void mg_hop(const MGGeom &m, const GaugeView<GSOA64> &U, const float2 *nv, int par, int s,
                                       int n, int k2, int ch2, double ph, Cpx<double> h[12]) {
  Cpx<double> psi[12], u[9];
#pragma unroll
  for (int comp = 0; comp < 12; comp++) {
    if (comp / 6 == ch2) {
      const float2 a = nv[nidx(m, k2, 1 - par, n, comp)];
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

// Y[B][d][col][row], d = 0..7 the directions (Y_d), d = 8 the self block X;
// col = ch2 nvec + k2 (the vector acted on), row = ch nvec + k:
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
  const SiteC c = mg_site(m, B, threadIdx.x);
  for (int i = threadIdx.x; i < nc * nc; i += blockDim.x) xs[i / nc][i % nc] = make_double2(0, 0);
  __syncthreads();
  for (int d = 0; d < 9; d++) {
    int n = 0, inblock = 1;
    double ph = 1.0;
    if (d < 8) {
      const int mu = d >> 1;
      const bool fwd = !(d & 1);
      int y[4] = {c.x[0], c.x[1], c.x[2], c.x[3]};
      y[mu] = fwd ? (y[mu] + 1) % m.L[mu] : (y[mu] + m.L[mu] - 1) % m.L[mu];
      n = ((y[3] * m.L[2] + y[2]) * m.L[1] + y[1]) * (m.L[0] / 2) + (y[0] >> 1);
      inblock = mg_block_of(m, y) == B;
      if (mu == 3 && ((fwd && c.x[3] == m.L[3] - 1) || (!fwd && c.x[3] == 0))) ph = t_bc;
    }
    for (int col = 0; col < nc; col++) {
      const int ch2 = col / nvec, k2 = col % nvec;
      Cpx<double> h[12];
      switch (d) {
        case 0: mg_hop<0, true>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 1: mg_hop<0, false>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 2: mg_hop<1, true>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 3: mg_hop<1, false>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 4: mg_hop<2, true>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 5: mg_hop<2, false>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 6: mg_hop<3, true>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        case 7: mg_hop<3, false>(m, U, nv, c.par, c.s, n, k2, ch2, ph, h); break;
        default:  // the local term A v_col (v_col itself without clover)
#pragma unroll
          for (int comp = 0; comp < 12; comp++) {
            if (comp / 6 == ch2) {
              const float2 a = nv[nidx(m, k2, c.par, c.s, comp)];
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
          const float2 a = nv[nidx(m, k, c.par, c.s, comp)];
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
          float *y = reinterpret_cast<float *>(Y + (((size_t)B * 9 + d) * nc + col) * nc + row);
          y[im] = (float)val;
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < nc * nc; i += blockDim.x) {
    const double2 v = xs[i / nc][i % nc];
    Y[((size_t)B * 9 + 8) * nc * nc + i] = make_float2((float)v.x, (float)v.y);
  }
}

// out = A_c in: one warp per aggregate, lane = row
__global__ void k_mg_capply(MGGeom m, const float2 *Y, const float2 *in, float2 *out) {
  const int B = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int row = threadIdx.x & 31;
  if (B >= m.nblocks || row >= m.nc) return;
  const int nc = m.nc;
  float re = 0.f, im = 0.f;
  for (int d = 0; d < 9; d++) {
    const float2 *x = in + (size_t)mg_cnbr(m, B, d) * nc;
    const float2 *Yd = Y + ((size_t)B * 9 + d) * nc * nc;
    for (int col = 0; col < nc; col++) {
      const float2 a = Yd[col * nc + row], v = x[col];
      re = fmaf(a.x, v.x, fmaf(-a.y, v.y, re));
      im = fmaf(a.x, v.y, fmaf(a.y, v.x, im));
    }
  }
  out[(size_t)B * nc + row] = make_float2(re, im);
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
// FP64 -> FP32, same element order
__global__ void k_mg_to32(int64_t n, const double2 *in, float2 *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
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
  // FP64 full vectors: b, x, r; e1, s, q (the cycle); tmp (one parity, A in)
  DevBuf b, x, r, e1, s, q, tmp;
  std::vector<std::unique_ptr<DevBuf>> Z, W;  // flexible GCR directions
  // coarse FP32 vectors
  DevBuf cb, cx, cr, crt, cp, cv, ct;
  double setup_seconds = 0;
  long long coarse_iters = 0;

  int64_t nfull() const { return (int64_t)2 * m.Vp * 12; }
  int64_t ncoarse() const { return (int64_t)m.nblocks * m.nc; }
};

namespace {

using C = Cpx<double>;
double2 *f64(DevBuf &d) { return d.as<double2>(); }
float2 *f32(DevBuf &d) { return d.as<float2>(); }

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

void capply(MG &mg, cudaStream_t st, const float2 *in, float2 *out) {
  constexpr int warps = 4;
  k_mg_capply<<<(mg.m.nblocks + warps - 1) / warps, 32 * warps, 0, st>>>(mg.m, mg.Y.as<float2>(), in, out);
  QCU_CHECK_LAUNCH();
}

// x ~ A_c^-1 b: BiCGSTAB (FP32 vectors, FP64 scalars) from x = 0 to
// |r| <= coarse_tol |b| or coarse_maxiter iterations; returns the iterations
int coarse_solve(MG &mg, cudaStream_t st, const float2 *bv, float2 *xv) {
  const int64_t n = mg.ncoarse();
  const size_t bytes = (size_t)n * sizeof(float2);
  float2 *r = f32(mg.cr), *rt = f32(mg.crt), *p = f32(mg.cp), *v = f32(mg.cv), *t = f32(mg.ct);
  QCU_CUDA(cudaMemsetAsync(xv, 0, bytes, st));
  QCU_CUDA(cudaMemsetAsync(p, 0, bytes, st));
  QCU_CUDA(cudaMemsetAsync(v, 0, bytes, st));
  QCU_CUDA(cudaMemcpyAsync(r, bv, bytes, cudaMemcpyDeviceToDevice, st));
  QCU_CUDA(cudaMemcpyAsync(rt, bv, bytes, cudaMemcpyDeviceToDevice, st));
  double d[3];
  dots(mg, st, n, bv, bv, d);
  const double bb = d[2];
  if (!(bb > 0)) return 0;
  const double target = mg.p.coarse_tol * mg.p.coarse_tol * bb;
  C rho(1, 0), alpha(1, 0), omega(1, 0);
  int it = 0;
  while (it < mg.p.coarse_maxiter) {
    dots(mg, st, n, rt, r, d);
    const C rho1(d[0], d[1]);
    if (rho1.norm2() == 0) break;
    const C beta = cdiv(rho1, rho) * cdiv(alpha, omega);
    lin3(st, n, p, C(1, 0), r, beta, p, -(beta * omega), v);  // p = r + beta (p - omega v)
    capply(mg, st, p, v);
    dots(mg, st, n, rt, v, d);
    const C rtv(d[0], d[1]);
    if (rtv.norm2() == 0) break;
    alpha = cdiv(rho1, rtv);
    lin3(st, n, r, C(1, 0), r, -alpha, v);  // s = r - alpha v (kept in r)
    capply(mg, st, r, t);
    dots(mg, st, n, t, r, d);  // <t, s>, |t|^2
    it++;
    if (!(d[2] > 0)) {  // t = 0: s is already the residual of x + alpha p
      lin3(st, n, xv, C(1, 0), xv, alpha, p);
      break;
    }
    omega = C(d[0] / d[2], d[1] / d[2]);
    lin3(st, n, xv, C(1, 0), xv, alpha, p, omega, r);  // x += alpha p + omega s
    lin3(st, n, r, C(1, 0), r, -omega, t);             // r = s - omega t
    rho = rho1;
    dots(mg, st, n, r, r, d);
    if (!(d[2] == d[2])) throw Error(3, "mg: the coarse solve produced a non-finite residual");
    if (d[2] <= target) break;
  }
  return it;
}

// steps MR iterations on M e = r from e (start: s = r - M e, or s = r when e = 0)
void smooth(MG &mg, Context &ctx, const double2 *r, double2 *e, int steps, bool e_zero) {
  cudaStream_t st = ctx.stream;
  const int64_t n = mg.nfull();
  double2 *s = f64(mg.s), *q = f64(mg.q);
  if (e_zero) {
    QCU_CUDA(cudaMemsetAsync(e, 0, (size_t)n * sizeof(double2), st));
    QCU_CUDA(cudaMemcpyAsync(s, r, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  } else {
    mat(mg, ctx, e, q);
    lin3(st, n, s, C(1, 0), r, C(-1, 0), q);
  }
  for (int k = 0; k < steps; k++) {
    mat(mg, ctx, s, q);
    double d[3];
    dots(mg, st, n, q, s, d);  // <M s, s>, |M s|^2
    if (!(d[2] > 0)) break;
    const C a(d[0] / d[2], d[1] / d[2]);
    lin3(st, n, e, C(1, 0), e, a, s);
    lin3(st, n, s, C(1, 0), s, -a, q);
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
    mat(mg, ctx, e, f64(mg.q));
    lin3(st, n, f64(mg.e1), C(1, 0), r, C(-1, 0), f64(mg.q));
    rc = f64(mg.e1);
  }
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, rc, f32(mg.cb));
  QCU_CHECK_LAUNCH();
  mg.coarse_iters += coarse_solve(mg, st, f32(mg.cb), f32(mg.cx));
  k_mg_prolong<<<m.nblocks, m.bsites, 0, st>>>(m, nv, f32(mg.cx), e, mg.p.nu_pre > 0 ? 1 : 0);
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
    mg->part.ensure((size_t)MG_RED_GRID * 3 * sizeof(double));
    mg->part_h.resize((size_t)MG_RED_GRID * 3);
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
      k_mg_to32<<<mg_grid(n), MG_RED, 0, st>>>(n, vf, mg->nv.as<float2>() + (size_t)k * n);
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
  mg->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return mg.release();
}

void mg_free(MG *mg) { delete mg; }

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
  double2 *b = f64(mg.b), *x = f64(mg.x), *r = f64(mg.r), *q = f64(mg.q);
  for (int par = 0; par < 2; par++)
    launch_convert(AOS64, SOA64, Vh, static_cast<const char *>(b_pyq) + par * half_pyq, nullptr, b + par * half,
                   nullptr, st);
  QCU_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double2), st));
  QCU_CUDA(cudaMemcpyAsync(r, b, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  MGInfo info;
  mg.coarse_iters = 0;
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
  info.status = ST_MAXITER;
  while (info.outer < maxiter) {
    for (int j = 0; j < mg.p.gcr_k && info.outer < maxiter; j++) {
      double2 *z = f64(*mg.Z[j]), *w = f64(*mg.W[j]);
      cycle(mg, ctx, r, z);
      mat(mg, ctx, z, w);
      for (int i = 0; i < j; i++) {  // w_j -= <w_i, w_j> w_i (w_i normalised), z_j likewise
        dots(mg, st, n, f64(*mg.W[i]), w, d);
        const C beta(d[0], d[1]);
        lin3(st, n, w, C(1, 0), w, -beta, f64(*mg.W[i]));
        lin3(st, n, z, C(1, 0), z, -beta, f64(*mg.Z[i]));
      }
      dots(mg, st, n, w, r, d);  // <w, r>, |w|^2
      if (!(d[2] > 0) || !(d[0] == d[0]) || !(d[1] == d[1])) {
        info.status = d[2] == d[2] ? ST_BREAKDOWN : ST_NAN;
        break;
      }
      const double inv_norm = 1.0 / std::sqrt(d[2]);
      lin3(st, n, w, C(inv_norm, 0), w);
      lin3(st, n, z, C(inv_norm, 0), z);
      const C alpha(d[0] * inv_norm, d[1] * inv_norm);  // <w / |w|, r>
      lin3(st, n, x, C(1, 0), x, alpha, z);
      lin3(st, n, r, C(1, 0), r, -alpha, w);
      info.outer++;
      dots(mg, st, n, r, r, d);
      rr = d[2];
      if (rr <= target) break;
    }
    if (info.status == ST_BREAKDOWN || info.status == ST_NAN) break;
    // restart from the FP64 true residual
    mat(mg, ctx, x, q);
    lin3(st, n, r, C(1, 0), b, C(-1, 0), q);
    dots(mg, st, n, r, r, d);
    rr = d[2];
    if (rr <= target) {
      info.status = ST_CONVERGED;
      break;
    }
  }
  if (info.status == ST_BREAKDOWN || info.status == ST_NAN) {
    mat(mg, ctx, x, q);
    lin3(st, n, r, C(1, 0), b, C(-1, 0), q);
    dots(mg, st, n, r, r, d);
    rr = d[2];
  }
  info.true_residual = std::sqrt(rr / bb);
  info.coarse_iters = (int)std::min<long long>(mg.coarse_iters, 0x7fffffff);
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
  k_mg_prolong<<<m.nblocks, m.bsites, 0, st>>>(m, nv, c0, e, 0);
  QCU_CHECK_LAUNCH();
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, e, c1);
  QCU_CHECK_LAUNCH();
  lin3(st, nc, c1, C(1, 0), c1, C(-1, 0), c0);
  dots(mg, st, nc, c1, c1, d);
  dots(mg, st, nc, c0, c0, d0);
  *orth_err = std::sqrt(d[2] / d0[2]);
  // A_c c against P^dag M P c
  mat(mg, ctx, e, q);
  k_mg_restrict<<<m.nblocks, m.bsites, 0, st>>>(m, nv, q, c1);
  QCU_CHECK_LAUNCH();
  capply(mg, st, c0, c2);
  dots(mg, st, nc, c1, c1, d0);
  lin3(st, nc, c2, C(1, 0), c2, C(-1, 0), c1);
  dots(mg, st, nc, c2, c2, d);
  *galerkin_err = std::sqrt(d[2] / d0[2]);
}

}  // namespace qcu
