// Parallel-transport layers of the learned preconditioner: forward,
// input-gradient (adjoint) and weight-gradient kernels, the training loss
// and an Adam step.  FP32 arithmetic; weights FP32 (training) or bf16
// (inference).  See nn.h for the layer definition.
#include <cuda_bf16.h>

#include "nn.h"

namespace qcu {

using F2 = float2;

__device__ __forceinline__ F2 cmul(F2 a, F2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ F2 cmulc(F2 a, F2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ F2 cadd(F2 a, F2 b) { return make_float2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ int hop_bar(int h) { return h == 0 ? 0 : (h & 1 ? h + 1 : h - 1); }

// neighbour of site s (parity par) in direction mu, step +-1; also whether
// the hop crosses the t boundary
__device__ __forceinline__ int nbr(const Geom &g, int s, int par, int mu, int fwd, bool &tcross) {
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int xodd = (y + z + t + par) & 1;
  tcross = false;
  switch (mu) {
    case 0:
      return fwd ? (xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s) : (xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1));
    case 1:
      return fwd ? (y == g.Ly - 1 ? s - (g.Ly - 1) * g.sy : s + g.sy) : (y == 0 ? s + (g.Ly - 1) * g.sy : s - g.sy);
    case 2:
      return fwd ? (z == g.Lz - 1 ? s - (g.Lz - 1) * g.sz : s + g.sz) : (z == 0 ? s + (g.Lz - 1) * g.sz : s - g.sz);
    default:
      tcross = fwd ? (t == g.Lt - 1) : (t == 0);
      return fwd ? (t == g.Lt - 1 ? s - (g.Lt - 1) * g.st : s + g.st) : (t == 0 ? s + (g.Lt - 1) * g.st : s - g.st);
  }
}

// v <- T_h applied at (s, par): transported colour vectors of CIN channels
// read from `in` on the neighbouring site.  Returns false if the hop's source
// parity holds no input (in_mask).
template <int CIN>
__device__ __forceinline__ bool transport(const Geom &g, const PtcArgs &a, const float2 *in_sample, int s, int par,
                                          int h, F2 v[CIN][3]) {
  const int src_par = h == 0 ? par : 1 - par;
  if (!(a.in_mask >> src_par & 1)) return false;
  const size_t slab = (size_t)src_par * g.Vh;
  if (h == 0) {
    const F2 *p = in_sample + (slab + s) * CIN * 3;
#pragma unroll
    for (int b = 0; b < CIN; b++)
#pragma unroll
      for (int c = 0; c < 3; c++) v[b][c] = p[b * 3 + c];
    return true;
  }
  const int mu = (h - 1) >> 1, fwd = (h & 1);
  bool tc;
  const int n = nbr(g, s, par, mu, fwd, tc);
  Cpx<float> u[9];
  const GaugeView<GSOA32> U{a.gauge, pad_sites(g.Vh)};
  link_load<GSOA32, float>(U, mu, fwd ? par : 1 - par, fwd ? s : n, u);
  const float ph = tc ? a.t_bc : 1.f;
  const F2 *p = in_sample + (slab + n) * CIN * 3;
#pragma unroll
  for (int b = 0; b < CIN; b++) {
    F2 q[3];
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = p[b * 3 + c];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      F2 acc = make_float2(0.f, 0.f);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const Cpx<float> m = fwd ? u[r * 3 + c] : u[c * 3 + r].conj();
        acc = cadd(acc, cmul(make_float2(m.re, m.im), q[c]));
      }
      v[b][r] = make_float2(acc.x * ph, acc.y * ph);
    }
  }
  return true;
}

// load the layer's weights into shared memory, as float2 [9][COUT][CIN]
template <int CIN, int COUT>
__device__ __forceinline__ void load_weights(const PtcArgs &a, F2 *W) {
  for (int k = threadIdx.x; k < NN_HOPS * COUT * CIN; k += blockDim.x) {
    const int h = k / (COUT * CIN), ab = k % (COUT * CIN), ao = ab / CIN, bi = ab % CIN;
    // adjoint: W'[h][a][b] = conj(W[hbar][b][a]) from a [9][CIN][COUT] source
    const int src = a.adjoint ? (hop_bar(h) * CIN + bi) * COUT + ao : k;
    F2 w;
    if (a.w) {
      w = a.w[src];
    } else {
      const uint32_t q = a.w16[src];
      w = make_float2(__uint_as_float(q << 16), __uint_as_float(q & 0xffff0000u));
    }
    if (a.adjoint) w.y = -w.y;
    W[k] = w;
  }
}

// which output site a flat thread index covers: (sample, parity, site)
__device__ __forceinline__ bool decode(const Geom &g, const PtcArgs &a, long long idx, int &b, int &par, int &s) {
  const int np = (a.out_mask & 1) + (a.out_mask >> 1 & 1);
  const long long per = (long long)np * g.Vh;
  if (idx >= per * a.B) return false;
  b = (int)(idx / per);
  const long long r = idx % per;
  const int which = (int)(r / g.Vh);
  s = (int)(r % g.Vh);
  par = np == 2 ? which : (a.out_mask == 1 ? 0 : 1);
  return true;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_ptc(Geom g, PtcArgs a) {
  __shared__ F2 W[NN_HOPS * COUT * CIN];
  load_weights<CIN, COUT>(a, W);
  __syncthreads();
  int b, par, s;
  if (!decode(g, a, blockIdx.x * (long long)blockDim.x + threadIdx.x, b, par, s)) return;
  const float2 *in_sample = a.in + (size_t)b * 2 * g.Vh * CIN * 3;
  F2 acc[COUT][3];
  F2 *out = a.out + (((size_t)b * 2 + par) * g.Vh + s) * COUT * 3;
#pragma unroll
  for (int o = 0; o < COUT; o++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[o][c] = a.accumulate ? out[o * 3 + c] : make_float2(0.f, 0.f);
  for (int h = 0; h < NN_HOPS; h++) {
    F2 v[CIN][3];
    if (!transport<CIN>(g, a, in_sample, s, par, h, v)) continue;
#pragma unroll
    for (int bi = 0; bi < CIN; bi++)
#pragma unroll
      for (int o = 0; o < COUT; o++) {
        const F2 w = W[(h * COUT + o) * CIN + bi];
#pragma unroll
        for (int c = 0; c < 3; c++) acc[o][c] = cadd(acc[o][c], cmul(w, v[bi][c]));
      }
  }
#pragma unroll
  for (int o = 0; o < COUT; o++)
#pragma unroll
    for (int c = 0; c < 3; c++) out[o * 3 + c] = acc[o][c];
}

// weight gradient: every lane runs the same hop loop (zeros where a hop does
// not apply) so the warp reductions stay converged
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_ptc_wgrad(Geom g, PtcArgs a, F2 *grad) {
  __shared__ F2 sg[NN_HOPS * COUT * CIN];
  for (int k = threadIdx.x; k < NN_HOPS * COUT * CIN; k += blockDim.x) sg[k] = make_float2(0.f, 0.f);
  __syncthreads();
  int b = 0, par = 0, s = 0;
  const bool active = decode(g, a, blockIdx.x * (long long)blockDim.x + threadIdx.x, b, par, s);
  F2 d[COUT][3];
  const float2 *in_sample = a.in + (size_t)b * 2 * g.Vh * CIN * 3;
  if (active) {
    const F2 *dp = a.out + (((size_t)b * 2 + par) * g.Vh + s) * COUT * 3;
#pragma unroll
    for (int o = 0; o < COUT; o++)
#pragma unroll
      for (int c = 0; c < 3; c++) d[o][c] = dp[o * 3 + c];
  }
  const int lane = threadIdx.x & 31;
  for (int h = 0; h < NN_HOPS; h++) {
    F2 v[CIN][3];
    bool ok = active && transport<CIN>(g, a, in_sample, s, par, h, v);
    if (!ok) {
#pragma unroll
      for (int bi = 0; bi < CIN; bi++)
#pragma unroll
        for (int c = 0; c < 3; c++) v[bi][c] = make_float2(0.f, 0.f);
    }
    if (!__any_sync(0xffffffffu, ok)) continue;
#pragma unroll
    for (int o = 0; o < COUT; o++)
#pragma unroll
      for (int bi = 0; bi < CIN; bi++) {
        F2 q = make_float2(0.f, 0.f);
        if (ok) {
#pragma unroll
          for (int c = 0; c < 3; c++) q = cadd(q, cmulc(d[o][c], v[bi][c]));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          q.x += __shfl_xor_sync(0xffffffffu, q.x, off);
          q.y += __shfl_xor_sync(0xffffffffu, q.y, off);
        }
        if (lane == 0) {
          F2 *t = &sg[(h * COUT + o) * CIN + bi];
          atomicAdd(&t->x, q.x);
          atomicAdd(&t->y, q.y);
        }
      }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NN_HOPS * COUT * CIN; k += blockDim.x) {
    atomicAdd(&grad[k].x, sg[k].x);
    atomicAdd(&grad[k].y, sg[k].y);
  }
}

// delta = (o - e) / (|e|^2 B), loss[i] += |o - e|^2 / |e|^2 over the odd sites
__global__ void k_nn_loss(Geom g, int B, const F2 *o, const F2 *e, const float *enorm2, F2 *delta, float *loss) {
  const long long n = (long long)B * g.Vh;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(idx / g.Vh), s = (int)(idx % g.Vh);
    const size_t off = (((size_t)b * 2 + 1) * g.Vh + s) * 12;
    const float inv = 1.f / enorm2[b];
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const F2 d = make_float2(o[off + k].x - e[off + k].x, o[off + k].y - e[off + k].y);
      acc += d.x * d.x + d.y * d.y;
      delta[off + k] = make_float2(d.x * inv / B, d.y * inv / B);
    }
    atomicAdd(&loss[b], acc * inv);
  }
}

__global__ void k_adam(int n, float *p, const float *gr, float *m, float *v, uint32_t *p16, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
  __syncthreads();  // launched as a single block: every updated value is visible below
  // bf16 copy, one complex (two reals) per word
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += gridDim.x * blockDim.x) {
    const __nv_bfloat16 re = __float2bfloat16_rn(p[2 * i]), im = __float2bfloat16_rn(p[2 * i + 1]);
    p16[i] = (uint32_t)__bfloat16_as_ushort(re) | ((uint32_t)__bfloat16_as_ushort(im) << 16);
  }
}

__global__ void k_to_bf16(int n, const float *p, uint32_t *p16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += gridDim.x * blockDim.x) {
    const __nv_bfloat16 re = __float2bfloat16_rn(p[2 * i]), im = __float2bfloat16_rn(p[2 * i + 1]);
    p16[i] = (uint32_t)__bfloat16_as_ushort(re) | ((uint32_t)__bfloat16_as_ushort(im) << 16);
  }
}

__global__ void k_soa64_to_nn(int Vh, const double2 *in, F2 *nn) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < Vh; s += gridDim.x * blockDim.x) {
    const double2 *p = in + blk_base<12>(s);
    F2 *o = nn + ((size_t)Vh + s) * 12;  // parity 1 slab
#pragma unroll
    for (int c = 0; c < 12; c++) {
      const double2 d = p[c * SB];
      o[c] = make_float2((float)d.x, (float)d.y);
    }
  }
}

__global__ void k_nn_to_soa64(int Vh, const F2 *nn, double2 *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < Vh; s += gridDim.x * blockDim.x) {
    double2 *p = out + blk_base<12>(s);
    const F2 *q = nn + ((size_t)Vh + s) * 12;
#pragma unroll
    for (int c = 0; c < 12; c++) p[c * SB] = make_double2(q[c].x, q[c].y);
  }
}

static long long out_sites(const Geom &g, const PtcArgs &a) {
  const int np = (a.out_mask & 1) + (a.out_mask >> 1 & 1);
  return (long long)np * g.Vh * a.B;
}

void launch_ptc(int cin, int cout, const Geom &g, const PtcArgs &a, cudaStream_t s) {
  const long long n = out_sites(g, a);
  const int blocks = (int)((n + 127) / 128);
  if (cin == 4 && cout == 16) k_ptc<4, 16><<<blocks, 128, 0, s>>>(g, a);
  else if (cin == 16 && cout == 4) k_ptc<16, 4><<<blocks, 128, 0, s>>>(g, a);
  else throw Error(1, "ptc layer: channels must be 4->16 or 16->4");
  QCU_CHECK_LAUNCH();
}

void launch_ptc_wgrad(int cin, int cout, const Geom &g, const PtcArgs &a, float2 *grad, cudaStream_t s) {
  const long long n = out_sites(g, a);
  const int blocks = (int)((n + 127) / 128);
  if (cin == 4 && cout == 16) k_ptc_wgrad<4, 16><<<blocks, 128, 0, s>>>(g, a, grad);
  else if (cin == 16 && cout == 4) k_ptc_wgrad<16, 4><<<blocks, 128, 0, s>>>(g, a, grad);
  else throw Error(1, "ptc layer: channels must be 4->16 or 16->4");
  QCU_CHECK_LAUNCH();
}

void launch_nn_loss(const Geom &g, int B, const float2 *o, const float2 *e, const float *enorm2, float2 *delta,
                    float *loss, cudaStream_t s) {
  k_nn_loss<<<blas_grid(g.Vh * B), BLAS_BLOCK, 0, s>>>(g, B, o, e, enorm2, delta, loss);
  QCU_CHECK_LAUNCH();
}

void launch_adam(int n, float *p, const float *grad, float *m, float *v, uint32_t *p16, float lr, float b1, float b2,
                 float eps, int step, cudaStream_t s) {
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  k_adam<<<1, 256, 0, s>>>(n, p, grad, m, v, p16, lr, b1, b2, eps, c1, c2);
  QCU_CHECK_LAUNCH();
}

void launch_to_bf16(int n, const float *p, uint32_t *p16, cudaStream_t s) {
  k_to_bf16<<<8, 256, 0, s>>>(n, p, p16);
  QCU_CHECK_LAUNCH();
}

void launch_soa64_to_nn(int Vh, const void *in, float2 *nn_odd, cudaStream_t s) {
  k_soa64_to_nn<<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, static_cast<const double2 *>(in), nn_odd);
  QCU_CHECK_LAUNCH();
}

void launch_nn_to_soa64(int Vh, const float2 *nn_odd, void *out, cudaStream_t s) {
  k_nn_to_soa64<<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, nn_odd, static_cast<double2 *>(out));
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
