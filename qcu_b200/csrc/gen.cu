// Seeded field generators and the gauge packer.
//
// Random numbers come from a counter-based generator: SplitMix64's output
// function (Steele, Lea & Flood, OOPSLA 2014) evaluated at (hashed seed +
// counter * golden gamma).  Every field element owns fixed counters, so the
// integers are identical to the CPU generator used by the tests; Gaussian
// variates use Box-Muller.  qcu itself used cuRAND XORWOW for its random
// initial guess (src/lattice_cuda.cu:3-14); this project does not reproduce
// cuRAND's streams.
#include "internal.h"
#include "rng.cuh"

namespace qcu {

__device__ __forceinline__ Cpx<double> rng_cgauss(uint64_t seed, uint64_t k) {
  const double u1 = rng_uniform(seed, 2 * k), u2 = rng_uniform(seed, 2 * k + 1);
  const double r = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  return Cpx<double>(r * cs, r * sn);
}

using C = Cpx<double>;

__device__ void mat_mul3(const C *a, const C *b, C *c) {
  C t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 3; k++) t[r * 3 + k] = a[r * 3] * b[k] + a[r * 3 + 1] * b[3 + k] + a[r * 3 + 2] * b[6 + k];
#pragma unroll
  for (int i = 0; i < 9; i++) c[i] = t[i];
}

// Gram-Schmidt on rows 0 and 1; row 2 = conj(row0 x row1) so det = 1
__device__ void reunitarise(C *m) {
  double n0 = m[0].norm2() + m[1].norm2() + m[2].norm2();
  n0 = 1.0 / sqrt(n0);
#pragma unroll
  for (int c = 0; c < 3; c++) m[c] = m[c] * n0;
  C pr = cdotmul(m[0], m[3]) + cdotmul(m[1], m[4]) + cdotmul(m[2], m[5]);
#pragma unroll
  for (int c = 0; c < 3; c++) m[3 + c] -= pr * m[c];
  double n1 = m[3].norm2() + m[4].norm2() + m[5].norm2();
  n1 = 1.0 / sqrt(n1);
#pragma unroll
  for (int c = 0; c < 3; c++) m[3 + c] = m[3 + c] * n1;
  m[6] = (m[1] * m[5] - m[2] * m[4]).conj();
  m[7] = (m[2] * m[3] - m[0] * m[5]).conj();
  m[8] = (m[0] * m[4] - m[1] * m[3]).conj();
}

// exp(i eps H), H Hermitian: Taylor series (16 terms) after scaling by 2^-s
// until the Frobenius norm is <= 1/4, then s squarings.
__device__ void expi_herm(const C *h, double eps, C *out) {
  C a[9];
  double nrm = 0;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    a[k] = C(-eps * h[k].im, eps * h[k].re);
    nrm += a[k].norm2();
  }
  nrm = sqrt(nrm);
  int s = 0;
  while (nrm > 0.25 && s < 60) {
    nrm *= 0.5;
    s++;
  }
  const double sc = ldexp(1.0, -s);
#pragma unroll
  for (int k = 0; k < 9; k++) a[k] = a[k] * sc;
  C res[9], term[9];
#pragma unroll
  for (int k = 0; k < 9; k++) res[k] = term[k] = C((k % 4 == 0) ? 1.0 : 0.0, 0.0);
  for (int n = 1; n <= 16; n++) {
    mat_mul3(term, a, term);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      term[k] = term[k] * (1.0 / n);
      res[k] += term[k];
    }
  }
  for (int q = 0; q < s; q++) mat_mul3(res, res, res);
#pragma unroll
  for (int k = 0; k < 9; k++) out[k] = res[k];
}

// kind 0: Haar SU(3) (Gaussian rows + Gram-Schmidt); kind 1: exp(i eps H) with
// H = sum_a h_a lambda_a / 2, h_a ~ N(0,1); kind 2: unit links
__global__ void k_gauge_random(int64_t nlink, double2 *gauge, int kind, double eps, uint64_t seed) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < nlink; l += (int64_t)gridDim.x * blockDim.x) {
    C m[9];
    if (kind == 0) {
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = rng_cgauss(seed, (uint64_t)(9 * l + k));
      reunitarise(m);
    } else if (kind == 1) {
      double h8[8];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        C z = rng_cgauss(seed, (uint64_t)(4 * l + k));
        h8[2 * k] = z.re;
        h8[2 * k + 1] = z.im;
      }
      const double s3 = 0.57735026918962576450914878050196;
      C H[9];
      H[0] = C(0.5 * (h8[2] + s3 * h8[7]), 0);
      H[4] = C(0.5 * (-h8[2] + s3 * h8[7]), 0);
      H[8] = C(0.5 * (-2.0 * s3 * h8[7]), 0);
      H[1] = C(0.5 * h8[0], -0.5 * h8[1]);
      H[3] = H[1].conj();
      H[2] = C(0.5 * h8[3], -0.5 * h8[4]);
      H[6] = H[2].conj();
      H[5] = C(0.5 * h8[5], -0.5 * h8[6]);
      H[7] = H[5].conj();
      expi_herm(H, eps, m);
      reunitarise(m);
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) m[k] = C((k % 4 == 0) ? 1.0 : 0.0, 0.0);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) gauge[9 * l + k] = make_double2(m[k].re, m[k].im);
  }
}

// kind 0: complex normal N(0,1) per component; kind 1: uniform (0,1] re and im
__global__ void k_fermion_random(int64_t n, double2 *psi, int kind, uint64_t seed) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if (kind == 0) {
      C z = rng_cgauss(seed, (uint64_t)k);
      psi[k] = make_double2(z.re, z.im);
    } else {
      psi[k] = make_double2(rng_uniform(seed, 2 * (uint64_t)k), rng_uniform(seed, 2 * (uint64_t)k + 1));
    }
  }
}

__global__ void k_uniform_soa64(int Vh, double2 *out, uint64_t seed) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < Vh; s += gridDim.x * blockDim.x) {
    double2 *o = out + blk_base<12>(s);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      const uint64_t k = (uint64_t)s * 12 + c;
      o[c * SB] = make_double2(rng_uniform(seed, 2 * k), rng_uniform(seed, 2 * k + 1));
    }
  }
}

// PyQuda gauge -> reconstruct-12 storage (rows 0 and 1 of every link)
template <int G>
__global__ void k_gauge_pack(int Vh, const double2 *__restrict__ in, void *out) {
  const int64_t n = (int64_t)8 * Vh;
  const int64_t Vp = pad_sites(Vh);
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slab = l / Vh;
    const int s = (int)(l % Vh);
    double2 v[6];
#pragma unroll
    for (int k = 0; k < 6; k++) v[k] = in[l * 9 + k];
    if constexpr (G == GSOA64) {
      double2 *o = static_cast<double2 *>(out) + slab * 6 * Vp + blk_base<6>(s);
#pragma unroll
      for (int k = 0; k < 6; k++) o[k * SB] = v[k];
    } else if constexpr (G == GSOA32) {
      float4 *o = static_cast<float4 *>(out) + slab * 3 * Vp + blk_base<3>(s);
#pragma unroll
      for (int k = 0; k < 3; k++)
        o[k * SB] = make_float4((float)v[2 * k].x, (float)v[2 * k].y, (float)v[2 * k + 1].x, (float)v[2 * k + 1].y);
    } else {
      char *blk = static_cast<char *>(out) + slab * Vp * 24 + (int64_t)(s >> 5) * G16_BLOCK_BYTES;
      unsigned w[6];
#pragma unroll
      for (int k = 0; k < 6; k++) w[k] = fix16_pack((float)v[k].x, (float)v[k].y);
      reinterpret_cast<uint4 *>(blk)[s & 31] = make_uint4(w[0], w[1], w[2], w[3]);
      reinterpret_cast<uint2 *>(blk + 512)[s & 31] = make_uint2(w[4], w[5]);
    }
  }
}

static int gen_grid(int64_t n, int block) {
  int64_t g = (n + block - 1) / block;
  return (int)(g > 148 * 64 ? 148 * 64 : (g < 1 ? 1 : g));
}

void launch_gauge_random(const Geom &g, void *gauge, int kind, double eps, uint64_t seed, cudaStream_t s) {
  const int64_t nlink = (int64_t)8 * g.Vh;
  k_gauge_random<<<gen_grid(nlink, 128), 128, 0, s>>>(nlink, static_cast<double2 *>(gauge), kind, eps, seed);
  QCU_CHECK_LAUNCH();
}

void launch_fermion_random(void *psi, int64_t n, int kind, uint64_t seed, cudaStream_t s) {
  k_fermion_random<<<gen_grid(n, 256), 256, 0, s>>>(n, static_cast<double2 *>(psi), kind, seed);
  QCU_CHECK_LAUNCH();
}

void launch_uniform_soa64(int Vh, void *out, uint64_t seed, cudaStream_t s) {
  k_uniform_soa64<<<gen_grid(Vh, 256), 256, 0, s>>>(Vh, static_cast<double2 *>(out), seed);
  QCU_CHECK_LAUNCH();
}

size_t gauge_bytes(int gkind, int Vh) {
  const size_t Vp = pad_sites(Vh);
  switch (gkind) {
    case GSOA64: return 8 * 6 * Vp * 16;
    case GSOA32: return 8 * 3 * Vp * 16;
    case GSOA16: return 8 * 3 * Vp * 8;
    default: return (size_t)8 * 9 * Vh * 16;
  }
}

void launch_gauge_pack(int gkind, const Geom &g, const void *pyq, void *out, cudaStream_t s) {
  const int64_t n = (int64_t)8 * g.Vh;
  const double2 *in = static_cast<const double2 *>(pyq);
  switch (gkind) {
    case GSOA64: k_gauge_pack<GSOA64><<<gen_grid(n, 256), 256, 0, s>>>(g.Vh, in, out); break;
    case GSOA32: k_gauge_pack<GSOA32><<<gen_grid(n, 256), 256, 0, s>>>(g.Vh, in, out); break;
    case GSOA16: k_gauge_pack<GSOA16><<<gen_grid(n, 256), 256, 0, s>>>(g.Vh, in, out); break;
    default: throw Error(1, "unsupported gauge kind");
  }
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
