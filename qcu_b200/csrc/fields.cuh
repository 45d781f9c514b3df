// Device-side views of the lattice fields and the Wilson stencil core.
//
// Internal fields use a site-blocked layout: sites are grouped in blocks of
// SB = 32 (one warp), and within a block every 16-byte (8-byte for 16-bit
// links) component is stored for the 32 sites contiguously:
//     element (site s, component c) at ((s / 32) * NC + c) * 32 + s % 32
// so a warp's load of one component is one contiguous 512 (256) byte
// segment, and the components of a site sit at compile-time offsets from one
// base pointer (no per-component address arithmetic).  Vh is padded to a
// multiple of 32; padding sites are never read or written.
// Spinor kinds (one parity):
//   AOS64 : PyQuda's own layout, complex128 [site][spin*3+colour]
//           (python/PyQuda/pyquda/field.py:78,230) -- used by the legacy ABI
//           so a single dslash needs no layout conversion at all.
//   AOS64W: the same layout, read and written with 32-byte accesses; for
//           fields whose base is 32-byte aligned (the legacy dslash checks)
//   SOA64 : double2, NC = 12 (one complex per 16-byte load)
//   SOA32 : float4,  NC = 6: float4 j = 3 * q + c holds colour c of spins 2q
//           and 2q + 1 as (re, re, im, im), the lane pairs of the paired FP32
//           instructions (hop32.cuh)
//   SOA16 : 12 words per site + float norm[Vh]: 16-bit fixed point
//           (offset-binary 16-bit, value/norm * 32767) scaled by the per-site max |component|;
//           word k = 6 q + 2 c + (re, im) holds spin 2q (low half) and 2q + 1 (high
//           half) of colour c.  A block of 32 sites is [32 x words 0-7][32 x words 8-11]
//           (1024 + 512 B): one 32-byte and one 16-byte load per site.  Fixed point keeps
//           15 bits of mantissa relative to the site maximum where FP16 keeps 11.
// Gauge kinds (reconstruct-12: rows 0 and 1 stored, row 2 = conj(r0 x r1),
// include/define.h:198-206), one slab of Vh_pad sites per (dir, parity):
//   GAOS64 : PyQuda layout complex128 [dir][par][site][3][3], rows 0-1 read
//   GSOA64 : double2, NC = 6
//   GSOA32 : float4,  NC = 3
//   GSOA16 : 6 words per link (word e = element e of rows 0-1, 16-bit fixed point,
//            |U_ij| <= 1); a block of 32 sites is [32 x words 0-3][32 x words 4-5]
//            (512 + 256 B): one 16-byte and one 8-byte load per link
#pragma once
#include "cplx.cuh"

namespace qcu {

enum SpinorKind { AOS64 = 0, SOA64 = 1, SOA32 = 2, SOA16 = 3, AOS64W = 4 };
enum GaugeKind { GAOS64 = 0, GSOA64 = 1, GSOA32 = 2, GSOA16 = 3 };

template <int K> struct SpinorReal { using T = float; };
template <> struct SpinorReal<AOS64> { using T = double; };
template <> struct SpinorReal<SOA64> { using T = double; };
template <> struct SpinorReal<AOS64W> { using T = double; };

// 16-bit fixed point: two values per 32-bit word, each stored offset-binary
// (u = v + 32768, v = round(x * 32767) in [-32767, 32767]).
constexpr float FIX16_SCALE = 32767.0f;
__device__ __forceinline__ unsigned fix16_pack(float a, float b) {
  const int ia = __float2int_rn(a * FIX16_SCALE), ib = __float2int_rn(b * FIX16_SCALE);
  return (((unsigned)ia & 0xffffu) | ((unsigned)ib << 16)) ^ 0x80008000u;
}
// decode without int->float conversions: byte-permuting u under the exponent
// bits of 2^23 gives the float 2^23 + u exactly, and subtracting 2^23 + 32768
// (exact, same exponent) leaves v -- one PRMT and one FADD per value.
__device__ __forceinline__ float2 fix16_unpack(unsigned w) {
  const float lo = __int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8421376.0f;
  const float hi = __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8421376.0f;
  return make_float2(lo, hi);
}

// Two values times k into one word (as fix16_pack(a * k / 32767, b * k /
// 32767)): adding 1.5 * 2^23 + 32768 rounds a float in [-32767, 32767] to the
// nearest integer in the low mantissa bits, already offset-binary, and one
// byte permute takes the two low halves.
constexpr float FIX16_ROUND = 12615680.0f;  // 1.5 * 2^23 + 32768
__device__ __forceinline__ unsigned fix16_pack_k(float a, float b, float k) {
  const float ra = fmaf(a, k, FIX16_ROUND), rb = fmaf(b, k, FIX16_ROUND);
  return __byte_perm(__float_as_uint(ra), __float_as_uint(rb), 0x5410);
}

// 256-bit global accesses (one request for 32 bytes; sm_100): p 32-byte aligned
__device__ __forceinline__ void ldg256(const void *p, unsigned (&w)[8]) {
  asm("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
      : "l"(p));
}
__device__ __forceinline__ void stg256(void *p, const unsigned (&w)[8]) {
  asm volatile("st.global.v8.u32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]),
               "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}

// site-blocked indexing
constexpr int SB = 32;
__host__ __device__ __forceinline__ int pad_sites(int Vh) { return (Vh + SB - 1) / SB * SB; }
template <int NC>
__host__ __device__ __forceinline__ size_t blk_base(int s) {
  return (size_t)(s >> 5) * NC * SB + (s & (SB - 1));
}

// SOA16: the 12 words of site s (words 0-7 at w8, 8-11 at w4)
constexpr int S16_BLOCK_BYTES = 32 * 48;
__host__ __device__ __forceinline__ size_t s16_w8(int s) { return (size_t)(s >> 5) * S16_BLOCK_BYTES + (s & 31) * 32; }
__host__ __device__ __forceinline__ size_t s16_w4(int s) {
  return (size_t)(s >> 5) * S16_BLOCK_BYTES + 1024 + (s & 31) * 16;
}
__device__ __forceinline__ void s16_load_words(const void *base, int s, unsigned (&w)[12]) {
  unsigned a[8];
  ldg256(static_cast<const char *>(base) + s16_w8(s), a);
  const uint4 b = __ldg(reinterpret_cast<const uint4 *>(static_cast<const char *>(base) + s16_w4(s)));
#pragma unroll
  for (int k = 0; k < 8; k++) w[k] = a[k];
  w[8] = b.x;
  w[9] = b.y;
  w[10] = b.z;
  w[11] = b.w;
}
__device__ __forceinline__ void s16_store_words(void *base, int s, const unsigned (&w)[12]) {
  unsigned a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = w[k];
  stg256(static_cast<char *>(base) + s16_w8(s), a);
  *reinterpret_cast<uint4 *>(static_cast<char *>(base) + s16_w4(s)) = make_uint4(w[8], w[9], w[10], w[11]);
}
// GSOA16: the 6 words of the link of site s in a slab starting `slab_sites` sites in
constexpr int G16_BLOCK_BYTES = 32 * 24;
__device__ __forceinline__ void g16_load_words(const void *base, size_t slab_sites, int s, unsigned (&w)[6]) {
  const char *blk = static_cast<const char *>(base) + slab_sites * 24 + (size_t)(s >> 5) * G16_BLOCK_BYTES;
  const uint4 a = __ldg(reinterpret_cast<const uint4 *>(blk) + (s & 31));
  const uint2 b = __ldg(reinterpret_cast<const uint2 *>(blk + 512) + (s & 31));
  w[0] = a.x;
  w[1] = a.y;
  w[2] = a.z;
  w[3] = a.w;
  w[4] = b.x;
  w[5] = b.y;
}

// Lattice geometry of one parity (half lattice).  Site index
// i = ((t*Lz + z)*Ly + y)*Lxh + xh, the PyQuda/qcu ordering.
struct Geom {
  int Lxh, Ly, Lz, Lt;
  int sy, sz, st;  // index strides of y, z, t
  int Vh;
  // reciprocal multipliers of Lxh, Ly, Lz: n / d = umulhi(n, m) for every
  // site index n (set by make_geom when that is exact, else 0: plain division)
  unsigned m_lxh = 0, m_ly = 0, m_lz = 0;
};

// n / d for 0 <= n < 2^31.  With m = ceil(2^32 / d) = (2^32 + e) / d, 0 <= e < d,
// n m / 2^32 = n / d + n e / (d 2^32), and the floor is exact while n e < 2^32
// (division by invariant integers, Granlund and Montgomery 1994); the host sets
// m only where Vh * d < 2^32 guarantees that, and 0 otherwise.
__host__ __device__ __forceinline__ int geom_div(int n, int d, unsigned m) {
#ifdef __CUDA_ARCH__
  return m ? (int)__umulhi((unsigned)n, m) : n / d;
#else
  return n / d;
#endif
}

// coordinates (xh, y, z, t) of site s of one parity
__host__ __device__ __forceinline__ void site_coords(const Geom &g, int s, int &xh, int &y, int &z, int &t) {
  const int r1 = geom_div(s, g.Lxh, g.m_lxh);
  xh = s - r1 * g.Lxh;
  const int r2 = geom_div(r1, g.Ly, g.m_ly);
  y = r1 - r2 * g.Ly;
  t = geom_div(r2, g.Lz, g.m_lz);
  z = r2 - t * g.Lz;
}

// ------------------------------------------------------------------ spinors
template <int K>
struct SpinorView {
  void *p;
  float *norm;  // SOA16 only
  int stride;
};

template <int K, typename T>
__device__ __forceinline__ void spinor_load(const SpinorView<K> &v, int s, Cpx<T> out[12]) {
  if constexpr (K == AOS64) {
    const double2 *p = static_cast<const double2 *>(v.p) + (size_t)s * 12;
#pragma unroll
    for (int c = 0; c < 12; c++) {
      double2 d = __ldg(p + c);
      out[c] = Cpx<T>((T)d.x, (T)d.y);
    }
  } else if constexpr (K == AOS64W) {
    // 32-byte loads (two complex numbers each) of a 32-byte aligned field: a
    // warp's request over 32 site-major records costs as many L1 wavefronts
    // as a 16-byte one, for twice the data
    const double2 *p = static_cast<const double2 *>(v.p) + (size_t)s * 12;
#pragma unroll
    for (int c = 0; c < 12; c += 2) {
      unsigned w[8];
      ldg256(p + c, w);
      out[c] = Cpx<T>((T)__hiloint2double(w[1], w[0]), (T)__hiloint2double(w[3], w[2]));
      out[c + 1] = Cpx<T>((T)__hiloint2double(w[5], w[4]), (T)__hiloint2double(w[7], w[6]));
    }
  } else if constexpr (K == SOA64) {
    const double2 *p = static_cast<const double2 *>(v.p) + blk_base<12>(s);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      double2 d = __ldg(p + c * SB);
      out[c] = Cpx<T>((T)d.x, (T)d.y);
    }
  } else if constexpr (K == SOA32) {
    const float4 *p = static_cast<const float4 *>(v.p) + blk_base<6>(s);
#pragma unroll
    for (int j = 0; j < 6; j++) {  // j = 3 * (spin pair) + colour
      float4 d = __ldg(p + j * SB);
      const int a = (j / 3) * 6 + j % 3;  // spin 2 * (j / 3), then spin 2 * (j / 3) + 1
      out[a] = Cpx<T>((T)d.x, (T)d.z);
      out[a + 3] = Cpx<T>((T)d.y, (T)d.w);
    }
  } else {
    const float nrm = __ldg(v.norm + s) * (1.0f / FIX16_SCALE);
    unsigned w[12];
    s16_load_words(v.p, s, w);
#pragma unroll
    for (int k = 0; k < 12; k++) {  // word k = 6 * (spin pair) + 2 * colour + (re, im)
      const float2 f = fix16_unpack(w[k]);
      const int a = (k / 6) * 6 + (k % 6) / 2;
      if (k % 2 == 0) {
        out[a].re = (T)(f.x * nrm);
        out[a + 3].re = (T)(f.y * nrm);
      } else {
        out[a].im = (T)(f.x * nrm);
        out[a + 3].im = (T)(f.y * nrm);
      }
    }
  }
}

template <int K, typename T>
__device__ __forceinline__ void spinor_store(const SpinorView<K> &v, int s, const Cpx<T> in[12]) {
  if constexpr (K == AOS64) {
    double2 *p = static_cast<double2 *>(v.p) + (size_t)s * 12;
#pragma unroll
    for (int c = 0; c < 12; c++) p[c] = make_double2((double)in[c].re, (double)in[c].im);
  } else if constexpr (K == AOS64W) {
    double2 *p = static_cast<double2 *>(v.p) + (size_t)s * 12;
#pragma unroll
    for (int c = 0; c < 12; c += 2) {
      const double v4[4] = {(double)in[c].re, (double)in[c].im, (double)in[c + 1].re, (double)in[c + 1].im};
      unsigned w[8];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        w[2 * k] = (unsigned)__double2loint(v4[k]);
        w[2 * k + 1] = (unsigned)__double2hiint(v4[k]);
      }
      stg256(p + c, w);
    }
  } else if constexpr (K == SOA64) {
    double2 *p = static_cast<double2 *>(v.p) + blk_base<12>(s);
#pragma unroll
    for (int c = 0; c < 12; c++) p[c * SB] = make_double2((double)in[c].re, (double)in[c].im);
  } else if constexpr (K == SOA32) {
    float4 *p = static_cast<float4 *>(v.p) + blk_base<6>(s);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const int a = (j / 3) * 6 + j % 3;
      p[j * SB] = make_float4((float)in[a].re, (float)in[a + 3].re, (float)in[a].im, (float)in[a + 3].im);
    }
  } else {
    float mx = 0.f;
#pragma unroll
    for (int c = 0; c < 12; c++) mx = fmaxf(mx, fmaxf(fabsf((float)in[c].re), fabsf((float)in[c].im)));
    const float k = mx > 0.f ? FIX16_SCALE / mx : 0.f;
    unsigned w[12];
#pragma unroll
    for (int q = 0; q < 12; q++) {
      const int a = (q / 6) * 6 + (q % 6) / 2;
      w[q] = q % 2 == 0 ? fix16_pack_k((float)in[a].re, (float)in[a + 3].re, k)
                        : fix16_pack_k((float)in[a].im, (float)in[a + 3].im, k);
    }
    s16_store_words(v.p, s, w);
    v.norm[s] = mx;
  }
}

// ------------------------------------------------------------------ gauge
template <int G>
struct GaugeView {
  const void *p;
  int stride;  // sites per (dir, parity) slab: Vh for GAOS64, pad_sites(Vh) otherwise
};

__device__ __forceinline__ void su3_row2(Cpx<float> *m) {
  m[6] = (m[1] * m[5] - m[2] * m[4]).conj();
  m[7] = (m[2] * m[3] - m[0] * m[5]).conj();
  m[8] = (m[0] * m[4] - m[1] * m[3]).conj();
}

// rows 0 and 1 of U_dir(site) on parity par, then row 2 = conj(row0 x row1)
template <int G, typename T>
__device__ __forceinline__ void link_load(const GaugeView<G> &u, int dir, int par, int s, Cpx<T> m[9]) {
  const size_t slab = (size_t)(dir * 2 + par) * u.stride;
  if constexpr (G == GAOS64) {
    const double2 *p = static_cast<const double2 *>(u.p) + (slab + s) * 9;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double2 d = __ldg(p + k);
      m[k] = Cpx<T>((T)d.x, (T)d.y);
    }
  } else if constexpr (G == GSOA64) {
    const double2 *p = static_cast<const double2 *>(u.p) + slab * 6 + blk_base<6>(s);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double2 d = __ldg(p + k * SB);
      m[k] = Cpx<T>((T)d.x, (T)d.y);
    }
  } else if constexpr (G == GSOA32) {
    const float4 *p = static_cast<const float4 *>(u.p) + slab * 3 + blk_base<3>(s);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float4 d = __ldg(p + k * SB);
      m[2 * k] = Cpx<T>((T)d.x, (T)d.y);
      m[2 * k + 1] = Cpx<T>((T)d.z, (T)d.w);
    }
  } else {
    unsigned w[6];
    g16_load_words(u.p, slab, s, w);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const float2 f = fix16_unpack(w[k]);
      m[k] = Cpx<T>((T)(f.x * (1.0f / FIX16_SCALE)), (T)(f.y * (1.0f / FIX16_SCALE)));
    }
  }
  m[6] = (m[1] * m[5] - m[2] * m[4]).conj();
  m[7] = (m[2] * m[3] - m[0] * m[5]).conj();
  m[8] = (m[0] * m[4] - m[1] * m[3]).conj();
}

// ------------------------------------------------------------------ stencil
// DeGrand-Rossi gamma matrices: row r of gamma_mu has one non-zero entry, in
// column GCOL[mu][r], with value GRE + i*GIM.  These are the projections qcu
// hard-codes in src/wilson_dslash.cu:56-243.
__host__ __device__ constexpr int gcol(int mu, int r) {
  return (mu < 2) ? (3 - r) : ((r + 2) & 3);
}
__host__ __device__ constexpr int gre(int mu, int r) {
  return mu == 1 ? ((r == 0 || r == 3) ? -1 : 1) : (mu == 3 ? 1 : 0);
}
__host__ __device__ constexpr int gim(int mu, int r) {
  return mu == 0 ? (r < 2 ? 1 : -1) : (mu == 2 ? ((r == 0 || r == 3) ? 1 : -1) : 0);
}

// acc += f U (1 - gamma_mu) psi   (FWD)   or   acc += f U^dag (1 + gamma_mu) psi   (!FWD)
// (f applied only when SCALED).  The projector has rank 2: rows 0,1 give
// h_k = psi_k + sigma*g_k*psi_col(k); rows 2,3 are sigma*g_m * h_col(m).
template <int MU, bool FWD, bool SCALED, typename T>
__device__ __forceinline__ void hop(Cpx<T> acc[12], const Cpx<T> psi[12], const Cpx<T> u[9], T f) {
  constexpr int S = FWD ? -1 : 1;
  Cpx<T> h[2][3], uh[2][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    h[0][c] = psi[c] + unit_mul<S * gre(MU, 0), S * gim(MU, 0)>(psi[gcol(MU, 0) * 3 + c]);
    h[1][c] = psi[3 + c] + unit_mul<S * gre(MU, 1), S * gim(MU, 1)>(psi[gcol(MU, 1) * 3 + c]);
  }
#pragma unroll
  for (int k = 0; k < 2; k++) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
      Cpx<T> s;
      if constexpr (FWD) {
        s = u[r * 3 + 0] * h[k][0];
        s += u[r * 3 + 1] * h[k][1];
        s += u[r * 3 + 2] * h[k][2];
      } else {
        s = cdotmul(u[0 * 3 + r], h[k][0]);
        s += cdotmul(u[1 * 3 + r], h[k][1]);
        s += cdotmul(u[2 * 3 + r], h[k][2]);
      }
      if constexpr (SCALED) s = s * f;
      uh[k][r] = s;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[c] += uh[0][c];
    acc[3 + c] += uh[1][c];
    acc[6 + c] += unit_mul<S * gre(MU, 2), S * gim(MU, 2)>(uh[gcol(MU, 2)][c]);
    acc[9 + c] += unit_mul<S * gre(MU, 3), S * gim(MU, 3)>(uh[gcol(MU, 3)][c]);
  }
}

// One hop: neighbour spinor n, link U_MU on (lpar, ls), boundary phase ph
// (the FP64 kinds; FP32 and 16-bit spinors take the paired path of hop32.cuh).
template <int MU, bool FWD, int K, int G, typename T>
__device__ __forceinline__ void hop_from(Cpx<T> acc[12], const SpinorView<K> &in, const GaugeView<G> &U, int n,
                                         int lpar, int ls, T ph) {
  Cpx<T> psi[12], u[9];
  spinor_load<K, T>(in, n, psi);
  link_load<G, T>(U, MU, lpar, ls, u);
  hop<MU, FWD, MU == 3, T>(acc, psi, u, ph);
}

// Hopping term D_{p <- 1-p} at output site s of parity `par`:
//   sum_mu U_mu(x)(1-g_mu) in(x+mu) + U_mu(x-mu)^+ (1+g_mu) in(x-mu)
// periodic in x,y,z; t-boundary hops multiplied by t_bc.
template <int K, int G, typename T>
__device__ __forceinline__ void wilson_hop_site(Cpx<T> acc[12], const SpinorView<K> &in, const GaugeView<G> &U,
                                                const Geom &g, int s, int par, T t_bc) {
#pragma unroll
  for (int c = 0; c < 12; c++) acc[c] = Cpx<T>(0, 0);
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int xodd = (y + z + t + par) & 1;  // full x = 2*xh + xodd
  int n;
  // x
  n = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  hop_from<0, true>(acc, in, U, n, par, s, T(1));
  n = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  hop_from<0, false>(acc, in, U, n, 1 - par, n, T(1));
  // y
  n = (y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  hop_from<1, true>(acc, in, U, n, par, s, T(1));
  n = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  hop_from<1, false>(acc, in, U, n, 1 - par, n, T(1));
  // z
  n = (z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  hop_from<2, true>(acc, in, U, n, par, s, T(1));
  n = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  hop_from<2, false>(acc, in, U, n, 1 - par, n, T(1));
  // t
  n = (t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  hop_from<3, true>(acc, in, U, n, par, s, (t == g.Lt - 1) ? t_bc : T(1));
  n = (t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
  hop_from<3, false>(acc, in, U, n, 1 - par, n, (t == 0) ? t_bc : T(1));
}

// ------------------------------------------------------------------ clover
// Packed clover (or inverse clover) per site: two Hermitian 6x6 chiral blocks
// (spins {0,1} and {2,3} in the DeGrand-Rossi basis), each 36 reals:
//   d[0..5] real diagonal, then L[i][j] (i>j) complex at i(i-1)/2 + j.
// Site-blocked like the spinors:
// CSOA64: double2, NC = 36 per site (block b at components 18b..18b+17:
//         the diagonal packed in 3 double2, then the 15 complex entries)
// CSOA32: float4,  NC = 18 per site (block b at components 9b..9b+8)
enum CloverKind { CSOA64 = 0, CSOA32 = 1 };
template <int C>
struct CloverView {
  const void *p;
  int stride;  // unused by the site-blocked layout (kept for symmetry with GaugeView)
};

template <int C, typename T>
__device__ __forceinline__ void clover_block_load(const CloverView<C> &cv, int blk, int s, T d[6], Cpx<T> L[15]) {
  if constexpr (C == CSOA64) {
    const double2 *p = static_cast<const double2 *>(cv.p) + blk_base<36>(s) + blk * 18 * SB;
    double2 q[18];
#pragma unroll
    for (int k = 0; k < 18; k++) q[k] = __ldg(p + k * SB);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      d[2 * k] = (T)q[k].x;
      d[2 * k + 1] = (T)q[k].y;
    }
#pragma unroll
    for (int k = 0; k < 15; k++) L[k] = Cpx<T>((T)q[3 + k].x, (T)q[3 + k].y);
  } else {
    const float4 *p = static_cast<const float4 *>(cv.p) + blk_base<18>(s) + blk * 9 * SB;
    float f[36];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float4 q = __ldg(p + k * SB);
      f[4 * k] = q.x;
      f[4 * k + 1] = q.y;
      f[4 * k + 2] = q.z;
      f[4 * k + 3] = q.w;
    }
#pragma unroll
    for (int k = 0; k < 6; k++) d[k] = (T)f[k];
#pragma unroll
    for (int k = 0; k < 15; k++) L[k] = Cpx<T>((T)f[6 + 2 * k], (T)f[7 + 2 * k]);
  }
}

// v <- C v for both chiral blocks of one site
template <int C, typename T>
__device__ __forceinline__ void clover_apply_site(const CloverView<C> &cv, int s, Cpx<T> v[12]) {
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    T d[6];
    Cpx<T> L[15];
    clover_block_load<C, T>(cv, blk, s, d, L);
    Cpx<T> x[6], y[6];
#pragma unroll
    for (int i = 0; i < 6; i++) x[i] = v[blk * 6 + i];
#pragma unroll
    for (int i = 0; i < 6; i++) y[i] = x[i] * d[i];
#pragma unroll
    for (int i = 1; i < 6; i++) {
#pragma unroll
      for (int j = 0; j < i; j++) {
        const Cpx<T> l = L[i * (i - 1) / 2 + j];
        y[i] += l * x[j];
        y[j] += cdotmul(l, x[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < 6; i++) v[blk * 6 + i] = y[i];
  }
}

}  // namespace qcu
