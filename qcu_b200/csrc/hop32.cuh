// FP32-arithmetic hopping term (FP32 and 16-bit spinors) on spin-paired registers.
//
// sm_100 issues two FP32 lanes per instruction (FFMA2 / FADD2 / FMUL2 on a
// float2).  The FP32 spinor storage (SOA32) keeps spins 0 and 1 -- and spins 2
// and 3 -- of one colour side by side, so a 16-byte load yields two such lane
// pairs, (re s0, re s1) and (im s0, im s1).  The rank-2 projector of the z and
// t hops combines spin 0 with 2 and spin 1 with 3, lane by lane; the x and y
// hops cross the lanes (0 with 3, 1 with 2) and are projected and
// reconstructed with scalar instructions.  The colour matrix-vector product,
// the largest share of the arithmetic, acts on both spins of the projected
// half spinor at once: every link element is held as a broadcast pair
// (u, u), built once per hop, and multiplies the pair (h0, h1).  The same
// arithmetic as the scalar hop (src/wilson_dslash.cu:56-243 of qcu), with half
// the FP32 instructions in the projection, the product and the reconstruction.
// The 16-bit spinors (SOA16) store the same lane pairs in one word each: one
// byte permute per value decodes them up to a constant offset, which the
// projection of a hop removes itself, exactly (fmak_biased, comb_biased).
#pragma once
#include "fields.cuh"

namespace qcu {

// One colour triplet of two spins, as lane pairs: re[c] = (re of spin a, re of
// spin b), im[c] likewise.
struct SpinPair {
  float2 re[3], im[3];
};
// One FP32 site: spins (0,1) and (2,3).
struct Site2 {
  SpinPair up, lo;
};
// One SU(3) link with every element broadcast to both lanes: re[r*3+c] = (Re U_rc, Re U_rc).
struct Link2 {
  float2 re[9], im[9];
};

__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
// a * (k0, k1) + c with compile-time constants k in {-1, 1}
template <int K0, int K1>
__device__ __forceinline__ float2 fmak(float2 a, float2 c) {
  if constexpr (K0 == 1 && K1 == 1) return add2(c, a);
  else if constexpr (K0 == -1 && K1 == -1) return add2(c, neg2(a));
  else return fma2(a, make_float2((float)K0, (float)K1), c);
}

constexpr float K16 = 8421376.0f;  // 2^23 + 32768: offset of a biased 16-bit value

// The same on biased inputs a = K16 + v_a, c = K16 + v_c (16-bit spinors):
// returns v_c + k v_a exactly.  A lane with k = -1 needs nothing (the offsets
// cancel in c - a); a lane with k = +1 first takes 2 K16 off c.  Every step is
// exact: the operands are integers below 2^24 and the sums cancel to |v| <= 65534.
template <int K0, int K1>
__device__ __forceinline__ float2 fmak_biased(float2 a, float2 c) {
  if constexpr (K0 == 1 || K1 == 1)
    c = add2(c, make_float2(K0 == 1 ? -2.0f * K16 : 0.0f, K1 == 1 ? -2.0f * K16 : 0.0f));
  return fmak<K0, K1>(a, c);
}
// scalar form: v_a + q, where q is a biased value times the unit SG (+1 or -1)
template <int SG>
__device__ __forceinline__ float comb_biased(float ra, float q) {
  if constexpr (SG > 0) return (ra - 2.0f * K16) + q;
  else return ra + q;
}
// sign (+1/-1) of the real and imaginary component of unit_mul<RE, IM>(z) relative to z's components
__host__ __device__ constexpr int unit_sign_re(int re, int im) { return re != 0 ? re : -im; }
__host__ __device__ constexpr int unit_sign_im(int re, int im) { return re != 0 ? re : im; }

// ------------------------------------------------------------------ SOA32 site I/O
__device__ __forceinline__ void site2_load(const SpinorView<SOA32> &v, int s, Site2 &o) {
  const float4 *p = static_cast<const float4 *>(v.p) + blk_base<6>(s);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float4 d = __ldg(p + c * SB), e = __ldg(p + (3 + c) * SB);
    o.up.re[c] = make_float2(d.x, d.y);
    o.up.im[c] = make_float2(d.z, d.w);
    o.lo.re[c] = make_float2(e.x, e.y);
    o.lo.im[c] = make_float2(e.z, e.w);
  }
}

__device__ __forceinline__ void site2_store(const SpinorView<SOA32> &v, int s, const Site2 &w) {
  float4 *p = static_cast<float4 *>(v.p) + blk_base<6>(s);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    p[c * SB] = make_float4(w.up.re[c].x, w.up.re[c].y, w.up.im[c].x, w.up.im[c].y);
    p[(3 + c) * SB] = make_float4(w.lo.re[c].x, w.lo.re[c].y, w.lo.im[c].x, w.lo.im[c].y);
  }
}

// canonical component order (spin * 3 + colour) <-> lane pairs; register renaming only
__device__ __forceinline__ void site2_to_cpx(const Site2 &w, Cpx<float> v[12]) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    v[c] = Cpx<float>(w.up.re[c].x, w.up.im[c].x);
    v[3 + c] = Cpx<float>(w.up.re[c].y, w.up.im[c].y);
    v[6 + c] = Cpx<float>(w.lo.re[c].x, w.lo.im[c].x);
    v[9 + c] = Cpx<float>(w.lo.re[c].y, w.lo.im[c].y);
  }
}
__device__ __forceinline__ void cpx_to_site2(const Cpx<float> v[12], Site2 &w) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w.up.re[c] = make_float2(v[c].re, v[3 + c].re);
    w.up.im[c] = make_float2(v[c].im, v[3 + c].im);
    w.lo.re[c] = make_float2(v[6 + c].re, v[9 + c].re);
    w.lo.im[c] = make_float2(v[6 + c].im, v[9 + c].im);
  }
}

__device__ __forceinline__ void site2_scale(Site2 &w, float2 f) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w.up.re[c] = mul2(w.up.re[c], f);
    w.up.im[c] = mul2(w.up.im[c], f);
    w.lo.re[c] = mul2(w.lo.re[c], f);
    w.lo.im[c] = mul2(w.lo.im[c], f);
  }
}
// w += f * x
__device__ __forceinline__ void site2_axpy(Site2 &w, float2 f, const Site2 &x) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w.up.re[c] = fma2(x.up.re[c], f, w.up.re[c]);
    w.up.im[c] = fma2(x.up.im[c], f, w.up.im[c]);
    w.lo.re[c] = fma2(x.lo.re[c], f, w.lo.re[c]);
    w.lo.im[c] = fma2(x.lo.im[c], f, w.lo.im[c]);
  }
}

// ------------------------------------------------------------------ SOA16 site I/O
// One 16-bit word -> its two values as a lane pair, in units of the stored
// scale (the decode of fix16_unpack, with one paired subtraction).
__device__ __forceinline__ float2 fix16_unpack2(unsigned w) {
  const float2 b = make_float2(__int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)),
                               __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
  return add2(b, bc2(-8421376.0f));
}

// SOA16 site in units of norm/32767 (word k = 6 q + 2 c + (re, im) is the lane
// pair of spins 2q, 2q + 1); returns the site norm.
__device__ __forceinline__ float site16_load_raw(const SpinorView<SOA16> &v, int s, Site2 &o) {
  unsigned w[12];
  s16_load_words(v.p, s, w);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o.up.re[c] = fix16_unpack2(w[2 * c]);
    o.up.im[c] = fix16_unpack2(w[2 * c + 1]);
    o.lo.re[c] = fix16_unpack2(w[6 + 2 * c]);
    o.lo.im[c] = fix16_unpack2(w[6 + 2 * c + 1]);
  }
  return __ldg(v.norm + s);
}

// The same site with the decode's offset left in: every value is r = K16 + v
// (K16 = 2^23 + 32768, v the integer value), exactly as the byte permute
// makes it.  The projection of a hop removes the offset itself (hop2), in
// fewer operations than decoding each value first.
__device__ __forceinline__ float2 fix16_biased2(unsigned w) {
  return make_float2(__int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)),
                     __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
}
// the same with the two halves exchanged: (spin b, spin a)
__device__ __forceinline__ float2 fix16_biased2_swapped(unsigned w) {
  return make_float2(__int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)),
                     __int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)));
}
// SWAP_LO: the lower spins come as (spin 3, spin 2), the lane order in which
// the x and y projections combine them with spins 0 and 1 (the byte permute
// places each half where it is wanted, at no cost)
template <bool SWAP_LO>
__device__ __forceinline__ float site16_load_biased(const SpinorView<SOA16> &v, int s, Site2 &o) {
  unsigned w[12];
  s16_load_words(v.p, s, w);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o.up.re[c] = fix16_biased2(w[2 * c]);
    o.up.im[c] = fix16_biased2(w[2 * c + 1]);
    if constexpr (SWAP_LO) {
      o.lo.re[c] = fix16_biased2_swapped(w[6 + 2 * c]);
      o.lo.im[c] = fix16_biased2_swapped(w[6 + 2 * c + 1]);
    } else {
      o.lo.re[c] = fix16_biased2(w[6 + 2 * c]);
      o.lo.im[c] = fix16_biased2(w[6 + 2 * c + 1]);
    }
  }
  return __ldg(v.norm + s);
}

// pack a lane pair times k (k = 32767 / norm) into one word (fix16_pack_k, paired)
__device__ __forceinline__ unsigned fix16_pack2(float2 v, float2 k) {
  const float2 r = fma2(v, k, bc2(FIX16_ROUND));
  return __byte_perm(__float_as_uint(r.x), __float_as_uint(r.y), 0x5410);
}

__device__ __forceinline__ void site16_store(const SpinorView<SOA16> &v, int s, const Site2 &x) {
  float mx = 0.f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(x.up.re[c].x), fabsf(x.up.re[c].y)), fmaxf(fabsf(x.up.im[c].x), fabsf(x.up.im[c].y))));
    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(x.lo.re[c].x), fabsf(x.lo.re[c].y)), fmaxf(fabsf(x.lo.im[c].x), fabsf(x.lo.im[c].y))));
  }
  const float2 k = bc2(mx > 0.f ? FIX16_SCALE / mx : 0.f);
  unsigned w[12];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w[2 * c] = fix16_pack2(x.up.re[c], k);
    w[2 * c + 1] = fix16_pack2(x.up.im[c], k);
    w[6 + 2 * c] = fix16_pack2(x.lo.re[c], k);
    w[6 + 2 * c + 1] = fix16_pack2(x.lo.im[c], k);
  }
  s16_store_words(v.p, s, w);
  v.norm[s] = mx;
}

// a site of an FP32 (SOA32) or 16-bit (SOA16) field as lane pairs, in value units
template <int K>
__device__ __forceinline__ void site_load2(const SpinorView<K> &v, int s, Site2 &o) {
  if constexpr (K == SOA32) {
    site2_load(v, s, o);
  } else {
    static_assert(K == SOA16, "paired site I/O: SOA32 or SOA16");
    const float nrm = site16_load_raw(v, s, o);
    site2_scale(o, bc2(nrm * (1.0f / FIX16_SCALE)));
  }
}
template <int K>
__device__ __forceinline__ void site_store2(const SpinorView<K> &v, int s, const Site2 &w) {
  if constexpr (K == SOA32) site2_store(v, s, w);
  else site16_store(v, s, w);
}

// ------------------------------------------------------------------ links
// row 2 = conj(row0 x row1), each element as one FMUL and three FFMA per
// component, then broadcast (k = 3 * r + c).  Scalar: a paired instruction
// takes the FMA pipe for two lanes, so a broadcast pair would cost twice.
__device__ __forceinline__ Cpx<float> conj_cross(const Cpx<float> &a, const Cpx<float> &b, const Cpx<float> &c,
                                                 const Cpx<float> &d) {  // conj(a b - c d)
  const float re = fmaf(a.re, b.re, fmaf(-a.im, b.im, fmaf(-c.re, d.re, c.im * d.im)));
  const float im = fmaf(c.re, d.im, fmaf(c.im, d.re, fmaf(-a.re, b.im, -(a.im * b.re))));
  return Cpx<float>(re, im);
}
__device__ __forceinline__ void link2_row2(Link2 &m) {
  Cpx<float> r[6];
#pragma unroll
  for (int k = 0; k < 6; k++) r[k] = Cpx<float>(m.re[k].x, m.im[k].x);
  const Cpx<float> r6 = conj_cross(r[1], r[5], r[2], r[4]);
  const Cpx<float> r7 = conj_cross(r[2], r[3], r[0], r[5]);
  const Cpx<float> r8 = conj_cross(r[0], r[4], r[1], r[3]);
  m.re[6] = bc2(r6.re);
  m.im[6] = bc2(r6.im);
  m.re[7] = bc2(r7.re);
  m.im[7] = bc2(r7.im);
  m.re[8] = bc2(r8.re);
  m.im[8] = bc2(r8.im);
}

// GSOA16 rows 0-1 are integers (units of 1/32767), so the rebuilt row 2 is
// in units of 1/32767^2: the hop multiplies its share of the product by the
// extra 1/32767 (hop2, R2F), on two lane pairs instead of six scalars.
template <int G>
constexpr bool link2_row2_raw() {
  return G == GSOA16;
}
constexpr float LINK16_ROW2_F = 1.0f / FIX16_SCALE;

// GSOA32: rows 0-1 as stored, row 2 rebuilt.  Returns the unit of the
// elements (1).
// GSOA16: rows 0-1 in units of 1/32767, row 2 rebuilt in units of 1/32767^2.
// Returns the unit of rows 0-1 (1/32767), applied once to the whole hop sum.
template <int G>
__device__ __forceinline__ float link2_load(const GaugeView<G> &u, int dir, int par, int s, Link2 &m) {
  const size_t slab = (size_t)(dir * 2 + par) * u.stride;
  if constexpr (G == GSOA32) {
    const float4 *p = static_cast<const float4 *>(u.p) + slab * 3 + blk_base<3>(s);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float4 d = __ldg(p + k * SB);
      m.re[2 * k] = bc2(d.x);
      m.im[2 * k] = bc2(d.y);
      m.re[2 * k + 1] = bc2(d.z);
      m.im[2 * k + 1] = bc2(d.w);
    }
    link2_row2(m);
    return 1.0f;
  } else {
    static_assert(G == GSOA16, "FP32 hop: GSOA32 or GSOA16 links");
    unsigned w[6];
    g16_load_words(u.p, slab, s, w);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const float2 a = fix16_unpack(w[k]);
      m.re[k] = bc2(a.x);
      m.im[k] = bc2(a.y);
    }
    link2_row2(m);
    return 1.0f / FIX16_SCALE;
  }
}

// ------------------------------------------------------------------ one hop
// acc += f U (1 - gamma_mu) psi (FWD) or f U^dag (1 + gamma_mu) psi (!FWD).
// f (the time-boundary phase, times the neighbour's norm for 16-bit spinors)
// scales the projected half spinor; it is taken as 1 unless MU == 3 or
// SCALED.  Gamma conventions as gcol / gre / gim in fields.cuh.
// BIASED: psi holds the biased values of a 16-bit spinor (site16_load_biased);
// the projection returns exact values all the same.
// R2F: row 2 of u is in units of r2f times those of rows 0-1 (link2_row2_raw).
// With BIASED, the x and y hops (MU < 2) take psi with its lower spins
// swapped (site16_load_biased<true>), so that their projection, too, runs
// lane by lane.
template <int MU, bool FWD, bool SCALED, bool BIASED = false, bool R2F = false>
__device__ __forceinline__ void hop2(Site2 &acc, const Site2 &psi, const Link2 &u, float ph, float r2f = 1.0f) {
  constexpr int S = FWD ? -1 : 1;
  SpinPair h, uh;
  // rows 0, 1 of the projector: h_r = psi_r + S g(mu,r) psi_gcol(mu,r)
  if constexpr (MU >= 2 || BIASED) {  // lane-aligned: gcol = 2, 3, or 3, 2 against swapped lower spins
    constexpr int A0 = S * gre(MU, 0), A1 = S * gre(MU, 1), B0 = S * gim(MU, 0), B1 = S * gim(MU, 1);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if constexpr (BIASED) {
        if constexpr (A0 != 0) {
          h.re[c] = fmak_biased<A0, A1>(psi.lo.re[c], psi.up.re[c]);
          h.im[c] = fmak_biased<A0, A1>(psi.lo.im[c], psi.up.im[c]);
        } else {
          h.re[c] = fmak_biased<-B0, -B1>(psi.lo.im[c], psi.up.re[c]);
          h.im[c] = fmak_biased<B0, B1>(psi.lo.re[c], psi.up.im[c]);
        }
      } else if constexpr (A0 != 0) {
        h.re[c] = fmak<A0, A1>(psi.lo.re[c], psi.up.re[c]);
        h.im[c] = fmak<A0, A1>(psi.lo.im[c], psi.up.im[c]);
      } else {
        h.re[c] = fmak<-B0, -B1>(psi.lo.im[c], psi.up.re[c]);
        h.im[c] = fmak<B0, B1>(psi.lo.re[c], psi.up.im[c]);
      }
    }
  } else {  // gcol = 3, 2: crossed lanes, scalar
#pragma unroll
    for (int c = 0; c < 3; c++) {  // h_0 from spin 3 (lane y), h_1 from spin 2 (lane x)
      constexpr int R0 = S * gre(MU, 0), I0 = S * gim(MU, 0), R1 = S * gre(MU, 1), I1 = S * gim(MU, 1);
      const Cpx<float> q0 = unit_mul<R0, I0>(Cpx<float>(psi.lo.re[c].y, psi.lo.im[c].y));
      const Cpx<float> q1 = unit_mul<R1, I1>(Cpx<float>(psi.lo.re[c].x, psi.lo.im[c].x));
      if constexpr (BIASED) {
        h.re[c] = make_float2(comb_biased<unit_sign_re(R0, I0)>(psi.up.re[c].x, q0.re),
                              comb_biased<unit_sign_re(R1, I1)>(psi.up.re[c].y, q1.re));
        h.im[c] = make_float2(comb_biased<unit_sign_im(R0, I0)>(psi.up.im[c].x, q0.im),
                              comb_biased<unit_sign_im(R1, I1)>(psi.up.im[c].y, q1.im));
      } else {
        h.re[c] = make_float2(psi.up.re[c].x + q0.re, psi.up.re[c].y + q1.re);
        h.im[c] = make_float2(psi.up.im[c].x + q0.im, psi.up.im[c].y + q1.im);
      }
    }
  }
  // U^dag h takes row 2 of U with colour 2 of h only: its factor goes there
  constexpr bool R2_ON_H = R2F && !FWD;
  if constexpr (MU == 3 || SCALED) {
    const float2 f = bc2(ph);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 fc = (R2_ON_H && c == 2) ? bc2(ph * r2f) : f;
      h.re[c] = mul2(h.re[c], fc);
      h.im[c] = mul2(h.im[c], fc);
    }
  } else if constexpr (R2_ON_H) {
    h.re[2] = mul2(h.re[2], bc2(r2f));
    h.im[2] = mul2(h.im[2], bc2(r2f));
  }
  // colour product on both spins at once
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 re, im;
    if constexpr (FWD) {  // U h
      re = mul2(u.re[r * 3], h.re[0]);
      im = mul2(u.re[r * 3], h.im[0]);
      re = fma2(neg2(u.im[r * 3]), h.im[0], re);
      im = fma2(u.im[r * 3], h.re[0], im);
#pragma unroll
      for (int c = 1; c < 3; c++) {
        re = fma2(u.re[r * 3 + c], h.re[c], re);
        im = fma2(u.re[r * 3 + c], h.im[c], im);
        re = fma2(neg2(u.im[r * 3 + c]), h.im[c], re);
        im = fma2(u.im[r * 3 + c], h.re[c], im);
      }
    } else {  // U^dag h
      re = mul2(u.re[r], h.re[0]);
      im = mul2(u.re[r], h.im[0]);
      re = fma2(u.im[r], h.im[0], re);
      im = fma2(neg2(u.im[r]), h.re[0], im);
#pragma unroll
      for (int c = 1; c < 3; c++) {
        re = fma2(u.re[c * 3 + r], h.re[c], re);
        im = fma2(u.re[c * 3 + r], h.im[c], im);
        re = fma2(u.im[c * 3 + r], h.im[c], re);
        im = fma2(neg2(u.im[c * 3 + r]), h.re[c], im);
      }
    }
    if constexpr (R2F && FWD) {
      if (r == 2) {  // U h takes row 2 of U in row 2 of the result only
        re = mul2(re, bc2(r2f));
        im = mul2(im, bc2(r2f));
      }
    }
    uh.re[r] = re;
    uh.im[r] = im;
  }
  // rows 0, 1 of the result; rows 2, 3 = S g(mu,r) uh_gcol(mu,r)
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc.up.re[c] = add2(acc.up.re[c], uh.re[c]);
    acc.up.im[c] = add2(acc.up.im[c], uh.im[c]);
  }
  if constexpr (MU >= 2) {  // gcol = 0, 1: lane-aligned
    constexpr int A2 = S * gre(MU, 2), A3 = S * gre(MU, 3), B2 = S * gim(MU, 2), B3 = S * gim(MU, 3);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if constexpr (A2 != 0) {
        acc.lo.re[c] = fmak<A2, A3>(uh.re[c], acc.lo.re[c]);
        acc.lo.im[c] = fmak<A2, A3>(uh.im[c], acc.lo.im[c]);
      } else {
        acc.lo.re[c] = fmak<-B2, -B3>(uh.im[c], acc.lo.re[c]);
        acc.lo.im[c] = fmak<B2, B3>(uh.re[c], acc.lo.im[c]);
      }
    }
  } else {  // gcol = 1, 0: crossed lanes, scalar
#pragma unroll
    for (int c = 0; c < 3; c++) {  // row 2 from uh_1 (lane y), row 3 from uh_0 (lane x)
      const Cpx<float> v2 = unit_mul<S * gre(MU, 2), S * gim(MU, 2)>(Cpx<float>(uh.re[c].y, uh.im[c].y));
      const Cpx<float> v3 = unit_mul<S * gre(MU, 3), S * gim(MU, 3)>(Cpx<float>(uh.re[c].x, uh.im[c].x));
      acc.lo.re[c].x += v2.re;
      acc.lo.im[c].x += v2.im;
      acc.lo.re[c].y += v3.re;
      acc.lo.im[c].y += v3.im;
    }
  }
}

template <int MU, bool FWD, int K, int G>
__device__ __forceinline__ float hop2_from(Site2 &acc, const SpinorView<K> &in, const GaugeView<G> &U, int n,
                                           int lpar, int ls, float ph) {
  Site2 psi;
  Link2 u;
  if constexpr (K == SOA16) ph *= site16_load_biased<(MU < 2)>(in, n, psi) * (1.0f / FIX16_SCALE);
  else site2_load(in, n, psi);
  const float unit = link2_load<G>(U, MU, lpar, ls, u);
  hop2<MU, FWD, K == SOA16, K == SOA16, link2_row2_raw<G>()>(acc, psi, u, ph, LINK16_ROW2_F);
  return unit;
}

// Hopping term D_{p <- 1-p} at output site s of parity par, FP32 or 16-bit spinors:
// acc = the sum over the eight hops in units of the returned value (1/32767
// for 16-bit links, 1 for FP32 links), which the caller folds into its own
// scale factor.  Neighbour indexing as wilson_hop_site.
template <int K, int G>
__device__ __forceinline__ float wilson_hop_site2(Site2 &acc, const SpinorView<K> &in, const GaugeView<G> &U,
                                                  const Geom &g, int s, int par, float t_bc) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc.up.re[c] = acc.up.im[c] = acc.lo.re[c] = acc.lo.im[c] = make_float2(0.f, 0.f);
  }
  int xh, y, z, t;
  site_coords(g, s, xh, y, z, t);
  const int xodd = (y + z + t + par) & 1;
  int n;
  float unit;
  n = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  unit = hop2_from<0, true>(acc, in, U, n, par, s, 1.f);
  n = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  hop2_from<0, false>(acc, in, U, n, 1 - par, n, 1.f);
  n = (y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  hop2_from<1, true>(acc, in, U, n, par, s, 1.f);
  n = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  hop2_from<1, false>(acc, in, U, n, 1 - par, n, 1.f);
  n = (z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  hop2_from<2, true>(acc, in, U, n, par, s, 1.f);
  n = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  hop2_from<2, false>(acc, in, U, n, 1 - par, n, 1.f);
  n = (t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  hop2_from<3, true>(acc, in, U, n, par, s, (t == g.Lt - 1) ? t_bc : 1.f);
  n = (t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
  hop2_from<3, false>(acc, in, U, n, 1 - par, n, (t == 0) ? t_bc : 1.f);
  return unit;
}

}  // namespace qcu
