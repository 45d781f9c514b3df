// Domain-decomposed hopping term: ncclDslashQcu on a grid of ranks.
//
// qcu splits the global lattice over a 4-D grid of MPI ranks, one GPU each
// (include/lattice_set.h:89-128, include/lattice_dslash.h:11-197,
// src/wilson_dslash.cu:246-1234): every rank holds its local sub-lattice in
// PyQuda layout, and every hop that leaves the sub-lattice in a partitioned
// direction takes its neighbour's contribution from a face exchanged with
// the neighbouring rank.  The same result here, B200-first:
//
//   1. k_dd_pack: one thread per input site; a site on the low face of a
//      partitioned direction mu projects its spinor for the neighbour's
//      forward hop, (1 - gamma_mu) psi -> 2 spins x 3 colours; a site on the
//      high face multiplies the projection for the neighbour's backward hop
//      by its own link, U_mu(x)^dag (1 + gamma_mu) psi (the link lives on the
//      sending rank).  Six complex numbers per face site cross the link
//      instead of twelve.
//   2. the faces are exchanged on a stream of their own: NCCL point-to-point
//      (grouped send/recv to the two neighbours of every partitioned
//      direction), or device-to-device copies when all ranks of a grid are
//      emulated in one process on one GPU (qcuDslashDDEmulate, the test of
//      the kernels and the exchange schedule without a second GPU); the
//      interior sites, whose hops read no face, are computed meanwhile on
//      the library stream, the boundary sites (a list built once per
//      lattice, partition and parity) once the faces have landed;
//   3. k_dd_dslash: one thread per output site, the eight hops in the order
//      of the single-GPU kernel; a hop that crosses a partitioned boundary
//      reads the received face (forward: multiply by the local link;
//      backward: already multiplied) and reconstructs the four spins.  The
//      arithmetic of every hop is the single-GPU kernel's, operation for
//      operation, so the result equals the single-GPU dslash of the global
//      lattice bit for bit.
//
// Rank <-> grid coordinate (qcu's mapping, lattice_set.h:89-95): t fastest,
// rank = ((gx * Gy + gy) * Gz + gz) * Gt + gt; neighbours wrap periodically.
// Every local extent must be even, so that local and global site parities
// agree.  NCCL is opened with dlopen at the first distributed call, so the
// library has no load-time dependency on it and, in a process that already
// loaded NCCL (torch), uses that copy.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "dd.h"
#include "rng.cuh"

namespace qcu {

// ---------------------------------------------------------------- plan
DDPlan dd_plan(const int latt[4], const int grid[4], int rank) {
  require(latt != nullptr && grid != nullptr, "dd: null lattice or grid");
  DDPlan p;
  p.nranks = 1;
  for (int d = 0; d < 4; d++) {
    require(grid[d] >= 1, "dd: grid sizes must be >= 1");
    require(latt[d] >= 2 && latt[d] % 2 == 0, "dd: every local lattice extent must be even and >= 2");
    p.grid[d] = grid[d];
    p.latt[d] = latt[d];
    p.nranks *= grid[d];
  }
  require(rank >= 0 && rank < p.nranks, "dd: rank out of range for the grid");
  p.rank = rank;
  const int G[4] = {grid[0], grid[1], grid[2], grid[3]};
  p.coord[0] = rank / G[3] / G[2] / G[1];
  p.coord[1] = rank / G[3] / G[2] % G[1];
  p.coord[2] = rank / G[3] % G[2];
  p.coord[3] = rank % G[3];
  const int stride[4] = {G[1] * G[2] * G[3], G[2] * G[3], G[3], 1};
  for (int d = 0; d < 4; d++) {
    const int c = p.coord[d];
    p.fwd[d] = rank + ((c + 1) % G[d] - c) * stride[d];
    p.bwd[d] = rank + ((c + G[d] - 1) % G[d] - c) * stride[d];
  }
  const int Lxh = latt[0] / 2, Ly = latt[1], Lz = latt[2], Lt = latt[3];
  const int64_t faces[4] = {(int64_t)Ly * Lz * Lt / 2, (int64_t)Lxh * Lz * Lt, (int64_t)Lxh * Ly * Lt,
                            (int64_t)Lxh * Ly * Lz};
  for (int d = 0; d < 4; d++) p.face[d] = G[d] > 1 ? (int)faces[d] : 0;
  return p;
}

std::vector<DDOp> dd_schedule(const DDPlan &p) {
  // per partitioned direction, the same four steps in the same order on every
  // rank; with a grid of 2 the two neighbours are one rank, and its two
  // messages pair up with this rank's two receives by order
  std::vector<DDOp> ops;
  for (int d = 0; d < 4; d++) {
    if (p.grid[d] == 1) continue;
    const int n = p.face[d] * DD_FACE_COMPLEX;
    ops.push_back({DD_SEND, d, 0, p.bwd[d], n});  // send[d][0]: my low face, for bwd's forward hops
    ops.push_back({DD_RECV, d, 0, p.fwd[d], n});  // halo[d][0]: fwd's low face, for my forward hops
    ops.push_back({DD_SEND, d, 1, p.fwd[d], n});  // send[d][1]: U^dag-multiplied high face, for fwd's backward hops
    ops.push_back({DD_RECV, d, 1, p.bwd[d], n});  // halo[d][1]: bwd's high face, for my backward hops
  }
  return ops;
}

// ---------------------------------------------------------------- device
struct DDDev {
  Geom g;
  int part;                  // bit d: direction d is partitioned
  double2 *send[4][2];       // [d][0] low face (projected), [d][1] high face (U^dag projected)
  const double2 *halo[4][2]; // [d][0] from the forward rank, [d][1] from the backward rank
};

struct Coord {
  int x, y, z, t;
};
__device__ __forceinline__ Coord dd_coord(const Geom &g, int s, int par) {
  Coord c;
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  c.y = r % g.Ly;
  r /= g.Ly;
  c.z = r % g.Lz;
  c.t = r / g.Lz;
  c.x = 2 * xh + ((c.y + c.z + c.t + par) & 1);
  return c;
}
// index of a site in the face orthogonal to direction MU (the same for the
// two sites a hop joins, which differ only in their MU coordinate)
template <int MU>
__device__ __forceinline__ int dd_face_index(const Geom &g, const Coord &c) {
  if constexpr (MU == 0) return ((c.t * g.Lz + c.z) * g.Ly + c.y) >> 1;
  else if constexpr (MU == 1) return (c.t * g.Lz + c.z) * g.Lxh + (c.x >> 1);
  else if constexpr (MU == 2) return (c.t * g.Ly + c.y) * g.Lxh + (c.x >> 1);
  else return (c.z * g.Ly + c.y) * g.Lxh + (c.x >> 1);
}
template <int MU>
__device__ __forceinline__ int dd_pos(const Coord &c) {
  return MU == 0 ? c.x : (MU == 1 ? c.y : (MU == 2 ? c.z : c.t));
}
template <int MU>
__device__ __forceinline__ int dd_extent(const Geom &g) {
  return MU == 0 ? 2 * g.Lxh : (MU == 1 ? g.Ly : (MU == 2 ? g.Lz : g.Lt));
}

// the three stages of hop<> (fields.cuh), separately
template <int MU, bool FWD>
__device__ __forceinline__ void dd_project(const Cpx<double> psi[12], Cpx<double> h[2][3]) {
  constexpr int S = FWD ? -1 : 1;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    h[0][c] = psi[c] + unit_mul<S * gre(MU, 0), S * gim(MU, 0)>(psi[gcol(MU, 0) * 3 + c]);
    h[1][c] = psi[3 + c] + unit_mul<S * gre(MU, 1), S * gim(MU, 1)>(psi[gcol(MU, 1) * 3 + c]);
  }
}
template <bool FWD>
__device__ __forceinline__ void dd_colour(const Cpx<double> u[9], const Cpx<double> h[2][3], Cpx<double> uh[2][3]) {
#pragma unroll
  for (int k = 0; k < 2; k++) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
      Cpx<double> s;
      if constexpr (FWD) {
        s = u[r * 3 + 0] * h[k][0];
        s += u[r * 3 + 1] * h[k][1];
        s += u[r * 3 + 2] * h[k][2];
      } else {
        s = cdotmul(u[0 * 3 + r], h[k][0]);
        s += cdotmul(u[1 * 3 + r], h[k][1]);
        s += cdotmul(u[2 * 3 + r], h[k][2]);
      }
      uh[k][r] = s;
    }
  }
}
template <int MU, bool FWD>
__device__ __forceinline__ void dd_reconstruct(Cpx<double> acc[12], const Cpx<double> uh[2][3]) {
  constexpr int S = FWD ? -1 : 1;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[c] += uh[0][c];
    acc[3 + c] += uh[1][c];
    acc[6 + c] += unit_mul<S * gre(MU, 2), S * gim(MU, 2)>(uh[gcol(MU, 2)][c]);
    acc[9 + c] += unit_mul<S * gre(MU, 3), S * gim(MU, 3)>(uh[gcol(MU, 3)][c]);
  }
}

__device__ __forceinline__ void dd_face_store(double2 *buf, int f, const Cpx<double> v[2][3]) {
  double2 *p = buf + (size_t)f * DD_FACE_COMPLEX;
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int c = 0; c < 3; c++) p[k * 3 + c] = make_double2(v[k][c].re, v[k][c].im);
}
__device__ __forceinline__ void dd_face_load(const double2 *buf, int f, Cpx<double> v[2][3]) {
  const double2 *p = buf + (size_t)f * DD_FACE_COMPLEX;
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 d = __ldg(p + k * 3 + c);
      v[k][c] = Cpx<double>(d.x, d.y);
    }
}

template <int MU>
__device__ __forceinline__ void dd_pack_dir(const DDDev &d, const GaugeView<GAOS64> &U, const Coord &c,
                                            const Cpx<double> psi[12], int s, int par) {
  if (!(d.part >> MU & 1)) return;
  const int pos = dd_pos<MU>(c);
  const int f = dd_face_index<MU>(d.g, c);
  if (pos == 0) {  // the backward rank's forward hops land here
    Cpx<double> h[2][3];
    dd_project<MU, true>(psi, h);
    dd_face_store(d.send[MU][0], f, h);
  }
  if (pos == dd_extent<MU>(d.g) - 1) {  // the forward rank's backward hops: U_mu(x)^dag on this rank
    Cpx<double> h[2][3], uh[2][3], u[9];
    dd_project<MU, false>(psi, h);
    link_load<GAOS64, double>(U, MU, par, s, u);
    dd_colour<false>(u, h, uh);
    dd_face_store(d.send[MU][1], f, uh);
  }
}

// faces of the input spinor (parity par), PyQuda layout
__global__ void k_dd_pack(DDDev d, const double2 *__restrict__ in, const void *gauge, int par) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= d.g.Vh) return;
  const Coord c = dd_coord(d.g, s, par);
  bool on_face = false;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const int pos = mu == 0 ? c.x : (mu == 1 ? c.y : (mu == 2 ? c.z : c.t));
    const int L = mu == 0 ? 2 * d.g.Lxh : (mu == 1 ? d.g.Ly : (mu == 2 ? d.g.Lz : d.g.Lt));
    on_face |= (d.part >> mu & 1) && (pos == 0 || pos == L - 1);
  }
  if (!on_face) return;
  Cpx<double> psi[12];
  spinor_load<AOS64, double>(SpinorView<AOS64>{const_cast<double2 *>(in), nullptr, d.g.Vh}, s, psi);
  const GaugeView<GAOS64> U{gauge, d.g.Vh};
  dd_pack_dir<0>(d, U, c, psi, s, par);
  dd_pack_dir<1>(d, U, c, psi, s, par);
  dd_pack_dir<2>(d, U, c, psi, s, par);
  dd_pack_dir<3>(d, U, c, psi, s, par);
}

// one hop of the output site s: local neighbour n (periodic inside the
// sub-lattice) or, across a partitioned boundary, the received face
template <int MU, bool FWD>
__device__ __forceinline__ void dd_hop(Cpx<double> acc[12], const DDDev &d, const SpinorView<AOS64> &in,
                                       const GaugeView<GAOS64> &U, const Coord &c, int s, int n, int par) {
  const int pos = dd_pos<MU>(c);
  const bool cross = (d.part >> MU & 1) && (FWD ? pos == dd_extent<MU>(d.g) - 1 : pos == 0);
  if (!cross) {
    // the single-GPU hop: link U_mu(x) (forward) or U_mu(x - mu) (backward, on the neighbour)
    hop_from<MU, FWD>(acc, in, U, n, FWD ? par : 1 - par, FWD ? s : n, 1.0);
    return;
  }
  const int f = dd_face_index<MU>(d.g, c);
  Cpx<double> uh[2][3];
  if constexpr (FWD) {
    Cpx<double> h[2][3], u[9];
    dd_face_load(d.halo[MU][0], f, h);
    link_load<GAOS64, double>(U, MU, par, s, u);
    dd_colour<true>(u, h, uh);
  } else {
    dd_face_load(d.halo[MU][1], f, uh);
  }
  dd_reconstruct<MU, FWD>(acc, uh);
}

// a site on the face of a partitioned direction: one of its hops reads a received face
__device__ __forceinline__ bool dd_on_face(const DDDev &d, const Coord &c) {
  bool on = false;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const int pos = mu == 0 ? c.x : (mu == 1 ? c.y : (mu == 2 ? c.z : c.t));
    const int L = mu == 0 ? 2 * d.g.Lxh : (mu == 1 ? d.g.Ly : (mu == 2 ? d.g.Lz : d.g.Lt));
    on |= (d.part >> mu & 1) && (pos == 0 || pos == L - 1);
  }
  return on;
}

// the output sites of parity par that read a received face (any order: each
// site is computed on its own)
__global__ void k_dd_boundary_list(DDDev d, int par, int *list, int *count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= d.g.Vh) return;
  if (dd_on_face(d, dd_coord(d.g, s, par))) list[atomicAdd(count, 1)] = s;
}

// mode 0: every output site; 1: the interior (no hop reads a received face),
// which runs while the faces are in flight; 2: the nlist boundary sites of
// list, after the faces landed
__global__ void __launch_bounds__(DSLASH_BLOCK, 3)
    k_dd_dslash(DDDev d, const double2 *__restrict__ in, const void *gauge, double2 *out, int par, int mode,
                const int *list, int nlist) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (mode == 2) {
    if (s >= nlist) return;
    s = list[s];
  } else if (s >= d.g.Vh) {
    return;
  }
  const Geom &g = d.g;
  const SpinorView<AOS64> inv{const_cast<double2 *>(in), nullptr, g.Vh};
  const GaugeView<GAOS64> U{gauge, g.Vh};
  const Coord c = dd_coord(g, s, par);
  if (mode == 1 && dd_on_face(d, c)) return;
  const int xh = c.x >> 1, xodd = c.x & 1;
  Cpx<double> acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = Cpx<double>(0, 0);
  // neighbour indices as wilson_hop_site (fields.cuh)
  int n = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  dd_hop<0, true>(acc, d, inv, U, c, s, n, par);
  n = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  dd_hop<0, false>(acc, d, inv, U, c, s, n, par);
  n = (c.y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  dd_hop<1, true>(acc, d, inv, U, c, s, n, par);
  n = (c.y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  dd_hop<1, false>(acc, d, inv, U, c, s, n, par);
  n = (c.z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  dd_hop<2, true>(acc, d, inv, U, c, s, n, par);
  n = (c.z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  dd_hop<2, false>(acc, d, inv, U, c, s, n, par);
  n = (c.t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  dd_hop<3, true>(acc, d, inv, U, c, s, n, par);
  n = (c.t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
  dd_hop<3, false>(acc, d, inv, U, c, s, n, par);
  spinor_store<AOS64, double>(SpinorView<AOS64>{out, nullptr, g.Vh}, s, acc);
}

// ---------------------------------------------------------------- vector kernels of the distributed solver
// out = a x + b y + c z on n complex numbers (y, z optional); out may alias any input
__global__ void k_dd_lin3(int64_t n, double2 *out, double2 a, const double2 *x, double2 b, const double2 *y,
                          double2 c, const double2 *z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const Cpx<double> xa(x[i].x, x[i].y);
    Cpx<double> v = Cpx<double>(a.x, a.y) * xa;
    if (y) v += Cpx<double>(b.x, b.y) * Cpx<double>(y[i].x, y[i].y);
    if (z) v += Cpx<double>(c.x, c.y) * Cpx<double>(z[i].x, z[i].y);
    out[i] = make_double2(v.re, v.im);
  }
}
// block partials of Re<a,b>, Im<a,b>, |a|^2 (<a,b> = sum conj(a) b)
constexpr int DD_RED_BLOCK = 256;
__global__ void __launch_bounds__(DD_RED_BLOCK) k_dd_dots(int64_t n, const double2 *a, const double2 *b, double *part) {
  double v[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 x = a[i], y = b[i];
    v[0] += x.x * y.x + x.y * y.y;
    v[1] += x.x * y.y - x.y * y.x;
    v[2] += x.x * x.x + x.y * x.y;
  }
  __shared__ double sh[3][DD_RED_BLOCK];
  for (int k = 0; k < 3; k++) sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int w = DD_RED_BLOCK / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 3; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) part[blockIdx.x * 3 + k] = sh[k][0];
}
// qcu's random start on the odd sites (include/lattice_bistabcg.h:108-109),
// the value of each element fixed by its GLOBAL site: element (global odd
// half-index G, component c) uses counters 2(12 G + c) and 2(12 G + c) + 1 --
// the same field as the single-GPU solver's start on the global lattice
__global__ void k_dd_uniform_odd(DDDev d, double2 *x, uint64_t seed, int4 origin, int4 glatt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= d.g.Vh) return;
  const Coord c = dd_coord(d.g, s, 1);
  const int64_t X = origin.x + c.x, Y = origin.y + c.y, Z = origin.z + c.z, T = origin.w + c.t;
  const int64_t G = ((T * glatt.z + Z) * glatt.y + Y) * (glatt.x / 2) + (X >> 1);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const uint64_t e = (uint64_t)G * 12 + k;
    x[(size_t)s * 12 + k] = make_double2(rng_uniform(seed, 2 * e), rng_uniform(seed, 2 * e + 1));
  }
}

// ---------------------------------------------------------------- host: one or all ranks of a grid
namespace {
// face buffers of one rank: send[d][0..1], halo[d][0..1]
struct DDBufs {
  DevBuf send[4][2], halo[4][2];
  void ensure(const DDPlan &p) {
    for (int d = 0; d < 4; d++)
      for (int k = 0; k < 2; k++) {
        const size_t bytes = (size_t)std::max(p.face[d], 1) * DD_FACE_COMPLEX * sizeof(double2);
        send[d][k].ensure(bytes);
        halo[d][k].ensure(bytes);
      }
  }
  DDDev dev(const DDPlan &p, const Geom &g) {
    DDDev d;
    d.g = g;
    d.part = 0;
    for (int m = 0; m < 4; m++) {
      if (p.grid[m] > 1) d.part |= 1 << m;
      for (int k = 0; k < 2; k++) {
        d.send[m][k] = send[m][k].as<double2>();
        d.halo[m][k] = halo[m][k].as<double2>();
      }
    }
    return d;
  }
};
// the boundary sites of one output parity (the same on every rank: equal
// local lattices and partitioned directions), built on first use
struct DDBoundary {
  DevBuf list, count;
  int n = -1;
  int key[5] = {0, 0, 0, 0, -1};  // Lxh, Ly, Lz, Lt, partitioned directions
};
struct DDSpace {
  std::vector<std::unique_ptr<DDBufs>> ranks;
  DDBoundary bnd[2];
  DDBufs &at(int r) {
    while ((int)ranks.size() <= r) ranks.push_back(std::make_unique<DDBufs>());
    return *ranks[r];
  }
};

struct NcclApi {
  void *lib = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*allReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*groupStart)() = nullptr;
  ncclResult_t (*groupEnd)() = nullptr;
  const char *(*errorString)(ncclResult_t) = nullptr;
};
NcclApi &nccl() {
  static std::mutex mu;
  static NcclApi api;
  std::lock_guard<std::mutex> lk(mu);
  if (api.lib) return api;
  void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  require(h != nullptr, "dd: NCCL (libnccl.so.2) could not be loaded");
  auto sym = [&](const char *n) {
    void *f = dlsym(h, n);
    require(f != nullptr, std::string("dd: NCCL symbol missing: ") + n);
    return f;
  };
  api.getUniqueId = reinterpret_cast<decltype(api.getUniqueId)>(sym("ncclGetUniqueId"));
  api.commInitRank = reinterpret_cast<decltype(api.commInitRank)>(sym("ncclCommInitRank"));
  api.commDestroy = reinterpret_cast<decltype(api.commDestroy)>(sym("ncclCommDestroy"));
  api.send = reinterpret_cast<decltype(api.send)>(sym("ncclSend"));
  api.recv = reinterpret_cast<decltype(api.recv)>(sym("ncclRecv"));
  api.allReduce = reinterpret_cast<decltype(api.allReduce)>(sym("ncclAllReduce"));
  api.groupStart = reinterpret_cast<decltype(api.groupStart)>(sym("ncclGroupStart"));
  api.groupEnd = reinterpret_cast<decltype(api.groupEnd)>(sym("ncclGroupEnd"));
  api.errorString = reinterpret_cast<decltype(api.errorString)>(sym("ncclGetErrorString"));
  api.lib = h;
  return api;
}
void nccl_check(ncclResult_t r, const char *what) {
  if (r != ncclSuccess) throw Error(2, std::string("dd: ") + what + ": " + nccl().errorString(r));
}
struct DDComm {
  ncclComm_t comm = nullptr;
  int nranks = 0, rank = -1;
};
DDComm &comm_of(const Context &ctx) { return per_device<DDComm>(ctx); }

// the stream the faces travel on, beside the library stream, and the two
// events that order it: faces packed -> exchange; exchange done -> boundary
struct DDStreams {
  cudaStream_t comm = nullptr;
  cudaEvent_t packed = nullptr, landed = nullptr;
  void ensure() {
    if (comm) return;
    QCU_CUDA(cudaStreamCreateWithFlags(&comm, cudaStreamNonBlocking));
    QCU_CUDA(cudaEventCreateWithFlags(&packed, cudaEventDisableTiming));
    QCU_CUDA(cudaEventCreateWithFlags(&landed, cudaEventDisableTiming));
  }
};

// The distributed operators on this process's ranks: every rank of the grid
// (emulated, faces exchanged by device copies) or this process's one rank
// (faces exchanged with NCCL).  The caller holds the context lock.
class DDRun {
 public:
  DDRun(Context &ctx, const int latt[4], const int grid[4], bool emulate)
      : ctx_(ctx), g_(make_geom(latt)), emulate_(emulate) {
    DDSpace &sp = per_device<DDSpace>(ctx);
    if (emulate) {
      const int n = dd_plan(latt, grid, 0).nranks;
      for (int r = 0; r < n; r++) plans_.push_back(dd_plan(latt, grid, r));
    } else {
      DDComm &c = comm_of(ctx);
      require(c.comm != nullptr,
              "ncclDslashQcu/ncclBistabCgQcu with grid != {1,1,1,1}: no communicator on this device (qcuCommInit)");
      plans_.push_back(dd_plan(latt, grid, c.rank));
      require(plans_[0].nranks == c.nranks, "dd: the grid's rank count differs from the communicator's");
      comm_ = c.comm;
    }
    for (size_t r = 0; r < plans_.size(); r++) {
      sp.at((int)r).ensure(plans_[r]);
      dev_.push_back(sp.at((int)r).dev(plans_[r], g_));
      bufs_.push_back(&sp.at((int)r));
    }
  }
  int domains() const { return (int)plans_.size(); }
  const Geom &geom() const { return g_; }
  const DDPlan &plan(int r) const { return plans_[r]; }
  const DDDev &dev(int r) const { return dev_[r]; }

  // out[r] = D_{par <- 1-par} in[r] on every domain (PyQuda-layout halves).
  // The faces are packed on the library stream and exchanged on a stream of
  // their own while the interior sites are computed; the boundary sites
  // follow once the faces have landed.
  void dslash(int par, const std::vector<const void *> &gauge, const std::vector<const void *> &in,
              const std::vector<void *> &out) {
    const cudaStream_t st = ctx_.stream;
    if (dev_[0].part == 0) {  // nothing partitioned: one pass, no exchange
      for (int r = 0; r < domains(); r++) launch_dd_dslash(dev_[r], in[r], gauge[r], out[r], par, 0, st);
      return;
    }
    DDStreams &ss = per_device<DDStreams>(ctx_);
    ss.ensure();
    const DDBoundary &bl = boundary(par);
    for (int r = 0; r < domains(); r++) launch_pack(dev_[r], in[r], gauge[r], 1 - par, st);
    QCU_CUDA(cudaEventRecord(ss.packed, st));
    QCU_CUDA(cudaStreamWaitEvent(ss.comm, ss.packed, 0));
    exchange(ss.comm);
    QCU_CUDA(cudaEventRecord(ss.landed, ss.comm));
    for (int r = 0; r < domains(); r++) launch_dd_dslash(dev_[r], in[r], gauge[r], out[r], par, 1, st);
    QCU_CUDA(cudaStreamWaitEvent(st, ss.landed, 0));
    for (int r = 0; r < domains(); r++)
      launch_dd_dslash(dev_[r], in[r], gauge[r], out[r], par, 2, st, bl.list.as<int>(), bl.n);
  }

  // v[0..n) summed over all ranks of the grid (over the domains of this
  // process when emulating, then across processes with NCCL); v holds this
  // process's per-domain values, domain-major: v[d * n + k]
  void allsum(std::vector<double> &v, int n) {
    std::vector<double> tot(n, 0.0);
    for (int r = 0; r < domains(); r++)
      for (int k = 0; k < n; k++) tot[k] += v[(size_t)r * n + k];
    if (!emulate_) {
      red_.ensure(n * sizeof(double));
      QCU_CUDA(cudaMemcpyAsync(red_.p, tot.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx_.stream));
      nccl_check(nccl().allReduce(red_.p, red_.p, n, ncclDouble, ncclSum, comm_, ctx_.stream), "ncclAllReduce");
      QCU_CUDA(cudaMemcpyAsync(tot.data(), red_.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
      QCU_CUDA(cudaStreamSynchronize(ctx_.stream));
    }
    v = tot;
  }

 private:
  void exchange(cudaStream_t st) {
    if (!emulate_) {
      NcclApi &n = nccl();
      const std::vector<DDOp> ops = dd_schedule(plans_[0]);
      DDBufs &b = *bufs_[0];
      nccl_check(n.groupStart(), "ncclGroupStart");
      for (const DDOp &op : ops) {
        const size_t cnt = (size_t)op.count * 2;  // complex128 as pairs of doubles
        if (op.kind == DD_SEND)
          nccl_check(n.send(b.send[op.dir][op.slot].p, cnt, ncclDouble, op.peer, comm_, st), "ncclSend");
        else
          nccl_check(n.recv(b.halo[op.dir][op.slot].p, cnt, ncclDouble, op.peer, comm_, st), "ncclRecv");
      }
      nccl_check(n.groupEnd(), "ncclGroupEnd");
      return;
    }
    // every rank's schedule carried out as device copies: a send of rank r to
    // peer q is matched with q's next receive from r
    const int n = domains();
    std::vector<std::vector<DDOp>> sched;
    for (int r = 0; r < n; r++) sched.push_back(dd_schedule(plans_[r]));
    std::vector<std::vector<int>> next_recv(n, std::vector<int>(n, 0));
    for (int r = 0; r < n; r++) {
      for (const DDOp &op : sched[r]) {
        if (op.kind != DD_SEND) continue;
        const int q = op.peer;
        int seen = 0, idx = -1;
        for (size_t k = 0; k < sched[q].size(); k++) {
          const DDOp &o = sched[q][k];
          if (o.kind == DD_RECV && o.peer == r) {
            if (seen == next_recv[q][r]) {
              idx = (int)k;
              break;
            }
            seen++;
          }
        }
        require(idx >= 0, "dd: exchange schedule has a send without a matching receive");
        next_recv[q][r]++;
        const DDOp &rv = sched[q][idx];
        require(rv.count == op.count, "dd: send and receive sizes differ");
        QCU_CUDA(cudaMemcpyAsync(bufs_[q]->halo[rv.dir][rv.slot].p, bufs_[r]->send[op.dir][op.slot].p,
                                 (size_t)op.count * sizeof(double2), cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  static void launch_pack(const DDDev &d, const void *in, const void *gauge, int par, cudaStream_t s) {
    k_dd_pack<<<(d.g.Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK, DSLASH_BLOCK, 0, s>>>(
        d, static_cast<const double2 *>(in), gauge, par);
    QCU_CHECK_LAUNCH();
  }
  static void launch_dd_dslash(const DDDev &d, const void *in, const void *gauge, void *out, int par, int mode,
                               cudaStream_t s, const int *list = nullptr, int nlist = 0) {
    const int n = mode == 2 ? nlist : d.g.Vh;
    if (n <= 0) return;
    k_dd_dslash<<<(n + DSLASH_BLOCK - 1) / DSLASH_BLOCK, DSLASH_BLOCK, 0, s>>>(
        d, static_cast<const double2 *>(in), gauge, static_cast<double2 *>(out), par, mode, list, nlist);
    QCU_CHECK_LAUNCH();
  }
  // the boundary sites of output parity par, built once per lattice and partition
  const DDBoundary &boundary(int par) {
    DDBoundary &b = per_device<DDSpace>(ctx_).bnd[par];
    const int key[5] = {g_.Lxh, g_.Ly, g_.Lz, g_.Lt, dev_[0].part};
    if (b.n >= 0 && std::equal(key, key + 5, b.key)) return b;
    b.list.ensure((size_t)g_.Vh * sizeof(int));
    b.count.ensure(sizeof(int));
    QCU_CUDA(cudaMemsetAsync(b.count.p, 0, sizeof(int), ctx_.stream));
    k_dd_boundary_list<<<(g_.Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK, DSLASH_BLOCK, 0, ctx_.stream>>>(
        dev_[0], par, b.list.as<int>(), b.count.as<int>());
    QCU_CHECK_LAUNCH();
    int n = 0;
    QCU_CUDA(cudaMemcpyAsync(&n, b.count.p, sizeof(int), cudaMemcpyDeviceToHost, ctx_.stream));
    QCU_CUDA(cudaStreamSynchronize(ctx_.stream));
    b.n = n;
    std::copy(key, key + 5, b.key);
    return b;
  }

  Context &ctx_;
  Geom g_;
  bool emulate_;
  ncclComm_t comm_ = nullptr;
  std::vector<DDPlan> plans_;
  std::vector<DDDev> dev_;
  std::vector<DDBufs *> bufs_;
  DevBuf red_;
};

std::vector<const void *> split_c(const void *all, size_t bytes, int n) {
  std::vector<const void *> v;
  for (int r = 0; r < n; r++) v.push_back(static_cast<const char *>(all) + bytes * r);
  return v;
}
std::vector<void *> split(void *all, size_t bytes, int n) {
  std::vector<void *> v;
  for (int r = 0; r < n; r++) v.push_back(static_cast<char *>(all) + bytes * r);
  return v;
}

// qcu's solver on the grid (include/lattice_bistabcg.h:101-132,221-340):
// b'_o = b_o + kappa D_oe b_e; BiCGSTAB on M_pc = 1 - kappa^2 D_oe D_eo from
// qcu's random start until the iterated, grid-wide ||r||^2 < tol (absolute)
// or maxiter iterations; x_e = b_e + kappa D_eo x_o.  Scalars and inner
// products are formed on the host from every rank's sums.
DDSolveResult dd_bicgstab(DDRun &run, const std::vector<const void *> &gauge, const std::vector<void *> &x,
                          const std::vector<const void *> &b, double kappa, double tol, int maxiter, uint64_t seed,
                          const int glatt[4]) {
  const Geom &g = run.geom();
  const int R = run.domains();
  const int64_t n = (int64_t)g.Vh * 12;
  const size_t half = (size_t)n * sizeof(double2);
  Context &ctx = context();
  const cudaStream_t st = ctx.stream;
  // per domain: b', r, rt, p, v, s, t, tmp, x_o
  enum { BP, RR, RT, PP, VV, SS, TT, TMP, XO, NV };
  std::vector<std::vector<std::unique_ptr<DevBuf>>> w(R);
  for (int r = 0; r < R; r++)
    for (int k = 0; k < NV; k++) {
      w[r].push_back(std::make_unique<DevBuf>());
      w[r][k]->ensure(half);
    }
  auto V = [&](int k) {
    std::vector<void *> v;
    for (int r = 0; r < R; r++) v.push_back(w[r][k]->p);
    return v;
  };
  auto VC = [&](int k) {
    std::vector<const void *> v;
    for (int r = 0; r < R; r++) v.push_back(w[r][k]->p);
    return v;
  };
  const int grid_blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  auto lin3 = [&](int r, void *out, Cpx<double> a, const void *xx, Cpx<double> bb = {0, 0}, const void *y = nullptr,
                  Cpx<double> c = {0, 0}, const void *z = nullptr) {
    k_dd_lin3<<<grid_blocks, 256, 0, st>>>(n, static_cast<double2 *>(out), make_double2(a.re, a.im),
                                           static_cast<const double2 *>(xx), make_double2(bb.re, bb.im),
                                           static_cast<const double2 *>(y), make_double2(c.re, c.im),
                                           static_cast<const double2 *>(z));
    QCU_CHECK_LAUNCH();
  };
  DevBuf part;
  part.ensure((size_t)grid_blocks * 3 * sizeof(double));
  std::vector<double> ph((size_t)grid_blocks * 3);
  // grid-wide Re<a,b>, Im<a,b>, |a|^2
  auto dots = [&](int ka, int kb) {
    std::vector<double> v((size_t)R * 3, 0.0);
    for (int r = 0; r < R; r++) {
      k_dd_dots<<<grid_blocks, DD_RED_BLOCK, 0, st>>>(n, static_cast<const double2 *>(w[r][ka]->p),
                                                     static_cast<const double2 *>(w[r][kb]->p), part.as<double>());
      QCU_CHECK_LAUNCH();
      QCU_CUDA(cudaMemcpyAsync(ph.data(), part.p, ph.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      QCU_CUDA(cudaStreamSynchronize(st));
      for (int i = 0; i < grid_blocks; i++)
        for (int k = 0; k < 3; k++) v[(size_t)r * 3 + k] += ph[(size_t)i * 3 + k];
    }
    run.allsum(v, 3);
    return v;
  };
  const double k2 = kappa * kappa;
  // out = M_pc in = in - kappa^2 D_oe D_eo in
  auto mpc = [&](int kin, int kout) {
    run.dslash(0, gauge, VC(kin), V(TMP));
    run.dslash(1, gauge, VC(TMP), V(kout));
    for (int r = 0; r < R; r++) lin3(r, w[r][kout]->p, {-k2, 0}, w[r][kout]->p, {1, 0}, w[r][kin]->p);
  };
  std::vector<const void *> be, bo;
  std::vector<void *> xe, xo_out;
  for (int r = 0; r < R; r++) {
    be.push_back(b[r]);
    bo.push_back(static_cast<const char *>(b[r]) + half);
    xe.push_back(x[r]);
    xo_out.push_back(static_cast<char *>(x[r]) + half);
  }
  // b'_o = b_o + kappa D_oe b_e
  run.dslash(1, gauge, be, V(TMP));
  for (int r = 0; r < R; r++) lin3(r, w[r][BP]->p, {1, 0}, bo[r], {kappa, 0}, w[r][TMP]->p);
  // random start
  for (int r = 0; r < R; r++) {
    const DDPlan &p = run.plan(r);
    const int4 origin = make_int4(p.coord[0] * p.latt[0], p.coord[1] * p.latt[1], p.coord[2] * p.latt[2],
                                  p.coord[3] * p.latt[3]);
    k_dd_uniform_odd<<<(g.Vh + 127) / 128, 128, 0, st>>>(run.dev(r), static_cast<double2 *>(w[r][XO]->p), seed,
                                                          origin, make_int4(glatt[0], glatt[1], glatt[2], glatt[3]));
    QCU_CHECK_LAUNCH();
  }
  mpc(XO, VV);
  for (int r = 0; r < R; r++) {
    lin3(r, w[r][RR]->p, {1, 0}, w[r][BP]->p, {-1, 0}, w[r][VV]->p);
    QCU_CUDA(cudaMemcpyAsync(w[r][RT]->p, w[r][RR]->p, half, cudaMemcpyDeviceToDevice, st));
    QCU_CUDA(cudaMemsetAsync(w[r][PP]->p, 0, half, st));
    QCU_CUDA(cudaMemsetAsync(w[r][VV]->p, 0, half, st));
  }
  Cpx<double> rho(1, 0), alpha(1, 0), omega(1, 0);
  DDSolveResult res;
  res.r2 = dots(RR, RR)[2];
  for (int it = 0; it < maxiter && !(res.r2 < tol); it++) {
    std::vector<double> d = dots(RT, RR);
    const Cpx<double> rho_n(d[0], d[1]);
    const Cpx<double> beta = cdiv(rho_n, rho) * cdiv(alpha, omega);
    rho = rho_n;
    for (int r = 0; r < R; r++)  // p = r + beta (p - omega v)
      lin3(r, w[r][PP]->p, {1, 0}, w[r][RR]->p, beta, w[r][PP]->p, Cpx<double>(0, 0) - beta * omega, w[r][VV]->p);
    mpc(PP, VV);
    d = dots(RT, VV);
    alpha = cdiv(rho, Cpx<double>(d[0], d[1]));
    for (int r = 0; r < R; r++) lin3(r, w[r][SS]->p, {1, 0}, w[r][RR]->p, Cpx<double>(0, 0) - alpha, w[r][VV]->p);
    mpc(SS, TT);
    d = dots(TT, SS);
    omega = Cpx<double>(d[0] / d[2], d[1] / d[2]);
    for (int r = 0; r < R; r++) {
      lin3(r, w[r][XO]->p, {1, 0}, w[r][XO]->p, alpha, w[r][PP]->p, omega, w[r][SS]->p);
      lin3(r, w[r][RR]->p, {1, 0}, w[r][SS]->p, Cpx<double>(0, 0) - omega, w[r][TT]->p);
    }
    res.r2 = dots(RR, RR)[2];
    res.iterations = it + 1;
    require(res.r2 == res.r2, "dd: the solve produced a non-finite residual");
  }
  // x_o, and x_e = b_e + kappa D_eo x_o
  run.dslash(0, gauge, VC(XO), V(TMP));
  for (int r = 0; r < R; r++) {
    QCU_CUDA(cudaMemcpyAsync(xo_out[r], w[r][XO]->p, half, cudaMemcpyDeviceToDevice, st));
    lin3(r, xe[r], {1, 0}, be[r], {kappa, 0}, w[r][TMP]->p);
  }
  QCU_CUDA(cudaStreamSynchronize(st));
  return res;
}
}  // namespace

void dd_dslash_emulate(void *out_all, const void *in_all, const void *gauge_all, const int latt[4], int parity,
                       const int grid[4]) {
  require(out_all && in_all && gauge_all, "dd: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDRun run(ctx, latt, grid, true);
  const Geom &g = run.geom();
  const int n = run.domains();
  const size_t half = (size_t)g.Vh * 12 * sizeof(double2), gauge_sz = (size_t)g.Vh * 8 * 9 * sizeof(double2);
  QCU_CUDA(cudaDeviceSynchronize());
  run.dslash(parity, split_c(gauge_all, gauge_sz, n), split_c(in_all, half, n), split(out_all, half, n));
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

void dd_dslash_nccl(void *out, const void *in, const void *gauge, const int latt[4], int parity, const int grid[4]) {
  require(out && in && gauge, "dslash: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDRun run(ctx, latt, grid, false);
  QCU_CUDA(cudaDeviceSynchronize());
  run.dslash(parity, {gauge}, {in}, {out});
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

DDSolveResult dd_solve(void *x, const void *b, const void *gauge, const int latt[4], const int grid[4], bool emulate,
                       double kappa, double tol, int maxiter, uint64_t seed) {
  require(x && b && gauge, "solve: null pointer argument");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDRun run(ctx, latt, grid, emulate);
  const Geom &g = run.geom();
  const int n = run.domains();
  const size_t full = (size_t)g.Vh * 24 * sizeof(double2), gauge_sz = (size_t)g.Vh * 8 * 9 * sizeof(double2);
  int glatt[4];
  for (int d = 0; d < 4; d++) glatt[d] = latt[d] * grid[d];
  QCU_CUDA(cudaDeviceSynchronize());
  return dd_bicgstab(run, split_c(gauge, gauge_sz, n), split(x, full, n), split_c(b, full, n), kappa, tol, maxiter,
                     seed, glatt);
}

void dd_unique_id(void *id) {
  require(id != nullptr, "dd: null id buffer");
  ncclUniqueId u;
  nccl_check(nccl().getUniqueId(&u), "ncclGetUniqueId");
  memcpy(id, &u, sizeof(u));
}

void dd_comm_init(const void *id, int nranks, int rank) {
  require(id != nullptr && nranks >= 1 && rank >= 0 && rank < nranks, "dd: bad communicator arguments");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDComm &c = comm_of(ctx);
  require(c.comm == nullptr, "dd: this device already has a communicator (qcuCommFree first)");
  ncclUniqueId u;
  memcpy(&u, id, sizeof(u));
  nccl_check(nccl().commInitRank(&c.comm, nranks, u, rank), "ncclCommInitRank");
  c.nranks = nranks;
  c.rank = rank;
}

void dd_comm_free() {
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDComm &c = comm_of(ctx);
  if (c.comm) nccl().commDestroy(c.comm);
  c = DDComm();
}

}  // namespace qcu
