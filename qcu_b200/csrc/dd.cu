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
//   2. the faces are exchanged: NCCL point-to-point on the library stream
//      (grouped send/recv to the two neighbours of every partitioned
//      direction), or device-to-device copies when all ranks of a grid are
//      emulated in one process on one GPU (qcuDslashDDEmulate, the test of
//      the kernels and the exchange schedule without a second GPU);
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

__global__ void __launch_bounds__(DSLASH_BLOCK, 3)
    k_dd_dslash(DDDev d, const double2 *__restrict__ in, const void *gauge, double2 *out, int par) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= d.g.Vh) return;
  const Geom &g = d.g;
  const SpinorView<AOS64> inv{const_cast<double2 *>(in), nullptr, g.Vh};
  const GaugeView<GAOS64> U{gauge, g.Vh};
  const Coord c = dd_coord(g, s, par);
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

// ---------------------------------------------------------------- host: buffers and launches
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
struct DDSpace {
  std::vector<std::unique_ptr<DDBufs>> ranks;
  DDBufs &at(int r) {
    while ((int)ranks.size() <= r) ranks.push_back(std::make_unique<DDBufs>());
    return *ranks[r];
  }
};

void launch_pack(const DDDev &d, const void *in, const void *gauge, int par, cudaStream_t s) {
  k_dd_pack<<<(d.g.Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK, DSLASH_BLOCK, 0, s>>>(d, static_cast<const double2 *>(in),
                                                                               gauge, par);
  QCU_CHECK_LAUNCH();
}
void launch_dd_dslash(const DDDev &d, const void *in, const void *gauge, void *out, int par, cudaStream_t s) {
  k_dd_dslash<<<(d.g.Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK, DSLASH_BLOCK, 0, s>>>(
      d, static_cast<const double2 *>(in), gauge, static_cast<double2 *>(out), par);
  QCU_CHECK_LAUNCH();
}
}  // namespace

void dd_dslash_emulate(void *out_all, const void *in_all, const void *gauge_all, const int latt[4], int parity,
                       const int grid[4]) {
  require(out_all && in_all && gauge_all, "dd: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  const DDPlan p0 = dd_plan(latt, grid, 0);
  const Geom g = make_geom(latt);
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDSpace &sp = per_device<DDSpace>(ctx);
  const cudaStream_t st = ctx.stream;
  const size_t half = (size_t)g.Vh * 12 * sizeof(double2), gauge_sz = (size_t)g.Vh * 8 * 9 * sizeof(double2);
  auto in_of = [&](int r) { return static_cast<const char *>(in_all) + half * r; };
  auto out_of = [&](int r) { return static_cast<char *>(out_all) + half * r; };
  auto gauge_of = [&](int r) { return static_cast<const char *>(gauge_all) + gauge_sz * r; };
  QCU_CUDA(cudaDeviceSynchronize());
  std::vector<DDPlan> plans;
  for (int r = 0; r < p0.nranks; r++) {
    plans.push_back(dd_plan(latt, grid, r));
    sp.at(r).ensure(plans[r]);
  }
  for (int r = 0; r < p0.nranks; r++)
    launch_pack(sp.at(r).dev(plans[r], g), in_of(r), gauge_of(r), 1 - parity, st);
  // the exchange schedule of every rank, carried out as device copies: a send
  // of rank r to peer q is matched with q's next receive from r
  std::vector<std::vector<DDOp>> sched;
  for (int r = 0; r < p0.nranks; r++) sched.push_back(dd_schedule(plans[r]));
  std::vector<std::vector<int>> next_recv(p0.nranks, std::vector<int>(p0.nranks, 0));
  for (int r = 0; r < p0.nranks; r++) {
    for (const DDOp &op : sched[r]) {
      if (op.kind != DD_SEND) continue;
      const int q = op.peer;
      // q's receives from r, in q's order
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
      QCU_CUDA(cudaMemcpyAsync(sp.at(q).halo[rv.dir][rv.slot].p, sp.at(r).send[op.dir][op.slot].p,
                               (size_t)op.count * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    }
  }
  for (int r = 0; r < p0.nranks; r++)
    launch_dd_dslash(sp.at(r).dev(plans[r], g), in_of(r), gauge_of(r), out_of(r), parity, st);
  QCU_CUDA(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------- NCCL
namespace {
struct NcclApi {
  void *lib = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
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
}  // namespace

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

void dd_dslash_nccl(void *out, const void *in, const void *gauge, const int latt[4], int parity, const int grid[4]) {
  require(out && in && gauge, "dslash: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  DDComm &c = comm_of(ctx);
  require(c.comm != nullptr, "ncclDslashQcu with grid != {1,1,1,1}: no communicator on this device (qcuCommInit)");
  const DDPlan p = dd_plan(latt, grid, c.rank);
  require(p.nranks == c.nranks, "ncclDslashQcu: the grid's rank count differs from the communicator's");
  const Geom g = make_geom(latt);
  DDBufs &b = per_device<DDSpace>(ctx).at(0);
  b.ensure(p);
  const DDDev dv = b.dev(p, g);
  const cudaStream_t st = ctx.stream;
  QCU_CUDA(cudaDeviceSynchronize());
  launch_pack(dv, in, gauge, 1 - parity, st);
  const std::vector<DDOp> ops = dd_schedule(p);
  NcclApi &n = nccl();
  nccl_check(n.groupStart(), "ncclGroupStart");
  for (const DDOp &op : ops) {
    const size_t cnt = (size_t)op.count * 2;  // complex128 as pairs of doubles
    if (op.kind == DD_SEND) nccl_check(n.send(b.send[op.dir][op.slot].p, cnt, ncclDouble, op.peer, c.comm, st), "ncclSend");
    else nccl_check(n.recv(b.halo[op.dir][op.slot].p, cnt, ncclDouble, op.peer, c.comm, st), "ncclRecv");
  }
  nccl_check(n.groupEnd(), "ncclGroupEnd");
  launch_dd_dslash(dv, in, gauge, out, parity, st);
  QCU_CUDA(cudaStreamSynchronize(st));
}

}  // namespace qcu
