// Host side of the learned preconditioner: the network object, its
// application (FP32 arithmetic, bf16 weights), gradients and Adam training
// steps.  The network approximates M_pc^{-1} on the odd sites:
//   hidden = L1(r)  (4 -> 16 channels, both parities; r lives on odd sites)
//   N(r)   = L2(hidden) (16 -> 4 channels, odd sites)
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "nn.h"
#include "solver.h"

namespace qcu {

constexpr int NN_W1 = NN_HOPS * NN_C_HID * NN_C_IN;   // complex weights of layer 1 ([9][16][4])
constexpr int NN_W2 = NN_HOPS * NN_C_OUT * NN_C_HID;  // layer 2 ([9][4][16])
constexpr int NN_NPARAM = 2 * (NN_W1 + NN_W2);        // reals

struct NNet {
  DevBuf w, w16, m, v, grad;       // FP32 master, bf16 copy, Adam moments, gradient
  DevBuf in, hid, out, delta2, delta1, target, enorm, loss;  // work fields (grown to batch x lattice)
  DevBuf err;   // set by the tensor-core layers if a wait timed out
  DevBuf hid16; // hidden field of the tensor-core layers (bf16 pairs)
  int tensor_cores = 1;
  int step = 0;
  int batch_cap = 0, vh_cap = 0;
  float2 *w1() const { return w.as<float2>(); }
  float2 *w2() const { return w.as<float2>() + NN_W1; }
  uint32_t *w16_1() const { return w16.as<uint32_t>(); }
  uint32_t *w16_2() const { return w16.as<uint32_t>() + NN_W1; }
  void ensure(int B, int Vh) {
    if (B <= batch_cap && Vh <= vh_cap) return;
    batch_cap = std::max(B, batch_cap);
    vh_cap = std::max(Vh, vh_cap);
    const size_t f4 = (size_t)batch_cap * 2 * vh_cap * NN_C_IN * 3 * sizeof(float2);
    const size_t f16 = (size_t)batch_cap * 2 * vh_cap * NN_C_HID * 3 * sizeof(float2);
    in.ensure(f4);
    out.ensure(f4);
    target.ensure(f4);
    delta2.ensure(f4);
    hid.ensure(f16);
    delta1.ensure(f16);
    enorm.ensure(batch_cap * sizeof(float));
    loss.ensure(batch_cap * sizeof(float));
  }
};

// staging spinor for the complex128 <-> complex64 conversions (one per device, never freed)
static Spinor &stage() { return per_device<Spinor>(context()); }

static void refresh_bf16(NNet &n, cudaStream_t s) { launch_to_bf16(NN_NPARAM, n.w.as<float>(), n.w16.as<uint32_t>(), s); }

NNet *nn_create(uint64_t seed, double scale) {
  auto *n = new NNet();
  n->w.ensure(NN_NPARAM * sizeof(float));
  n->w16.ensure(NN_NPARAM / 2 * sizeof(uint32_t));
  n->err.ensure(sizeof(int));
  QCU_CUDA(cudaMemset(n->err.p, 0, sizeof(int)));
  n->m.ensure(NN_NPARAM * sizeof(float));
  n->v.ensure(NN_NPARAM * sizeof(float));
  n->grad.ensure(NN_NPARAM * sizeof(float));
  // identity start: hidden channels 0-3 copy the input (W1[0]), the output
  // copies them back (W2[0]); every other weight small and random
  std::vector<float> h(NN_NPARAM);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, (float)scale);
  for (auto &x : h) x = nd(rng);
  for (int a = 0; a < NN_C_IN; a++) {
    h[2 * ((0 * NN_C_HID + a) * NN_C_IN + a)] = 1.f;
    h[2 * ((0 * NN_C_HID + a) * NN_C_IN + a) + 1] = 0.f;
    h[2 * (NN_W1 + (0 * NN_C_OUT + a) * NN_C_HID + a)] = 1.f;
    h[2 * (NN_W1 + (0 * NN_C_OUT + a) * NN_C_HID + a) + 1] = 0.f;
  }
  Context &ctx = context();
  QCU_CUDA(cudaMemcpy(n->w.p, h.data(), NN_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  QCU_CUDA(cudaMemset(n->m.p, 0, NN_NPARAM * sizeof(float)));
  QCU_CUDA(cudaMemset(n->v.p, 0, NN_NPARAM * sizeof(float)));
  QCU_CUDA(cudaMemset(n->grad.p, 0, NN_NPARAM * sizeof(float)));
  refresh_bf16(*n, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  return n;
}

void nn_free(NNet *n) { delete n; }
int nn_nparam() { return NN_NPARAM; }

void nn_get(NNet &n, float *host) { QCU_CUDA(cudaMemcpy(host, n.w.p, NN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost)); }
void nn_set(NNet &n, const float *host) {
  Context &ctx = context();
  QCU_CUDA(cudaMemcpy(n.w.p, host, NN_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  refresh_bf16(n, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

// N(in) for B samples whose odd halves are in n.in; result in n.out (odd halves).
// bf16 = true: inference weights; false: FP32 master weights (training)
static void forward(NNet &n, const GaugeHandle &G, int B, bool bf16, cudaStream_t s) {
  PtcArgs a;
  a.gauge = G.g32.p;
  a.t_bc = (float)G.t_bc;
  a.B = B;
  a.in = n.in.as<float2>();
  a.out = n.hid.as<float2>();
  a.in_mask = 2;
  a.out_mask = 3;
  if (bf16) a.w16 = n.w16_1();
  else a.w = n.w1();
  launch_ptc(NN_C_IN, NN_C_HID, G.g, a, s);
  PtcArgs b2 = a;
  b2.in = n.hid.as<float2>();
  b2.out = n.out.as<float2>();
  b2.in_mask = 3;
  b2.out_mask = 2;
  b2.w = nullptr;
  b2.w16 = nullptr;
  if (bf16) b2.w16 = n.w16_2();
  else b2.w = n.w2();
  launch_ptc(NN_C_HID, NN_C_OUT, G.g, b2, s);
}

// z = N(r) on odd-parity SOA64 spinors (z may be r): the tensor-core layers,
// or the FMA layers through the NN layout
static void apply_soa64(NNet &n, const GaugeHandle &G, const void *r64, void *z64, cudaStream_t s) {
  const int Vh = G.g.Vh;
  if (n.tensor_cores) {
    n.hid16.ensure(nn_hid16_bytes(Vh));
    launch_nn_tc(G.g, G.g16.p, (float)G.t_bc, n.w16_1(), n.w16_2(), r64, n.hid16.p, z64, n.err.as<int>(),
                 context().sms, s);
    return;
  }
  launch_soa64_to_nn(Vh, r64, n.in.as<float2>(), s);
  forward(n, G, 1, true, s);
  launch_nn_to_soa64(Vh, n.out.as<float2>(), z64, s);
}

void nn_check(NNet &n) {
  int e = 0;
  QCU_CUDA(cudaMemcpy(&e, n.err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    QCU_CUDA(cudaMemset(n.err.p, 0, sizeof(int)));
    throw Error(2, "network: a tensor-core layer timed out waiting for its MMAs");
  }
}

void nn_set_tensor_cores(NNet &n, int on) { n.tensor_cores = on ? 1 : 0; }

void nn_apply_pyq(NNet &n, const GaugeHandle &G, void *out, const void *in) {
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  const int Vh = G.g.Vh;
  if (!n.tensor_cores) n.ensure(1, Vh);  // the FMA layers' work fields
  QCU_CUDA(cudaDeviceSynchronize());
  // complex128 -> FP64 blocked layout, the network, and back
  Spinor &t = stage();
  t.alloc(SOA64, Vh);
  launch_convert(AOS64, SOA64, Vh, in, nullptr, t.data.p, nullptr, ctx.stream);
  apply_soa64(n, G, t.data.p, t.data.p, ctx.stream);
  launch_convert(SOA64, AOS64, Vh, t.data.p, nullptr, out, nullptr, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  nn_check(n);
}

// gradient of L = mean_i |N(r_i) - e_i|^2 / |e_i|^2 over a batch of odd half
// spinors (complex128 PyQuda layout [B][Vh][4][3]); optionally an Adam step
double nn_train_step(NNet &n, const GaugeHandle &G, const void *r, const void *e, int B, double lr, float *grad_host) {
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  const int Vh = G.g.Vh;
  cudaStream_t s = ctx.stream;
  n.ensure(B, Vh);
  QCU_CUDA(cudaDeviceSynchronize());
  // inputs: odd slabs of samples b (parity 0 slabs are never read: in_mask = 2)
  Spinor &t = stage();
  t.alloc(SOA64, Vh);
  const size_t half = spinor_bytes(AOS64, Vh);
  std::vector<float> enorm(B);
  for (int b = 0; b < B; b++) {
    const char *rb = static_cast<const char *>(r) + b * half;
    const char *eb = static_cast<const char *>(e) + b * half;
    launch_convert(AOS64, SOA64, Vh, rb, nullptr, t.data.p, nullptr, s);
    launch_soa64_to_nn(Vh, t.data.p, n.in.as<float2>() + (size_t)b * 2 * Vh * 12, s);
    launch_convert(AOS64, SOA64, Vh, eb, nullptr, t.data.p, nullptr, s);
    launch_soa64_to_nn(Vh, t.data.p, n.target.as<float2>() + (size_t)b * 2 * Vh * 12, s);
    launch_dots(SOA64, Vh, t.data.p, nullptr, t.data.p, nullptr, ctx, s);
    QCU_CUDA(cudaMemcpyAsync(ctx.st_host, ctx.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
    QCU_CUDA(cudaStreamSynchronize(s));
    enorm[b] = (float)ctx.st_host->sums[2];
    require(enorm[b] > 0.f, "training target with zero norm");
  }
  QCU_CUDA(cudaMemcpyAsync(n.enorm.p, enorm.data(), B * sizeof(float), cudaMemcpyHostToDevice, s));
  QCU_CUDA(cudaMemsetAsync(n.loss.p, 0, B * sizeof(float), s));
  QCU_CUDA(cudaMemsetAsync(n.grad.p, 0, NN_NPARAM * sizeof(float), s));
  forward(n, G, B, false, s);
  launch_nn_loss(G.g, B, n.out.as<float2>(), n.target.as<float2>(), n.enorm.as<float>(), n.delta2.as<float2>(),
                 n.loss.as<float>(), s);
  // dL/dW2: delta2 (odd) against the hidden field
  PtcArgs a;
  a.gauge = G.g32.p;
  a.t_bc = (float)G.t_bc;
  a.B = B;
  a.in = n.hid.as<float2>();
  a.out = n.delta2.as<float2>();
  a.in_mask = 3;
  a.out_mask = 2;
  launch_ptc_wgrad(NN_C_HID, NN_C_OUT, G.g, a, n.grad.as<float2>() + NN_W1, s);
  // delta1 = L2^dag delta2 on both parities
  PtcArgs d = a;
  d.in = n.delta2.as<float2>();
  d.out = n.delta1.as<float2>();
  d.in_mask = 2;
  d.out_mask = 3;
  d.adjoint = 1;
  d.w = n.w2();
  launch_ptc(NN_C_OUT, NN_C_HID, G.g, d, s);
  // dL/dW1: delta1 against the input
  PtcArgs g1 = a;
  g1.in = n.in.as<float2>();
  g1.out = n.delta1.as<float2>();
  g1.in_mask = 2;
  g1.out_mask = 3;
  launch_ptc_wgrad(NN_C_IN, NN_C_HID, G.g, g1, n.grad.as<float2>(), s);
  std::vector<float> loss(B);
  QCU_CUDA(cudaMemcpyAsync(loss.data(), n.loss.p, B * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (grad_host) QCU_CUDA(cudaMemcpyAsync(grad_host, n.grad.p, NN_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (lr > 0) {
    n.step++;
    launch_adam(NN_NPARAM, n.w.as<float>(), n.grad.as<float>(), n.m.as<float>(), n.v.as<float>(),
                n.w16.as<uint32_t>(), (float)lr, 0.9f, 0.999f, 1e-8f, n.step, s);
  }
  QCU_CUDA(cudaStreamSynchronize(s));
  double tot = 0;
  for (float l : loss) tot += l;
  return tot / B;
}

// GCR preconditioner application on FP64 blocked odd spinors: z = N(r)
void nn_apply_soa64(NNet &n, const GaugeHandle &G, const void *r64, void *z64, cudaStream_t s) {
  apply_soa64(n, G, r64, z64, s);
}

void nn_prepare(NNet &n, int Vh) {
  if (n.tensor_cores) n.hid16.ensure(nn_hid16_bytes(Vh));
  else n.ensure(1, Vh);
}

}  // namespace qcu
