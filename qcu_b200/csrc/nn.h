// Gauge-equivariant parallel-transport network used as a learned
// preconditioner (an approximation of M_pc^{-1} on the odd sites).
//
// A field with C channels holds C colour vectors per site: float2
// [B][2 parities][Vh][C][3] ("NN layout"; for C = 4 one parity is exactly a
// PyQuda half spinor in complex64).  One parallel-transport layer maps
//     out_a(x) = sum_{h=0..8} sum_b W[h][a][b] (T_h in_b)(x)
// with T_0 = identity, T_{1+2mu} in(x) = U_mu(x) in(x+mu) and
// T_{2+2mu} in(x) = U_mu(x-mu)^dag in(x-mu) (t-boundary phase included).
// W acts on channels only, T on colour only, so the layer commutes with
// gauge transformations.  The adjoint of T_h is T_hbar (forward <-> backward
// of the same direction), so the input gradient of a layer is the same
// kernel run with hops swapped and weights conjugate-transposed.
#pragma once
#include "internal.h"

namespace qcu {

constexpr int NN_HOPS = 9;
constexpr int NN_C_IN = 4, NN_C_HID = 16, NN_C_OUT = 4;

struct PtcArgs {
  const float2 *in = nullptr;   // [B][2][Vh][cin][3]
  float2 *out = nullptr;        // [B][2][Vh][cout][3]
  const float2 *w = nullptr;    // [9][cout][cin] complex FP32 (or null: use w16)
  const uint32_t *w16 = nullptr;  // same, as packed bf16 pairs (re, im)
  const void *gauge = nullptr;  // GSOA32 packed links
  int B = 1;
  int out_mask = 3;  // bit p: compute output parity p (others are left untouched)
  int in_mask = 3;   // bit q: input is non-zero on parity q (others skipped)
  int adjoint = 0;   // 1: hops replaced by their adjoints, weights by W^dag (input gradient)
  float t_bc = 1.f;
  int accumulate = 0;  // 1: out += layer(in)
};

// forward (or adjoint) layer; cin/cout in {4, 16}
void launch_ptc(int cin, int cout, const Geom &g, const PtcArgs &a, cudaStream_t s);
// the network's forward pass with bf16 weights on the tensor cores
// (nn_tc.cu): z64 = N(r64) on odd-parity FP64 site-blocked spinors (SOA64;
// z64 may be r64), through a hidden field stored as bf16 pairs
// (nn_hid16_bytes); the transported inputs are rounded to bf16, accumulation
// is FP32; err is set to 1 if a wait of the kernel timed out
void launch_nn_tc(const Geom &g, const void *gauge16, float t_bc, const uint32_t *w16_1, const uint32_t *w16_2,
                  const void *r64, void *hid16, void *z64, int *err, int sms, cudaStream_t s);
size_t nn_hid16_bytes(int Vh);

// grad[h][a][b] += sum_x sum_colour delta_a(x) conj((T_h in_b)(x)), over the
// output parities in a.out_mask (a.out holds delta).  grad: [9][cout][cin] complex FP32.
void launch_ptc_wgrad(int cin, int cout, const Geom &g, const PtcArgs &a, float2 *grad, cudaStream_t s);

// loss: delta_i = (o_i - e_i) / |e_i|^2 on parity 1, sums_i |o_i - e_i|^2 / |e_i|^2 -> loss[i]
void launch_nn_loss(const Geom &g, int B, const float2 *o, const float2 *e, const float *enorm2, float2 *delta,
                    float *loss, cudaStream_t s);

// Adam step on n real parameters; also refreshes the bf16 copy (pairs)
void launch_adam(int n, float *p, const float *grad, float *m, float *v, uint32_t *p16, float lr, float b1, float b2,
                 float eps, int step, cudaStream_t s);

// FP32 weights -> packed bf16 pairs
void launch_to_bf16(int n, const float *p, uint32_t *p16, cudaStream_t s);

// solver-side conversions: odd-parity FP64 blocked spinor (SOA64) <-> NN layout (B = 1, C = 4)
void launch_soa64_to_nn(int Vh, const void *in, float2 *nn_odd, cudaStream_t s);
void launch_nn_to_soa64(int Vh, const float2 *nn_odd, void *out, cudaStream_t s);

struct NNet;
struct GaugeHandle;
NNet *nn_create(uint64_t seed, double scale);
void nn_free(NNet *n);
int nn_nparam();
void nn_get(NNet &n, float *host);
void nn_set(NNet &n, const float *host);
void nn_apply_pyq(NNet &n, const GaugeHandle &G, void *out, const void *in);
double nn_train_step(NNet &n, const GaugeHandle &G, const void *r, const void *e, int B, double lr, float *grad_host);
void nn_apply_soa64(NNet &n, const GaugeHandle &G, const void *r64, void *z64, cudaStream_t s);
void nn_prepare(NNet &n, int Vh);
// throws if a tensor-core layer of the network reported a timed-out wait
void nn_check(NNet &n);
// 1: inference runs the tensor-core layers (default); 0: the FMA layers
void nn_set_tensor_cores(NNet &n, int on);

}  // namespace qcu
