// Multi-right-hand-side hopping term on the tcgen05 tensor cores (mrhs_tc.cu).
#pragma once
#include "internal.h"

namespace qcu {

struct GaugeHandle;

// rows of a multi-rhs field (right-hand sides padded to 64 or 128) and its bytes (one parity)
int mrhs_rows(int nrhs);
size_t mrhs_bytes(int Vh, int nrhs);

// out = D_{par <- 1-par} in for every right-hand side: multi-rhs FP16 fields,
// GSOA16 links; *err set if a wait in the kernel timed out
void launch_mrhs_tc(const Geom &g, const void *gauge16, double t_bc, const void *in, void *out, int nrhs, int par,
                    int *err, int sms, cudaStream_t s);
// PyQuda half spinors [nrhs][Vh][12] complex128 <-> multi-rhs FP16 field
void launch_mrhs_pack(const void *pyq, void *mrhs, int Vh, int nrhs, cudaStream_t s);
void launch_mrhs_unpack(const void *mrhs, void *pyq, int Vh, int nrhs, cudaStream_t s);
void launch_mrhs_random(void *mrhs, int Vh, int nrhs, unsigned long long seed, cudaStream_t s);

// on a gauge handle: the operator on PyQuda-layout fields, and the kernel's
// time per application (ms, CUDA events) on resident seeded fields
void handle_dslash_mrhs(GaugeHandle &G, void *out, const void *in, int nrhs, int par);
double handle_dslash_mrhs_time(GaugeHandle &G, int nrhs, int par, int iters);

}  // namespace qcu
