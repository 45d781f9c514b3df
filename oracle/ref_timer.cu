// Times qcu's own hopping kernel -- wilson_dslash, src/wilson_dslash.cu:9-245
// of the reference, compiled from its sources into oracle/_ref/libqcu_ref.so
// by ref.mk, which links this file into the same library so that its
// launches go through the same CUDA runtime as qcu's -- the way qcu launches it (src/draft.cu:14-15: one thread per
// site of one parity, blocks of 32, include/lattice_set.h), on qcu's internal
// layouts, with CUDA events around back-to-back launches.  BENCHMARK / TEST
// INFRASTRUCTURE ONLY: the product library never loads this file or qcu.
//
// The inputs arrive in PyQuda layout and are put into qcu's layouts by qcu's
// own permutation kernels (src/lattice_cuda.cu:41-211), out of place; the
// first launch's output is permuted back so the caller can check it.
#include <cuda_runtime.h>

#include <cstdio>

// qcu's kernels (defined in qcu's objects of the same library; launched through their host stubs)
__global__ void wilson_dslash(void *device_U, void *device_src, void *device_dest, void *device_lat_xyzt,
                              const int device_parity);
__global__ void _tzyxsc2sctzyx(void *device_fermi, void *device__fermi, int lat_4dim);
__global__ void _sctzyx2tzyxsc(void *device_fermi, void *device__fermi, int lat_4dim);
__global__ void _dptzyxcc2ccdptzyx(void *device_gauge, void *device__gauge, int lat_4dim);

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      fprintf(stderr, "ref_timer: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      rc = 2;                                                                         \
      goto done;                                                                      \
    }                                                                                 \
  } while (0)

// out_pyq, in_pyq: half spinors, gauge_pyq: the full gauge, all complex128 in
// PyQuda layout on the device; latt = {Lx, Ly, Lz, Lt}.  Returns 0 on success;
// *ms = mean milliseconds per launch of `iters` launches.
extern "C" int qcu_ref_wilson_dslash_timed(void *out_pyq, const void *in_pyq, const void *gauge_pyq,
                                           const int latt[4], int parity, int iters, double *ms) {
  int rc = 0;
  const int lat[5] = {latt[0] / 2, latt[1], latt[2], latt[3], latt[0] / 2 * latt[1] * latt[2] * latt[3]};
  const int vh = lat[4];
  if (latt[0] % 2 != 0 || vh % 32 != 0 || iters < 1) return 1;  // qcu's own constraints (lattice_set.h:103-110)
  const size_t c128 = 16;
  void *U = nullptr, *src = nullptr, *dst = nullptr, *dlat = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const dim3 grid(vh / 32), block(32);
  float t = 0.f;
  CK(cudaMalloc(&U, (size_t)vh * 2 * 4 * 9 * c128));
  CK(cudaMalloc(&src, (size_t)vh * 12 * c128));
  CK(cudaMalloc(&dst, (size_t)vh * 12 * c128));
  CK(cudaMalloc(&dlat, sizeof(lat)));
  CK(cudaMemcpy(dlat, lat, sizeof(lat), cudaMemcpyHostToDevice));
  CK(cudaDeviceSynchronize());
  _dptzyxcc2ccdptzyx<<<grid, block>>>(const_cast<void *>(gauge_pyq), U, vh);
  _tzyxsc2sctzyx<<<grid, block>>>(const_cast<void *>(in_pyq), src, vh);
  wilson_dslash<<<grid, block>>>(U, src, dst, dlat, parity);
  _sctzyx2tzyxsc<<<grid, block>>>(dst, out_pyq, vh);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  for (int i = 0; i < 3; i++) wilson_dslash<<<grid, block>>>(U, src, dst, dlat, parity);  // warm-up
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, 0));
  for (int i = 0; i < iters; i++) wilson_dslash<<<grid, block>>>(U, src, dst, dlat, parity);
  CK(cudaEventRecord(e1, 0));
  CK(cudaEventSynchronize(e1));
  CK(cudaGetLastError());
  CK(cudaEventElapsedTime(&t, e0, e1));
  *ms = (double)t / iters;
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(U);
  cudaFree(src);
  cudaFree(dst);
  cudaFree(dlat);
  return rc;
}
