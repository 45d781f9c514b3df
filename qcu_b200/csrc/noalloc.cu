// dslashCloverQcuNoAlloc: the clover hopping term for callers that must not
// allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a framework whose
// caching allocator has already reserved the device memory it is allowed to
// use, a job running under a hard per-process device-memory cap, or a
// latency-critical path where an allocation (and the synchronisation it can
// imply) is not acceptable.  dslashCloverQcu needs scratch memory for the
// inverse clover field of the output parity; this variant keeps that scratch
// in a file-scope __device__ array instead, so a call allocates nothing.
//
// Limits and rules:
//  * at most NOALLOC_MAX_VH sites per parity (16^4 = 32768, e.g. 16^4, 16^3x8,
//    8^3x64); the array is 32768 * 576 B = 18 MiB per device;
//  * the driver reserves that array on a device when the library's device
//    code is loaded there: with lazy module loading (the CUDA 12 default)
//    that is the first use on that device, typically this entry point's first
//    call; with CUDA_MODULE_LOADING=EAGER it is when the library is loaded.
//    A caller under a hard memory cap should make the first call early, while
//    the 18 MiB are still available; the array is then held until the process
//    exits;
//  * every call looks up the array's device address with that device current
//    (cudaGetSymbolAddress, cheap once the module is loaded), so a call after
//    cudaDeviceReset finds the array of the new context;
//  * every call synchronises the device and runs on the legacy default
//    stream: no call may be made while any stream of the process is being
//    captured, and a call cannot itself be captured;
//  * every call reuses the same array, which keeps the previous call's
//    contents; calls that overlap on the GPU (from several host threads)
//    race on it.  A call returns after its work has completed.
#include "internal.h"

namespace qcu {

constexpr int NOALLOC_MAX_VH = 32768;

// scratch: packed inverse clover (2 chiral blocks x 18 double2 per site) and
// the zero-pivot counter
static __device__ __align__(256) double2 g_noalloc_clover[(size_t)NOALLOC_MAX_VH * 2 * 18];
static __device__ __align__(256) int g_noalloc_bad;

struct NoAllocSlot {
  void *clover = nullptr;
  int *bad = nullptr;
};

// device addresses of the scratch in the current device's context
static NoAllocSlot noalloc_slot() {
  NoAllocSlot s;
  void *c = nullptr, *b = nullptr;
  QCU_CUDA(cudaGetSymbolAddress(&c, g_noalloc_clover));
  QCU_CUDA(cudaGetSymbolAddress(&b, g_noalloc_bad));
  s.clover = c;
  s.bad = static_cast<int *>(b);
  return s;
}

int noalloc_max_vh() { return NOALLOC_MAX_VH; }

void clover_dslash_noalloc(void *out, const void *in, const void *gauge, const int latt[4], int parity) {
  require(out && in && gauge, "dslash: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  const Geom g = make_geom(latt);
  require(g.Vh <= NOALLOC_MAX_VH, "lattice too large for dslashCloverQcuNoAlloc: " + std::to_string(g.Vh) +
                                      " sites per parity, the static scratch holds " +
                                      std::to_string(NOALLOC_MAX_VH));
  const NoAllocSlot slot = noalloc_slot();
  const cudaStream_t s = 0;  // legacy default stream: no stream object to create
  QCU_CUDA(cudaDeviceSynchronize());
  QCU_CUDA(cudaMemsetAsync(slot.bad, 0, sizeof(int), s));  // the counter must start at zero
  // clover of the output parity with qcu's unit normalisation, inverted into the scratch
  launch_clover_build(g, gauge, parity, 1.0, nullptr, slot.clover, slot.bad, s);
  DslashArgs d;
  d.in = in;
  d.out = out;
  d.gauge = gauge;
  d.parity = parity;
  d.t_bc = 1.0;
  d.a = 1.0;
  d.clover = slot.clover;
  Context none;  // no reductions: the launch touches neither solver state nor partials
  launch_dslash(AOS64, GAOS64, CSOA64, g, d, none, s);
  int nbad = 0;
  QCU_CUDA(cudaMemcpyAsync(&nbad, slot.bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  QCU_CUDA(cudaStreamSynchronize(s));
  require(nbad == 0, "clover term is singular on " + std::to_string(nbad) + " site blocks");
}

}  // namespace qcu
