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
//    8^3x64); the array is 32768 * 576 B = 18 MiB and every GPU that loads
//    the library holds it until the process exits;
//  * the first call on a device does a one-time set-up with that device
//    current: it looks up the array's device address (and the driver may
//    reserve the kernels' local memory at their first launch); make that first
//    call before any stream capture;
//  * every call reuses the same array, which keeps the previous call's
//    contents; calls that overlap on the GPU (from several host threads, or
//    on different streams) race on it.  The call itself runs on the legacy
//    default stream and returns after its work has completed.
#include <mutex>

#include "internal.h"

namespace qcu {

constexpr int NOALLOC_MAX_VH = 32768;
constexpr int NOALLOC_MAX_DEVICES = 64;

// scratch: packed inverse clover (2 chiral blocks x 18 double2 per site) and
// the zero-pivot counter
static __device__ __align__(256) double2 g_noalloc_clover[(size_t)NOALLOC_MAX_VH * 2 * 18];
static __device__ __align__(256) int g_noalloc_bad[64];

struct NoAllocSlot {
  void *clover = nullptr;
  int *bad = nullptr;
};

// device address of the scratch on the current device (looked up once per device)
static NoAllocSlot noalloc_slot() {
  static std::mutex mu;
  static NoAllocSlot slots[NOALLOC_MAX_DEVICES];
  int dev = 0;
  QCU_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < NOALLOC_MAX_DEVICES, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(mu);
  NoAllocSlot &s = slots[dev];
  if (s.clover == nullptr) {
    void *c = nullptr, *b = nullptr;
    QCU_CUDA(cudaGetSymbolAddress(&c, g_noalloc_clover));
    QCU_CUDA(cudaGetSymbolAddress(&b, g_noalloc_bad));
    s.clover = c;
    s.bad = static_cast<int *>(b);
  }
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
