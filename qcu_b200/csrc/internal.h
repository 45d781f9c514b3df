// Host-side internals shared by the translation units of libqcu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "fields.cuh"
#include "reduce.cuh"

namespace qcu {

// ---------------------------------------------------------------- errors
// Errors never exit the process and never cross the C ABI as exceptions:
// internal code throws qcu::Error, every extern "C" entry point catches it,
// records it as the thread's last error and returns a status.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
void set_last_error(int code, const std::string &msg);
void clear_last_error();

#define QCU_CUDA(call)                                                                                     \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      throw ::qcu::Error(2, std::string("CUDA error '") + cudaGetErrorString(e_) + "' at " + __FILE__ + ":" + \
                                std::to_string(__LINE__));                                                 \
  } while (0)

// every kernel launch goes through this check, which also counts it
void note_launch(long long n);
long long launch_count();
void set_launch_count(long long v);
#define QCU_CHECK_LAUNCH()           \
  do {                               \
    QCU_CUDA(cudaGetLastError());    \
    ::qcu::note_launch(1);           \
  } while (0)

inline void require(bool ok, const std::string &msg) {
  if (!ok) throw Error(1, msg);
}

// ---------------------------------------------------------------- geometry
Geom make_geom(const int latt[4]);  // validates: all > 0, Lx even

constexpr int DSLASH_BLOCK = 128;
constexpr int BLAS_BLOCK = 256;
constexpr int MAX_REDUCE_BLOCKS = 148 * 8;  // one resident wave of 256-thread blocks on B200

inline int blas_grid(int n) {
  int g = (n + BLAS_BLOCK - 1) / BLAS_BLOCK;
  return g > MAX_REDUCE_BLOCKS ? MAX_REDUCE_BLOCKS : (g < 1 ? 1 : g);
}

// bytes of one parity spinor in each storage kind
size_t spinor_bytes(int kind, int Vh);
size_t spinor_norm_bytes(int kind, int Vh);

// ---------------------------------------------------------------- device buffers
struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  cudaStream_t stream = nullptr;  // the context stream the buffer was allocated on (and is freed on)
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf();
  void ensure(size_t bytes);  // grow-only
  void release();
  template <typename T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// one parity spinor in internal storage
struct Spinor {
  int kind = SOA64;
  int Vh = 0;
  DevBuf data, norm;
  void alloc(int k, int vh);
  template <int K>
  SpinorView<K> view() const {
    return SpinorView<K>{data.p, norm.as<float>(), Vh};
  }
};

// ---------------------------------------------------------------- per-device context
// Streams, the solver state block and the reduction partials persist across
// API calls (one context per device, created on first use).
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  SolverState *st = nullptr;       // device
  SolverState *st_host = nullptr;  // pinned mirror
  double *partials = nullptr;      // blocks * RED_MAXV doubles (grown to the largest grid used)
  size_t partials_blocks = 0;
  int sms = 148;                   // multiprocessors of the device
  // scratch of the legacy clover call (dslashCloverQcu): the inverse clover
  // of the output parity and its zero-pivot counter.  Per device, used only
  // under `mu`; allocated on first use and kept until exit.
  DevBuf *legacy_clover = nullptr;
  DevBuf *legacy_bad = nullptr;
  std::mutex mu;
  void ensure_partials(size_t blocks);
};
Context &context();  // current device's context

// One T per device, created on first use and kept until exit: the work
// buffers of a solve live on the device they were allocated on, so each
// device gets its own (callers hold that device's Context::mu while using it).
template <typename T>
T &per_device(const Context &ctx) {
  static std::mutex mu;
  static std::map<int, T *> objs;
  std::lock_guard<std::mutex> lk(mu);
  T *&p = objs[ctx.device];
  if (p == nullptr) p = new T();
  return *p;
}

// ---------------------------------------------------------------- kernels (launchers)
struct DslashArgs {
  const void *in = nullptr;
  const float *in_norm = nullptr;
  void *out = nullptr;
  float *out_norm = nullptr;
  const void *x1 = nullptr;  // epilogue sources: out = a*w + b1*x1 + b2*x2
  const float *x1_norm = nullptr;
  const void *x2 = nullptr;
  const float *x2_norm = nullptr;
  const void *rt = nullptr;  // shadow residual for the fused <rt, out>
  const float *rt_norm = nullptr;
  const void *gauge = nullptr;
  const void *clover = nullptr;  // packed inverse clover of the output parity, or null
  int parity = 0;
  double t_bc = 1.0, a = 1.0, b1 = 0.0, b2 = 0.0;
  int red = 0;  // RedKind
  int gate = GATE_ALWAYS;
  int fin = FIN_STORE;
};
enum RedKind { RED_NONE = 0, RED_DOT_RT = 1, RED_TS_TT = 2, RED_NORM = 3 };

// kind: spinor storage (AOS64/SOA64/SOA32/SOA16); gkind: gauge storage; ckind: clover storage
void launch_dslash(int kind, int gkind, int ckind, const Geom &g, const DslashArgs &a, Context &ctx,
                   cudaStream_t s);

// the vectors of one BiCGSTAB solve: r..t and the partial solution x in the
// inner precision, x64/r64 the FP64 solution and true residual
struct VecSet {
  void *r, *rt, *p, *v, *s, *t, *x;
  float *rn, *rtn, *pn, *vn, *sn, *tn, *xn;
  void *x64, *r64;
};
void launch_pupdate(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s);
void launch_supdate(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s);
void launch_xrupdate(int kind, int Vh, const VecSet &vs, Context &ctx, int gate, cudaStream_t s);
void launch_xfold(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s);
void launch_rconv(int kind, int Vh, const VecSet &vs, Context &ctx, int gate, cudaStream_t s);
void launch_init(int kind, int Vh, const VecSet &vs, Context &ctx, cudaStream_t s);
// device-side loop condition for a graph WHILE node: continue while !st->done (at most cap passes)
void launch_loop_cond(SolverState *st, cudaGraphConditionalHandle h, unsigned cap, cudaStream_t s);
void launch_convert(int kin, int kout, int Vh, const void *in, const float *in_n, void *out, float *out_n,
                    cudaStream_t s);
void launch_axpby(int kind, int Vh, double a, void *x, float *xn, double b, void *y, float *yn, cudaStream_t s);
// st->sums[0..3] = Re<a,b>, Im<a,b>, |a|^2, |b|^2
void launch_dots(int kind, int Vh, void *a, float *an, void *b, float *bn, Context &ctx, cudaStream_t s);

// gauge: PyQuda complex128 [4][2][Vh][3][3] -> reconstruct-12 internal storage
void launch_gauge_pack(int gkind, const Geom &g, const void *pyq, void *out, cudaStream_t s);
size_t gauge_bytes(int gkind, int Vh);

// clover: build A = 1 - coeff/8 sum g_mu g_nu (Q - Q^+) on parity `par` from the
// PyQuda gauge, packed (CSOA64); optionally also its inverse
void launch_clover_build(const Geom &g, const void *gauge_pyq, int par, double coeff, void *A64, void *Ainv64,
                         int *bad, cudaStream_t s);
void launch_clover_to32(int Vh, const void *c64, void *c32, cudaStream_t s);
// out = C in for a packed clover C (AOS64 or SOA64 spinors)
void launch_clover_apply(int kind, int Vh, const void *c64, const void *in, void *out, cudaStream_t s);
size_t clover_bytes(int ckind, int Vh);

// seeded generators (PyQuda layouts, complex128)
void launch_gauge_random(const Geom &g, void *gauge, int kind, double eps, uint64_t seed, cudaStream_t s);
void launch_fermion_random(void *psi, int64_t n, int kind, uint64_t seed, cudaStream_t s);
// internal-layout uniform (0,1] field whose element (site, comp) uses counter site*12+comp
void launch_uniform_soa64(int Vh, void *out, uint64_t seed, cudaStream_t s);

}  // namespace qcu
