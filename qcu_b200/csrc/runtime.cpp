// Runtime support: error recording, device buffers, the per-device context.
#include <atomic>
#include <cstring>
#include <map>
#include <memory>

#include "internal.h"

namespace qcu {

// ---------------------------------------------------------------- errors
static thread_local int g_err_code = 0;
static thread_local std::string g_err_msg;

void set_last_error(int code, const std::string &msg) {
  g_err_code = code;
  g_err_msg = msg;
  if (getenv("QCU_QUIET") == nullptr) fprintf(stderr, "qcu: %s\n", msg.c_str());
}
void clear_last_error() {
  g_err_code = 0;
  g_err_msg.clear();
}
int last_error(char *buf, int len) {
  if (buf && len > 0) {
    strncpy(buf, g_err_msg.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return g_err_code;
}

// ---------------------------------------------------------------- launch counter
static std::atomic<long long> g_launches{0};
void note_launch(long long n) { g_launches += n; }
long long launch_count() { return g_launches.load(); }
void set_launch_count(long long v) { g_launches = v; }

// ---------------------------------------------------------------- geometry
Geom make_geom(const int latt[4]) {
  require(latt != nullptr, "lattice size pointer is null");
  for (int d = 0; d < 4; d++) require(latt[d] > 0, "lattice sizes must be positive");
  require(latt[0] % 2 == 0, "Lx must be even for the even-odd layout");
  const int64_t vh = (int64_t)latt[0] / 2 * latt[1] * latt[2] * latt[3];
  require(vh < (1LL << 28), "lattice too large (Vh must be < 2^28)");
  Geom g;
  g.Lxh = latt[0] / 2;
  g.Ly = latt[1];
  g.Lz = latt[2];
  g.Lt = latt[3];
  g.sy = g.Lxh;
  g.sz = g.Lxh * g.Ly;
  g.st = g.Lxh * g.Ly * g.Lz;
  g.Vh = (int)vh;
  // reciprocal multipliers, exact for every site index while Vh * d < 2^32 (geom_div)
  auto magic = [&](int d) -> unsigned {
    if (d < 2 || (uint64_t)(vh + 64) * (uint64_t)d >= (1ULL << 32)) return 0u;  // padded indices too
    return (unsigned)(((1ULL << 32) + (uint64_t)d - 1) / (uint64_t)d);
  };
  g.m_lxh = magic(g.Lxh);
  g.m_ly = magic(g.Ly);
  g.m_lz = magic(g.Lz);
  return g;
}

size_t spinor_bytes(int kind, int Vh) {
  const size_t Vp = pad_sites(Vh);  // site-blocked kinds are padded to whole blocks of 32
  switch (kind) {
    case AOS64: return (size_t)Vh * 12 * 16;
    case SOA64: return Vp * 12 * 16;
    case SOA32: return Vp * 12 * 8;
    case SOA16: return Vp * 12 * 4;
  }
  return 0;
}
size_t spinor_norm_bytes(int kind, int Vh) { return kind == SOA16 ? (size_t)pad_sites(Vh) * 4 : 0; }

// ---------------------------------------------------------------- buffers
// Device buffers come from a memory pool of the library's own, ordered on the
// context stream, that keeps freed memory for reuse (release threshold: never).
// A gauge handle loaded and freed per solve then costs no cudaMalloc/cudaFree,
// whose page mapping on multi-GB buffers took 10-300 ms per call on B200.
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static cudaMemPool_t pool_for(int dev) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  QCU_CUDA(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = UINT64_MAX;
  QCU_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  g_pools[dev] = pool;
  return pool;
}

DevBuf::~DevBuf() { release(); }
void DevBuf::release() {
  if (p) cudaFreeAsync(p, stream);
  p = nullptr;
  n = 0;
}
void DevBuf::ensure(size_t bytes) {
  if (bytes <= n) return;
  release();
  if (bytes == 0) return;
  Context &ctx = context();
  stream = ctx.stream;
  QCU_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool_for(ctx.device), stream));
  n = bytes;
}

void Spinor::alloc(int k, int vh) {
  kind = k;
  Vh = vh;
  data.ensure(spinor_bytes(k, vh));
  // 16-bit spinors are read and written with 32-byte accesses
  require(reinterpret_cast<uintptr_t>(data.p) % 32 == 0, "spinor buffer is not 32-byte aligned");
  if (k == SOA16) norm.ensure(spinor_norm_bytes(k, vh));
}

// ---------------------------------------------------------------- context
void Context::ensure_partials(size_t blocks) {
  if (blocks <= partials_blocks) return;
  if (partials) cudaFree(partials);
  partials = nullptr;
  QCU_CUDA(cudaMalloc(&partials, blocks * RED_MAXV * sizeof(double)));
  partials_blocks = blocks;
}

static std::mutex g_ctx_mu;
static std::map<int, std::unique_ptr<Context>> g_ctx;

Context &context() {
  int dev = 0;
  QCU_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto it = g_ctx.find(dev);
  if (it != g_ctx.end()) return *it->second;
  auto c = std::make_unique<Context>();
  c->device = dev;
  QCU_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  QCU_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev));
  QCU_CUDA(cudaMalloc(&c->st, sizeof(SolverState)));
  QCU_CUDA(cudaMemset(c->st, 0, sizeof(SolverState)));
  QCU_CUDA(cudaMallocHost(&c->st_host, sizeof(SolverState)));
  memset(c->st_host, 0, sizeof(SolverState));
  c->ensure_partials(MAX_REDUCE_BLOCKS);
  Context &ref = *c;
  g_ctx[dev] = std::move(c);
  return ref;
}

}  // namespace qcu
