// Allocation-free AC effective-Hamiltonian apply (FP64).
//
// Some callers cannot let a library call cudaMalloc: a host framework whose
// caching allocator (PyTorch, CUDA.jl) has already reserved the device memory,
// so a library allocation fails or forces the pool to be flushed, and callers
// that must not add the implicit device synchronisation that cudaMalloc /
// cudaFree can cause in the middle of their own stream work.  For them,
// imps_ac_apply_noalloc runs the same GL.x -> level mix -> .GR pipeline as
// imps_ac_apply, with every intermediate held in one file-scope device array of
// fixed size instead of library-allocated buffers.  The caller passes all
// inputs and outputs as device pointers (the MPO tensor as a small host array).
//
// Limits and sharing rules (also stated in include/imps_b200.h):
//  * the array is kNoAllocScratchBytes (64 MiB) on every device that loads the
//    library, held until the process exits.  This file is its own CUDA module, and
//    with lazy module loading the array comes into being when its address is
//    first looked up; imps_ctx_create does that lookup (noalloc_prepare), so the
//    array exists as soon as a context is created on the device, before the
//    caller's allocator reserves the rest of the memory;
//  * the intermediates need 16 * Dl * d * Dr * (m + n) bytes plus the MPO
//    tensor (at most 64 KiB); larger problems are rejected with IMPS_INVALID_ARG;
//  * every call uses the same array and leaves its contents behind, so calls
//    whose GPU work overlaps (other streams, other host threads) race;
//  * the call is asynchronous: its work is queued on the context's stream, which
//    the caller orders against its own producers and consumers of GL, GR, x, y
//    (or shares through imps_ctx_set_stream);
//  * W_host is copied into the array during the call.
#include <atomic>
#include <mutex>

#include "imps_internal.h"

namespace imps {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr size_t kNoAllocWBytes = size_t(64) << 10;

// The scratch array.  In host code `g_noalloc_scratch` names a host-side
// stand-in, not device memory: only the address from cudaGetSymbolAddress may
// be handed to kernels.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
// Per-device address of the array.  Contexts on several host threads may look it
// up at the same time: the lookup itself runs under a mutex and the published
// pointer is atomic.
std::atomic<void*> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

// Once per device, with that device current: the array's device address.
void* scratch_address(int device) {
  IMPS_REQUIRE(device >= 0 && device < kMaxDevices, IMPS_INVALID_ARG, "device ordinal out of range");
  void* p = g_scratch_addr[device].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  p = g_scratch_addr[device].load(std::memory_order_relaxed);
  if (!p) {
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    IMPS_REQUIRE(e == cudaSuccess && p != nullptr, IMPS_CUDA_ERROR,
                 std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device].store(p, std::memory_order_release);
  }
  return p;
}

// Disables the per-kernel event timers (they create CUDA events) for one call.
struct NoProfile {
  Context* ctx;
  bool old;
  explicit NoProfile(Context* c) : ctx(c), old(c->profile) { ctx->profile = false; }
  ~NoProfile() { ctx->profile = old; }
};

}  // namespace

void ac_apply_noalloc(Context* ctx, int Dl, int d, int Dr, int m, int n, const cplx* W_host, const dcplx* GL,
                      const dcplx* GR, const dcplx* x, dcplx* y) {
  IMPS_REQUIRE(Dl > 0 && d > 0 && Dr > 0 && m > 0 && n > 0, IMPS_INVALID_ARG, "empty dimension");
  IMPS_REQUIRE(d <= 8, IMPS_INVALID_ARG, "physical dimension above 8 is not supported");
  const size_t wbytes = (size_t)m * d * n * d * sizeof(dcplx);
  const size_t t1 = (size_t)Dl * m * d * Dr, t2 = (size_t)Dl * d * Dr * n;
  const size_t need = (t1 + t2) * sizeof(dcplx);
  IMPS_REQUIRE(wbytes <= kNoAllocWBytes, IMPS_INVALID_ARG, "no-alloc AC apply: MPO tensor larger than 64 KiB");
  IMPS_REQUIRE(need <= kNoAllocScratchBytes - kNoAllocWBytes, IMPS_INVALID_ARG,
               "no-alloc AC apply: intermediates need " + std::to_string(need) +
                   " bytes, above the fixed scratch of " + std::to_string(kNoAllocScratchBytes - kNoAllocWBytes) +
                   " bytes");
  // block pattern of W (fixed array, no heap)
  std::pair<int, int> nz[256];
  int nnz = 0;
  bool hit[64] = {false};
  IMPS_REQUIRE(n <= 64 && m <= 64, IMPS_INVALID_ARG, "no-alloc AC apply: more than 64 MPO levels");
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      bool nzb = false;
      for (int u = 0; u < d && !nzb; ++u)
        for (int s = 0; s < d; ++s)
          if (W_host[i + (size_t)m * (u + (size_t)d * (j + (size_t)n * s))] != cplx(0.0, 0.0)) {
            nzb = true;
            break;
          }
      if (nzb) {
        IMPS_REQUIRE(nnz < 256, IMPS_INVALID_ARG, "no-alloc AC apply: too many MPO blocks");
        nz[nnz++] = {i, j};
        hit[j] = true;
      }
    }
  NoProfile np(ctx);
  unsigned char* base = static_cast<unsigned char*>(scratch_address(ctx->device));
  dcplx* Wd = reinterpret_cast<dcplx*>(base);
  dcplx* T1 = reinterpret_cast<dcplx*>(base + kNoAllocWBytes);
  dcplx* T2 = T1 + t1;
  IMPS_CUDA(cudaMemcpyAsync(Wd, W_host, wbytes, cudaMemcpyHostToDevice, ctx->stream));
  zgemm_fp64(ctx, OP_N, OP_N, Dl * m, d * Dr, Dl, 1.0, GL, (int64_t)Dl * m, 0, x, Dl, 0, 0.0, T1, (int64_t)Dl * m, 0, 1);
  // right levels without any block read as zero (the array keeps the previous call's data)
  for (int q = 0; q < n; ++q)
    if (!hit[q]) zfill(ctx, (int64_t)Dl * d * Dr, 0.0, T2 + (int64_t)Dl * d * Dr * q);
  MixPlan pl;
  pl.Db = Dl; pl.R = m; pl.P = d; pl.Q = n; pl.S = d; pl.C = Dr;
  pl.in_r = Dl; pl.in_s = (int64_t)Dl * m; pl.in_c = (int64_t)Dl * m * d;
  pl.out_p = Dl; pl.out_q = (int64_t)Dl * d * Dr; pl.out_c = (int64_t)Dl * d;
  pl.M = Wd;
  level_mix_nz(ctx, pl, nz, nnz, T1, T2);
  zgemm_fp64(ctx, OP_N, OP_N, Dl * d, Dr, Dr * n, 1.0, T2, (int64_t)Dl * d, 0, GR, (int64_t)Dr * n, 0, 0.0, y,
             (int64_t)Dl * d, 0, 1);
  ctx->n_ac_apply++;
}

size_t noalloc_scratch_bytes() { return kNoAllocScratchBytes - kNoAllocWBytes; }

void noalloc_prepare(int device) { (void)scratch_address(device); }

}  // namespace imps
