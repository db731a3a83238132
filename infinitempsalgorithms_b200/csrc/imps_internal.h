// Internal declarations of the imps_b200 runtime (not part of the C ABI).
//
// Storage convention everywhere: column-major complex128 (interleaved re, im),
// exactly the Julia layout of the reference, so a host array of the reference
// can be copied byte for byte.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <set>
#include <tuple>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/imps_b200.h"

namespace imps {

using cplx = std::complex<double>;
using dcplx = double2;  // device complex

// Error carried from the depths of the runtime to the C ABI.
struct Error : public std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define IMPS_CUDA(call)                                                               \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      if (e_ == cudaErrorMemoryAllocation)                                            \
        throw ::imps::Error(IMPS_OOM, std::string("out of device memory: ") + #call); \
      throw ::imps::Error(IMPS_CUDA_ERROR, std::string(cudaGetErrorString(e_)) +      \
                                               " at " + __FILE__ + ":" +              \
                                               std::to_string(__LINE__));             \
    }                                                                                 \
  } while (0)

#define IMPS_REQUIRE(cond, status, msg)        \
  do {                                         \
    if (!(cond)) throw ::imps::Error(status, msg); \
  } while (0)

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  explicit DevBuf(size_t b) { alloc(b); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t b) {
    release();
    if (b) IMPS_CUDA(cudaMalloc(&ptr, b));
    bytes = b;
  }
  // Grow-only: keeps the allocation when it is already large enough.
  void ensure(size_t b) { if (b > bytes) alloc(b); }
  void release() { if (ptr) cudaFree(ptr); ptr = nullptr; bytes = 0; }
  dcplx* z() const { return static_cast<dcplx*>(ptr); }
  double* d() const { return static_cast<double*>(ptr); }
};

// Kernel timing accumulated per kernel class (CUDA events on the context stream).
struct KernelStat {
  int64_t launches = 0;
  double ms = 0.0;
  double flops = 0.0;   // algorithmic flops (or bytes for memory-bound kernels)
};

enum GemmPrecision { PREC_FP64 = 0, PREC_SPLIT_I8 = 1 };

struct SplitOperand;
// (pointer, side, op, rows, K, ld, slices) -> split planes of an operand that is
// constant for the current scope (environments during a solve, site tensors
// during an environment build)
using SplitKey = std::tuple<const void*, int, int, int, int, int64_t, int>;

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int precision = PREC_FP64;
  int nslices = 5;           // int8 slices per operand in split mode
  int max_adaptive_slices = 6;  // adaptive mode: a tolerance needing more slices runs in FP64
  bool adaptive_slices = false;
  int fp64_engine = 0;       // FP64 GEMM kernel: 0 = DMMA tensor cores, 1 = SIMT DFMA (env IMPS_FP64_ENGINE)
  std::string last_error;
  // named grow-only scratch buffers
  std::map<std::string, DevBuf> scratch;
  // reduction scratch (per-block partials) and pinned host staging
  DevBuf red;
  double* host_pinned = nullptr;
  size_t host_pinned_bytes = 0;
  int* dev_info = nullptr;
  // device error flag of the bounded waits (split GEMM) and its pinned host copy;
  // armed while a kernel that may set it has not been checked at a synchronisation
  int* err_dev = nullptr;
  int* err_host = nullptr;
  bool err_armed = false;
  void* qr_count_ptr = nullptr;       // completion counter of the QR small products, zeroed at this address
  long long wait_cycles = 2000000000LL;  // bound of each pipeline wait (~1 s at 1.9 GHz)
  // profiling
  bool profile = false;
  const char* prof_tag = "";           // call-site tag appended to kernel classes when profiling
  std::set<std::string> profile_only;  // when non-empty, only these kernel classes are timed
  std::vector<cudaEvent_t> event_pool; // reusable timing events
  std::map<std::string, KernelStat> stats;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  double pending_flops_dummy = 0;
  std::vector<double> pending_flops;
  // counters
  int64_t n_ac_apply = 0, n_c_apply = 0, n_push = 0, n_gemm = 0, n_kernels = 0, n_qr = 0;
  double gemm_flops = 0.0;  // real flops of every complex GEMM requested (8 M N K), either precision
  double qr_flops = 0.0;    // real flops of the Householder QRpos factorizations (factor + Q)
  int num_sms = 148;
  // split-precision state
  double split_tol = 1e-10;            // accuracy requested by the running solver
  int force_fp64 = 0;                  // > 0: every GEMM in FP64 (gauge, Galerkin, energy)
  std::multiset<const void*> const_ptrs;
  std::map<SplitKey, std::shared_ptr<SplitOperand>> split_cache;
  std::shared_ptr<SplitOperand> split_scratch[2];
  // split operands released by a ConstScope, kept (with their device buffers) for the
  // next constant operands: no cudaMalloc / cudaFree, and so no implicit device
  // synchronisation, per solve
  std::vector<std::shared_ptr<SplitOperand>> split_pool;
  int64_t split_calls = 0, split_cache_hits = 0;
  // split GEMM launches, their algorithmic work (8 M N K real flops of the complex
  // product each computes) and the int8 operations the tensor pipe executes for it
  int64_t split_launches = 0;
  double split_alg_flops = 0.0, split_exec_ops = 0.0;

  // cap on the named scratch workspace below (0 = none); growing past it is IMPS_OOM
  size_t workspace_limit = 0;
  DevBuf& buf(const std::string& name, size_t bytes) {
    DevBuf& b = scratch[name];
    if (bytes > b.bytes && workspace_limit > 0) {
      size_t total = 0;
      for (const auto& kv : scratch) total += kv.second.bytes;
      if (total - b.bytes + bytes > workspace_limit)
        throw Error(IMPS_OOM, "workspace limit of " + std::to_string(workspace_limit) + " bytes reached (buffer '" +
                                  name + "' needs " + std::to_string(bytes) + " bytes)");
    }
    b.ensure(bytes);
    return b;
  }
  double* pinned(size_t bytes);
};

// Marks operands constant for the lifetime of the scope (their int8 splits are cached).
struct ConstScope {
  Context* ctx;
  std::vector<const void*> ptrs;
  ConstScope(Context* c, std::vector<const void*> p) : ctx(c), ptrs(std::move(p)) {
    for (auto q : ptrs) ctx->const_ptrs.insert(q);
  }
  ~ConstScope() {
    for (auto q : ptrs) {
      auto it = ctx->const_ptrs.find(q);
      if (it != ctx->const_ptrs.end()) ctx->const_ptrs.erase(it);
      if (ctx->const_ptrs.count(q) == 0) {
        for (auto it2 = ctx->split_cache.begin(); it2 != ctx->split_cache.end();) {
          if (std::get<0>(it2->first) == q) {
            ctx->split_pool.push_back(std::move(it2->second));
            if (ctx->split_pool.size() > 8) ctx->split_pool.erase(ctx->split_pool.begin());
            it2 = ctx->split_cache.erase(it2);
          } else {
            ++it2;
          }
        }
      }
    }
  }
};
// Tags the kernels launched while alive with a call site (profiling attribution).
struct ProfTag {
  Context* ctx;
  const char* old;
  ProfTag(Context* c, const char* tag) : ctx(c), old(c->prof_tag) { ctx->prof_tag = tag; }
  ~ProfTag() { ctx->prof_tag = old; }
};
// Forces FP64 for every GEMM while alive.
struct Fp64Scope {
  Context* ctx;
  explicit Fp64Scope(Context* c) : ctx(c) { ctx->force_fp64++; }
  ~Fp64Scope() { ctx->force_fp64--; }
};
// One-time per-device setup (kernel attributes) safe to reach from several host threads:
// the setup may run more than once when threads race, so it must be idempotent.
struct DeviceOnce {
  std::atomic<uint64_t> done{0};
  template <class F>
  void run(int device, F&& f) {
    const uint64_t bit = 1ull << (device & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    f();
    done.fetch_or(bit, std::memory_order_release);
  }
};

// Inside an Fp64Scope: lets the split engine serve the GEMMs at accuracy tol while alive,
// when the context runs the split engine with adaptive slice counts (the slice count then
// follows tol; a fixed count could not reach an arbitrary tolerance).
struct SplitAllowScope {
  Context* ctx;
  int saved;
  double old_tol;
  bool on;
  SplitAllowScope(Context* c, double tol)
      : ctx(c), saved(c->force_fp64), old_tol(c->split_tol),
        on(c->precision == PREC_SPLIT_I8 && c->adaptive_slices) {
    if (on) {
      ctx->force_fp64 = 0;
      ctx->split_tol = tol;
    }
  }
  ~SplitAllowScope() {
    if (on) {
      ctx->force_fp64 = saved;
      ctx->split_tol = old_tol;
    }
  }
};
// Raises the most slices the adaptive split engine may use while alive (above it: FP64).
struct MaxSlicesScope {
  Context* ctx;
  int old;
  MaxSlicesScope(Context* c, int s) : ctx(c), old(c->max_adaptive_slices) { ctx->max_adaptive_slices = s; }
  ~MaxSlicesScope() { ctx->max_adaptive_slices = old; }
};
// Sets the accuracy the split GEMMs must meet while alive.
struct TolScope {
  Context* ctx;
  double old;
  TolScope(Context* c, double tol) : ctx(c), old(c->split_tol) { ctx->split_tol = tol; }
  ~TolScope() { ctx->split_tol = old; }
};

// Slices the split engine would use right now (0 = FP64 engine).  Adaptive mode picks
// the smallest s whose truncation floor meets ctx->split_tol; s >= 7 falls back to FP64.
int active_slices(const Context* ctx);
// the smallest slice count whose truncation floor meets tol (clamped to 2..8)
int slices_for_tol(double tol);
// Relative accuracy of the GEMM engine currently selected (0 for FP64).
double split_floor(const Context* ctx);

// RAII timer for one kernel class on the context stream (active when profiling).
struct ScopedTimer {
  Context* ctx;
  std::string name;
  double flops;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ScopedTimer(Context* c, const char* n, double f);
  ~ScopedTimer();
};

// ---------------------------------------------------------------------------
// Objects behind the opaque ABI handles
// ---------------------------------------------------------------------------
struct MpoSite {
  int m = 0, d = 0, n = 0;       // left levels, physical dim, right levels
  std::vector<cplx> W;           // dense (m, d, n, d), column-major
  DevBuf Wdev;                   // same on device
  // nonzero (i, j) blocks, 0-based
  std::vector<std::pair<int, int>> nz;
  bool block_nonzero(int i, int j) const;
  cplx at(int i, int u, int j, int s) const { return W[i + (size_t)m * (u + (size_t)d * (j + (size_t)n * s))]; }
};

}  // namespace imps

struct imps_mpo {
  imps::Context* ctx;
  int device = 0;
  int N;
  std::vector<imps::MpoSite> sites;
  std::vector<imps::MpoSite> closing;  // closing column (m, d, 1, d) of each site, for the Schur energy
  bool isidentitylevel(int i) const;  // 1-based level label
  bool isemptylevel(int i) const;
};

struct imps_state {
  imps::Context* ctx;
  int device = 0;
  int N;
  std::vector<int> d;     // physical dim per site
  std::vector<int> chi;   // chi[l] = bond dimension right of site l (bond N-1 == bond 0)
  std::vector<imps::DevBuf> AL, AR, C, AC;
  int Dl(int l) const { return chi[((l - 1) % N + N) % N]; }
  int Dr(int l) const { return chi[((l % N) + N) % N]; }
  size_t site_elems(int l) const { return (size_t)Dl(l) * d[l] * Dr(l); }
  size_t bond_elems(int l) const { return (size_t)Dr(l) * Dr(l); }
};

struct imps_envs {
  imps::Context* ctx;
  int device = 0;
  int N;
  std::vector<int> Dl, Dr, ml, nr;
  std::vector<imps::DevBuf> lefts, rights;   // (Dl, ml, Dl), (Dr, nr, Dr)
  // previous environments kept as the warm start of the next build
  std::vector<imps::DevBuf> init_lefts, init_rights;
  // Permuted copy of the left environment used by the C Hamiltonian:
  // GLp[l][a + D (a' + D w)] = lefts[l][a, w, a'].  Rebuilt lazily.
  std::vector<imps::DevBuf> GLp;
  std::vector<bool> GLp_valid;
  int64_t version = 0;
  imps_env_info last;
  // operator-scale estimates |lambda| of the AC / C problems (split-precision accuracy targets)
  std::vector<double> hest_ac, hest_c;
};

namespace imps {

// ---------------------------------------------------------------------------
// Kernels / building blocks (defined in the .cu files)
// ---------------------------------------------------------------------------
enum Op { OP_N = 0, OP_T = 1, OP_C = 2 };

// Column-major complex GEMM: C = alpha op(A) op(B) + beta C, batched with strides
// (in complex elements).  Dispatches on ctx->precision for the large products.
void zgemm(Context* ctx, Op opA, Op opB, int M, int N, int K, cplx alpha, const dcplx* A, int64_t lda,
           int64_t strideA, const dcplx* B, int64_t ldb, int64_t strideB, cplx beta, dcplx* C, int64_t ldc,
           int64_t strideC, int batch, bool allow_split = true);
// Always the FP64 engine.
void zgemm_fp64(Context* ctx, Op opA, Op opB, int M, int N, int K, cplx alpha, const dcplx* A, int64_t lda,
                int64_t strideA, const dcplx* B, int64_t ldb, int64_t strideB, cplx beta, dcplx* C,
                int64_t ldc, int64_t strideC, int batch);

// Strided block-sparse level mixing (the MPO contraction between the GEMMs):
// out[b,p,q,c] = sum_{(r,q) in nz} sum_s M[r,p,q,s] in[b,r,s,c], b contiguous.
struct MixPlan {
  int Db, P, S, C;            // extents of b, p (out phys), s (in phys), c
  int R, Q;                   // extents of r (in level) and q (out level)
  int64_t in_r, in_s, in_c;   // input strides (b stride = 1)
  int64_t out_p, out_q, out_c;
  const dcplx* M;             // dense (R, P, Q, S) column-major
  std::vector<std::pair<int, int>> nz;  // (r, q) nonzero blocks
  cplx scale = cplx(1.0, 0.0);
};
void level_mix(Context* ctx, const MixPlan& plan, const dcplx* in, dcplx* out);
// same with the block list given as a pointer (uses no heap memory; plan.nz is ignored)
void level_mix_nz(Context* ctx, const MixPlan& plan, const std::pair<int, int>* nz, int nnz, const dcplx* in,
                  dcplx* out);

// BLAS-1 style helpers (deterministic two-pass reductions)
void zcopy(Context* ctx, int64_t n, const dcplx* x, dcplx* y);
void zscal(Context* ctx, int64_t n, cplx a, dcplx* x);
void zaxpy(Context* ctx, int64_t n, cplx a, const dcplx* x, dcplx* y);        // y += a x
void zaxpby(Context* ctx, int64_t n, cplx a, const dcplx* x, cplx b, dcplx* y); // y = a x + b y
void zfill(Context* ctx, int64_t n, cplx v, dcplx* x);
void zset_identity(Context* ctx, int D, dcplx* X, int64_t ld, cplx diag);
double dznrm2(Context* ctx, int64_t n, const dcplx* x);
cplx zdotc(Context* ctx, int64_t n, const dcplx* x, const dcplx* y);  // sum conj(x) y
// One classical Gram-Schmidt projection w <- w - V h with h = V^H w, all on the device
// and one host synchronisation: returns ||w_new||^2, writes h (host) and, if nw_old2
// is given, ||w_old||^2.
double proj_pass(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, dcplx* w, cplx* h_host,
                 double* nw_old2);
// Classical Gram-Schmidt with iterative refinement of w against the nv columns of V
// (KrylovKit's ClassicalGramSchmidtIR, eta = 1/sqrt(2), at most three projections):
// h (host) receives the accumulated coefficients; returns the final ||w||.  Each
// update is fused with the next projection's dots, one host synchronisation per
// projection after the first.  A non-finite norm raises IMPS_INVALID_ARG.
double gs_project(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, dcplx* w, std::vector<cplx>& h);
// w += sum_j coef[j] V[:, j]
void zgemv_acc(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, const cplx* coef, dcplx* w);
// y = sum_j coef[j] V[:, j]
void zgemv_set(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, const cplx* coef, dcplx* y);
// X (m x n, ldx) -> Y = X^H (n x m, ldy)
void zconj_transpose(Context* ctx, int m, int n, const dcplx* X, int64_t ldx, dcplx* Y, int64_t ldy);
// trace(L * V) with L, V  D x D (regularize! coefficient, sum L[a,b] V[b,a])
cplx ztrace_prod(Context* ctx, int D, const dcplx* L, int64_t ldl, const dcplx* V, int64_t ldv);
void zadd_diag(Context* ctx, int D, dcplx* X, int64_t ld, cplx v);
void zfill2d(Context* ctx, int rows, int cols, cplx v, dcplx* Y, int64_t ldy);
// X[:, lvl-slice] strided copy helpers
void zcopy2d(Context* ctx, int rows, int cols, const dcplx* X, int64_t ldx, dcplx* Y, int64_t ldy);

// Orthogonal factorizations with a non-negative real diagonal (QRpos / LQpos).
// Q overwrites nothing: results go to Q (m x k) and R (k x n), k = min(m, n).
void qrpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* Q, dcplx* R);
void lqpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, dcplx* Q);
// The two halves of QRpos / LQpos: the factorisation (R or L, phase-fixed) keeps its
// reflectors in the named slot; Q is formed from them on request, any time before the
// next factorisation into the same slot.  Q == nullptr in qrpos / lqpos skips Q.
void qr_factor(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* R, const char* slot);
void qr_form_q(Context* ctx, int m, int n, dcplx* Q, const char* slot);
void lq_factor(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, const char* slot);
void lq_form_q(Context* ctx, int m, int n, dcplx* Q, const char* slot);

// Reads the device error flag if a kernel that may set it ran since the last check
// (synchronises the stream); a set flag is cleared and raised as IMPS_TIMEOUT.
void check_device_errors(Context* ctx);

// Host <-> device
void upload(Context* ctx, void* dst, const void* src, size_t bytes);
void download(Context* ctx, void* dst, const void* src, size_t bytes);

// ---------------------------------------------------------------------------
// Tensor-network operations (heff.cu)
// ---------------------------------------------------------------------------
// AC effective Hamiltonian y = H_AC x for site `site` (0-based); `Wover` optionally
// replaces the site's MPO tensor (used for the closing-column energy).
void ac_apply(Context* ctx, const imps_envs* envs, const imps_mpo* mpo, int site, const dcplx* x, dcplx* y,
              const MpoSite* Wover = nullptr, const dcplx* GRover = nullptr, int64_t GRover_ld = 0);
void c_apply(Context* ctx, imps_envs* envs, int site, const dcplx* x, dcplx* y);
// (re)build the permuted left environment GLp[l] used by c_apply
void ensure_GLp(Context* ctx, imps_envs* envs, int l);
// identity-channel pushes with distinct above/below tensors (transfermatrix.jl:5-66)
void push_left_id(Context* ctx, int Dl, int d, int Dr, const dcplx* L, const dcplx* above, const dcplx* below,
                  dcplx* out);
void push_right_id(Context* ctx, int Dl, int d, int Dr, const dcplx* R, const dcplx* above, const dcplx* below,
                   dcplx* out);
// Level-resolved pushes: out_q = sum_{(l,q)} push_slice(L_l, W[l,:,q,:], A)
void push_left_levels(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* L, int64_t L_level_stride,
                      int64_t L_ld, const std::vector<std::pair<int, int>>& blocks, int q_count,
                      const std::vector<int>& q_targets, const dcplx* A, dcplx* out, int64_t out_level_stride,
                      int64_t out_ld, bool accumulate);
void push_right_levels(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* R,
                       int64_t R_level_stride, int64_t R_ld, const std::vector<std::pair<int, int>>& blocks,
                       const std::vector<int>& q_targets, const dcplx* A, dcplx* out, int64_t out_level_stride,
                       int64_t out_ld, bool accumulate);
// AC apply with all intermediates in a fixed file-scope device array (noalloc.cu)
void ac_apply_noalloc(Context* ctx, int Dl, int d, int Dr, int m, int n, const cplx* W_host, const dcplx* GL,
                      const dcplx* GR, const dcplx* x, dcplx* y);
size_t noalloc_scratch_bytes();
// Loads the no-alloc array on `device` (current) and caches its address.
void noalloc_prepare(int device);
// W^I (alg 1) / W^II (alg 2) tensor (m-1, d, n-1, d) of the Schur site tensor W (m, d, n, d)
// approximating exp(delta H) (timeevo_mpo.cu; host only).
void timeevompo_site(int m, int d, int n, const cplx* W, cplx delta, int alg, cplx* out);
// Full MPO pushes (transfer_leftenv!/transfer_rightenv!)
void push_mpo_left(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* L, const dcplx* A, dcplx* out);
void push_mpo_right(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* R, const dcplx* A,
                    dcplx* out);

}  // namespace imps
