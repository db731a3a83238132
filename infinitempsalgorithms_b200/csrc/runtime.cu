// Context, transfers, timing and the memory-bound vector kernels (Krylov
// orthogonalisation, norms, axpy, transposes).  Reductions are two-pass and
// deterministic: per-block partials in a fixed order, then one final block.
#include "imps_internal.h"

#include <algorithm>
#include <vector>
#include <cmath>
#include <cstring>

namespace imps {

namespace {
constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 1184;  // 8 x 148 SMs

__device__ __forceinline__ dcplx cmul(dcplx a, dcplx b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ dcplx cmulc(dcplx a, dcplx b) {  // conj(a) * b
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}

int red_blocks(int64_t n) {
  int64_t b = (n + kRedThreads - 1) / kRedThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, kMaxRedBlocks));
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; ++i) r += sh[i];
  }
  __syncthreads();
  return r;
}

__global__ void k_nrm2_partial(int64_t n, const dcplx* __restrict__ x, double* __restrict__ part) {
  __shared__ double sh[kRedThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx v = x[i];
    s = fma(v.x, v.x, fma(v.y, v.y, s));
  }
  double r = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void k_dotc_partial(int64_t n, const dcplx* __restrict__ x, const dcplx* __restrict__ y,
                               double* __restrict__ part) {
  __shared__ double sh[kRedThreads / 32];
  double sr = 0.0, si = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx p = cmulc(x[i], y[i]);
    sr += p.x;
    si += p.y;
  }
  double r = block_sum<kRedThreads>(sr, sh);
  double q = block_sum<kRedThreads>(si, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r;
    part[2 * blockIdx.x + 1] = q;
  }
}

// Sum `ncol` columns of partials (each `nb` long, stride ld) in a fixed order.
__global__ void k_final_sum(int nb, int ncol, const double* __restrict__ part, int64_t ld, double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  for (int c = 0; c < ncol; ++c) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i + ld * c];
    double r = block_sum<kRedThreads>(s, sh);
    if (threadIdx.x == 0) out[c] = r;
  }
}

// One block per column: out[c] = sum_i part[i + ld c] (same order as k_final_sum).
__global__ void k_final_sum_cols(int nb, const double* __restrict__ part, int64_t ld, double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i + ld * c];
  double r = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) out[c] = r;
}

// Projection pass, step 1: partials of h_j = <V_j, w> for a chunk of up to CH
// vectors (columns 2 j0 + 2 j, +1 of `part`) and, when norm_col >= 0, of ||w||^2.
template <int CH>
__global__ void k_proj_dots(int64_t n, int nv, const dcplx* __restrict__ V, int64_t ldv, const dcplx* __restrict__ w,
                            double* __restrict__ part, int64_t ldp, int col0, int norm_col) {
  __shared__ double sh[kRedThreads / 32];
  double ar[CH], ai[CH], nn = 0.0;
#pragma unroll
  for (int j = 0; j < CH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const dcplx wi = w[i];
    nn = fma(wi.x, wi.x, fma(wi.y, wi.y, nn));
#pragma unroll
    for (int j = 0; j < CH; ++j) {
      if (j < nv) {
        const dcplx p = cmulc(V[i + ldv * j], wi);
        ar[j] += p.x;
        ai[j] += p.y;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < CH; ++j) {
    if (j < nv) {
      const double r = block_sum<kRedThreads>(ar[j], sh);
      const double q = block_sum<kRedThreads>(ai[j], sh);
      if (threadIdx.x == 0) {
        part[blockIdx.x + ldp * (col0 + 2 * j)] = r;
        part[blockIdx.x + ldp * (col0 + 2 * j + 1)] = q;
      }
    }
  }
  if (norm_col >= 0) {
    const double r = block_sum<kRedThreads>(nn, sh);
    if (threadIdx.x == 0) part[blockIdx.x + ldp * norm_col] = r;
  }
}

// Projection pass, step 2: w -= sum_j h_j V_j for up to 32 vectors, h read from the
// device (interleaved re/im at hdev[2 j0 ..]); on the last chunk also the partials
// of the new ||w||^2 (one per block) go to `npart`.
__global__ void k_proj_update(int64_t n, int nv, const dcplx* __restrict__ V, int64_t ldv,
                              const double* __restrict__ hdev, dcplx* __restrict__ w, double* __restrict__ npart) {
  __shared__ double2 c[32];
  __shared__ double sh[kRedThreads / 32];
  if (threadIdx.x < nv) c[threadIdx.x] = make_double2(-hdev[2 * threadIdx.x], -hdev[2 * threadIdx.x + 1]);
  __syncthreads();
  double nn = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx acc = w[i];
    for (int j = 0; j < nv; ++j) {
      const dcplx p = cmul(c[j], V[i + ldv * j]);
      acc.x += p.x;
      acc.y += p.y;
    }
    w[i] = acc;
    nn = fma(acc.x, acc.x, fma(acc.y, acc.y, nn));
  }
  if (npart) {
    const double r = block_sum<kRedThreads>(nn, sh);
    if (threadIdx.x == 0) npart[blockIdx.x] = r;
  }
}

// Gram-Schmidt projections against a basis of nv <= NV columns, one kernel per pass.
// The rows are taken in chunks of GS_ROWS.  A GS_STAGES-deep cp.async ring stages each
// chunk of V[chunk, 0:nv] and w[chunk] from HBM into shared memory (coalesced: 64
// consecutive rows per column), so several chunks are in flight per block while the
// current one is used: the pending update w <- w - V h (the column partial sums of a row
// combined through shared memory), then the chunk's contribution to h'_j = <V_j, w> for
// every column, GS_THREADS / NV threads per column.  Few registers per thread.
// Partials: part[blockIdx.x + ldp k], k < 2 nv the dots (re, im), k = 2 nv the norm^2
// of w (after the update).
constexpr int GS_THREADS = 256;
constexpr int GS_ROWS = 64;
constexpr int GS_QP = GS_THREADS / GS_ROWS;
constexpr int GS_STAGES = 3;

template <int NV>
constexpr size_t gs_smem_bytes() {
  return (size_t)GS_STAGES * (NV + 1) * GS_ROWS * sizeof(dcplx);
}

__device__ __forceinline__ void gs_cp16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

template <int NV, bool UPDATE>
__global__ void __launch_bounds__(GS_THREADS) k_gs_pass(int64_t n, int nv, const dcplx* __restrict__ V, int64_t ldv,
                                                       const double* __restrict__ hdev, dcplx* __restrict__ w,
                                                       double* __restrict__ part, int64_t ldp) {
  constexpr int TPC = GS_THREADS / NV;   // threads per column in the dot phase
  constexpr int RPD = GS_ROWS / TPC;     // rows per thread in the dot phase
  constexpr int STAGE = (NV + 1) * GS_ROWS;
  extern __shared__ __align__(16) dcplx gs_sm[];   // [stage][NV + 1][GS_ROWS]: columns, then w
  __shared__ dcplx as[GS_ROWS];
  __shared__ dcplx apart[UPDATE ? GS_QP : 1][GS_ROWS];
  __shared__ dcplx cs[NV];
  __shared__ double nred[GS_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31;
  if (UPDATE && tid < NV)
    cs[tid] = tid < nv ? make_double2(-hdev[2 * tid], -hdev[2 * tid + 1]) : make_double2(0.0, 0.0);
  const int r1 = tid % GS_ROWS, q = tid / GS_ROWS;   // load / update phase: row r1, columns q + GS_QP u
  const int jd = tid / TPC, sd = tid % TPC;          // dot phase: column jd, rows sd + TPC u
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(gs_sm));
  const int64_t nchunks = (n + GS_ROWS - 1) / GS_ROWS;
  auto issue = [&](int stage, int64_t chunk) {
    const int64_t i = chunk * GS_ROWS + r1;
    const bool ok = i < n;
#pragma unroll
    for (int u = 0; u < NV / GS_QP; ++u) {
      const int j = q + GS_QP * u;
      const bool live = ok && j < nv;
      gs_cp16(sbase + 16u * (uint32_t)(stage * STAGE + j * GS_ROWS + r1), live ? (const void*)(V + i + ldv * j) : V,
              live ? 16 : 0);
    }
    if (q == 0) gs_cp16(sbase + 16u * (uint32_t)(stage * STAGE + NV * GS_ROWS + r1), ok ? (const void*)(w + i) : w,
                        ok ? 16 : 0);
  };
  // chunk t of this block is blockIdx.x + t gridDim.x
  int64_t t_issue = 0;
#pragma unroll
  for (int st = 0; st < GS_STAGES - 1; ++st) {
    const int64_t c = blockIdx.x + t_issue * gridDim.x;
    if (c < nchunks) issue(st, c);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    ++t_issue;
  }
  double dre = 0.0, dim = 0.0, nrm = 0.0;
  for (int64_t t = 0;; ++t) {
    const int64_t chunk = blockIdx.x + t * gridDim.x;
    if (chunk >= nchunks) break;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(GS_STAGES - 2) : "memory");
    __syncthreads();
    {
      const int64_t c = blockIdx.x + t_issue * gridDim.x;
      if (c < nchunks) issue((int)(t_issue % GS_STAGES), c);
      asm volatile("cp.async.commit_group;\n" ::: "memory");
      ++t_issue;
    }
    const dcplx* Vs = gs_sm + (t % GS_STAGES) * STAGE;
    const dcplx* ws = Vs + NV * GS_ROWS;
    const int64_t i = chunk * GS_ROWS + r1;
    const dcplx* arow = ws;
    if (UPDATE) {
      double ar = 0.0, ai = 0.0;
#pragma unroll
      for (int u = 0; u < NV / GS_QP; ++u) {
        const int j = q + GS_QP * u;
        const dcplx c = cs[j], v = Vs[j * GS_ROWS + r1];
        ar = fma(c.x, v.x, fma(-c.y, v.y, ar));
        ai = fma(c.x, v.y, fma(c.y, v.x, ai));
      }
      apart[q][r1] = make_double2(ar, ai);
      __syncthreads();
      if (tid < GS_ROWS) {
        dcplx wi = ws[tid];
#pragma unroll
        for (int k = 0; k < GS_QP; ++k) {
          wi.x += apart[k][tid].x;
          wi.y += apart[k][tid].y;
        }
        if (i < n) w[i] = wi;
        as[tid] = wi;
        nrm = fma(wi.x, wi.x, fma(wi.y, wi.y, nrm));
      }
      __syncthreads();
      arow = as;
    } else if (tid < GS_ROWS) {
      const dcplx wi = ws[tid];
      nrm = fma(wi.x, wi.x, fma(wi.y, wi.y, nrm));
    }
    if (jd < nv) {
#pragma unroll
      for (int u = 0; u < RPD; ++u) {
        const int r = sd + TPC * u;
        const dcplx v = Vs[jd * GS_ROWS + r], a = arow[r];
        dre = fma(v.x, a.x, fma(v.y, a.y, dre));
        dim = fma(v.x, a.y, fma(-v.y, a.x, dim));
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
  for (int o = TPC / 2; o >= 1; o >>= 1) {
    dre += __shfl_xor_sync(0xffffffffu, dre, o);
    dim += __shfl_xor_sync(0xffffffffu, dim, o);
  }
  if (sd == 0 && jd < nv) {
    part[blockIdx.x + ldp * (2 * jd)] = dre;
    part[blockIdx.x + ldp * (2 * jd + 1)] = dim;
  }
  for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
  if (lane == 0) nred[tid >> 5] = nrm;
  __syncthreads();
  if (tid == 0) {
    double tsum = 0.0;
    for (int k = 0; k < GS_THREADS / 32; ++k) tsum += nred[k];
    part[blockIdx.x + ldp * (2 * nv)] = tsum;
  }
}

struct CoefPack {
  double2 c[32];
};

__global__ void k_gemv_acc(int64_t n, int nv, const dcplx* __restrict__ V, int64_t ldv, CoefPack coef,
                           dcplx* __restrict__ w, int set) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx acc = set ? make_double2(0.0, 0.0) : w[i];
    for (int j = 0; j < nv; ++j) {
      dcplx p = cmul(coef.c[j], V[i + ldv * j]);
      acc.x += p.x;
      acc.y += p.y;
    }
    w[i] = acc;
  }
}

__global__ void k_scal(int64_t n, double2 a, dcplx* x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = cmul(a, x[i]);
}
__global__ void k_axpby(int64_t n, double2 a, const dcplx* __restrict__ x, double2 b, dcplx* __restrict__ y,
                        int use_b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx v = cmul(a, x[i]);
    if (use_b) {
      dcplx u = cmul(b, y[i]);
      v.x += u.x;
      v.y += u.y;
    }
    y[i] = v;
  }
}
__global__ void k_axpy(int64_t n, double2 a, const dcplx* __restrict__ x, dcplx* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx v = cmul(a, x[i]);
    dcplx u = y[i];
    y[i] = make_double2(u.x + v.x, u.y + v.y);
  }
}
__global__ void k_fill(int64_t n, double2 v, dcplx* x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}
__global__ void k_set_identity(int D, dcplx* X, int64_t ld, double2 diag) {
  int64_t total = (int64_t)D * D;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int a = (int)(t % D), b = (int)(t / D);
    X[a + ld * b] = (a == b) ? diag : make_double2(0.0, 0.0);
  }
}

// 32 x 32 tiled conjugate transpose: Y[j + ldy i] = conj(X[i + ldx j]).
__global__ void k_conj_transpose(int m, int n, const dcplx* __restrict__ X, int64_t ldx, dcplx* __restrict__ Y,
                                 int64_t ldy) {
  __shared__ dcplx tile[32][33];
  int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = i0 + threadIdx.x, j = j0 + r;
    if (i < m && j < n) tile[r][threadIdx.x] = X[i + ldx * j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int j = j0 + threadIdx.x, i = i0 + r;
    if (i < m && j < n) {
      dcplx v = tile[threadIdx.x][r];
      Y[j + ldy * i] = make_double2(v.x, -v.y);
    }
  }
}

// partials of sum_{a,b} L[a,b] V[b,a]
__global__ void k_trace_prod_partial(int D, const dcplx* __restrict__ L, int64_t ldl, const dcplx* __restrict__ V,
                                     int64_t ldv, double* __restrict__ part) {
  __shared__ double sh[kRedThreads / 32];
  double sr = 0.0, si = 0.0;
  int64_t total = (int64_t)D * D;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int a = (int)(t % D), b = (int)(t / D);
    dcplx p = cmul(L[a + ldl * b], V[b + ldv * a]);
    sr += p.x;
    si += p.y;
  }
  double r = block_sum<kRedThreads>(sr, sh);
  double q = block_sum<kRedThreads>(si, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r;
    part[2 * blockIdx.x + 1] = q;
  }
}

__global__ void k_copy2d(int rows, int cols, const dcplx* __restrict__ X, int64_t ldx, dcplx* __restrict__ Y,
                         int64_t ldy, int add) {
  int64_t total = (int64_t)rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t % rows), c = (int)(t / rows);
    dcplx v = X[r + ldx * c];
    if (add) {
      dcplx u = Y[r + ldy * c];
      v.x += u.x;
      v.y += u.y;
    }
    Y[r + ldy * c] = v;
  }
}

__global__ void k_add_diag(int D, dcplx* X, int64_t ld, double2 v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D; i += gridDim.x * blockDim.x) {
    dcplx u = X[i + ld * i];
    X[i + ld * i] = make_double2(u.x + v.x, u.y + v.y);
  }
}
__global__ void k_fill2d(int rows, int cols, dcplx* Y, int64_t ldy, double2 v) {
  int64_t total = (int64_t)rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t % rows), c = (int)(t / rows);
    Y[r + ldy * c] = v;
  }
}

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

inline double2 d2(cplx z) { return make_double2(z.real(), z.imag()); }

void check_launch(Context* ctx) {
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("kernel launch: ") + cudaGetErrorString(e));
}

}  // namespace

double* Context::pinned(size_t bytes) {
  if (bytes > host_pinned_bytes) {
    if (host_pinned) cudaFreeHost(host_pinned);
    host_pinned = nullptr;
    size_t b = std::max<size_t>(bytes, 1 << 16);
    IMPS_CUDA(cudaMallocHost((void**)&host_pinned, b));
    host_pinned_bytes = b;
  }
  return host_pinned;
}

static cudaEvent_t pooled_event(Context* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

ScopedTimer::ScopedTimer(Context* c, const char* n, double f) : ctx(c), flops(f) {
  if (!ctx->profile) return;
  if (!ctx->profile_only.empty() && ctx->profile_only.count(n) == 0) return;
  name = n;
  if (ctx->prof_tag && ctx->prof_tag[0]) name = name + "@" + ctx->prof_tag;
  e0 = pooled_event(ctx);
  e1 = pooled_event(ctx);
  cudaEventRecord(e0, ctx->stream);
}
ScopedTimer::~ScopedTimer() {
  if (e0) {
    cudaEventRecord(e1, ctx->stream);
    ctx->pending.push_back({name, {e0, e1}});
    ctx->pending_flops.push_back(flops);
  }
}

// The error flag rides along with a synchronisation that happens anyway.
static void err_copy(Context* ctx) {
  if (ctx->err_armed)
    IMPS_CUDA(cudaMemcpyAsync(ctx->err_host, ctx->err_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
}
static void err_after_sync(Context* ctx) {
  if (!ctx->err_armed) return;
  ctx->err_armed = false;
  if (ctx->err_host[0] != 0) {
    ctx->err_host[0] = 0;
    IMPS_CUDA(cudaMemsetAsync(ctx->err_dev, 0, sizeof(int), ctx->stream));
    throw Error(IMPS_TIMEOUT, "a bounded device wait of the split GEMM pipeline ran out");
  }
}
void check_device_errors(Context* ctx) {
  if (!ctx->err_armed) return;
  err_copy(ctx);
  IMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  err_after_sync(ctx);
}

void upload(Context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  IMPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  err_copy(ctx);
  IMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  err_after_sync(ctx);
}
void download(Context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  IMPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  err_copy(ctx);
  IMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  err_after_sync(ctx);
}

void zcopy(Context* ctx, int64_t n, const dcplx* x, dcplx* y) {
  if (n <= 0 || x == y) return;
  IMPS_CUDA(cudaMemcpyAsync(y, x, n * sizeof(dcplx), cudaMemcpyDeviceToDevice, ctx->stream));
}
void zscal(Context* ctx, int64_t n, cplx a, dcplx* x) {
  if (n <= 0) return;
  k_scal<<<grid_for(n), 256, 0, ctx->stream>>>(n, d2(a), x);
  check_launch(ctx);
}
void zaxpy(Context* ctx, int64_t n, cplx a, const dcplx* x, dcplx* y) {
  if (n <= 0) return;
  k_axpy<<<grid_for(n), 256, 0, ctx->stream>>>(n, d2(a), x, y);
  check_launch(ctx);
}
void zaxpby(Context* ctx, int64_t n, cplx a, const dcplx* x, cplx b, dcplx* y) {
  if (n <= 0) return;
  k_axpby<<<grid_for(n), 256, 0, ctx->stream>>>(n, d2(a), x, d2(b), y, b != cplx(0.0, 0.0));
  check_launch(ctx);
}
void zfill(Context* ctx, int64_t n, cplx v, dcplx* x) {
  if (n <= 0) return;
  k_fill<<<grid_for(n), 256, 0, ctx->stream>>>(n, d2(v), x);
  check_launch(ctx);
}
void zset_identity(Context* ctx, int D, dcplx* X, int64_t ld, cplx diag) {
  if (D <= 0) return;
  k_set_identity<<<grid_for((int64_t)D * D), 256, 0, ctx->stream>>>(D, X, ld, d2(diag));
  check_launch(ctx);
}

double dznrm2(Context* ctx, int64_t n, const dcplx* x) {
  if (n <= 0) return 0.0;
  int nb = red_blocks(n);
  DevBuf& red = ctx->buf("red_part", (size_t)(nb + 8) * sizeof(double));
  DevBuf& out = ctx->buf("red_out", 64 * sizeof(double));
  ScopedTimer t(ctx, "blas1", (double)n * 16);
  k_nrm2_partial<<<nb, kRedThreads, 0, ctx->stream>>>(n, x, red.d());
  check_launch(ctx);
  k_final_sum<<<1, kRedThreads, 0, ctx->stream>>>(nb, 1, red.d(), nb, out.d());
  check_launch(ctx);
  double h;
  download(ctx, &h, out.d(), sizeof(double));
  return std::sqrt(h);
}

cplx zdotc(Context* ctx, int64_t n, const dcplx* x, const dcplx* y) {
  if (n <= 0) return cplx(0.0, 0.0);
  int nb = red_blocks(n);
  DevBuf& red = ctx->buf("red_part", (size_t)(2 * nb + 8) * sizeof(double));
  DevBuf& out = ctx->buf("red_out", 64 * sizeof(double));
  ScopedTimer t(ctx, "blas1", (double)n * 32);
  (void)out;
  k_dotc_partial<<<nb, kRedThreads, 0, ctx->stream>>>(n, x, y, red.d());
  check_launch(ctx);
  double h[2];
  {
    // per-block (re, im) partials summed on the host in block order (deterministic)
    std::vector<double> p(2 * nb);
    download(ctx, p.data(), red.d(), p.size() * sizeof(double));
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < nb; ++i) { sr += p[2 * i]; si += p[2 * i + 1]; }
    h[0] = sr;
    h[1] = si;
  }
  return cplx(h[0], h[1]);
}

static void gemv_common(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, const cplx* coef, dcplx* w,
                        int set) {
  ScopedTimer t(ctx, "orth", (double)n * 16 * (nv + 2));
  int done = 0;
  bool first = true;
  while (done < nv || (first && set)) {
    int cnt = std::min(32, nv - done);
    CoefPack p;
    for (int j = 0; j < cnt; ++j) p.c[j] = d2(coef[done + j]);
    k_gemv_acc<<<grid_for(n), 256, 0, ctx->stream>>>(n, cnt, V + ldv * (int64_t)done, ldv, p, w,
                                                      (first && set) ? 1 : 0);
    check_launch(ctx);
    done += cnt;
    first = false;
    if (cnt == 0) break;
  }
}

void zgemv_acc(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, const cplx* coef, dcplx* w) {
  if (nv <= 0) return;
  gemv_common(ctx, n, nv, V, ldv, coef, w, 0);
}
void zgemv_set(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, const cplx* coef, dcplx* y) {
  gemv_common(ctx, n, nv, V, ldv, coef, y, 1);
}

double proj_pass(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, dcplx* w, cplx* h_host,
                 double* nw_old2) {
  // columns of the partials: 2 nv dot columns, then ||w_old||^2, then ||w_new||^2
  const int nb = std::min(red_blocks(n), 592);
  constexpr int CH = 8;
  const int ncol = 2 * nv + 2;
  DevBuf& red = ctx->buf("proj_part", (size_t)nb * ncol * sizeof(double));
  DevBuf& out = ctx->buf("proj_out", (size_t)ncol * sizeof(double));
  ScopedTimer t(ctx, "orth", (double)n * 16 * (2 * nv + 3));
  const int norm_col = nw_old2 ? 2 * nv : -1;
  if (nv == 0 && nw_old2) {
    k_proj_dots<CH><<<nb, kRedThreads, 0, ctx->stream>>>(n, 0, V, ldv, w, red.d(), nb, 0, norm_col);
    check_launch(ctx);
  }
  for (int c0 = 0; c0 < nv; c0 += CH) {
    const int nvc = std::min(CH, nv - c0);
    k_proj_dots<CH><<<nb, kRedThreads, 0, ctx->stream>>>(n, nvc, V + ldv * (int64_t)c0, ldv, w, red.d(), nb, 2 * c0,
                                                         c0 == 0 ? norm_col : -1);
    check_launch(ctx);
  }
  const int ndots = 2 * nv + (nw_old2 ? 1 : 0);
  if (ndots > 0) {
    k_final_sum_cols<<<ndots, kRedThreads, 0, ctx->stream>>>(nb, red.d(), nb, out.d());
    check_launch(ctx);
  }
  for (int c0 = 0; c0 < nv || (nv == 0 && c0 == 0); c0 += 32) {
    const int cnt = std::min(32, nv - c0);
    const bool last = c0 + 32 >= nv;
    k_proj_update<<<nb, kRedThreads, 0, ctx->stream>>>(n, cnt, V + ldv * (int64_t)c0, ldv, out.d() + 2 * c0, w,
                                                       last ? red.d() + (size_t)nb * (2 * nv + 1) : nullptr);
    check_launch(ctx);
    if (nv == 0) break;
  }
  k_final_sum_cols<<<1, kRedThreads, 0, ctx->stream>>>(nb, red.d() + (size_t)nb * (2 * nv + 1), nb,
                                                       out.d() + 2 * nv + 1);
  check_launch(ctx);
  std::vector<double> hv(ncol);
  download(ctx, hv.data(), out.d(), hv.size() * sizeof(double));
  for (int j = 0; j < nv; ++j) h_host[j] = cplx(hv[2 * j], hv[2 * j + 1]);
  if (nw_old2) *nw_old2 = hv[2 * nv];
  return hv[2 * nv + 1];
}

namespace {
template <int NV>
int gs_blocks_for(int64_t n) {
  // resident blocks per SM by shared memory (the ring plus the static arrays), at most 8
  const int per_sm = std::max(1, std::min(8, (int)((220 * 1024) / (gs_smem_bytes<NV>() + 8 * 1024))));
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + GS_ROWS - 1) / GS_ROWS, (int64_t)148 * per_sm));
}
template <int NV, bool UPDATE>
void launch_gs_kernel(Context* ctx, int nb, int64_t n, int nv, const dcplx* V, int64_t ldv, const double* hdev,
                      dcplx* w, double* part, int64_t ldp) {
  static DeviceOnce attr;
  attr.run(ctx->device, [] {
    IMPS_CUDA(cudaFuncSetAttribute(k_gs_pass<NV, UPDATE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)gs_smem_bytes<NV>()));
  });
  k_gs_pass<NV, UPDATE><<<nb, GS_THREADS, gs_smem_bytes<NV>(), ctx->stream>>>(n, nv, V, ldv, hdev, w, part, ldp);
}
int gs_pass_blocks(int64_t n, int nv) {
  return nv <= 8 ? gs_blocks_for<8>(n) : nv <= 16 ? gs_blocks_for<16>(n) : gs_blocks_for<32>(n);
}
void gs_pass(Context* ctx, bool update, int64_t n, int nv, const dcplx* V, int64_t ldv, const double* hdev, dcplx* w,
             double* part, int64_t ldp, double* out) {
  const int nb = gs_pass_blocks(n, nv);
  if (nv <= 8) {
    if (update) launch_gs_kernel<8, true>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
    else launch_gs_kernel<8, false>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
  } else if (nv <= 16) {
    if (update) launch_gs_kernel<16, true>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
    else launch_gs_kernel<16, false>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
  } else {
    if (update) launch_gs_kernel<32, true>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
    else launch_gs_kernel<32, false>(ctx, nb, n, nv, V, ldv, hdev, w, part, ldp);
  }
  check_launch(ctx);
  k_final_sum_cols<<<2 * nv + 1, kRedThreads, 0, ctx->stream>>>(nb, part, ldp, out);
  check_launch(ctx);
}
const char* kNonFinite =
    "non-finite value (NaN or Inf) in the Krylov iteration: the operator or the start vector holds one";
}  // namespace

double gs_project(Context* ctx, int64_t n, int nv, const dcplx* V, int64_t ldv, dcplx* w, std::vector<cplx>& h) {
  h.assign(nv, cplx(0.0, 0.0));
  if (nv <= 0) {
    const double nw = dznrm2(ctx, n, w);
    IMPS_REQUIRE(std::isfinite(nw), IMPS_INVALID_ARG, kNonFinite);
    return nw;
  }
  if (nv > 32) {
    // wide bases: the chunked two-kernel projection
    std::vector<cplx> h1(nv);
    double nw0 = 0.0;
    double nw1 = proj_pass(ctx, n, nv, V, ldv, w, h1.data(), &nw0);
    IMPS_REQUIRE(std::isfinite(nw0) && std::isfinite(nw1), IMPS_INVALID_ARG, kNonFinite);
    for (int j = 0; j < nv; ++j) h[j] += h1[j];
    for (int pass = 1; pass < 3 && nw1 < 0.5 * nw0; ++pass) {
      nw0 = nw1;
      nw1 = proj_pass(ctx, n, nv, V, ldv, w, h1.data(), nullptr);
      for (int j = 0; j < nv; ++j) h[j] += h1[j];
    }
    return std::sqrt(std::max(nw1, 0.0));
  }
  const int nb = gs_pass_blocks(n, nv);
  const int ncol = 2 * nv + 1;
  DevBuf& part = ctx->buf("gs_part", (size_t)nb * ncol * sizeof(double));
  DevBuf& outb = ctx->buf("gs_out", (size_t)3 * ncol * sizeof(double));
  double* out[3] = {outb.d(), outb.d() + ncol, outb.d() + 2 * ncol};
  ScopedTimer t(ctx, "orth", (double)n * 16 * (nv + 1));
  // projection 1 (dots of w), then its update fused with the dots of projection 2
  gs_pass(ctx, false, n, nv, V, ldv, nullptr, w, part.d(), nb, out[0]);
  gs_pass(ctx, true, n, nv, V, ldv, out[0], w, part.d(), nb, out[1]);
  std::vector<double> hv(2 * ncol);
  download(ctx, hv.data(), out[0], hv.size() * sizeof(double));
  double nw0 = hv[2 * nv], nw1 = hv[ncol + 2 * nv];
  IMPS_REQUIRE(std::isfinite(nw0) && std::isfinite(nw1), IMPS_INVALID_ARG, kNonFinite);
  for (int j = 0; j < nv; ++j) h[j] = cplx(hv[2 * j], hv[2 * j + 1]);
  // iterative refinement (KrylovKit's ClassicalGramSchmidtIR, eta = 1/sqrt(2)): apply the
  // pending projection while the last one shrank ||w|| below eta of its previous value,
  // at most three projections in all
  int cur = 1;
  std::vector<double> hn(hv.begin() + ncol, hv.end());
  for (int pass = 1; pass < 3 && nw1 < 0.5 * nw0; ++pass) {
    const int nxt = cur == 1 ? 2 : 1;
    gs_pass(ctx, true, n, nv, V, ldv, out[cur], w, part.d(), nb, out[nxt]);
    for (int j = 0; j < nv; ++j) h[j] += cplx(hn[2 * j], hn[2 * j + 1]);
    download(ctx, hn.data(), out[nxt], ncol * sizeof(double));
    nw0 = nw1;
    nw1 = hn[2 * nv];
    IMPS_REQUIRE(std::isfinite(nw1), IMPS_INVALID_ARG, kNonFinite);
    cur = nxt;
  }
  return std::sqrt(std::max(nw1, 0.0));
}

void zconj_transpose(Context* ctx, int m, int n, const dcplx* X, int64_t ldx, dcplx* Y, int64_t ldy) {
  if (m <= 0 || n <= 0) return;
  dim3 grid((m + 31) / 32, (n + 31) / 32), block(32, 8);
  ScopedTimer t(ctx, "permute", (double)m * n * 32);
  k_conj_transpose<<<grid, block, 0, ctx->stream>>>(m, n, X, ldx, Y, ldy);
  check_launch(ctx);
}

cplx ztrace_prod(Context* ctx, int D, const dcplx* L, int64_t ldl, const dcplx* V, int64_t ldv) {
  int64_t n = (int64_t)D * D;
  int nb = red_blocks(n);
  DevBuf& red = ctx->buf("red_part", (size_t)(2 * nb + 8) * sizeof(double));
  k_trace_prod_partial<<<nb, kRedThreads, 0, ctx->stream>>>(D, L, ldl, V, ldv, red.d());
  check_launch(ctx);
  std::vector<double> p(2 * nb);
  download(ctx, p.data(), red.d(), p.size() * sizeof(double));
  double sr = 0.0, si = 0.0;
  for (int i = 0; i < nb; ++i) { sr += p[2 * i]; si += p[2 * i + 1]; }
  return cplx(sr, si);
}

void zcopy2d(Context* ctx, int rows, int cols, const dcplx* X, int64_t ldx, dcplx* Y, int64_t ldy) {
  if (rows <= 0 || cols <= 0) return;
  k_copy2d<<<grid_for((int64_t)rows * cols), 256, 0, ctx->stream>>>(rows, cols, X, ldx, Y, ldy, 0);
  check_launch(ctx);
}

void zadd_diag(Context* ctx, int D, dcplx* X, int64_t ld, cplx v) {
  if (D <= 0) return;
  k_add_diag<<<grid_for(D), 256, 0, ctx->stream>>>(D, X, ld, d2(v));
  check_launch(ctx);
}
void zfill2d(Context* ctx, int rows, int cols, cplx v, dcplx* Y, int64_t ldy) {
  if (rows <= 0 || cols <= 0) return;
  k_fill2d<<<grid_for((int64_t)rows * cols), 256, 0, ctx->stream>>>(rows, cols, Y, ldy, d2(v));
  check_launch(ctx);
}

}  // namespace imps
