// FP64 complex GEMM engine (the plain method).  Column-major, op(A) in
// {N, T, C}, op(B) in {N, T, C}, strided batches.
//
// Tiling: 64 x 64 complex output tile per CTA of 256 threads, 4 x 4 complex
// accumulators per thread (strided by 16 so shared-memory reads of a warp hit
// consecutive addresses), K tile of 8 staged through shared memory with a
// register prefetch of the next tile.  Each complex MAC is 4 DFMA.
#include "imps_internal.h"
#include "split_gemm.h"

#include <cmath>

namespace imps {
namespace {

constexpr int BM = 64, BN = 64, BK = 8, NT = 256;

__device__ __forceinline__ double2 conj2(double2 v) { return make_double2(v.x, -v.y); }

template <int OPA, int OPB, bool BETA>
__global__ void __launch_bounds__(NT, 2)
    k_zgemm(int M, int N, int K, double2 alpha, const double2* __restrict__ A, int64_t lda, int64_t sA,
            const double2* __restrict__ B, int64_t ldb, int64_t sB, double2 beta, double2* __restrict__ C,
            int64_t ldc, int64_t sC) {
  __shared__ double2 As[2][BK][BM + 1];
  __shared__ double2 Bs[2][BK][BN + 1];
  const int bz = blockIdx.z;
  A += sA * bz;
  B += sB * bz;
  C += sC * bz;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;

  // global-load coordinates: 2 A elements and 2 B elements per thread per K tile
  int am[2], ak[2], bk[2], bn[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    if (OPA == OP_N) { am[r] = tid & 63; ak[r] = (tid >> 6) + 4 * r; }
    else { ak[r] = tid & 7; am[r] = (tid >> 3) + 32 * r; }
    if (OPB == OP_N) { bk[r] = tid & 7; bn[r] = (tid >> 3) + 32 * r; }
    else { bn[r] = tid & 63; bk[r] = (tid >> 6) + 4 * r; }
  }
  double2 ra[2], rb[2];
  auto load_tile = [&](int k0) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int gm = m0 + am[r], gk = k0 + ak[r];
      double2 v = make_double2(0.0, 0.0);
      if (gm < M && gk < K) {
        v = (OPA == OP_N) ? A[gm + lda * gk] : A[gk + lda * gm];
        if (OPA == OP_C) v = conj2(v);
      }
      ra[r] = v;
      int gn = n0 + bn[r], gk2 = k0 + bk[r];
      double2 u = make_double2(0.0, 0.0);
      if (gn < N && gk2 < K) {
        u = (OPB == OP_N) ? B[gk2 + ldb * gn] : B[gn + ldb * gk2];
        if (OPB == OP_C) u = conj2(u);
      }
      rb[r] = u;
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      As[buf][ak[r]][am[r]] = ra[r];
      Bs[buf][bk[r]][bn[r]] = rb[r];
    }
  };

  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);

  const int ktiles = (K + BK - 1) / BK;
  load_tile(0);
  store_tile(0);
  __syncthreads();
  for (int kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) load_tile((kt + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
    if (kt + 1 < ktiles) {
      store_tile(buf ^ 1);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + tx + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + ty + 16 * j;
      if (gn >= N) continue;
      double2 v = acc[i][j];
      double2 o = make_double2(alpha.x * v.x - alpha.y * v.y, alpha.x * v.y + alpha.y * v.x);
      if (BETA) {
        double2 c = C[gm + ldc * gn];
        o.x += beta.x * c.x - beta.y * c.y;
        o.y += beta.x * c.y + beta.y * c.x;
      }
      C[gm + ldc * gn] = o;
    }
  }
}

template <int OPA, int OPB>
void launch(Context* ctx, int M, int N, int K, double2 alpha, const dcplx* A, int64_t lda, int64_t sA,
            const dcplx* B, int64_t ldb, int64_t sB, double2 beta, dcplx* C, int64_t ldc, int64_t sC, int batch,
            bool use_beta) {
  dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, batch);
  if (use_beta)
    k_zgemm<OPA, OPB, true><<<grid, NT, 0, ctx->stream>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
  else
    k_zgemm<OPA, OPB, false><<<grid, NT, 0, ctx->stream>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
}

}  // namespace

void zgemm_fp64(Context* ctx, Op opA, Op opB, int M, int N, int K, cplx alpha, const dcplx* A, int64_t lda,
                int64_t strideA, const dcplx* B, int64_t ldb, int64_t strideB, cplx beta, dcplx* C, int64_t ldc,
                int64_t strideC, int batch) {
  if (M <= 0 || N <= 0 || batch <= 0) return;
  IMPS_REQUIRE(batch <= 65535, IMPS_INVALID_ARG, "zgemm: batch too large");
  IMPS_REQUIRE((N + BN - 1) / BN <= 65535, IMPS_INVALID_ARG, "zgemm: N too large");
  if (K <= 0) {
    // C = beta C
    for (int b = 0; b < batch; ++b) {
      for (int n = 0; n < N; ++n) {
        if (beta == cplx(0.0, 0.0)) zfill(ctx, M, cplx(0.0, 0.0), C + strideC * b + ldc * n);
        else zscal(ctx, M, beta, C + strideC * b + ldc * n);
      }
    }
    return;
  }
  double2 a = make_double2(alpha.real(), alpha.imag()), bt = make_double2(beta.real(), beta.imag());
  bool use_beta = beta != cplx(0.0, 0.0);
  ScopedTimer t(ctx, "zgemm_fp64", 8.0 * M * (double)N * K * batch);
  ctx->n_gemm++;
  ctx->n_kernels++;
#define IMPS_GEMM_CASE(OA, OB)                                                                              \
  if (opA == OA && opB == OB) {                                                                             \
    launch<OA, OB>(ctx, M, N, K, a, A, lda, strideA, B, ldb, strideB, bt, C, ldc, strideC, batch, use_beta); \
  }
  IMPS_GEMM_CASE(OP_N, OP_N)
  IMPS_GEMM_CASE(OP_N, OP_T)
  IMPS_GEMM_CASE(OP_N, OP_C)
  IMPS_GEMM_CASE(OP_T, OP_N)
  IMPS_GEMM_CASE(OP_C, OP_N)
  IMPS_GEMM_CASE(OP_T, OP_T)
  IMPS_GEMM_CASE(OP_C, OP_C)
  IMPS_GEMM_CASE(OP_T, OP_C)
  IMPS_GEMM_CASE(OP_C, OP_T)
#undef IMPS_GEMM_CASE
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("zgemm launch: ") + cudaGetErrorString(e));
}

int slices_for_tol(double tol) {
  // the truncation error of s slices is below 2^-7s of the row/column scales; keep
  // a 2^4 margin for the sum over K and the spread inside a row
  if (!(tol > 0)) return 7;
  int s = (int)std::ceil((-std::log2(tol) + 4.0) / 7.0);
  return std::min(7, std::max(2, s));
}

int active_slices(const Context* ctx) {
  if (ctx->precision != PREC_SPLIT_I8 || ctx->force_fp64 > 0) return 0;
  const int s = ctx->adaptive_slices ? slices_for_tol(ctx->split_tol) : ctx->nslices;
  return s >= 7 ? 0 : s;  // seven slices cost about as much as the FP64 engine
}

double split_floor(const Context* ctx) {
  const int s = active_slices(ctx);
  return s == 0 ? 0.0 : 16.0 * std::ldexp(1.0, -7 * s);
}

static std::shared_ptr<SplitOperand> get_split(Context* ctx, int side, Op op, int rows, int K, const dcplx* X,
                                               int64_t ld, int s) {
  const bool constant = ctx->const_ptrs.count(X) > 0;
  SplitKey key{X, side, (int)op, rows, K, ld, s};
  if (constant) {
    auto it = ctx->split_cache.find(key);
    if (it != ctx->split_cache.end()) {
      ctx->split_cache_hits++;
      return it->second;
    }
  }
  std::shared_ptr<SplitOperand> S;
  if (constant) {
    S = std::make_shared<SplitOperand>();
  } else {
    // transient operand: reuse one scratch object per side of this context
    if (!ctx->split_scratch[side]) ctx->split_scratch[side] = std::make_shared<SplitOperand>();
    S = ctx->split_scratch[side];
  }
  if (side == 0) split_operand_a(ctx, *S, op, rows, K, X, ld, s);
  else split_operand_b(ctx, *S, op, K, rows, X, ld, s);
  if (constant) ctx->split_cache[key] = S;
  return S;
}

void zgemm(Context* ctx, Op opA, Op opB, int M, int N, int K, cplx alpha, const dcplx* A, int64_t lda,
           int64_t strideA, const dcplx* B, int64_t ldb, int64_t strideB, cplx beta, dcplx* C, int64_t ldc,
           int64_t strideC, int batch, bool allow_split) {
  ctx->gemm_flops += 8.0 * (double)M * (double)N * (double)K * (double)batch;
  const int s = active_slices(ctx);
  const bool split = s > 0 && allow_split && opA != OP_T && opB != OP_T && alpha.imag() == 0.0 &&
                     (beta == cplx(0.0, 0.0) || beta == cplx(1.0, 0.0)) && M >= 64 && N >= 64 && K >= 32 &&
                     (double)M * N * K >= 33554432.0;
  if (!split) {
    zgemm_fp64(ctx, opA, opB, M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, batch);
    return;
  }
  for (int b = 0; b < batch; ++b) {
    const dcplx* Ab = A + strideA * b;
    const dcplx* Bb = B + strideB * b;
    auto SA = get_split(ctx, 0, opA, M, K, Ab, lda, s);
    auto SB = get_split(ctx, 1, opB, N, K, Bb, ldb, s);
    ctx->split_calls++;
    split_gemm(ctx, *SA, *SB, s, alpha.real(), beta == cplx(1.0, 0.0), C + strideC * b, ldc);
  }
}

}  // namespace imps
