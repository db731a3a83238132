// FP64 complex GEMM engine (the plain method).  Column-major, op(A) in
// {N, T, C}, op(B) in {N, T, C}, strided batches.
//
// Tiling: 64 x 64 complex output tile per CTA of 256 threads, 4 x 4 complex
// accumulators per thread (strided by 16 so shared-memory reads of a warp hit
// consecutive addresses), K tile of 8 staged through shared memory with a
// register prefetch of the next tile.  Each complex MAC is 4 DFMA.
#include "imps_internal.h"
#include "split_gemm.h"

#include <atomic>
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

// ---------------------------------------------------------------------------
// FP64 tensor-core variant: mma.sync m8n8k4 f64 (DMMA).  128 x 64 complex output
// tile per CTA of 8 warps (4 x 2 warps of 32 x 32), K stage of 16 complex, a
// 3-stage cp.async ring (zero-filled at the matrix edges).  A complex product is
// four real DMMAs per 8 x 8 block: re += ar br - ai bi, im += ar bi + ai br; the
// conjugate of an operand only flips the sign of its imaginary fragment.
// Shared tiles are k-major rows of double2 with one element of padding.
// ---------------------------------------------------------------------------
// Tile shapes of the DMMA engine: TM = 128 (8 warps, one CTA per SM by registers and
// shared memory) for large grids; TM = 64 (4 warps, two CTAs per SM) for grids that would
// not fill the SMs twice over with 128-row tiles (the skinny products of the blocked QR).
namespace dm {
constexpr int BN = 64, BK = 16, STAGES = 3;
template <int TM>
struct Tile {
  static constexpr int BM = TM, NT = 2 * TM, WM = TM / 32;
  static constexpr int LDA = BM + 1, LDB = BN + 1;
  static constexpr int A_ELEMS = BK * LDA, B_ELEMS = BK * LDB;
  static constexpr int SMEM = STAGES * (A_ELEMS + B_ELEMS) * 16;
};
}  // namespace dm

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int OPA, int OPB, bool BETA, int TM>
__global__ void __launch_bounds__(2 * TM, 128 / TM)
    k_zgemm_dmma(int M, int N, int K, double2 alpha, const double2* __restrict__ A, int64_t lda, int64_t sA,
                 const double2* __restrict__ B, int64_t ldb, int64_t sB, double2 beta, double2* __restrict__ C,
                 int64_t ldc, int64_t sC) {
  using T = dm::Tile<TM>;
  extern __shared__ __align__(16) double2 smem_dm[];
  double2* As = smem_dm;                             // [STAGES][BK][LDA]
  double2* Bs = smem_dm + dm::STAGES * T::A_ELEMS;   // [STAGES][BK][LDB]
  const int bz = blockIdx.z;
  A += sA * bz;
  B += sB * bz;
  C += sC * bz;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % T::WM, wn = warp / T::WM;  // warp tile origin (32 * wm, 32 * wn)
  const int m0 = blockIdx.x * T::BM, n0 = blockIdx.y * dm::BN;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dm));

  auto issue = [&](int stage, int k0) {
    // A tile: BM x BK complex, 8 per thread (NT = 2 BM)
    static_assert(dm::BN == 64 && dm::BK == 16 && (TM == 64 || TM == 128), "load mapping assumes these tiles");
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      int m, k;
      if (OPA == OP_N) { m = tid & (TM - 1); k = (tid / TM) + 2 * r; }
      else { k = tid & 15; m = (tid >> 4) + (T::NT / 16) * r; }
      const int gm = m0 + m, gk = k0 + k;
      const bool ok = gm < M && gk < K;
      const double2* src = ok ? ((OPA == OP_N) ? A + gm + lda * (int64_t)gk : A + gk + lda * (int64_t)gm) : A;
      cp_async16(sbase + 16u * (stage * T::A_ELEMS + k * T::LDA + m), src, ok ? 16 : 0);
    }
    // B tile: BK x BN complex, 1024 / NT per thread
#pragma unroll
    for (int r = 0; r < 1024 / T::NT; ++r) {
      int n, k;
      if (OPB == OP_N) { k = tid & 15; n = (tid >> 4) + (T::NT / 16) * r; }
      else { n = tid & 63; k = (tid >> 6) + (T::NT / 64) * r; }
      const int gn = n0 + n, gk = k0 + k;
      const bool ok = gn < N && gk < K;
      const double2* src = ok ? ((OPB == OP_N) ? B + gk + ldb * (int64_t)gn : B + gn + ldb * (int64_t)gk) : B;
      cp_async16(sbase + 16u * (dm::STAGES * T::A_ELEMS + stage * T::B_ELEMS + k * T::LDB + n), src, ok ? 16 : 0);
    }
  };

  double cre[4][4][2], cim[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0;

  const int ktiles = (K + dm::BK - 1) / dm::BK;
#pragma unroll
  for (int st = 0; st < dm::STAGES - 1; ++st) {
    if (st < ktiles) issue(st, st * dm::BK);
    cp_async_commit();
  }
  const int fr = lane >> 2, fk = lane & 3;  // fragment row/col (A: row m, col k; B: col n, row k)
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<dm::STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + dm::STAGES - 1;
      if (nk < ktiles) issue(nk % dm::STAGES, nk * dm::BK);
      cp_async_commit();
    }
    const double2* as = As + (kt % dm::STAGES) * T::A_ELEMS;
    const double2* bs = Bs + (kt % dm::STAGES) * T::B_ELEMS;
#pragma unroll
    for (int kb = 0; kb < dm::BK; kb += 4) {
      double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v = as[(kb + fk) * T::LDA + 32 * wm + 8 * i + fr];
        ar[i] = v.x;
        ai[i] = (OPA == OP_C) ? -v.y : v.y;
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 v = bs[(kb + fk) * T::LDB + 32 * wn + 8 * j + fr];
        br[j] = v.x;
        bi[j] = (OPB == OP_C) ? -v.y : v.y;
      }
      // the two updates of one accumulator are 32 MMAs apart
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(cre[i][j][0], cre[i][j][1], ar[i], br[j]);
          dmma(cim[i][j][0], cim[i][j][1], ar[i], bi[j]);
        }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(cre[i][j][0], cre[i][j][1], nai[i], bi[j]);
          dmma(cim[i][j][0], cim[i][j][1], ai[i], br[j]);
        }
    }
  }
  cp_async_wait<0>();
  // D fragment: row = lane >> 2, cols 2 (lane & 3) + {0, 1} of each 8 x 8 block
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + 32 * wm + 8 * i + fr;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int gn = n0 + 32 * wn + 8 * j + 2 * fk + e;
        if (gn >= N) continue;
        const double vr = cre[i][j][e], vi = cim[i][j][e];
        double2 o = make_double2(alpha.x * vr - alpha.y * vi, alpha.x * vi + alpha.y * vr);
        if (BETA) {
          const double2 c = C[gm + ldc * (int64_t)gn];
          o.x += beta.x * c.x - beta.y * c.y;
          o.y += beta.x * c.y + beta.y * c.x;
        }
        C[gm + ldc * (int64_t)gn] = o;
      }
    }
  }
}

template <int OPA, int OPB, int TM>
void launch_dmma(Context* ctx, int M, int N, int K, double2 alpha, const dcplx* A, int64_t lda, int64_t sA,
                 const dcplx* B, int64_t ldb, int64_t sB, double2 beta, dcplx* C, int64_t ldc, int64_t sC, int batch,
                 bool use_beta) {
  using T = dm::Tile<TM>;
  // the dynamic shared-memory opt-in is per device and per kernel instance; setting it
  // twice (two host threads racing here) is harmless
  static std::atomic<uint64_t> attr_set[2];
  auto kern = use_beta ? k_zgemm_dmma<OPA, OPB, true, TM> : k_zgemm_dmma<OPA, OPB, false, TM>;
  const uint64_t bit = 1ull << (ctx->device & 63);
  std::atomic<uint64_t>& done = attr_set[use_beta ? 1 : 0];
  if (!(done.load() & bit)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, T::SMEM);
    if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("zgemm smem opt-in: ") + cudaGetErrorString(e));
    done.fetch_or(bit);
  }
  dim3 grid((M + T::BM - 1) / T::BM, (N + dm::BN - 1) / dm::BN, batch);
  kern<<<grid, T::NT, T::SMEM, ctx->stream>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
}

template <int OPA, int OPB>
void launch(Context* ctx, int M, int N, int K, double2 alpha, const dcplx* A, int64_t lda, int64_t sA,
            const dcplx* B, int64_t ldb, int64_t sB, double2 beta, dcplx* C, int64_t ldc, int64_t sC, int batch,
            bool use_beta) {
  if (ctx->fp64_engine == 1) {
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, batch);
    if (use_beta)
      k_zgemm<OPA, OPB, true><<<grid, NT, 0, ctx->stream>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
    else
      k_zgemm<OPA, OPB, false><<<grid, NT, 0, ctx->stream>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc,
                                                              sC);
    return;
  }
  // 128-row tiles unless they would give fewer than two CTAs per SM; then 64-row tiles,
  // two of which fit an SM
  const int64_t tiles128 = (int64_t)((M + 127) / 128) * ((N + dm::BN - 1) / dm::BN) * batch;
  if (tiles128 >= 2 * 148) launch_dmma<OPA, OPB, 128>(ctx, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC,
                                                       batch, use_beta);
  else launch_dmma<OPA, OPB, 64>(ctx, M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch, use_beta);
}

}  // namespace

void zgemm_fp64(Context* ctx, Op opA, Op opB, int M, int N, int K, cplx alpha, const dcplx* A, int64_t lda,
                int64_t strideA, const dcplx* B, int64_t ldb, int64_t strideB, cplx beta, dcplx* C, int64_t ldc,
                int64_t strideC, int batch) {
  if (M <= 0 || N <= 0 || batch <= 0) return;
  IMPS_REQUIRE(batch <= 65535, IMPS_INVALID_ARG, "zgemm: batch too large");
  IMPS_REQUIRE((N + dm::BN - 1) / dm::BN <= 65535, IMPS_INVALID_ARG, "zgemm: N too large");
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
  if (!(tol > 0)) return 8;
  int s = (int)std::ceil((-std::log2(tol) + 4.0) / 7.0);
  return std::min(8, std::max(2, s));
}

int active_slices(const Context* ctx) {
  if (ctx->precision != PREC_SPLIT_I8 || ctx->force_fp64 > 0) return 0;
  if (!ctx->adaptive_slices) return ctx->nslices;  // a fixed count is used as given
  // adaptive: beyond max_adaptive_slices (6 unless a scope raises it) the FP64 engine
  const int s = slices_for_tol(ctx->split_tol);
  return s > ctx->max_adaptive_slices ? 0 : s;
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
    // reuse a pooled operand: the smallest whose planes already fit, else the largest
    auto rup = [](int64_t x) { return (x + 127) / 128 * 128; };
    const size_t need = (size_t)(side == 0 ? rup(2 * (int64_t)rows) : rup(rows)) * rup(2 * (int64_t)K) * s;
    int best = -1;
    for (int i = 0; i < (int)ctx->split_pool.size(); ++i) {
      const size_t have = ctx->split_pool[i]->data.bytes;
      if (best < 0) { best = i; continue; }
      const size_t cur = ctx->split_pool[best]->data.bytes;
      const bool fits = have >= need, cur_fits = cur >= need;
      if ((fits && (!cur_fits || have < cur)) || (!fits && !cur_fits && have > cur)) best = i;
    }
    if (best >= 0) {
      S = ctx->split_pool[best];
      ctx->split_pool.erase(ctx->split_pool.begin() + best);
    } else {
      S = std::make_shared<SplitOperand>();
    }
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
