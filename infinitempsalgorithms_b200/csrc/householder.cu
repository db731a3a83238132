// QRpos / LQpos on the device by blocked Householder QR, written here (no
// vendor solver library): FiniteMPSAlgorithms' `leftorth(.; alg = QRpos())` and
// `rightorth(.; alg = LQpos())` as used in src/states/ortho.jl:150, 188, 214-225.
//
// M (m x n) = Q R with Q (m x k) isometric, R (k x n) upper trapezoidal with a real
// non-negative diagonal, k = min(m, n).  The reflectors follow LAPACK's zgeqr2
// convention (H = I - tau v v^H with v[0] = 1 and beta = -sign(Re alpha) ||x|| real,
// the trailing columns updated with H^H), so R and Q agree with a LAPACK QR up to
// the final phase fix Q[:, i] *= ph_i, R[i, :] *= conj(ph_i), ph_i = R_ii / |R_ii|.
//
// Blocked right-looking algorithm over panels of NB columns:
//  * k_qr_panel: one thread-block cluster of QR_CL CTAs factors the panel
//    A[p:m, p:p+b].  Each thread keeps RPT rows of the panel in registers for the
//    whole panel; per column the cluster reduces ||x||^2 (one value) and then the
//    NB-1 inner products needed both for the trailing columns of the panel and for
//    the compact-WY factor T (LAPACK zlarft, T[0:c, c] = -tau_c T[0:c, 0:c] V^H v_c),
//    each through distributed shared memory after one cluster barrier.  The kernel
//    writes R (upper part of A), V (explicit, unit diagonal, zeros above), tau and T.
//  * the trailing matrix A2 = A[p:m, p+b:n] <- (I - V T V^H)^H A2 = A2 - V T^H (V^H A2),
//    FP64 GEMMs on the DMMA engine; the long-K product V^H A2 is split into row
//    chunks (one batched GEMM) and summed in a fixed order.
//  * Q = H_1 ... H_k [I; 0] by the same block reflectors applied backwards:
//    Q[p:m, p:k] <- (I - V T V^H) Q[p:m, p:k].
// LQpos is QRpos of the conjugate transpose.
#include <algorithm>

#include "imps_internal.h"

namespace imps {

void scale_q_r(Context* ctx, int m, int n, int k, dcplx* Q, int64_t ldq, dcplx* R, int64_t ldr, const dcplx* ph);

namespace {

constexpr int QR_CL = 8;     // CTAs per cluster (portable cluster size)
constexpr int QR_NT = 512;   // threads per CTA
constexpr int QR_G = QR_CL * QR_NT;
constexpr int QR_NBMAX = 16;
constexpr int QR_KC = 256;   // rows per split-K chunk of the V^H X products

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// all threads of every CTA of the cluster; release / acquire order the shared
// (and global) writes before the barrier with the reads after it
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ double ld_peer(const double* local, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_addr(local)), "r"(rank));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
  return v;
}

__device__ __forceinline__ dcplx cmul(dcplx a, dcplx b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ dcplx cmulc(dcplx a, dcplx b) {  // conj(a) * b
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}

// Householder factorization of the panel A[0:R, 0:b] (lda), b <= NB.  Row il of the
// panel is held by cluster thread g = rank * QR_NT + tid with il = g + k QR_G, k < RPT.
// Outputs: A (R above/on the diagonal, v below), V (R x b, ldv: v with unit diagonal
// and zeros above), tau[0:b], T (b x b, ldt, upper triangular).
template <int NB, int RPT>
__global__ void __cluster_dims__(QR_CL, 1, 1) __launch_bounds__(QR_NT, 1)
    k_qr_panel(int R, int b, dcplx* __restrict__ A, int64_t lda, dcplx* __restrict__ V, int64_t ldv,
               dcplx* __restrict__ tau, dcplx* __restrict__ T, int ldt) {
  __shared__ double red_ssq[2];              // CTA partial of ||x||^2, by column parity
  __shared__ double alpha_sh[2][2];          // alpha (CTA 0 only), by parity
  __shared__ double red_w[2][2 * NB];        // CTA partials of the NB-1 inner products, by parity
  __shared__ double wsum[QR_NT / 32][2 * NB];
  __shared__ dcplx wfin[NB];
  __shared__ dcplx Tsh[NB][NB + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rank = cluster_rank();
  const int g = (int)rank * QR_NT + tid;

  dcplx x[RPT][NB];
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int il = g + k * QR_G;
#pragma unroll
    for (int j = 0; j < NB; ++j)
      x[k][j] = (il < R && j < b) ? A[il + lda * (int64_t)j] : make_double2(0.0, 0.0);
  }
  if (rank == 0)
    for (int e = tid; e < NB * (NB + 1); e += QR_NT) Tsh[e / (NB + 1)][e % (NB + 1)] = make_double2(0.0, 0.0);

  for (int c = 0; c < b; ++c) {
    const int par = c & 1;
    // (a) ||x_below||^2 over the rows below the diagonal; alpha = row c (CTA 0, thread c)
    double ssq = 0.0;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int il = g + k * QR_G;
#pragma unroll
      for (int j = 0; j < NB; ++j)
        if (j == c && il > c && il < R) ssq = fma(x[k][j].x, x[k][j].x, fma(x[k][j].y, x[k][j].y, ssq));
    }
    if (g == c) {
#pragma unroll
      for (int j = 0; j < NB; ++j)
        if (j == c) {
          alpha_sh[par][0] = x[0][j].x;
          alpha_sh[par][1] = x[0][j].y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) ssq += __shfl_down_sync(0xffffffffu, ssq, o);
    if (lane == 0) wsum[warp][0] = ssq;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int q = 0; q < QR_NT / 32; ++q) s += wsum[q][0];
      red_ssq[par] = s;
    }
    cluster_sync();
    // (b) the reflector, computed identically by every thread of the cluster
    double xs = 0.0;
    for (uint32_t q = 0; q < QR_CL; ++q) xs += ld_peer(&red_ssq[par], q);
    const dcplx al = make_double2(ld_peer(&alpha_sh[par][0], 0), ld_peer(&alpha_sh[par][1], 0));
    dcplx tc, scale;
    double beta;
    if (xs == 0.0 && al.y == 0.0) {
      tc = make_double2(0.0, 0.0);
      scale = make_double2(0.0, 0.0);
      beta = al.x;
    } else {
      beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xs), al.x);
      tc = make_double2((beta - al.x) / beta, -al.y / beta);
      // 1 / (alpha - beta)
      const double dr = al.x - beta, di = al.y, den = dr * dr + di * di;
      scale = make_double2(dr / den, -di / den);
    }
    // (c) v (kept in vk), R diagonal; inner products of v with V[:, 0:c] (for T) and
    // with the trailing panel columns (for their update), slot s <-> column s < c ? s : s+1
    dcplx vk[RPT];
    double acc[2 * NB];
#pragma unroll
    for (int s = 0; s < 2 * NB; ++s) acc[s] = 0.0;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int il = g + k * QR_G;
      dcplx v = make_double2(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        if (j == c && il < R) {
          if (il > c) {
            v = cmul(x[k][j], scale);
            x[k][j] = v;
          } else if (il == c) {
            v = make_double2(1.0, 0.0);
            x[k][j] = make_double2(beta, 0.0);
          }
        }
      }
      vk[k] = v;
#pragma unroll
      for (int j = 0; j < NB - 1; ++j) {
        if (j < c) {
          // V[il, j] = x (il > j), 1 (il == j), 0 above
          const dcplx vj = il > j ? x[k][j] : (il == j ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0));
          const dcplx p = cmulc(vj, v);
          acc[2 * j] += p.x;
          acc[2 * j + 1] += p.y;
        } else if (j + 1 < b) {
          const dcplx p = cmulc(v, x[k][j + 1]);
          acc[2 * j] += p.x;
          acc[2 * j + 1] += p.y;
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 2 * (NB - 1); ++s) {
      double t = acc[s];
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) wsum[warp][s] = t;
    }
    __syncthreads();
    if (tid < 2 * (NB - 1)) {
      double s = 0.0;
      for (int q = 0; q < QR_NT / 32; ++q) s += wsum[q][tid];
      red_w[par][tid] = s;
    }
    cluster_sync();
    if (tid < NB - 1) {
      double sr = 0.0, si = 0.0;
      for (uint32_t q = 0; q < QR_CL; ++q) {
        sr += ld_peer(&red_w[par][2 * tid], q);
        si += ld_peer(&red_w[par][2 * tid + 1], q);
      }
      wfin[tid] = make_double2(sr, si);
    }
    __syncthreads();
    // (d) trailing panel columns: x[:, c'] -= conj(tau) v w_{c'}
    const dcplx ctc = make_double2(tc.x, -tc.y);
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const dcplx cv = cmul(ctc, vk[k]);
#pragma unroll
      for (int j = 1; j < NB; ++j) {
        if (j > c && j < b) {
          const dcplx p = cmul(cv, wfin[j - 1]);
          x[k][j].x -= p.x;
          x[k][j].y -= p.y;
        }
      }
    }
    // (e) T[0:c, c] = -tau_c T[0:c, 0:c] z with z_l = <V_l, v_c> (slots l < c)
    if (rank == 0) {
      if (tid < c) {
        dcplx s = make_double2(0.0, 0.0);
        for (int l = tid; l < c; ++l) {
          const dcplx p = cmul(Tsh[tid][l], wfin[l]);
          s.x += p.x;
          s.y += p.y;
        }
        const dcplx t = cmul(tc, s);
        Tsh[tid][c] = make_double2(-t.x, -t.y);
      }
      if (tid == 0) {
        Tsh[c][c] = tc;
        tau[c] = tc;
      }
    }
  }
  // write back: the panel (R above the diagonal, v below) and the explicit V
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int il = g + k * QR_G;
    if (il >= R) continue;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      if (j < b) {
        A[il + lda * (int64_t)j] = x[k][j];
        V[il + ldv * (int64_t)j] = il > j ? x[k][j] : (il == j ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0));
      }
    }
  }
  if (rank == 0) {
    __syncthreads();
    for (int e = tid; e < b * b; e += QR_NT) {
      const int i = e % b, j = e / b;
      T[i + (int64_t)ldt * j] = Tsh[i][j];
    }
  }
  // no CTA may leave while a peer can still read its shared memory
  cluster_sync();
}

__global__ void k_extract_r(int k, int n, const dcplx* __restrict__ A, int64_t lda, dcplx* __restrict__ R,
                            int64_t ldr, dcplx* __restrict__ ph) {
  int64_t tot = (int64_t)k * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t % k), c = (int)(t / k);
    dcplx v = (r <= c) ? A[r + lda * c] : make_double2(0.0, 0.0);
    R[r + ldr * c] = v;
    if (r == c) {
      double a = hypot(v.x, v.y);
      ph[r] = (a > 0.0) ? make_double2(v.x / a, v.y / a) : make_double2(1.0, 0.0);
    }
  }
}

// out[i] = sum_c part[i + stride c] over nc partials, in a fixed order
__global__ void k_sum_partials(int64_t len, int nc, const dcplx* __restrict__ part, int64_t stride,
                               dcplx* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    dcplx s = make_double2(0.0, 0.0);
    for (int c = 0; c < nc; ++c) {
      const dcplx v = part[i + stride * c];
      s.x += v.x;
      s.y += v.y;
    }
    out[i] = s;
  }
}

template <int NB, int RPT>
void launch_panel(Context* ctx, int R, int b, dcplx* A, int64_t lda, dcplx* V, int64_t ldv, dcplx* tau, dcplx* T,
                  int ldt) {
  k_qr_panel<NB, RPT><<<QR_CL, QR_NT, 0, ctx->stream>>>(R, b, A, lda, V, ldv, tau, T, ldt);
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("qr panel launch: ") + cudaGetErrorString(e));
}

// Panel width for a panel of R rows: the registers of a thread hold RPT rows x NB columns.
int panel_width(int R) {
  if (R <= QR_G) return 16;
  if (R <= 2 * QR_G) return 8;
  if (R <= 4 * QR_G) return 4;
  return 2;
}

// W (b x N) = V^H X with V (K x b) and X (K x N) sharing the leading dimension ld and a
// long K: split into chunks of QR_KC rows (one batched GEMM over the full chunks and
// one for the remainder), then a deterministic sum of the partial products.
void gemm_vhx(Context* ctx, int b, int N, int K, const dcplx* Vm, const dcplx* X, int64_t ld, dcplx* part,
              dcplx* W) {
  const int nfull = K / QR_KC, rem = K - nfull * QR_KC;
  const int nc = nfull + (rem > 0 ? 1 : 0);
  const int64_t pstride = (int64_t)b * N;
  if (nc == 1) {
    zgemm_fp64(ctx, OP_C, OP_N, b, N, K, 1.0, Vm, ld, 0, X, ld, 0, 0.0, W, b, 0, 1);
    return;
  }
  if (nfull > 0)
    zgemm_fp64(ctx, OP_C, OP_N, b, N, QR_KC, 1.0, Vm, ld, QR_KC, X, ld, QR_KC, 0.0, part, b, pstride, nfull);
  if (rem > 0)
    zgemm_fp64(ctx, OP_C, OP_N, b, N, rem, 1.0, Vm + (int64_t)nfull * QR_KC, ld, 0, X + (int64_t)nfull * QR_KC, ld, 0,
               0.0, part + pstride * nfull, b, 0, 1);
  const int g = (int)std::min<int64_t>((pstride + 255) / 256, 148 * 8);
  k_sum_partials<<<std::max(g, 1), 256, 0, ctx->stream>>>(pstride, nc, part, pstride, W);
  ctx->n_kernels++;
}

}  // namespace

void qrpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* Q, dcplx* R) {
  IMPS_REQUIRE(m > 0 && n > 0, IMPS_INVALID_ARG, "qrpos: empty matrix");
  IMPS_REQUIRE(m <= 8 * QR_G, IMPS_INVALID_ARG, "qrpos: more than 32768 rows is not supported");
  ctx->n_qr++;
  const int k = std::min(m, n);
  const double qf = 8.0 * (2.0 * m * (double)n * k - 2.0 / 3.0 * k * (double)k * k) * 2.0;
  ctx->qr_flops += qf;
  ScopedTimer t(ctx, "qr", qf);
  const int npan_max = (k + 1) / 2;
  DevBuf& Ab = ctx->buf("qr_a", (size_t)m * n * sizeof(dcplx));
  DevBuf& Vb = ctx->buf("qr_v", (size_t)m * k * sizeof(dcplx));
  DevBuf& Tb = ctx->buf("qr_t", (size_t)npan_max * QR_NBMAX * QR_NBMAX * sizeof(dcplx));
  DevBuf& taub = ctx->buf("qr_tau", (size_t)k * sizeof(dcplx));
  DevBuf& ph = ctx->buf("qr_ph", (size_t)k * sizeof(dcplx));
  DevBuf& Wb = ctx->buf("qr_w", (size_t)QR_NBMAX * std::max(n, k) * sizeof(dcplx));
  DevBuf& W2b = ctx->buf("qr_w2", (size_t)QR_NBMAX * std::max(n, k) * sizeof(dcplx));
  DevBuf& Pb = ctx->buf("qr_part", (size_t)QR_NBMAX * std::max(n, k) * ((m + QR_KC - 1) / QR_KC) * sizeof(dcplx));
  zcopy2d(ctx, m, n, M, ldm, Ab.z(), m);
  dcplx* A = Ab.z();
  std::vector<std::pair<int, int>> panels;  // (p, b)
  for (int p = 0; p < k;) {
    const int Rr = m - p;
    const int b = std::min(panel_width(Rr), k - p);
    dcplx* Ap = A + p + (int64_t)m * p;
    dcplx* Vp = Vb.z() + p + (int64_t)m * p;
    dcplx* Tp = Tb.z() + (size_t)panels.size() * QR_NBMAX * QR_NBMAX;
    switch (panel_width(Rr)) {
      case 16: launch_panel<16, 1>(ctx, Rr, b, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
      case 8: launch_panel<8, 2>(ctx, Rr, b, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
      case 4: launch_panel<4, 4>(ctx, Rr, b, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
      default: launch_panel<2, 8>(ctx, Rr, b, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
    }
    const int n2 = n - p - b;
    if (n2 > 0) {
      dcplx* A2 = A + p + (int64_t)m * (p + b);
      // W = V^H A2, W2 = T^H W, A2 -= V W2
      gemm_vhx(ctx, b, n2, Rr, Vp, A2, m, Pb.z(), Wb.z());
      zgemm_fp64(ctx, OP_C, OP_N, b, n2, b, 1.0, Tp, QR_NBMAX, 0, Wb.z(), b, 0, 0.0, W2b.z(), b, 0, 1);
      zgemm_fp64(ctx, OP_N, OP_N, Rr, n2, b, -1.0, Vp, m, 0, W2b.z(), b, 0, 1.0, A2, m, 0, 1);
    }
    panels.push_back({p, b});
    p += b;
  }
  {
    int64_t tot = (int64_t)k * n;
    int g = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
    k_extract_r<<<std::max(g, 1), 256, 0, ctx->stream>>>(k, n, A, m, R, k, ph.z());
    ctx->n_kernels++;
  }
  // Q = H_1 ... H_k [I; 0], block reflectors applied from the last panel back
  zfill2d(ctx, m, k, 0.0, Q, m);
  zadd_diag(ctx, k, Q, m, 1.0);
  for (int t = (int)panels.size() - 1; t >= 0; --t) {
    const int p = panels[t].first, b = panels[t].second;
    const int Rr = m - p, nc = k - p;
    dcplx* Vp = Vb.z() + p + (int64_t)m * p;
    dcplx* Tp = Tb.z() + (size_t)t * QR_NBMAX * QR_NBMAX;
    dcplx* Qs = Q + p + (int64_t)m * p;
    gemm_vhx(ctx, b, nc, Rr, Vp, Qs, m, Pb.z(), Wb.z());
    zgemm_fp64(ctx, OP_N, OP_N, b, nc, b, 1.0, Tp, QR_NBMAX, 0, Wb.z(), b, 0, 0.0, W2b.z(), b, 0, 1);
    zgemm_fp64(ctx, OP_N, OP_N, Rr, nc, b, -1.0, Vp, m, 0, W2b.z(), b, 0, 1.0, Qs, m, 0, 1);
  }
  scale_q_r(ctx, m, n, k, Q, m, R, k, ph.z());
}

void lqpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, dcplx* Q) {
  // M (m x n) = L Q  <=>  M^H = Q^H L^H : QRpos of M^H (n x m) gives Q' (n x k), R' (k x m)
  const int k = std::min(m, n);
  DevBuf& MH = ctx->buf("lq_mh", (size_t)m * n * sizeof(dcplx));
  DevBuf& Qp = ctx->buf("lq_q", (size_t)n * k * sizeof(dcplx));
  DevBuf& Rp = ctx->buf("lq_r", (size_t)k * m * sizeof(dcplx));
  zconj_transpose(ctx, m, n, M, ldm, MH.z(), n);
  qrpos(ctx, n, m, MH.z(), n, Qp.z(), Rp.z());
  zconj_transpose(ctx, k, m, Rp.z(), k, L, m);   // L = R'^H  (m x k)
  zconj_transpose(ctx, n, k, Qp.z(), n, Q, k);   // Q = Q'^H  (k x n)
}

}  // namespace imps
