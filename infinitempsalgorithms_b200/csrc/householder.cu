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
// Two-level blocked right-looking algorithm:
//  * k_qr_panel: one thread-block cluster of QR_CL CTAs factors the panel
//    A[p:m, p:p+b] (b <= 16), the panel rows staged in shared memory.  Per column a
//    single cluster reduction (distributed shared memory after one cluster barrier)
//    gives ||x||^2, the inner products with the trailing panel columns and those with
//    the earlier reflectors needed for the compact-WY factor T (LAPACK zlarft,
//    T[0:c, c] = -tau_c T[0:c, 0:c] V^H v_c).  The kernel writes R (upper part of A),
//    V (explicit, unit diagonal, zeros above), tau and T.
//  * inner panels update only the rest of their outer block of QR_NBO columns; the
//    outer block's T is merged from the panels' factors (k_merge_t, with G = V^H V),
//    and the trailing matrix A2 <- (I - V T V^H)^H A2 = A2 - (V T^H) (A2^H V)^H is updated
//    once per outer block by FP64 GEMMs on the DMMA engine (the long-K product A2^H V
//    split into row chunks, one batched GEMM, summed in a fixed order).
//  * Q = H_1 ... H_k [I; 0] by the outer block reflectors applied backwards:
//    Q[P:m, P:k] <- (I - V T V^H) Q[P:m, P:k].
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
constexpr int QR_NBO = 64;   // outer block: columns per compact-WY trailing update
constexpr size_t QR_PANEL_SMEM = (size_t)QR_NBMAX * QR_NT * sizeof(dcplx);  // NB RPT = 16 for every panel kind
constexpr int QR_MAXCHUNK = 32;  // most row chunks of a split-K X^H V product

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
// store v into the same shared variable of CTA `rank` of the cluster (made visible to
// that CTA by the next cluster barrier's release / acquire)
__device__ __forceinline__ void st_peer(double* local, uint32_t rank, double v) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_addr(local)), "r"(rank));
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}

__device__ __forceinline__ dcplx cmul(dcplx a, dcplx b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ dcplx cmulc(dcplx a, dcplx b) {  // conj(a) * b
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}

// Sum of val[s] over the 32 lanes of a warp for NV slots by a reduce-scatter: log2(NV)
// exchange rounds of halving width (NV - 1 shuffles in all), then plain rounds over the
// lanes that share a slot.  Returns the warp total of slot lane / (32 / NV).
template <int NV>
__device__ __forceinline__ double warp_reduce_scatter(double (&val)[NV], int lane) {
  int half = NV;
#pragma unroll
  for (int o = 16; o >= 32 / NV; o >>= 1) {
    half >>= 1;
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int v = 0; v < NV / 2; ++v) {
      if (v < half) {
        const double send = up ? val[v] : val[v + half];
        const double keep = up ? val[v + half] : val[v];
        val[v] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
  }
  double r = val[0];
#pragma unroll
  for (int o = 32 / NV / 2; o >= 1; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

// Householder factorization of the panel A[0:R, 0:b] (lda), b <= NB.  Row il of the
// panel belongs to cluster thread g = rank * QR_NT + tid with il = g + k QR_G, k < RPT,
// and lives in shared memory (NB RPT QR_NT complex = 128 KiB per CTA).
// One cluster reduction per column: ||x_c below||^2, d_j = x_c^H x_j (j > c, trailing
// panel columns) and e_l = V_l^H x_c (l < c, for T), all over the rows below c, together
// with row c of the panel (held by thread c of CTA 0).  With v = [1; scale x_c below]:
//   v^H x_j = x_j[c] + conj(scale) d_j,   V_l^H v = conj(V_l[c]) + scale e_l.
// Outputs: A (R above/on the diagonal, v below), V (R x b, ldv: v with unit diagonal and
// zeros above; the zabove rows before row 0 are zeroed too), tau[0:b], T (b x b, ldt).
template <int NB, int RPT>
__global__ void __cluster_dims__(QR_CL, 1, 1) __launch_bounds__(QR_NT, 1)
    k_qr_panel(int R, int b, int zabove, dcplx* __restrict__ A, int64_t lda, dcplx* __restrict__ V, int64_t ldv,
               dcplx* __restrict__ tau, dcplx* __restrict__ T, int ldt) {
  constexpr int NV = 2 * NB;       // reduction slots: [0] ||x||^2, [1 + 2s, 2 + 2s] complex slot s
  constexpr int SPL = 32 / NV;     // lanes per slot after the reduce-scatter
  extern __shared__ dcplx xs[];    // xs[(k NB + j) QR_NT + tid]
  __shared__ double wsum[QR_NT / 32][NV];
  __shared__ double red[2][QR_CL][NV];   // partials pushed by every CTA of the cluster
  __shared__ double rowc[2][2 * NB];     // row c of the panel, pushed by CTA 0
  __shared__ double fin[NV + 2 * NB];
  __shared__ dcplx Tsh[NB][NB + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rank = cluster_rank();
  const int g = (int)rank * QR_NT + tid;
#define XS(k, j) xs[((k) * NB + (j)) * QR_NT + tid]

#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int il = g + k * QR_G;
#pragma unroll
    for (int j = 0; j < NB; ++j) XS(k, j) = (il < R && j < b) ? A[il + lda * (int64_t)j] : make_double2(0.0, 0.0);
  }
  if (rank == 0)
    for (int e = tid; e < NB * (NB + 1); e += QR_NT) Tsh[e / (NB + 1)][e % (NB + 1)] = make_double2(0.0, 0.0);

  for (int c = 0; c < b; ++c) {
    const int par = c & 1;
    double val[NV];
#pragma unroll
    for (int s = 0; s < NV; ++s) val[s] = 0.0;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int il = g + k * QR_G;
      if (il > c && il < R) {
        const dcplx xc = XS(k, c);
        val[0] = fma(xc.x, xc.x, fma(xc.y, xc.y, val[0]));
#pragma unroll
        for (int s = 0; s < NB - 1; ++s) {
          dcplx p = make_double2(0.0, 0.0);
          if (s < c) p = cmulc(XS(k, s), xc);                // e_s
          else if (s + 1 < b) p = cmulc(xc, XS(k, s + 1));   // d_{s+1}
          val[1 + 2 * s] += p.x;
          val[2 + 2 * s] += p.y;
        }
      }
    }
    const double wv = warp_reduce_scatter<NV>(val, lane);
    if (lane % SPL == 0) wsum[warp][lane / SPL] = wv;
    __syncthreads();
    // push this CTA's partials (and, from CTA 0, row c of the panel: thread c's row
    // in shared memory) into every CTA of the cluster; no remote loads
    if (tid < NV) {
      double t = 0.0;
      for (int q = 0; q < QR_NT / 32; ++q) t += wsum[q][tid];
#pragma unroll
      for (uint32_t q = 0; q < QR_CL; ++q) st_peer(&red[par][rank][tid], q, t);
    } else if (rank == 0 && tid < NV + 2 * NB * QR_CL) {
      const int e = tid - NV, slot = e % (2 * NB), dst = e / (2 * NB);
      const dcplx x = xs[(slot >> 1) * QR_NT + c];   // XS(0, slot / 2) of thread c
      st_peer(&rowc[par][slot], (uint32_t)dst, (slot & 1) ? x.y : x.x);
    }
    cluster_sync();
    if (tid < NV) {
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < QR_CL; ++q) t += red[par][q][tid];
      fin[tid] = t;
    } else if (tid < NV + 2 * NB) {
      fin[tid] = rowc[par][tid - NV];
    }
    __syncthreads();
    // the reflector (LAPACK zlarfg), computed identically by every thread
    const double xsq = fin[0];
    const dcplx al = make_double2(fin[NV + 2 * c], fin[NV + 2 * c + 1]);
    dcplx tc, scale;
    double beta;
    if (xsq == 0.0 && al.y == 0.0) {
      tc = make_double2(0.0, 0.0);
      scale = make_double2(0.0, 0.0);
      beta = al.x;
    } else {
      beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xsq), al.x);
      tc = make_double2((beta - al.x) / beta, -al.y / beta);
      const double dr = al.x - beta, di = al.y, den = dr * dr + di * di;
      scale = make_double2(dr / den, -di / den);   // 1 / (alpha - beta)
    }
    const dcplx ctc = make_double2(tc.x, -tc.y), cs = make_double2(scale.x, -scale.y);
    // v into column c, R diagonal, trailing panel columns x_j -= conj(tau) v (v^H x_j)
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int il = g + k * QR_G;
      if (il < c || il >= R) continue;
      dcplx v;
      if (il == c) {
        v = make_double2(1.0, 0.0);
        XS(k, c) = make_double2(beta, 0.0);
      } else {
        v = cmul(XS(k, c), scale);
        XS(k, c) = v;
      }
      const dcplx cv = cmul(ctc, v);
#pragma unroll
      for (int j = 1; j < NB; ++j) {
        if (j > c && j < b) {
          const dcplx dj = make_double2(fin[1 + 2 * (j - 1)], fin[2 + 2 * (j - 1)]);
          const dcplx rj = make_double2(fin[NV + 2 * j], fin[NV + 2 * j + 1]);
          const dcplx t = cmul(cs, dj);
          const dcplx w = make_double2(rj.x + t.x, rj.y + t.y);
          const dcplx p = cmul(cv, w);
          dcplx x = XS(k, j);
          x.x -= p.x;
          x.y -= p.y;
          XS(k, j) = x;
        }
      }
    }
    // T[0:c, c] = -tau T[0:c, 0:c] z with z_l = V_l^H v = conj(V_l[c]) + scale e_l (LAPACK zlarft)
    if (rank == 0) {
      if (tid < c) {
        dcplx sacc = make_double2(0.0, 0.0);
        for (int l = tid; l < c; ++l) {
          const dcplx el = make_double2(fin[1 + 2 * l], fin[2 + 2 * l]);
          const dcplx se = cmul(scale, el);
          const dcplx z = make_double2(fin[NV + 2 * l] + se.x, -fin[NV + 2 * l + 1] + se.y);
          const dcplx p = cmul(Tsh[tid][l], z);
          sacc.x += p.x;
          sacc.y += p.y;
        }
        const dcplx t = cmul(tc, sacc);
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
        const dcplx x = XS(k, j);
        A[il + lda * (int64_t)j] = x;
        V[il + ldv * (int64_t)j] = il > j ? x : (il == j ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0));
      }
    }
  }
#undef XS
  for (int r = g; r < zabove; r += QR_G)
    for (int j = 0; j < b; ++j) V[(int64_t)(r - zabove) + ldv * (int64_t)j] = make_double2(0.0, 0.0);
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

// Compact-WY factor of an outer block from the factors of its inner panels (LAPACK
// zlarft, block form): T = [[T1, -T1 (V1^H V2) T2], [0, T2]] applied panel by panel,
// with G = V^H V of the whole outer block.  One CTA; T is bo x bo (ld bo).
struct PanelList {
  int n;
  short off[QR_NBO / 2 + 1];
  short w[QR_NBO / 2];
};

// T, G and the panels' products live in shared memory for the whole merge (one CTA).
constexpr size_t QR_MERGE_SMEM = (size_t)2 * QR_NBO * (QR_NBO + 1) * sizeof(dcplx);

__global__ void __launch_bounds__(256) k_merge_t(int bo, PanelList pl, const dcplx* __restrict__ Tin,
                                                 const dcplx* __restrict__ G, dcplx* __restrict__ Tb) {
  extern __shared__ __align__(16) dcplx msm[];
  const int ld = bo + 1;
  dcplx* Ts = msm;                            // Ts[r + ld c]
  dcplx* Gs = msm + (size_t)QR_NBO * (QR_NBO + 1);
  __shared__ dcplx Xs[QR_NBO][QR_NBMAX];
  const int tid = threadIdx.x;
  for (int e = tid; e < bo * bo; e += blockDim.x) {
    const int r = e % bo, c = e / bo;
    int t = 0;
    while (t + 1 < pl.n && pl.off[t + 1] <= c) ++t;
    const int o = pl.off[t];
    dcplx v = make_double2(0.0, 0.0);
    if (r >= o && r < o + pl.w[t]) v = Tin[(size_t)t * QR_NBMAX * QR_NBMAX + (r - o) + QR_NBMAX * (c - o)];
    Ts[r + ld * c] = v;
    if (pl.n > 1) Gs[r + ld * c] = G[r + (int64_t)bo * c];
  }
  __syncthreads();
  for (int t = 1; t < pl.n; ++t) {
    const int c0 = pl.off[t], bt = pl.w[t];
    const dcplx* Tt = Tin + (size_t)t * QR_NBMAX * QR_NBMAX;
    for (int e = tid; e < c0 * bt; e += blockDim.x) {
      const int r = e % c0, u = e / c0;
      dcplx sacc = make_double2(0.0, 0.0);
      for (int l = r; l < c0; ++l) {
        const dcplx p = cmul(Ts[r + ld * l], Gs[l + ld * (c0 + u)]);
        sacc.x += p.x;
        sacc.y += p.y;
      }
      Xs[r][u] = sacc;
    }
    __syncthreads();
    for (int e = tid; e < c0 * bt; e += blockDim.x) {
      const int r = e % c0, u = e / c0;
      dcplx sacc = make_double2(0.0, 0.0);
      for (int v = 0; v <= u; ++v) {
        const dcplx p = cmul(Xs[r][v], Tt[v + QR_NBMAX * u]);
        sacc.x += p.x;
        sacc.y += p.y;
      }
      Ts[r + ld * (c0 + u)] = make_double2(-sacc.x, -sacc.y);
    }
    __syncthreads();
  }
  for (int e = tid; e < bo * bo; e += blockDim.x) Tb[e] = Ts[(e % bo) + ld * (e / bo)];
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
void launch_panel(Context* ctx, int R, int b, int zabove, dcplx* A, int64_t lda, dcplx* V, int64_t ldv, dcplx* tau,
                  dcplx* T, int ldt) {
  static_assert(NB * RPT == QR_NBMAX, "panel shared-memory size");
  static DeviceOnce attr;
  attr.run(ctx->device, [] {
    IMPS_CUDA(cudaFuncSetAttribute(k_qr_panel<NB, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)QR_PANEL_SMEM));
  });
  k_qr_panel<NB, RPT><<<QR_CL, QR_NT, QR_PANEL_SMEM, ctx->stream>>>(R, b, zabove, A, lda, V, ldv, tau, T, ldt);
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

// Small-product path for the updates inside an outer block (N <= 48 columns against
// b <= 16 reflectors): on these shapes a DMMA GEMM launch is all pipeline fill, so one
// kernel forms the long-K product and a second applies it.
constexpr int XS_NT = 256;   // threads of the X^H V kernel
constexpr int XS_ROWS = 64;  // rows staged in shared memory per step (one step per CTA)
constexpr int XS_MAXO = 16;  // outputs per thread: N b <= 4096
constexpr int XS_LD = XS_ROWS + 1;

// Wh (N x b, ld N) = X^H V over K rows, X (K x N) and V (K x b) with leading dimension ld.
// CTA g sums rows [g kc, (g + 1) kc) into part[g]; the last CTA to finish (counter) adds
// the partials in CTA order, so the result does not depend on scheduling, resets the
// counter and, when T is given, forms Z (b x N, ld b) = op(T) Wh^H (op = C or N).
__global__ void __launch_bounds__(XS_NT) k_xhv_small(int K, int N, int b, int kc, const dcplx* __restrict__ X,
                                                      const dcplx* __restrict__ Vm, int64_t ld,
                                                      dcplx* __restrict__ part, unsigned* __restrict__ counter,
                                                      dcplx* __restrict__ Wh, const dcplx* __restrict__ T, int ldt,
                                                      int conjT, dcplx* __restrict__ Z) {
  extern __shared__ dcplx sh[];  // [N + b columns][XS_LD rows], later the summed Wh
  __shared__ bool last;
  const int nb = N * b, W = N + b, tid = threadIdx.x;
  const int k0 = blockIdx.x * kc, k1 = min(K, k0 + kc);
  dcplx acc[XS_MAXO];
#pragma unroll
  for (int i = 0; i < XS_MAXO; ++i) acc[i] = make_double2(0.0, 0.0);
  for (int r0 = k0; r0 < k1; r0 += XS_ROWS) {
    const int nr = min(XS_ROWS, k1 - r0);
    __syncthreads();
    for (int e = tid; e < XS_ROWS * W; e += XS_NT) {
      const int r = e % XS_ROWS, col = e / XS_ROWS;  // consecutive threads walk rows: coalesced
      dcplx v = make_double2(0.0, 0.0);
      if (r < nr) v = (col < N) ? X[(int64_t)(r0 + r) + ld * col] : Vm[(int64_t)(r0 + r) + ld * (col - N)];
      sh[r + XS_LD * col] = v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < XS_MAXO; ++i) {
      const int o = tid + XS_NT * i;
      if (o < nb) {
        const dcplx* xc = sh + XS_LD * (o % N);
        const dcplx* vc = sh + XS_LD * (N + o / N);
        for (int r = 0; r < nr; ++r) {
          const dcplx x = xc[r], v = vc[r];
          acc[i].x = fma(x.x, v.x, fma(x.y, v.y, acc[i].x));
          acc[i].y = fma(x.x, v.y, fma(-x.y, v.x, acc[i].y));
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < XS_MAXO; ++i) {
    const int o = tid + XS_NT * i;
    if (o < nb) part[(int64_t)blockIdx.x * nb + o] = acc[i];
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  __syncthreads();
  for (int o = tid; o < nb; o += XS_NT) {
    dcplx t = make_double2(0.0, 0.0);
    int g = 0;
    for (; g + 4 <= (int)gridDim.x; g += 4) {  // four loads in flight, added in CTA order
      const dcplx v0 = __ldcg(&part[(int64_t)g * nb + o]), v1 = __ldcg(&part[(int64_t)(g + 1) * nb + o]);
      const dcplx v2 = __ldcg(&part[(int64_t)(g + 2) * nb + o]), v3 = __ldcg(&part[(int64_t)(g + 3) * nb + o]);
      t.x += v0.x; t.y += v0.y;
      t.x += v1.x; t.y += v1.y;
      t.x += v2.x; t.y += v2.y;
      t.x += v3.x; t.y += v3.y;
    }
    for (; g < (int)gridDim.x; ++g) {
      const dcplx v = __ldcg(&part[(int64_t)g * nb + o]);
      t.x += v.x;
      t.y += v.y;
    }
    Wh[o] = t;
    sh[o] = t;  // nb <= XS_LD * (N + b)
  }
  if (tid == 0) *counter = 0u;
  if (!Z) return;
  __syncthreads();
  // Z[i, n] = sum_l op(T)[i, l] conj(Wh[n, l])
  for (int e = tid; e < nb; e += XS_NT) {
    const int i = e % b, n = e / b;
    dcplx z = make_double2(0.0, 0.0);
    for (int l = 0; l < b; ++l) {
      dcplx t = conjT ? T[l + (int64_t)ldt * i] : T[i + (int64_t)ldt * l];
      if (conjT) t.y = -t.y;
      const dcplx w = sh[n + N * l];  // conj(w) below
      z.x += t.x * w.x + t.y * w.y;
      z.y += t.y * w.x - t.x * w.y;
    }
    Z[e] = z;
  }
}

// A2 (R x N, lda) -= V (R x b, ldv) Z (b x N), b <= 16, N <= 64: a thread per element,
// 64 rows x 4 columns per CTA (row loads coalesced, V rows shared through L1).
__global__ void __launch_bounds__(256) k_apply_small(int R, int N, int b, const dcplx* __restrict__ Vm, int64_t ldv,
                                                     const dcplx* __restrict__ Z, dcplx* __restrict__ A2,
                                                     int64_t lda) {
  const int r = blockIdx.x * 64 + (threadIdx.x & 63);
  const int n = blockIdx.y * 4 + (threadIdx.x >> 6);
  if (r >= R || n >= N) return;
  dcplx a = A2[r + lda * n];
#pragma unroll
  for (int i = 0; i < QR_NBMAX; ++i) {
    if (i < b) {
      const dcplx v = Vm[r + ldv * i], z = __ldg(&Z[i + b * n]);
      a.x -= v.x * z.x - v.y * z.y;
      a.y -= v.x * z.y + v.y * z.x;
    }
  }
  A2[r + lda * n] = a;
}

// Wh = X^H V (and Z = op(T) Wh^H when T is given) by k_xhv_small.
void xhv_small(Context* ctx, int N, int b, int K, const dcplx* X, const dcplx* Vm, int64_t ld, dcplx* part,
               dcplx* Wh, const dcplx* T, int ldt, bool conjT, dcplx* Z) {
  IMPS_REQUIRE(N * b <= XS_NT * XS_MAXO && N <= QR_NBO && b <= QR_NBO, IMPS_INVALID_ARG, "xhv_small: shape");
  DevBuf& cnt = ctx->buf("qr_xhv_count", 256);
  if (ctx->qr_count_ptr != cnt.ptr) {  // a new counter starts at zero; each launch leaves it at zero
    IMPS_CUDA(cudaMemsetAsync(cnt.ptr, 0, 256, ctx->stream));
    ctx->qr_count_ptr = cnt.ptr;
  }
  // one staged chunk of XS_ROWS rows per CTA, at most 64 partials (more rows per CTA past
  // that): the last CTA sums g N b values
  int g = std::max(1, std::min(64, (K + XS_ROWS - 1) / XS_ROWS));
  const int kc = (K + g - 1) / g;
  g = (K + kc - 1) / kc;
  ScopedTimer tm(ctx, "qr_small", 8.0 * N * b * (double)K);
  const size_t smem = (size_t)XS_LD * (N + b) * sizeof(dcplx);
  static DeviceOnce attr;
  attr.run(ctx->device, [] {
    IMPS_CUDA(cudaFuncSetAttribute(k_xhv_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)((size_t)XS_LD * 2 * QR_NBO * sizeof(dcplx))));
  });
  k_xhv_small<<<g, XS_NT, smem, ctx->stream>>>(K, N, b, kc, X, Vm, ld, part, static_cast<unsigned*>(cnt.ptr), Wh,
                                               T, ldt, conjT ? 1 : 0, Z);
  ctx->n_kernels++;
  IMPS_CUDA(cudaPeekAtLastError());
}

void apply_small(Context* ctx, int R, int N, int b, const dcplx* Vm, int64_t ldv, const dcplx* Z, dcplx* A2,
                 int64_t lda) {
  IMPS_REQUIRE(b <= QR_NBMAX && N <= QR_NBO, IMPS_INVALID_ARG, "apply_small: shape");
  ScopedTimer tm(ctx, "qr_small", 8.0 * R * N * (double)b);
  k_apply_small<<<dim3((R + 63) / 64, (N + 3) / 4), 256, 0, ctx->stream>>>(R, N, b, Vm, ldv, Z, A2, lda);
  ctx->n_kernels++;
  IMPS_CUDA(cudaPeekAtLastError());
}

// Wh (N x b, ld N) = X^H V with X (K x N) and V (K x b) sharing the leading dimension ld
// and a long K.  The long side N goes on the GEMM's 128-row output tile; K is split into
// row chunks (one batched GEMM over the full chunks and one for the remainder) so that
// about two CTAs per SM are busy, then the partial products are summed in a fixed order.
void gemm_xhv(Context* ctx, int N, int b, int K, const dcplx* X, const dcplx* Vm, int64_t ld, dcplx* part,
              dcplx* Wh) {
  const int tiles = ((N + 127) / 128) * ((b + 63) / 64);
  int nc = std::max(1, std::min({(2 * 148 + tiles - 1) / tiles, QR_MAXCHUNK, K / 64}));
  int kc = (K + nc - 1) / nc;
  kc = (kc + 15) / 16 * 16;
  nc = (K + kc - 1) / kc;
  if (nc == 1) {
    zgemm_fp64(ctx, OP_C, OP_N, N, b, K, 1.0, X, ld, 0, Vm, ld, 0, 0.0, Wh, N, 0, 1);
    return;
  }
  const int nfull = K / kc, rem = K - nfull * kc;
  const int64_t pstride = (int64_t)N * b;
  if (nfull > 0)
    zgemm_fp64(ctx, OP_C, OP_N, N, b, kc, 1.0, X, ld, kc, Vm, ld, kc, 0.0, part, N, pstride, nfull);
  if (rem > 0)
    zgemm_fp64(ctx, OP_C, OP_N, N, b, rem, 1.0, X + (int64_t)nfull * kc, ld, 0, Vm + (int64_t)nfull * kc, ld, 0,
               0.0, part + pstride * nfull, N, 0, 1);
  const int g = (int)std::min<int64_t>((pstride + 255) / 256, 148 * 8);
  k_sum_partials<<<std::max(g, 1), 256, 0, ctx->stream>>>(pstride, nc, part, pstride, Wh);
  ctx->n_kernels++;
}

// A2 (R x N) <- A2 - Y Wh^H with Y = V op(T) (R x b): one block-reflector application
// given Wh = A2^H V (op = C: A2 <- (I - V T V^H)^H A2; op = N: A2 <- (I - V T V^H) A2).
void apply_block(Context* ctx, int R, int N, int b, const dcplx* Vp, int64_t ldv, const dcplx* Tp, int ldt, Op opT,
                 const dcplx* Wh, dcplx* Y, dcplx* A2, int64_t lda) {
  zgemm_fp64(ctx, OP_N, opT, R, b, b, 1.0, Vp, ldv, 0, Tp, ldt, 0, 0.0, Y, R, 0, 1);
  zgemm_fp64(ctx, OP_N, OP_C, R, N, b, -1.0, Y, R, 0, Wh, N, 0, 1.0, A2, lda, 0, 1);
}

}  // namespace

// Factorisation half of QRpos: A = H_1 ... H_k [R; 0].  The explicit reflectors V, the
// compact-WY factor of every outer block and the diagonal phases stay in the slot's
// buffers (`<slot>_v`, `<slot>_t`, `<slot>_ph`) until the next factorisation into the
// same slot, so that Q can be formed later (qr_form_q) or not at all.  R gets the
// positive-diagonal phase fix.
void qr_factor(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* R, const char* slot) {
  IMPS_REQUIRE(m > 0 && n > 0, IMPS_INVALID_ARG, "qrpos: empty matrix");
  IMPS_REQUIRE(m <= 8 * QR_G, IMPS_INVALID_ARG, "qrpos: more than 32768 rows is not supported");
  ctx->n_qr++;
  const int k = std::min(m, n);
  const double qf = 8.0 * (2.0 * m * (double)n * k - 2.0 / 3.0 * k * (double)k * k);
  ctx->qr_flops += qf;
  ScopedTimer t(ctx, "qr", qf);
  const std::string sl(slot);
  const int nob = (k + QR_NBO - 1) / QR_NBO;
  const int wmax = std::max({n, k, QR_NBO});
  DevBuf& Ab = ctx->buf("qr_a", (size_t)m * n * sizeof(dcplx));
  DevBuf& Vb = ctx->buf(sl + "_v", (size_t)m * k * sizeof(dcplx));
  DevBuf& Tin = ctx->buf("qr_tin", (size_t)(QR_NBO / 2) * QR_NBMAX * QR_NBMAX * sizeof(dcplx));
  DevBuf& Tbig = ctx->buf(sl + "_t", (size_t)nob * QR_NBO * QR_NBO * sizeof(dcplx));
  DevBuf& Gb = ctx->buf("qr_g", (size_t)QR_NBO * QR_NBO * sizeof(dcplx));
  DevBuf& taub = ctx->buf("qr_tau", (size_t)k * sizeof(dcplx));
  DevBuf& ph = ctx->buf(sl + "_ph", (size_t)k * sizeof(dcplx));
  DevBuf& Wb = ctx->buf("qr_w", (size_t)QR_NBO * wmax * sizeof(dcplx));
  DevBuf& Yb = ctx->buf("qr_y", (size_t)QR_NBO * m * sizeof(dcplx));
  // partial products: the split-K GEMMs' chunks, or k_xhv_small's (up to 2 CTAs per SM)
  DevBuf& Pb = ctx->buf("qr_part", std::max((size_t)QR_NBO * wmax * QR_MAXCHUNK,
                                            (size_t)2 * ctx->num_sms * QR_NBO * QR_NBO) * sizeof(dcplx));
  DevBuf& Zb = ctx->buf("qr_z", (size_t)QR_NBMAX * QR_NBO * sizeof(dcplx));
  zcopy2d(ctx, m, n, M, ldm, Ab.z(), m);
  dcplx* A = Ab.z();
  int nblk = 0;
  for (int P = 0; P < k;) {
    const int bo = std::min(QR_NBO, k - P);
    PanelList pl;
    pl.n = 0;
    // inner panels; each also updates the rest of its outer block
    for (int p = P; p < P + bo;) {
      const int Rr = m - p;
      const int b = std::min(panel_width(Rr), P + bo - p);
      dcplx* Ap = A + p + (int64_t)m * p;
      dcplx* Vp = Vb.z() + p + (int64_t)m * p;
      dcplx* Tp = Tin.z() + (size_t)pl.n * QR_NBMAX * QR_NBMAX;
      switch (panel_width(Rr)) {
        case 16: launch_panel<16, 1>(ctx, Rr, b, p - P, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
        case 8: launch_panel<8, 2>(ctx, Rr, b, p - P, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
        case 4: launch_panel<4, 4>(ctx, Rr, b, p - P, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
        default: launch_panel<2, 8>(ctx, Rr, b, p - P, Ap, m, Vp, m, taub.z() + p, Tp, QR_NBMAX); break;
      }
      pl.off[pl.n] = (short)(p - P);
      pl.w[pl.n] = (short)b;
      pl.n++;
      const int n2in = P + bo - (p + b);
      if (n2in > 0) {
        // A2 <- A2 - V T^H (A2^H V)^H for the rest of the outer block
        dcplx* A2 = A + p + (int64_t)m * (p + b);
        xhv_small(ctx, n2in, b, Rr, A2, Vp, m, Pb.z(), Wb.z(), Tp, QR_NBMAX, true, Zb.z());
        apply_small(ctx, Rr, n2in, b, Vp, m, Zb.z(), A2, m);
      }
      p += b;
    }
    pl.off[pl.n] = (short)bo;
    // compact-WY factor of the outer block, then its trailing update
    const int RrB = m - P;
    dcplx* Vblk = Vb.z() + P + (int64_t)m * P;
    dcplx* Tb = Tbig.z() + (size_t)nblk * QR_NBO * QR_NBO;
    if (pl.n > 1) gemm_xhv(ctx, bo, bo, RrB, Vblk, Vblk, m, Pb.z(), Gb.z());
    static DeviceOnce merge_attr;
    merge_attr.run(ctx->device, [] {
      IMPS_CUDA(cudaFuncSetAttribute(k_merge_t, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QR_MERGE_SMEM));
    });
    k_merge_t<<<1, 256, QR_MERGE_SMEM, ctx->stream>>>(bo, pl, Tin.z(), Gb.z(), Tb);
    ctx->n_kernels++;
    const int n2 = n - (P + bo);
    if (n2 > 0) {
      dcplx* A2 = A + P + (int64_t)m * (P + bo);
      gemm_xhv(ctx, n2, bo, RrB, A2, Vblk, m, Pb.z(), Wb.z());
      apply_block(ctx, RrB, n2, bo, Vblk, m, Tb, bo, OP_C, Wb.z(), Yb.z(), A2, m);
    }
    ++nblk;
    P += bo;
  }
  {
    int64_t tot = (int64_t)k * n;
    int g = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
    k_extract_r<<<std::max(g, 1), 256, 0, ctx->stream>>>(k, n, A, m, R, k, ph.z());
    ctx->n_kernels++;
  }
  scale_q_r(ctx, 0, n, k, nullptr, 1, R, k, ph.z());  // R rows by conj(phase)
}

// Q (m x k, ld m) of the last qr_factor(m, n, ...) into `slot`:
// Q = H_1 ... H_k [I; 0] with the outer blocks applied from the last back, then the
// columns scaled by the diagonal phases (the positive-diagonal convention of QRpos).
void qr_form_q(Context* ctx, int m, int n, dcplx* Q, const char* slot) {
  const int k = std::min(m, n);
  const double qf = 8.0 * (2.0 * m * (double)n * k - 2.0 / 3.0 * k * (double)k * k);
  ctx->qr_flops += qf;
  ScopedTimer t(ctx, "qr", qf);
  const std::string sl(slot);
  const int nob = (k + QR_NBO - 1) / QR_NBO;
  const int wmax = std::max({n, k, QR_NBO});
  DevBuf& Vb = ctx->buf(sl + "_v", (size_t)m * k * sizeof(dcplx));
  DevBuf& Tbig = ctx->buf(sl + "_t", (size_t)nob * QR_NBO * QR_NBO * sizeof(dcplx));
  DevBuf& ph = ctx->buf(sl + "_ph", (size_t)k * sizeof(dcplx));
  DevBuf& Wb = ctx->buf("qr_w", (size_t)QR_NBO * wmax * sizeof(dcplx));
  DevBuf& Yb = ctx->buf("qr_y", (size_t)QR_NBO * m * sizeof(dcplx));
  DevBuf& Pb = ctx->buf("qr_part", (size_t)QR_NBO * wmax * QR_MAXCHUNK * sizeof(dcplx));
  zfill2d(ctx, m, k, 0.0, Q, m);
  zadd_diag(ctx, k, Q, m, 1.0);
  for (int t = nob - 1; t >= 0; --t) {
    const int P = t * QR_NBO, bo = std::min(QR_NBO, k - P);
    const int RrB = m - P, nc = k - P;
    dcplx* Vblk = Vb.z() + P + (int64_t)m * P;
    dcplx* Tb = Tbig.z() + (size_t)t * QR_NBO * QR_NBO;
    dcplx* Qs = Q + P + (int64_t)m * P;
    gemm_xhv(ctx, nc, bo, RrB, Qs, Vblk, m, Pb.z(), Wb.z());
    apply_block(ctx, RrB, nc, bo, Vblk, m, Tb, bo, OP_N, Wb.z(), Yb.z(), Qs, m);
  }
  scale_q_r(ctx, m, 0, k, Q, m, nullptr, k, ph.z());  // Q columns by phase
}

void qrpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* Q, dcplx* R) {
  qr_factor(ctx, m, n, M, ldm, R, "qr");
  if (Q) qr_form_q(ctx, m, n, Q, "qr");
}

// M (m x n) = L Q  <=>  M^H = Q^H L^H : QRpos of M^H (n x m) gives Q' (n x k), R' (k x m)
void lq_factor(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, const char* slot) {
  const int k = std::min(m, n);
  DevBuf& MH = ctx->buf("lq_mh", (size_t)m * n * sizeof(dcplx));
  DevBuf& Rp = ctx->buf("lq_r", (size_t)k * m * sizeof(dcplx));
  zconj_transpose(ctx, m, n, M, ldm, MH.z(), n);
  qr_factor(ctx, n, m, MH.z(), n, Rp.z(), slot);
  zconj_transpose(ctx, k, m, Rp.z(), k, L, m);  // L = R'^H  (m x k)
}

void lq_form_q(Context* ctx, int m, int n, dcplx* Q, const char* slot) {
  const int k = std::min(m, n);
  DevBuf& Qp = ctx->buf("lq_q", (size_t)n * k * sizeof(dcplx));
  qr_form_q(ctx, n, m, Qp.z(), slot);
  zconj_transpose(ctx, n, k, Qp.z(), n, Q, k);  // Q = Q'^H  (k x n)
}

void lqpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, dcplx* Q) {
  lq_factor(ctx, m, n, M, ldm, L, "qr");
  if (Q) lq_form_q(ctx, m, n, Q, "qr");
}

}  // namespace imps
