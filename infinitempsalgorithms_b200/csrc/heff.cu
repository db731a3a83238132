// Effective Hamiltonians and transfer pushes as GEMM -> level mix -> GEMM.
//
//   AC:  T1 = GL (Dl m x Dl) x (Dl x d Dr)            [effective.jl:90-102]
//        T2[b,u,c,j] = sum_{i,s} W[i,u,j,s] T1[b,i,s,c] (block-sparse level mix)
//        y  = T2 (Dl d x Dr n) GR (Dr n x Dr)
//   C:   U  = x (D x D) GR (D x n D);  y = GLp (D x D n) U (D n x D)   [effective.jl:72-76]
//   pushes: the same two-GEMM pattern with conj(A) on one side    [transfermatrix.jl, envs.jl:104-231]
#include "imps_internal.h"

#include <algorithm>

namespace imps {
namespace {

constexpr int kMaxNz = 256;
constexpr int kMaxQ = 64;

struct MixArgs {
  int Db, R, P, Q, S, Cn;
  int64_t in_r, in_s, in_c, out_p, out_q, out_c;
  double2 scale;
  int nq;
  short qval[kMaxQ];
  short qstart[kMaxQ + 1];
  short rval[kMaxNz];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

template <int P>
__global__ void __launch_bounds__(128) k_level_mix(const MixArgs a, const double2* __restrict__ M,
                                                   const double2* __restrict__ in, double2* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.Db) return;
  for (int c = blockIdx.y; c < a.Cn; c += gridDim.y) {
    const double2* inb = in + b + a.in_c * c;
    double2* outb = out + b + a.out_c * c;
    for (int iq = 0; iq < a.nq; ++iq) {
      const int q = a.qval[iq];
      double2 acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = make_double2(0.0, 0.0);
      for (int t = a.qstart[iq]; t < a.qstart[iq + 1]; ++t) {
        const int r = a.rval[t];
        for (int s = 0; s < a.S; ++s) {
          const double2 v = inb[a.in_r * r + a.in_s * s];
#pragma unroll
          for (int p = 0; p < P; ++p) {
            const double2 w = __ldg(&M[r + (int64_t)a.R * (p + (int64_t)P * (q + (int64_t)a.Q * s))]);
            acc[p].x = fma(w.x, v.x, fma(-w.y, v.y, acc[p].x));
            acc[p].y = fma(w.x, v.y, fma(w.y, v.x, acc[p].y));
          }
        }
      }
#pragma unroll
      for (int p = 0; p < P; ++p) outb[a.out_p * p + a.out_q * q] = cmul(a.scale, acc[p]);
    }
  }
}

__global__ void k_scale_cols_rows(int m, int n, int k, dcplx* Q, int64_t ldq, dcplx* R, int64_t ldr,
                                  const dcplx* __restrict__ ph) {
  // Q[:, i] *= ph[i] (m x k), R[i, :] *= conj(ph[i]) (k x n)
  int64_t tq = (int64_t)m * k, tr = (int64_t)k * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tq + tr; t += (int64_t)gridDim.x * blockDim.x) {
    if (t < tq) {
      int r = (int)(t % m), c = (int)(t / m);
      Q[r + ldq * c] = cmul(ph[c], Q[r + ldq * c]);
    } else {
      int64_t u = t - tq;
      int r = (int)(u % k), c = (int)(u / k);
      double2 p = ph[r];
      R[r + ldr * c] = cmul(make_double2(p.x, -p.y), R[r + ldr * c]);
    }
  }
}

}  // namespace

void level_mix_nz(Context* ctx, const MixPlan& plan, const std::pair<int, int>* nz_in, int nnz, const dcplx* in,
                  dcplx* out) {
  MixArgs a;
  a.Db = plan.Db; a.R = plan.R; a.P = plan.P; a.Q = plan.Q; a.S = plan.S; a.Cn = plan.C;
  a.in_r = plan.in_r; a.in_s = plan.in_s; a.in_c = plan.in_c;
  a.out_p = plan.out_p; a.out_q = plan.out_q; a.out_c = plan.out_c;
  a.scale = make_double2(plan.scale.real(), plan.scale.imag());
  IMPS_REQUIRE(nnz <= kMaxNz, IMPS_INVALID_ARG, "level_mix: too many MPO blocks");
  // group the nonzero (r, q) blocks by q (insertion sort into a fixed array: no heap use)
  std::pair<int, int> nz[kMaxNz];
  for (int t = 0; t < nnz; ++t) {
    std::pair<int, int> v = nz_in[t];
    int u = t;
    while (u > 0 && (nz[u - 1].second > v.second || (nz[u - 1].second == v.second && nz[u - 1].first > v.first))) {
      nz[u] = nz[u - 1];
      --u;
    }
    nz[u] = v;
  }
  a.nq = 0;
  for (int t = 0; t < nnz; ++t) {
    if (a.nq == 0 || a.qval[a.nq - 1] != nz[t].second) {
      IMPS_REQUIRE(a.nq < kMaxQ, IMPS_INVALID_ARG, "level_mix: too many MPO levels");
      a.qval[a.nq] = (short)nz[t].second;
      a.qstart[a.nq] = (short)t;
      a.nq++;
    }
    a.rval[t] = (short)nz[t].first;
  }
  a.qstart[a.nq] = (short)nnz;
  if (a.nq == 0 || plan.Db <= 0 || plan.C <= 0) return;
  dim3 block(128);
  dim3 grid((plan.Db + 127) / 128, std::min(plan.C, 65535));
  double bytes = 16.0 * plan.Db * (double)plan.C * (plan.R * plan.S + plan.P * a.nq);
  ScopedTimer t(ctx, "level_mix", bytes);
  switch (plan.P) {
#define IMPS_MIX_CASE(PP) \
  case PP: k_level_mix<PP><<<grid, block, 0, ctx->stream>>>(a, plan.M, in, out); break;
    IMPS_MIX_CASE(1) IMPS_MIX_CASE(2) IMPS_MIX_CASE(3) IMPS_MIX_CASE(4)
    IMPS_MIX_CASE(5) IMPS_MIX_CASE(6) IMPS_MIX_CASE(7) IMPS_MIX_CASE(8)
#undef IMPS_MIX_CASE
    default: throw Error(IMPS_INVALID_ARG, "level_mix: physical dimension above 8 is not supported");
  }
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("level_mix launch: ") + cudaGetErrorString(e));
}

void level_mix(Context* ctx, const MixPlan& plan, const dcplx* in, dcplx* out) {
  level_mix_nz(ctx, plan, plan.nz.data(), (int)plan.nz.size(), in, out);
}

// Phase fix shared by qrpos/lqpos (see linalg.cu)
void scale_q_r(Context* ctx, int m, int n, int k, dcplx* Q, int64_t ldq, dcplx* R, int64_t ldr, const dcplx* ph) {
  int64_t tot = (int64_t)m * k + (int64_t)k * n;
  int g = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
  k_scale_cols_rows<<<std::max(g, 1), 256, 0, ctx->stream>>>(m, n, k, Q, ldq, R, ldr, ph);
  ctx->n_kernels++;
}

// ---------------------------------------------------------------------------
// AC / C effective Hamiltonians
// ---------------------------------------------------------------------------
void ac_apply(Context* ctx, const imps_envs* envs, const imps_mpo* mpo, int site, const dcplx* x, dcplx* y,
              const MpoSite* Wover, const dcplx* GRover, int64_t GRover_ld) {
  const MpoSite& W = Wover ? *Wover : mpo->sites[site % mpo->N];
  const int Dl = envs->Dl[site], Dr = envs->Dr[site];
  const int m = W.m, d = W.d, n = W.n;
  IMPS_REQUIRE(m == envs->ml[site], IMPS_DIM_MISMATCH, "ac_apply: MPO left levels != environment levels");
  const dcplx* GL = envs->lefts[site].z();
  const dcplx* GR = GRover ? GRover : envs->rights[site].z();
  IMPS_REQUIRE(GRover || n == envs->nr[site], IMPS_DIM_MISMATCH, "ac_apply: MPO right levels != environment");
  const int64_t gr_ld = GRover ? GRover_ld : (int64_t)Dr * n;
  ctx->n_ac_apply++;
  const int64_t t1n = (int64_t)Dl * m * d * Dr, t2n = (int64_t)Dl * d * Dr * n;
  DevBuf& T1 = ctx->buf("ac_t1", t1n * sizeof(dcplx));
  DevBuf& T2 = ctx->buf("ac_t2", t2n * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl * m, d * Dr, Dl, 1.0, GL, (int64_t)Dl * m, 0, x, Dl, 0, 0.0, T1.z(), (int64_t)Dl * m, 0, 1);
  MixPlan pl;
  pl.Db = Dl; pl.R = m; pl.P = d; pl.Q = n; pl.S = d; pl.C = Dr;
  pl.in_r = Dl; pl.in_s = (int64_t)Dl * m; pl.in_c = (int64_t)Dl * m * d;
  pl.out_p = Dl; pl.out_q = (int64_t)Dl * d * Dr; pl.out_c = (int64_t)Dl * d;
  pl.M = W.Wdev.z();
  pl.nz = W.nz;
  // levels q without any nonzero block must read as zero in the second GEMM
  {
    std::vector<bool> hit(n, false);
    for (auto& b : W.nz) hit[b.second] = true;
    for (int q = 0; q < n; ++q)
      if (!hit[q]) zfill(ctx, (int64_t)Dl * d * Dr, 0.0, T2.z() + (int64_t)Dl * d * Dr * q);
  }
  level_mix(ctx, pl, T1.z(), T2.z());
  zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr * n, 1.0, T2.z(), (int64_t)Dl * d, 0, GR, gr_ld, 0, 0.0, y,
        (int64_t)Dl * d, 0, 1);
}

void ensure_GLp(Context* ctx, imps_envs* envs, int l) {
  if (envs->GLp_valid[l]) return;
  const int D = envs->Dl[l], w = envs->ml[l];
  envs->GLp[l].ensure((size_t)D * D * w * sizeof(dcplx));
  // GLp[a + D (a' + D w)] = GL[a, w, a'] via the level mix with an identity level map
  DevBuf& Id = ctx->buf("glp_id", (size_t)w * w * sizeof(dcplx));
  std::vector<cplx> idh((size_t)w * w, cplx(0.0, 0.0));
  for (int i = 0; i < w; ++i) idh[i + (size_t)w * i] = 1.0;
  upload(ctx, Id.ptr, idh.data(), idh.size() * sizeof(dcplx));
  MixPlan pl;
  pl.Db = D; pl.R = w; pl.P = 1; pl.Q = w; pl.S = 1; pl.C = D;
  pl.in_r = D; pl.in_s = 0; pl.in_c = (int64_t)D * w;
  pl.out_p = 0; pl.out_q = (int64_t)D * D; pl.out_c = D;
  pl.M = Id.z();
  for (int i = 0; i < w; ++i) pl.nz.push_back({i, i});
  level_mix(ctx, pl, envs->lefts[l].z(), envs->GLp[l].z());
  envs->GLp_valid[l] = true;
}

void c_apply(Context* ctx, imps_envs* envs, int site, const dcplx* x, dcplx* y) {
  const int N = envs->N;
  const int l1 = (site + 1) % N;
  const int D = envs->Dr[site];
  const int w = envs->nr[site];
  IMPS_REQUIRE(envs->Dl[l1] == D && envs->ml[l1] == w, IMPS_DIM_MISMATCH, "c_apply: environment shapes disagree");
  ensure_GLp(ctx, envs, l1);
  ctx->n_c_apply++;
  DevBuf& U = ctx->buf("c_u", (size_t)D * D * w * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, D, w * D, D, 1.0, x, D, 0, envs->rights[site].z(), D, 0, 0.0, U.z(), D, 0, 1);
  zgemm(ctx, OP_N, OP_N, D, D, D * w, 1.0, envs->GLp[l1].z(), D, 0, U.z(), (int64_t)D * w, 0, 0.0, y, D, 0, 1);
}

// ---------------------------------------------------------------------------
// Transfer pushes
// ---------------------------------------------------------------------------
void push_left_id(Context* ctx, int Dl, int d, int Dr, const dcplx* L, const dcplx* above, const dcplx* below,
                  dcplx* out) {
  ctx->n_push++;
  DevBuf& Y = ctx->buf("push_y", (size_t)Dl * d * Dr * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl, d * Dr, Dl, 1.0, L, Dl, 0, above, Dl, 0, 0.0, Y.z(), Dl, 0, 1);
  zgemm(ctx, OP_C, OP_N, Dr, Dr, Dl * d, 1.0, below, (int64_t)Dl * d, 0, Y.z(), (int64_t)Dl * d, 0, 0.0, out, Dr, 0, 1);
}

void push_right_id(Context* ctx, int Dl, int d, int Dr, const dcplx* R, const dcplx* above, const dcplx* below,
                   dcplx* out) {
  ctx->n_push++;
  DevBuf& Y = ctx->buf("push_y", (size_t)Dl * d * Dr * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, 1.0, above, (int64_t)Dl * d, 0, R, Dr, 0, 0.0, Y.z(), (int64_t)Dl * d, 0, 1);
  zgemm(ctx, OP_N, OP_C, Dl, Dl, d * Dr, 1.0, Y.z(), Dl, 0, below, Dl, 0, 0.0, out, Dl, 0, 1);
}

void push_left_levels(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* L, int64_t L_level_stride,
                      int64_t L_ld, const std::vector<std::pair<int, int>>& blocks, int q_count,
                      const std::vector<int>& q_targets, const dcplx* A, dcplx* out, int64_t out_level_stride,
                      int64_t out_ld, bool accumulate) {
  (void)q_count;
  if (blocks.empty()) return;
  ctx->n_push++;
  std::vector<int> ls;
  for (auto& b : blocks) ls.push_back(b.first);
  std::sort(ls.begin(), ls.end());
  ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
  const int64_t ysz = (int64_t)Dl * d * Dr;
  DevBuf& Y = ctx->buf("pushl_y", (size_t)ysz * W.m * sizeof(dcplx));
  DevBuf& Z = ctx->buf("pushl_z", (size_t)ysz * W.n * sizeof(dcplx));
  for (int l : ls)
    zgemm(ctx, OP_N, OP_N, Dl, d * Dr, Dl, 1.0, L + L_level_stride * l, L_ld, 0, A, Dl, 0, 0.0, Y.z() + ysz * l, Dl,
          0, 1);
  MixPlan pl;
  pl.Db = Dl; pl.R = W.m; pl.P = d; pl.Q = W.n; pl.S = d; pl.C = Dr;
  pl.in_r = ysz; pl.in_s = Dl; pl.in_c = (int64_t)Dl * d;
  pl.out_p = Dl; pl.out_q = ysz; pl.out_c = (int64_t)Dl * d;
  pl.M = W.Wdev.z();
  pl.nz = blocks;
  level_mix(ctx, pl, Y.z(), Z.z());
  for (int q : q_targets) {
    bool any = false;
    for (auto& b : blocks) any |= (b.second == q);
    if (!any) continue;
    zgemm(ctx, OP_C, OP_N, Dr, Dr, Dl * d, 1.0, A, (int64_t)Dl * d, 0, Z.z() + ysz * q, (int64_t)Dl * d, 0,
          accumulate ? 1.0 : 0.0, out + out_level_stride * q, out_ld, 0, 1);
  }
}

void push_right_levels(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* R,
                       int64_t R_level_stride, int64_t R_ld, const std::vector<std::pair<int, int>>& blocks,
                       const std::vector<int>& q_targets, const dcplx* A, dcplx* out, int64_t out_level_stride,
                       int64_t out_ld, bool accumulate) {
  // out_i = sum_{(i,l)} push_slice_right(R_l, W[i,:,l,:], A); blocks are (i, l) pairs
  if (blocks.empty()) return;
  ctx->n_push++;
  std::vector<int> ls;
  for (auto& b : blocks) ls.push_back(b.second);
  std::sort(ls.begin(), ls.end());
  ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
  const int64_t ysz = (int64_t)Dl * d * Dr;
  DevBuf& Y = ctx->buf("pushr_y", (size_t)ysz * W.n * sizeof(dcplx));
  DevBuf& Z = ctx->buf("pushr_z", (size_t)ysz * W.m * sizeof(dcplx));
  for (int l : ls)
    zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, 1.0, A, (int64_t)Dl * d, 0, R + R_level_stride * l, R_ld, 0, 0.0,
          Y.z() + ysz * l, (int64_t)Dl * d, 0, 1);
  // Z_i[a', u, b] = sum_{l, s} W[i, u, l, s] Y_l[a', s, b]: mixing over the transposed tensor
  MixPlan pl;
  pl.Db = Dl; pl.R = W.n; pl.P = d; pl.Q = W.m; pl.S = d; pl.C = Dr;
  pl.in_r = ysz; pl.in_s = Dl; pl.in_c = (int64_t)Dl * d;
  pl.out_p = Dl; pl.out_q = ysz; pl.out_c = (int64_t)Dl * d;
  pl.M = W.Wdev.z() + (int64_t)W.m * W.d * W.n * W.d;  // transposed copy Wt[j,u,i,s] = W[i,u,j,s]
  for (auto& b : blocks) pl.nz.push_back({b.second, b.first});
  level_mix(ctx, pl, Y.z(), Z.z());
  for (int q : q_targets) {
    bool any = false;
    for (auto& b : blocks) any |= (b.first == q);
    if (!any) continue;
    zgemm(ctx, OP_N, OP_C, Dl, Dl, d * Dr, 1.0, Z.z() + ysz * q, Dl, 0, A, Dl, 0, accumulate ? 1.0 : 0.0,
          out + out_level_stride * q, out_ld, 0, 1);
  }
}

void push_mpo_left(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* L, const dcplx* A, dcplx* out) {
  ctx->n_push++;
  const int m = W.m, n = W.n;
  DevBuf& Y = ctx->buf("ac_t1", (size_t)Dl * m * d * Dr * sizeof(dcplx));
  DevBuf& Z = ctx->buf("ac_t2", (size_t)Dl * d * n * Dr * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl * m, d * Dr, Dl, 1.0, L, (int64_t)Dl * m, 0, A, Dl, 0, 0.0, Y.z(), (int64_t)Dl * m, 0, 1);
  MixPlan pl;
  pl.Db = Dl; pl.R = m; pl.P = d; pl.Q = n; pl.S = d; pl.C = Dr;
  pl.in_r = Dl; pl.in_s = (int64_t)Dl * m; pl.in_c = (int64_t)Dl * m * d;
  pl.out_p = Dl; pl.out_q = (int64_t)Dl * d; pl.out_c = (int64_t)Dl * d * n;
  pl.M = W.Wdev.z();
  pl.nz = W.nz;
  std::vector<bool> hit(n, false);
  for (auto& b : W.nz) hit[b.second] = true;
  bool any_missing = false;
  for (int q = 0; q < n; ++q) any_missing |= !hit[q];
  if (any_missing) zfill(ctx, (int64_t)Dl * d * n * Dr, 0.0, Z.z());
  level_mix(ctx, pl, Y.z(), Z.z());
  zgemm(ctx, OP_C, OP_N, Dr, n * Dr, Dl * d, 1.0, A, (int64_t)Dl * d, 0, Z.z(), (int64_t)Dl * d, 0, 0.0, out, Dr, 0, 1);
}

void push_mpo_right(Context* ctx, const MpoSite& W, int Dl, int d, int Dr, const dcplx* R, const dcplx* A,
                    dcplx* out) {
  ctx->n_push++;
  const int m = W.m, n = W.n;
  DevBuf& Y = ctx->buf("ac_t1", (size_t)Dl * d * n * Dr * sizeof(dcplx));
  DevBuf& Z = ctx->buf("ac_t2", (size_t)Dl * m * d * Dr * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl * d, n * Dr, Dr, 1.0, A, (int64_t)Dl * d, 0, R, Dr, 0, 0.0, Y.z(), (int64_t)Dl * d, 0, 1);
  MixPlan pl;
  pl.Db = Dl; pl.R = n; pl.P = d; pl.Q = m; pl.S = d; pl.C = Dr;
  pl.in_r = (int64_t)Dl * d; pl.in_s = Dl; pl.in_c = (int64_t)Dl * d * n;
  pl.out_p = (int64_t)Dl * m; pl.out_q = Dl; pl.out_c = (int64_t)Dl * m * d;
  pl.M = W.Wdev.z() + (int64_t)W.m * W.d * W.n * W.d;
  for (auto& b : W.nz) pl.nz.push_back({b.second, b.first});
  std::vector<bool> hit(m, false);
  for (auto& b : W.nz) hit[b.first] = true;
  bool any_missing = false;
  for (int q = 0; q < m; ++q) any_missing |= !hit[q];
  if (any_missing) zfill(ctx, (int64_t)Dl * m * d * Dr, 0.0, Z.z());
  level_mix(ctx, pl, Y.z(), Z.z());
  zgemm(ctx, OP_N, OP_C, Dl * m, Dl, d * Dr, 1.0, Z.z(), (int64_t)Dl * m, 0, A, Dl, 0, 0.0, out, (int64_t)Dl * m, 0, 1);
}

}  // namespace imps
