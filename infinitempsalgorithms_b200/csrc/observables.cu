// Dense-MPO channel environments, two-point correlators and the entanglement
// spectrum on the device:
//   dominant_env          envs.jl:34-99 (identity or dense-MPO transfer matrix of one
//                         unit cell, :LM Arnoldi from v0 = ones, unit norm)
//   envs_build_dense      DMRGCache(psi, ::DenseIMPO), envs.jl:284-304, with
//                         normalize_envs! (envs.jl:559-584)
//   energy_dense          expectationvalue(psi, ::DenseIMPO, envs), expval.jl:60-79
//   correlator            correlators.jl:13-42
//   entanglement_spectrum toolbox.jl:9-14: singular values of C[loc] by one-sided
//                         (Hestenes) Jacobi rotations, all column pairs of a round
//                         rotated in parallel (round-robin schedule), one CTA per pair
#include "observables.h"

#include <algorithm>
#include <cmath>

#include "gauge.h"

namespace imps {
namespace {

constexpr int kJacThreads = 256;

__device__ __forceinline__ double block_sum256(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  for (int q = 0; q < kJacThreads / 32; ++q) r += sh[q];
  __syncthreads();
  return r;
}

// Player at position `pos` of round `r` in the round-robin schedule of P (even)
// players: position 0 is fixed, the other P-1 rotate by one per round.
__device__ __forceinline__ int rr_player(int pos, int r, int P) {
  return pos == 0 ? 0 : ((pos - 1 + r) % (P - 1)) + 1;
}

// One round of one-sided Jacobi: CTA k orthogonalises columns (a, b) = players at
// positions k and P-1-k.  Columns >= ncol are zero padding (never rotated).  With
// gamma = u_a^H u_b = |gamma| e^{i phi}, the real Jacobi rotation of the Gram matrix
// [[alpha, |gamma|], [|gamma|, beta]] applied to (u_a, e^{-i phi} u_b) makes them
// orthogonal.  *rot counts the rotations performed (the convergence test of a sweep).
__global__ void __launch_bounds__(kJacThreads) k_jacobi_round(int n, int ncol, int P, int r, dcplx* __restrict__ U,
                                                          int64_t ldu, double tol, int* __restrict__ rot,
                                                          dcplx* __restrict__ V, int nv, int64_t ldv) {
  __shared__ double sh[kJacThreads / 32];
  const int k = blockIdx.x;
  int a = rr_player(k, r, P), b = rr_player(P - 1 - k, r, P);
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  if (b >= ncol) return;
  dcplx* ua = U + ldu * (int64_t)a;
  dcplx* ub = U + ldu * (int64_t)b;
  double al = 0.0, be = 0.0, gr = 0.0, gi = 0.0;
  for (int i = threadIdx.x; i < n; i += kJacThreads) {
    const dcplx x = ua[i], y = ub[i];
    al = fma(x.x, x.x, fma(x.y, x.y, al));
    be = fma(y.x, y.x, fma(y.y, y.y, be));
    gr = fma(x.x, y.x, fma(x.y, y.y, gr));   // Re conj(x) y
    gi = fma(x.x, y.y, fma(-x.y, y.x, gi));  // Im conj(x) y
  }
  al = block_sum256(al, sh);
  be = block_sum256(be, sh);
  gr = block_sum256(gr, sh);
  gi = block_sum256(gi, sh);
  const double g = hypot(gr, gi);
  if (!(g > tol * sqrt(al * be)) || g == 0.0) return;
  const double zeta = (be - al) / (2.0 * g);
  const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
  const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
  const double er = gr / g, ei = gi / g;  // e^{i phi}
  for (int i = threadIdx.x; i < n; i += kJacThreads) {
    const dcplx x = ua[i], y = ub[i];
    // y' = e^{-i phi} y
    const double ypr = er * y.x + ei * y.y, ypi = er * y.y - ei * y.x;
    const double nxr = c * x.x - s * ypr, nxi = c * x.y - s * ypi;
    const double nyr = s * x.x + c * ypr, nyi = s * x.y + c * ypi;
    ua[i] = make_double2(nxr, nxi);
    // back to the original phase of column b: e^{i phi} y''
    ub[i] = make_double2(er * nyr - ei * nyi, er * nyi + ei * nyr);
  }
  // the same rotation on the columns of V (right singular vectors), if requested
  if (V) {
    dcplx* va = V + ldv * (int64_t)a;
    dcplx* vb = V + ldv * (int64_t)b;
    for (int i = threadIdx.x; i < nv; i += kJacThreads) {
      const dcplx x = va[i], y = vb[i];
      const double ypr = er * y.x + ei * y.y, ypi = er * y.y - ei * y.x;
      const double nxr = c * x.x - s * ypr, nxi = c * x.y - s * ypi;
      const double nyr = s * x.x + c * ypr, nyi = s * x.y + c * ypi;
      va[i] = make_double2(nxr, nxi);
      vb[i] = make_double2(er * nyr - ei * nyi, er * nyi + ei * nyr);
    }
  }
  if (threadIdx.x == 0) atomicAdd(rot, 1);
}

// out[:, j] = scale_j * in[:, perm[j]] for j < k (column gather with optional scaling)
__global__ void k_gather_cols(int rows, int k, const dcplx* __restrict__ in, int64_t ldi, const int* __restrict__ perm,
                              const double* __restrict__ scale, dcplx* __restrict__ out, int64_t ldo) {
  const int64_t tot = (int64_t)rows * k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % rows), j = (int)(t / rows);
    const dcplx v = in[i + ldi * (int64_t)perm[j]];
    const double f = scale ? scale[j] : 1.0;
    out[i + ldo * (int64_t)j] = make_double2(v.x * f, v.y * f);
  }
}

__global__ void k_col_norms2(int n, int ncol, const dcplx* __restrict__ U, int64_t ldu, double* __restrict__ out) {
  __shared__ double sh[kJacThreads / 32];
  const int j = blockIdx.x;
  if (j >= ncol) return;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kJacThreads) {
    const dcplx x = U[i + ldu * (int64_t)j];
    s = fma(x.x, x.x, fma(x.y, x.y, s));
  }
  s = block_sum256(s, sh);
  if (threadIdx.x == 0) out[j] = s;
}

void check(Context* ctx) {
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("observables launch: ") + cudaGetErrorString(e));
}

}  // namespace

std::vector<double> singular_values_sq(Context* ctx, int m, int n, const dcplx* A, int64_t lda) {
  IMPS_REQUIRE(m > 0 && n > 0, IMPS_INVALID_ARG, "singular values: empty matrix");
  const int P = n + (n & 1);
  DevBuf& U = ctx->buf("jac_u", (size_t)m * P * sizeof(dcplx));
  DevBuf& flag = ctx->buf("jac_flag", 64);
  DevBuf& nr = ctx->buf("jac_norms", (size_t)P * sizeof(double));
  zcopy2d(ctx, m, n, A, lda, U.z(), m);
  ScopedTimer tm(ctx, "jacobi_svd", 0.0);
  const double tol = 1e-15 * std::sqrt((double)m);
  for (int sweep = 0; sweep < 60; ++sweep) {
    IMPS_CUDA(cudaMemsetAsync(flag.ptr, 0, sizeof(int), ctx->stream));
    for (int r = 0; r < P - 1; ++r) {
      k_jacobi_round<<<P / 2, kJacThreads, 0, ctx->stream>>>(m, n, P, r, U.z(), m, tol, static_cast<int*>(flag.ptr),
                                                             nullptr, 0, 0);
      check(ctx);
    }
    int rot = 0;
    download(ctx, &rot, flag.ptr, sizeof(int));
    if (rot == 0) break;
  }
  k_col_norms2<<<n, kJacThreads, 0, ctx->stream>>>(m, n, U.z(), m, nr.d());
  check(ctx);
  std::vector<double> s2(n);
  download(ctx, s2.data(), nr.ptr, n * sizeof(double));
  std::sort(s2.begin(), s2.end(), [](double x, double y) { return x > y; });
  return s2;
}

int svd_thin(Context* ctx, int m, int n, const dcplx* A, int64_t lda, int kmax, double cutoff, dcplx* U,
             std::vector<double>& s, dcplx* V) {
  IMPS_REQUIRE(m > 0 && n > 0, IMPS_INVALID_ARG, "svd: empty matrix");
  if (m < n) {
    // A = (A^H)^H: the SVD of A^H with the roles of U and V exchanged
    DevBuf& AH = ctx->buf("svd_ah", (size_t)m * n * sizeof(dcplx));
    zconj_transpose(ctx, m, n, A, lda, AH.z(), n);
    DevBuf& Ut = ctx->buf("svd_ut", (size_t)n * std::min(m, kmax > 0 ? kmax : m) * sizeof(dcplx));
    const int k = svd_thin(ctx, n, m, AH.z(), n, kmax, cutoff, Ut.z(), s, U);
    // V = U' (n x k) of the transposed problem
    zcopy2d(ctx, n, k, Ut.z(), n, V, n);
    return k;
  }
  const int P = n + (n & 1);
  DevBuf& W = ctx->buf("svd_w", (size_t)m * P * sizeof(dcplx));
  DevBuf& Vw = ctx->buf("svd_v", (size_t)n * P * sizeof(dcplx));
  DevBuf& flag = ctx->buf("jac_flag", 64);
  DevBuf& nr = ctx->buf("jac_norms", (size_t)P * sizeof(double));
  zcopy2d(ctx, m, n, A, lda, W.z(), m);
  zset_identity(ctx, n, Vw.z(), n, 1.0);
  ScopedTimer tm(ctx, "jacobi_svd", 0.0);
  const double tol = 1e-15 * std::sqrt((double)m);
  for (int sweep = 0; sweep < 60; ++sweep) {
    IMPS_CUDA(cudaMemsetAsync(flag.ptr, 0, sizeof(int), ctx->stream));
    for (int r = 0; r < P - 1; ++r) {
      k_jacobi_round<<<P / 2, kJacThreads, 0, ctx->stream>>>(m, n, P, r, W.z(), m, tol, static_cast<int*>(flag.ptr),
                                                             Vw.z(), n, n);
      check(ctx);
    }
    int rot = 0;
    download(ctx, &rot, flag.ptr, sizeof(int));
    if (rot == 0) break;
  }
  k_col_norms2<<<n, kJacThreads, 0, ctx->stream>>>(m, n, W.z(), m, nr.d());
  check(ctx);
  std::vector<double> n2(n);
  download(ctx, n2.data(), nr.ptr, n * sizeof(double));
  std::vector<int> perm(n);
  for (int j = 0; j < n; ++j) perm[j] = j;
  std::stable_sort(perm.begin(), perm.end(), [&](int x, int y) { return n2[x] > n2[y]; });
  int k = kmax > 0 ? std::min(kmax, n) : n;
  while (k > 1 && std::sqrt(std::max(n2[perm[k - 1]], 0.0)) <= cutoff) --k;
  s.resize(k);
  std::vector<double> inv(k);
  for (int j = 0; j < k; ++j) {
    s[j] = std::sqrt(std::max(n2[perm[j]], 0.0));
    inv[j] = s[j] > 0.0 ? 1.0 / s[j] : 0.0;
  }
  // the doubles first: an int array of odd length before them would misalign them
  DevBuf& pb = ctx->buf("svd_perm", (size_t)k * (sizeof(int) + sizeof(double)));
  double* sd = static_cast<double*>(pb.ptr);
  int* pd = reinterpret_cast<int*>(static_cast<char*>(pb.ptr) + (size_t)k * sizeof(double));
  upload(ctx, pd, perm.data(), (size_t)k * sizeof(int));
  upload(ctx, sd, inv.data(), (size_t)k * sizeof(double));
  auto grid = [](int64_t t) { return (int)std::max<int64_t>(1, std::min<int64_t>((t + 255) / 256, 148 * 8)); };
  // U = W[:, perm] / s (columns of exactly zero singular value stay zero), V = Vw[:, perm]
  k_gather_cols<<<grid((int64_t)m * k), 256, 0, ctx->stream>>>(m, k, W.z(), m, pd, sd, U, m);
  check(ctx);
  k_gather_cols<<<grid((int64_t)n * k), 256, 0, ctx->stream>>>(n, k, Vw.z(), n, pd, nullptr, V, n);
  check(ctx);
  return k;
}

std::vector<double> entanglement_spectrum(Context* ctx, imps_state* st, int bond) {
  Fp64Scope fp64(ctx);
  const int b = ((bond % st->N) + st->N) % st->N;
  const int D = st->Dr(b);
  std::vector<double> p = singular_values_sq(ctx, D, D, st->C[b].z(), D);
  double tot = 0.0;
  for (double v : p) tot += v;
  IMPS_REQUIRE(tot > 0.0, IMPS_INVALID_ARG, "entanglement spectrum: zero center matrix");
  for (double& v : p) v /= tot;
  return p;
}

KrylovResult dominant_env(Context* ctx, imps_state* st, const imps_mpo* mpo, int side, double tol, int krylovdim,
                          int maxiter, dcplx* out) {
  Fp64Scope fp64(ctx);
  const int N = st->N;
  const int D = st->Dl(0);
  const int w = mpo ? mpo->sites[0].m : 1;
  const int64_t n = (int64_t)D * w * D;
  DevBuf& a = ctx->buf("domenv_a", (size_t)n * sizeof(dcplx));
  DevBuf& b = ctx->buf("domenv_b", (size_t)n * sizeof(dcplx));
  DevBuf& v0 = ctx->buf("domenv_v0", (size_t)n * sizeof(dcplx));
  LinOp op = [&](const dcplx* v, dcplx* o) {
    const dcplx* cur = v;
    for (int k = 0; k < N; ++k) {
      const int l = side == 0 ? k : N - 1 - k;
      dcplx* dst = (k == N - 1) ? o : ((k % 2 == 0) ? a.z() : b.z());
      const int Dl = st->Dl(l), d = st->d[l], Dr = st->Dr(l);
      if (!mpo) {
        if (side == 0) push_left_id(ctx, Dl, d, Dr, cur, st->AL[l].z(), st->AL[l].z(), dst);
        else push_right_id(ctx, Dl, d, Dr, cur, st->AR[l].z(), st->AR[l].z(), dst);
      } else {
        const MpoSite& W = mpo->sites[l % mpo->N];
        if (side == 0) push_mpo_left(ctx, W, Dl, d, Dr, cur, st->AL[l].z(), dst);
        else push_mpo_right(ctx, W, Dl, d, Dr, cur, st->AR[l].z(), dst);
      }
      cur = dst;
    }
  };
  zfill(ctx, n, cplx(1.0, 0.0), v0.z());
  KrylovResult r = arnoldi_dominant(ctx, n, op, v0.z(), out, tol, krylovdim, maxiter, true);
  const double nv = dznrm2(ctx, n, out);
  zscal(ctx, n, 1.0 / nv, out);
  return r;
}

KrylovResult envs_build_dense(Context* ctx, imps_envs* envs, imps_state* st, const imps_mpo* mpo, double tol,
                              int krylovdim, int maxiter) {
  Fp64Scope fp64(ctx);
  const int N = st->N;
  IMPS_REQUIRE(envs->N == N && mpo->N > 0 && N % mpo->N == 0, IMPS_DIM_MISMATCH,
               "dense environments: unit cells of state, MPO and environments differ");
  KrylovResult rl = dominant_env(ctx, st, mpo, 0, tol, krylovdim, maxiter, envs->lefts[0].z());
  KrylovResult rr = dominant_env(ctx, st, mpo, 1, tol, krylovdim, maxiter, envs->rights[N - 1].z());
  for (int l = 1; l < N; ++l)
    push_mpo_left(ctx, mpo->sites[(l - 1) % mpo->N], st->Dl(l - 1), st->d[l - 1], st->Dr(l - 1),
                  envs->lefts[l - 1].z(), st->AL[l - 1].z(), envs->lefts[l].z());
  for (int l = N - 2; l >= 0; --l)
    push_mpo_right(ctx, mpo->sites[(l + 1) % mpo->N], st->Dl(l + 1), st->d[l + 1], st->Dr(l + 1),
                   envs->rights[l + 1].z(), st->AR[l + 1].z(), envs->rights[l].z());
  for (int l = 0; l < N; ++l) envs->GLp_valid[l] = false;
  // normalize_envs!: unit-norm right environments, lefts[i+1] /= <C_i, H_C(i) C_i>
  for (int i = 0; i < N; ++i) {
    const int64_t nr = (int64_t)envs->Dr[i] * envs->nr[i] * envs->Dr[i];
    const double rn = dznrm2(ctx, nr, envs->rights[i].z());
    if (rn > 0) zscal(ctx, nr, 1.0 / rn, envs->rights[i].z());
    const int D = st->Dr(i);
    DevBuf& hc = ctx->buf("dense_hc", (size_t)D * D * sizeof(dcplx));
    c_apply(ctx, envs, i, st->C[i].z(), hc.z());
    const cplx lam = zdotc(ctx, (int64_t)D * D, st->C[i].z(), hc.z());
    if (std::abs(lam) > 0) {
      const int l1 = (i + 1) % N;
      const int64_t nl = (int64_t)envs->Dl[l1] * envs->ml[l1] * envs->Dl[l1];
      zscal(ctx, nl, 1.0 / lam, envs->lefts[l1].z());
      envs->GLp_valid[l1] = false;
    }
  }
  envs->version++;
  KrylovResult r;
  r.converged = rl.converged && rr.converged;
  r.numops = rl.numops + rr.numops;
  r.numiter = rl.numiter + rr.numiter;
  r.normres = std::max(rl.normres, rr.normres);
  r.value = rl.value;
  return r;
}

cplx energy_dense(Context* ctx, imps_envs* envs, const imps_mpo* mpo, imps_state* st) {
  Fp64Scope fp64(ctx);
  cplx E = 0.0;
  for (int i = 0; i < st->N; ++i) {
    const int64_t n = st->site_elems(i);
    DevBuf& y = ctx->buf("dense_e", (size_t)n * sizeof(dcplx));
    ac_apply(ctx, envs, mpo, i, st->AC[i].z(), y.z());
    E += zdotc(ctx, n, st->AC[i].z(), y.z());
  }
  return E / state_dot(ctx, st);
}

void apply_local(Context* ctx, int Dl, int d, int Dr, const dcplx* O_dev, const dcplx* A, dcplx* out) {
  // out[:, :, b] = A[:, :, b] O^T  (out[a, u, b] = sum_s O[u, s] A[a, s, b])
  zgemm_fp64(ctx, OP_N, OP_T, Dl, d, d, 1.0, A, Dl, (int64_t)Dl * d, O_dev, d, 0, 0.0, out, Dl, (int64_t)Dl * d, Dr);
}

std::vector<cplx> correlator(Context* ctx, imps_state* st, const cplx* O1, const cplx* O2, int i,
                             const std::vector<int>& js) {
  Fp64Scope fp64(ctx);
  const int N = st->N;
  IMPS_REQUIRE(!js.empty() && js[0] > i, IMPS_INVALID_ARG, "correlator: i should be smaller than j");
  for (size_t k = 1; k < js.size(); ++k)
    IMPS_REQUIRE(js[k] > js[k - 1], IMPS_INVALID_ARG, "correlator: js must increase");
  auto site = [&](int l) { return ((l - 1) % N + N) % N; };  // 1-based -> 0-based periodic
  const int si = site(i);
  const int dmax = *std::max_element(st->d.begin(), st->d.end());
  DevBuf& Od = ctx->buf("corr_o", (size_t)2 * dmax * dmax * sizeof(dcplx));
  const int d1 = st->d[si];
  upload(ctx, Od.ptr, O1, (size_t)d1 * d1 * sizeof(dcplx));
  size_t mx = 0;
  int Dmax = 0;
  for (int l = 0; l < N; ++l) {
    mx = std::max(mx, st->site_elems(l));
    Dmax = std::max(Dmax, std::max(st->Dl(l), st->Dr(l)));
  }
  DevBuf& OA = ctx->buf("corr_oa", mx * sizeof(dcplx));
  DevBuf& Va = ctx->buf("corr_va", (size_t)Dmax * Dmax * sizeof(dcplx));
  DevBuf& Vb = ctx->buf("corr_vb", (size_t)Dmax * Dmax * sizeof(dcplx));
  DevBuf& Ib = ctx->buf("corr_id", (size_t)Dmax * Dmax * sizeof(dcplx));
  DevBuf& E = ctx->buf("corr_e", (size_t)Dmax * Dmax * sizeof(dcplx));
  // V = push_env_left(I, O1 AC_i, AC_i)
  {
    const int Dl = st->Dl(si), Dr = st->Dr(si);
    zset_identity(ctx, Dl, Ib.z(), Dl, 1.0);
    apply_local(ctx, Dl, d1, Dr, Od.z(), st->AC[si].z(), OA.z());
    push_left_id(ctx, Dl, d1, Dr, Ib.z(), OA.z(), st->AC[si].z(), Va.z());
  }
  dcplx* V = Va.z();
  dcplx* Vn = Vb.z();
  std::vector<cplx> out(js.size());
  int ctr = i;
  for (size_t k = 0; k < js.size(); ++k) {
    const int j = js[k];
    for (int l = ctr + 1; l <= j - 1; ++l) {
      const int s = site(l);
      push_left_id(ctx, st->Dl(s), st->d[s], st->Dr(s), V, st->AR[s].z(), st->AR[s].z(), Vn);
      std::swap(V, Vn);
    }
    const int sj = site(j);
    const int Dl = st->Dl(sj), d = st->d[sj], Dr = st->Dr(sj);
    upload(ctx, Od.z() + dmax * dmax, O2, (size_t)d * d * sizeof(dcplx));
    apply_local(ctx, Dl, d, Dr, Od.z() + dmax * dmax, st->AR[sj].z(), OA.z());
    push_left_id(ctx, Dl, d, Dr, V, OA.z(), st->AR[sj].z(), E.z());
    zset_identity(ctx, Dr, Ib.z(), Dr, 1.0);
    out[k] = ztrace_prod(ctx, Dr, E.z(), Dr, Ib.z(), Dr);
    ctr = j;  // as the reference (correlators.jl:34): the next j transfers from ctr + 1
  }
  const cplx nrm = state_dot(ctx, st);
  for (auto& v : out) v /= nrm;
  return out;
}

}  // namespace imps
