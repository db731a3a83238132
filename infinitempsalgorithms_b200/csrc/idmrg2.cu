// Two-site IDMRG (IDMRG2) on the device.
//   sweep   src/algorithms/groundstates/idmrg.jl:113-185 (_localupdate_sweep_idmrg2!)
//   split   idmrg.jl:107-111 (_idmrg2_split: tsvd with truncdim(D), normalize!(s))
//   divs    idmrg.jl:89-95 (_div_tail = A / C, _frontdiv = C \ A)
//   AC2     src/algorithms/groundstates/effective.jl:113-197 (two-site effective Hamiltonian)
//
// The two-site action is the one-site pattern with a second level mix:
//   T1 = GL (Dl m x Dl) x (Dl x d1 d2 Dr)
//   T2[b,u1,s2,c,j]  = sum_{i,s1} W1[i,u1,j,s1] T1[b,i,s1,s2,c]
//   T3[b,u1,u2,c,k]  = sum_{j,s2} W2[j,u2,k,s2] T2[b,u1,s2,c,j]
//   y  = T3 (Dl d1 d2 x Dr n) GR (Dr n x Dr)
// Bond dimensions change at every split (k = min(D, Dl d1, d2 Dr)); the state's and the
// environments' per-bond dimensions are updated as the sweep goes, and each tensor is
// re-allocated to its new shape when it is rewritten.  The whole sweep runs in FP64.
#include "algos.h"
#include "observables.h"

#include <cmath>

namespace imps {
namespace {

// Y = diag(s) X (rows) or X diag(s) (cols), rows x cols column-major, in place allowed
__global__ void k_scale_diag(int rows, int cols, const dcplx* __restrict__ X, int64_t ldx, dcplx* Y, int64_t ldy,
                             const dcplx* __restrict__ s, int by_row) {
  const int64_t tot = (int64_t)rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(t % rows), c = (int)(t / rows);
    const double2 a = s[by_row ? r : c];
    const double2 x = X[r + ldx * c];
    Y[r + ldy * c] = make_double2(a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x);
  }
}

__global__ void k_set_diag(int k, const dcplx* __restrict__ s, dcplx* C) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) C[i + (int64_t)k * i] = s[i];
}

void launched(Context* ctx) {
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string("idmrg2 launch: ") + cudaGetErrorString(e));
}

int grid_for(int64_t t) { return (int)std::max<int64_t>(1, std::min<int64_t>((t + 255) / 256, 148 * 8)); }

void reshape(DevBuf& b, int64_t elems) {
  const size_t bytes = (size_t)elems * sizeof(dcplx);
  if (b.bytes != bytes) b.alloc(bytes);
}

struct Sweep2 {
  Context* ctx;
  imps_envs* E;
  const imps_mpo* H;
  imps_state* st;
  int D;
  double tol;
  int kdim, maxiter;
  bool eager;
  int N;
  // singular values of bonds written by a split in this sweep (empty: C[b] is a general matrix)
  std::vector<std::vector<cplx>> sdiag;

  const MpoSite& W(int l) const { return H->sites[((l % N) + N) % N % H->N]; }

  void scale(int rows, int cols, const dcplx* X, dcplx* Y, const std::vector<cplx>& s, bool by_row) {
    DevBuf& sd = ctx->buf("idmrg2_s", s.size() * sizeof(dcplx));
    upload(ctx, sd.ptr, s.data(), s.size() * sizeof(dcplx));
    const int64_t tot = (int64_t)rows * cols;
    if (tot == 0) return;
    k_scale_diag<<<grid_for(tot), 256, 0, ctx->stream>>>(rows, cols, X, rows, Y, rows, sd.z(), by_row ? 1 : 0);
    launched(ctx);
  }

  void set_bond(int b, int k) {
    b = ((b % N) + N) % N;
    st->chi[b] = k;
    E->Dr[b] = k;
    E->Dl[(b + 1) % N] = k;
  }

  // inverse of a general bond matrix through its SVD: C^{-1} = V diag(1/s) U^H
  void general_inverse(int k, const dcplx* Cm, dcplx* Cinv) {
    DevBuf& U = ctx->buf("idmrg2_inv_u", (size_t)k * k * sizeof(dcplx));
    DevBuf& V = ctx->buf("idmrg2_inv_v", (size_t)k * k * sizeof(dcplx));
    std::vector<double> s;
    const int r = svd_thin(ctx, k, k, Cm, k, k, -1.0, U.z(), s, V.z());
    IMPS_REQUIRE(r == k && s[k - 1] > 0.0, IMPS_INVALID_ARG, "IDMRG2: singular bond matrix");
    std::vector<cplx> inv(k);
    for (int i = 0; i < k; ++i) inv[i] = 1.0 / s[i];
    scale(k, k, V.z(), V.z(), inv, false);
    zgemm_fp64(ctx, OP_N, OP_C, k, k, k, 1.0, V.z(), k, 0, U.z(), k, 0, 0.0, Cinv, k, 0, 1);
  }

  // X = A / C[b] (A: rows x k) or X = C[b] \ A (A: k x cols)
  void divide(int b, bool tail, int other, const dcplx* A, dcplx* X) {
    b = ((b % N) + N) % N;
    const int k = st->chi[b];
    if (!sdiag[b].empty()) {
      std::vector<cplx> inv(k);
      for (int i = 0; i < k; ++i) {
        IMPS_REQUIRE(sdiag[b][i] != cplx(0.0, 0.0), IMPS_INVALID_ARG, "IDMRG2: singular bond matrix");
        inv[i] = 1.0 / sdiag[b][i];
      }
      if (tail) scale(other, k, A, X, inv, false);
      else scale(k, other, A, X, inv, true);
      return;
    }
    DevBuf& Ci = ctx->buf("idmrg2_cinv", (size_t)k * k * sizeof(dcplx));
    general_inverse(k, st->C[b].z(), Ci.z());
    if (tail) zgemm_fp64(ctx, OP_N, OP_N, other, k, k, 1.0, A, other, 0, Ci.z(), k, 0, 0.0, X, other, 0, 1);
    else zgemm_fp64(ctx, OP_N, OP_N, k, other, k, 1.0, Ci.z(), k, 0, A, k, 0, 0.0, X, k, 0, 1);
  }

  // Y = A C[b] (A: rows x k) or Y = C[b] A (A: k x cols)
  void mul_c(int b, bool right, int other, const dcplx* A, dcplx* Y) {
    b = ((b % N) + N) % N;
    const int k = st->chi[b];
    if (!sdiag[b].empty()) {
      if (right) scale(other, k, A, Y, sdiag[b], false);
      else scale(k, other, A, Y, sdiag[b], true);
      return;
    }
    if (right) zgemm_fp64(ctx, OP_N, OP_N, other, k, k, 1.0, A, other, 0, st->C[b].z(), k, 0, 0.0, Y, other, 0, 1);
    else zgemm_fp64(ctx, OP_N, OP_N, k, other, k, 1.0, st->C[b].z(), k, 0, A, k, 0, 0.0, Y, k, 0, 1);
  }

  // lefts[s] = transfer of lefts[s-1] through AL[s-1]; rights[s] = through AR[s+1]
  void tl(int s) {
    s = ((s % N) + N) % N;
    const int sm = (s - 1 + N) % N;
    const int Dl = st->Dl(sm), d = st->d[sm], Dr = st->Dr(sm);
    reshape(E->lefts[s], (int64_t)Dr * E->ml[s] * Dr);
    push_mpo_left(ctx, W(sm), Dl, d, Dr, E->lefts[sm].z(), st->AL[sm].z(), E->lefts[s].z());
    E->GLp_valid[s] = false;
  }
  void tr(int s) {
    s = ((s % N) + N) % N;
    const int q = (s + 1) % N;
    const int Dl = st->Dl(q), d = st->d[q], Dr = st->Dr(q);
    reshape(E->rights[s], (int64_t)Dl * E->nr[s] * Dl);
    push_mpo_right(ctx, W(q), Dl, d, Dr, E->rights[q].z(), st->AR[q].z(), E->rights[s].z());
  }

  // lowest eigenpair of the two-site Hamiltonian of window (p, p+1) from the :ACAR / :ALAC guess
  double solve(int p, bool acar, DevBuf& x) {
    const int q = (p + 1) % N;
    const int Dl = st->Dl(p), k1 = st->Dr(p), Dr = st->Dr(q), d1 = st->d[p], d2 = st->d[q];
    const int64_t n = (int64_t)Dl * d1 * d2 * Dr;
    reshape(x, n);
    const dcplx* A1 = acar ? st->AC[p].z() : st->AL[p].z();
    const dcplx* A2 = acar ? st->AR[q].z() : st->AC[q].z();
    zgemm_fp64(ctx, OP_N, OP_N, Dl * d1, d2 * Dr, k1, 1.0, A1, (int64_t)Dl * d1, 0, A2, k1, 0, 0.0, x.z(),
               (int64_t)Dl * d1, 0, 1);
    ConstScope cs(ctx, {E->lefts[p].ptr, E->rights[q].ptr});
    ProfTag tag(ctx, "eig_ac2");
    LinOp op = [&](const dcplx* v, dcplx* out) { ac2_apply(ctx, E, H, p, v, out); };
    KrylovResult r = lanczos_eigsolve(ctx, n, op, x.z(), x.z(), tol, kdim, maxiter, eager);
    return r.value.real();
  }

  // _idmrg2_split of the window (p, p+1): AL[p] = u, C[p] = diag(s / |s|), AR[p+1] = v
  void split(int p, const DevBuf& x) {
    const int q = (p + 1) % N;
    const int Dl = st->Dl(p), Dr = st->Dr(q), d1 = st->d[p], d2 = st->d[q];
    const int m = Dl * d1, n = d2 * Dr;
    DevBuf& U = ctx->buf("idmrg2_u", (size_t)m * std::min({m, n, D}) * sizeof(dcplx));
    DevBuf& V = ctx->buf("idmrg2_v", (size_t)n * std::min({m, n, D}) * sizeof(dcplx));
    std::vector<double> s;
    ProfTag tag(ctx, "split2");
    const int k = svd_thin(ctx, m, n, x.z(), m, D, -1.0, U.z(), s, V.z());
    double nrm = 0.0;
    for (int i = 0; i < k; ++i) nrm += s[i] * s[i];
    nrm = std::sqrt(nrm);
    IMPS_REQUIRE(nrm > 0.0 && std::isfinite(nrm), IMPS_INVALID_ARG, "IDMRG2: zero or non-finite two-site vector");
    std::vector<cplx> sc(k);
    for (int i = 0; i < k; ++i) sc[i] = s[i] / nrm;
    set_bond(p, k);
    reshape(st->AL[p], (int64_t)m * k);
    zcopy(ctx, (int64_t)m * k, U.z(), st->AL[p].z());
    reshape(st->C[p], (int64_t)k * k);
    zfill(ctx, (int64_t)k * k, 0.0, st->C[p].z());
    DevBuf& sd = ctx->buf("idmrg2_sdiag", (size_t)k * sizeof(dcplx));
    upload(ctx, sd.ptr, sc.data(), (size_t)k * sizeof(dcplx));
    k_set_diag<<<grid_for(k), 256, 0, ctx->stream>>>(k, sd.z(), st->C[p].z());
    launched(ctx);
    reshape(st->AR[q], (int64_t)k * n);
    zconj_transpose(ctx, n, k, V.z(), n, st->AR[q].z(), k);
    sdiag[p] = sc;
  }

  // AC[q] = C[p] AR[q] (the bond left of q);  AC[p] = AL[p] C[p]
  void ac_from_right(int q) {
    q = ((q % N) + N) % N;
    const int b = (q - 1 + N) % N;
    const int64_t cols = (int64_t)st->d[q] * st->Dr(q);
    reshape(st->AC[q], (int64_t)st->Dl(q) * cols);
    mul_c(b, false, (int)cols, st->AR[q].z(), st->AC[q].z());
  }
  void ac_from_left(int p) {
    p = ((p % N) + N) % N;
    const int rows = st->Dl(p) * st->d[p];
    reshape(st->AC[p], (int64_t)rows * st->Dr(p));
    mul_c(p, true, rows, st->AL[p].z(), st->AC[p].z());
  }

  void run(double* Eout, double* epsout) {
    N = st->N;
    sdiag.assign(N, {});
    DevBuf& x = ctx->buf("idmrg2_x", 16);
    // left to right, windows (p, p+1) as :ACAR
    for (int p = 0; p < N - 1; ++p) {
      solve(p, true, x);
      split(p, x);
      ac_from_right(p + 1);
      tl(p + 1);
      tr(p);
    }
    // edge: AL[N-1] = AC[N-1] / C[N-1], AC[0] = AL[0] C[0], wrap window (N-1, 0) as :ALAC
    {
      const int l = N - 1, rows = st->Dl(l) * st->d[l];
      DevBuf& t = ctx->buf("idmrg2_t", (size_t)rows * st->Dr(l) * sizeof(dcplx));
      divide(l, true, rows, st->AC[l].z(), t.z());
      reshape(st->AL[l], (int64_t)rows * st->Dr(l));
      zcopy(ctx, (int64_t)rows * st->Dr(l), t.z(), st->AL[l].z());
      ac_from_left(0);
    }
    solve(N - 1, false, x);
    split(N - 1, x);
    ac_from_left(N - 1);
    ac_from_right(0);
    {
      const int rows = st->Dl(0) * st->d[0];
      reshape(st->AL[0], (int64_t)rows * st->Dr(0));
      divide(0, true, rows, st->AC[0].z(), st->AL[0].z());
    }
    const std::vector<cplx> c_old = sdiag[N - 1];
    tl(0);
    tr(N - 1);
    // right to left, windows (p, p+1) as :ALAC
    for (int p = N - 2; p >= 0; --p) {
      solve(p, false, x);
      split(p, x);
      ac_from_left(p);
      ac_from_right(p + 1);
      tl(p + 1);
      tr(p);
    }
    // edge: AC[N-1] = C[N-2] AR[N-1], AR[0] = C[N-1] \ AC[0], window (N-1, 0) as :ACAR
    ac_from_right(N - 1);
    {
      const int cols = st->d[0] * st->Dr(0);
      reshape(st->AR[0], (int64_t)st->Dl(0) * cols);
      divide(N - 1, false, cols, st->AC[0].z(), st->AR[0].z());
    }
    const double Elast = solve(N - 1, true, x);
    split(N - 1, x);
    {
      // AR[N-1] = C[N-2] \ (AL[N-1] C[N-1])
      const int l = N - 1, rows = st->Dl(l) * st->d[l], k = st->Dr(l);
      DevBuf& t = ctx->buf("idmrg2_t", (size_t)rows * k * sizeof(dcplx));
      mul_c(l, true, rows, st->AL[l].z(), t.z());
      const int cols = st->d[l] * k;
      reshape(st->AR[l], (int64_t)st->Dl(l) * cols);
      divide(N - 2, false, cols, t.z(), st->AR[l].z());
    }
    ac_from_right(0);
    tl(0);
    tr(N - 1);
    // ||C[0] - C_old||_F over the zero-padded diagonals
    double e2 = 0.0;
    const std::vector<cplx>& c_new = sdiag[N - 1];
    for (size_t i = 0; i < std::max(c_new.size(), c_old.size()); ++i) {
      const cplx a = i < c_new.size() ? c_new[i] : cplx(0.0, 0.0);
      const cplx b = i < c_old.size() ? c_old[i] : cplx(0.0, 0.0);
      e2 += std::norm(a - b);
    }
    for (int l = 0; l < N; ++l) E->GLp_valid[l] = false;
    if (epsout) *epsout = std::sqrt(e2);
    if (Eout) *Eout = Elast;
  }
};

}  // namespace

void ac2_apply(Context* ctx, const imps_envs* E, const imps_mpo* H, int p, const dcplx* x, dcplx* y) {
  const int N = E->N;
  const int q = (p + 1) % N;
  const MpoSite& W1 = H->sites[p % H->N];
  const MpoSite& W2 = H->sites[q % H->N];
  const int Dl = E->Dl[p], Dr = E->Dr[q];
  const int m = W1.m, mid = W1.n, n = W2.n, d1 = W1.d, d2 = W2.d;
  IMPS_REQUIRE(m == E->ml[p] && n == E->nr[q] && W2.m == mid, IMPS_DIM_MISMATCH,
               "ac2_apply: MPO levels do not match the environments");
  const int64_t cols = (int64_t)d1 * d2 * Dr;
  DevBuf& T1 = ctx->buf("ac2_t1", (size_t)Dl * m * cols * sizeof(dcplx));
  DevBuf& T2 = ctx->buf("ac2_t2", (size_t)Dl * cols * mid * sizeof(dcplx));
  DevBuf& T3 = ctx->buf("ac2_t3", (size_t)Dl * cols * n * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dl * m, (int)cols, Dl, 1.0, E->lefts[p].z(), (int64_t)Dl * m, 0, x, Dl, 0, 0.0, T1.z(),
        (int64_t)Dl * m, 0, 1);
  auto zero_unhit = [&](const MpoSite& Wx, int levels, dcplx* T) {
    std::vector<bool> hit(levels, false);
    for (auto& b : Wx.nz) hit[b.second] = true;
    for (int j = 0; j < levels; ++j)
      if (!hit[j]) zfill(ctx, (int64_t)Dl * cols, 0.0, T + (int64_t)Dl * cols * j);
  };
  MixPlan p1;
  p1.Db = Dl; p1.R = m; p1.P = d1; p1.Q = mid; p1.S = d1; p1.C = d2 * Dr;
  p1.in_r = Dl; p1.in_s = (int64_t)Dl * m; p1.in_c = (int64_t)Dl * m * d1;
  p1.out_p = Dl; p1.out_q = (int64_t)Dl * cols; p1.out_c = (int64_t)Dl * d1;
  p1.M = W1.Wdev.z();
  p1.nz = W1.nz;
  zero_unhit(W1, mid, T2.z());
  level_mix(ctx, p1, T1.z(), T2.z());
  MixPlan p2;
  p2.Db = Dl * d1; p2.R = mid; p2.P = d2; p2.Q = n; p2.S = d2; p2.C = Dr;
  p2.in_r = (int64_t)Dl * cols; p2.in_s = (int64_t)Dl * d1; p2.in_c = (int64_t)Dl * d1 * d2;
  p2.out_p = (int64_t)Dl * d1; p2.out_q = (int64_t)Dl * cols; p2.out_c = (int64_t)Dl * d1 * d2;
  p2.M = W2.Wdev.z();
  p2.nz = W2.nz;
  zero_unhit(W2, n, T3.z());
  level_mix(ctx, p2, T2.z(), T3.z());
  zgemm(ctx, OP_N, OP_N, Dl * d1 * d2, Dr, Dr * n, 1.0, T3.z(), (int64_t)Dl * d1 * d2, 0, E->rights[q].z(),
        (int64_t)Dr * n, 0, 0.0, y, (int64_t)Dl * d1 * d2, 0, 1);
}

void idmrg2_sweep(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, int D, double tol, int kdim,
                  int maxiter, bool eager, double* Eout, double* epsout) {
  IMPS_REQUIRE(st->N >= 2, IMPS_INVALID_ARG, "IDMRG2 requires unit cell length >= 2");
  IMPS_REQUIRE(D >= 1, IMPS_INVALID_ARG, "IDMRG2: truncation dimension must be positive");
  IMPS_REQUIRE(E->N == st->N, IMPS_DIM_MISMATCH, "state / environment unit cells differ");
  Fp64Scope fp64(ctx);
  Sweep2 s{ctx, E, H, st, D, tol, kdim, maxiter, eager, st->N, {}};
  s.run(Eout, epsout);
}

}  // namespace imps
