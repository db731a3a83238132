// Krylov solvers with the basis in HBM and the small projected problems in
// FP64 on the host (smallla.cu).  Orthogonalisation is classical Gram-Schmidt
// with one re-orthogonalisation pass (CGS2): two fused multi-dot passes and two
// multi-axpy passes over the basis per expansion, all coalesced and
// bandwidth-bound.
//
// These restate the solvers the reference reaches through KrylovKit
// (src/utility.jl:180-265, 379-393; src/algorithms/groundstates/envs.jl:14-19;
// src/algorithms/timeevo/tdvp.jl:14-20); the CPU oracle implements the very same
// algorithms so trajectories can be compared step for step.
#include "krylov.h"

#include <algorithm>
#include <cmath>

#include "smallla.h"

namespace imps {
namespace {

// Classical Gram-Schmidt with iterative refinement (KrylovKit's
// ClassicalGramSchmidtIR, eta = 1/sqrt(2)): w <- w - V h; the projection is
// repeated while it shrank ||w|| below eta times its previous value (at most three
// passes).  Returns the accumulated coefficients (host) and the final ||w||.
double cgs2(Context* ctx, int64_t n, int nv, const dcplx* V, dcplx* w, std::vector<cplx>& h) {
  return gs_project(ctx, n, nv, V, n, w, h);
}

std::vector<cplx> herm_part(const std::vector<cplx>& H, int ldh, int m) {
  std::vector<cplx> S((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i)
      S[i + (size_t)m * j] = 0.5 * (H[i + (size_t)ldh * j] + std::conj(H[j + (size_t)ldh * i]));
  return S;
}

void phase_align(Context* ctx, int64_t n, const dcplx* x0n, dcplx* x) {
  cplx ov = zdotc(ctx, n, x0n, x);
  double a = std::abs(ov);
  if (a > 0) zscal(ctx, n, std::conj(ov) / a, x);
}

}  // namespace

KrylovResult lanczos_eigsolve(Context* ctx, int64_t n, const LinOp& A, const dcplx* x0, dcplx* x, double tol,
                              int krylovdim, int maxiter, bool eager) {
  KrylovResult res;
  const int kdim = (int)std::min<int64_t>(krylovdim, n);
  IMPS_REQUIRE(kdim >= 1, IMPS_INVALID_ARG, "eigsolve: empty problem");
  DevBuf& Vb = ctx->buf("kry_V", (size_t)n * (kdim + 1) * sizeof(dcplx));
  DevBuf& X0 = ctx->buf("kry_x0", (size_t)n * sizeof(dcplx));
  dcplx* V = Vb.z();
  double beta0 = dznrm2(ctx, n, x0);
  IMPS_REQUIRE(std::isfinite(beta0), IMPS_INVALID_ARG, "eigsolve: the starting vector holds NaN or Inf");
  IMPS_REQUIRE(beta0 > 0, IMPS_INVALID_ARG, "eigsolve: zero starting vector");
  zaxpby(ctx, n, 1.0 / beta0, x0, 0.0, X0.z());
  zcopy(ctx, n, X0.z(), V);
  const int ldh = kdim + 1;
  std::vector<cplx> H((size_t)ldh * kdim, 0.0), h;
  res.numiter = 1;
  int nvec = 1;
  std::vector<double> theta;
  std::vector<cplx> U;
  while (true) {
    const int k = nvec - 1;
    dcplx* w = V + n * (int64_t)nvec;
    A(V + n * (int64_t)k, w);
    res.numops++;
    double beta = cgs2(ctx, n, nvec, V, w, h);
    for (int i = 0; i <= k; ++i) H[i + (size_t)ldh * k] = h[i];
    H[k + 1 + (size_t)ldh * k] = beta;
    const int m = k + 1;
    herm_eig(m, herm_part(H, ldh, m), theta, U);
    std::vector<double> rr(m);
    double tmax = 0.0;
    for (int j = 0; j < m; ++j) {
      rr[j] = std::abs(beta * U[(m - 1) + (size_t)m * j]);
      tmax = std::max(tmax, std::abs(theta[j]));
    }
    const bool breakdown = beta <= 1e-14 * std::max(1.0, tmax);
    const bool full = (m == kdim);
    auto finish = [&](bool conv) {
      std::vector<cplx> u(m);
      for (int i = 0; i < m; ++i) u[i] = U[i + (size_t)m * 0];
      zgemv_set(ctx, n, m, V, n, u.data(), x);
      double nx = dznrm2(ctx, n, x);
      zscal(ctx, n, 1.0 / nx, x);
      if (conv) phase_align(ctx, n, X0.z(), x);
      res.converged = conv ? 1 : 0;
      res.normres = rr[0];
      res.value = theta[0];
      return res;
    };
    if (eager || full || breakdown) {
      if (rr[0] <= tol || breakdown) return finish(true);
    }
    if (full) {
      if (res.numiter >= maxiter) return finish(false);
      int nconv = 0;
      for (int j = 0; j < m; ++j) nconv += rr[j] <= tol;
      const int keep = std::max(1, (3 * kdim + 2 * nconv) / 5);
      DevBuf& T = ctx->buf("kry_tmp", (size_t)n * keep * sizeof(dcplx));
      DevBuf& Ud = ctx->buf("kry_U", (size_t)m * keep * sizeof(dcplx));
      upload(ctx, Ud.ptr, U.data(), (size_t)m * keep * sizeof(dcplx));
      zgemm_fp64(ctx, OP_N, OP_N, (int)n, keep, m, 1.0, V, n, 0, Ud.z(), m, 0, 0.0, T.z(), n, 0, 1);
      // next basis vector w / beta goes to slot `keep`
      zaxpby(ctx, n, 1.0 / beta, w, 0.0, V + n * (int64_t)keep);
      zcopy(ctx, n * keep, T.z(), V);
      std::fill(H.begin(), H.end(), cplx(0.0, 0.0));
      for (int j = 0; j < keep; ++j) {
        H[j + (size_t)ldh * j] = theta[j];
        H[keep + (size_t)ldh * j] = beta * U[(m - 1) + (size_t)m * j];
      }
      nvec = keep + 1;
      res.numiter++;
    } else {
      zscal(ctx, n, 1.0 / beta, w);
      nvec++;
    }
  }
}

KrylovResult gmres(Context* ctx, int64_t n, const LinOp& A, const dcplx* b, dcplx* x, double tol, int krylovdim,
                   int maxiter, cplx a0, cplx a1) {
  KrylovResult res;
  const int kdim = (int)std::min<int64_t>(krylovdim, n);
  DevBuf& Vb = ctx->buf("kry_V", (size_t)n * (kdim + 1) * sizeof(dcplx));
  dcplx* V = Vb.z();
  auto op = [&](const dcplx* v, dcplx* out) {
    res.numops++;
    A(v, out);
    zaxpby(ctx, n, a0, v, a1, out);  // out = a0 v + a1 A v
  };
  // Mixed precision = iterative refinement: the residual b - op(x) that defines
  // convergence is always evaluated with the FP64 engine; the Krylov cycles in
  // between run on the split engine and solve the correction equation to the
  // engine's relative accuracy.
  const double inner_floor = split_floor(ctx);
  auto true_op = [&](const dcplx* v, dcplx* out) {
    Fp64Scope f(ctx);
    op(v, out);
  };
  // r = b - op(x)
  true_op(x, V);
  zaxpby(ctx, n, 1.0, b, -1.0, V);
  double beta = dznrm2(ctx, n, V);
  res.normres = beta;
  if (beta <= tol) {
    res.converged = 1;
    return res;
  }
  const int ldr = kdim + 1;
  std::vector<cplx> h;
  while (true) {
    res.numiter++;
    zscal(ctx, n, 1.0 / beta, V);
    std::vector<cplx> R((size_t)ldr * kdim, 0.0), g(kdim + 1, 0.0), sn(kdim, 0.0);
    std::vector<double> cs(kdim, 0.0);
    g[0] = beta;
    int kused = 0;
    for (int k = 0; k < kdim; ++k) {
      dcplx* w = V + n * (int64_t)(k + 1);
      op(V + n * (int64_t)k, w);
      double hn = cgs2(ctx, n, k + 1, V, w, h);
      std::vector<cplx> col(k + 2, 0.0);
      for (int i = 0; i <= k; ++i) col[i] = h[i];
      col[k + 1] = hn;
      for (int j = 0; j < k; ++j) {
        cplx t1 = cs[j] * col[j] + sn[j] * col[j + 1];
        col[j + 1] = -std::conj(sn[j]) * col[j] + cs[j] * col[j + 1];
        col[j] = t1;
      }
      cplx a = col[k], bb = col[k + 1];
      double nrm = std::hypot(std::abs(a), std::abs(bb));
      if (nrm == 0.0) { cs[k] = 1.0; sn[k] = 0.0; }
      else if (std::abs(a) == 0.0) { cs[k] = 0.0; sn[k] = std::conj(bb) / std::abs(bb); }
      else { cs[k] = std::abs(a) / nrm; sn[k] = (a / std::abs(a)) * std::conj(bb) / nrm; }
      col[k] = cs[k] * a + sn[k] * bb;
      col[k + 1] = 0.0;
      g[k + 1] = -std::conj(sn[k]) * g[k];
      g[k] = cs[k] * g[k];
      for (int i = 0; i <= k + 1; ++i) R[i + (size_t)ldr * k] = col[i];
      kused = k + 1;
      if (std::abs(g[k + 1]) <= std::max(tol, inner_floor * beta) || hn <= 1e-300) break;
      zscal(ctx, n, 1.0 / hn, w);
    }
    std::vector<cplx> y(kused, 0.0);
    for (int i = kused - 1; i >= 0; --i) {
      cplx s = g[i];
      for (int j = i + 1; j < kused; ++j) s -= R[i + (size_t)ldr * j] * y[j];
      y[i] = s / R[i + (size_t)ldr * i];
    }
    zgemv_acc(ctx, n, kused, V, n, y.data(), x);
    true_op(x, V);
    zaxpby(ctx, n, 1.0, b, -1.0, V);
    beta = dznrm2(ctx, n, V);
    res.normres = beta;
    if (beta <= tol) {
      res.converged = 1;
      return res;
    }
    if (res.numiter >= maxiter) return res;
  }
}

KrylovResult exponentiate(Context* ctx, int64_t n, const LinOp& A, cplx t, const dcplx* x0, dcplx* x, double tol,
                          int krylovdim, int maxiter) {
  KrylovResult res;
  zcopy(ctx, n, x0, x);
  if (t == cplx(0.0, 0.0)) {
    res.converged = 1;
    return res;
  }
  const int kdim = (int)std::min<int64_t>(krylovdim, n);
  DevBuf& Vb = ctx->buf("kry_V", (size_t)n * (kdim + 1) * sizeof(dcplx));
  dcplx* V = Vb.z();
  const int ldh = kdim + 1;
  cplx remaining = t;
  const double absT = std::abs(t);
  std::vector<cplx> h, E;
  while (true) {
    double beta = dznrm2(ctx, n, x);
    if (beta == 0.0) {
      res.converged = 1;
      return res;
    }
    res.numiter++;
    zaxpby(ctx, n, 1.0 / beta, x, 0.0, V);
    std::vector<cplx> H((size_t)ldh * kdim, 0.0);
    cplx tau = remaining;
    int m = 0;
    double err = 0.0;
    while (true) {
      const int k = m;
      dcplx* w = V + n * (int64_t)(k + 1);
      A(V + n * (int64_t)k, w);
      res.numops++;
      double hn = cgs2(ctx, n, k + 1, V, w, h);
      for (int i = 0; i <= k; ++i) H[i + (size_t)ldh * k] = h[i];
      H[k + 1 + (size_t)ldh * k] = hn;
      m = k + 1;
      std::vector<cplx> Hs = herm_part(H, ldh, m);
      double dmax = 0.0;
      for (int i = 0; i < m; ++i) dmax = std::max(dmax, std::abs(Hs[i + (size_t)m * i]));
      const bool breakdown = hn <= 1e-14 * std::max(1.0, dmax);
      herm_expm_e1(m, Hs, tau, E);
      err = beta * hn * std::abs(E[m - 1]);
      if (breakdown || err <= tol * std::abs(tau) / absT) break;
      if (m == kdim) {
        while (err > tol * std::abs(tau) / absT && std::abs(tau) > 1e-300) {
          tau = tau / 2.0;
          herm_expm_e1(m, Hs, tau, E);
          err = beta * hn * std::abs(E[m - 1]);
        }
        break;
      }
      zscal(ctx, n, 1.0 / hn, w);
    }
    std::vector<cplx> coef(m);
    for (int i = 0; i < m; ++i) coef[i] = beta * E[i];
    zgemv_set(ctx, n, m, V, n, coef.data(), x);
    remaining -= tau;
    res.normres = err;
    if (std::abs(remaining) <= 1e-15 * absT) {
      res.converged = 1;
      return res;
    }
    if (res.numiter >= maxiter) return res;
  }
}

KrylovResult arnoldi_dominant(Context* ctx, int64_t n, const LinOp& A, const dcplx* x0, dcplx* x, double tol,
                              int krylovdim, int maxiter, bool eager) {
  // Krylov-Schur form A V[:, :m] = V[:, :m+1] H[:m+1, :m], with H upper Hessenberg
  // apart from the leading keep x keep Schur block and its coupling row after a
  // restart.  A full basis restarts from the leading `keep` Schur vectors of
  // H[:m, :m] (ordered by |lambda|) plus the residual vector, which keeps the
  // subspace of the dominant Ritz values (KrylovKit's schursolve restart).
  KrylovResult res;
  const int kdim = (int)std::min<int64_t>(krylovdim, n);
  DevBuf& Vb = ctx->buf("arn_V", (size_t)n * (kdim + 1) * sizeof(dcplx));
  DevBuf& X0 = ctx->buf("arn_x0", (size_t)n * sizeof(dcplx));
  dcplx* V = Vb.z();
  double nx0 = dznrm2(ctx, n, x0);
  IMPS_REQUIRE(std::isfinite(nx0), IMPS_INVALID_ARG, "arnoldi: the starting vector holds NaN or Inf");
  IMPS_REQUIRE(nx0 > 0, IMPS_INVALID_ARG, "arnoldi: zero starting vector");
  zaxpby(ctx, n, 1.0 / nx0, x0, 0.0, X0.z());
  zcopy(ctx, n, X0.z(), V);
  const int ldh = kdim + 1;
  std::vector<cplx> H((size_t)ldh * kdim, 0.0), h, lam, Y;
  res.numiter = 1;
  int nvec = 1;
  while (true) {
    const int k = nvec - 1;
    dcplx* w = V + n * (int64_t)nvec;
    A(V + n * (int64_t)k, w);
    res.numops++;
    double hn = cgs2(ctx, n, nvec, V, w, h);
    for (int i = 0; i <= k; ++i) H[i + (size_t)ldh * k] = h[i];
    H[k + 1 + (size_t)ldh * k] = hn;
    const int m = k + 1;
    std::vector<cplx> Hm((size_t)m * m);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) Hm[i + (size_t)m * j] = H[i + (size_t)ldh * j];
    gen_eig(m, Hm, lam, Y);
    int jd = 0;
    for (int j = 1; j < m; ++j)
      if (std::abs(lam[j]) > std::abs(lam[jd])) jd = j;
    std::vector<cplx> y(m);
    for (int i = 0; i < m; ++i) y[i] = Y[i + (size_t)m * jd];
    // residual of the Ritz pair: |row m of H . y| times the unit residual vector
    cplx ry = 0.0;
    for (int j = 0; j < m; ++j) ry += H[m + (size_t)ldh * j] * y[j];
    const double rnorm = std::abs(ry);
    const bool breakdown = hn <= 1e-14 * std::max(1.0, std::abs(lam[jd]));
    const bool full = (m == kdim);
    auto ritz = [&]() {
      zgemv_set(ctx, n, m, V, n, y.data(), x);
      double nv = dznrm2(ctx, n, x);
      zscal(ctx, n, 1.0 / nv, x);
    };
    if (eager || full || breakdown) {
      if (rnorm <= tol || breakdown) {
        ritz();
        phase_align(ctx, n, X0.z(), x);
        res.converged = 1;
        res.normres = rnorm;
        res.value = lam[jd];
        return res;
      }
    }
    if (full) {
      if (res.numiter >= maxiter) {
        ritz();
        res.normres = rnorm;
        res.value = lam[jd];
        return res;
      }
      // Krylov-Schur restart
      std::vector<cplx> T, Z;
      schur_sorted(m, Hm, T, Z);
      const int nconv = rnorm <= tol ? 1 : 0;
      const int keep = std::max(1, std::min(m - 1, (3 * kdim + 2 * nconv) / 5));
      DevBuf& Tb = ctx->buf("arn_tmp", (size_t)n * keep * sizeof(dcplx));
      DevBuf& Zd = ctx->buf("arn_Z", (size_t)m * keep * sizeof(dcplx));
      upload(ctx, Zd.ptr, Z.data(), (size_t)m * keep * sizeof(dcplx));
      zgemm_fp64(ctx, OP_N, OP_N, (int)n, keep, m, 1.0, V, n, 0, Zd.z(), m, 0, 0.0, Tb.z(), n, 0, 1);
      // residual direction (unit after scaling) moves to slot `keep`
      zscal(ctx, n, 1.0 / hn, w);
      zcopy(ctx, n, w, V + n * (int64_t)keep);
      zcopy(ctx, n * keep, Tb.z(), V);
      std::vector<cplx> Hn((size_t)ldh * kdim, 0.0);
      for (int j = 0; j < keep; ++j) {
        for (int i = 0; i <= j; ++i) Hn[i + (size_t)ldh * j] = T[i + (size_t)m * j];
        cplx bcoef = 0.0;
        for (int l = 0; l < m; ++l) bcoef += H[m + (size_t)ldh * l] * Z[l + (size_t)m * j];
        Hn[keep + (size_t)ldh * j] = bcoef;
      }
      H.swap(Hn);
      nvec = keep + 1;
      res.numiter++;
    } else {
      zscal(ctx, n, 1.0 / hn, w);
      nvec++;
    }
  }
}

}  // namespace imps
