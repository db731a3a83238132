// Small dense eigenproblems of the Krylov solvers (projected matrices of
// dimension <= krylovdim, i.e. <= 64): FP64 on the host thread that drives the
// stream, between launches.
//   herm_eig : cyclic complex Jacobi (Ritz values of the Hermitian Lanczos
//              projection, ascending order)
//   gen_eig  : complex Schur form of an upper-Hessenberg matrix by shifted QR
//              (Givens), eigenvectors by back substitution (Arnoldi Ritz pairs)
#include "smallla.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace imps {

void herm_eig(int n, const std::vector<cplx>& Ain, std::vector<double>& w, std::vector<cplx>& V) {
  std::vector<cplx> A(Ain);
  V.assign((size_t)n * n, cplx(0.0, 0.0));
  for (int i = 0; i < n; ++i) V[i + (size_t)n * i] = 1.0;
  auto a = [&](int i, int j) -> cplx& { return A[i + (size_t)n * j]; };
  // symmetrise
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      cplx s = 0.5 * (a(i, j) + std::conj(a(j, i)));
      a(i, j) = s;
      a(j, i) = std::conj(s);
    }
  double fro = 0.0;
  for (auto& z : A) fro += std::norm(z);
  fro = std::sqrt(fro);
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (i != j) off += std::norm(a(i, j));
    if (std::sqrt(off) <= 1e-17 * std::max(fro, 1e-300)) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        cplx apq = a(p, q);
        double b = std::abs(apq);
        if (b <= 1e-300) continue;
        cplx eph = apq / b;  // e^{i phi}
        double app = a(p, p).real(), aqq = a(q, q).real();
        double theta = 0.5 * std::atan2(2.0 * b, app - aqq);
        double c = std::cos(theta), s = std::sin(theta);
        // U (rows p,q; cols p,q) = [[c, -s], [s e^{-i phi}, c e^{-i phi}]]
        cplx upp = c, upq = -s, uqp = s * std::conj(eph), uqq = c * std::conj(eph);
        // A <- A U (columns)
        for (int i = 0; i < n; ++i) {
          cplx xp = a(i, p), xq = a(i, q);
          a(i, p) = xp * upp + xq * uqp;
          a(i, q) = xp * upq + xq * uqq;
        }
        // A <- U^H A (rows)
        for (int j = 0; j < n; ++j) {
          cplx xp = a(p, j), xq = a(q, j);
          a(p, j) = std::conj(upp) * xp + std::conj(uqp) * xq;
          a(q, j) = std::conj(upq) * xp + std::conj(uqq) * xq;
        }
        a(p, q) = 0.0;
        a(q, p) = 0.0;
        a(p, p) = a(p, p).real();
        a(q, q) = a(q, q).real();
        for (int i = 0; i < n; ++i) {
          cplx xp = V[i + (size_t)n * p], xq = V[i + (size_t)n * q];
          V[i + (size_t)n * p] = xp * upp + xq * uqp;
          V[i + (size_t)n * q] = xp * upq + xq * uqq;
        }
      }
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return a(x, x).real() < a(y, y).real(); });
  w.resize(n);
  std::vector<cplx> Vs((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    w[j] = a(idx[j], idx[j]).real();
    for (int i = 0; i < n; ++i) Vs[i + (size_t)n * j] = V[i + (size_t)n * idx[j]];
  }
  V.swap(Vs);
}

void gen_eig(int n, const std::vector<cplx>& Hin, std::vector<cplx>& lam, std::vector<cplx>& Y) {
  std::vector<cplx> H(Hin);
  std::vector<cplx> Z((size_t)n * n, cplx(0.0, 0.0));
  for (int i = 0; i < n; ++i) Z[i + (size_t)n * i] = 1.0;
  auto h = [&](int i, int j) -> cplx& { return H[i + (size_t)n * j]; };
  // reduce to Hessenberg form (Householder) -- Arnoldi matrices already are, this is a guard
  for (int k = 0; k < n - 2; ++k) {
    double alpha = 0.0;
    for (int i = k + 2; i < n; ++i) alpha += std::norm(h(i, k));
    if (alpha == 0.0) continue;
    std::vector<cplx> v(n, 0.0);
    double nx = std::sqrt(alpha + std::norm(h(k + 1, k)));
    cplx x0 = h(k + 1, k);
    cplx ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : cplx(1.0, 0.0);
    v[k + 1] = x0 + ph * nx;
    for (int i = k + 2; i < n; ++i) v[i] = h(i, k);
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += std::norm(v[i]);
    if (vn == 0.0) continue;
    // H <- P H P, P = I - 2 v v^H / vn
    for (int j = 0; j < n; ++j) {
      cplx s = 0.0;
      for (int i = k + 1; i < n; ++i) s += std::conj(v[i]) * h(i, j);
      s *= 2.0 / vn;
      for (int i = k + 1; i < n; ++i) h(i, j) -= v[i] * s;
    }
    for (int i = 0; i < n; ++i) {
      cplx s = 0.0;
      for (int j = k + 1; j < n; ++j) s += h(i, j) * v[j];
      s *= 2.0 / vn;
      for (int j = k + 1; j < n; ++j) h(i, j) -= s * std::conj(v[j]);
    }
    for (int i = 0; i < n; ++i) {
      cplx s = 0.0;
      for (int j = k + 1; j < n; ++j) s += Z[i + (size_t)n * j] * v[j];
      s *= 2.0 / vn;
      for (int j = k + 1; j < n; ++j) Z[i + (size_t)n * j] -= s * std::conj(v[j]);
    }
    for (int i = k + 2; i < n; ++i) h(i, k) = 0.0;
  }
  // shifted QR iterations to complex Schur form
  const double eps = 2.220446049250313e-16;
  int hi = n - 1, it = 0, total = 0;
  std::vector<double> cs(n);
  std::vector<cplx> sn(n);
  while (hi > 0 && total < 100 * n) {
    int l = hi;
    while (l > 0) {
      double s = std::abs(h(l - 1, l - 1)) + std::abs(h(l, l));
      if (s == 0.0) s = 1.0;
      if (std::abs(h(l, l - 1)) <= eps * s) break;
      --l;
    }
    if (l == hi) {
      if (hi > 0) h(hi, hi - 1) = 0.0;
      --hi;
      it = 0;
      continue;
    }
    if (l > 0) h(l, l - 1) = 0.0;
    cplx a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
    cplx mu;
    if (it > 0 && it % 10 == 0) {
      mu = d + cplx(std::abs(c), 0.0);  // exceptional shift
    } else {
      cplx tr = a + d, det = a * d - b * c;
      cplx disc = std::sqrt(tr * tr / 4.0 - det);
      cplx m1 = tr / 2.0 + disc, m2 = tr / 2.0 - disc;
      mu = (std::abs(m1 - d) < std::abs(m2 - d)) ? m1 : m2;
    }
    for (int k = l; k <= hi; ++k) h(k, k) -= mu;
    for (int k = l; k < hi; ++k) {
      cplx x = h(k, k), y = h(k + 1, k);
      double r = std::sqrt(std::norm(x) + std::norm(y));
      double ck;
      cplx sk;
      if (r == 0.0) { ck = 1.0; sk = 0.0; }
      else if (std::abs(x) == 0.0) { ck = 0.0; sk = std::conj(y) / std::abs(y); }
      else { ck = std::abs(x) / r; sk = (x / std::abs(x)) * std::conj(y) / r; }
      cs[k] = ck;
      sn[k] = sk;
      for (int j = k; j < n; ++j) {
        cplx u = h(k, j), v = h(k + 1, j);
        h(k, j) = ck * u + sk * v;
        h(k + 1, j) = -std::conj(sk) * u + ck * v;
      }
    }
    for (int k = l; k < hi; ++k) {
      double ck = cs[k];
      cplx sk = sn[k];
      int rmax = std::min(k + 2, hi);
      for (int i = 0; i <= rmax; ++i) {
        cplx u = h(i, k), v = h(i, k + 1);
        h(i, k) = ck * u + std::conj(sk) * v;
        h(i, k + 1) = -sk * u + ck * v;
      }
      for (int i = 0; i < n; ++i) {
        cplx u = Z[i + (size_t)n * k], v = Z[i + (size_t)n * (k + 1)];
        Z[i + (size_t)n * k] = ck * u + std::conj(sk) * v;
        Z[i + (size_t)n * (k + 1)] = -sk * u + ck * v;
      }
    }
    for (int k = l; k <= hi; ++k) h(k, k) += mu;
    ++it;
    ++total;
  }
  lam.resize(n);
  for (int i = 0; i < n; ++i) lam[i] = h(i, i);
  // eigenvectors of the triangular factor, mapped back by Z
  Y.assign((size_t)n * n, cplx(0.0, 0.0));
  std::vector<cplx> y(n);
  for (int j = 0; j < n; ++j) {
    std::fill(y.begin(), y.end(), cplx(0.0, 0.0));
    y[j] = 1.0;
    for (int i = j - 1; i >= 0; --i) {
      cplx s = 0.0;
      for (int k = i + 1; k <= j; ++k) s += h(i, k) * y[k];
      cplx den = h(i, i) - lam[j];
      if (std::abs(den) < 1e-300) den = cplx(1e-300, 0.0);
      y[i] = -s / den;
    }
    double nrm = 0.0;
    std::vector<cplx> x(n, 0.0);
    for (int i = 0; i < n; ++i) {
      cplx s = 0.0;
      for (int k = 0; k <= j; ++k) s += Z[i + (size_t)n * k] * y[k];
      x[i] = s;
      nrm += std::norm(s);
    }
    nrm = std::sqrt(nrm);
    for (int i = 0; i < n; ++i) Y[i + (size_t)n * j] = x[i] / nrm;
  }
}

void herm_expm_e1(int m, const std::vector<cplx>& Hs, cplx t, std::vector<cplx>& out) {
  std::vector<double> th;
  std::vector<cplx> U;
  herm_eig(m, Hs, th, U);
  out.assign(m, 0.0);
  for (int j = 0; j < m; ++j) {
    cplx coef = std::exp(t * th[j]) * std::conj(U[0 + (size_t)m * j]);
    for (int i = 0; i < m; ++i) out[i] += U[i + (size_t)m * j] * coef;
  }
}

}  // namespace imps
