// Small dense eigenproblems of the Krylov solvers (projected matrices of
// dimension <= krylovdim, i.e. <= 64): FP64 on the host thread that drives the
// stream, between launches.
//   herm_eig     : Householder reduction of the Hermitian matrix to a real
//                  symmetric tridiagonal one (phases moved into a diagonal
//                  unitary), then implicit QR steps with Wilkinson shifts
//                  (Golub & Van Loan, Matrix Computations, alg. 8.3.2/8.3.3)
//                  with the rotations accumulated; ascending eigenvalues.
//   complex_schur: Householder reduction to Hessenberg form, then shifted QR
//                  (Givens) to the complex Schur form T = Z^H H Z.
//   schur_sorted : the Schur form reordered so that |T[k,k]| is non-increasing
//                  (adjacent swaps by the eigenvector of each 2 x 2 block, as in
//                  LAPACK's ztrexc); the Krylov-Schur restart keeps its leading
//                  columns.
//   gen_eig      : eigenpairs of a general matrix from its Schur form
//                  (back substitution), used for the Arnoldi Ritz pairs.
#include "smallla.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace imps {
namespace {

constexpr double kEps = 2.220446049250313e-16;

// One implicit symmetric QR step with a Wilkinson shift on the unreduced block
// [l, h] of the tridiagonal (a, b) (b[k] couples k and k+1), rotations applied
// to the columns of the real n x n matrix Z.
void tridiag_qr_step(int n, std::vector<double>& a, std::vector<double>& b, int l, int h, std::vector<double>& Z) {
  const double dd = 0.5 * (a[h - 1] - a[h]);
  const double bh = b[h - 1];
  double mu;
  if (dd == 0.0) mu = a[h] - std::abs(bh);
  else mu = a[h] - bh * bh / (dd + std::copysign(std::hypot(dd, bh), dd));
  double x = a[l] - mu, z = b[l];
  for (int k = l; k < h; ++k) {
    const double r = std::hypot(x, z);
    const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
    if (k > l) b[k - 1] = r;
    const double ak = a[k], ak1 = a[k + 1], bk = b[k];
    a[k] = c * c * ak + 2.0 * c * s * bk + s * s * ak1;
    a[k + 1] = s * s * ak - 2.0 * c * s * bk + c * c * ak1;
    b[k] = c * s * (ak1 - ak) + (c * c - s * s) * bk;
    if (k + 1 < h) {
      x = b[k];
      z = s * b[k + 1];
      b[k + 1] = c * b[k + 1];
    }
    double* zk = Z.data() + (size_t)n * k;
    double* zk1 = Z.data() + (size_t)n * (k + 1);
    for (int i = 0; i < n; ++i) {
      const double u = zk[i], v = zk1[i];
      zk[i] = c * u + s * v;
      zk1[i] = -s * u + c * v;
    }
  }
}

// Householder reduction H <- P^H H P of a general matrix to upper Hessenberg form,
// P accumulated into Z (Z <- Z P).  For a Hermitian input the result is tridiagonal.
void hessenberg(int n, std::vector<cplx>& H, std::vector<cplx>& Z) {
  auto h = [&](int i, int j) -> cplx& { return H[i + (size_t)n * j]; };
  std::vector<cplx> v(n);
  for (int k = 0; k < n - 2; ++k) {
    double alpha = 0.0;
    for (int i = k + 2; i < n; ++i) alpha += std::norm(h(i, k));
    if (alpha == 0.0) continue;
    const double nx = std::sqrt(alpha + std::norm(h(k + 1, k)));
    const cplx x0 = h(k + 1, k);
    const cplx ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : cplx(1.0, 0.0);
    std::fill(v.begin(), v.end(), cplx(0.0, 0.0));
    v[k + 1] = x0 + ph * nx;
    for (int i = k + 2; i < n; ++i) v[i] = h(i, k);
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += std::norm(v[i]);
    if (vn == 0.0) continue;
    const double f = 2.0 / vn;
    for (int j = 0; j < n; ++j) {  // rows: H <- (I - f v v^H) H
      cplx s = 0.0;
      for (int i = k + 1; i < n; ++i) s += std::conj(v[i]) * h(i, j);
      s *= f;
      for (int i = k + 1; i < n; ++i) h(i, j) -= v[i] * s;
    }
    for (int i = 0; i < n; ++i) {  // columns: H <- H (I - f v v^H)
      cplx s = 0.0;
      for (int j = k + 1; j < n; ++j) s += h(i, j) * v[j];
      s *= f;
      for (int j = k + 1; j < n; ++j) h(i, j) -= s * std::conj(v[j]);
    }
    for (int i = 0; i < n; ++i) {
      cplx s = 0.0;
      for (int j = k + 1; j < n; ++j) s += Z[i + (size_t)n * j] * v[j];
      s *= f;
      for (int j = k + 1; j < n; ++j) Z[i + (size_t)n * j] -= s * std::conj(v[j]);
    }
    for (int i = k + 2; i < n; ++i) h(i, k) = 0.0;
  }
}

}  // namespace

void herm_eig(int n, const std::vector<cplx>& Ain, std::vector<double>& w, std::vector<cplx>& V) {
  std::vector<cplx> A((size_t)n * n);
  // Hermitian part of the input
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i)
      A[i + (size_t)n * j] = 0.5 * (Ain[i + (size_t)n * j] + std::conj(Ain[j + (size_t)n * i]));
  std::vector<cplx> Q((size_t)n * n, cplx(0.0, 0.0));
  for (int i = 0; i < n; ++i) Q[i + (size_t)n * i] = 1.0;
  hessenberg(n, A, Q);
  // T = Q^H A Q is tridiagonal with real diagonal; D = diag(p) makes the off-diagonal
  // real and non-negative: (D^H T D)[k+1,k] = |T[k+1,k]| for p[k+1] = p[k] e_k / |e_k|
  std::vector<double> a(n), b(std::max(n - 1, 0));
  std::vector<cplx> p(n, cplx(1.0, 0.0));
  for (int k = 0; k < n; ++k) a[k] = A[k + (size_t)n * k].real();
  for (int k = 0; k + 1 < n; ++k) {
    const cplx e = A[(k + 1) + (size_t)n * k];
    const double ae = std::abs(e);
    b[k] = ae;
    p[k + 1] = ae > 0.0 ? p[k] * (e / ae) : p[k];
  }
  std::vector<double> Z((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Z[i + (size_t)n * i] = 1.0;
  int h = n - 1, guard = 0;
  while (h > 0 && guard < 60 * n) {
    if (std::abs(b[h - 1]) <= kEps * (std::abs(a[h - 1]) + std::abs(a[h]))) {
      b[h - 1] = 0.0;
      --h;
      continue;
    }
    int l = h - 1;
    while (l > 0 && std::abs(b[l - 1]) > kEps * (std::abs(a[l - 1]) + std::abs(a[l]))) --l;
    if (l > 0) b[l - 1] = 0.0;
    tridiag_qr_step(n, a, b, l, h, Z);
    ++guard;
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return a[x] < a[y]; });
  // V = Q D Z, columns in ascending eigenvalue order
  w.resize(n);
  V.assign((size_t)n * n, cplx(0.0, 0.0));
  std::vector<cplx> QD((size_t)n * n);
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) QD[i + (size_t)n * k] = Q[i + (size_t)n * k] * p[k];
  for (int j = 0; j < n; ++j) {
    const int c = idx[j];
    w[j] = a[c];
    cplx* vj = V.data() + (size_t)n * j;
    for (int k = 0; k < n; ++k) {
      const double zkc = Z[k + (size_t)n * c];
      if (zkc == 0.0) continue;
      const cplx* qk = QD.data() + (size_t)n * k;
      for (int i = 0; i < n; ++i) vj[i] += qk[i] * zkc;
    }
  }
}

void complex_schur(int n, const std::vector<cplx>& Hin, std::vector<cplx>& Tout, std::vector<cplx>& Zout) {
  std::vector<cplx> T(Hin), Z((size_t)n * n, cplx(0.0, 0.0));
  for (int i = 0; i < n; ++i) Z[i + (size_t)n * i] = 1.0;
  hessenberg(n, T, Z);
  auto h = [&](int i, int j) -> cplx& { return T[i + (size_t)n * j]; };
  int hi = n - 1, it = 0, total = 0;
  std::vector<double> cs(n);
  std::vector<cplx> sn(n);
  while (hi > 0 && total < 100 * n) {
    int l = hi;
    while (l > 0) {
      double s = std::abs(h(l - 1, l - 1)) + std::abs(h(l, l));
      if (s == 0.0) s = 1.0;
      if (std::abs(h(l, l - 1)) <= kEps * s) break;
      --l;
    }
    if (l == hi) {
      if (hi > 0) h(hi, hi - 1) = 0.0;
      --hi;
      it = 0;
      continue;
    }
    if (l > 0) h(l, l - 1) = 0.0;
    const cplx a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
    cplx mu;
    if (it > 0 && it % 10 == 0) {
      mu = d + cplx(std::abs(c), 0.0);  // exceptional shift
    } else {
      const cplx tr = a + d, det = a * d - b * c;
      const cplx disc = std::sqrt(tr * tr / 4.0 - det);
      const cplx m1 = tr / 2.0 + disc, m2 = tr / 2.0 - disc;
      mu = (std::abs(m1 - d) < std::abs(m2 - d)) ? m1 : m2;
    }
    for (int k = l; k <= hi; ++k) h(k, k) -= mu;
    for (int k = l; k < hi; ++k) {
      const cplx x = h(k, k), y = h(k + 1, k);
      const double r = std::sqrt(std::norm(x) + std::norm(y));
      double ck;
      cplx sk;
      if (r == 0.0) { ck = 1.0; sk = 0.0; }
      else if (std::abs(x) == 0.0) { ck = 0.0; sk = std::conj(y) / std::abs(y); }
      else { ck = std::abs(x) / r; sk = (x / std::abs(x)) * std::conj(y) / r; }
      cs[k] = ck;
      sn[k] = sk;
      for (int j = k; j < n; ++j) {
        const cplx u = h(k, j), v = h(k + 1, j);
        h(k, j) = ck * u + sk * v;
        h(k + 1, j) = -std::conj(sk) * u + ck * v;
      }
    }
    for (int k = l; k < hi; ++k) {
      const double ck = cs[k];
      const cplx sk = sn[k];
      const int rmax = std::min(k + 2, hi);
      for (int i = 0; i <= rmax; ++i) {
        const cplx u = h(i, k), v = h(i, k + 1);
        h(i, k) = ck * u + std::conj(sk) * v;
        h(i, k + 1) = -sk * u + ck * v;
      }
      for (int i = 0; i < n; ++i) {
        const cplx u = Z[i + (size_t)n * k], v = Z[i + (size_t)n * (k + 1)];
        Z[i + (size_t)n * k] = ck * u + std::conj(sk) * v;
        Z[i + (size_t)n * (k + 1)] = -sk * u + ck * v;
      }
    }
    for (int k = l; k <= hi; ++k) h(k, k) += mu;
    ++it;
    ++total;
  }
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) h(i, j) = 0.0;
  Tout.swap(T);
  Zout.swap(Z);
}

void schur_sorted(int n, const std::vector<cplx>& H, std::vector<cplx>& T, std::vector<cplx>& Z) {
  complex_schur(n, H, T, Z);
  auto t = [&](int i, int j) -> cplx& { return T[i + (size_t)n * j]; };
  // bubble the diagonal into non-increasing modulus by adjacent swaps; the block
  // [[t11, t12], [0, t22]] has the eigenvector x = (t12, t22 - t11) for t22, so the
  // unitary G = [x/|x|, (-conj x2, conj x1)/|x|] brings t22 to the top
  for (int pass = 0; pass < n; ++pass) {
    bool swapped = false;
    for (int k = 0; k + 1 < n; ++k) {
      const cplx t11 = t(k, k), t22 = t(k + 1, k + 1);
      if (!(std::abs(t22) > std::abs(t11))) continue;
      cplx g1 = t(k, k + 1), g2 = t22 - t11;
      const double nr = std::sqrt(std::norm(g1) + std::norm(g2));
      if (nr == 0.0) continue;
      g1 /= nr;
      g2 /= nr;
      // G = [[g1, -conj(g2)], [g2, conj(g1)]]
      for (int j = 0; j < n; ++j) {  // rows k, k+1 <- G^H rows
        const cplx u = t(k, j), v = t(k + 1, j);
        t(k, j) = std::conj(g1) * u + std::conj(g2) * v;
        t(k + 1, j) = -g2 * u + g1 * v;
      }
      for (int i = 0; i < n; ++i) {  // cols k, k+1 <- cols G
        const cplx u = t(i, k), v = t(i, k + 1);
        t(i, k) = u * g1 + v * g2;
        t(i, k + 1) = -u * std::conj(g2) + v * std::conj(g1);
        const cplx zu = Z[i + (size_t)n * k], zv = Z[i + (size_t)n * (k + 1)];
        Z[i + (size_t)n * k] = zu * g1 + zv * g2;
        Z[i + (size_t)n * (k + 1)] = -zu * std::conj(g2) + zv * std::conj(g1);
      }
      t(k + 1, k) = 0.0;
      t(k, k) = t22;
      t(k + 1, k + 1) = t11;
      swapped = true;
    }
    if (!swapped) break;
  }
}

void gen_eig(int n, const std::vector<cplx>& Hin, std::vector<cplx>& lam, std::vector<cplx>& Y) {
  std::vector<cplx> T, Z;
  complex_schur(n, Hin, T, Z);
  auto h = [&](int i, int j) -> cplx { return T[i + (size_t)n * j]; };
  lam.resize(n);
  for (int i = 0; i < n; ++i) lam[i] = h(i, i);
  // eigenvectors of the triangular factor, mapped back by Z
  Y.assign((size_t)n * n, cplx(0.0, 0.0));
  std::vector<cplx> y(n), x(n);
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
