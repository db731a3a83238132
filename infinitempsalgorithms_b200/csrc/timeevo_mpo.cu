// W^I / W^II time-evolution MPO tensors (timeevompo(H::SparseIMPO, delta, WI()/WII()),
// src/algorithms/timeevo/w1w2.jl:26-45).  The reference's per-site kernel lives in the
// unvendored FiniteMPSAlgorithms package; this restates the published construction it
// cites (Zaletel, Mong, Karrasch, Moore, Pollmann, PRB 91, 165112 (2015),
// arXiv:1407.1832).  It builds a few tensors of size (m-1) d (n-1) d once per
// evolution, so it runs on the host (setup, like imps_mpo_create); the MPO it makes is
// applied on the device.
//
// Schur site tensor W (m, d, n, d): D = W[0,:,n-1,:], C_b = W[0,:,b,:], B_a = W[a,:,n-1,:],
// A_ab = W[a,:,b,:] (a, b interior levels).  With s = sqrt(delta):
//   W^I  = [[1 + delta D, s C], [s B, A]]
//   W^II : for every interior pair (a, b), E = exp(M) with M the 4 x 4 block operator on
//          the auxiliary states (0, c, b, bc): M[x,x] = delta D, M[c,0] = s C_b,
//          M[b,0] = s B_a, M[bc,0] = A_ab, M[bc,c] = s B_a, M[bc,b] = s C_b; then
//          W_D = E[0,0], W_C(b) = E[c,0], W_B(a) = E[b,0], W_A(a,b) = E[bc,0].
// The exponential is taken by scaling and squaring of a truncated Taylor series.
#include <cmath>
#include <complex>
#include <vector>

#include "imps_internal.h"

namespace imps {
namespace {

using Mat = std::vector<cplx>;  // column-major n x n

Mat matmul(int n, const Mat& X, const Mat& Y) {
  Mat Z((size_t)n * n, cplx(0.0, 0.0));
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) {
      const cplx y = Y[k + (size_t)n * j];
      if (y == cplx(0.0, 0.0)) continue;
      for (int i = 0; i < n; ++i) Z[i + (size_t)n * j] += X[i + (size_t)n * k] * y;
    }
  return Z;
}

// exp(M): M / 2^q with ||M / 2^q||_1 <= 1/2, Taylor series to 24 terms (the truncation
// is below 2^-24 / 24! relative), then q squarings.
Mat expm(int n, const Mat& M) {
  double nrm = 0.0;
  for (int j = 0; j < n; ++j) {
    double c = 0.0;
    for (int i = 0; i < n; ++i) c += std::abs(M[i + (size_t)n * j]);
    nrm = std::max(nrm, c);
  }
  int q = 0;
  while (nrm > 0.5) {
    nrm *= 0.5;
    ++q;
  }
  const double sc = std::ldexp(1.0, -q);
  Mat A(M);
  for (auto& v : A) v *= sc;
  Mat E((size_t)n * n, cplx(0.0, 0.0)), T((size_t)n * n, cplx(0.0, 0.0));
  for (int i = 0; i < n; ++i) E[i + (size_t)n * i] = T[i + (size_t)n * i] = 1.0;
  for (int k = 1; k <= 24; ++k) {
    T = matmul(n, T, A);
    for (auto& v : T) v /= (double)k;
    for (size_t e = 0; e < E.size(); ++e) E[e] += T[e];
  }
  for (int k = 0; k < q; ++k) E = matmul(n, E, E);
  return E;
}

}  // namespace

void timeevompo_site(int m, int d, int n, const cplx* W, cplx delta, int alg, cplx* out) {
  IMPS_REQUIRE(m >= 2 && n >= 2 && d >= 1, IMPS_INVALID_ARG, "timeevompo: Schur tensors need >= 2 levels");
  IMPS_REQUIRE(alg == 1 || alg == 2, IMPS_INVALID_ARG, "timeevompo: alg must be 1 (WI) or 2 (WII)");
  auto w = [&](int i, int u, int j, int s) { return W[i + (size_t)m * (u + (size_t)d * (j + (size_t)n * s))]; };
  const int kl = m - 2, kr = n - 2, mo = m - 1, no = n - 1;
  auto o = [&](int i, int u, int j, int s) -> cplx& {
    return out[i + (size_t)mo * (u + (size_t)d * (j + (size_t)no * s))];
  };
  for (size_t e = 0; e < (size_t)mo * d * no * d; ++e) out[e] = 0.0;
  const cplx sq = std::sqrt(delta);
  if (alg == 1) {
    for (int u = 0; u < d; ++u)
      for (int s = 0; s < d; ++s) {
        o(0, u, 0, s) = (u == s ? 1.0 : 0.0) + delta * w(0, u, n - 1, s);
        for (int b = 0; b < kr; ++b) o(0, u, b + 1, s) = sq * w(0, u, b + 1, s);
        for (int a = 0; a < kl; ++a) {
          o(a + 1, u, 0, s) = sq * w(a + 1, u, n - 1, s);
          for (int b = 0; b < kr; ++b) o(a + 1, u, b + 1, s) = w(a + 1, u, b + 1, s);
        }
      }
    return;
  }
  const int N4 = 4 * d;
  // block (x, y) of the 4d x 4d generator, x = target aux state, y = source
  auto build = [&](int a, int b) {
    Mat M((size_t)N4 * N4, cplx(0.0, 0.0));
    auto put = [&](int x, int y, auto&& f) {
      for (int u = 0; u < d; ++u)
        for (int s = 0; s < d; ++s) M[(x * d + u) + (size_t)N4 * (y * d + s)] = f(u, s);
    };
    for (int x = 0; x < 4; ++x) put(x, x, [&](int u, int s) { return delta * w(0, u, n - 1, s); });
    if (b >= 0) {
      put(1, 0, [&](int u, int s) { return sq * w(0, u, b + 1, s); });
      put(3, 2, [&](int u, int s) { return sq * w(0, u, b + 1, s); });
    }
    if (a >= 0) {
      put(2, 0, [&](int u, int s) { return sq * w(a + 1, u, n - 1, s); });
      put(3, 1, [&](int u, int s) { return sq * w(a + 1, u, n - 1, s); });
    }
    if (a >= 0 && b >= 0) put(3, 0, [&](int u, int s) { return w(a + 1, u, b + 1, s); });
    return expm(N4, M);
  };
  auto take = [&](const Mat& E, int x, int oi, int oj) {
    for (int u = 0; u < d; ++u)
      for (int s = 0; s < d; ++s) o(oi, u, oj, s) = E[(x * d + u) + (size_t)N4 * s];
  };
  take(build(-1, -1), 0, 0, 0);
  for (int b = 0; b < kr; ++b) take(build(-1, b), 1, 0, b + 1);
  for (int a = 0; a < kl; ++a) {
    take(build(a, -1), 2, a + 1, 0);
    for (int b = 0; b < kr; ++b) take(build(a, b), 3, a + 1, b + 1);
  }
}

}  // namespace imps
