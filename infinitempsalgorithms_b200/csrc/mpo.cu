// Schur MPO storage (SparseIMPO, src/operators/mpohamiltonian.jl:33-133) and
// its level predicates.  Each site keeps the dense tompotensor (m, d, n, d) and,
// right behind it on the device, the level-transposed copy Wt[j,u,i,s] = W[i,u,j,s]
// used by right pushes.
#include "mpo.h"

#include <cmath>

namespace imps {

bool MpoSite::block_nonzero(int i, int j) const {
  if (i < 0 || i >= m || j < 0 || j >= n) return false;
  for (int u = 0; u < d; ++u)
    for (int s = 0; s < d; ++s)
      if (at(i, u, j, s) != cplx(0.0, 0.0)) return true;
  return false;
}

void make_mpo_site(Context* ctx, MpoSite& S, int m, int d, int n, const cplx* W) {
  IMPS_REQUIRE(m > 0 && d > 0 && n > 0, IMPS_INVALID_ARG, "MPO tensor with an empty dimension");
  IMPS_REQUIRE(d <= 8, IMPS_INVALID_ARG, "physical dimension above 8 is not supported");
  S.m = m;
  S.d = d;
  S.n = n;
  const size_t tot = (size_t)m * d * n * d;
  S.W.assign(W, W + tot);
  std::vector<cplx> both(2 * tot);
  for (size_t k = 0; k < tot; ++k) both[k] = S.W[k];
  for (int i = 0; i < m; ++i)
    for (int u = 0; u < d; ++u)
      for (int j = 0; j < n; ++j)
        for (int s = 0; s < d; ++s)
          both[tot + j + (size_t)n * (u + (size_t)d * (i + (size_t)m * s))] = S.at(i, u, j, s);
  S.Wdev.ensure(2 * tot * sizeof(dcplx));
  upload(ctx, S.Wdev.ptr, both.data(), both.size() * sizeof(dcplx));
  S.nz.clear();
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j)
      if (S.block_nonzero(i, j)) S.nz.push_back({i, j});
}

void make_closing_column(Context* ctx, const MpoSite& W, MpoSite& out) {
  std::vector<cplx> col((size_t)W.m * W.d * 1 * W.d);
  for (int i = 0; i < W.m; ++i)
    for (int u = 0; u < W.d; ++u)
      for (int s = 0; s < W.d; ++s) col[i + (size_t)W.m * (u + (size_t)W.d * (0 + 1 * (size_t)s))] = W.at(i, u, W.n - 1, s);
  make_mpo_site(ctx, out, W.m, W.d, 1, col.data());
}

}  // namespace imps

namespace {
// isapprox(block, one(block); atol): Frobenius distance to the identity
bool is_identity_block(const imps::MpoSite& W, int i, int j, double atol) {
  double nrm = 0.0;
  for (int u = 0; u < W.d; ++u)
    for (int s = 0; s < W.d; ++s) nrm += std::norm(W.at(i, u, j, s) - (u == s ? 1.0 : 0.0));
  return std::sqrt(nrm) <= atol;
}
}  // namespace

// isidentitylevel (mpohamiltonian.jl:100-109), level i 1-based
bool imps_mpo::isidentitylevel(int i) const {
  if (i == 1) return true;
  for (const auto& W : sites) {
    const int m = W.m, n = W.n;
    if (i == m && m == n) continue;
    if (i > m - 1 || i > n - 1) return false;
    if (!is_identity_block(W, i - 1, i - 1, 1e-14)) return false;
  }
  return true;
}

// isemptylevel (mpohamiltonian.jl:122-133)
bool imps_mpo::isemptylevel(int i) const {
  if (i == 1) return false;
  for (const auto& W : sites)
    if (i == W.n) return false;
  for (const auto& W : sites) {
    const int m = W.m, n = W.n;
    bool dz = (i > m - 1 || i > n - 1) || !W.block_nonzero(i - 1, i - 1);
    bool cz = (i > n - 1) || !W.block_nonzero(0, i - 1);
    bool bz = (i > m - 1) || !W.block_nonzero(i - 1, n - 1);
    if (!(dz && cz && bz)) return false;
  }
  return true;
}
