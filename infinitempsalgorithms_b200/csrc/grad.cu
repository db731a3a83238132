// Energy gradients of a canonical iMPS by the adjoint of the environment fixed points.
//
// The reference has no gradient code; these two operations extend its API for
// gradient-based iMPS optimisation.  The energy per unit cell of a canonical
// state is E = sum_site <AC| H_AC |AC> over the closing column, with the left
// environments GL the fixed points of the left transfer recursion
// (src/algorithms/groundstates/envs.jl:321-518).  The adjoint of that linear
// fixed-point system, (1 - T_L)^T lambda = dE/dGL, is solved by the right
// environments GR of the same Schur levels (the right recursion is the transpose
// of the left one), so every derivative is one contraction with environments that
// the solver already holds: no unrolled iterations, nothing stored per iteration.
//
//   dE/dW_site[i,u,j,s] = sum conj(AC[b,u,c']) GL[b,i,a] AC[a,s,c] GR[c,j,c']
//   dE/dconj(AL_site)   = (H_AC(AC) - lambda AC) C_site^H,  lambda = <AC|H_AC|AC> / <AC|AC>
//
// The first is exact for every block except the two identity blocks of the
// Schur form (first level -> first level, last -> last), whose "derivative" is
// extensive and is returned as zero.  The second is the Wirtinger gradient of the
// normalised energy functional E(A) of the uniform MPS generated by A = AL.
#include "algos.h"
#include "gauge.h"
#include "imps_internal.h"

#include <algorithm>
#include <vector>

namespace imps {

void energy_grad_mpo(Context* ctx, const imps_envs* E, const imps_mpo* H, const imps_state* st, int site,
                     cplx* G_host) {
  Fp64Scope fp64(ctx);
  ProfTag tag(ctx, "grad");
  const MpoSite& W = H->sites[site % H->N];
  const int Dl = E->Dl[site], Dr = E->Dr[site];
  const int m = W.m, d = W.d, n = W.n;
  IMPS_REQUIRE(m == E->ml[site] && n == E->nr[site], IMPS_DIM_MISMATCH,
               "energy_grad_mpo: MPO levels != environment levels");
  IMPS_REQUIRE(st->Dl(site) == Dl && st->Dr(site) == Dr && st->d[site] == d, IMPS_DIM_MISMATCH,
               "energy_grad_mpo: state and environment shapes disagree");
  const dcplx* GL = E->lefts[site].z();
  const dcplx* GR = E->rights[site].z();
  const dcplx* AC = st->AC[site].z();
  const int64_t blk = (int64_t)Dr * Dl;  // one (c, b) plane
  DevBuf& P = ctx->buf("grad_p", (size_t)blk * m * d * sizeof(dcplx));
  DevBuf& Q = ctx->buf("grad_q", (size_t)blk * n * d * sizeof(dcplx));
  // P[(c,b), i + m s] = sum_a AC[a,s,c] GL[b,i,a]   (AC_s^T GL_i^T, one batch over s per level i)
  for (int i = 0; i < m; ++i)
    zgemm(ctx, OP_T, OP_T, Dr, Dl, Dl, 1.0, AC, (int64_t)Dl * d, Dl, GL + (int64_t)Dl * i, (int64_t)Dl * m, 0, 0.0,
          P.z() + blk * i, Dr, blk * m, d);
  // Q[(c,b), j + n u] = sum_c' GR[c,j,c'] conj(AC[b,u,c'])   (GR_j AC_u^H, one batch over u per level j)
  for (int j = 0; j < n; ++j)
    zgemm(ctx, OP_N, OP_C, Dr, Dl, Dr, 1.0, GR + (int64_t)Dr * j, (int64_t)Dr * n, 0, AC, (int64_t)Dl * d, Dl, 0.0,
          Q.z() + blk * j, Dr, blk * n, d);
  // G[(i,s), (j,u)] = sum_(c,b) P Q: a long-K product, split over K into batches summed on the host
  const int M = m * d, N = n * d;
  const int64_t kc = std::max<int64_t>(4096, (blk + 255) / 256);
  const int64_t nfull = blk / kc, rem = blk - nfull * kc;
  const int64_t nout = nfull + (rem > 0 ? 1 : 0);
  DevBuf& Gp = ctx->buf("grad_gp", (size_t)nout * M * N * sizeof(dcplx));
  if (nfull > 0)
    zgemm(ctx, OP_T, OP_N, M, N, (int)kc, 1.0, P.z(), blk, kc, Q.z(), blk, kc, 0.0, Gp.z(), M, (int64_t)M * N,
          (int)nfull);
  if (rem > 0)
    zgemm(ctx, OP_T, OP_N, M, N, (int)rem, 1.0, P.z() + nfull * kc, blk, 0, Q.z() + nfull * kc, blk, 0, 0.0,
          Gp.z() + nfull * M * N, M, 0, 1);
  std::vector<cplx> hp((size_t)nout * M * N);
  download(ctx, hp.data(), Gp.ptr, hp.size() * sizeof(dcplx));
  for (int s = 0; s < d; ++s)
    for (int i = 0; i < m; ++i)
      for (int u = 0; u < d; ++u)
        for (int j = 0; j < n; ++j) {
          cplx acc = 0.0;
          const size_t r = i + (size_t)m * s, c = j + (size_t)n * u;
          for (int64_t b = 0; b < nout; ++b) acc += hp[(size_t)b * M * N + r + (size_t)M * c];
          const bool identity_block = (i == 0 && j == 0) || (i == m - 1 && j == n - 1);
          G_host[i + (size_t)m * (u + (size_t)d * (j + (size_t)n * s))] = identity_block ? cplx(0.0) : acc;
        }
}

void energy_grad_al(Context* ctx, const imps_envs* E, const imps_mpo* H, const imps_state* st, int site, dcplx* g) {
  Fp64Scope fp64(ctx);
  ProfTag tag(ctx, "grad");
  const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
  IMPS_REQUIRE(E->Dl[site] == Dl && E->Dr[site] == Dr, IMPS_DIM_MISMATCH,
               "energy_grad_al: state and environment shapes disagree");
  const int64_t nel = (int64_t)Dl * d * Dr;
  DevBuf& y = ctx->buf("grad_y", nel * sizeof(dcplx));
  ac_apply(ctx, E, H, site, st->AC[site].z(), y.z());
  const cplx num = zdotc(ctx, nel, st->AC[site].z(), y.z());
  const cplx den = zdotc(ctx, nel, st->AC[site].z(), st->AC[site].z());
  zaxpy(ctx, nel, -num / den, st->AC[site].z(), y.z());
  zgemm(ctx, OP_N, OP_C, Dl * d, Dr, Dr, 1.0, y.z(), (int64_t)Dl * d, 0, st->C[site].z(), Dr, 0, 0.0, g,
        (int64_t)Dl * d, 0, 1);
}

}  // namespace imps
