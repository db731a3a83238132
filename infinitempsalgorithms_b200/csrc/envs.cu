// DMRGCache(psi, H::SparseIMPO) on the device (src/algorithms/groundstates/envs.jl:321-518),
// step for step: per-level cycle-through sweeps, regularized GMRES solves on the
// identity / closing levels, diagonal-channel solves elsewhere, per-site
// regularize! afterwards.  Levels are 1-based in the comments (as in the
// reference) and 0-based in memory.
//
// Device layout: lefts[l] is (Dl, ml, Dl) and rights[l] is (Dr, nr, Dr), column
// major; the level slice X[:, i, :] is a D x D matrix with leading dimension D*levels.
#include "envs.h"

#include <algorithm>
#include <cmath>

#include "krylov.h"

namespace imps {
namespace {

struct Slice {
  dcplx* p;
  int64_t ld;
};
Slice lslice(imps_envs* e, int l, int lvl) {
  return {e->lefts[l].z() + (int64_t)e->Dl[l] * lvl, (int64_t)e->Dl[l] * e->ml[l]};
}
Slice rslice(imps_envs* e, int l, int lvl) {
  return {e->rights[l].z() + (int64_t)e->Dr[l] * lvl, (int64_t)e->Dr[l] * e->nr[l]};
}

struct Builder {
  Context* ctx;
  imps_envs* E;
  const imps_state* st;
  const imps_mpo* H;
  double tol;
  int maxiter, kdim;
  imps_env_info info{};
  std::vector<DevBuf>* initL;
  std::vector<DevBuf>* initR;
  bool warm;

  int N() const { return E->N; }

  // _left_cyclethrough! (envs.jl:121-136): lefts[site+1][:, i, :] = sum_{l<=i} push_slice(...)
  void left_cyclethrough(int i) {
    for (int site = 0; site < N(); ++site) {
      const int snext = (site + 1) % N();
      const MpoSite& W = H->sites[site];
      const int ms = W.m, ns = W.n;
      if (!(i <= ns - 1)) continue;
      std::vector<std::pair<int, int>> blocks;
      for (int l = 1; l <= std::min(i, ms); ++l)
        if (W.block_nonzero(l - 1, i - 1)) blocks.push_back({l - 1, i - 1});
      push_target_left(site, snext, W, blocks, i - 1);
    }
  }
  // _left_closing_sweep! (envs.jl:143-156)
  void left_closing_sweep() {
    for (int site = 0; site < N(); ++site) {
      const int snext = (site + 1) % N();
      const MpoSite& W = H->sites[site];
      const int ms = W.m, ns = W.n;
      std::vector<std::pair<int, int>> blocks;
      for (int l = 1; l <= ms; ++l)
        if (W.block_nonzero(l - 1, ns - 1)) blocks.push_back({l - 1, ns - 1});
      push_target_left(site, snext, W, blocks, ns - 1);
    }
  }
  void push_target_left(int site, int snext, const MpoSite& W, const std::vector<std::pair<int, int>>& blocks, int q) {
    const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
    Slice out = lslice(E, snext, q);
    if (blocks.empty()) {
      zfill2d(ctx, Dr, Dr, 0.0, out.p, out.ld);
      return;
    }
    info.pushes += (int)blocks.size();
    push_left_levels(ctx, W, Dl, d, Dr, E->lefts[site].z(), Dl, (int64_t)Dl * E->ml[site], blocks, W.n, {q},
                     st->AL[site].z(), E->lefts[snext].z(), Dr, (int64_t)Dr * E->ml[snext], false);
  }
  // _right_cyclethrough! (envs.jl:162-177)
  void right_cyclethrough(int i) {
    for (int site = N() - 1; site >= 0; --site) {
      const int sprev = (site - 1 + N()) % N();
      const MpoSite& W = H->sites[site];
      const int ms = W.m, ns = W.n;
      if (!(i <= ms)) continue;
      std::vector<std::pair<int, int>> blocks;
      for (int l = i; l <= ns; ++l)
        if (W.block_nonzero(i - 1, l - 1)) blocks.push_back({i - 1, l - 1});
      const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
      Slice out = rslice(E, sprev, i - 1);
      if (blocks.empty()) {
        zfill2d(ctx, Dl, Dl, 0.0, out.p, out.ld);
        continue;
      }
      info.pushes += (int)blocks.size();
      push_right_levels(ctx, W, Dl, d, Dr, E->rights[site].z(), Dr, (int64_t)Dr * E->nr[site], blocks, {i - 1},
                        st->AR[site].z(), E->rights[sprev].z(), Dl, (int64_t)Dl * E->nr[sprev], false);
    }
  }

  // x <- solution of (1 - op) x = rhs with GMRES (linsolve with a0 = 1, a1 = -1)
  void solve(const LinOp& op, int D, Slice target, const dcplx* prev_contig) {
    // GMRES refines in FP64, so the inner Krylov cycles only need a moderate accuracy
    TolScope inner(ctx, 1e-6);
    const int64_t n = (int64_t)D * D;
    DevBuf& rhs = ctx->buf("env_rhs", n * sizeof(dcplx));
    DevBuf& x = ctx->buf("env_x", n * sizeof(dcplx));
    zcopy2d(ctx, D, D, target.p, target.ld, rhs.z(), D);
    zcopy(ctx, n, prev_contig, x.z());
    KrylovResult r = gmres(ctx, n, op, rhs.z(), x.z(), tol, kdim, maxiter, 1.0, -1.0);
    info.solves++;
    info.gmres_iters += r.numiter;
    info.gmres_ops += r.numops;
    info.max_normres = std::max(info.max_normres, r.normres);
    if (!r.converged) info.converged = 0;
    zcopy2d(ctx, D, D, x.z(), D, target.p, target.ld);
  }

  // previous value of a level (warm start = init_lefts/init_rights, else the current zeros)
  const dcplx* prev_left(int lvl) {
    const int D = E->Dl[0];
    DevBuf& p = ctx->buf("env_prev", (size_t)D * D * sizeof(dcplx));
    const dcplx* src = warm ? (*initL)[0].z() : E->lefts[0].z();
    zcopy2d(ctx, D, D, src + (int64_t)D * lvl, (int64_t)D * E->ml[0], p.z(), D);
    return p.z();
  }
  const dcplx* prev_right(int lvl) {
    const int N1 = N() - 1, D = E->Dr[N1];
    DevBuf& p = ctx->buf("env_prev", (size_t)D * D * sizeof(dcplx));
    const dcplx* src = warm ? (*initR)[N1].z() : E->rights[N1].z();
    zcopy2d(ctx, D, D, src + (int64_t)D * lvl, (int64_t)D * E->nr[N1], p.z(), D);
    return p.z();
  }

  // regularize!(X, rho, I): X -= tr(rho X) I
  void regularize(int D, dcplx* X, int64_t ldx, const dcplx* rho) {
    cplx c = ztrace_prod(ctx, D, rho, D, X, ldx);
    zadd_diag(ctx, D, X, ldx, -c);
  }

  void run() {
    const int N = this->N();
    info.converged = 1;
    // right-hand-side sweeps: error of the split engine kept well below the solver tolerance
    TolScope rhs_tol(ctx, tol * 1e-2);
    const int DN = st->Dr(N - 1);
    // rho_r = C[N] C[N]^H (left solves), rho_l = C[N]^H C[N] (right solves)
    DevBuf& rho_r = ctx->buf("env_rho_r", (size_t)DN * DN * sizeof(dcplx));
    DevBuf& rho_l = ctx->buf("env_rho_l", (size_t)DN * DN * sizeof(dcplx));
    zgemm(ctx, OP_N, OP_C, DN, DN, DN, 1.0, st->C[N - 1].z(), DN, 0, st->C[N - 1].z(), DN, 0, 0.0, rho_r.z(), DN, 0, 1, false);
    zgemm(ctx, OP_C, OP_N, DN, DN, DN, 1.0, st->C[N - 1].z(), DN, 0, st->C[N - 1].z(), DN, 0, 0.0, rho_l.z(), DN, 0, 1, false);
    int jmax = 0;
    for (int l = 0; l < N; ++l) jmax = std::max(jmax, E->nr[l]);
    jmax -= 1;
    const int D0 = E->Dl[0];
    // identity-channel left transfer chain T_AL^N with the regularization
    LinOp opL_reg = [&](const dcplx* v, dcplx* out) {
      DevBuf& a = ctx->buf("env_tm_a", (size_t)D0 * D0 * sizeof(dcplx));
      DevBuf& b = ctx->buf("env_tm_b", (size_t)D0 * D0 * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = 0; l < N; ++l) {
        dcplx* dst = (l == N - 1) ? out : ((l % 2 == 0) ? a.z() : b.z());
        push_left_id(ctx, st->Dl(l), st->d[l], st->Dr(l), cur, st->AL[l].z(), st->AL[l].z(), dst);
        info.pushes++;
        cur = dst;
      }
      regularize(D0, out, D0, rho_r.z());
    };
    // ---- left environments (envs.jl:363-421)
    for (int i = 2; i <= jmax; ++i) {
      if (i <= E->ml[0] - 1) {
        const dcplx* prev = prev_left(i - 1);
        DevBuf& prevc = ctx->buf("env_prev_keep", (size_t)D0 * D0 * sizeof(dcplx));
        zcopy(ctx, (int64_t)D0 * D0, prev, prevc.z());
        left_cyclethrough(i);
        if (H->isidentitylevel(i)) {
          solve(opL_reg, D0, lslice(E, 0, i - 1), prevc.z());
          if (N > 1) left_cyclethrough(i);
          regularize_left_level(i - 1, false);
        } else {
          if (!H->isemptylevel(i)) {
            LinOp op = diag_left_op(i);
            solve(op, D0, lslice(E, 0, i - 1), prevc.z());
          }
          if (N > 1) left_cyclethrough(i);
        }
      } else {
        left_cyclethrough(i);
      }
    }
    // ---- closing level of the left environments (envs.jl:424-455)
    {
      const int i = E->ml[0];
      const dcplx* prev = prev_left(i - 1);
      DevBuf& prevc = ctx->buf("env_prev_keep", (size_t)D0 * D0 * sizeof(dcplx));
      zcopy(ctx, (int64_t)D0 * D0, prev, prevc.z());
      left_closing_sweep();
      solve(opL_reg, D0, lslice(E, 0, i - 1), prevc.z());
      if (N > 1) left_closing_sweep();
      regularize_left_level(-1, true);
    }
    // ---- right environments (envs.jl:461-515)
    const int DRN = E->Dr[N - 1];
    LinOp opR_reg = [&](const dcplx* v, dcplx* out) {
      DevBuf& a = ctx->buf("env_tm_a", (size_t)DRN * DRN * sizeof(dcplx));
      DevBuf& b = ctx->buf("env_tm_b", (size_t)DRN * DRN * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = N - 1, k = 0; l >= 0; --l, ++k) {
        dcplx* dst = (l == 0) ? out : ((k % 2 == 0) ? a.z() : b.z());
        push_right_id(ctx, st->Dl(l), st->d[l], st->Dr(l), cur, st->AR[l].z(), st->AR[l].z(), dst);
        info.pushes++;
        cur = dst;
      }
      regularize(DRN, out, DRN, rho_l.z());
    };
    for (int i = jmax; i >= 1; --i) {
      if (i <= E->nr[N - 1] - 1) {
        const dcplx* prev = prev_right(i - 1);
        DevBuf& prevc = ctx->buf("env_prev_keep", (size_t)DRN * DRN * sizeof(dcplx));
        zcopy(ctx, (int64_t)DRN * DRN, prev, prevc.z());
        right_cyclethrough(i);
        if (H->isidentitylevel(i)) {
          solve(opR_reg, DRN, rslice(E, N - 1, i - 1), prevc.z());
          if (N > 1) right_cyclethrough(i);
          for (int l = 0; l < N; ++l) {
            const int D = E->Dr[l];
            DevBuf& rho = ctx->buf("env_rho_site", (size_t)D * D * sizeof(dcplx));
            zgemm(ctx, OP_C, OP_N, D, D, D, 1.0, st->C[l].z(), D, 0, st->C[l].z(), D, 0, 0.0, rho.z(), D, 0, 1, false);
            Slice s = rslice(E, l, i - 1);
            regularize(D, s.p, s.ld, rho.z());
          }
        } else {
          if (!H->isemptylevel(i)) {
            LinOp op = diag_right_op(i);
            solve(op, DRN, rslice(E, N - 1, i - 1), prevc.z());
          }
          if (N > 1) right_cyclethrough(i);
        }
      } else {
        right_cyclethrough(i);
      }
    }
  }

  // per-site regularize! of a left level (closing: each site's own last level)
  void regularize_left_level(int lvl, bool closing) {
    for (int l = 0; l < N(); ++l) {
      const int D = E->Dl[l];
      const int prevsite = (l - 1 + N()) % N();
      DevBuf& rho = ctx->buf("env_rho_site", (size_t)D * D * sizeof(dcplx));
      zgemm(ctx, OP_N, OP_C, D, D, D, 1.0, st->C[prevsite].z(), D, 0, st->C[prevsite].z(), D, 0, 0.0, rho.z(), D, 0,
            1, false);
      Slice s = lslice(E, l, closing ? E->ml[l] - 1 : lvl);
      regularize(D, s.p, s.ld, rho.z());
    }
  }

  // diagonal channel chain: X -> push_slice(X, W_l[i,i], AL_l) over the unit cell
  LinOp diag_left_op(int i) {
    return [this, i](const dcplx* v, dcplx* out) {
      const int N = this->N();
      bool zero = false;
      for (int l = 0; l < N; ++l) {
        const MpoSite& W = H->sites[l];
        if (!(i <= std::min(W.m, W.n)) || !W.block_nonzero(i - 1, i - 1)) zero = true;
      }
      const int D = E->Dl[0];
      if (zero) {
        zfill(ctx, (int64_t)D * D, 0.0, out);
        return;
      }
      DevBuf& a = ctx->buf("env_tm_a", (size_t)D * D * sizeof(dcplx));
      DevBuf& b = ctx->buf("env_tm_b", (size_t)D * D * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = 0; l < N; ++l) {
        dcplx* dst = (l == N - 1) ? out : ((l % 2 == 0) ? a.z() : b.z());
        const int Dl = st->Dl(l), d = st->d[l], Dr = st->Dr(l);
        // single block (i-1, i-1): L_l = cur (contiguous, level stride 0), output to dst
        push_left_levels(ctx, H->sites[l], Dl, d, Dr, cur, 0, Dl, {{i - 1, i - 1}}, H->sites[l].n, {i - 1},
                         st->AL[l].z(), dst, 0, Dr, false);
        info.pushes++;
        cur = dst;
      }
    };
  }
  LinOp diag_right_op(int i) {
    return [this, i](const dcplx* v, dcplx* out) {
      const int N = this->N();
      bool zero = false;
      for (int l = 0; l < N; ++l) {
        const MpoSite& W = H->sites[l];
        if (!(i <= std::min(W.m, W.n)) || !W.block_nonzero(i - 1, i - 1)) zero = true;
      }
      const int D = E->Dr[N - 1];
      if (zero) {
        zfill(ctx, (int64_t)D * D, 0.0, out);
        return;
      }
      DevBuf& a = ctx->buf("env_tm_a", (size_t)D * D * sizeof(dcplx));
      DevBuf& b = ctx->buf("env_tm_b", (size_t)D * D * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = N - 1, k = 0; l >= 0; --l, ++k) {
        dcplx* dst = (l == 0) ? out : ((k % 2 == 0) ? a.z() : b.z());
        const int Dl = st->Dl(l), d = st->d[l], Dr = st->Dr(l);
        push_right_levels(ctx, H->sites[l], Dl, d, Dr, cur, 0, Dr, {{i - 1, i - 1}}, {i - 1}, st->AR[l].z(), dst, 0,
                          Dl, false);
        info.pushes++;
        cur = dst;
      }
    };
  }
};

}  // namespace

void envs_allocate(imps_envs* E, const imps_state* st, const imps_mpo* H) {
  const int N = st->N;
  IMPS_REQUIRE(H->N >= 1 && N % H->N == 0, IMPS_DIM_MISMATCH, "state unit cell must be a multiple of the MPO's");
  E->N = N;
  E->Dl.resize(N);
  E->Dr.resize(N);
  E->ml.resize(N);
  E->nr.resize(N);
  E->lefts.resize(N);
  E->rights.resize(N);
  E->init_lefts.resize(N);
  E->init_rights.resize(N);
  E->GLp.resize(N);
  E->GLp_valid.assign(N, false);
  E->hest_ac.assign(N, 0.0);
  E->hest_c.assign(N, 0.0);
  for (int l = 0; l < N; ++l) {
    const MpoSite& W = H->sites[l % H->N];
    IMPS_REQUIRE(W.d == st->d[l], IMPS_DIM_MISMATCH, "MPO physical dimension != state physical dimension");
    E->Dl[l] = st->Dl(l);
    E->Dr[l] = st->Dr(l);
    E->ml[l] = W.m;
    E->nr[l] = W.n;
    E->lefts[l].ensure((size_t)E->Dl[l] * W.m * E->Dl[l] * sizeof(dcplx));
    E->rights[l].ensure((size_t)E->Dr[l] * W.n * E->Dr[l] * sizeof(dcplx));
  }
  IMPS_REQUIRE(H->sites[(N - 1) % H->N].n == H->sites[0].m, IMPS_DIM_MISMATCH,
               "operator level chain does not close over the ket unit cell");
}

imps_env_info envs_build(Context* ctx, imps_envs* E, const imps_state* st, const imps_mpo* H, double tol, int maxiter,
                         int krylovdim, bool warm) {
  const int N = E->N;
  IMPS_REQUIRE(st->N == N, IMPS_DIM_MISMATCH, "state / environment unit cells differ");
  for (int l = 0; l < N; ++l)
    IMPS_REQUIRE(E->Dl[l] == st->Dl(l) && E->Dr[l] == st->Dr(l), IMPS_DIM_MISMATCH,
                 "environment bond dimensions differ from the state's");
  // keep the previous environments as the warm start (init_lefts / init_rights), start from zeros
  for (int l = 0; l < N; ++l) {
    if (warm) {
      std::swap(E->lefts[l], E->init_lefts[l]);
      std::swap(E->rights[l], E->init_rights[l]);
      E->lefts[l].ensure(E->init_lefts[l].bytes);
      E->rights[l].ensure(E->init_rights[l].bytes);
    }
    const int Dl = E->Dl[l], Dr = E->Dr[l];
    zfill(ctx, (int64_t)Dl * E->ml[l] * Dl, 0.0, E->lefts[l].z());
    zfill(ctx, (int64_t)Dr * E->nr[l] * Dr, 0.0, E->rights[l].z());
    Slice s = lslice(E, l, 0);
    zset_identity(ctx, Dl, s.p, s.ld, 1.0);
    Slice r = rslice(E, l, E->nr[l] - 1);
    zset_identity(ctx, Dr, r.p, r.ld, 1.0);
    E->GLp_valid[l] = false;
  }
  // the site tensors are constant for the whole build: their int8 splits are cached
  std::vector<const void*> cptrs;
  for (int l = 0; l < N; ++l) {
    cptrs.push_back(st->AL[l].ptr);
    cptrs.push_back(st->AR[l].ptr);
  }
  ConstScope cs(ctx, cptrs);
  Builder b;
  b.ctx = ctx;
  b.E = E;
  b.st = st;
  b.H = H;
  b.tol = tol;
  b.maxiter = maxiter;
  b.kdim = std::min(E->Dl[0] * E->Dl[0], krylovdim);
  b.initL = &E->init_lefts;
  b.initR = &E->init_rights;
  b.warm = warm;
  b.run();
  E->version++;
  E->last = b.info;
  return b.info;
}

}  // namespace imps
