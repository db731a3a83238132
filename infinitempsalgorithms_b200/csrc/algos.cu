// Observables and algorithm steps on the device:
//   calc_galerkin       (src/algorithms/groundstates/vumps.jl:111-124)
//   Schur energy        (src/observables/expval.jl:93-112)
//   local expectation   (expval.jl:33-37)
//   localupdate_step!   (vumps.jl:7-19), one VUMPS iteration (vumps.jl:51-85)
//   TDVP timestep       (src/algorithms/timeevo/tdvp.jl:34-53)
//   IDMRG sweep         (src/algorithms/groundstates/idmrg.jl:12-33)
#include "algos.h"

#include <algorithm>
#include <cmath>

#include "envs.h"
#include "gauge.h"
#include "krylov.h"
#include "mpo.h"

namespace imps {

namespace {
double dyn_tol(double eps, double factor, int iter) {
  // updatetol(DynamicTol(alg, tol_min = 1e-14, tol_max = 1e-4, factor), iter, eps) (utility.jl:153-157)
  iter = std::max(iter, 1);
  return std::min(std::max(eps * factor / std::sqrt((double)iter), 1e-14), 1e-4);
}
}  // namespace

double galerkin(Context* ctx, imps_envs* E, const imps_mpo* H, const imps_state* st) {
  Fp64Scope fp64(ctx);  // the Galerkin residual is always FP64
  ProfTag tag(ctx, "galerkin");
  double eps = 0.0;
  for (int site = 0; site < st->N; ++site) {
    const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
    const int64_t n = (int64_t)Dl * d * Dr;
    DevBuf& x = ctx->buf("gal_x", n * sizeof(dcplx));
    DevBuf& q = ctx->buf("gal_q", (size_t)Dr * Dr * sizeof(dcplx));
    ac_apply(ctx, E, H, site, st->AC[site].z(), x.z());
    double nx = dznrm2(ctx, n, x.z());
    zscal(ctx, n, 1.0 / nx, x.z());
    zgemm(ctx, OP_C, OP_N, Dr, Dr, Dl * d, 1.0, st->AL[site].z(), (int64_t)Dl * d, 0, x.z(), (int64_t)Dl * d, 0, 0.0,
          q.z(), Dr, 0, 1, false);
    zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, -1.0, st->AL[site].z(), (int64_t)Dl * d, 0, q.z(), Dr, 0, 1.0, x.z(),
          (int64_t)Dl * d, 0, 1, false);
    eps = std::max(eps, dznrm2(ctx, n, x.z()));
  }
  return eps;
}

cplx energy(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st) {
  Fp64Scope fp64(ctx);
  ProfTag tag(ctx, "energy");
  cplx e = 0.0;
  for (int site = 0; site < st->N; ++site) {
    const MpoSite& col = H->closing[site % H->N];
    const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
    const int64_t n = (int64_t)Dl * d * Dr;
    DevBuf& y = ctx->buf("en_y", n * sizeof(dcplx));
    const dcplx* GRe = E->rights[site].z() + (int64_t)Dr * (E->nr[site] - 1);
    ac_apply(ctx, E, H, site, st->AC[site].z(), y.z(), &col, GRe, (int64_t)Dr * E->nr[site]);
    (void)d;
    e += zdotc(ctx, n, st->AC[site].z(), y.z());
  }
  return e / state_dot(ctx, st);
}

cplx local_expval(Context* ctx, imps_state* st, int site, const cplx* O) {
  Fp64Scope fp64(ctx);
  const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
  const int64_t n = (int64_t)Dl * d * Dr;
  DevBuf& y = ctx->buf("lexp_y", n * sizeof(dcplx));
  DevBuf& Od = ctx->buf("lexp_o", (size_t)d * d * sizeof(dcplx));
  upload(ctx, Od.ptr, O, (size_t)d * d * sizeof(dcplx));
  // Y[a, u, b] = sum_s O[u, s] AC[a, s, b]
  MixPlan pl;
  pl.Db = Dl; pl.R = 1; pl.P = d; pl.Q = 1; pl.S = d; pl.C = Dr;
  pl.in_r = 0; pl.in_s = Dl; pl.in_c = (int64_t)Dl * d;
  pl.out_p = Dl; pl.out_q = 0; pl.out_c = (int64_t)Dl * d;
  pl.M = Od.z();
  pl.nz = {{0, 0}};
  level_mix(ctx, pl, st->AC[site].z(), y.z());
  cplx v = zdotc(ctx, n, st->AC[site].z(), y.z());
  return v / state_dot(ctx, st);
}

namespace {
// Lanczos on the split engine, then (if the engine's accuracy floor is above the
// requested tolerance) an FP64 Lanczos polish warm-started from the split result.
// `hest` is a running estimate of |lambda|, the scale of the matvec error.
KrylovResult mixed_eigsolve(Context* ctx, int64_t n, const LinOp& op, const dcplx* x0, dcplx* x, double tol, int kdim,
                            int maxiter, bool eager, double& hest) {
  if (ctx->precision != PREC_SPLIT_I8 || ctx->force_fp64 > 0)
    return lanczos_eigsolve(ctx, n, op, x0, x, tol, kdim, maxiter, eager);
  const double scale = hest > 0 ? hest : 1.0;
  KrylovResult r1;
  double floor_abs;
  {
    TolScope ts(ctx, tol / (8.0 * scale));
    floor_abs = split_floor(ctx) * scale;
    r1 = lanczos_eigsolve(ctx, n, op, x0, x, std::max(tol, floor_abs), kdim, maxiter, eager);
  }
  hest = std::max(std::abs(r1.value), 1e-300);
  if (floor_abs <= tol) return r1;
  KrylovResult r2;
  {
    Fp64Scope fp64(ctx);
    r2 = lanczos_eigsolve(ctx, n, op, x, x, tol, kdim, maxiter, eager);
  }
  r2.numops += r1.numops;
  r2.numiter += r1.numiter;
  return r2;
}
}  // namespace

KrylovResult eigsolve_ac(Context* ctx, imps_envs* E, const imps_mpo* H, int site, const dcplx* x0, dcplx* x,
                         double tol, int kdim, int maxiter, bool eager) {
  const int64_t n = (int64_t)E->Dl[site] * H->sites[site % H->N].d * E->Dr[site];
  ConstScope cs(ctx, {E->lefts[site].ptr, E->rights[site].ptr});
  ProfTag tag(ctx, "eig_ac");
  LinOp op = [&](const dcplx* v, dcplx* out) { ac_apply(ctx, E, H, site, v, out); };
  return mixed_eigsolve(ctx, n, op, x0, x, tol, kdim, maxiter, eager, E->hest_ac[site]);
}

KrylovResult eigsolve_c(Context* ctx, imps_envs* E, int site, const dcplx* x0, dcplx* x, double tol, int kdim,
                        int maxiter, bool eager) {
  const int64_t n = (int64_t)E->Dr[site] * E->Dr[site];
  const int l1 = (site + 1) % E->N;
  ensure_GLp(ctx, E, l1);
  ConstScope cs(ctx, {E->GLp[l1].ptr, E->rights[site].ptr});
  ProfTag tag(ctx, "eig_c");
  LinOp op = [&](const dcplx* v, dcplx* out) { c_apply(ctx, E, site, v, out); };
  return mixed_eigsolve(ctx, n, op, x0, x, tol, kdim, maxiter, eager, E->hest_c[site]);
}

// The Lanczos exponentiate has no residual refinement: its error estimate
// (beta h_{m+1,m} |e_m^T exp(tau H_m) e_1|) assumes matvecs exact well below the
// tolerance, which a sliced product does not give, and with inexact matvecs the
// sub-step halving can shrink tau without end (a D=512 TFIM step did not finish
// in 230 s in split precision; 0.44 s in FP64).  TDVP integrates in FP64 in both
// precision modes; the environment solves of the step may still use the split
// engine, since their GMRES refines against an FP64 residual.
KrylovResult expo_ac(Context* ctx, imps_envs* E, const imps_mpo* H, int site, cplx dt, const dcplx* x0, dcplx* x,
                     double tol, int kdim, int maxiter) {
  const int64_t n = (int64_t)E->Dl[site] * H->sites[site % H->N].d * E->Dr[site];
  Fp64Scope fp64(ctx);
  ConstScope cs(ctx, {E->lefts[site].ptr, E->rights[site].ptr});
  const double scale = (E->hest_ac[site] > 0 ? E->hest_ac[site] : 1.0) * std::max(std::abs(dt), 1e-300);
  TolScope ts(ctx, tol / (8.0 * scale));
  LinOp op = [&](const dcplx* v, dcplx* out) { ac_apply(ctx, E, H, site, v, out); };
  return exponentiate(ctx, n, op, dt, x0, x, tol, kdim, maxiter);
}

KrylovResult expo_c(Context* ctx, imps_envs* E, int site, cplx dt, const dcplx* x0, dcplx* x, double tol, int kdim,
                    int maxiter) {
  Fp64Scope fp64(ctx);  // see expo_ac
  const int64_t n = (int64_t)E->Dr[site] * E->Dr[site];
  const int l1 = (site + 1) % E->N;
  ensure_GLp(ctx, E, l1);
  ConstScope cs(ctx, {E->GLp[l1].ptr, E->rights[site].ptr});
  const double scale = (E->hest_c[site] > 0 ? E->hest_c[site] : 1.0) * std::max(std::abs(dt), 1e-300);
  TolScope ts(ctx, tol / (8.0 * scale));
  LinOp op = [&](const dcplx* v, dcplx* out) { c_apply(ctx, E, site, v, out); };
  return exponentiate(ctx, n, op, dt, x0, x, tol, kdim, maxiter);
}

void vumps_localupdate(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, double tol, int kdim, int maxiter,
                       bool eager, int* nac, int* nc) {
  int ac_ops = 0, c_ops = 0;
  for (int site = 0; site < st->N; ++site) {
    const int Dl = st->Dl(site), d = st->d[site], Dr = st->Dr(site);
    DevBuf& ac = ctx->buf("lu_ac", (size_t)Dl * d * Dr * sizeof(dcplx));
    DevBuf& c = ctx->buf("lu_c", (size_t)Dr * Dr * sizeof(dcplx));
    KrylovResult r1 = eigsolve_ac(ctx, E, H, site, st->AC[site].z(), ac.z(), tol, kdim, maxiter, eager);
    KrylovResult r2 = eigsolve_c(ctx, E, site, st->C[site].z(), c.z(), tol, kdim, maxiter, eager);
    ac_ops += r1.numops;
    c_ops += r2.numops;
    ProfTag tag(ctx, "regauge");
    regauge(ctx, Dl, d, Dr, ac.z(), c.z(), st->AL[site].z());
  }
  if (nac) *nac = ac_ops;
  if (nc) *nc = c_ops;
}

imps_vumps_info vumps_iter(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, int iter, double eps) {
  imps_vumps_info info{};
  const int siter = iter - 1;
  int nac = 0, nc = 0;
  vumps_localupdate(ctx, E, H, st, dyn_tol(eps, 1e-3, siter), 30, 300, true, &nac, &nc);
  const int N = st->N, DN = st->Dr(N - 1);
  DevBuf& c0 = ctx->buf("vumps_c0", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), c0.z());
  GaugeResult g;
  {
    ProfTag tag(ctx, "gauge");
    g = from_al(ctx, st, c0.z(), dyn_tol(eps, 1e-6, siter), 300);
  }
  imps_env_info ei;
  {
    ProfTag tag(ctx, "envs");
    ei = envs_build(ctx, E, st, H, dyn_tol(eps, 1e-4, siter), 300, 30, true);
  }
  info.galerkin = galerkin(ctx, E, H, st);
  cplx e = energy(ctx, E, H, st);
  info.energy_re = e.real();
  info.energy_im = e.imag();
  info.ac_matvecs = nac;
  info.c_matvecs = nc;
  info.gauge_iters = g.niter;
  info.env_gmres_ops = ei.gmres_ops;
  info.env = ei;
  return info;
}

KrylovResult tdvp_step(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, cplx dt, double tol, int kdim,
                       int maxiter, double gauge_tol, int gauge_maxiter) {
  const int N = st->N;
  KrylovResult agg;
  agg.converged = 1;
  size_t acs = 0, cs = 0;
  for (int l = 0; l < N; ++l) {
    acs += st->site_elems(l);
    cs += st->bond_elems(l);
  }
  DevBuf& ACn = ctx->buf("tdvp_ac", acs * sizeof(dcplx));
  DevBuf& Cn = ctx->buf("tdvp_c", cs * sizeof(dcplx));
  std::vector<dcplx*> pac(N), pc(N);
  size_t oa = 0, oc = 0;
  for (int l = 0; l < N; ++l) {
    pac[l] = ACn.z() + oa;
    pc[l] = Cn.z() + oc;
    oa += st->site_elems(l);
    oc += st->bond_elems(l);
  }
  for (int l = 0; l < N; ++l) {
    ProfTag tag(ctx, "expo");
    KrylovResult r1 = expo_ac(ctx, E, H, l, dt, st->AC[l].z(), pac[l], tol, kdim, maxiter);
    KrylovResult r2 = expo_c(ctx, E, l, dt, st->C[l].z(), pc[l], tol, kdim, maxiter);
    agg.numops += r1.numops + r2.numops;
    agg.numiter += r1.numiter + r2.numiter;
    agg.converged &= r1.converged & r2.converged;
    agg.normres = std::max({agg.normres, r1.normres, r2.normres});
  }
  {
    ProfTag tag(ctx, "regauge");
    for (int l = 0; l < N; ++l) regauge(ctx, st->Dl(l), st->d[l], st->Dr(l), pac[l], pc[l], st->AL[l].z());
  }
  const int DN = st->Dr(N - 1);
  DevBuf& c0 = ctx->buf("vumps_c0", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), c0.z());
  {
    ProfTag tag(ctx, "gauge");
    from_al(ctx, st, c0.z(), gauge_tol, gauge_maxiter);
  }
  {
    ProfTag tag(ctx, "envs");
    envs_build(ctx, E, st, H, 1e-10, 300, 30, true);
  }
  return agg;
}

void idmrg_sweep(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, double tol, int kdim, int maxiter,
                 bool eager, double* Eout, double* epsout) {
  const int N = st->N;
  const int DN = st->Dr(N - 1);
  DevBuf& Cold = ctx->buf("idmrg_cold", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), Cold.z());
  for (int pos = 0; pos < N; ++pos) {
    const int Dl = st->Dl(pos), d = st->d[pos], Dr = st->Dr(pos);
    const int64_t n = (int64_t)Dl * d * Dr;
    DevBuf& ac = ctx->buf("idmrg_ac", n * sizeof(dcplx));
    eigsolve_ac(ctx, E, H, pos, st->AC[pos].z(), ac.z(), tol, kdim, maxiter, eager);
    qrpos(ctx, Dl * d, Dr, ac.z(), (int64_t)Dl * d, st->AL[pos].z(), st->C[pos].z());
    if (pos != N - 1) zcopy(ctx, n, st->AL[pos].z(), st->AC[pos].z());
    else zcopy(ctx, n, ac.z(), st->AC[pos].z());
    const int nxt = (pos + 1) % N;
    DevBuf& tmp = ctx->buf("idmrg_env", E->lefts[nxt].bytes);
    push_mpo_left(ctx, H->sites[pos % H->N], Dl, d, Dr, E->lefts[pos].z(), st->AL[pos].z(), tmp.z());
    zcopy(ctx, (int64_t)(E->lefts[nxt].bytes / sizeof(dcplx)), tmp.z(), E->lefts[nxt].z());
    E->GLp_valid[nxt] = false;
  }
  double Elast = 0.0;
  for (int pos = N - 1; pos >= 0; --pos) {
    const int Dl = st->Dl(pos), d = st->d[pos], Dr = st->Dr(pos);
    const int64_t n = (int64_t)Dl * d * Dr;
    DevBuf& ac = ctx->buf("idmrg_ac", n * sizeof(dcplx));
    KrylovResult r = eigsolve_ac(ctx, E, H, pos, st->AC[pos].z(), ac.z(), tol, kdim, maxiter, eager);
    Elast = r.value.real();
    const int prv = (pos - 1 + N) % N;
    lqpos(ctx, Dl, d * Dr, ac.z(), Dl, st->C[prv].z(), st->AR[pos].z());
    if (pos != 0) zcopy(ctx, n, st->AR[pos].z(), st->AC[pos].z());
    else zcopy(ctx, n, ac.z(), st->AC[pos].z());
    DevBuf& tmp = ctx->buf("idmrg_env", E->rights[prv].bytes);
    push_mpo_right(ctx, H->sites[pos % H->N], Dl, d, Dr, E->rights[pos].z(), st->AR[pos].z(), tmp.z());
    zcopy(ctx, (int64_t)(E->rights[prv].bytes / sizeof(dcplx)), tmp.z(), E->rights[prv].z());
  }
  for (int l = 0; l < N; ++l) E->GLp_valid[l] = false;
  DevBuf& diff = ctx->buf("idmrg_diff", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), diff.z());
  zaxpy(ctx, (int64_t)DN * DN, -1.0, Cold.z(), diff.z());
  if (epsout) *epsout = dznrm2(ctx, (int64_t)DN * DN, diff.z());
  if (Eout) *Eout = Elast;
}

}  // namespace imps
