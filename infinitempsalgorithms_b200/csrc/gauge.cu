// Gauge fixing on the device: uniform_leftorth! / uniform_rightorth!
// (src/states/ortho.jl:125-202), regauge! (:214-219), the CanonicalIMPS
// constructors (src/states/canonicalmps.jl:151-195), gauge_step!
// (src/algorithms/groundstates/vumps.jl:23-31) and dot(psi, psi)
// (canonicalmps.jl:262-269).  All factorizations are FP64 QRpos / LQpos.
#include "gauge.h"

#include <algorithm>
#include <cmath>
#include <string>

#include "krylov.h"

namespace imps {
namespace {

double eig_tol_from(double eps) {
  // _GAUGE_ALG_EIGSOLVE = alg_eigsolve(ishermitian = false, tol_factor = 1) (ortho.jl:6):
  // updatetol(alg, 1, eps^2) = clamp(eps^2, tol_min = 1e-14, tol_max = 1e-4)
  return std::min(std::max(eps * eps, 1e-14), 1e-4);
}

// Copies of the input site tensors (the sweep may write into storage aliasing A).
std::vector<dcplx*> work_copy(Context* ctx, const imps_state* st, const std::vector<const dcplx*>& A,
                              const char* name) {
  size_t total = 0;
  for (int l = 0; l < st->N; ++l) total += st->site_elems(l);
  DevBuf& W = ctx->buf(name, total * sizeof(dcplx));
  std::vector<dcplx*> out(st->N);
  size_t off = 0;
  for (int l = 0; l < st->N; ++l) {
    out[l] = W.z() + off;
    zcopy(ctx, st->site_elems(l), A[l], out[l]);
    off += st->site_elems(l);
  }
  return out;
}

double diff_norm(Context* ctx, int64_t n, const dcplx* a, const dcplx* b) {
  DevBuf& T = ctx->buf("gauge_diff", n * sizeof(dcplx));
  zcopy(ctx, n, a, T.z());
  zaxpy(ctx, n, -1.0, b, T.z());
  return dznrm2(ctx, n, T.z());
}

// The transfer-matrix eigensolve of a gauge sweep.  Its fixed point only seeds the next
// sweep, whose own FP64 convergence test decides, so the products may run on the split
// engine at a tenth of the eigensolver tolerance (the site tensors are constant over the
// eigensolve: their splits are cached).  When that tolerance needs more than six slices,
// a solve to 1e-8 at up to six slices seeds a solve whose products use up to eight
// (truncation below 2^-56 of the row and column scales, the accuracy of an FP64 product;
// about 1.8x faster than the FP64 engine on the 1024 x 4096 x 1024 products of d = 4,
// D = 1024).
void gauge_eigsolve(Context* ctx, int64_t n, const LinOp& op, const dcplx* c0, dcplx* ev, double etol,
                    const std::vector<const void*>& cptrs) {
  ConstScope cs(ctx, cptrs);
  const bool split = ctx->precision == PREC_SPLIT_I8 && ctx->adaptive_slices;
  if (split && etol < 1e-8 && slices_for_tol(0.1 * etol) >= 7) {
    DevBuf& seed = ctx->buf("gauge_seed", (size_t)n * sizeof(dcplx));
    {
      SplitAllowScope sa(ctx, 1e-9);
      arnoldi_dominant(ctx, n, op, c0, seed.z(), 1e-8, 30, 300, true);
    }
    SplitAllowScope sa(ctx, 0.1 * etol);
    MaxSlicesScope ms(ctx, 8);
    arnoldi_dominant(ctx, n, op, seed.z(), ev, etol, 30, 300, true);
    return;
  }
  SplitAllowScope sa(ctx, 0.1 * etol);
  arnoldi_dominant(ctx, n, op, c0, ev, etol, 30, 300, true);
}

// Reflector storage of site i's factorisation in a gauge sweep.
std::string sweep_slot(int i) { return "gauge_sweep" + std::to_string(i); }

// A sweep only needs its L (R) factors to go on; its AR (AL) tensors are read by the
// transfer-matrix eigensolve that starts the next iteration (from eig_miniter on) and
// are the result when the iteration stops.  Other sweeps leave Q unformed; `it` counts
// the sweeps done, this one included.
bool sweep_q_needed(double eps, double tol, int it, int maxiter, int eig_miniter) {
  return eps < tol || it > maxiter || it >= eig_miniter;
}

}  // namespace

GaugeResult uniform_leftorth(Context* ctx, imps_state* st, const std::vector<const dcplx*>& A, const dcplx* C0,
                             double tol, int maxiter, int eig_miniter) {
  Fp64Scope fp64(ctx);  // gauge fixing stays FP64
  const int N = st->N;
  GaugeResult res;
  std::vector<dcplx*> Aw = work_copy(ctx, st, A, "gauge_awork");
  const int DN = st->Dr(N - 1);
  {
    DevBuf& t = ctx->buf("gauge_c0", (size_t)DN * DN * sizeof(dcplx));
    zcopy(ctx, (int64_t)DN * DN, C0, t.z());
    double nc = dznrm2(ctx, (int64_t)DN * DN, t.z());
    zaxpby(ctx, (int64_t)DN * DN, 1.0 / nc, t.z(), 0.0, st->C[N - 1].z());
  }
  DevBuf& Cpre = ctx->buf("gauge_cpre", (size_t)DN * DN * sizeof(dcplx));
  DevBuf& M = ctx->buf("gauge_m", [&] {
    size_t mx = 0;
    for (int l = 0; l < N; ++l) mx = std::max(mx, st->site_elems(l));
    return mx * sizeof(dcplx);
  }());
  double eps = INFINITY;
  int it = 0;
  while (true) {
    if (it >= eig_miniter) {
      ProfTag ptag(ctx, "gauge_eig");
      double etol = eig_tol_from(eps);
      LinOp op = [&](const dcplx* v, dcplx* out) {
        DevBuf& a = ctx->buf("gauge_tm_a", (size_t)DN * DN * sizeof(dcplx));
        DevBuf& b = ctx->buf("gauge_tm_b", (size_t)DN * DN * sizeof(dcplx));
        const dcplx* cur = v;
        for (int l = 0; l < N; ++l) {
          dcplx* dst = (l == N - 1) ? out : ((l % 2 == 0) ? a.z() : b.z());
          push_left_id(ctx, st->Dl(l), st->d[l], st->Dr(l), cur, Aw[l], st->AL[l].z(), dst);
          cur = dst;
        }
      };
      DevBuf& ev = ctx->buf("gauge_evec", (size_t)DN * DN * sizeof(dcplx));
      {
        std::vector<const void*> cptrs;
        for (int l = 0; l < N; ++l) {
          cptrs.push_back(Aw[l]);
          cptrs.push_back(st->AL[l].ptr);
        }
        gauge_eigsolve(ctx, (int64_t)DN * DN, op, st->C[N - 1].z(), ev.z(), etol, cptrs);
      }
      qrpos(ctx, DN, DN, ev.z(), DN, nullptr, st->C[N - 1].z());  // the R factor only
    }
    zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), Cpre.z());
    for (int i = 0; i < N; ++i) {
      const int Dl = st->Dl(i), d = st->d[i], Dr = st->Dr(i);
      const dcplx* Cprev = st->C[(i - 1 + N) % N].z();
      zgemm(ctx, OP_N, OP_N, Dl, d * Dr, Dl, 1.0, Cprev, Dl, 0, Aw[i], Dl, 0, 0.0, M.z(), Dl, 0, 1, false);
      qr_factor(ctx, Dl * d, Dr, M.z(), (int64_t)Dl * d, st->C[i].z(), sweep_slot(i).c_str());
    }
    double nc = dznrm2(ctx, (int64_t)DN * DN, st->C[N - 1].z());
    zscal(ctx, (int64_t)DN * DN, 1.0 / nc, st->C[N - 1].z());
    eps = diff_norm(ctx, (int64_t)DN * DN, st->C[N - 1].z(), Cpre.z());
    ++it;
    if (sweep_q_needed(eps, tol, it, maxiter, eig_miniter)) {
      ProfTag ptag(ctx, "gauge_q");
      for (int i = 0; i < N; ++i) qr_form_q(ctx, st->Dl(i) * st->d[i], st->Dr(i), st->AL[i].z(), sweep_slot(i).c_str());
    }
    if (eps < tol || it > maxiter) {
      res.niter = it;
      res.err = eps;
      res.converged = eps < tol;
      return res;
    }
  }
}

GaugeResult uniform_rightorth(Context* ctx, imps_state* st, const std::vector<const dcplx*>& A, const dcplx* C0,
                              double tol, int maxiter, int eig_miniter) {
  Fp64Scope fp64(ctx);
  const int N = st->N;
  GaugeResult res;
  std::vector<dcplx*> Aw = work_copy(ctx, st, A, "gauge_awork");
  const int DN = st->Dr(N - 1);
  {
    DevBuf& t = ctx->buf("gauge_c0", (size_t)DN * DN * sizeof(dcplx));
    zcopy(ctx, (int64_t)DN * DN, C0, t.z());
    double nc = dznrm2(ctx, (int64_t)DN * DN, t.z());
    zaxpby(ctx, (int64_t)DN * DN, 1.0 / nc, t.z(), 0.0, st->C[N - 1].z());
  }
  DevBuf& Cpre = ctx->buf("gauge_cpre", (size_t)DN * DN * sizeof(dcplx));
  DevBuf& M = ctx->buf("gauge_m", [&] {
    size_t mx = 0;
    for (int l = 0; l < N; ++l) mx = std::max(mx, st->site_elems(l));
    return mx * sizeof(dcplx);
  }());
  double eps = INFINITY;
  int it = 0;
  while (true) {
    if (it >= eig_miniter) {
      ProfTag ptag(ctx, "gauge_eig");
      double etol = eig_tol_from(eps);
      LinOp op = [&](const dcplx* v, dcplx* out) {
        DevBuf& a = ctx->buf("gauge_tm_a", (size_t)DN * DN * sizeof(dcplx));
        DevBuf& b = ctx->buf("gauge_tm_b", (size_t)DN * DN * sizeof(dcplx));
        const dcplx* cur = v;
        for (int l = N - 1, k = 0; l >= 0; --l, ++k) {
          dcplx* dst = (l == 0) ? out : ((k % 2 == 0) ? a.z() : b.z());
          push_right_id(ctx, st->Dl(l), st->d[l], st->Dr(l), cur, Aw[l], st->AR[l].z(), dst);
          cur = dst;
        }
      };
      DevBuf& ev = ctx->buf("gauge_evec", (size_t)DN * DN * sizeof(dcplx));
      {
        std::vector<const void*> cptrs;
        for (int l = 0; l < N; ++l) {
          cptrs.push_back(Aw[l]);
          cptrs.push_back(st->AR[l].ptr);
        }
        gauge_eigsolve(ctx, (int64_t)DN * DN, op, st->C[N - 1].z(), ev.z(), etol, cptrs);
      }
      lqpos(ctx, DN, DN, ev.z(), DN, st->C[N - 1].z(), nullptr);  // the L factor only
    }
    zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), Cpre.z());
    for (int i = N - 1; i >= 0; --i) {
      const int Dl = st->Dl(i), d = st->d[i], Dr = st->Dr(i);
      zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, 1.0, Aw[i], (int64_t)Dl * d, 0, st->C[i].z(), Dr, 0, 0.0, M.z(),
            (int64_t)Dl * d, 0, 1, false);
      lq_factor(ctx, Dl, d * Dr, M.z(), Dl, st->C[(i - 1 + N) % N].z(), sweep_slot(i).c_str());
    }
    double nc = dznrm2(ctx, (int64_t)DN * DN, st->C[N - 1].z());
    zscal(ctx, (int64_t)DN * DN, 1.0 / nc, st->C[N - 1].z());
    eps = diff_norm(ctx, (int64_t)DN * DN, st->C[N - 1].z(), Cpre.z());
    ++it;
    if (sweep_q_needed(eps, tol, it, maxiter, eig_miniter)) {
      ProfTag ptag(ctx, "gauge_q");
      for (int i = 0; i < N; ++i) lq_form_q(ctx, st->Dl(i), st->d[i] * st->Dr(i), st->AR[i].z(), sweep_slot(i).c_str());
    }
    if (eps < tol || it > maxiter) {
      res.niter = it;
      res.err = eps;
      res.converged = eps < tol;
      return res;
    }
  }
}

void mul_AL_C(Context* ctx, imps_state* st) {
  for (int l = 0; l < st->N; ++l) {
    const int Dl = st->Dl(l), d = st->d[l], Dr = st->Dr(l);
    zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, 1.0, st->AL[l].z(), (int64_t)Dl * d, 0, st->C[l].z(), Dr, 0, 0.0,
          st->AC[l].z(), (int64_t)Dl * d, 0, 1, false);
  }
}

void check_full_rank(const imps_state* st) {
  for (int l = 0; l < st->N; ++l) {
    const int Dl = st->Dl(l), d = st->d[l], Dr = st->Dr(l);
    IMPS_REQUIRE(Dr <= Dl * d && Dl <= Dr * d, IMPS_DIM_MISMATCH,
                 "bond profile is not full rank (Dr <= Dl*d and Dl <= Dr*d required at every site)");
  }
}

GaugeResult canonicalize(Context* ctx, imps_state* st, const std::vector<const dcplx*>& As, double tol, int maxiter) {
  check_full_rank(st);
  const int N = st->N, DN = st->Dr(N - 1);
  DevBuf& I = ctx->buf("canon_id", (size_t)DN * DN * sizeof(dcplx));
  zset_identity(ctx, DN, I.z(), DN, 1.0);
  GaugeResult r1 = uniform_leftorth(ctx, st, As, I.z(), tol, maxiter, 10);
  std::vector<const dcplx*> al(N);
  for (int l = 0; l < N; ++l) al[l] = st->AL[l].z();
  DevBuf& c0 = ctx->buf("canon_c0", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, st->C[N - 1].z(), c0.z());
  GaugeResult r2 = uniform_rightorth(ctx, st, al, c0.z(), tol, maxiter, 10);
  mul_AL_C(ctx, st);
  GaugeResult r;
  r.niter = r1.niter + r2.niter;
  r.converged = r1.converged && r2.converged;
  r.err = std::max(r1.err, r2.err);
  return r;
}

GaugeResult from_al(Context* ctx, imps_state* st, const dcplx* C0, double tol, int maxiter) {
  // st->AL holds the (candidate) left-canonical tensors
  const int N = st->N, DN = st->Dr(N - 1);
  std::vector<const dcplx*> al(N);
  for (int l = 0; l < N; ++l) al[l] = st->AL[l].z();
  DevBuf& c0 = ctx->buf("canon_c0", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, C0, c0.z());
  GaugeResult r = uniform_rightorth(ctx, st, al, c0.z(), tol, maxiter, 10);
  mul_AL_C(ctx, st);
  return r;
}

void regauge(Context* ctx, int Dl, int d, int Dr, const dcplx* AC, const dcplx* C, dcplx* AL) {
  Fp64Scope fp64(ctx);
  DevBuf& Qac = ctx->buf("reg_qac", (size_t)Dl * d * Dr * sizeof(dcplx));
  DevBuf& Rac = ctx->buf("reg_rac", (size_t)Dr * Dr * sizeof(dcplx));
  DevBuf& Qc = ctx->buf("reg_qc", (size_t)Dr * Dr * sizeof(dcplx));
  DevBuf& Rc = ctx->buf("reg_rc", (size_t)Dr * Dr * sizeof(dcplx));
  qrpos(ctx, Dl * d, Dr, AC, (int64_t)Dl * d, Qac.z(), Rac.z());
  qrpos(ctx, Dr, Dr, C, Dr, Qc.z(), Rc.z());
  zgemm(ctx, OP_N, OP_C, Dl * d, Dr, Dr, 1.0, Qac.z(), (int64_t)Dl * d, 0, Qc.z(), Dr, 0, 0.0, AL, (int64_t)Dl * d,
        0, 1, false);
}

cplx state_dot(Context* ctx, imps_state* st) {
  Fp64Scope fp64(ctx);
  const int N = st->N, D0 = st->Dl(0);
  DevBuf& v0 = ctx->buf("dot_v0", (size_t)D0 * D0 * sizeof(dcplx));
  DevBuf& ev = ctx->buf("dot_ev", (size_t)D0 * D0 * sizeof(dcplx));
  zset_identity(ctx, D0, v0.z(), D0, 1.0);
  LinOp op = [&](const dcplx* v, dcplx* out) {
    DevBuf& a = ctx->buf("dot_tm_a", (size_t)D0 * D0 * sizeof(dcplx) * 4);
    DevBuf& b = ctx->buf("dot_tm_b", (size_t)D0 * D0 * sizeof(dcplx) * 4);
    const dcplx* cur = v;
    for (int l = 0; l < N; ++l) {
      dcplx* dst = (l == N - 1) ? out : ((l % 2 == 0) ? a.z() : b.z());
      push_left_id(ctx, st->Dl(l), st->d[l], st->Dr(l), cur, st->AL[l].z(), st->AL[l].z(), dst);
      cur = dst;
    }
  };
  KrylovResult r = arnoldi_dominant(ctx, (int64_t)D0 * D0, op, v0.z(), ev.z(), 1e-10, 30, 300, true);
  return r.value;
}

}  // namespace imps
