// Gauge fixing and state constructors on the device (see gauge.cu).
#pragma once
#include "imps_internal.h"

namespace imps {

struct GaugeResult {
  int niter = 0;
  int converged = 0;
  double err = 0.0;
};

// uniform_leftorth! writing st->AL and st->C from site tensors A and C0.
GaugeResult uniform_leftorth(Context* ctx, imps_state* st, const std::vector<const dcplx*>& A, const dcplx* C0,
                             double tol, int maxiter, int eig_miniter);
// uniform_rightorth! writing st->AR and st->C.
GaugeResult uniform_rightorth(Context* ctx, imps_state* st, const std::vector<const dcplx*>& A, const dcplx* C0,
                              double tol, int maxiter, int eig_miniter);
// AC[l] = AL[l] C[l]
void mul_AL_C(Context* ctx, imps_state* st);
// CanonicalIMPS(As)
GaugeResult canonicalize(Context* ctx, imps_state* st, const std::vector<const dcplx*>& As, double tol, int maxiter);
// CanonicalIMPS(st->AL, C0) / gauge_step!: right gauge fix keeping st->AL, then AC = AL C.
GaugeResult from_al(Context* ctx, imps_state* st, const dcplx* C0, double tol, int maxiter);
// regauge!(AC, C) -> AL
void regauge(Context* ctx, int Dl, int d, int Dr, const dcplx* AC, const dcplx* C, dcplx* AL);
// dot(psi, psi)
cplx state_dot(Context* ctx, imps_state* st);

}  // namespace imps
