// Device-resident Krylov solvers (KrylovKit's eigsolve / linsolve / exponentiate /
// schursolve as called by the reference, restated; see krylov.cu).
#pragma once
#include <functional>

#include "imps_internal.h"

namespace imps {

struct KrylovResult {
  int converged = 0;
  int numiter = 0;
  int numops = 0;
  double normres = 0.0;
  cplx value = 0.0;
};

// y = A x on device vectors of length n
using LinOp = std::function<void(const dcplx* x, dcplx* y)>;

// Smallest-real eigenpair of a Hermitian map (thick-restart Lanczos, CGS2).
// x may alias x0.  Returned vector: unit norm, <x0, x> real non-negative.
KrylovResult lanczos_eigsolve(Context* ctx, int64_t n, const LinOp& A, const dcplx* x0, dcplx* x, double tol,
                              int krylovdim, int maxiter, bool eager);
// (a0 + a1 A) x = b, restarted GMRES; x holds x0 on entry and the solution on exit.
KrylovResult gmres(Context* ctx, int64_t n, const LinOp& A, const dcplx* b, dcplx* x, double tol, int krylovdim,
                   int maxiter, cplx a0, cplx a1);
// x = exp(t A) x0 for Hermitian A (Lanczos with sub-stepping). x may alias x0.
KrylovResult exponentiate(Context* ctx, int64_t n, const LinOp& A, cplx t, const dcplx* x0, dcplx* x, double tol,
                          int krylovdim, int maxiter);
// Dominant (largest |lambda|) eigenpair of a general map (Arnoldi, Ritz restart).
KrylovResult arnoldi_dominant(Context* ctx, int64_t n, const LinOp& A, const dcplx* x0, dcplx* x, double tol,
                              int krylovdim, int maxiter, bool eager);

}  // namespace imps
