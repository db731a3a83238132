// Dense-MPO channel environments, correlators and entanglement spectra (observables.cu).
#pragma once
#include <vector>

#include "imps_internal.h"
#include "krylov.h"

namespace imps {

// Squared singular values (descending) of the m x n matrix A, by one-sided Jacobi.
std::vector<double> singular_values_sq(Context* ctx, int m, int n, const dcplx* A, int64_t lda);
// Thin SVD A = U diag(s) V^H by one-sided Jacobi (descending s), truncated to at most
// kmax (> 0) values and to those above `cutoff` (at least one kept); U (m x k), V (n x k)
// column-major with leading dimensions m and n.  Returns k.
int svd_thin(Context* ctx, int m, int n, const dcplx* A, int64_t lda, int kmax, double cutoff, dcplx* U,
             std::vector<double>& s, dcplx* V);
// entanglement_spectrum(psi, loc): normalised squared Schmidt values of bond `bond` (0-based).
std::vector<double> entanglement_spectrum(Context* ctx, imps_state* st, int bond);
// dominant_env([W,] psi; side) into out (D x w x D, unit norm); mpo == nullptr: identity channel.
// side 0 = left (AL pushes), 1 = right (AR pushes).
KrylovResult dominant_env(Context* ctx, imps_state* st, const imps_mpo* mpo, int side, double tol, int krylovdim,
                          int maxiter, dcplx* out);
// DMRGCache(psi, ::DenseIMPO) with normalize_envs!, into envs.
KrylovResult envs_build_dense(Context* ctx, imps_envs* envs, imps_state* st, const imps_mpo* mpo, double tol,
                              int krylovdim, int maxiter);
// expectationvalue(psi, ::DenseIMPO, envs).
cplx energy_dense(Context* ctx, imps_envs* envs, const imps_mpo* mpo, imps_state* st);
// out[a, u, b] = sum_s O[u, s] A[a, s, b] (O on the device, d x d column-major).
void apply_local(Context* ctx, int Dl, int d, int Dr, const dcplx* O_dev, const dcplx* A, dcplx* out);
// correlator(psi, O1, O2, i, js) (1-based sites, host operators d x d).
std::vector<cplx> correlator(Context* ctx, imps_state* st, const cplx* O1, const cplx* O2, int i,
                             const std::vector<int>& js);

}  // namespace imps
