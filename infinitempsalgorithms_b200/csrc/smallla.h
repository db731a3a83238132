// Small dense FP64 eigenproblems used by the Krylov solvers (see smallla.cu).
#pragma once
#include <complex>
#include <vector>

namespace imps {
using cplx = std::complex<double>;
// Hermitian n x n (column-major) -> ascending eigenvalues w, eigenvectors V (columns).
void herm_eig(int n, const std::vector<cplx>& A, std::vector<double>& w, std::vector<cplx>& V);
// Complex Schur form H = Z T Z^H (T upper triangular, Z unitary), column-major.
void complex_schur(int n, const std::vector<cplx>& H, std::vector<cplx>& T, std::vector<cplx>& Z);
// Same with the diagonal of T ordered by non-increasing modulus.
void schur_sorted(int n, const std::vector<cplx>& H, std::vector<cplx>& T, std::vector<cplx>& Z);
// General n x n (column-major) -> eigenvalues lam, unit eigenvectors Y (columns).
void gen_eig(int n, const std::vector<cplx>& H, std::vector<cplx>& lam, std::vector<cplx>& Y);
// exp(t Hs) e1 for a Hermitian m x m matrix.
void herm_expm_e1(int m, const std::vector<cplx>& Hs, cplx t, std::vector<cplx>& out);
}  // namespace imps
