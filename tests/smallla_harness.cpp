// Host-only harness of the Krylov solvers' small eigenproblems (csrc/smallla.cu),
// compiled with the host C++ compiler by tests/test_smallla.py: no GPU involved.
#include "../infinitempsalgorithms_b200/csrc/smallla.cu"

extern "C" {
void h_herm_eig(int n, const double* A, double* w, double* V) {
  const imps::cplx* a0 = reinterpret_cast<const imps::cplx*>(A);
  std::vector<imps::cplx> a(a0, a0 + (size_t)n * n);
  std::vector<double> ww;
  std::vector<imps::cplx> vv;
  imps::herm_eig(n, a, ww, vv);
  for (int i = 0; i < n; ++i) w[i] = ww[i];
  for (size_t i = 0; i < vv.size(); ++i) reinterpret_cast<imps::cplx*>(V)[i] = vv[i];
}
void h_schur_sorted(int n, const double* H, double* T, double* Z) {
  const imps::cplx* h0 = reinterpret_cast<const imps::cplx*>(H);
  std::vector<imps::cplx> h(h0, h0 + (size_t)n * n);
  std::vector<imps::cplx> t, z;
  imps::schur_sorted(n, h, t, z);
  for (size_t i = 0; i < t.size(); ++i) reinterpret_cast<imps::cplx*>(T)[i] = t[i];
  for (size_t i = 0; i < z.size(); ++i) reinterpret_cast<imps::cplx*>(Z)[i] = z[i];
}
void h_gen_eig(int n, const double* H, double* lam, double* Y) {
  const imps::cplx* h0 = reinterpret_cast<const imps::cplx*>(H);
  std::vector<imps::cplx> h(h0, h0 + (size_t)n * n);
  std::vector<imps::cplx> l, y;
  imps::gen_eig(n, h, l, y);
  for (int i = 0; i < n; ++i) reinterpret_cast<imps::cplx*>(lam)[i] = l[i];
  for (size_t i = 0; i < y.size(); ++i) reinterpret_cast<imps::cplx*>(Y)[i] = y[i];
}
}
