// Observables and algorithm steps (see algos.cu).
#pragma once
#include "imps_internal.h"
#include "krylov.h"

namespace imps {
double galerkin(Context* ctx, imps_envs* E, const imps_mpo* H, const imps_state* st);
cplx energy(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st);
cplx local_expval(Context* ctx, imps_state* st, int site, const cplx* O);
// energy gradients (grad.cu): dE/dW[site] into G_host (m, d, n, d); dE/dconj(AL[site]) into g (device)
void energy_grad_mpo(Context* ctx, const imps_envs* E, const imps_mpo* H, const imps_state* st, int site,
                     cplx* G_host);
void energy_grad_al(Context* ctx, const imps_envs* E, const imps_mpo* H, const imps_state* st, int site, dcplx* g);
KrylovResult eigsolve_ac(Context* ctx, imps_envs* E, const imps_mpo* H, int site, const dcplx* x0, dcplx* x,
                         double tol, int kdim, int maxiter, bool eager);
KrylovResult eigsolve_c(Context* ctx, imps_envs* E, int site, const dcplx* x0, dcplx* x, double tol, int kdim,
                        int maxiter, bool eager);
KrylovResult expo_ac(Context* ctx, imps_envs* E, const imps_mpo* H, int site, cplx dt, const dcplx* x0, dcplx* x,
                     double tol, int kdim, int maxiter);
KrylovResult expo_c(Context* ctx, imps_envs* E, int site, cplx dt, const dcplx* x0, dcplx* x, double tol, int kdim,
                    int maxiter);
void vumps_localupdate(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, double tol, int kdim, int maxiter,
                       bool eager, int* nac, int* nc);
imps_vumps_info vumps_iter(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, int iter, double eps);
KrylovResult tdvp_step(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, cplx dt, double tol, int kdim,
                       int maxiter, double gauge_tol, int gauge_maxiter);
void idmrg_sweep(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, double tol, int kdim, int maxiter,
                 bool eager, double* Eout, double* epsout);
// two-site IDMRG (idmrg2.cu): y = AC2 Hamiltonian of window (p, p+1) applied to x (Dl, d1, d2, Dr)
void ac2_apply(Context* ctx, const imps_envs* E, const imps_mpo* H, int p, const dcplx* x, dcplx* y);
// one _localupdate_sweep_idmrg2! with truncdim(D); bond dimensions of st and E change in place
void idmrg2_sweep(Context* ctx, imps_envs* E, const imps_mpo* H, imps_state* st, int D, double tol, int kdim,
                  int maxiter, bool eager, double* Eout, double* epsout);
}  // namespace imps
