// MPO application by VOMPS on the device (see mult.cu).
#pragma once
#include "gauge.h"
#include "imps_internal.h"
#include "krylov.h"

// Environments of the <bra|W|ket> channel (MultCache): lefts[l] (bra bond, w, ket bond)
// left of site l, rights[l] (ket bond, w, bra bond) right of site l.  W, bra and ket are
// borrowed and must outlive the object; sweeps update the bra in place.
struct imps_mult_envs {
  imps::Context* ctx;
  int device = 0;
  int N = 0;
  const imps_mpo* W = nullptr;
  imps_state* bra = nullptr;
  const imps_state* ket = nullptr;
  std::vector<imps::DevBuf> lefts, rights;
};

namespace imps {
void push_ternary_left(Context* ctx, const MpoSite& W, int Db, int Dbr, int Da, int Dar, const dcplx* L,
                       const dcplx* below, const dcplx* above, dcplx* out);
void push_ternary_right(Context* ctx, const MpoSite& W, int Dal, int Da, int Dbl, int Db, const dcplx* R,
                        const dcplx* above, const dcplx* below, dcplx* out);
void mult_ac(Context* ctx, const MpoSite& W, int Db, int Da, int Dar, int Dbr, const dcplx* GL, const dcplx* GR,
             const dcplx* x, dcplx* y);
void mult_c(Context* ctx, int w, int Db, int Da, int Dbr, const dcplx* GL, const dcplx* GR, const dcplx* C,
            dcplx* y);
void mult_envs_allocate(imps_mult_envs* E);
KrylovResult mult_fixedpoints(Context* ctx, imps_mult_envs* E, double tol, int maxiter, bool warm);
double mult_galerkin(Context* ctx, imps_mult_envs* E);
double mult_sweep(Context* ctx, imps_mult_envs* E, double gauge_tol, int gauge_maxiter, double env_tol,
                  int env_maxiter);
imps_state* mult_guess(Context* ctx, const imps_mpo* W, const imps_state* ket, int D, double tol, int maxiter,
                       GaugeResult* gres);
}  // namespace imps
