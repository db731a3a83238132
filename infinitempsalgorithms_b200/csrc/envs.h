// Schur-MPO environments on the device (see envs.cu).
#pragma once
#include "imps_internal.h"

namespace imps {
void envs_allocate(imps_envs* E, const imps_state* st, const imps_mpo* H);
imps_env_info envs_build(Context* ctx, imps_envs* E, const imps_state* st, const imps_mpo* H, double tol, int maxiter,
                         int krylovdim, bool warm);
}  // namespace imps
