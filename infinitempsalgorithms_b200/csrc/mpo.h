// Schur MPO site construction (see mpo.cu).
#pragma once
#include "imps_internal.h"

namespace imps {
void make_mpo_site(Context* ctx, MpoSite& S, int m, int d, int n, const cplx* W);
// the closing column W[:, :, n-1, :] as an (m, d, 1, d) tensor (Schur energy, expval.jl:104-108)
void make_closing_column(Context* ctx, const MpoSite& W, MpoSite& out);
}  // namespace imps
