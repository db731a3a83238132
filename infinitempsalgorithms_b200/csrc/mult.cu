// MPO application y ~ W psi by VOMPS on the device:
//   ternary pushes          src/transfermatrix.jl:77-107
//   MultCache fixed points  src/algorithms/arithmetics/mult.jl:93-158 (mixed_fixedpoints)
//   local maps              mult.jl:226-230 (_mapAC), :705-716 (_mapC with operator.C = I)
//   Galerkin residual       mult.jl:586-593, :278-284
//   VOMPS iteration         src/algorithms/arithmetics/envs.jl:51-93 (compression_sweeps!)
//   initial guess           mult.jl:848-870 (svdguess_mult), compress.jl:161-190 (_lazy_svd_guess)
// W is any MPO held as an imps_mpo (the dense DenseIMPO channel: AL = AR = AC = W, C = I).
// Every product of the channel is the one-site pattern GEMM -> level mix -> GEMM with a
// bra (below) and a ket (above) of different bond dimensions.  FP64 throughout.
#include "gauge.h"
#include "krylov.h"
#include "mult.h"
#include "observables.h"

#include <cmath>

namespace imps {
namespace {

void launched(Context* ctx, const char* what) {
  ctx->n_kernels++;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) throw Error(IMPS_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kEnvKrylovDim = 30;   // Defaults.krylovdim

int grid_for(int64_t t) { return (int)std::max<int64_t>(1, std::min<int64_t>((t + 255) / 256, 148 * 8)); }

// v[k] = exp(2 pi i frac(k phi)), phi the golden-ratio conjugate: the deterministic start of
// the environment eigensolves (the reference draws randn)
__global__ void k_env_start(int64_t n, dcplx* v) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double f = fmod((double)k * 0.6180339887498949, 1.0);
    double s, c;
    sincospi(2.0 * f, &s, &c);
    v[k] = make_double2(c, s);
  }
}

// B[(wl + Wl bl), u, (wr + Wr br)] = sum_d W[wl,u,wr,d] A[bl,d,br]   (operators/linalg.jl:15-20)
__global__ void k_mult_site(int wl, int d, int wr, int bl, int br, const dcplx* __restrict__ W,
                            const dcplx* __restrict__ A, dcplx* __restrict__ B) {
  const int64_t rows = (int64_t)wl * bl, cols = (int64_t)wr * br, tot = rows * d * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t % rows, rest = t / rows;
    const int u = (int)(rest % d);
    const int64_t c = rest / d;
    const int iwl = (int)(r % wl), ibl = (int)(r / wl), iwr = (int)(c % wr), ibr = (int)(c / wr);
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < d; ++s) {
      const dcplx w = W[iwl + (int64_t)wl * (u + (int64_t)d * (iwr + (int64_t)wr * s))];
      const dcplx a = A[ibl + (int64_t)bl * (s + (int64_t)d * ibr)];
      sr += w.x * a.x - w.y * a.y;
      si += w.x * a.y + w.y * a.x;
    }
    B[t] = make_double2(sr, si);
  }
}

// B[(wl + Wl bl), u, f] = sum_{wr, s} W[wl,u,wr,s] Tb[bl,s,wr,f]
__global__ void k_mult_carry(int wl, int d, int wr, int bl, int f, const dcplx* __restrict__ W,
                             const dcplx* __restrict__ Tb, dcplx* __restrict__ B) {
  const int64_t rows = (int64_t)wl * bl, tot = rows * d * f;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t % rows, rest = t / rows;
    const int u = (int)(rest % d), jf = (int)(rest / d);
    const int iwl = (int)(r % wl), ibl = (int)(r / wl);
    double sr = 0.0, si = 0.0;
    for (int iwr = 0; iwr < wr; ++iwr)
      for (int s = 0; s < d; ++s) {
        const dcplx w = W[iwl + (int64_t)wl * (u + (int64_t)d * (iwr + (int64_t)wr * s))];
        const dcplx x = Tb[ibl + (int64_t)bl * (s + (int64_t)d * (iwr + (int64_t)wr * jf))];
        sr += w.x * x.x - w.y * x.y;
        si += w.x * x.y + w.y * x.x;
      }
    B[t] = make_double2(sr, si);
  }
}

// Y[br, wr, f] = X[wr, br, f] (swap of the two leading dims)
__global__ void k_swap01(int a, int b, int64_t c, const dcplx* __restrict__ X, dcplx* __restrict__ Y) {
  const int64_t tot = (int64_t)a * b * c;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % a);
    const int64_t rest = t / a;
    const int j = (int)(rest % b);
    const int64_t k = rest / b;
    Y[j + (int64_t)b * (i + (int64_t)a * k)] = X[t];
  }
}

// X[r, c] *= s[c] (real), rows x cols column-major
__global__ void k_scale_cols_real(int rows, int cols, dcplx* X, const double* __restrict__ s) {
  const int64_t tot = (int64_t)rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const double a = s[t / rows];
    X[t].x *= a;
    X[t].y *= a;
  }
}

void scale_cols(Context* ctx, int rows, int cols, dcplx* X, const std::vector<double>& s) {
  DevBuf& sd = ctx->buf("mult_scale", s.size() * sizeof(double));
  upload(ctx, sd.ptr, s.data(), s.size() * sizeof(double));
  k_scale_cols_real<<<grid_for((int64_t)rows * cols), 256, 0, ctx->stream>>>(rows, cols, X, sd.d());
  launched(ctx, "mult scale");
}

}  // namespace

// ---------------------------------------------------------------------------
// Channel products
// ---------------------------------------------------------------------------
void push_ternary_left(Context* ctx, const MpoSite& W, int Db, int Dbr, int Da, int Dar, const dcplx* L,
                       const dcplx* below, const dcplx* above, dcplx* out) {
  ctx->n_push++;
  const int w = W.m, wr = W.n, d = W.d;
  DevBuf& Y = ctx->buf("mult_t1", (size_t)Db * w * d * Dar * sizeof(dcplx));
  DevBuf& Z = ctx->buf("mult_t2", (size_t)Db * d * wr * Dar * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Db * w, d * Dar, Da, 1.0, L, (int64_t)Db * w, 0, above, Da, 0, 0.0, Y.z(),
        (int64_t)Db * w, 0, 1);
  MixPlan pl;
  pl.Db = Db; pl.R = w; pl.P = d; pl.Q = wr; pl.S = d; pl.C = Dar;
  pl.in_r = Db; pl.in_s = (int64_t)Db * w; pl.in_c = (int64_t)Db * w * d;
  pl.out_p = Db; pl.out_q = (int64_t)Db * d; pl.out_c = (int64_t)Db * d * wr;
  pl.M = W.Wdev.z();
  pl.nz = W.nz;
  {
    std::vector<bool> hit(wr, false);
    for (auto& b : W.nz) hit[b.second] = true;
    bool any = false;
    for (int q = 0; q < wr; ++q) any |= !hit[q];
    if (any) zfill(ctx, (int64_t)Db * d * wr * Dar, 0.0, Z.z());
  }
  level_mix(ctx, pl, Y.z(), Z.z());
  zgemm(ctx, OP_C, OP_N, Dbr, wr * Dar, Db * d, 1.0, below, (int64_t)Db * d, 0, Z.z(), (int64_t)Db * d, 0, 0.0, out,
        Dbr, 0, 1);
}

void push_ternary_right(Context* ctx, const MpoSite& W, int Dal, int Da, int Dbl, int Db, const dcplx* R,
                        const dcplx* above, const dcplx* below, dcplx* out) {
  ctx->n_push++;
  const int wl = W.m, w = W.n, d = W.d;
  DevBuf& Y = ctx->buf("mult_t1", (size_t)Dal * d * w * Db * sizeof(dcplx));
  DevBuf& Z = ctx->buf("mult_t2", (size_t)Dal * wl * d * Db * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Dal * d, w * Db, Da, 1.0, above, (int64_t)Dal * d, 0, R, Da, 0, 0.0, Y.z(),
        (int64_t)Dal * d, 0, 1);
  MixPlan pl;
  pl.Db = Dal; pl.R = w; pl.P = d; pl.Q = wl; pl.S = d; pl.C = Db;
  pl.in_r = (int64_t)Dal * d; pl.in_s = Dal; pl.in_c = (int64_t)Dal * d * w;
  pl.out_p = (int64_t)Dal * wl; pl.out_q = Dal; pl.out_c = (int64_t)Dal * wl * d;
  pl.M = W.Wdev.z() + (int64_t)W.m * W.d * W.n * W.d;
  for (auto& b : W.nz) pl.nz.push_back({b.second, b.first});
  {
    std::vector<bool> hit(wl, false);
    for (auto& b : W.nz) hit[b.first] = true;
    bool any = false;
    for (int q = 0; q < wl; ++q) any |= !hit[q];
    if (any) zfill(ctx, (int64_t)Dal * wl * d * Db, 0.0, Z.z());
  }
  level_mix(ctx, pl, Y.z(), Z.z());
  zgemm(ctx, OP_N, OP_C, Dal * wl, Dbl, d * Db, 1.0, Z.z(), (int64_t)Dal * wl, 0, below, Dbl, 0, 0.0, out,
        (int64_t)Dal * wl, 0, 1);
}

void mult_ac(Context* ctx, const MpoSite& W, int Db, int Da, int Dar, int Dbr, const dcplx* GL, const dcplx* GR,
             const dcplx* x, dcplx* y) {
  const int w = W.m, wr = W.n, d = W.d;
  DevBuf& T1 = ctx->buf("mult_t1", (size_t)Db * w * d * Dar * sizeof(dcplx));
  DevBuf& T2 = ctx->buf("mult_t2", (size_t)Db * d * Dar * wr * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Db * w, d * Dar, Da, 1.0, GL, (int64_t)Db * w, 0, x, Da, 0, 0.0, T1.z(), (int64_t)Db * w,
        0, 1);
  MixPlan pl;
  pl.Db = Db; pl.R = w; pl.P = d; pl.Q = wr; pl.S = d; pl.C = Dar;
  pl.in_r = Db; pl.in_s = (int64_t)Db * w; pl.in_c = (int64_t)Db * w * d;
  pl.out_p = Db; pl.out_q = (int64_t)Db * d * Dar; pl.out_c = (int64_t)Db * d;
  pl.M = W.Wdev.z();
  pl.nz = W.nz;
  {
    std::vector<bool> hit(wr, false);
    for (auto& b : W.nz) hit[b.second] = true;
    for (int q = 0; q < wr; ++q)
      if (!hit[q]) zfill(ctx, (int64_t)Db * d * Dar, 0.0, T2.z() + (int64_t)Db * d * Dar * q);
  }
  level_mix(ctx, pl, T1.z(), T2.z());
  zgemm(ctx, OP_N, OP_N, Db * d, Dbr, Dar * wr, 1.0, T2.z(), (int64_t)Db * d, 0, GR, (int64_t)Dar * wr, 0, 0.0, y,
        (int64_t)Db * d, 0, 1);
}

void mult_c(Context* ctx, int w, int Db, int Da, int Dbr, const dcplx* GL, const dcplx* GR, const dcplx* C,
            dcplx* y) {
  // GL (Db, w, Da), C (Da, Da), GR (Da, w, Dbr): y = GLp (Db x Da w) U (Da w x Dbr), U = C GR
  DevBuf& U = ctx->buf("mult_t1", (size_t)Da * w * Dbr * sizeof(dcplx));
  DevBuf& Gp = ctx->buf("mult_t2", (size_t)Db * Da * w * sizeof(dcplx));
  zgemm(ctx, OP_N, OP_N, Da, w * Dbr, Da, 1.0, C, Da, 0, GR, Da, 0, 0.0, U.z(), Da, 0, 1);
  DevBuf& Id = ctx->buf("mult_id", (size_t)w * w * sizeof(dcplx));
  std::vector<cplx> idh((size_t)w * w, cplx(0.0, 0.0));
  for (int i = 0; i < w; ++i) idh[i + (size_t)w * i] = 1.0;
  upload(ctx, Id.ptr, idh.data(), idh.size() * sizeof(dcplx));
  MixPlan pl;  // Gp[b + Db (c + Da q)] = GL[b, q, c]
  pl.Db = Db; pl.R = w; pl.P = 1; pl.Q = w; pl.S = 1; pl.C = Da;
  pl.in_r = Db; pl.in_s = 0; pl.in_c = (int64_t)Db * w;
  pl.out_p = 0; pl.out_q = (int64_t)Db * Da; pl.out_c = Db;
  pl.M = Id.z();
  for (int i = 0; i < w; ++i) pl.nz.push_back({i, i});
  level_mix(ctx, pl, GL, Gp.z());
  zgemm(ctx, OP_N, OP_N, Db, Dbr, Da * w, 1.0, Gp.z(), Db, 0, U.z(), (int64_t)Da * w, 0, 0.0, y, Db, 0, 1);
}

// ---------------------------------------------------------------------------
// Environments
// ---------------------------------------------------------------------------
namespace {
const MpoSite& wsite(const imps_mult_envs* E, int l) { return E->W->sites[((l % E->N) + E->N) % E->N % E->W->N]; }
}  // namespace

void mult_envs_allocate(imps_mult_envs* E) {
  const int N = E->N;
  E->lefts.resize(N);
  E->rights.resize(N);
  for (int l = 0; l < N; ++l) {
    const MpoSite& W = wsite(E, l);
    E->lefts[l].ensure((size_t)E->bra->Dl(l) * W.m * E->ket->Dl(l) * sizeof(dcplx));
    E->rights[l].ensure((size_t)E->ket->Dr(l) * W.n * E->bra->Dr(l) * sizeof(dcplx));
  }
}

KrylovResult mult_fixedpoints(Context* ctx, imps_mult_envs* E, double tol, int maxiter, bool warm) {
  Fp64Scope fp64(ctx);
  const int N = E->N;
  const imps_state* bra = E->bra;
  const imps_state* ket = E->ket;
  const int Dl = bra->Dl(0), Da = ket->Dl(0), Dw = wsite(E, 0).m;
  KrylovResult agg;
  {
    const int64_t n = (int64_t)Dl * Dw * Da;
    DevBuf& v0 = ctx->buf("mult_v0", n * sizeof(dcplx));
    if (warm) zcopy(ctx, n, E->lefts[0].z(), v0.z());
    else {
      k_env_start<<<grid_for(n), 256, 0, ctx->stream>>>(n, v0.z());
      launched(ctx, "mult env start");
    }
    size_t mx = 0;
    for (int l = 0; l < N; ++l) mx = std::max(mx, (size_t)bra->Dr(l) * wsite(E, l).n * ket->Dr(l));
    LinOp op = [&](const dcplx* v, dcplx* out) {
      DevBuf& a = ctx->buf("mult_tm_a", mx * sizeof(dcplx));
      DevBuf& b = ctx->buf("mult_tm_b", mx * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = 0; l < N; ++l) {
        dcplx* dst = (l == N - 1) ? out : ((l % 2 == 0) ? a.z() : b.z());
        push_ternary_left(ctx, wsite(E, l), bra->Dl(l), bra->Dr(l), ket->Dl(l), ket->Dr(l), cur, bra->AL[l].z(),
                          ket->AL[l].z(), dst);
        cur = dst;
      }
    };
    KrylovResult r = arnoldi_dominant(ctx, n, op, v0.z(), E->lefts[0].z(), tol, kEnvKrylovDim, maxiter, true);
    agg.numops += r.numops;
    agg.numiter += r.numiter;
    agg.converged = r.converged;
    agg.normres = r.normres;
    for (int l = 1; l < N; ++l)
      push_ternary_left(ctx, wsite(E, l - 1), bra->Dl(l - 1), bra->Dr(l - 1), ket->Dl(l - 1), ket->Dr(l - 1),
                        E->lefts[l - 1].z(), bra->AL[l - 1].z(), ket->AL[l - 1].z(), E->lefts[l].z());
  }
  {
    const int Dar = ket->Dr(N - 1), Dbr = bra->Dr(N - 1), Dwr = wsite(E, N - 1).n;
    const int64_t n = (int64_t)Dar * Dwr * Dbr;
    DevBuf& v0 = ctx->buf("mult_v0", n * sizeof(dcplx));
    if (warm) zcopy(ctx, n, E->rights[N - 1].z(), v0.z());
    else {
      k_env_start<<<grid_for(n), 256, 0, ctx->stream>>>(n, v0.z());
      launched(ctx, "mult env start");
    }
    size_t mx = 0;
    for (int l = 0; l < N; ++l) mx = std::max(mx, (size_t)ket->Dl(l) * wsite(E, l).m * bra->Dl(l));
    LinOp op = [&](const dcplx* v, dcplx* out) {
      DevBuf& a = ctx->buf("mult_tm_a", mx * sizeof(dcplx));
      DevBuf& b = ctx->buf("mult_tm_b", mx * sizeof(dcplx));
      const dcplx* cur = v;
      for (int l = N - 1, k = 0; l >= 0; --l, ++k) {
        dcplx* dst = (l == 0) ? out : ((k % 2 == 0) ? a.z() : b.z());
        push_ternary_right(ctx, wsite(E, l), ket->Dl(l), ket->Dr(l), bra->Dl(l), bra->Dr(l), cur, ket->AR[l].z(),
                           bra->AR[l].z(), dst);
        cur = dst;
      }
    };
    KrylovResult r = arnoldi_dominant(ctx, n, op, v0.z(), E->rights[N - 1].z(), tol, kEnvKrylovDim, maxiter,
                                      true);
    agg.numops += r.numops;
    agg.numiter += r.numiter;
    agg.converged = agg.converged && r.converged;
    agg.normres = std::max(agg.normres, r.normres);
    for (int l = N - 2; l >= 0; --l)
      push_ternary_right(ctx, wsite(E, l + 1), ket->Dl(l + 1), ket->Dr(l + 1), bra->Dl(l + 1), bra->Dr(l + 1),
                         E->rights[l + 1].z(), ket->AR[l + 1].z(), bra->AR[l + 1].z(), E->rights[l].z());
  }
  // normalisation: each GR to unit Frobenius norm, then GL[l+1] /= <below.C[l], mapC(GL[l+1], GR[l], above.C[l])>
  for (int l = 0; l < N; ++l) {
    const int64_t n = (int64_t)ket->Dr(l) * wsite(E, l).n * bra->Dr(l);
    const double nr = dznrm2(ctx, n, E->rights[l].z());
    IMPS_REQUIRE(nr > 0.0 && std::isfinite(nr), IMPS_INVALID_ARG, "ternary environment: zero or non-finite fixed point");
    zscal(ctx, n, 1.0 / nr, E->rights[l].z());
  }
  for (int l = 0; l < N; ++l) {
    const int nx = (l + 1) % N;
    const int Db = bra->Dr(l), Dk = ket->Dr(l), w = wsite(E, l).n;
    DevBuf& Cn = ctx->buf("mult_cnew", (size_t)Db * Db * sizeof(dcplx));
    mult_c(ctx, w, Db, Dk, Db, E->lefts[nx].z(), E->rights[l].z(), ket->C[l].z(), Cn.z());
    const cplx lam = zdotc(ctx, (int64_t)Db * Db, bra->C[l].z(), Cn.z());
    IMPS_REQUIRE(lam != cplx(0.0, 0.0), IMPS_INVALID_ARG, "ternary environment: local overlap lambda = 0");
    zscal(ctx, (int64_t)Db * w * Dk, 1.0 / lam, E->lefts[nx].z());
  }
  return agg;
}

namespace {
// ACnew of site l and CNew of bond l into the given buffers
void local_maps(Context* ctx, imps_mult_envs* E, int l, dcplx* ac, dcplx* c) {
  const imps_state* bra = E->bra;
  const imps_state* ket = E->ket;
  const int N = E->N;
  if (ac)
    mult_ac(ctx, wsite(E, l), bra->Dl(l), ket->Dl(l), ket->Dr(l), bra->Dr(l), E->lefts[l].z(), E->rights[l].z(),
            ket->AC[l].z(), ac);
  if (c)
    mult_c(ctx, wsite(E, l).n, bra->Dr(l), ket->Dr(l), bra->Dr(l), E->lefts[(l + 1) % N].z(), E->rights[l].z(),
           ket->C[l].z(), c);
}
}  // namespace

double mult_galerkin(Context* ctx, imps_mult_envs* E) {
  Fp64Scope fp64(ctx);
  const imps_state* bra = E->bra;
  double eps = 0.0;
  for (int l = 0; l < E->N; ++l) {
    const int Dl = bra->Dl(l), d = bra->d[l], Dr = bra->Dr(l);
    const int64_t n = (int64_t)Dl * d * Dr;
    DevBuf& ac = ctx->buf("mult_gal_ac", n * sizeof(dcplx));
    DevBuf& q = ctx->buf("mult_gal_q", (size_t)Dr * Dr * sizeof(dcplx));
    local_maps(ctx, E, l, ac.z(), nullptr);
    const double nr = dznrm2(ctx, n, ac.z());
    IMPS_REQUIRE(nr > 0.0 && std::isfinite(nr), IMPS_INVALID_ARG, "mult: zero or non-finite local map");
    zscal(ctx, n, 1.0 / nr, ac.z());
    zgemm(ctx, OP_C, OP_N, Dr, Dr, Dl * d, 1.0, bra->AL[l].z(), (int64_t)Dl * d, 0, ac.z(), (int64_t)Dl * d, 0, 0.0,
          q.z(), Dr, 0, 1);
    zgemm(ctx, OP_N, OP_N, Dl * d, Dr, Dr, -1.0, bra->AL[l].z(), (int64_t)Dl * d, 0, q.z(), Dr, 0, 1.0, ac.z(),
          (int64_t)Dl * d, 0, 1);
    eps = std::max(eps, dznrm2(ctx, n, ac.z()));
  }
  return eps;
}

double mult_sweep(Context* ctx, imps_mult_envs* E, double gauge_tol, int gauge_maxiter, double env_tol,
                  int env_maxiter) {
  Fp64Scope fp64(ctx);
  imps_state* bra = E->bra;
  const int N = E->N;
  // localupdate: AC / C maps with the current environments for every site, then regauge
  size_t tot_ac = 0, tot_c = 0;
  for (int l = 0; l < N; ++l) {
    tot_ac += bra->site_elems(l);
    tot_c += bra->bond_elems(l);
  }
  DevBuf& acs = ctx->buf("mult_acs", tot_ac * sizeof(dcplx));
  DevBuf& cs = ctx->buf("mult_cs", tot_c * sizeof(dcplx));
  std::vector<dcplx*> pac(N), pc(N);
  size_t oa = 0, oc = 0;
  for (int l = 0; l < N; ++l) {
    pac[l] = acs.z() + oa;
    pc[l] = cs.z() + oc;
    oa += bra->site_elems(l);
    oc += bra->bond_elems(l);
    local_maps(ctx, E, l, pac[l], pc[l]);
  }
  for (int l = 0; l < N; ++l) regauge(ctx, bra->Dl(l), bra->d[l], bra->Dr(l), pac[l], pc[l], bra->AL[l].z());
  // gauge_step!: right gauge fix keeping the candidate ALs, from the current C[N-1]
  const int DN = bra->Dr(N - 1);
  DevBuf& c0 = ctx->buf("mult_c0", (size_t)DN * DN * sizeof(dcplx));
  zcopy(ctx, (int64_t)DN * DN, bra->C[N - 1].z(), c0.z());
  from_al(ctx, bra, c0.z(), gauge_tol, gauge_maxiter);
  // recalculate!: fixed points warm-started from the current ones
  mult_fixedpoints(ctx, E, env_tol, env_maxiter, true);
  return mult_galerkin(ctx, E);
}

// ---------------------------------------------------------------------------
// svdguess_mult: the product's site tensors streamed right to left with truncation
// ---------------------------------------------------------------------------
imps_state* mult_guess(Context* ctx, const imps_mpo* W, const imps_state* ket, int D, double tol, int maxiter,
                       GaugeResult* gres) {
  Fp64Scope fp64(ctx);
  const int N = ket->N;
  IMPS_REQUIRE(N % W->N == 0, IMPS_DIM_MISMATCH, "incompatible unit-cell lengths of MPS and MPO");
  IMPS_REQUIRE(D >= 1, IMPS_INVALID_ARG, "mult: bond dimension must be positive");
  auto Wl = [&](int l) -> const MpoSite& { return W->sites[l % W->N]; };
  for (int l = 0; l < N; ++l)
    IMPS_REQUIRE(Wl(l).d == ket->d[l], IMPS_DIM_MISMATCH, "MPO physical dimension != state physical dimension");
  std::vector<DevBuf> out(N);
  std::vector<int> outL(N), outR(N);
  DevBuf& Bb = ctx->buf("guess_b", 16);
  int Brows = 0, Bcols = 0;  // B as (rows, d, cols)
  auto site = [&](int i, const dcplx* carry, int f) {
    const MpoSite& Wi = Wl(i);
    const int wl = Wi.m, d = Wi.d, wr = Wi.n;
    const int bl = ket->Dl(i), br = ket->Dr(i);
    Brows = wl * bl;
    if (!carry) {
      Bcols = wr * br;
      Bb.ensure((size_t)Brows * d * Bcols * sizeof(dcplx));
      k_mult_site<<<grid_for((int64_t)Brows * d * Bcols), 256, 0, ctx->stream>>>(wl, d, wr, bl, br, Wi.Wdev.z(),
                                                                                 ket->AL[i].z(), Bb.z());
      launched(ctx, "mult site");
      return;
    }
    Bcols = f;
    // l4[wr, br, f] -> l4p[br, wr, f]; Tb = AL (bl d x br) l4p (br x wr f) = Tb[bl, d, wr, f]
    DevBuf& l4p = ctx->buf("guess_l4p", (size_t)wr * br * f * sizeof(dcplx));
    k_swap01<<<grid_for((int64_t)wr * br * f), 256, 0, ctx->stream>>>(wr, br, f, carry, l4p.z());
    launched(ctx, "mult swap");
    DevBuf& Tb = ctx->buf("guess_tb", (size_t)bl * d * wr * f * sizeof(dcplx));
    zgemm(ctx, OP_N, OP_N, bl * d, wr * f, br, 1.0, ket->AL[i].z(), (int64_t)bl * d, 0, l4p.z(), br, 0, 0.0, Tb.z(),
          (int64_t)bl * d, 0, 1);
    Bb.ensure((size_t)Brows * d * f * sizeof(dcplx));
    k_mult_carry<<<grid_for((int64_t)Brows * d * f), 256, 0, ctx->stream>>>(wl, d, wr, bl, f, Wi.Wdev.z(), Tb.z(),
                                                                            Bb.z());
    launched(ctx, "mult carry");
  };
  // tsvd(B, (1,), (2, 3); truncdim(D)): B (rows x d cols) = U diag(s) V^H
  DevBuf& Ub = ctx->buf("guess_u", 16);
  DevBuf& Vb = ctx->buf("guess_v", 16);
  DevBuf& carry = ctx->buf("guess_carry", 16);
  auto tsvd_rows = [&](int d, std::vector<double>& s) {
    const int m = Brows, n = d * Bcols, kk = std::min({D, m, n});
    Ub.ensure((size_t)m * kk * sizeof(dcplx));
    Vb.ensure((size_t)n * kk * sizeof(dcplx));
    return svd_thin(ctx, m, n, Bb.z(), m, D, -1.0, Ub.z(), s, Vb.z());
  };
  site(N - 1, nullptr, 0);
  for (int i = N - 1; i >= 1; --i) {
    const int d = Wl(i).d;
    std::vector<double> s;
    const int k = tsvd_rows(d, s);
    const int cols = Bcols;
    out[i].alloc((size_t)k * d * cols * sizeof(dcplx));
    zconj_transpose(ctx, d * cols, k, Vb.z(), (int64_t)d * cols, out[i].z(), k);   // V^H (k x d cols)
    outL[i] = k;
    outR[i] = cols;
    const int rows = Brows;
    carry.ensure((size_t)rows * k * sizeof(dcplx));
    zcopy(ctx, (int64_t)rows * k, Ub.z(), carry.z());
    scale_cols(ctx, rows, k, carry.z(), s);
    site(i - 1, carry.z(), k);
  }
  {
    const int d = Wl(0).d;
    std::vector<double> s;
    const int k = tsvd_rows(d, s);
    const int cols = Bcols, rows = Brows;
    // out[0] = diag(s) V^H  (k x d cols)
    DevBuf& v3 = ctx->buf("guess_v3", (size_t)k * d * cols * sizeof(dcplx));
    zcopy(ctx, (int64_t)d * cols * k, Vb.z(), v3.z());
    scale_cols(ctx, d * cols, k, v3.z(), s);
    out[0].alloc((size_t)k * d * cols * sizeof(dcplx));
    zconj_transpose(ctx, d * cols, k, v3.z(), (int64_t)d * cols, out[0].z(), k);
    outL[0] = k;
    outR[0] = cols;
    if (N >= 2) {
      // u^T absorbed into the right leg of site N-1: A[a, s, b] = sum_bb NL[a, s, bb] u[bb, b]
      const int l = N - 1, r = outL[l] * Wl(l).d;
      IMPS_REQUIRE(outR[l] == rows, IMPS_DIM_MISMATCH, "mult guess: wrap bond mismatch");
      DevBuf t;
      t.alloc((size_t)r * k * sizeof(dcplx));
      zgemm(ctx, OP_N, OP_N, r, k, rows, 1.0, out[l].z(), r, 0, Ub.z(), rows, 0, 0.0, t.z(), r, 0, 1);
      out[l] = std::move(t);
      outR[l] = k;
    } else {
      // one site: the second bond of the approximate guess by another SVD, (k d) x cols
      const int m = k * d, n = cols;
      std::vector<double> s2;
      DevBuf& U2 = ctx->buf("guess_u2", (size_t)m * std::min({D, m, n}) * sizeof(dcplx));
      DevBuf& V2 = ctx->buf("guess_v2", (size_t)n * std::min({D, m, n}) * sizeof(dcplx));
      const int k2 = svd_thin(ctx, m, n, out[0].z(), m, D, -1.0, U2.z(), s2, V2.z());
      DevBuf t;
      t.alloc((size_t)m * k2 * sizeof(dcplx));
      zcopy(ctx, (int64_t)m * k2, U2.z(), t.z());
      scale_cols(ctx, m, k2, t.z(), s2);
      out[0] = std::move(t);
      outR[0] = k2;
      IMPS_REQUIRE(k2 == k, IMPS_DIM_MISMATCH, "mult guess: one-site bonds differ after truncation");
    }
  }
  for (int l = 0; l < N; ++l)
    IMPS_REQUIRE(outR[l] == outL[(l + 1) % N], IMPS_DIM_MISMATCH, "mult guess: bond chain mismatch");
  imps_state* st = new imps_state();
  try {
    st->ctx = ctx;
    st->device = ctx->device;
    st->N = N;
    st->d = ket->d;
    st->chi = outR;
    st->AL.resize(N);
    st->AR.resize(N);
    st->C.resize(N);
    st->AC.resize(N);
    for (int l = 0; l < N; ++l) {
      st->AL[l].alloc(st->site_elems(l) * sizeof(dcplx));
      st->AR[l].alloc(st->site_elems(l) * sizeof(dcplx));
      st->AC[l].alloc(st->site_elems(l) * sizeof(dcplx));
      st->C[l].alloc(st->bond_elems(l) * sizeof(dcplx));
    }
    std::vector<const dcplx*> ptrs(N);
    for (int l = 0; l < N; ++l) ptrs[l] = out[l].z();
    GaugeResult g = canonicalize(ctx, st, ptrs, tol, maxiter);
    if (gres) *gres = g;
  } catch (...) {
    delete st;
    throw;
  }
  return st;
}

}  // namespace imps
