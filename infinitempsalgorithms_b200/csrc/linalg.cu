// QRpos / LQpos on the device (FiniteMPSAlgorithms `leftorth(.; alg = QRpos())`
// and `rightorth(.; alg = LQpos())` as used in src/states/ortho.jl:150, 188, 214-225).
//
// Householder QR from cuSOLVER (zgeqrf + zungqr), then a phase fix that makes
// diag(R) real and non-negative: Q[:, i] *= ph_i, R[i, :] *= conj(ph_i) with
// ph_i = R_ii / |R_ii| (1 when R_ii == 0).  LQ is QR of the conjugate transpose.
#include "imps_internal.h"

namespace imps {

void scale_q_r(Context* ctx, int m, int n, int k, dcplx* Q, int64_t ldq, dcplx* R, int64_t ldr, const dcplx* ph);

namespace {

__global__ void k_extract_r(int k, int n, const dcplx* __restrict__ A, int64_t lda, dcplx* __restrict__ R,
                            int64_t ldr, dcplx* __restrict__ ph) {
  int64_t tot = (int64_t)k * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t % k), c = (int)(t / k);
    dcplx v = (r <= c) ? A[r + lda * c] : make_double2(0.0, 0.0);
    R[r + ldr * c] = v;
    if (r == c) {
      double a = hypot(v.x, v.y);
      ph[r] = (a > 0.0) ? make_double2(v.x / a, v.y / a) : make_double2(1.0, 0.0);
    }
  }
}

}  // namespace

void qrpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* Q, dcplx* R) {
  IMPS_REQUIRE(m > 0 && n > 0, IMPS_INVALID_ARG, "qrpos: empty matrix");
  ctx->n_qr++;
  const int k = std::min(m, n);
  const double qf = 8.0 * (2.0 * m * (double)n * k - 2.0 / 3.0 * k * (double)k * k) * 2.0;
  ctx->qr_flops += qf;
  ScopedTimer t(ctx, "qr", qf);
  DevBuf& Abuf = ctx->buf("qr_a", (size_t)m * n * sizeof(dcplx));
  DevBuf& tau = ctx->buf("qr_tau", (size_t)k * sizeof(dcplx));
  DevBuf& ph = ctx->buf("qr_ph", (size_t)k * sizeof(dcplx));
  zcopy2d(ctx, m, n, M, ldm, Abuf.z(), m);
  cuDoubleComplex* A = reinterpret_cast<cuDoubleComplex*>(Abuf.ptr);
  int lw1 = 0, lw2 = 0;
  IMPS_SOLVER(cusolverDnZgeqrf_bufferSize(ctx->solver, m, n, A, m, &lw1));
  IMPS_SOLVER(cusolverDnZungqr_bufferSize(ctx->solver, m, k, k, A, m, reinterpret_cast<cuDoubleComplex*>(tau.ptr), &lw2));
  int lw = std::max(lw1, lw2);
  DevBuf& work = ctx->buf("qr_work", (size_t)std::max(lw, 1) * sizeof(cuDoubleComplex));
  IMPS_SOLVER(cusolverDnZgeqrf(ctx->solver, m, n, A, m, reinterpret_cast<cuDoubleComplex*>(tau.ptr),
                               reinterpret_cast<cuDoubleComplex*>(work.ptr), lw, ctx->dev_info));
  {
    int64_t tot = (int64_t)k * n;
    int g = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
    k_extract_r<<<std::max(g, 1), 256, 0, ctx->stream>>>(k, n, Abuf.z(), m, R, k, ph.z());
    ctx->n_kernels++;
  }
  IMPS_SOLVER(cusolverDnZungqr(ctx->solver, m, k, k, A, m, reinterpret_cast<cuDoubleComplex*>(tau.ptr),
                               reinterpret_cast<cuDoubleComplex*>(work.ptr), lw, ctx->dev_info));
  zcopy2d(ctx, m, k, Abuf.z(), m, Q, m);
  scale_q_r(ctx, m, n, k, Q, m, R, k, ph.z());
}

void lqpos(Context* ctx, int m, int n, const dcplx* M, int64_t ldm, dcplx* L, dcplx* Q) {
  // M (m x n) = L Q  <=>  M^H = Q^H L^H : QRpos of M^H (n x m) gives Q' (n x k), R' (k x m)
  const int k = std::min(m, n);
  DevBuf& MH = ctx->buf("lq_mh", (size_t)m * n * sizeof(dcplx));
  DevBuf& Qp = ctx->buf("lq_q", (size_t)n * k * sizeof(dcplx));
  DevBuf& Rp = ctx->buf("lq_r", (size_t)k * m * sizeof(dcplx));
  zconj_transpose(ctx, m, n, M, ldm, MH.z(), n);
  qrpos(ctx, n, m, MH.z(), n, Qp.z(), Rp.z());
  zconj_transpose(ctx, k, m, Rp.z(), k, L, m);   // L = R'^H  (m x k)
  zconj_transpose(ctx, n, k, Qp.z(), n, Q, k);   // Q = Q'^H  (k x n)
}

}  // namespace imps
