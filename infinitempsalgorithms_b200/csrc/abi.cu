// The extern "C" boundary (include/imps_b200.h).  Every entry point catches
// exceptions and maps them to IMPS_* status codes; the message is kept in the
// context (imps_ctx_last_error) and in a thread-local fallback.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <string>

#include "algos.h"
#include "envs.h"
#include "gauge.h"
#include "imps_internal.h"
#include "krylov.h"
#include "mpo.h"
#include "mult.h"
#include "observables.h"

struct imps_ctx {
  imps::Context c;
};

namespace {
thread_local std::string g_last_error;

template <class F>
int guard(imps::Context* ctx, F&& f) {
  try {
    if (ctx) cudaSetDevice(ctx->device);
    int r = f();
    // a bounded wait that ran out inside this call surfaces here at the latest
    if (ctx) imps::check_device_errors(ctx);
    return r;
  } catch (const imps::Error& e) {
    g_last_error = e.what();
    if (ctx) ctx->last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc& e) {
    g_last_error = "host allocation failed";
    if (ctx) ctx->last_error = g_last_error;
    return IMPS_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    if (ctx) ctx->last_error = e.what();
    return IMPS_CUDA_ERROR;
  }
}

const imps::dcplx* zc(const double* p) { return reinterpret_cast<const imps::dcplx*>(p); }
imps::dcplx* zm(double* p) { return reinterpret_cast<imps::dcplx*>(p); }
const imps::cplx* hc(const double* p) { return reinterpret_cast<const imps::cplx*>(p); }

void fill_info(imps_krylov_info* info, const imps::KrylovResult& r) {
  if (!info) return;
  info->converged = r.converged;
  info->numiter = r.numiter;
  info->numops = r.numops;
  info->pad = 0;
  info->normres = r.normres;
  info->value_re = r.value.real();
  info->value_im = r.value.imag();
}

void fill_gauge(imps_gauge_info* info, const imps::GaugeResult& g) {
  if (!info) return;
  info->niter = g.niter;
  info->converged = g.converged;
  info->err = g.err;
}

imps::DevBuf& state_field(imps_state* st, int field, int site) {
  IMPS_REQUIRE(site >= 0 && site < st->N, IMPS_INVALID_ARG, "site index out of range");
  switch (field) {
    case IMPS_AL: return st->AL[site];
    case IMPS_AR: return st->AR[site];
    case IMPS_C: return st->C[site];
    case IMPS_AC: return st->AC[site];
    default: throw imps::Error(IMPS_INVALID_ARG, "unknown state field");
  }
}
size_t field_elems(const imps_state* st, int field, int site) {
  return field == IMPS_C ? st->bond_elems(site) : st->site_elems(site);
}

void check_site(const imps_envs* E, int site) {
  IMPS_REQUIRE(E && site >= 0 && site < E->N, IMPS_INVALID_ARG, "site index out of range");
}

int conv_status(int converged) { return converged ? IMPS_OK : IMPS_NOT_CONVERGED; }
}  // namespace

extern "C" {

const char* imps_status_string(int s) {
  switch (s) {
    case IMPS_OK: return "ok";
    case IMPS_NOT_CONVERGED: return "not converged";
    case IMPS_DIM_MISMATCH: return "dimension mismatch";
    case IMPS_INVALID_ARG: return "invalid argument";
    case IMPS_OOM: return "out of memory";
    case IMPS_CUDA_ERROR: return "CUDA error";
    case IMPS_TIMEOUT: return "timeout";
    case IMPS_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

int imps_ctx_create(int device, imps_ctx** out) {
  if (!out) return IMPS_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    g_last_error = "no CUDA device visible";
    return IMPS_NO_DEVICE;
  }
  if (device < 0 || device >= n) return IMPS_INVALID_ARG;
  imps_ctx* h = new imps_ctx();
  int r = guard(nullptr, [&] {
    imps::Context& c = h->c;
    c.device = device;
    IMPS_CUDA(cudaSetDevice(device));
    IMPS_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.own_stream = true;
    IMPS_CUDA(cudaMalloc((void**)&c.dev_info, sizeof(int) * 4));
    IMPS_CUDA(cudaMalloc((void**)&c.err_dev, sizeof(int) * 4));
    IMPS_CUDA(cudaMemset(c.err_dev, 0, sizeof(int) * 4));
    IMPS_CUDA(cudaMallocHost((void**)&c.err_host, sizeof(int) * 4));
    c.err_host[0] = 0;
    cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, device);
    if (const char* e = std::getenv("IMPS_FP64_ENGINE")) c.fp64_engine = std::atoi(e) == 1 ? 1 : 0;
    // the allocation-free entry point's fixed array is created with the context,
    // before the caller's allocator takes the rest of the device memory
    imps::noalloc_prepare(device);
    return IMPS_OK;
  });
  if (r != IMPS_OK) {
    delete h;
    return r;
  }
  *out = h;
  return IMPS_OK;
}

int imps_ctx_destroy(imps_ctx* h) {
  if (!h) return IMPS_OK;
  imps::Context& c = h->c;
  cudaSetDevice(c.device);
  cudaStreamSynchronize(c.stream);
  for (auto& p : c.pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  for (auto e : c.event_pool) cudaEventDestroy(e);
  c.scratch.clear();
  c.red.release();
  if (c.host_pinned) cudaFreeHost(c.host_pinned);
  if (c.dev_info) cudaFree(c.dev_info);
  if (c.err_dev) cudaFree(c.err_dev);
  if (c.err_host) cudaFreeHost(c.err_host);
  if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
  delete h;
  return IMPS_OK;
}

int imps_ctx_set_stream(imps_ctx* h, void* stream) {
  if (!h) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context& c = h->c;
    IMPS_CUDA(cudaStreamSynchronize(c.stream));
    if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
    c.stream = static_cast<cudaStream_t>(stream);
    c.own_stream = false;
    return IMPS_OK;
  });
}

int imps_ctx_set_precision(imps_ctx* h, int mode, int nslices) {
  if (!h) return IMPS_INVALID_ARG;
  if (mode != IMPS_PREC_FP64 && mode != IMPS_PREC_SPLIT_I8) return IMPS_INVALID_ARG;
  if (nslices > 8) return IMPS_INVALID_ARG;
  if (mode == IMPS_PREC_SPLIT_I8 && nslices > 0 && nslices < 2) return IMPS_INVALID_ARG;
  h->c.precision = mode;
  h->c.adaptive_slices = nslices <= 0;
  if (nslices > 0) h->c.nslices = nslices;
  return IMPS_OK;
}

int imps_ctx_synchronize(imps_ctx* h) {
  if (!h) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    IMPS_CUDA(cudaStreamSynchronize(h->c.stream));
    return IMPS_OK;
  });
}

int imps_ctx_set_wait_limit(imps_ctx* h, int64_t cycles) {
  if (!h || cycles < 0) return IMPS_INVALID_ARG;
  h->c.wait_cycles = cycles > 0 ? (long long)cycles : 2000000000LL;
  return IMPS_OK;
}

int imps_ctx_set_workspace_limit(imps_ctx* h, int64_t bytes) {
  if (!h || bytes < 0) return IMPS_INVALID_ARG;
  h->c.workspace_limit = (size_t)bytes;
  return IMPS_OK;
}

int imps_ctx_workspace_bytes(imps_ctx* h, int64_t* bytes) {
  if (!h || !bytes) return IMPS_INVALID_ARG;
  size_t total = 0;
  for (const auto& kv : h->c.scratch) total += kv.second.bytes;
  *bytes = (int64_t)total;
  return IMPS_OK;
}

int imps_ctx_counters_ext(imps_ctx* h, int64_t* c, int n) {
  if (!h || !c || n < 0) return IMPS_INVALID_ARG;
  const imps::Context& x = h->c;
  const int64_t all[11] = {x.n_ac_apply, x.n_c_apply, x.n_push, x.n_gemm, x.n_kernels, x.n_qr,
                           (int64_t)x.gemm_flops, (int64_t)x.qr_flops, x.split_launches,
                           (int64_t)x.split_alg_flops, (int64_t)x.split_exec_ops};
  for (int i = 0; i < n; ++i) c[i] = i < 11 ? all[i] : 0;
  return IMPS_OK;
}

const char* imps_ctx_last_error(const imps_ctx* h) {
  if (!h) return g_last_error.c_str();
  return h->c.last_error.c_str();
}

int imps_ctx_profile(imps_ctx* h, int enable) {
  if (!h) return IMPS_INVALID_ARG;
  h->c.profile = enable != 0;
  return IMPS_OK;
}

static void flush_profile(imps::Context& c) {
  if (c.pending.empty()) return;
  cudaStreamSynchronize(c.stream);
  for (size_t i = 0; i < c.pending.size(); ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.pending[i].second.first, c.pending[i].second.second);
    imps::KernelStat& s = c.stats[c.pending[i].first];
    s.launches++;
    s.ms += ms;
    s.flops += c.pending_flops[i];
    c.event_pool.push_back(c.pending[i].second.first);
    c.event_pool.push_back(c.pending[i].second.second);
  }
  c.pending.clear();
  c.pending_flops.clear();
}

int imps_ctx_profile_get(imps_ctx* h, const char* cls, int64_t* launches, double* total_ms, double* work) {
  if (!h || !cls) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    flush_profile(h->c);
    auto it = h->c.stats.find(cls);
    if (launches) *launches = it == h->c.stats.end() ? 0 : it->second.launches;
    if (total_ms) *total_ms = it == h->c.stats.end() ? 0.0 : it->second.ms;
    if (work) *work = it == h->c.stats.end() ? 0.0 : it->second.flops;
    return IMPS_OK;
  });
}

int imps_ctx_profile_classes(imps_ctx* h, const char* csv) {
  if (!h) return IMPS_INVALID_ARG;
  h->c.profile_only.clear();
  if (csv) {
    std::string s(csv), cur;
    for (char ch : s) {
      if (ch == ',') { if (!cur.empty()) h->c.profile_only.insert(cur); cur.clear(); }
      else cur += ch;
    }
    if (!cur.empty()) h->c.profile_only.insert(cur);
  }
  return IMPS_OK;
}

int imps_ctx_profile_dump(imps_ctx* h, char* buf, int64_t len) {
  if (!h || !buf || len <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    flush_profile(h->c);
    std::string out;
    for (auto& kv : h->c.stats) {
      char line[256];
      snprintf(line, sizeof(line), "%s %lld %.6f %.6e\n", kv.first.c_str(), (long long)kv.second.launches,
               kv.second.ms, kv.second.flops);
      out += line;
    }
    IMPS_REQUIRE((int64_t)out.size() < len, IMPS_INVALID_ARG, "profile dump buffer too small");
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return IMPS_OK;
  });
}

int imps_ctx_profile_reset(imps_ctx* h) {
  if (!h) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    flush_profile(h->c);
    h->c.stats.clear();
    return IMPS_OK;
  });
}

int imps_ctx_counters(imps_ctx* h, int64_t* c) {
  if (!h || !c) return IMPS_INVALID_ARG;
  c[0] = h->c.n_ac_apply;
  c[1] = h->c.n_c_apply;
  c[2] = h->c.n_push;
  c[3] = h->c.n_gemm;
  c[4] = h->c.n_kernels;
  c[5] = h->c.n_qr;
  c[6] = (int64_t)h->c.gemm_flops;
  c[7] = (int64_t)h->c.qr_flops;
  return IMPS_OK;
}

// ------------------------------------------------------------------ MPO
int imps_mpo_create(imps_ctx* h, int N, const int* m, const int* d, const int* n, const double* const* W,
                    imps_mpo** out) {
  if (!h || !out || !m || !d || !n || !W || N <= 0) return IMPS_INVALID_ARG;
  *out = nullptr;
  imps_mpo* mpo = new imps_mpo();
  int r = guard(&h->c, [&] {
    mpo->ctx = &h->c;
    mpo->device = h->c.device;
    mpo->N = N;
    mpo->sites.resize(N);
    mpo->closing.resize(N);
    for (int l = 0; l < N; ++l) {
      IMPS_REQUIRE(W[l] != nullptr, IMPS_INVALID_ARG, "null MPO tensor");
      imps::make_mpo_site(&h->c, mpo->sites[l], m[l], d[l], n[l], hc(W[l]));
      imps::make_closing_column(&h->c, mpo->sites[l], mpo->closing[l]);
    }
    for (int l = 0; l < N; ++l) {
      int l1 = (l + 1) % N;
      IMPS_REQUIRE(n[l] == m[l1], IMPS_DIM_MISMATCH, "level chain mismatch between neighbouring MPO tensors");
    }
    return IMPS_OK;
  });
  if (r != IMPS_OK) {
    delete mpo;
    return r;
  }
  *out = mpo;
  return IMPS_OK;
}

// Destroy functions never dereference the context: an object may outlive it.
int imps_mpo_destroy(imps_mpo* mpo) {
  if (!mpo) return IMPS_OK;
  cudaSetDevice(mpo->device);
  cudaDeviceSynchronize();
  delete mpo;
  return IMPS_OK;
}

// ------------------------------------------------------------------ state
int imps_state_create(imps_ctx* h, int N, const int* d, const int* chi, imps_state** out) {
  if (!h || !out || !d || !chi || N <= 0) return IMPS_INVALID_ARG;
  *out = nullptr;
  imps_state* st = new imps_state();
  int r = guard(&h->c, [&] {
    st->ctx = &h->c;
    st->device = h->c.device;
    st->N = N;
    st->d.assign(d, d + N);
    st->chi.assign(chi, chi + N);
    for (int l = 0; l < N; ++l) IMPS_REQUIRE(d[l] > 0 && chi[l] > 0, IMPS_INVALID_ARG, "empty dimension");
    st->AL.resize(N);
    st->AR.resize(N);
    st->C.resize(N);
    st->AC.resize(N);
    for (int l = 0; l < N; ++l) {
      size_t se = st->site_elems(l) * sizeof(imps::dcplx), be = st->bond_elems(l) * sizeof(imps::dcplx);
      st->AL[l].ensure(se);
      st->AR[l].ensure(se);
      st->AC[l].ensure(se);
      st->C[l].ensure(be);
      IMPS_CUDA(cudaMemsetAsync(st->AL[l].ptr, 0, se, h->c.stream));
      IMPS_CUDA(cudaMemsetAsync(st->AR[l].ptr, 0, se, h->c.stream));
      IMPS_CUDA(cudaMemsetAsync(st->AC[l].ptr, 0, se, h->c.stream));
      IMPS_CUDA(cudaMemsetAsync(st->C[l].ptr, 0, be, h->c.stream));
    }
    return IMPS_OK;
  });
  if (r != IMPS_OK) {
    delete st;
    return r;
  }
  *out = st;
  return IMPS_OK;
}

int imps_state_destroy(imps_state* st) {
  if (!st) return IMPS_OK;
  cudaSetDevice(st->device);
  cudaDeviceSynchronize();
  delete st;
  return IMPS_OK;
}

int imps_state_set(imps_state* st, int field, int site, const double* host) {
  if (!st || !host) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::DevBuf& b = state_field(st, field, site);
    imps::upload(st->ctx, b.ptr, host, field_elems(st, field, site) * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_state_get(const imps_state* st, int field, int site, double* host) {
  if (!st || !host) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::DevBuf& b = state_field(const_cast<imps_state*>(st), field, site);
    imps::download(st->ctx, host, b.ptr, field_elems(st, field, site) * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_state_copy(imps_state* dst, const imps_state* src) {
  if (!dst || !src) return IMPS_INVALID_ARG;
  return guard(dst->ctx, [&] {
    IMPS_REQUIRE(dst->N == src->N && dst->d == src->d && dst->chi == src->chi, IMPS_DIM_MISMATCH,
                 "state shapes differ");
    for (int l = 0; l < src->N; ++l) {
      imps::zcopy(dst->ctx, src->site_elems(l), src->AL[l].z(), dst->AL[l].z());
      imps::zcopy(dst->ctx, src->site_elems(l), src->AR[l].z(), dst->AR[l].z());
      imps::zcopy(dst->ctx, src->site_elems(l), src->AC[l].z(), dst->AC[l].z());
      imps::zcopy(dst->ctx, src->bond_elems(l), src->C[l].z(), dst->C[l].z());
    }
    return IMPS_OK;
  });
}

int imps_state_canonicalize(imps_state* st, const double* const* As, double tol, int maxiter, imps_gauge_info* info) {
  if (!st || !As) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::Context* ctx = st->ctx;
    size_t total = 0;
    for (int l = 0; l < st->N; ++l) total += st->site_elems(l);
    imps::DevBuf& in = ctx->buf("canon_in", total * sizeof(imps::dcplx));
    std::vector<const imps::dcplx*> ptrs(st->N);
    size_t off = 0;
    for (int l = 0; l < st->N; ++l) {
      IMPS_REQUIRE(As[l] != nullptr, IMPS_INVALID_ARG, "null site tensor");
      imps::upload(ctx, in.z() + off, As[l], st->site_elems(l) * sizeof(imps::dcplx));
      ptrs[l] = in.z() + off;
      off += st->site_elems(l);
    }
    imps::GaugeResult g = imps::canonicalize(ctx, st, ptrs, tol, maxiter);
    fill_gauge(info, g);
    return conv_status(g.converged);
  });
}

int imps_state_from_al(imps_state* st, const double* const* ALs, const double* C0, double tol, int maxiter,
                       imps_gauge_info* info) {
  if (!st || !ALs || !C0) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::Context* ctx = st->ctx;
    for (int l = 0; l < st->N; ++l) {
      IMPS_REQUIRE(ALs[l] != nullptr, IMPS_INVALID_ARG, "null site tensor");
      imps::upload(ctx, st->AL[l].ptr, ALs[l], st->site_elems(l) * sizeof(imps::dcplx));
    }
    const int DN = st->Dr(st->N - 1);
    imps::DevBuf& c0 = ctx->buf("abi_c0", (size_t)DN * DN * sizeof(imps::dcplx));
    imps::upload(ctx, c0.ptr, C0, (size_t)DN * DN * sizeof(imps::dcplx));
    imps::GaugeResult g = imps::from_al(ctx, st, c0.z(), tol, maxiter);
    fill_gauge(info, g);
    return conv_status(g.converged);
  });
}

int imps_gauge_step(imps_state* st, double tol, int maxiter, imps_gauge_info* info) {
  if (!st) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::Context* ctx = st->ctx;
    const int DN = st->Dr(st->N - 1);
    imps::DevBuf& c0 = ctx->buf("vumps_c0", (size_t)DN * DN * sizeof(imps::dcplx));
    imps::zcopy(ctx, (int64_t)DN * DN, st->C[st->N - 1].z(), c0.z());
    imps::GaugeResult g = imps::from_al(ctx, st, c0.z(), tol, maxiter);
    fill_gauge(info, g);
    return conv_status(g.converged);
  });
}

int imps_state_dot(imps_state* st, double* re, double* im) {
  if (!st) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::cplx v = imps::state_dot(st->ctx, st);
    if (re) *re = v.real();
    if (im) *im = v.imag();
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ envs
int imps_envs_create(imps_ctx* h, const imps_state* st, const imps_mpo* mpo, imps_envs** out) {
  if (!h || !st || !mpo || !out) return IMPS_INVALID_ARG;
  *out = nullptr;
  imps_envs* E = new imps_envs();
  int r = guard(&h->c, [&] {
    E->ctx = &h->c;
    E->device = h->c.device;
    imps::envs_allocate(E, st, mpo);
    for (int l = 0; l < E->N; ++l) {
      imps::zfill(&h->c, (int64_t)(E->lefts[l].bytes / sizeof(imps::dcplx)), 0.0, E->lefts[l].z());
      imps::zfill(&h->c, (int64_t)(E->rights[l].bytes / sizeof(imps::dcplx)), 0.0, E->rights[l].z());
    }
    return IMPS_OK;
  });
  if (r != IMPS_OK) {
    delete E;
    return r;
  }
  *out = E;
  return IMPS_OK;
}

int imps_envs_destroy(imps_envs* E) {
  if (!E) return IMPS_OK;
  cudaSetDevice(E->device);
  cudaDeviceSynchronize();
  delete E;
  return IMPS_OK;
}

int imps_envs_build(imps_envs* E, const imps_state* st, const imps_mpo* mpo, double tol, int maxiter, int krylovdim,
                    int warm, imps_env_info* info) {
  if (!E || !st || !mpo) return IMPS_INVALID_ARG;
  if (tol <= 0 || maxiter <= 0 || krylovdim <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps_env_info ei = imps::envs_build(E->ctx, E, st, mpo, tol, maxiter, krylovdim, warm != 0);
    if (info) *info = ei;
    return conv_status(ei.converged);
  });
}

int imps_envs_get(const imps_envs* E, int side, int site, double* host) {
  if (!E || !host) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    const imps::DevBuf& b = side == 0 ? E->lefts[site] : E->rights[site];
    size_t n = side == 0 ? (size_t)E->Dl[site] * E->ml[site] * E->Dl[site] : (size_t)E->Dr[site] * E->nr[site] * E->Dr[site];
    imps::download(E->ctx, host, b.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_envs_set(imps_envs* E, int side, int site, const double* host) {
  if (!E || !host) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    imps::DevBuf& b = side == 0 ? E->lefts[site] : E->rights[site];
    size_t n = side == 0 ? (size_t)E->Dl[site] * E->ml[site] * E->Dl[site] : (size_t)E->Dr[site] * E->nr[site] * E->Dr[site];
    imps::upload(E->ctx, b.ptr, host, n * sizeof(imps::dcplx));
    E->GLp_valid[site] = false;
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ Heff
int imps_ac_apply_dev(imps_envs* E, const imps_mpo* mpo, int site, const void* x, void* y) {
  if (!E || !mpo || !x || !y) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    imps::ac_apply(E->ctx, E, mpo, site, static_cast<const imps::dcplx*>(x), static_cast<imps::dcplx*>(y));
    return IMPS_OK;
  });
}

int imps_ac_apply(imps_envs* E, const imps_mpo* mpo, int site, const double* x, double* y) {
  if (!E || !mpo || !x || !y) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    imps::Context* ctx = E->ctx;
    const int64_t n = (int64_t)E->Dl[site] * mpo->sites[site % mpo->N].d * E->Dr[site];
    imps::DevBuf& xd = ctx->buf("abi_x", n * sizeof(imps::dcplx));
    imps::DevBuf& yd = ctx->buf("abi_y", n * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, x, n * sizeof(imps::dcplx));
    imps::ac_apply(ctx, E, mpo, site, xd.z(), yd.z());
    imps::download(ctx, y, yd.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_ac_apply_noalloc(imps_ctx* h, int Dl, int d, int Dr, int m, int n, const double* W_host, const void* GL,
                          const void* GR, const void* x, void* y) {
  if (!h || !W_host || !GL || !GR || !x || !y) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::ac_apply_noalloc(&h->c, Dl, d, Dr, m, n, hc(W_host), static_cast<const imps::dcplx*>(GL),
                           static_cast<const imps::dcplx*>(GR), static_cast<const imps::dcplx*>(x),
                           static_cast<imps::dcplx*>(y));
    return IMPS_OK;
  });
}

int imps_c_apply_dev(imps_envs* E, int site, const void* x, void* y) {
  if (!E || !x || !y) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    imps::c_apply(E->ctx, E, site, static_cast<const imps::dcplx*>(x), static_cast<imps::dcplx*>(y));
    return IMPS_OK;
  });
}

int imps_c_apply(imps_envs* E, int site, const double* x, double* y) {
  if (!E || !x || !y) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    imps::Context* ctx = E->ctx;
    const int64_t n = (int64_t)E->Dr[site] * E->Dr[site];
    imps::DevBuf& xd = ctx->buf("abi_x", n * sizeof(imps::dcplx));
    imps::DevBuf& yd = ctx->buf("abi_y", n * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, x, n * sizeof(imps::dcplx));
    imps::c_apply(ctx, E, site, xd.z(), yd.z());
    imps::download(ctx, y, yd.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ pushes
static int push_id_common(imps_ctx* h, int Dl, int d, int Dr, const double* X, const double* above,
                          const double* below, double* out, bool left) {
  if (!h || !X || !above || !below || !out || Dl <= 0 || d <= 0 || Dr <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    const int Din = left ? Dl : Dr, Dout = left ? Dr : Dl;
    const int64_t sa = (int64_t)Dl * d * Dr;
    imps::DevBuf& xd = ctx->buf("abi_x", (size_t)Din * Din * sizeof(imps::dcplx));
    imps::DevBuf& ad = ctx->buf("abi_a", sa * sizeof(imps::dcplx));
    imps::DevBuf& bd = ctx->buf("abi_b", sa * sizeof(imps::dcplx));
    imps::DevBuf& od = ctx->buf("abi_y", (size_t)Dout * Dout * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, X, (size_t)Din * Din * sizeof(imps::dcplx));
    imps::upload(ctx, ad.ptr, above, sa * sizeof(imps::dcplx));
    imps::upload(ctx, bd.ptr, below, sa * sizeof(imps::dcplx));
    if (left) imps::push_left_id(ctx, Dl, d, Dr, xd.z(), ad.z(), bd.z(), od.z());
    else imps::push_right_id(ctx, Dl, d, Dr, xd.z(), ad.z(), bd.z(), od.z());
    imps::download(ctx, out, od.ptr, (size_t)Dout * Dout * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_push_left(imps_ctx* h, int Dl, int d, int Dr, const double* L, const double* above, const double* below,
                   double* out) {
  return push_id_common(h, Dl, d, Dr, L, above, below, out, true);
}
int imps_push_right(imps_ctx* h, int Dl, int d, int Dr, const double* R, const double* above, const double* below,
                    double* out) {
  return push_id_common(h, Dl, d, Dr, R, above, below, out, false);
}

static int push_mpo_common(imps_ctx* h, const imps_mpo* mpo, int site, int Dl, int Dr, const double* X,
                           const double* A, double* out, bool left) {
  if (!h || !mpo || !X || !A || !out || Dl <= 0 || Dr <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    IMPS_REQUIRE(site >= 0, IMPS_INVALID_ARG, "site index out of range");
    imps::Context* ctx = &h->c;
    const imps::MpoSite& W = mpo->sites[site % mpo->N];
    const int d = W.d;
    const int64_t sa = (int64_t)Dl * d * Dr;
    const int64_t nin = left ? (int64_t)Dl * W.m * Dl : (int64_t)Dr * W.n * Dr;
    const int64_t nout = left ? (int64_t)Dr * W.n * Dr : (int64_t)Dl * W.m * Dl;
    imps::DevBuf& xd = ctx->buf("abi_x", nin * sizeof(imps::dcplx));
    imps::DevBuf& ad = ctx->buf("abi_a", sa * sizeof(imps::dcplx));
    imps::DevBuf& od = ctx->buf("abi_y", nout * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, X, nin * sizeof(imps::dcplx));
    imps::upload(ctx, ad.ptr, A, sa * sizeof(imps::dcplx));
    if (left) imps::push_mpo_left(ctx, W, Dl, d, Dr, xd.z(), ad.z(), od.z());
    else imps::push_mpo_right(ctx, W, Dl, d, Dr, xd.z(), ad.z(), od.z());
    imps::download(ctx, out, od.ptr, nout * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_push_mpo_left(imps_ctx* h, const imps_mpo* mpo, int site, int Dl, int Dr, const double* L, const double* A,
                       double* out) {
  return push_mpo_common(h, mpo, site, Dl, Dr, L, A, out, true);
}
int imps_push_mpo_right(imps_ctx* h, const imps_mpo* mpo, int site, int Dl, int Dr, const double* R, const double* A,
                        double* out) {
  return push_mpo_common(h, mpo, site, Dl, Dr, R, A, out, false);
}

// ------------------------------------------------------------------ GEMM
int imps_zgemm(imps_ctx* h, int opA, int opB, int M, int N, int K, double alpha_re, double alpha_im,
               const void* A, int64_t lda, const void* B, int64_t ldb, double beta_re, double beta_im, void* Cp,
               int64_t ldc) {
  if (!h || !A || !B || !Cp || M < 0 || N < 0 || K < 0) return IMPS_INVALID_ARG;
  if (opA < 0 || opA > 2 || opB < 0 || opB > 2) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::zgemm(&h->c, (imps::Op)opA, (imps::Op)opB, M, N, K, imps::cplx(alpha_re, alpha_im),
                static_cast<const imps::dcplx*>(A), lda, 0, static_cast<const imps::dcplx*>(B), ldb, 0,
                imps::cplx(beta_re, beta_im), static_cast<imps::dcplx*>(Cp), ldc, 0, 1, true);
    IMPS_CUDA(cudaStreamSynchronize(h->c.stream));
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ factorizations
int imps_qrpos(imps_ctx* h, int m, int n, const double* M, double* Q, double* R) {
  if (!h || !M || !Q || !R || m <= 0 || n <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    const int k = std::min(m, n);
    imps::DevBuf& md = ctx->buf("abi_x", (size_t)m * n * sizeof(imps::dcplx));
    imps::DevBuf& qd = ctx->buf("abi_a", (size_t)m * k * sizeof(imps::dcplx));
    imps::DevBuf& rd = ctx->buf("abi_b", (size_t)k * n * sizeof(imps::dcplx));
    imps::upload(ctx, md.ptr, M, (size_t)m * n * sizeof(imps::dcplx));
    imps::qrpos(ctx, m, n, md.z(), m, qd.z(), rd.z());
    imps::download(ctx, Q, qd.ptr, (size_t)m * k * sizeof(imps::dcplx));
    imps::download(ctx, R, rd.ptr, (size_t)k * n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_lqpos(imps_ctx* h, int m, int n, const double* M, double* L, double* Q) {
  if (!h || !M || !Q || !L || m <= 0 || n <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    const int k = std::min(m, n);
    imps::DevBuf& md = ctx->buf("abi_x", (size_t)m * n * sizeof(imps::dcplx));
    imps::DevBuf& ld = ctx->buf("abi_a", (size_t)m * k * sizeof(imps::dcplx));
    imps::DevBuf& qd = ctx->buf("abi_b", (size_t)k * n * sizeof(imps::dcplx));
    imps::upload(ctx, md.ptr, M, (size_t)m * n * sizeof(imps::dcplx));
    imps::lqpos(ctx, m, n, md.z(), m, ld.z(), qd.z());
    imps::download(ctx, L, ld.ptr, (size_t)m * k * sizeof(imps::dcplx));
    imps::download(ctx, Q, qd.ptr, (size_t)k * n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_regauge(imps_ctx* h, int Dl, int d, int Dr, const double* AC, const double* C, double* AL) {
  if (!h || !AC || !C || !AL || Dl <= 0 || d <= 0 || Dr <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    IMPS_REQUIRE(Dl * d >= Dr, IMPS_DIM_MISMATCH, "regauge!: Dl*d must be >= Dr");
    imps::Context* ctx = &h->c;
    const int64_t sa = (int64_t)Dl * d * Dr;
    imps::DevBuf& a = ctx->buf("abi_x", sa * sizeof(imps::dcplx));
    imps::DevBuf& c = ctx->buf("abi_a", (size_t)Dr * Dr * sizeof(imps::dcplx));
    imps::DevBuf& o = ctx->buf("abi_y", sa * sizeof(imps::dcplx));
    imps::upload(ctx, a.ptr, AC, sa * sizeof(imps::dcplx));
    imps::upload(ctx, c.ptr, C, (size_t)Dr * Dr * sizeof(imps::dcplx));
    imps::regauge(ctx, Dl, d, Dr, a.z(), c.z(), o.z());
    imps::download(ctx, AL, o.ptr, sa * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ Krylov
static int krylov_host(imps::Context* ctx, int64_t n, const double* x0, double* x,
                       const std::function<imps::KrylovResult(const imps::dcplx*, imps::dcplx*)>& run,
                       imps_krylov_info* info) {
  imps::DevBuf& xd = ctx->buf("abi_kx0", n * sizeof(imps::dcplx));
  imps::DevBuf& yd = ctx->buf("abi_kx", n * sizeof(imps::dcplx));
  imps::upload(ctx, xd.ptr, x0, n * sizeof(imps::dcplx));
  imps::KrylovResult r = run(xd.z(), yd.z());
  imps::download(ctx, x, yd.ptr, n * sizeof(imps::dcplx));
  fill_info(info, r);
  return conv_status(r.converged);
}

int imps_eigsolve_ac(imps_envs* E, const imps_mpo* mpo, int site, const double* x0, double* x, double tol,
                     int krylovdim, int maxiter, int eager, imps_krylov_info* info) {
  if (!E || !mpo || !x0 || !x || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    const int64_t n = (int64_t)E->Dl[site] * mpo->sites[site % mpo->N].d * E->Dr[site];
    return krylov_host(E->ctx, n, x0, x, [&](const imps::dcplx* a, imps::dcplx* b) {
      return imps::eigsolve_ac(E->ctx, E, mpo, site, a, b, tol, krylovdim, maxiter, eager != 0);
    }, info);
  });
}

int imps_eigsolve_c(imps_envs* E, int site, const double* x0, double* x, double tol, int krylovdim, int maxiter,
                    int eager, imps_krylov_info* info) {
  if (!E || !x0 || !x || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    const int64_t n = (int64_t)E->Dr[site] * E->Dr[site];
    return krylov_host(E->ctx, n, x0, x, [&](const imps::dcplx* a, imps::dcplx* b) {
      return imps::eigsolve_c(E->ctx, E, site, a, b, tol, krylovdim, maxiter, eager != 0);
    }, info);
  });
}

int imps_exponentiate_ac(imps_envs* E, const imps_mpo* mpo, int site, double dt_re, double dt_im, const double* x0,
                         double* x, double tol, int krylovdim, int maxiter, imps_krylov_info* info) {
  if (!E || !mpo || !x0 || !x || tol <= 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    const int64_t n = (int64_t)E->Dl[site] * mpo->sites[site % mpo->N].d * E->Dr[site];
    return krylov_host(E->ctx, n, x0, x, [&](const imps::dcplx* a, imps::dcplx* b) {
      return imps::expo_ac(E->ctx, E, mpo, site, imps::cplx(dt_re, dt_im), a, b, tol, krylovdim, maxiter);
    }, info);
  });
}

int imps_exponentiate_c(imps_envs* E, int site, double dt_re, double dt_im, const double* x0, double* x, double tol,
                        int krylovdim, int maxiter, imps_krylov_info* info) {
  if (!E || !x0 || !x || tol <= 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    check_site(E, site);
    const int64_t n = (int64_t)E->Dr[site] * E->Dr[site];
    return krylov_host(E->ctx, n, x0, x, [&](const imps::dcplx* a, imps::dcplx* b) {
      return imps::expo_c(E->ctx, E, site, imps::cplx(dt_re, dt_im), a, b, tol, krylovdim, maxiter);
    }, info);
  });
}

namespace {
__global__ void k_diag_apply(int64_t n, const double2* __restrict__ dv, const double2* __restrict__ x,
                             double2* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 a = dv[i], b = x[i];
    y[i] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
}
imps::LinOp diag_op(imps::Context* ctx, int64_t n, const imps::dcplx* dv) {
  return [ctx, n, dv](const imps::dcplx* x, imps::dcplx* y) {
    int g = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_diag_apply<<<std::max(g, 1), 256, 0, ctx->stream>>>(n, dv, x, y);
    ctx->n_kernels++;
  };
}
}  // namespace

int imps_linsolve_diag(imps_ctx* h, int64_t n, const double* dvals, const double* b, const double* x0, double a0,
                       double a1, double tol, int krylovdim, int maxiter, double* x, imps_krylov_info* info) {
  if (!h || !dvals || !b || !x0 || !x || n <= 0 || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    imps::DevBuf& dv = ctx->buf("diag_d", n * sizeof(imps::dcplx));
    imps::DevBuf& bd = ctx->buf("diag_b", n * sizeof(imps::dcplx));
    imps::DevBuf& xd = ctx->buf("diag_x", n * sizeof(imps::dcplx));
    imps::upload(ctx, dv.ptr, dvals, n * sizeof(imps::dcplx));
    imps::upload(ctx, bd.ptr, b, n * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, x0, n * sizeof(imps::dcplx));
    imps::KrylovResult r = imps::gmres(ctx, n, diag_op(ctx, n, dv.z()), bd.z(), xd.z(), tol, krylovdim, maxiter, a0, a1);
    imps::download(ctx, x, xd.ptr, n * sizeof(imps::dcplx));
    fill_info(info, r);
    return conv_status(r.converged);
  });
}

int imps_exponentiate_diag(imps_ctx* h, int64_t n, const double* dvals, double dt_re, double dt_im, const double* x0,
                           double* x, double tol, int krylovdim, int maxiter, imps_krylov_info* info) {
  if (!h || !dvals || !x0 || !x || n <= 0 || tol <= 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    imps::DevBuf& dv = ctx->buf("diag_d", n * sizeof(imps::dcplx));
    imps::DevBuf& xd = ctx->buf("diag_x", n * sizeof(imps::dcplx));
    imps::DevBuf& yd = ctx->buf("diag_b", n * sizeof(imps::dcplx));
    imps::upload(ctx, dv.ptr, dvals, n * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, x0, n * sizeof(imps::dcplx));
    imps::KrylovResult r = imps::exponentiate(ctx, n, diag_op(ctx, n, dv.z()), imps::cplx(dt_re, dt_im), xd.z(),
                                              yd.z(), tol, krylovdim, maxiter);
    imps::download(ctx, x, yd.ptr, n * sizeof(imps::dcplx));
    fill_info(info, r);
    return conv_status(r.converged);
  });
}

// ------------------------------------------------------------------ observables
int imps_galerkin(imps_envs* E, const imps_mpo* mpo, const imps_state* st, double* eps) {
  if (!E || !mpo || !st || !eps) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    *eps = imps::galerkin(E->ctx, E, mpo, st);
    return IMPS_OK;
  });
}

int imps_energy(imps_envs* E, const imps_mpo* mpo, imps_state* st, double* re, double* im) {
  if (!E || !mpo || !st) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::cplx e = imps::energy(E->ctx, E, mpo, st);
    if (re) *re = e.real();
    if (im) *im = e.imag();
    return IMPS_OK;
  });
}

int imps_local_expval(imps_state* st, int site, const double* O, double* re, double* im) {
  if (!st || !O) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    IMPS_REQUIRE(site >= 0 && site < st->N, IMPS_INVALID_ARG, "site index out of range");
    imps::cplx v = imps::local_expval(st->ctx, st, site, hc(O));
    if (re) *re = v.real();
    if (im) *im = v.imag();
    return IMPS_OK;
  });
}

// -------------------------------------------- dense-MPO channel and observables
int imps_dominant_env(imps_state* st, const imps_mpo* mpo, int side, double tol, int krylovdim, int maxiter,
                      double* lambda, double* L_host, imps_krylov_info* info) {
  if (!st || (side != 0 && side != 1)) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    imps::Context* ctx = st->ctx;
    const int D = st->Dl(0), w = mpo ? mpo->sites[0].m : 1;
    const size_t n = (size_t)D * w * D;
    imps::DevBuf& out = ctx->buf("abi_domenv", n * sizeof(imps::dcplx));
    imps::KrylovResult r = imps::dominant_env(ctx, st, mpo, side, tol, krylovdim, maxiter, out.z());
    if (lambda) {
      lambda[0] = r.value.real();
      lambda[1] = r.value.imag();
    }
    if (L_host) imps::download(ctx, L_host, out.ptr, n * sizeof(imps::dcplx));
    fill_info(info, r);
    return conv_status(r.converged);
  });
}

int imps_envs_build_dense(imps_envs* E, imps_state* st, const imps_mpo* mpo, double tol, int krylovdim,
                          int maxiter, imps_krylov_info* info) {
  if (!E || !st || !mpo) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::KrylovResult r = imps::envs_build_dense(E->ctx, E, st, mpo, tol, krylovdim, maxiter);
    fill_info(info, r);
    return conv_status(r.converged);
  });
}

int imps_energy_dense(imps_envs* E, const imps_mpo* mpo, imps_state* st, double* re, double* im) {
  if (!E || !mpo || !st) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::cplx e = imps::energy_dense(E->ctx, E, mpo, st);
    if (re) *re = e.real();
    if (im) *im = e.imag();
    return IMPS_OK;
  });
}

int imps_correlator(imps_state* st, const double* O1, const double* O2, int i, int nj, const int* js, double* out) {
  if (!st || !O1 || !O2 || !js || !out || nj <= 0) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    std::vector<int> jv(js, js + nj);
    std::vector<imps::cplx> g = imps::correlator(st->ctx, st, hc(O1), hc(O2), i, jv);
    for (int k = 0; k < nj; ++k) {
      out[2 * k] = g[k].real();
      out[2 * k + 1] = g[k].imag();
    }
    return IMPS_OK;
  });
}

int imps_svd(imps_ctx* h, int m, int n, const double* A, int kmax, double cutoff, double* U, double* s, double* V,
             int* k) {
  if (!h || !A || !U || !s || !V || !k || m <= 0 || n <= 0) return IMPS_INVALID_ARG;
  return guard(&h->c, [&] {
    imps::Context* ctx = &h->c;
    const int r = std::min(m, n);
    imps::DevBuf& Ad = ctx->buf("abi_svd_a", (size_t)m * n * sizeof(imps::dcplx));
    imps::DevBuf& Ud = ctx->buf("abi_svd_u", (size_t)m * r * sizeof(imps::dcplx));
    imps::DevBuf& Vd = ctx->buf("abi_svd_v", (size_t)n * r * sizeof(imps::dcplx));
    imps::upload(ctx, Ad.ptr, A, (size_t)m * n * sizeof(imps::dcplx));
    std::vector<double> sv;
    const int kk = imps::svd_thin(ctx, m, n, Ad.z(), m, kmax, cutoff, Ud.z(), sv, Vd.z());
    imps::download(ctx, U, Ud.ptr, (size_t)m * kk * sizeof(imps::dcplx));
    imps::download(ctx, V, Vd.ptr, (size_t)n * kk * sizeof(imps::dcplx));
    std::copy(sv.begin(), sv.end(), s);
    *k = kk;
    return IMPS_OK;
  });
}

int imps_entanglement_spectrum(imps_state* st, int bond, double* p) {
  if (!st || !p) return IMPS_INVALID_ARG;
  return guard(st->ctx, [&] {
    std::vector<double> v = imps::entanglement_spectrum(st->ctx, st, bond);
    std::copy(v.begin(), v.end(), p);
    return IMPS_OK;
  });
}

int imps_timeevompo_tensor(int m, int d, int n, const double* W, double delta_re, double delta_im, int alg,
                           double* out) {
  if (!W || !out) return IMPS_INVALID_ARG;
  return guard(nullptr, [&] {
    imps::timeevompo_site(m, d, n, hc(W), imps::cplx(delta_re, delta_im), alg, reinterpret_cast<imps::cplx*>(out));
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ gradients
int imps_energy_grad_mpo(imps_envs* E, const imps_mpo* mpo, imps_state* st, int site, double* G) {
  if (!E || !mpo || !st || !G) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    IMPS_REQUIRE(site >= 0 && site < st->N && st->N == E->N, IMPS_INVALID_ARG, "site index out of range");
    imps::energy_grad_mpo(E->ctx, E, mpo, st, site, reinterpret_cast<imps::cplx*>(G));
    return IMPS_OK;
  });
}

int imps_energy_grad_al(imps_envs* E, const imps_mpo* mpo, imps_state* st, int site, double* g) {
  if (!E || !mpo || !st || !g) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    IMPS_REQUIRE(site >= 0 && site < st->N && st->N == E->N, IMPS_INVALID_ARG, "site index out of range");
    imps::Context* ctx = E->ctx;
    const size_t n = st->site_elems(site);
    imps::DevBuf& gd = ctx->buf("grad_al_out", n * sizeof(imps::dcplx));
    imps::energy_grad_al(ctx, E, mpo, st, site, gd.z());
    imps::download(ctx, g, gd.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

// ------------------------------------------------------------------ algorithms
int imps_vumps_localupdate(imps_envs* E, const imps_mpo* mpo, imps_state* st, double tol, int krylovdim, int maxiter,
                           int eager, int32_t* ac_matvecs, int32_t* c_matvecs) {
  if (!E || !mpo || !st || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    int a = 0, c = 0;
    imps::vumps_localupdate(E->ctx, E, mpo, st, tol, krylovdim, maxiter, eager != 0, &a, &c);
    if (ac_matvecs) *ac_matvecs = a;
    if (c_matvecs) *c_matvecs = c;
    return IMPS_OK;
  });
}

int imps_vumps_iter(imps_envs* E, const imps_mpo* mpo, imps_state* st, int iter, double eps, imps_vumps_info* info) {
  if (!E || !mpo || !st || iter < 1) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps_vumps_info v = imps::vumps_iter(E->ctx, E, mpo, st, iter, eps);
    if (info) *info = v;
    return IMPS_OK;
  });
}

int imps_vumps_iter_batch(int n, imps_envs* const* envs, const imps_mpo* const* mpos, imps_state* const* states,
                          const int* iters, const double* eps, imps_vumps_info* infos, int* status, int nthreads) {
  if (n < 0 || (n > 0 && (!envs || !mpos || !states || !iters || !eps || !infos || !status))) return IMPS_INVALID_ARG;
  if (n == 0) return IMPS_OK;
  // instances that share a context run one after another on one host thread; distinct
  // contexts (distinct streams) run on concurrent host threads
  std::vector<imps::Context*> keys;
  std::vector<std::vector<int>> groups;
  for (int i = 0; i < n; ++i) {
    if (!envs[i] || !mpos[i] || !states[i]) return IMPS_INVALID_ARG;
    imps::Context* c = envs[i]->ctx;
    auto it = std::find(keys.begin(), keys.end(), c);
    if (it == keys.end()) {
      keys.push_back(c);
      groups.emplace_back();
      groups.back().push_back(i);
    } else {
      groups[it - keys.begin()].push_back(i);
    }
  }
  std::atomic<int> next{0};
  auto worker = [&] {
    for (int g = next.fetch_add(1); g < (int)groups.size(); g = next.fetch_add(1))
      for (int i : groups[g]) status[i] = imps_vumps_iter(envs[i], mpos[i], states[i], iters[i], eps[i], &infos[i]);
  };
  const int nt = std::max(1, std::min<int>(nthreads > 0 ? nthreads : 16, (int)groups.size()));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  int worst = IMPS_OK;
  for (int i = 0; i < n; ++i)
    if (status[i] < 0 && (worst >= 0 || status[i] < worst)) worst = status[i];
  return worst;
}

int imps_tdvp_step(imps_envs* E, const imps_mpo* mpo, imps_state* st, double dt_re, double dt_im, double tol,
                   int krylovdim, int maxiter, double gauge_tol, int gauge_maxiter, imps_krylov_info* info) {
  if (!E || !mpo || !st || tol <= 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::KrylovResult r = imps::tdvp_step(E->ctx, E, mpo, st, imps::cplx(dt_re, dt_im), tol, krylovdim, maxiter,
                                           gauge_tol, gauge_maxiter);
    fill_info(info, r);
    return conv_status(r.converged);
  });
}

int imps_idmrg_sweep(imps_envs* E, const imps_mpo* mpo, imps_state* st, double tol, int krylovdim, int maxiter,
                     int eager, double* Eout, double* eps) {
  if (!E || !mpo || !st || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::idmrg_sweep(E->ctx, E, mpo, st, tol, krylovdim, maxiter, eager != 0, Eout, eps);
    return IMPS_OK;
  });
}

int imps_idmrg2_sweep(imps_envs* E, const imps_mpo* mpo, imps_state* st, int D, double tol, int krylovdim,
                      int maxiter, int eager, double* Eout, double* eps) {
  if (!E || !mpo || !st || D <= 0 || tol < 0 || krylovdim <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::idmrg2_sweep(E->ctx, E, mpo, st, D, tol, krylovdim, maxiter, eager != 0, Eout, eps);
    return IMPS_OK;
  });
}

int imps_ac2_apply(imps_envs* E, const imps_mpo* mpo, int p, const double* x, double* y) {
  if (!E || !mpo || !x || !y || p < 0 || p >= E->N) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::Context* ctx = E->ctx;
    IMPS_REQUIRE(E->N >= 2, IMPS_INVALID_ARG, "two-site window needs unit cell length >= 2");
    const int q = (p + 1) % E->N;
    const size_t n = (size_t)E->Dl[p] * mpo->sites[p % mpo->N].d * mpo->sites[q % mpo->N].d * E->Dr[q];
    imps::DevBuf& xd = ctx->buf("abi_ac2_x", n * sizeof(imps::dcplx));
    imps::DevBuf& yd = ctx->buf("abi_ac2_y", n * sizeof(imps::dcplx));
    imps::upload(ctx, xd.ptr, x, n * sizeof(imps::dcplx));
    {
      imps::Fp64Scope fp64(ctx);
      imps::ac2_apply(ctx, E, mpo, p, xd.z(), yd.z());
    }
    imps::download(ctx, y, yd.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_state_bonds(const imps_state* st, int* chi) {
  if (!st || !chi) return IMPS_INVALID_ARG;
  for (int l = 0; l < st->N; ++l) chi[l] = st->chi[l];
  return IMPS_OK;
}

int imps_mult_guess(const imps_mpo* W, const imps_state* psi, int D, double tol, int maxiter, imps_state** out,
                    imps_gauge_info* info) {
  if (!W || !psi || !out || D <= 0 || maxiter <= 0) return IMPS_INVALID_ARG;
  *out = nullptr;
  return guard(psi->ctx, [&] {
    IMPS_REQUIRE(W->ctx == psi->ctx, IMPS_INVALID_ARG, "MPO and state belong to different contexts");
    imps::GaugeResult g;
    *out = imps::mult_guess(psi->ctx, W, psi, D, tol, maxiter, &g);
    fill_gauge(info, g);
    return conv_status(g.converged);
  });
}

int imps_mult_envs_create(imps_state* bra, const imps_mpo* W, const imps_state* ket, double tol, int maxiter,
                          imps_mult_envs** out, imps_krylov_info* info) {
  if (!bra || !W || !ket || !out || maxiter <= 0) return IMPS_INVALID_ARG;
  *out = nullptr;
  imps_mult_envs* E = new imps_mult_envs();
  int r = guard(bra->ctx, [&] {
    IMPS_REQUIRE(W->ctx == bra->ctx && ket->ctx == bra->ctx, IMPS_INVALID_ARG,
                 "MPO and states belong to different contexts");
    IMPS_REQUIRE(bra->N == ket->N && ket->N % W->N == 0, IMPS_DIM_MISMATCH,
                 "incompatible unit-cell lengths of MPS and MPO");
    for (int l = 0; l < ket->N; ++l) {
      const imps::MpoSite& Ws = W->sites[l % W->N];
      IMPS_REQUIRE(Ws.d == ket->d[l] && bra->d[l] == ket->d[l], IMPS_DIM_MISMATCH,
                   "MPO physical dimension != state physical dimension");
      IMPS_REQUIRE(Ws.n == W->sites[(l + 1) % W->N].m, IMPS_DIM_MISMATCH, "MPO bond chain mismatch");
    }
    E->ctx = bra->ctx;
    E->device = bra->device;
    E->N = bra->N;
    E->W = W;
    E->bra = bra;
    E->ket = ket;
    imps::mult_envs_allocate(E);
    imps::KrylovResult k = imps::mult_fixedpoints(E->ctx, E, tol, maxiter, false);
    fill_info(info, k);
    return conv_status(k.converged);
  });
  if (r != IMPS_OK && r != IMPS_NOT_CONVERGED) {
    delete E;
    return r;
  }
  *out = E;
  return r;
}

int imps_mult_envs_destroy(imps_mult_envs* E) {
  if (!E) return IMPS_OK;
  cudaSetDevice(E->device);
  cudaDeviceSynchronize();
  delete E;
  return IMPS_OK;
}

int imps_mult_envs_get(const imps_mult_envs* E, int side, int site, double* host) {
  if (!E || !host || site < 0 || site >= E->N || (side != 0 && side != 1)) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    const imps::DevBuf& b = side == 0 ? E->lefts[site] : E->rights[site];
    const imps::MpoSite& Ws = E->W->sites[site % E->W->N];
    const size_t n = side == 0 ? (size_t)E->bra->Dl(site) * Ws.m * E->ket->Dl(site)
                               : (size_t)E->ket->Dr(site) * Ws.n * E->bra->Dr(site);
    imps::download(E->ctx, host, b.ptr, n * sizeof(imps::dcplx));
    return IMPS_OK;
  });
}

int imps_mult_local_maps(imps_mult_envs* E, int site, double* ac, double* c) {
  if (!E || site < 0 || site >= E->N) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    imps::Context* ctx = E->ctx;
    imps::Fp64Scope fp64(ctx);
    const imps_state* bra = E->bra;
    const imps_state* ket = E->ket;
    const imps::MpoSite& Ws = E->W->sites[site % E->W->N];
    if (ac) {
      imps::DevBuf& y = ctx->buf("abi_mult_ac", bra->site_elems(site) * sizeof(imps::dcplx));
      imps::mult_ac(ctx, Ws, bra->Dl(site), ket->Dl(site), ket->Dr(site), bra->Dr(site), E->lefts[site].z(),
                    E->rights[site].z(), ket->AC[site].z(), y.z());
      imps::download(ctx, ac, y.ptr, bra->site_elems(site) * sizeof(imps::dcplx));
    }
    if (c) {
      imps::DevBuf& y = ctx->buf("abi_mult_c", bra->bond_elems(site) * sizeof(imps::dcplx));
      imps::mult_c(ctx, Ws.n, bra->Dr(site), ket->Dr(site), bra->Dr(site), E->lefts[(site + 1) % E->N].z(),
                   E->rights[site].z(), ket->C[site].z(), y.z());
      imps::download(ctx, c, y.ptr, bra->bond_elems(site) * sizeof(imps::dcplx));
    }
    return IMPS_OK;
  });
}

int imps_mult_galerkin(imps_mult_envs* E, double* eps) {
  if (!E || !eps) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    *eps = imps::mult_galerkin(E->ctx, E);
    return IMPS_OK;
  });
}

int imps_mult_sweep(imps_mult_envs* E, double gauge_tol, int gauge_maxiter, double env_tol, int env_maxiter,
                    double* eps) {
  if (!E || !eps || gauge_maxiter <= 0 || env_maxiter <= 0) return IMPS_INVALID_ARG;
  return guard(E->ctx, [&] {
    *eps = imps::mult_sweep(E->ctx, E, gauge_tol, gauge_maxiter, env_tol, env_maxiter);
    return IMPS_OK;
  });
}

}  // extern "C"
