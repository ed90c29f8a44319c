// C ABI of librest_b200.so: context, tensor producers and the REST-shaped
// vj/vk entry points (declared in include/rest_b200.h).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rest_b200.h"
#include "rijk_common.cuh"
#include "rijk_internal.h"

using rijk::Geom;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool pooled = false;  // from the stream-ordered pool (freed with cudaFreeAsync)
};

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
int64_t round_up(int64_t a, int64_t b) { return cdiv(a, b) * b; }

}  // namespace

struct rijk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Geom g;
  bool have = false;
  int64_t naux_pad = 0;
  double* dB = nullptr;
  size_t dB_bytes = 0;  // the current tensor's size
  size_t dB_cap = 0;    // the allocation's size (it only grows: a smaller tensor reuses it)
  int* d_err = nullptr;   // device-side wait timeouts
  int* d_info = nullptr;  // Cholesky failing pivot
  DevBuf stage, W, w, Jpart, Jw, Cw, X, Kpart, din, dout, docc, mV, mLinv, mT, mLinvd, mOut, Cr, Y, Yp;
  // split-precision (tcgen05) state: BF16 hi/lo copies of the tensor, operands, partials
  DevBuf tcBhi, tcBlo, tcVhi, tcVlo, tcXhi, tcXlo, tcPart;
  int64_t tensor_version = 0, tc_version = -1;
  size_t scratch_budget = (size_t)4 << 30;
  int ht_cfg = 1, rk_cfg = 1;  // CTA shapes of the K kernels (fastest measured on B200)
  bool pinned = false;         // scratch and tensor may not be (re)allocated or freed
  std::string last;
  // per-kernel-class event timers
  struct ProfRec {
    int cls;
    cudaEvent_t a, b;
  };
  bool prof = false;
  std::vector<ProfRec> prof_pending;
  std::vector<cudaEvent_t> ev_pool;
  double prof_ms[RIJK_PROF_NCLASS] = {};
  int64_t prof_n[RIJK_PROF_NCLASS] = {};
};

namespace {

cudaEvent_t ev_get(rijk_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Brackets the launches issued in its scope with events when profiling is on.
struct ProfScope {
  rijk_ctx* c;
  int cls;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  ProfScope(rijk_ctx* c_, int cls_, cudaStream_t st_) : c(c_), cls(cls_), st(st_) {
    if (c->prof) {
      a = ev_get(c);
      cudaEventRecord(a, st);
    }
  }
  ~ProfScope() {
    if (c->prof && a) {
      cudaEvent_t b = ev_get(c);
      cudaEventRecord(b, st);
      c->prof_pending.push_back({cls, a, b});
    }
  }
};

}  // namespace

namespace {

int set_err(rijk_ctx* c, int code, const std::string& msg) {
  if (c) c->last = msg;
  return code;
}

int cuda_fail(rijk_ctx* c, cudaError_t e, const char* what) {
  return set_err(c, RIJK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RIJK_CK(call)                                         \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);  \
  } while (0)

void free_buf(rijk_ctx* ctx, DevBuf& b) {
  if (b.p) {
    if (b.pooled)
      cudaFreeAsync(b.p, ctx->stream);
    else
      cudaFree(b.p);
  }
  b.p = nullptr;
  b.bytes = 0;
  b.pooled = false;
}

// Frees the scratch only the metric step and the fit use (once per geometry):
// the metric, its factor and inverse, the fit's output panel and large staging.
// They come from the stream-ordered pool, so the frees are ordered after the
// fit on the context's stream and need no device synchronisation.
int release_fit_scratch(rijk_ctx* ctx) {
  if (ctx->pinned) return RIJK_OK;
  for (DevBuf* b : {&ctx->mV, &ctx->mLinv, &ctx->mT, &ctx->mLinvd, &ctx->mOut}) free_buf(ctx, *b);
  if (ctx->stage.bytes > ((size_t)256 << 20)) free_buf(ctx, ctx->stage);
  return RIJK_OK;
}

int ensure(rijk_ctx* ctx, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return RIJK_OK;
  if (ctx->pinned)
    return set_err(ctx, RIJK_ERR_TOO_LARGE,
                   "buffers are pinned: this call needs " + std::to_string(bytes) + " bytes of scratch");
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, RIJK_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  b.bytes = bytes;
  return RIJK_OK;
}

// Scratch used only by work on the context's own stream (staging, metric and
// fit buffers) comes from the device's stream-ordered pool: allocation and
// release are ordered on that stream, and the pool keeps freed memory for the
// next geometry instead of unmapping it.
int ensure_pooled(rijk_ctx* ctx, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return RIJK_OK;
  if (ctx->pinned)
    return set_err(ctx, RIJK_ERR_TOO_LARGE,
                   "buffers are pinned: this call needs " + std::to_string(bytes) + " bytes of scratch");
  free_buf(ctx, b);
  cudaError_t e = cudaMallocAsync(&b.p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return set_err(ctx, RIJK_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  b.bytes = bytes;
  b.pooled = true;
  return RIJK_OK;
}

#define RIJK_TRY(x)               \
  do {                            \
    int r_ = (x);                 \
    if (r_ != RIJK_OK) return r_; \
  } while (0)

cudaStream_t pick(rijk_ctx* ctx, void* s) { return s ? static_cast<cudaStream_t>(s) : ctx->stream; }

// Launch errors are reported immediately; device-side timeouts at the next sync.
int after_launch(rijk_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  return RIJK_OK;
}

int sync_and_check(rijk_ctx* ctx, cudaStream_t st) {
  RIJK_CK(cudaStreamSynchronize(st));
  int h = 0;
  RIJK_CK(cudaMemcpy(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    RIJK_CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
    if (h == rijk::DEV_NONFINITE)
      return set_err(ctx, RIJK_ERR_NONFINITE, "a density, orbital or occupation element read was NaN or Inf");
    if (h == rijk::DEV_TENSOR_MAP)
      return set_err(ctx, RIJK_ERR_CUDA, "a tensor map of the split exchange could not be encoded");
    return set_err(ctx, RIJK_ERR_TIMEOUT, "a device-side wait exceeded its time budget");
  }
  return RIJK_OK;
}

int check_spin(rijk_ctx* ctx, int spin) {
  if (spin != 1 && spin != 2) return set_err(ctx, RIJK_ERR_ARG, "spin_channel must be 1 or 2");
  return RIJK_OK;
}

int need_tensor(rijk_ctx* ctx) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!ctx->have) return set_err(ctx, RIJK_ERR_NO_TENSOR, "no fitted tensor loaded");
  RIJK_CK(cudaSetDevice(ctx->device));
  return RIJK_OK;
}

// Allocate the tile-packed tensor for (n, naux); pad rows are zero.
int alloc_tensor(rijk_ctx* ctx, int64_t n, int64_t naux) {
  if (n <= 0 || naux <= 0) return set_err(ctx, RIJK_ERR_ARG, "num_basis and num_auxbas must be positive");
  if (ctx->pinned) return set_err(ctx, RIJK_ERR_ARG, "buffers are pinned: no new tensor can be loaded");
  if (n > 46000) return set_err(ctx, RIJK_ERR_TOO_LARGE, "num_basis above 46000");
  Geom g = rijk::make_geom(n, naux);
  const int64_t naux_pad = round_up(naux, rijk::TS);
  const size_t bytes = (size_t)naux_pad * g.ldB * sizeof(double);
  if (ctx->dB && ctx->dB_cap < bytes) {
    cudaFree(ctx->dB);
    ctx->dB = nullptr;
    ctx->dB_bytes = ctx->dB_cap = 0;
  }
  if (!ctx->dB) {
    cudaError_t e = cudaMalloc(&ctx->dB, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      ctx->dB = nullptr;
      ctx->have = false;
      return set_err(ctx, RIJK_ERR_NOMEM, "tensor allocation of " + std::to_string(bytes) + " bytes failed");
    }
    ctx->dB_cap = bytes;
  }
  ctx->dB_bytes = bytes;
  if (naux_pad > naux)
    RIJK_CK(cudaMemsetAsync(ctx->dB + naux * g.ldB, 0, (size_t)(naux_pad - naux) * g.ldB * sizeof(double),
                            ctx->stream));
  ctx->g = g;
  ctx->naux_pad = naux_pad;
  ctx->g.ht_cfg = ctx->ht_cfg;
  ctx->g.rk_cfg = ctx->rk_cfg;
  ctx->tensor_version++;
  ctx->have = false;
  return RIJK_OK;
}

// Upload a host tensor (rimatr rows of npair, or ri3fn blocks of n*n) in chunks.
int upload_tensor(rijk_ctx* ctx, const double* host, int64_t n, int64_t naux, int kind) {
  RIJK_CK(cudaSetDevice(ctx->device));
  RIJK_TRY(alloc_tensor(ctx, n, naux));
  const Geom& g = ctx->g;
  const int64_t row = kind == 0 ? g.npair : n * n;
  const int64_t rows_per = std::max<int64_t>(1, std::min<int64_t>(naux, ((int64_t)256 << 20) / (row * 8)));
  RIJK_TRY(ensure_pooled(ctx, ctx->stage, (size_t)rows_per * row * 8));
  double* st = static_cast<double*>(ctx->stage.p);
  for (int64_t p0 = 0; p0 < naux; p0 += rows_per) {
    const int64_t np = std::min(rows_per, naux - p0);
    RIJK_CK(cudaMemcpyAsync(st, host + p0 * row, (size_t)np * row * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (kind == 0)
      rijk::launch_pack_rimatr(g, st, np, ctx->dB + p0 * g.ldB, ctx->stream);
    else
      rijk::launch_pack_ri3fn(g, st, np, ctx->dB + p0 * g.ldB, ctx->stream);
    RIJK_TRY(after_launch(ctx, "pack tensor"));
  }
  RIJK_TRY(sync_and_check(ctx, ctx->stream));
  ctx->have = true;
  return RIJK_OK;
}

int upload_square_padded(rijk_ctx* ctx, const double* host, int64_t n, int64_t np, DevBuf& dst) {
  RIJK_TRY(ensure_pooled(ctx, ctx->stage, (size_t)n * n * 8));
  RIJK_TRY(ensure_pooled(ctx, dst, (size_t)np * np * 8));
  RIJK_CK(cudaMemcpyAsync(ctx->stage.p, host, (size_t)n * n * 8, cudaMemcpyHostToDevice, ctx->stream));
  rijk::launch_pad_matrix(static_cast<double*>(ctx->stage.p), n, np, static_cast<double*>(dst.p), ctx->stream);
  return after_launch(ctx, "pad metric");
}

}  // namespace

namespace rijk {
void launch_fit_copy_back(const double* out, int64_t kc, double* dB, int64_t ldB, int64_t k0, int64_t rows,
                          cudaStream_t st);
}

namespace {

// B <- B * F (F = L^-T with klim upper, or a dense factor), chunked over the
// stored columns k so that the product never overwrites its own input.
int fit_in_place(rijk_ctx* ctx, const double* dF, int64_t ldf, int tb, int klim) {
  const Geom& g = ctx->g;
  const int64_t np = ctx->naux_pad;
  int64_t chunk = std::max<int64_t>(1024, (((int64_t)512 << 20) / (np * 8)) / 1024 * 1024);
  chunk = std::min(chunk, g.ldB);
  RIJK_TRY(ensure_pooled(ctx, ctx->mOut, (size_t)chunk * np * 8));
  double* out = static_cast<double*>(ctx->mOut.p);
  for (int64_t k0 = 0; k0 < g.ldB; k0 += chunk) {
    const int64_t kc = std::min(chunk, g.ldB - k0);
    rijk::launch_dgemm(kc, np, np, 1.0, ctx->dB + k0, g.ldB, 0, dF, ldf, tb, 0.0, out, kc, klim, 0, 1, 0, 0, 0,
                       ctx->d_err, ctx->stream);
    RIJK_TRY(after_launch(ctx, "fit gemm"));
    rijk::launch_fit_copy_back(out, kc, ctx->dB, g.ldB, k0, np, ctx->stream);
    RIJK_TRY(after_launch(ctx, "fit copy"));
  }
  ctx->tensor_version++;
  return RIJK_OK;
}

// ---- J ----------------------------------------------------------------------
int vj_dev(rijk_ctx* ctx, const double* d_dm, int spin, double scale, int mode, int out_kind, double* d_out,
           cudaStream_t st) {
  const Geom& g = ctx->g;
  const int splits = rijk::j_pass2_splits(g);
  RIJK_TRY(ensure(ctx, ctx->W, (size_t)spin * g.ldB * 8));
  RIJK_TRY(ensure(ctx, ctx->w, (size_t)spin * g.naux * 8));
  RIJK_TRY(ensure(ctx, ctx->Jpart, (size_t)splits * spin * g.ldB * 8));
  double* W = static_cast<double*>(ctx->W.p);
  double* w = static_cast<double*>(ctx->w.p);
  double* Jp = static_cast<double*>(ctx->Jpart.p);
  {
    ProfScope ps(ctx, RIJK_PROF_J_OTHER, st);
    rijk::launch_j_weights(g, d_dm, spin, mode, W, ctx->d_err, st);
  }
  {
    ProfScope ps(ctx, RIJK_PROF_J_PASS1, st);
    rijk::launch_j_pass1(g, ctx->dB, W, spin, w, st);
  }
  {
    ProfScope ps(ctx, RIJK_PROF_J_PASS2, st);
    rijk::launch_j_pass2(g, ctx->dB, w, spin, splits, Jp, st);
  }
  {
    ProfScope ps(ctx, RIJK_PROF_J_OTHER, st);
    rijk::launch_j_finalize(g, Jp, spin, splits, scale, out_kind, d_out, st);
  }
  return after_launch(ctx, "vj");
}

// ---- K, occupied-orbital form (and J from the same half-transform) -------------
// d_vj != nullptr: J of the densities D_s = C_s diag(occ_s) C_s^T as well.  The
// half-transform's epilogue reduces w_P,s = <C_s diag(sqrt occ), X_P,s> =
// B_P : D_s, which replaces J's first pass over the tensor; J's second pass
// and finalisation follow the K chunks.
int vk_occ_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo, const double* d_occ,
               int spin, double scale, double* d_out, cudaStream_t st, double j_scale = 0.0,
               double* d_vj = nullptr) {
  const Geom& g = ctx->g;
  int64_t nw[2] = {0, 0};
  for (int s = 0; s < spin; ++s) {
    nw[s] = homo[s] + 1;
    if (homo[s] < 0 || nw[s] > num_state) return set_err(ctx, RIJK_ERR_ARG, "homo out of range");
  }
  const int64_t ldx = round_up(g.n, 128);
  const int64_t coff[2] = {0, round_up(nw[0], rijk::TS)};
  const int64_t ocols_valid = spin == 2 ? coff[1] + nw[1] : nw[0];
  const int64_t ocols = round_up(ocols_valid, 128);  // a multiple of every half-transform CTA width
  RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ldx * ocols * 8));
  double* Cw = static_cast<double*>(ctx->Cw.p);
  {
    ProfScope ps(ctx, RIJK_PROF_K_OTHER, st);
    rijk::launch_k_prepare_c(g, d_eigv, g.n, g.n * num_state, d_occ, num_state, nw, spin, ldx, ocols, Cw, ctx->d_err,
                             st);
  }
  // X holds, per spin, the chunk's X_p back to back without padding (column
  // p nw + i), spin beta after spin alpha, and 32 spare columns for the rank
  // update's last k tile
  const int64_t xcols = nw[0] + (spin == 2 ? nw[1] : 0);
  const int64_t per_p = ldx * xcols * 8;
  const int64_t pchunk = std::max<int64_t>(1, std::min<int64_t>(g.naux, (int64_t)ctx->scratch_budget / per_p));
  RIJK_TRY(ensure(ctx, ctx->X, (size_t)(pchunk * xcols + rijk::TS) * ldx * 8));
  const int splits_max = rijk::k_rank_splits(g, pchunk, 0);
  RIJK_TRY(ensure(ctx, ctx->Kpart, (size_t)splits_max * rijk::k_block_pairs(g, 0) * 128 * 128 * 8));
  double* X = static_cast<double*>(ctx->X.p);
  double* Kp = static_cast<double*>(ctx->Kpart.p);
  double *jw = nullptr, *w = nullptr;
  int jsplits = 0;
  if (d_vj) {
    jsplits = rijk::j_pass2_splits(g);
    RIJK_TRY(ensure(ctx, ctx->Jw, (size_t)rijk::half_transform_warps(g, pchunk, ldx, ocols) * 2 * 8));
    RIJK_TRY(ensure(ctx, ctx->w, (size_t)spin * g.naux * 8));
    RIJK_TRY(ensure(ctx, ctx->Jpart, (size_t)jsplits * spin * g.ldB * 8));
    jw = static_cast<double*>(ctx->Jw.p);
    w = static_cast<double*>(ctx->w.p);
  }
  for (int64_t p0 = 0; p0 < g.naux; p0 += pchunk) {
    const int64_t np = std::min(pchunk, g.naux - p0);
    const rijk::XMap xm{nw[0], (int)nw[0], (int)coff[1], spin == 2 ? (int)nw[1] : 0, np * nw[0], nw[1]};
    {
      ProfScope ps(ctx, RIJK_PROF_K_HALF, st);
      rijk::launch_half_transform(g, ctx->dB, p0, np, Cw, ldx, ocols, ocols_valid, X, ldx, xm, ctx->d_err, st, jw, w,
                                  spin, spin == 2 ? (int)coff[1] : 1 << 30);
    }
    for (int s = 0; s < spin; ++s) {
      if (nw[s] == 0) continue;
      const int splits = rijk::k_rank_splits(g, np, 0);
      {
        ProfScope ps(ctx, RIJK_PROF_K_RANK, st);
        rijk::launch_k_rank_update(g, X + (s == 0 ? 0 : np * nw[0]) * ldx, ldx, np, nw[s], splits, 0, Kp,
                                   ctx->d_err, st);
      }
      ProfScope ps(ctx, RIJK_PROF_K_OTHER, st);
      rijk::launch_k_finalize(g, Kp, splits, 0, scale, p0 > 0 ? 1 : 0, 0, d_out + s * g.npair, st);
    }
  }
  if (d_vj) {
    double* Jp = static_cast<double*>(ctx->Jpart.p);
    {
      ProfScope ps(ctx, RIJK_PROF_J_PASS2, st);
      rijk::launch_j_pass2(g, ctx->dB, w, spin, jsplits, Jp, st);
    }
    ProfScope ps(ctx, RIJK_PROF_J_OTHER, st);
    rijk::launch_j_finalize(g, Jp, spin, jsplits, j_scale, 0, d_vj, st);
  }
  return after_launch(ctx, d_vj ? "vjk occ" : "vk occ");
}

// ---- K, density form ----------------------------------------------------------
int vk_dm_dev(rijk_ctx* ctx, const double* d_dm, int spin, double scale, int full, double* d_out, cudaStream_t st) {
  const Geom& g = ctx->g;
  const int64_t ldx = round_up(g.n, 128);
  RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ldx * ldx * 8));
  double* Dp = static_cast<double*>(ctx->Cw.p);
  const int64_t per_p = ldx * ldx * 8;
  const int64_t pchunk = std::max<int64_t>(1, std::min<int64_t>(g.naux, (int64_t)ctx->scratch_budget / per_p));
  RIJK_TRY(ensure(ctx, ctx->X, (size_t)pchunk * per_p));
  const int splits_max = rijk::k_rank_splits(g, pchunk, full);
  RIJK_TRY(ensure(ctx, ctx->Kpart, (size_t)splits_max * rijk::k_block_pairs(g, full) * 128 * 128 * 8));
  double* T = static_cast<double*>(ctx->X.p);
  double* Kp = static_cast<double*>(ctx->Kpart.p);
  const int64_t per_out = full ? g.n * g.n : g.npair;
  for (int s = 0; s < spin; ++s) {
    {
      ProfScope ps(ctx, RIJK_PROF_K_OTHER, st);
      rijk::launch_pad_square(d_dm + s * g.n * g.n, g.n, g.n, ldx, Dp, ctx->d_err, st);
    }
    for (int64_t p0 = 0; p0 < g.naux; p0 += pchunk) {
      const int64_t np = std::min(pchunk, g.naux - p0);
      {
        ProfScope ps(ctx, RIJK_PROF_K_HALF, st);
        rijk::launch_half_transform(g, ctx->dB, p0, np, Dp, ldx, ldx, g.n, T, ldx, rijk::XMap::dense(ldx),
                                    ctx->d_err, st);
      }
      const int splits = rijk::k_rank_splits(g, np, full);
      {
        ProfScope ps(ctx, RIJK_PROF_K_DM, st);
        rijk::launch_k_dm_update(g, T, ldx, ldx * ldx, ctx->dB, p0, np, splits, full, Kp, ctx->d_err, st);
      }
      ProfScope ps(ctx, RIJK_PROF_K_OTHER, st);
      rijk::launch_k_finalize(g, Kp, splits, full, scale, p0 > 0 ? 1 : 0, full ? 1 : 0, d_out + s * per_out, st);
    }
  }
  return after_launch(ctx, "vk dm");
}

// Host-pointer wrapper: copy inputs in, run, copy the result out, synchronise.
template <class F>
int host_call(rijk_ctx* ctx, const double* h_in, size_t in_doubles, double* h_out, size_t out_doubles, F&& body) {
  RIJK_TRY(ensure(ctx, ctx->din, in_doubles * 8));
  RIJK_TRY(ensure(ctx, ctx->dout, out_doubles * 8));
  double* din = static_cast<double*>(ctx->din.p);
  double* dout = static_cast<double*>(ctx->dout.p);
  RIJK_CK(cudaMemcpyAsync(din, h_in, in_doubles * 8, cudaMemcpyHostToDevice, ctx->stream));
  RIJK_TRY(body(din, dout));
  RIJK_CK(cudaMemcpyAsync(h_out, dout, out_doubles * 8, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx, ctx->stream);
}

}  // namespace

// ============================================================================
// extern "C"
// ============================================================================
extern "C" {

const char* rijk_status_string(int status) {
  switch (status) {
    case RIJK_OK: return "ok";
    case RIJK_ERR_ARG: return "invalid argument";
    case RIJK_ERR_CUDA: return "CUDA error";
    case RIJK_ERR_NOT_SPD: return "metric is not positive definite";
    case RIJK_ERR_NO_TENSOR: return "no fitted tensor loaded";
    case RIJK_ERR_TIMEOUT: return "device-side wait timed out";
    case RIJK_ERR_NOMEM: return "device out of memory";
    case RIJK_ERR_NONFINITE: return "non-finite input";
    case RIJK_ERR_TOO_LARGE: return "size above the supported maximum";
    default: return "unknown status";
  }
}

namespace {
// The stream-ordered pool returns freed memory to the system at every
// synchronisation unless told otherwise; let it keep up to 8 GiB for this
// process so that the next geometry's scratch comes back without new mappings.
void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), device) != done.end()) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = (uint64_t)8 << 30;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done.push_back(device);
}
}  // namespace

int rijk_ctx_create(int device, rijk_ctx** out) {
  if (!out) return RIJK_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return RIJK_ERR_CUDA;
  }
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) return RIJK_ERR_CUDA;
  if (major != 10) return RIJK_ERR_CUDA;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return RIJK_ERR_CUDA;
  rijk_ctx* c = new rijk_ctx();
  c->device = device;
  if (const char* s = getenv("RIJK_HT_CFG")) c->ht_cfg = std::max(0, std::min(RIJK_TILE_CFGS - 1, atoi(s)));
  if (const char* s = getenv("RIJK_RK_CFG")) c->rk_cfg = std::max(0, std::min(RIJK_TILE_CFGS - 1, atoi(s)));
  if (const char* s = getenv("RIJK_SCRATCH_BYTES")) {
    const long long v = atoll(s);
    if (v > (1 << 20)) c->scratch_budget = (size_t)v;
  }
  keep_pool_memory(device);
  // the error flag, the Cholesky pivot and the wait budget share one
  // allocation (d_err owns it; layout in rijk_common.cuh, ERR_WORDS)
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&c->d_err, rijk::ERR_WORDS * sizeof(int)) == cudaSuccess;
  if (ok) {
    c->d_info = c->d_err + 1;
    ok = cudaMemsetAsync(c->d_err, 0, rijk::ERR_WORDS * sizeof(int), c->stream) == cudaSuccess &&
         cudaStreamSynchronize(c->stream) == cudaSuccess;
  }
  if (!ok) {
    rijk_ctx_destroy(c);
    return RIJK_ERR_CUDA;
  }
  *out = c;
  return RIJK_OK;
}

int rijk_ctx_destroy(rijk_ctx* ctx) {
  if (!ctx) return RIJK_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[] = {&ctx->stage, &ctx->W,   &ctx->w,    &ctx->Jpart, &ctx->Cw,    &ctx->X,      &ctx->Kpart, &ctx->din,
                    &ctx->dout,  &ctx->docc, &ctx->mV, &ctx->mLinv, &ctx->mT, &ctx->mLinvd, &ctx->mOut,
                    &ctx->Cr,    &ctx->Y,    &ctx->Yp, &ctx->tcBhi, &ctx->tcBlo, &ctx->tcVhi, &ctx->tcVlo,
                    &ctx->tcXhi, &ctx->tcXlo, &ctx->tcPart, &ctx->Jw};
  for (DevBuf* b : bufs) free_buf(ctx, *b);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& r : ctx->prof_pending) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->dB) cudaFree(ctx->dB);
  if (ctx->d_err) cudaFree(ctx->d_err);  // d_info lives in the same allocation
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return RIJK_OK;
}

const char* rijk_ctx_last_error(const rijk_ctx* ctx) { return ctx ? ctx->last.c_str() : "null context"; }

int rijk_ctx_info(const rijk_ctx* ctx, int64_t* num_basis, int64_t* num_auxbas, int64_t* tensor_bytes) {
  if (!ctx) return RIJK_ERR_ARG;
  if (num_basis) *num_basis = ctx->have ? ctx->g.n : 0;
  if (num_auxbas) *num_auxbas = ctx->have ? ctx->g.naux : 0;
  if (tensor_bytes) *tensor_bytes = ctx->have ? (int64_t)ctx->dB_bytes : 0;
  return RIJK_OK;
}

void* rijk_ctx_stream(rijk_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t rijk_kernel_launches(void) { return rijk::launch_count(); }

int rijk_ctx_pin_buffers(rijk_ctx* ctx, int pinned) {
  if (!ctx) return RIJK_ERR_ARG;
  ctx->pinned = pinned != 0;
  return RIJK_OK;
}

int rijk_ctx_set_wait_budget(rijk_ctx* ctx, int64_t nanoseconds) {
  if (!ctx) return RIJK_ERR_ARG;
  if (nanoseconds != 0 && (nanoseconds < 10000000 || nanoseconds > 600000000000LL))
    return set_err(ctx, RIJK_ERR_ARG, "wait budget must be 0 (default) or between 10 ms and 600 s");
  RIJK_CK(cudaSetDevice(ctx->device));
  const uint64_t v = (uint64_t)nanoseconds;
  RIJK_CK(cudaMemcpyAsync(ctx->d_err + 2, &v, sizeof(v), cudaMemcpyHostToDevice, ctx->stream));
  RIJK_CK(cudaStreamSynchronize(ctx->stream));
  return RIJK_OK;
}

int rijk_ctx_selftest_timeout(rijk_ctx* ctx) {
  if (!ctx) return RIJK_ERR_ARG;
  RIJK_CK(cudaSetDevice(ctx->device));
  rijk::launch_wait_selftest(ctx->d_err, ctx->stream);
  RIJK_TRY(after_launch(ctx, "wait self-test"));
  return sync_and_check(ctx, ctx->stream);
}

int rijk_ctx_get_tiles(const rijk_ctx* ctx, int* half_transform_cfg, int* update_cfg) {
  if (!ctx || !half_transform_cfg || !update_cfg) return RIJK_ERR_ARG;
  *half_transform_cfg = ctx->ht_cfg;
  *update_cfg = ctx->rk_cfg;
  return RIJK_OK;
}

int rijk_ctx_set_tiles(rijk_ctx* ctx, int half_transform_cfg, int update_cfg) {
  if (!ctx || half_transform_cfg < 0 || half_transform_cfg >= RIJK_TILE_CFGS || update_cfg < 0 ||
      update_cfg >= RIJK_TILE_CFGS)
    return set_err(ctx, RIJK_ERR_ARG, "tile configuration out of range");
  ctx->ht_cfg = ctx->g.ht_cfg = half_transform_cfg;
  ctx->rk_cfg = ctx->g.rk_cfg = update_cfg;
  return RIJK_OK;
}

int rijk_ctx_autotune(rijk_ctx* ctx, int64_t ncols, int64_t sample_rows, int* best_half, int* best_update,
                      double* ms_out) {
  RIJK_TRY(need_tensor(ctx));
  if (ncols <= 0) return set_err(ctx, RIJK_ERR_ARG, "ncols must be positive");
  Geom g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int64_t np = std::max<int64_t>(1, std::min<int64_t>(g.naux, sample_rows > 0 ? sample_rows : 512));
  const int64_t ldx = round_up(g.n, 128);
  const int64_t ocols = round_up(ncols, 128);
  RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ldx * ocols * 8));
  RIJK_TRY(ensure(ctx, ctx->X, (size_t)(np * ncols + rijk::TS) * ldx * 8));
  // any non-zero operand times the same as the real one: fill C with a constant
  std::vector<double> ones((size_t)ldx * ocols, 0.0);
  for (int64_t c = 0; c < ncols; ++c)
    for (int64_t r = 0; r < g.n; ++r) ones[r + ldx * c] = 1.0 / (1.0 + (double)((r + c) % 7));
  RIJK_CK(cudaMemcpyAsync(ctx->Cw.p, ones.data(), ones.size() * 8, cudaMemcpyHostToDevice, st));
  cudaEvent_t a, b;
  RIJK_CK(cudaEventCreate(&a));
  RIJK_CK(cudaEventCreate(&b));
  double best_ht_ms = 1e30, best_rk_ms = 1e30;
  int bh = ctx->ht_cfg, br = ctx->rk_cfg;
  for (int cfg = 0; cfg < RIJK_TILE_CFGS; ++cfg) {
    g.ht_cfg = cfg;
    g.rk_cfg = cfg;
    const int splits = rijk::k_rank_splits(g, np, 0);
    RIJK_TRY(ensure(ctx, ctx->Kpart, (size_t)splits * rijk::k_block_pairs(g, 0) * 128 * 128 * 8));
    float t_ht = 0.f, t_rk = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // first repetition warms up
      RIJK_CK(cudaEventRecord(a, st));
      rijk::launch_half_transform(g, ctx->dB, 0, np, static_cast<double*>(ctx->Cw.p), ldx, ocols, ncols,
                                  static_cast<double*>(ctx->X.p), ldx, rijk::XMap{ncols, (int)ncols, 0, 0, 0, 0},
                                  ctx->d_err, st);
      RIJK_CK(cudaEventRecord(b, st));
      RIJK_CK(cudaEventSynchronize(b));
      RIJK_CK(cudaEventElapsedTime(&t_ht, a, b));
      RIJK_CK(cudaEventRecord(a, st));
      rijk::launch_k_rank_update(g, static_cast<double*>(ctx->X.p), ldx, np, ncols, splits, 0,
                                 static_cast<double*>(ctx->Kpart.p), ctx->d_err, st);
      RIJK_CK(cudaEventRecord(b, st));
      RIJK_CK(cudaEventSynchronize(b));
      RIJK_CK(cudaEventElapsedTime(&t_rk, a, b));
    }
    RIJK_TRY(after_launch(ctx, "autotune"));
    if (ms_out) {
      ms_out[2 * cfg] = t_ht;
      ms_out[2 * cfg + 1] = t_rk;
    }
    if (t_ht < best_ht_ms) {
      best_ht_ms = t_ht;
      bh = cfg;
    }
    if (t_rk < best_rk_ms) {
      best_rk_ms = t_rk;
      br = cfg;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  RIJK_TRY(sync_and_check(ctx, st));
  ctx->ht_cfg = ctx->g.ht_cfg = bh;
  ctx->rk_cfg = ctx->g.rk_cfg = br;
  if (best_half) *best_half = bh;
  if (best_update) *best_update = br;
  return RIJK_OK;
}

int rijk_ctx_profile(rijk_ctx* ctx, int enable) {
  if (!ctx) return RIJK_ERR_ARG;
  ctx->prof = enable != 0;
  return RIJK_OK;
}

int rijk_ctx_profile_read(rijk_ctx* ctx, double* ms, int64_t* launches) {
  if (!ctx) return RIJK_ERR_ARG;
  RIJK_CK(cudaSetDevice(ctx->device));
  for (auto& r : ctx->prof_pending) {
    RIJK_CK(cudaEventSynchronize(r.b));
    float t = 0.f;
    RIJK_CK(cudaEventElapsedTime(&t, r.a, r.b));
    ctx->prof_ms[r.cls] += t;
    ctx->prof_n[r.cls] += 1;
    ctx->ev_pool.push_back(r.a);
    ctx->ev_pool.push_back(r.b);
  }
  ctx->prof_pending.clear();
  for (int i = 0; i < RIJK_PROF_NCLASS; ++i) {
    if (ms) ms[i] = ctx->prof_ms[i];
    if (launches) launches[i] = ctx->prof_n[i];
    ctx->prof_ms[i] = 0.0;
    ctx->prof_n[i] = 0;
  }
  return RIJK_OK;
}

int rijk_ctx_tensor(rijk_ctx* ctx, const double** d_tensor, int64_t* row_stride) {
  RIJK_TRY(need_tensor(ctx));
  if (d_tensor) *d_tensor = ctx->dB;
  if (row_stride) *row_stride = ctx->g.ldB;
  return RIJK_OK;
}

int rijk_ctx_synchronize(rijk_ctx* ctx, void* stream) {
  if (!ctx) return RIJK_ERR_ARG;
  RIJK_CK(cudaSetDevice(ctx->device));
  return sync_and_check(ctx, pick(ctx, stream));
}

int rijk_set_rimatr(rijk_ctx* ctx, const double* rimatr, int64_t num_basis, int64_t num_auxbas) {
  if (!ctx || !rimatr) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  return upload_tensor(ctx, rimatr, num_basis, num_auxbas, 0);
}

int rijk_set_ri3fn(rijk_ctx* ctx, const double* ri3fn, int64_t num_basis, int64_t num_auxbas) {
  if (!ctx || !ri3fn) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  return upload_tensor(ctx, ri3fn, num_basis, num_auxbas, 1);
}

int rijk_tensor_alloc(rijk_ctx* ctx, int64_t num_basis, int64_t num_auxbas) {
  if (!ctx) return RIJK_ERR_ARG;
  RIJK_CK(cudaSetDevice(ctx->device));
  RIJK_TRY(alloc_tensor(ctx, num_basis, num_auxbas));
  RIJK_CK(cudaMemsetAsync(ctx->dB, 0, ctx->dB_bytes, ctx->stream));
  RIJK_TRY(sync_and_check(ctx, ctx->stream));
  ctx->have = true;
  return RIJK_OK;
}

int rijk_tensor_load_rows_dev(rijk_ctx* ctx, const double* d_rows, int64_t p0, int64_t np, int layout,
                              void* stream) {
  RIJK_TRY(need_tensor(ctx));
  if (!d_rows || p0 < 0 || np <= 0 || p0 + np > ctx->g.naux || (layout != 0 && layout != 1))
    return set_err(ctx, RIJK_ERR_ARG, "bad row range or layout");
  ctx->tensor_version++;
  if (layout == 0)
    rijk::launch_pack_rimatr(ctx->g, d_rows, np, ctx->dB + p0 * ctx->g.ldB, pick(ctx, stream));
  else
    rijk::launch_pack_ri3fn(ctx->g, d_rows, np, ctx->dB + p0 * ctx->g.ldB, pick(ctx, stream));
  return after_launch(ctx, "load rows");
}

int rijk_get_rimatr(rijk_ctx* ctx, double* rimatr) {
  RIJK_TRY(need_tensor(ctx));
  if (!rimatr) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  const Geom& g = ctx->g;
  const int64_t rows_per = std::max<int64_t>(1, std::min<int64_t>(g.naux, ((int64_t)256 << 20) / (g.npair * 8)));
  RIJK_TRY(ensure_pooled(ctx, ctx->stage, (size_t)rows_per * g.npair * 8));
  double* st = static_cast<double*>(ctx->stage.p);
  for (int64_t p0 = 0; p0 < g.naux; p0 += rows_per) {
    const int64_t np = std::min(rows_per, g.naux - p0);
    rijk::launch_unpack_rimatr(g, ctx->dB + p0 * g.ldB, np, st, ctx->stream);
    RIJK_TRY(after_launch(ctx, "unpack tensor"));
    RIJK_CK(cudaMemcpyAsync(rimatr + p0 * g.npair, st, (size_t)np * g.npair * 8, cudaMemcpyDeviceToHost,
                            ctx->stream));
  }
  return sync_and_check(ctx, ctx->stream);
}

namespace {

// The padded metric V is in ctx->mV and the three-centre rows in the tensor:
// factor V = L L^T, invert L and fit B = int3c L^-T in place.
int cholesky_fit(rijk_ctx* ctx, int64_t* failed_pivot) {
  const int64_t np = ctx->naux_pad;
  RIJK_TRY(ensure_pooled(ctx, ctx->mLinvd, (size_t)np * rijk::TS * 8));
  RIJK_TRY(ensure_pooled(ctx, ctx->mLinv, (size_t)np * np * 8));
  RIJK_TRY(ensure_pooled(ctx, ctx->mT, (size_t)np * np * 8));
  double* V = static_cast<double*>(ctx->mV.p);
  double* Linvd = static_cast<double*>(ctx->mLinvd.p);
  double* Linv = static_cast<double*>(ctx->mLinv.p);
  double* T = static_cast<double*>(ctx->mT.p);
  RIJK_CK(cudaMemsetAsync(ctx->d_info, 0, sizeof(int), ctx->stream));
  rijk::run_potrf(V, np, np, Linvd, ctx->d_info, ctx->d_err, ctx->stream);
  RIJK_TRY(after_launch(ctx, "potrf"));
  RIJK_TRY(sync_and_check(ctx, ctx->stream));
  int info = 0;
  RIJK_CK(cudaMemcpy(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost));
  if (info != 0) {
    if (failed_pivot) *failed_pivot = info;
    return set_err(ctx, RIJK_ERR_NOT_SPD, "metric not positive definite at pivot " + std::to_string(info));
  }
  rijk::run_trtri(V, np, np, Linvd, Linv, T, ctx->d_err, ctx->stream);
  RIJK_TRY(after_launch(ctx, "trtri"));
  // B^T = L^-1 (Q|mu nu)  <=>  B[k, P] = sum_Q int3c[k, Q] Linv[P, Q]
  RIJK_TRY(fit_in_place(ctx, Linv, np, 1, 2));
  RIJK_TRY(sync_and_check(ctx, ctx->stream));
  ctx->have = true;
  return release_fit_scratch(ctx);
}

struct PlanGuard {
  rijk::RiIntPlan* p = nullptr;
  ~PlanGuard() {
    if (p) rijk::ri_plan_destroy(p);
  }
};

const char* plan_error(int rc) {
  return rc == RIJK_ERR_TOO_LARGE ? "device integrals take AO shells with l <= 2 and auxiliary shells with l <= 4"
                                  : "invalid shell data or c2s table";
}

}  // namespace

int rijk_build_rimatr_cholesky(rijk_ctx* ctx, const double* aux_v, const double* int3c, int64_t num_basis,
                               int64_t num_auxbas, int64_t* failed_pivot) {
  if (failed_pivot) *failed_pivot = 0;
  if (!ctx || !aux_v || !int3c) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  RIJK_TRY(upload_tensor(ctx, int3c, num_basis, num_auxbas, 0));
  ctx->have = false;
  RIJK_TRY(upload_square_padded(ctx, aux_v, num_auxbas, ctx->naux_pad, ctx->mV));
  return cholesky_fit(ctx, failed_pivot);
}

int rijk_int2c2e_dev(const rijk_shells* aux, const double* const* c2s, double* d_out, void* stream) {
  if (!aux || !c2s || !d_out) return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PlanGuard pg;
  const int rc = rijk::ri_plan_create(nullptr, aux, c2s, st, &pg.p);
  if (rc != RIJK_OK) return rc;
  rijk::launch_int2c2e(pg.p, d_out, rijk::ri_plan_naux(pg.p), st);
  if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}

int rijk_int3c2e_dev(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, double* d_out,
                     void* stream) {
  if (!bas || !aux || !c2s || !d_out) return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PlanGuard pg;
  const int rc = rijk::ri_plan_create(bas, aux, c2s, st, &pg.p);
  if (rc != RIJK_OK) return rc;
  const int64_t n = rijk::ri_plan_nbas(pg.p), npair = n * (n + 1) / 2;
  const int nsh = rijk::ri_plan_aux_shells(pg.p);
  for (int k0 = 0; k0 < nsh; k0 += 64) {
    const int k1 = std::min(nsh, k0 + 64);
    rijk::launch_int3c2e(pg.p, k0, k1, d_out + rijk::ri_plan_aux_offset(pg.p, k0) * npair, st);
    if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  }
  return cudaStreamSynchronize(st) == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}

int rijk_build_rimatr_from_shells(rijk_ctx* ctx, const rijk_shells* bas, const rijk_shells* aux,
                                  const double* const* c2s, const double* metric_factor, int64_t* failed_pivot) {
  if (failed_pivot) *failed_pivot = 0;
  if (!ctx || !bas || !aux || !c2s) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  RIJK_CK(cudaSetDevice(ctx->device));
  PlanGuard pg;
  const int rc = rijk::ri_plan_create(bas, aux, c2s, ctx->stream, &pg.p);
  if (rc != RIJK_OK) return set_err(ctx, rc, plan_error(rc));
  const int64_t n = rijk::ri_plan_nbas(pg.p), naux = rijk::ri_plan_naux(pg.p);
  RIJK_TRY(alloc_tensor(ctx, n, naux));
  const Geom& g = ctx->g;
  // three-centre rows, a run of auxiliary shells at a time, packed as they come;
  // large runs keep every class kernel's grid wide
  const size_t chunk_bytes = std::max<size_t>(std::min<size_t>(ctx->scratch_budget / 2, (size_t)naux * g.npair * 8),
                                              (size_t)9 * g.npair * 8);
  RIJK_TRY(ensure_pooled(ctx, ctx->stage, std::max<size_t>(chunk_bytes, (size_t)naux * naux * 8)));
  double* st = static_cast<double*>(ctx->stage.p);
  const int nsh = rijk::ri_plan_aux_shells(pg.p);
  for (int k0 = 0; k0 < nsh;) {
    int k1 = k0 + 1;
    while (k1 < nsh &&
           (size_t)(rijk::ri_plan_aux_offset(pg.p, k1 + 1) - rijk::ri_plan_aux_offset(pg.p, k0)) * g.npair * 8 <=
               chunk_bytes)
      ++k1;
    const int64_t p0 = rijk::ri_plan_aux_offset(pg.p, k0), np = rijk::ri_plan_aux_offset(pg.p, k1) - p0;
    rijk::launch_int3c2e(pg.p, k0, k1, st, ctx->stream);
    RIJK_TRY(after_launch(ctx, "int3c2e"));
    rijk::launch_pack_rimatr(g, st, np, ctx->dB + p0 * g.ldB, ctx->stream);
    RIJK_TRY(after_launch(ctx, "pack tensor"));
    k0 = k1;
  }
  ctx->tensor_version++;
  const int64_t npad = ctx->naux_pad;
  if (metric_factor) {
    RIJK_TRY(upload_square_padded(ctx, metric_factor, naux, npad, ctx->mV));
    RIJK_TRY(fit_in_place(ctx, static_cast<double*>(ctx->mV.p), npad, 0, 0));
    RIJK_TRY(sync_and_check(ctx, ctx->stream));
    ctx->have = true;
    return release_fit_scratch(ctx);
  }
  RIJK_TRY(ensure_pooled(ctx, ctx->mV, (size_t)npad * npad * 8));
  rijk::launch_int2c2e(pg.p, st, naux, ctx->stream);
  RIJK_TRY(after_launch(ctx, "int2c2e"));
  rijk::launch_pad_matrix(st, naux, npad, static_cast<double*>(ctx->mV.p), ctx->stream);
  RIJK_TRY(after_launch(ctx, "pad metric"));
  return cholesky_fit(ctx, failed_pivot);
}

int rijk_fit_rimatr(rijk_ctx* ctx, const double* metric_factor, const double* int3c, int64_t num_basis,
                    int64_t num_auxbas) {
  if (!ctx || !metric_factor || !int3c) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  RIJK_TRY(upload_tensor(ctx, int3c, num_basis, num_auxbas, 0));
  ctx->have = false;
  const int64_t np = ctx->naux_pad;
  RIJK_TRY(upload_square_padded(ctx, metric_factor, num_auxbas, np, ctx->mV));
  RIJK_TRY(fit_in_place(ctx, static_cast<double*>(ctx->mV.p), np, 0, 0));
  RIJK_TRY(sync_and_check(ctx, ctx->stream));
  ctx->have = true;
  return release_fit_scratch(ctx);
}

// ---- J ------------------------------------------------------------------------
int rijk_vj_upper_dev(rijk_ctx* ctx, const double* d_dm, int spin_channel, double scaling_factor, int dm_mode,
                      double* d_vj, void* stream) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!d_dm || !d_vj || (dm_mode != 0 && dm_mode != 1)) return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  return vj_dev(ctx, d_dm, spin_channel, scaling_factor, dm_mode, 0, d_vj, pick(ctx, stream));
}

static int vj_host(rijk_ctx* ctx, const double* dm, int spin, double scale, int mode, int out_kind, double* out) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin));
  if (!dm || !out) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  const Geom& g = ctx->g;
  const size_t per = out_kind == 0 ? (size_t)g.npair : (size_t)(g.n * g.n);
  return host_call(ctx, dm, (size_t)spin * g.n * g.n, out, spin * per, [&](double* din, double* dout) {
    return vj_dev(ctx, din, spin, scale, mode, out_kind, dout, ctx->stream);
  });
}

int rijk_vj_upper_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor, double* vj) {
  return vj_host(ctx, dm, spin_channel, scaling_factor, 0, 0, vj);
}
int rijk_vj_upper_with_rimatr_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                double* vj) {
  return vj_host(ctx, dm, spin_channel, scaling_factor, 1, 0, vj);
}
int rijk_vj_full_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor, double* vj_full) {
  return vj_host(ctx, dm, spin_channel, scaling_factor, 0, 1, vj_full);
}

// ---- K ------------------------------------------------------------------------
int rijk_vk_upper_occ_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                          const double* d_occupation, int spin_channel, double scaling_factor, double* d_vk,
                          void* stream) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!d_eigv || !homo || !d_occupation || !d_vk || num_state <= 0)
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  return vk_occ_dev(ctx, d_eigv, num_state, homo, d_occupation, spin_channel, scaling_factor, d_vk,
                    pick(ctx, stream));
}

int rijk_vjk_upper_occ_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                           const double* d_occupation, int spin_channel, double j_scaling_factor,
                           double k_scaling_factor, double* d_vj, double* d_vk, void* stream) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!d_eigv || !homo || !d_occupation || !d_vj || !d_vk || num_state <= 0 || d_vj == d_vk)
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  return vk_occ_dev(ctx, d_eigv, num_state, homo, d_occupation, spin_channel, k_scaling_factor, d_vk,
                    pick(ctx, stream), j_scaling_factor, d_vj);
}

int rijk_vk_upper_with_ri_v(rijk_ctx* ctx, const double* eigv, int64_t num_state, const int64_t* homo,
                            const double* occupation, int spin_channel, double scaling_factor, double* vk) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!eigv || !homo || !occupation || !vk || num_state <= 0) return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  for (int s = 0; s < spin_channel; ++s) {
    if (homo[s] < 0 || homo[s] >= num_state) return set_err(ctx, RIJK_ERR_ARG, "homo out of range");
    for (int64_t i = 0; i <= homo[s]; ++i)
      if (!(occupation[s * num_state + i] >= 0.0)) return set_err(ctx, RIJK_ERR_ARG, "negative occupation");
  }
  const Geom& g = ctx->g;
  const size_t ne = (size_t)spin_channel * g.n * num_state;
  RIJK_TRY(ensure(ctx, ctx->docc, (size_t)spin_channel * num_state * 8));
  RIJK_CK(cudaMemcpyAsync(ctx->docc.p, occupation, (size_t)spin_channel * num_state * 8, cudaMemcpyHostToDevice,
                          ctx->stream));
  return host_call(ctx, eigv, ne, vk, (size_t)spin_channel * g.npair, [&](double* din, double* dout) {
    return vk_occ_dev(ctx, din, num_state, homo, static_cast<double*>(ctx->docc.p), spin_channel, scaling_factor,
                      dout, ctx->stream);
  });
}

int rijk_vjk_upper_with_ri_v(rijk_ctx* ctx, const double* eigv, int64_t num_state, const int64_t* homo,
                             const double* occupation, int spin_channel, double j_scaling_factor,
                             double k_scaling_factor, double* vj, double* vk) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!eigv || !homo || !occupation || !vj || !vk || num_state <= 0) return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  for (int s = 0; s < spin_channel; ++s) {
    if (homo[s] < 0 || homo[s] >= num_state) return set_err(ctx, RIJK_ERR_ARG, "homo out of range");
    for (int64_t i = 0; i <= homo[s]; ++i)
      if (!(occupation[s * num_state + i] >= 0.0)) return set_err(ctx, RIJK_ERR_ARG, "negative occupation");
  }
  const Geom& g = ctx->g;
  const size_t ne = (size_t)spin_channel * g.n * num_state;
  const size_t per = (size_t)spin_channel * g.npair;
  RIJK_TRY(ensure(ctx, ctx->docc, (size_t)spin_channel * num_state * 8));
  RIJK_CK(cudaMemcpyAsync(ctx->docc.p, occupation, (size_t)spin_channel * num_state * 8, cudaMemcpyHostToDevice,
                          ctx->stream));
  // J and K land side by side in the output staging buffer
  RIJK_TRY(ensure(ctx, ctx->din, ne * 8));
  RIJK_TRY(ensure(ctx, ctx->dout, 2 * per * 8));
  double* din = static_cast<double*>(ctx->din.p);
  double* dout = static_cast<double*>(ctx->dout.p);
  RIJK_CK(cudaMemcpyAsync(din, eigv, ne * 8, cudaMemcpyHostToDevice, ctx->stream));
  RIJK_TRY(vk_occ_dev(ctx, din, num_state, homo, static_cast<double*>(ctx->docc.p), spin_channel, k_scaling_factor,
                      dout + per, ctx->stream, j_scaling_factor, dout));
  RIJK_CK(cudaMemcpyAsync(vj, dout, per * 8, cudaMemcpyDeviceToHost, ctx->stream));
  RIJK_CK(cudaMemcpyAsync(vk, dout + per, per * 8, cudaMemcpyDeviceToHost, ctx->stream));
  return sync_and_check(ctx, ctx->stream);
}

int rijk_vk_upper_dm_dev(rijk_ctx* ctx, const double* d_dm, int spin_channel, double scaling_factor, double* d_vk,
                         void* stream) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!d_dm || !d_vk) return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  return vk_dm_dev(ctx, d_dm, spin_channel, scaling_factor, 0, d_vk, pick(ctx, stream));
}

static int vk_dm_host(rijk_ctx* ctx, const double* dm, int spin, double scale, int full, double* out) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin));
  if (!dm || !out) return set_err(ctx, RIJK_ERR_ARG, "null argument");
  const Geom& g = ctx->g;
  const size_t per = full ? (size_t)(g.n * g.n) : (size_t)g.npair;
  return host_call(ctx, dm, (size_t)spin * g.n * g.n, out, spin * per, [&](double* din, double* dout) {
    return vk_dm_dev(ctx, din, spin, scale, full, dout, ctx->stream);
  });
}

int rijk_vk_upper_with_ri_v_use_dm_only(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                        double* vk) {
  return vk_dm_host(ctx, dm, spin_channel, scaling_factor, 0, vk);
}
int rijk_vk_upper_with_rimatr_use_dm_only(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                          double* vk) {
  return vk_dm_host(ctx, dm, spin_channel, scaling_factor, 0, vk);
}
int rijk_vk_full_fromdm_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                  double* vk_full) {
  return vk_dm_host(ctx, dm, spin_channel, scaling_factor, 1, vk_full);
}

// ---- density matrix and energy -----------------------------------------------
int rijk_density_matrix(rijk_ctx* ctx, const double* eigv, int64_t num_basis, int64_t num_state, const int64_t* homo,
                        const double* occupation, int spin_channel, double* dm) {
  if (!ctx || !eigv || !homo || !occupation || !dm || num_basis <= 0 || num_state <= 0)
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  RIJK_TRY(check_spin(ctx, spin_channel));
  RIJK_CK(cudaSetDevice(ctx->device));
  const int64_t n = num_basis;
  const int64_t ld = round_up(n, 128);
  Geom g = rijk::make_geom(n, 1);
  RIJK_TRY(ensure(ctx, ctx->din, (size_t)spin_channel * n * num_state * 8));
  RIJK_TRY(ensure(ctx, ctx->docc, (size_t)spin_channel * num_state * 8));
  RIJK_TRY(ensure(ctx, ctx->dout, (size_t)spin_channel * ld * ld * 8));
  double* din = static_cast<double*>(ctx->din.p);
  double* dout = static_cast<double*>(ctx->dout.p);
  RIJK_CK(cudaMemcpyAsync(din, eigv, (size_t)spin_channel * n * num_state * 8, cudaMemcpyHostToDevice, ctx->stream));
  RIJK_CK(cudaMemcpyAsync(ctx->docc.p, occupation, (size_t)spin_channel * num_state * 8, cudaMemcpyHostToDevice,
                          ctx->stream));
  for (int s = 0; s < spin_channel; ++s) {
    const int64_t nw[2] = {homo[s] + 1, 0};
    if (homo[s] < 0 || nw[0] > num_state) return set_err(ctx, RIJK_ERR_ARG, "homo out of range");
    for (int64_t i = 0; i < nw[0]; ++i)
      if (!(occupation[s * num_state + i] >= 0.0)) return set_err(ctx, RIJK_ERR_ARG, "negative occupation");
    const int64_t kc = round_up(nw[0], 64);
    RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ld * kc * 8));
    double* Cw = static_cast<double*>(ctx->Cw.p);
    rijk::launch_k_prepare_c(g, din + s * n * num_state, n, 0, static_cast<double*>(ctx->docc.p) + s * num_state, 0,
                             nw, 1, ld, kc, Cw, ctx->d_err, ctx->stream);
    rijk::launch_dgemm(ld, ld, kc, 1.0, Cw, ld, 0, Cw, ld, 1, 0.0, dout + s * ld * ld, ld, 0, 0, 1, 0, 0, 0,
                       ctx->d_err, ctx->stream);
    RIJK_TRY(after_launch(ctx, "density"));
  }
  for (int s = 0; s < spin_channel; ++s)
    RIJK_CK(cudaMemcpy2DAsync(dm + s * n * n, n * 8, dout + s * ld * ld, ld * 8, n * 8, n, cudaMemcpyDeviceToHost,
                              ctx->stream));
  return sync_and_check(ctx, ctx->stream);
}

// ---- split-precision exchange (tcgen05) ----------------------------------------
static int tc_prepare(rijk_ctx* ctx, cudaStream_t st) {
  if (ctx->tc_version == ctx->tensor_version) return RIJK_OK;
  const Geom& g = ctx->g;
  const size_t bytes = (size_t)rijk::tc_tensor_elems(g) * 2;
  RIJK_TRY(ensure(ctx, ctx->tcBhi, bytes));
  RIJK_TRY(ensure(ctx, ctx->tcBlo, bytes));
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(g.naux, 1024));
  for (int64_t p0 = 0; p0 < g.naux; p0 += chunk)
    rijk::launch_split_tensor(g, ctx->dB, p0, std::min(chunk, g.naux - p0), ctx->tcBhi.p, ctx->tcBlo.p, st);
  RIJK_TRY(after_launch(ctx, "split tensor"));
  ctx->tc_version = ctx->tensor_version;
  return RIJK_OK;
}

// out (+)= scale sum_P (B_P V)(S)(B_P V)^T for the columns [c0, c0 + nc) of V, all of sign `sgn`
// With w: also w[p] += sgn <V, B_p V> (J's scalars of the same difference).
static int tc_lowrank_group(rijk_ctx* ctx, const double* d_V, int64_t ldv, int c0, int nc, int sgn, double scale,
                            int accumulate, double* d_out, cudaStream_t st, double* w = nullptr) {
  const Geom& g = ctx->g;
  const rijk::TcGeom t = rijk::make_tc_geom(g, nc);
  const size_t vbytes = (size_t)t.npad * 64 * t.nkb * 2;
  RIJK_TRY(ensure(ctx, ctx->tcVhi, vbytes));
  RIJK_TRY(ensure(ctx, ctx->tcVlo, vbytes));
  rijk::launch_split_cols(g, t, d_V + (int64_t)c0 * ldv, ldv, nc, ctx->tcVhi.p, ctx->tcVlo.p, st);
  const int64_t xper = (int64_t)t.nmb * t.nib * t.block_elems * 2;  // bytes per P per plane
  const int64_t pchunk = std::max<int64_t>(1, std::min<int64_t>(g.naux, (int64_t)ctx->scratch_budget / (2 * xper)));
  RIJK_TRY(ensure(ctx, ctx->tcXhi, (size_t)pchunk * xper));
  RIJK_TRY(ensure(ctx, ctx->tcXlo, (size_t)pchunk * xper));
  const int64_t pairs = (int64_t)t.nmb * (t.nmb + 1) / 2;
  const int splits_max = rijk::tc_rank_splits(t, pchunk);
  RIJK_TRY(ensure(ctx, ctx->tcPart, (size_t)splits_max * pairs * 128 * 128 * 4));
  rijk::TcJ jw{d_V + (int64_t)c0 * ldv, ldv, nc, (double)sgn, nullptr, w};
  if (w) {
    RIJK_TRY(ensure(ctx, ctx->Jw, (size_t)pchunk * 4 * t.nmb * 8));
    jw.wpart = static_cast<double*>(ctx->Jw.p);
  }
  for (int64_t p0 = 0; p0 < g.naux; p0 += pchunk) {
    const int64_t np = std::min(pchunk, g.naux - p0);
    {
      ProfScope ps(ctx, RIJK_PROF_K_HALF, st);
      rijk::launch_half_tc(g, t, ctx->tcBhi.p, ctx->tcBlo.p, p0, np, ctx->tcVhi.p, ctx->tcVlo.p, ctx->tcXhi.p,
                           ctx->tcXlo.p, ctx->d_err, st, w ? &jw : nullptr);
    }
    const int splits = rijk::tc_rank_splits(t, np);
    {
      ProfScope ps(ctx, RIJK_PROF_K_RANK, st);
      rijk::launch_rank_tc(g, t, ctx->tcXhi.p, ctx->tcXlo.p, np, sgn > 0 ? t.nib : 0, splits,
                           static_cast<float*>(ctx->tcPart.p), ctx->d_err, st);
    }
    ProfScope ps(ctx, RIJK_PROF_K_OTHER, st);
    rijk::launch_rank_tc_finalize(g, t, static_cast<float*>(ctx->tcPart.p), splits, scale,
                                  (accumulate || p0 > 0) ? 1 : 0, d_out, st);
  }
  return after_launch(ctx, "split exchange");
}

int rijk_vk_upper_lowrank_split_dev(rijk_ctx* ctx, const double* d_V, int64_t ld_v, int64_t ncols, int64_t npos,
                                    double scaling_factor, int accumulate, double* d_vk, void* stream) {
  RIJK_TRY(need_tensor(ctx));
  if (!d_V || !d_vk || ncols < 0 || npos < 0 || npos > ncols || ld_v < ctx->g.n || (ld_v & 1) ||
      (reinterpret_cast<uintptr_t>(d_V) & 15))
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  cudaStream_t st = pick(ctx, stream);
  RIJK_TRY(tc_prepare(ctx, st));
  bool first = !accumulate;
  if (ncols == 0 && first) RIJK_CK(cudaMemsetAsync(d_vk, 0, (size_t)ctx->g.npair * 8, st));
  for (int64_t c0 = 0; c0 < ncols;) {
    const int64_t end = c0 < npos ? npos : ncols;
    const int nc = (int)std::min<int64_t>(256, end - c0);
    RIJK_TRY(tc_lowrank_group(ctx, d_V, ld_v, (int)c0, nc, c0 < npos ? 1 : -1, scaling_factor, first ? 0 : 1, d_vk,
                              st));
    first = false;
    c0 += nc;
  }
  return RIJK_OK;
}

int rijk_vjk_upper_lowrank_split_dev(rijk_ctx* ctx, const double* d_V, int64_t ld_v, int64_t ncols, int64_t npos,
                                     double j_scaling_factor, double k_scaling_factor, int accumulate, double* d_vj,
                                     double* d_vk, void* stream) {
  RIJK_TRY(need_tensor(ctx));
  if (!d_V || !d_vj || !d_vk || d_vj == d_vk || ncols < 0 || npos < 0 || npos > ncols || ld_v < ctx->g.n ||
      (ld_v & 1) || (reinterpret_cast<uintptr_t>(d_V) & 15))
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  const Geom& g = ctx->g;
  cudaStream_t st = pick(ctx, stream);
  RIJK_TRY(tc_prepare(ctx, st));
  RIJK_TRY(ensure(ctx, ctx->w, (size_t)g.naux * 8));
  double* w = static_cast<double*>(ctx->w.p);
  RIJK_CK(cudaMemsetAsync(w, 0, (size_t)g.naux * 8, st));
  bool first = !accumulate;
  if (ncols == 0 && first) RIJK_CK(cudaMemsetAsync(d_vk, 0, (size_t)g.npair * 8, st));
  for (int64_t c0 = 0; c0 < ncols;) {
    const int64_t end = c0 < npos ? npos : ncols;
    const int nc = (int)std::min<int64_t>(256, end - c0);
    RIJK_TRY(tc_lowrank_group(ctx, d_V, ld_v, (int)c0, nc, c0 < npos ? 1 : -1, k_scaling_factor, first ? 0 : 1,
                              d_vk, st, w));
    first = false;
    c0 += nc;
  }
  const int jsplits = rijk::j_pass2_splits(g);
  RIJK_TRY(ensure(ctx, ctx->Jpart, (size_t)jsplits * g.ldB * 8));
  double* Jp = static_cast<double*>(ctx->Jpart.p);
  {
    ProfScope ps(ctx, RIJK_PROF_J_PASS2, st);
    rijk::launch_j_pass2(g, ctx->dB, w, 1, jsplits, Jp, st);
  }
  ProfScope ps(ctx, RIJK_PROF_J_OTHER, st);
  rijk::launch_j_finalize(g, Jp, 1, jsplits, j_scaling_factor, 0, d_vj, st);
  return after_launch(ctx, "split J and exchange");
}

int rijk_vk_upper_occ_split_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                                const double* d_occupation, int spin_channel, double scaling_factor, double* d_vk,
                                void* stream) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!d_eigv || !homo || !d_occupation || !d_vk || num_state <= 0) return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  const Geom& g = ctx->g;
  cudaStream_t st = pick(ctx, stream);
  const int64_t ldx = round_up(g.n, 128);
  for (int s = 0; s < spin_channel; ++s) {
    const int64_t nw[2] = {homo[s] + 1, 0};
    if (homo[s] < 0 || nw[0] > num_state) return set_err(ctx, RIJK_ERR_ARG, "homo out of range");
    const int64_t oc = round_up(nw[0], 64);
    RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ldx * oc * 8));
    double* Cw = static_cast<double*>(ctx->Cw.p);
    rijk::launch_k_prepare_c(g, d_eigv + (size_t)s * g.n * num_state, g.n, 0, d_occupation + (size_t)s * num_state, 0,
                             nw, 1, ldx, oc, Cw, ctx->d_err, st);
    RIJK_TRY(rijk_vk_upper_lowrank_split_dev(ctx, Cw, ldx, nw[0], nw[0], scaling_factor, 0, d_vk + s * g.npair, st));
  }
  return RIJK_OK;
}

int rijk_ao2mo(rijk_ctx* ctx, const double* eigv, int64_t num_state, int64_t row_begin, int64_t row_end,
               int64_t col_begin, int64_t col_end, int spin_channel, double* ri3mo) {
  RIJK_TRY(need_tensor(ctx));
  RIJK_TRY(check_spin(ctx, spin_channel));
  if (!eigv || !ri3mo || num_state <= 0 || row_begin < 0 || row_end <= row_begin || row_end > num_state ||
      col_begin < 0 || col_end <= col_begin || col_end > num_state)
    return set_err(ctx, RIJK_ERR_ARG, "bad argument");
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int64_t n = g.n, nrow = row_end - row_begin, ncol = col_end - col_begin;
  const int64_t ldx = round_up(n, 128);
  const int64_t ocols = round_up(ncol, 128);
  const int64_t nrp = round_up(nrow, 32);
  const int64_t ldy = round_up(nrow, 2);
  RIJK_TRY(ensure(ctx, ctx->din, (size_t)n * num_state * 8));
  RIJK_TRY(ensure(ctx, ctx->Cw, (size_t)ldx * ocols * 8));
  RIJK_TRY(ensure(ctx, ctx->Cr, (size_t)ldx * nrp * 8));
  const int64_t per_p = ldx * ocols * 8 + ldy * ncol * 8 * 2;
  const int64_t pchunk = std::max<int64_t>(1, std::min<int64_t>(g.naux, (int64_t)ctx->scratch_budget / per_p));
  RIJK_TRY(ensure(ctx, ctx->X, (size_t)pchunk * ldx * ocols * 8));
  RIJK_TRY(ensure(ctx, ctx->Y, (size_t)pchunk * ldy * ncol * 8));
  RIJK_TRY(ensure(ctx, ctx->Yp, (size_t)pchunk * nrow * ncol * 8));
  double* din = static_cast<double*>(ctx->din.p);
  double* Cc = static_cast<double*>(ctx->Cw.p);
  double* Cr = static_cast<double*>(ctx->Cr.p);
  double* X = static_cast<double*>(ctx->X.p);
  double* Y = static_cast<double*>(ctx->Y.p);
  double* Yp = static_cast<double*>(ctx->Yp.p);
  for (int s = 0; s < spin_channel; ++s) {
    double* out = ri3mo + (size_t)s * g.naux * nrow * ncol;
    RIJK_CK(cudaMemcpyAsync(din, eigv + (size_t)s * n * num_state, (size_t)n * num_state * 8, cudaMemcpyHostToDevice,
                            st));
    rijk::launch_gather_cols(din, n, n, col_begin, ncol, ldx, ocols, Cc, st);
    rijk::launch_gather_cols(din, n, n, row_begin, nrow, ldx, nrp, Cr, st);
    for (int64_t p0 = 0; p0 < g.naux; p0 += pchunk) {
      const int64_t np = std::min(pchunk, g.naux - p0);
      // X_p = B_p C[:, cols]  (FP64 DMMA half-transform)
      rijk::launch_half_transform(g, ctx->dB, p0, np, Cc, ldx, ocols, ncol, X, ldx, rijk::XMap::dense(ocols),
                                  ctx->d_err, st);
      // Y_p = C[:, rows]^T X_p  (batched over p)
      for (int64_t b0 = 0; b0 < np; b0 += 65535) {
        const int64_t nb = std::min<int64_t>(65535, np - b0);
        rijk::launch_dgemm(nrow, ncol, g.nt * rijk::TS, 1.0, Cr, ldx, 1, X + b0 * ldx * ocols, ldx, 0, 0.0,
                           Y + b0 * ldy * ncol, ldy, 0, 0, (int)nb, 0, ldx * ocols, ldy * ncol, ctx->d_err, st);
      }
      rijk::launch_ri3mo_permute(Y, ldy, ldy * ncol, np, nrow, ncol, Yp, st);
      RIJK_TRY(after_launch(ctx, "ao2mo"));
      // chunk rows p0..p0+np of every (a, i) column of REST's RIFull[naux, nrow, ncol]
      RIJK_CK(cudaMemcpy2DAsync(out + p0, (size_t)g.naux * 8, Yp, (size_t)np * 8, (size_t)np * 8,
                                (size_t)nrow * ncol, cudaMemcpyDeviceToHost, st));
    }
  }
  return sync_and_check(ctx, st);
}

// ---- grouped build over a molecule set -------------------------------------------
}  // extern "C"

struct rijk_group {
  int device = 0;
  int count = 0;
  std::vector<rijk_ctx*> ctxs;
  std::vector<int64_t> versions;  // each context's tensor version at creation
  rijk::GroupPlan plan{};
  void* mem = nullptr;  // descriptors, prefix sums, error words and every molecule's scratch
  int* d_err = nullptr;
  int sms = 148;
  std::string last;
};

extern "C" {

int rijk_group_create(rijk_ctx* const* ctxs, int count, const int64_t* nocc, int half_transform_cfg, int update_cfg,
                      rijk_group** out) {
  if (!ctxs || !nocc || !out || count <= 0) return RIJK_ERR_ARG;
  *out = nullptr;
  if (half_transform_cfg != 0 && half_transform_cfg != 1 && half_transform_cfg != 4) return RIJK_ERR_ARG;
  if (update_cfg != 0 && update_cfg != 1 && update_cfg != 4) return RIJK_ERR_ARG;
  const int device = ctxs[0] ? ctxs[0]->device : -1;
  for (int m = 0; m < count; ++m) {
    if (!ctxs[m] || !ctxs[m]->have || ctxs[m]->device != device) return RIJK_ERR_ARG;
    if (nocc[m] <= 0 || nocc[m] > ctxs[m]->g.n) return RIJK_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return RIJK_ERR_CUDA;
  const int BM = rijk::group_cta_rows(half_transform_cfg), BN = rijk::group_cta_cols(half_transform_cfg);
  const int subs = rijk::group_rank_subs(update_cfg);
  std::vector<rijk::GroupMol> mols(count);
  std::vector<int64_t> pre[6];
  int64_t tot[6] = {0, 0, 0, 0, 0, 0};
  // byte layout: descriptors | 6 prefix arrays | error words | per-molecule scratch
  size_t off = round_up((int64_t)count * sizeof(rijk::GroupMol), 256);
  const size_t pre_off = off;
  off += round_up(6 * (int64_t)count * 8, 256);
  const size_t err_off = off;
  off += 256;
  std::vector<size_t> mol_off(count);
  for (int m = 0; m < count; ++m) {
    const Geom& g = ctxs[m]->g;
    rijk::GroupMol& d = mols[m];
    d.B = ctxs[m]->dB;
    d.ldB = g.ldB;
    d.n = (int)g.n;
    d.nt = (int)g.nt;
    d.naux = (int)g.naux;
    d.nocc = (int)nocc[m];
    d.ldx = round_up(g.n, 128);
    d.ocols = (int)round_up(nocc[m], std::max(BN, 64));
    d.jsplits = (int)std::max<int64_t>(1, std::min<int64_t>(8, g.naux / 256));
    d.ksplits = (int)std::max<int64_t>(1, std::min<int64_t>(16, cdiv(g.naux * nocc[m], 32768)));
    d.nkb = cdiv(g.n, 128);
    d.pairs = d.nkb * (d.nkb + 1) / 2;
    d.npair = g.npair;
    {
      // orbitals ending 1..16 columns past a full block: the last full block's
      // CTAs compute them (shape 1 only), so no mostly empty block is launched
      const int full = (int)(nocc[m] / BN), rem = (int)(nocc[m] - (int64_t)full * BN);
      const int xr = rijk::group_remainder_cols(half_transform_cfg);
      d.xcol0 = (full >= 1 && rem > 0 && rem <= xr) ? full * BN : 0;
      d.ncb = d.xcol0 > 0 ? full : d.ocols / BN;
    }
    d.wper = (int)((d.ldx / BM) * d.ncb * rijk::group_cta_warps(half_transform_cfg));
    const int64_t counts[6] = {d.ldx * d.ocols, g.naux, g.naux * (d.ldx / BM) * d.ncb,
                               (int64_t)d.ksplits * d.pairs * subs, (int64_t)d.jsplits * cdiv(g.ldB / 2, 256),
                               g.npair};
    for (int ph = 0; ph < 6; ++ph) {
      pre[ph].push_back(tot[ph]);
      tot[ph] += counts[ph];
    }
    mol_off[m] = off;
    off += round_up(d.ldx * d.ocols * 8, 256) + round_up(g.naux * d.wper * 8, 256) + round_up(g.naux * 8, 256) +
           round_up((int64_t)d.jsplits * g.ldB * 8, 256) + round_up((g.naux * nocc[m] + rijk::TS) * d.ldx * 8, 256) +
           round_up((int64_t)d.ksplits * d.pairs * 128 * 128 * 8, 256);
  }
  void* mem = nullptr;
  if (cudaMalloc(&mem, off) != cudaSuccess) {
    cudaGetLastError();
    return RIJK_ERR_NOMEM;
  }
  char* base = static_cast<char*>(mem);
  for (int m = 0; m < count; ++m) {
    rijk::GroupMol& d = mols[m];
    const Geom& g = ctxs[m]->g;
    char* q = base + mol_off[m];
    auto take = [&](int64_t bytes) {
      char* r = q;
      q += round_up(bytes, 256);
      return reinterpret_cast<double*>(r);
    };
    d.Cw = take(d.ldx * d.ocols * 8);
    d.wpart = take(g.naux * d.wper * 8);
    d.w = take(g.naux * 8);
    d.Jpart = take((int64_t)d.jsplits * g.ldB * 8);
    d.X = take((g.naux * d.nocc + rijk::TS) * d.ldx * 8);
    d.Kpart = take((int64_t)d.ksplits * d.pairs * 128 * 128 * 8);
  }
  std::vector<int64_t> pre_flat;
  for (int ph = 0; ph < 6; ++ph) pre_flat.insert(pre_flat.end(), pre[ph].begin(), pre[ph].end());
  bool ok = cudaMemcpy(base, mols.data(), count * sizeof(rijk::GroupMol), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(base + pre_off, pre_flat.data(), pre_flat.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(base + err_off, 0, 256) == cudaSuccess;
  // X's spare columns are read (masked) by the rank update's last k tile
  for (int m = 0; ok && m < count; ++m)
    ok = cudaMemset(mols[m].X, 0, (size_t)(mols[m].naux * (int64_t)mols[m].nocc + rijk::TS) * mols[m].ldx * 8) ==
         cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cudaFree(mem);
    return RIJK_ERR_CUDA;
  }
  rijk_group* gr = new rijk_group();
  gr->device = device;
  gr->count = count;
  for (int m = 0; m < count; ++m) {
    gr->ctxs.push_back(ctxs[m]);
    gr->versions.push_back(ctxs[m]->tensor_version);
  }
  gr->mem = mem;
  gr->d_err = reinterpret_cast<int*>(base + err_off);
  gr->plan.mols = reinterpret_cast<rijk::GroupMol*>(base);
  gr->plan.count = count;
  for (int ph = 0; ph < 6; ++ph) {
    gr->plan.pre[ph] = reinterpret_cast<int64_t*>(base + pre_off) + (int64_t)ph * count;
    gr->plan.total[ph] = tot[ph];
  }
  gr->plan.ht_cfg = half_transform_cfg;
  gr->plan.rk_cfg = update_cfg;
  gr->plan.remainder = 0;
  for (int m = 0; m < count; ++m) gr->plan.remainder |= mols[m].xcol0 > 0 ? 1 : 0;
  int sms = 148;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  gr->sms = sms;
  *out = gr;
  return RIJK_OK;
}

int rijk_group_destroy(rijk_group* g) {
  if (!g) return RIJK_OK;
  cudaSetDevice(g->device);
  cudaDeviceSynchronize();
  if (g->mem) cudaFree(g->mem);
  delete g;
  return RIJK_OK;
}

int rijk_group_jk_occ_dev(rijk_group* g, const double* d_C, int64_t c_mol, int64_t c_row, int64_t c_col,
                          double k_scale, const int* d_active, double* d_out, int64_t out_mol, int64_t ldo,
                          void* stream) {
  if (!g || !d_C || !d_active || !d_out || ldo <= 0) return RIJK_ERR_ARG;
  for (int m = 0; m < g->count; ++m)
    if (!g->ctxs[m]->have || g->ctxs[m]->tensor_version != g->versions[m]) {
      g->last = "a context of the group has loaded another tensor since the group was created";
      return RIJK_ERR_ARG;
    }
  if (cudaSetDevice(g->device) != cudaSuccess) return RIJK_ERR_CUDA;
  rijk::launch_group(g->plan, d_C, c_mol, c_row, c_col, k_scale, d_out, out_mol, ldo, d_active, g->d_err, g->sms,
                     static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g->last = std::string("group build: ") + cudaGetErrorString(e);
    return RIJK_ERR_CUDA;
  }
  return RIJK_OK;
}

int rijk_group_synchronize(rijk_group* g, void* stream) {
  if (!g) return RIJK_ERR_ARG;
  if (cudaSetDevice(g->device) != cudaSuccess) return RIJK_ERR_CUDA;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return RIJK_ERR_CUDA;
  int h = 0;
  if (cudaMemcpy(&h, g->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return RIJK_ERR_CUDA;
  if (h != 0) {
    cudaMemset(g->d_err, 0, sizeof(int));
    g->last = "a device-side wait exceeded its time budget";
    return RIJK_ERR_TIMEOUT;
  }
  return RIJK_OK;
}

double rijk_energy_contraction(const double* a, const double* b, int64_t npair) {
  if (!a || !b || npair <= 0) return 0.0;
  double tot = 0.0, dg = 0.0;
  for (int64_t k = 0; k < npair; ++k) tot += a[k] * b[k];
  for (int64_t j = 0;; ++j) {
    const int64_t d = j * (j + 1) / 2 + j;
    if (d >= npair) break;
    dg += a[d] * b[d];
  }
  return (2.0 * tot - dg) * 0.5;
}

}  // extern "C"
