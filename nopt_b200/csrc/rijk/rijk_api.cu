// rijk_api.cu — the C ABI of librijk: context, set-up (metric, fitted tensor) and the
// Fock build.  See include/rijk.h for the reference functions each entry point replaces.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {

int mixed_prepare(rijk_ctx* ctx);
int mixed_exchange(rijk_ctx* ctx, const double* dMO, long nocc, double* dK);

int set_err(rijk_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return code;
}

int cuda_check(rijk_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return RIJK_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return set_err(ctx, RIJK_ERR_ALLOC, "%s: out of device memory", what);
  }
  return set_err(ctx, RIJK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int ensure(rijk_ctx* ctx, DeviceBuf& b, size_t bytes, const char* what) {
  if (b.bytes >= bytes && b.p) return RIJK_OK;
  if (bytes > 0 && ctx->fail_alloc_after >= 0) {  // rijk_selftest_alloc_failure
    if (ctx->fail_alloc_after == 0) return set_err(ctx, RIJK_ERR_ALLOC, "%s: out of device memory (injected)", what);
    --ctx->fail_alloc_after;
  }
  if (b.p) {  // the old buffer may still be read by work queued on the context's streams
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->j_stream) cudaStreamSynchronize(ctx->j_stream);
    cudaFree(b.p);
  }
  b.p = nullptr;
  b.bytes = 0;
  if (bytes == 0) return RIJK_OK;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) return cuda_check(ctx, e, what);
  b.bytes = bytes;
  return RIJK_OK;
}

cudaError_t ensure_smem_limit(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{fn, dev}];
  if (have >= bytes) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e == cudaSuccess) have = bytes;
  return e;
}

void prefer_max_shared(const void* fn) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, bool> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  bool& set = done[{fn, dev}];
  if (set) return;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) ==
      cudaSuccess)
    set = true;
  else
    cudaGetLastError();  // a hint only: the launch works without it
}

void release(DeviceBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

__global__ void k_pad_from_colmajor(const double* __restrict__ src, long naux, double* __restrict__ dst, long nauxp) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long total = nauxp * nauxp;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long q = idx / nauxp, p = idx % nauxp;
    dst[idx] = (q < naux && p < naux) ? src[q + p * naux] : 0.0;
  }
}

// Scale column k of the eigenvector matrix by lambda_k^-1/2 (0 for lambda_k <= 0, as
// S05_calc does, src/matr.cpp:383-386); count the dropped eigenvalues.
__global__ void k_scale_eigvecs(double* __restrict__ U, const double* __restrict__ w, long naux, int* ndrop) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long total = naux * naux;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long k = idx / naux;
    double l = w[k];
    double f = l > 0.0 ? 1.0 / sqrt(l) : 0.0;
    U[idx] *= f;
    if (idx % naux == 0 && !(l > 0.0)) atomicAdd(ndrop, 1);
  }
}

__global__ void k_identity(double* __restrict__ X, long n) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long total = n * n;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) X[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

__global__ void k_fock_matrix(const double* __restrict__ H, const double* __restrict__ J, const double* __restrict__ K,
                              double cj, double ck, long nn, double* __restrict__ F) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < nn; idx += static_cast<long>(gridDim.x) * blockDim.x) F[idx] = H[idx] + cj * J[idx] - ck * K[idx];
}

static unsigned grid1d(long total) {
  long b = (total + 255) / 256;
  return static_cast<unsigned>(std::min<long>(std::max<long>(b, 1), 148L * 16));
}

namespace {
std::mutex g_log_mu;
FILE* g_log = nullptr;
bool g_log_checked = false;
}  // namespace

void log_line(const std::string& json) {
  std::lock_guard<std::mutex> lock(g_log_mu);
  if (!g_log_checked) {
    g_log_checked = true;
    const char* path = std::getenv("RIJK_LOG");
    if (path && *path) g_log = std::fopen(path, "a");
  }
  if (!g_log) return;
  std::fputs(json.c_str(), g_log);
  std::fputc('\n', g_log);
  std::fflush(g_log);
}

void log_build(rijk_ctx* ctx, const char* call, long nocc, int precision) {
  const rijk_stats_t& st = ctx->stats;
  const char* prec = precision == RIJK_PREC_MIXED ? "mixed" : precision == RIJK_PREC_FP64_TC ? "fp64_tc" : "fp64";
  const double ms = st.ms_last_fock;
  char buf[640];
  std::snprintf(buf, sizeof(buf),
                "{\"call\": \"%s\", \"device\": %d, \"n\": %ld, \"naux\": %ld, \"q0\": %ld, \"n_c\": %ld, "
                "\"precision\": \"%s\", \"ms\": %.6g, \"ms_coulomb\": %.6g, \"ms_exchange\": %.6g, "
                "\"flops\": %.6g, \"bytes\": %.6g, \"tflops\": %.6g, \"gbs\": %.6g, \"kernels\": %d}",
                call, ctx->device, ctx->n, ctx->nq, ctx->q0, nocc, prec, ms, st.ms_coulomb, st.ms_exchange,
                st.flops_last_fock, st.bytes_last_fock, ms > 0 ? st.flops_last_fock / (ms * 1e9) : 0.0,
                ms > 0 ? st.bytes_last_fock / (ms * 1e6) : 0.0, st.kernels_last_fock);
  log_line(buf);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

void prof_mark(rijk_ctx* ctx, const char* name) {
  if (!ctx->profiling || ctx->npev >= 13) return;
  if (ctx->npev > 0) ctx->pname[ctx->npev - 1] = name;
  cudaEventRecord(ctx->pev[ctx->npev++], ctx->stream);
}

static void prof_begin(rijk_ctx* ctx) {
  ctx->npev = 0;
  if (ctx->profiling) cudaEventRecord(ctx->pev[ctx->npev++], ctx->stream);
}

static void prof_collect(rijk_ctx* ctx) {
  ctx->stats.profiled_stages = 0;
  if (!ctx->profiling || ctx->npev < 2) return;
  cudaEventSynchronize(ctx->pev[ctx->npev - 1]);
  int k = ctx->npev - 1;
  for (int i = 0; i < k && i < 12; ++i) {
    ctx->stats.ms_stage[i] = elapsed(ctx->pev[i], ctx->pev[i + 1]);
    std::snprintf(ctx->stats.stage_names[i], sizeof(ctx->stats.stage_names[i]), "%s", ctx->pname[i] ? ctx->pname[i] : "?");
  }
  ctx->stats.profiled_stages = k < 12 ? k : 12;
}

int fock_device_impl(rijk_ctx* ctx, const double* dD, const double* dMO, long nocc, double* dJ, double* dK,
                     int precision, cudaEvent_t mo_ready, cudaEvent_t j_done) {
  // naux here is the number of aux functions this context holds (a slice under rijk_set_aux_range)
  const long n = ctx->n, naux = ctx->nq, nt = ctx->nt, npad = ctx->npad, ntile = ctx->ntile;
  const long tile_elems = ntile * TILE2;
  cudaStream_t s = ctx->stream;
  int rc;
  int launches = 0;
  const int nsJ = coulomb_nsplit(tile_elems, naux, precision == RIJK_PREC_MIXED ? 8 : 2);
  if ((rc = ensure(ctx, ctx->Dt, tile_elems * sizeof(double), "Dt")) ||
      (rc = ensure(ctx, ctx->w, (1 + coulomb_w_mixed_chunks(ntile)) * naux * sizeof(double), "w")) ||  // w, partials
      (rc = ensure(ctx, ctx->Jpart, static_cast<size_t>(nsJ) * tile_elems * sizeof(double), "Jpart")))
    return rc;
  if (precision == RIJK_PREC_MIXED && (rc = mixed_prepare(ctx))) return rc;
  // the FP64 exchange's buffers, before anything is queued: growing one drains the streams
  const long noccp = round_up(nocc, 16);
  const long kdim = naux * noccp;
  const bool tc = precision == RIJK_PREC_FP64_TC;
  long kper_tc = 0;
  int nsK = 1;
  if (nocc > 0 && precision != RIJK_PREC_MIXED) {
    nsK = tc ? syrk_i8_parts(nt, kdim, ctx->device, &kper_tc) : syrk_nsplit(nt, kdim);
    if ((rc = ensure(ctx, ctx->MOp, noccp * npad * sizeof(double), "MOp")) ||
        (rc = ensure(ctx, ctx->XT, static_cast<size_t>(npad) * kdim * sizeof(double), "XT")) ||
        (rc = ensure(ctx, ctx->Kpart, static_cast<size_t>(nsK) * tile_elems * sizeof(double), "Kpart")))
      return rc;
  }
  // FP64 and FP64_TC: the Coulomb pair runs on the high-priority stream beside the half-transform, one
  // 256-thread CTA per SM, in the registers and warps the half-transform's two CTAs per SM leave free;
  // the pair is bound by HBM, the half-transform by the FP64 tensor pipe.  With per-kernel timing on,
  // the kernels run one after another instead.
  const bool side_j = precision != RIJK_PREC_MIXED && nocc > 0 && !ctx->profiling;
  cudaEventRecord(ctx->ev0, s);
  prof_begin(ctx);
  launch_pack_density(dD, n, npad, nt, static_cast<double*>(ctx->Dt.p), s);
  prof_mark(ctx, "pack_density");
  // The pair's CTAs (one or two an SM): the half-transform's time per byte of B grows with the orbitals,
  // so fewer orbitals leave a shorter window for the same bytes
  const int side_ctas = noccp <= 96 ? 2 * ctx->sms : ctx->sms;
  if (side_j) {
    cudaStream_t js = ctx->j_stream;
    cudaEventRecord(ctx->ev_pk, s);
    cudaStreamWaitEvent(js, ctx->ev_pk, 0);
    launch_coulomb_w(static_cast<const double*>(ctx->B.p), static_cast<const double*>(ctx->Dt.p), naux, tile_elems,
                     static_cast<double*>(ctx->w.p), js, side_ctas);
    // the same aux ranges as the pass run alone, so J's sums are the same
    launch_coulomb_j(static_cast<const double*>(ctx->B.p), static_cast<const double*>(ctx->w.p), naux, tile_elems, nsJ,
                     static_cast<double*>(ctx->Jpart.p), js, side_ctas);
    launch_unpack_sym(static_cast<double*>(ctx->Jpart.p), nsJ, ntile, n, dJ, js);
    launches += 4 + (nsJ > 1 ? 1 : 0);  // pack, w, j, unpack (+ split sum)
    cudaEventRecord(ctx->ev1, js);
    if (j_done) cudaEventRecord(j_done, js);
    cudaEventRecord(ctx->ev_jside, js);
  } else if (precision == RIJK_PREC_MIXED) {
    // mixed form: both passes over the split-BF16 copy (half the bytes of the FP64 passes)
    const long ntile2 = round_up(nt, 2) * (round_up(nt, 2) + 1) / 2;
    const __nv_bfloat16* Bm = static_cast<const __nv_bfloat16*>(ctx->Bmix.p);
    launch_coulomb_w_mixed(Bm, static_cast<const double*>(ctx->Dt.p), naux, ntile, ntile2,
                           static_cast<double*>(ctx->w.p), s);
    prof_mark(ctx, "coulomb_w_mixed");
    launch_coulomb_j_mixed(Bm, static_cast<const double*>(ctx->w.p), naux, ntile, ntile2, nsJ,
                           static_cast<double*>(ctx->Jpart.p), s);
    prof_mark(ctx, "coulomb_j_mixed");
  } else {
    launch_coulomb_w(static_cast<const double*>(ctx->B.p), static_cast<const double*>(ctx->Dt.p), naux, tile_elems,
                     static_cast<double*>(ctx->w.p), s);
    prof_mark(ctx, "coulomb_w");
    launch_coulomb_j(static_cast<const double*>(ctx->B.p), static_cast<const double*>(ctx->w.p), naux, tile_elems,
                     nsJ, static_cast<double*>(ctx->Jpart.p), s);
    prof_mark(ctx, "coulomb_j");
  }
  if (!side_j) {
    launch_unpack_sym(static_cast<double*>(ctx->Jpart.p), nsJ, ntile, n, dJ, s);
    prof_mark(ctx, "unpack_j");
    launches += (precision == RIJK_PREC_MIXED ? 5 : 4) + (nsJ > 1 ? 1 : 0);  // pack, w (+ chunk sum), j, unpack (+ split sum)
    cudaEventRecord(ctx->ev1, s);
    if (j_done) cudaEventRecord(j_done, s);
  }
  if (mo_ready && nocc > 0) cudaStreamWaitEvent(s, mo_ready, 0);

  if (nocc == 0) {
    cudaMemsetAsync(dK, 0, n * n * sizeof(double), s);
  } else if (precision == RIJK_PREC_MIXED) {
    rc = mixed_exchange(ctx, dMO, nocc, dK);
    if (rc) return rc;
    launches += ctx->stats.kernels_last_fock;
  } else {
    // About 20 us, so that the Coulomb CTAs, whose stream waits on an event, are resident before the
    // half-transform's thousands of CTAs queue (builds queued back to back: 240.5 -> 235.2 ms at
    // n_ao = 1856, where the pair alone takes 17.7 ms)
    if (side_j) {
      launch_delay(40000, s);
      ++launches;
    }
    launch_pack_mo(dMO, nocc, n, noccp, npad, static_cast<double*>(ctx->MOp.p), s);
    prof_mark(ctx, "pack_mo");
    launches += launch_xform_f64(static_cast<const double*>(ctx->B.p), static_cast<const double*>(ctx->MOp.p), naux,
                                 nt, noccp, static_cast<double*>(ctx->XT.p), s);
    prof_mark(ctx, "xform_f64");
    if (tc) {  // int8 digit planes of X^T, then K on tcgen05 (exact s32 products)
      rc = syrk_i8(ctx, static_cast<const double*>(ctx->XT.p), npad, nt, kdim, nsK, kper_tc,
                   static_cast<double*>(ctx->Kpart.p), s);
      if (rc) {
        if (side_j) cudaStreamWaitEvent(s, ctx->ev_jside, 0);  // nothing of the side stream outlives the call
        return rc;
      }
      prof_mark(ctx, "syrk_i8");
      ++launches;  // the digit-plane pass
    } else {
      launch_syrk_f64(static_cast<const double*>(ctx->XT.p), npad, nt, kdim, nsK, static_cast<double*>(ctx->Kpart.p),
                      s);
      prof_mark(ctx, "syrk_f64");
    }
    launch_unpack_sym(static_cast<double*>(ctx->Kpart.p), nsK, ntile, n, dK, s);
    prof_mark(ctx, "unpack_k");
    launches += 3 + (nsK > 1 ? 1 : 0);  // pack_mo, syrk, unpack (+ split sum); the half-transform counted above
  }
  if (side_j) cudaStreamWaitEvent(s, ctx->ev_jside, 0);  // J joins the build's stream
  cudaEventRecord(ctx->ev2, s);
  rc = cuda_check(ctx, cudaGetLastError(), "fock launch");
  if (rc) return rc;
  const double noccd = static_cast<double>(nocc);
  ctx->stats.flops_last_fock = 4.0 * static_cast<double>(tile_elems) * naux +
                               2.0 * noccd * npad * npad * naux + static_cast<double>(npad) * (npad + TILE) * noccd * naux;
  ctx->stats.bytes_last_fock = 2.0 * static_cast<double>(tile_elems) * naux *
                               (precision == RIJK_PREC_MIXED ? 2 * sizeof(__nv_bfloat16) : sizeof(double));
  ctx->stats.kernels_last_fock = launches;
  prof_collect(ctx);
  return RIJK_OK;
}

}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_create(rijk_ctx** out, int device) {
  if (!out) return RIJK_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RIJK_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return RIJK_ERR_ARG;
  rijk_ctx* ctx = new rijk_ctx;
  ctx->device = device;
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return RIJK_ERR_CUDA;
  }
  ctx->own_stream = true;
  if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    rijk_destroy(ctx);
    return RIJK_ERR_CUDA;
  }
  cudaEventCreateWithFlags(&ctx->ev_mo, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_j, cudaEventDisableTiming);
  {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&ctx->j_stream, cudaStreamNonBlocking, greatest) != cudaSuccess) {
      rijk_destroy(ctx);
      return RIJK_ERR_CUDA;
    }
  }
  cudaEventCreateWithFlags(&ctx->ev_pk, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_jside, cudaEventDisableTiming);
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  if (ctx->sms <= 0) ctx->sms = 148;
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  cudaEventCreate(&ctx->ev2);
  cudaEventCreate(&ctx->ev3);
  if (cublasCreate(&ctx->cublas) != CUBLAS_STATUS_SUCCESS || cusolverDnCreate(&ctx->cusolver) != CUSOLVER_STATUS_SUCCESS) {
    rijk_destroy(ctx);
    return RIJK_ERR_CUDA;
  }
  cublasSetStream(ctx->cublas, ctx->stream);
  cusolverDnSetStream(ctx->cusolver, ctx->stream);
  if (int rc = rijk::noalloc_resolve(ctx)) {
    rijk_destroy(ctx);
    return rc;
  }
  if (ensure(ctx, ctx->err, sizeof(int), "err")) {
    rijk_destroy(ctx);
    return RIJK_ERR_ALLOC;
  }
  cudaMemsetAsync(ctx->err.p, 0, sizeof(int), ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  *out = ctx;
  return RIJK_OK;
}

RIJK_API int rijk_destroy(rijk_ctx* ctx) {
  if (!ctx) return RIJK_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);  // before any buffer it may touch is freed
  if (ctx->j_stream) cudaStreamSynchronize(ctx->j_stream);
  DeviceBuf* bufs[] = {&ctx->M,  &ctx->B,     &ctx->Bmix,  &ctx->stageD, &ctx->stageMO, &ctx->stageJ,
                       &ctx->stageK, &ctx->Dt, &ctx->w,     &ctx->Jpart, &ctx->MOp,    &ctx->XT,
                       &ctx->Kpart, &ctx->err, &ctx->scratch, &ctx->eri_tab, &ctx->Xs, &ctx->Xe,
                       &ctx->s3.raw};
  for (DeviceBuf* b : bufs) release(*b);
  for (DeviceBuf& b : ctx->scf) release(b);
  if (ctx->cublas) cublasDestroy(ctx->cublas);
  if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->j_stream) cudaStreamDestroy(ctx->j_stream);
  cudaEvent_t evs[] = {ctx->ev0, ctx->ev1, ctx->ev2, ctx->ev3, ctx->ev_mo, ctx->ev_j, ctx->ev_pk, ctx->ev_jside};
  for (cudaEvent_t ev : evs)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : ctx->pev)
    if (ev) cudaEventDestroy(ev);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return RIJK_OK;
}

RIJK_API int rijk_set_stream(rijk_ctx* ctx, void* stream) {
  if (!ctx) return RIJK_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // work queued on the old stream ends first
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = s;
  ctx->own_stream = false;
  cublasSetStream(ctx->cublas, s);
  cusolverDnSetStream(ctx->cusolver, s);
  return RIJK_OK;
}

RIJK_API int rijk_last_error(const rijk_ctx* ctx, char* buf, int len) {
  if (!ctx || !buf || len <= 0) return RIJK_ERR_ARG;
  std::snprintf(buf, static_cast<size_t>(len), "%s", ctx->last_error.c_str());
  return RIJK_OK;
}

RIJK_API int rijk_set_profiling(rijk_ctx* ctx, int on) {
  if (!ctx) return RIJK_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (on && !ctx->pev[0])
    for (cudaEvent_t& e : ctx->pev) cudaEventCreate(&e);
  ctx->profiling = on != 0;
  return RIJK_OK;
}

RIJK_API int rijk_get_stats(const rijk_ctx* ctx, rijk_stats_t* out) {
  if (!ctx || !out) return RIJK_ERR_ARG;
  *out = ctx->stats;
  out->q0 = ctx->q0;
  out->nq = ctx->nq;
  return RIJK_OK;
}

RIJK_API int rijk_set_aux_range(rijk_ctx* ctx, long q0, long q1) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!ctx->have_metric) return set_err(ctx, RIJK_ERR_STATE, "rijk_set_aux_range: call rijk_set_metric first");
  if (q0 < 0 || q1 <= q0 || q1 > ctx->naux)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_set_aux_range: [%ld, %ld) not inside [0, %ld)", q0, q1, ctx->naux);
  cudaSetDevice(ctx->device);
  stream3c_cancel(ctx);
  ctx->q0 = q0;
  ctx->nq = q1 - q0;
  ctx->have_b = false;
  ctx->have_bmix = false;
  return RIJK_OK;
}

RIJK_API int rijk_set_metric(rijk_ctx* ctx, const double* PQ, long naux, int form) {
  if (!ctx) return RIJK_ERR_ARG;
  NvtxRange range("rijk_set_metric");
  return set_metric_impl(ctx, PQ, cudaMemcpyHostToDevice, naux, form);
}

namespace rijk {
int set_metric_impl(rijk_ctx* ctx, const double* PQ, cudaMemcpyKind kind, long naux, int form) {
  if (!PQ || naux <= 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_metric: null (P|Q) or naux <= 0");
  if (naux > 65535) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_metric: naux = %ld exceeds 65535", naux);
  if (form != RIJK_METRIC_INVSQRT && form != RIJK_METRIC_CHOLESKY)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_set_metric: unknown metric form %d", form);
  cudaSetDevice(ctx->device);
  stream3c_cancel(ctx);  // a new metric ends any streaming three-centre input in progress
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const long nauxp = round_up(naux, KC);
  int rc;
  DeviceBuf V, X, W, work, info;
  auto cleanup = [&]() {
    release(V);
    release(X);
    release(W);
    release(work);
    release(info);
  };
  if ((rc = ensure(ctx, V, naux * naux * sizeof(double), "metric V")) ||
      (rc = ensure(ctx, X, naux * naux * sizeof(double), "metric X")) ||
      (rc = ensure(ctx, W, naux * sizeof(double), "metric w")) || (rc = ensure(ctx, info, 2 * sizeof(int), "info")) ||
      (rc = ensure(ctx, ctx->M, nauxp * nauxp * sizeof(double), "metric M"))) {
    cleanup();
    return rc;
  }
  cudaEventRecord(ctx->ev0, s);
  rc = cuda_check(ctx, cudaMemcpyAsync(V.p, PQ, naux * naux * sizeof(double), kind, s), "copy (P|Q)");
  if (rc) { cleanup(); return rc; }
  cudaMemsetAsync(info.p, 0, 2 * sizeof(int), s);
  double* dV = static_cast<double*>(V.p);
  double* dX = static_cast<double*>(X.p);
  int* dinfo = static_cast<int*>(info.p);
  const int na = static_cast<int>(naux);
  if (form == RIJK_METRIC_INVSQRT) {
    int lwork = 0;
    if (cusolverDnDsyevd_bufferSize(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, na, dV, na,
                                    static_cast<double*>(W.p), &lwork) != CUSOLVER_STATUS_SUCCESS) {
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "syevd buffer query failed");
    }
    if ((rc = ensure(ctx, work, static_cast<size_t>(lwork) * sizeof(double), "syevd work"))) { cleanup(); return rc; }
    if (cusolverDnDsyevd(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, na, dV, na,
                         static_cast<double*>(W.p), static_cast<double*>(work.p), lwork, dinfo) != CUSOLVER_STATUS_SUCCESS) {
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "syevd failed");
    }
    // X = U diag(f) ; M = X U^T
    cudaMemcpyAsync(dX, dV, naux * naux * sizeof(double), cudaMemcpyDeviceToDevice, s);
    k_scale_eigvecs<<<grid1d(naux * naux), 256, 0, s>>>(dX, static_cast<const double*>(W.p), naux, dinfo + 1);
    const double one = 1.0, zero = 0.0;
    DeviceBuf Mt;
    if ((rc = ensure(ctx, Mt, naux * naux * sizeof(double), "metric tmp"))) { cleanup(); return rc; }
    cublasStatus_t st = cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_T, na, na, na, &one, dX, na, dV, na, &zero,
                                    static_cast<double*>(Mt.p), na);
    if (st != CUBLAS_STATUS_SUCCESS) {
      release(Mt);
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "dgemm for V^-1/2 failed");
    }
    k_pad_from_colmajor<<<grid1d(nauxp * nauxp), 256, 0, s>>>(static_cast<const double*>(Mt.p), naux,
                                                               static_cast<double*>(ctx->M.p), nauxp);
    cudaStreamSynchronize(s);
    release(Mt);
  } else {
    int lwork = 0;
    if (cusolverDnDpotrf_bufferSize(ctx->cusolver, CUBLAS_FILL_MODE_LOWER, na, dV, na, &lwork) !=
        CUSOLVER_STATUS_SUCCESS) {
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "potrf buffer query failed");
    }
    if ((rc = ensure(ctx, work, static_cast<size_t>(lwork) * sizeof(double), "potrf work"))) { cleanup(); return rc; }
    if (cusolverDnDpotrf(ctx->cusolver, CUBLAS_FILL_MODE_LOWER, na, dV, na, static_cast<double*>(work.p), lwork,
                         dinfo) != CUSOLVER_STATUS_SUCCESS) {
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "potrf failed");
    }
    k_identity<<<grid1d(naux * naux), 256, 0, s>>>(dX, naux);
    const double one = 1.0;
    if (cublasDtrsm(ctx->cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, na, na,
                    &one, dV, na, dX, na) != CUBLAS_STATUS_SUCCESS) {
      cleanup();
      return set_err(ctx, RIJK_ERR_SOLVER, "trsm for L^-1 failed");
    }
    k_pad_from_colmajor<<<grid1d(nauxp * nauxp), 256, 0, s>>>(dX, naux, static_cast<double*>(ctx->M.p), nauxp);
  }
  cudaEventRecord(ctx->ev1, s);
  int hinfo[2] = {0, 0};
  rc = cuda_check(ctx, cudaMemcpyAsync(hinfo, dinfo, 2 * sizeof(int), cudaMemcpyDeviceToHost, s), "info D2H");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(s), "set_metric");
  cleanup();
  if (rc) return rc;
  if (hinfo[0] != 0)
    return set_err(ctx, RIJK_ERR_SOLVER, "metric factorisation failed (info = %d): (P|Q) not positive definite?",
                   hinfo[0]);
  ctx->stats.ms_setup_metric = elapsed(ctx->ev0, ctx->ev1);
  ctx->naux = naux;
  ctx->q0 = 0;
  ctx->nq = naux;
  ctx->metric_form = form;
  ctx->have_metric = true;
  ctx->have_b = false;
  ctx->have_bmix = false;
  ctx->stats.naux = naux;
  if (hinfo[1] > 0) ctx->last_error = "warning: metric eigenvalues <= 0 dropped";
  return RIJK_OK;
}
}  // namespace rijk

RIJK_API int rijk_set_3c(rijk_ctx* ctx, const double* I3, long n, long naux, int layout) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!I3 || n <= 0 || naux <= 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_3c: null integrals or bad sizes");
  NvtxRange range("rijk_set_3c");
  cudaStream_t s = ctx->stream;
  return set_3c_impl(ctx, n, naux, layout, [&](long, long, long first, long count, double* raw, long ld) {
    if (count <= 0) return static_cast<int>(RIJK_OK);
    return cuda_check(ctx,
                      cudaMemcpy2DAsync(raw, ld * sizeof(double), I3 + first * naux, naux * sizeof(double),
                                        naux * sizeof(double), static_cast<size_t>(count), cudaMemcpyHostToDevice, s),
                      "H2D three-centre block");
  });
}

namespace rijk {
long rows_per_chunk(long n, long nauxp, int layout) {
  const long npad = round_up(n, TILE), nt = npad / TILE;
  const double budget = 2.0 * 1024 * 1024 * 1024;
  const long rows = std::max<long>(1, static_cast<long>(budget / (static_cast<double>(TILE) *
                                                                  (layout == RIJK_LAYOUT_NOPT_FULL ? n : npad) *
                                                                  nauxp * 8.0)));
  return std::min(rows, nt);
}

void pair_rows(int layout, long n, long mu0, long mu1, long* first, long* count) {
  if (layout == RIJK_LAYOUT_NOPT_FULL) {
    *first = mu0 * n;
    *count = (mu1 - mu0) * n;
  } else {
    *first = mu0 * (mu0 + 1) / 2;
    *count = mu1 * (mu1 + 1) / 2 - *first;
  }
}

int set_3c_impl(rijk_ctx* ctx, long n, long naux, int layout, const ChunkFill& fill) {
  if (n <= 0 || naux <= 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_3c: bad sizes");
  if (layout != RIJK_LAYOUT_NOPT_FULL && layout != RIJK_LAYOUT_PACKED)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_set_3c: unknown layout %d", layout);
  if (!ctx->have_metric) return set_err(ctx, RIJK_ERR_STATE, "rijk_set_3c: call rijk_set_metric first");
  if (naux != ctx->naux)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_set_3c: naux %ld differs from the metric's %ld", naux, ctx->naux);
  cudaSetDevice(ctx->device);
  stream3c_cancel(ctx);
  cudaStream_t s = ctx->stream;
  const long npad = round_up(n, TILE), nt = npad / TILE, ntile = nt * (nt + 1) / 2;
  const long nauxp = round_up(naux, KC);
  const long nq = ctx->nq, q0 = ctx->q0;
  int rc;
  ctx->have_b = false;
  ctx->have_bmix = false;
  release(ctx->Bmix);
  if ((rc = ensure(ctx, ctx->B, static_cast<size_t>(nq) * ntile * TILE2 * sizeof(double), "fitted tensor B")))
    return rc;
  // Raw integrals come in blocks of whole tile rows, at most ~2 GiB each.
  const long rows_per = rows_per_chunk(n, nauxp, layout);
  auto pairs_of = [&](long I0, long I1, long& first, long& count) {
    pair_rows(layout, n, I0 * TILE, std::min(I1 * TILE, n), &first, &count);
  };
  long maxcount = 0;
  for (long I0 = 0; I0 < nt; I0 += rows_per) {
    long f, c;
    pairs_of(I0, std::min(nt, I0 + rows_per), f, c);
    maxcount = std::max(maxcount, c);
  }
  DeviceBuf raw;
  if ((rc = ensure(ctx, raw, static_cast<size_t>(std::max<long>(maxcount, 1)) * nauxp * sizeof(double), "raw 3c block")))
    return rc;
  cudaMemsetAsync(raw.p, 0, raw.bytes, s);
  cudaMemsetAsync(ctx->B.p, 0, static_cast<size_t>(nq) * ntile * TILE2 * sizeof(double), s);
  float ms = 0.f;
  for (long I0 = 0; I0 < nt; I0 += rows_per) {
    long I1 = std::min(nt, I0 + rows_per);
    long first, count;
    pairs_of(I0, I1, first, count);
    rc = fill(I0 * TILE, std::min(I1 * TILE, n), first, count, static_cast<double*>(raw.p), nauxp);
    if (rc) { release(raw); return rc; }
    cudaEventRecord(ctx->ev0, s);
    launch_metric_contract_chunk(static_cast<const double*>(ctx->M.p) + q0 * nauxp, nauxp, nauxp - q0,
                                 static_cast<const double*>(raw.p), layout, n, nq, nt, I0, I1,
                                 static_cast<double*>(ctx->B.p), s,
                                 ctx->metric_form == RIJK_METRIC_CHOLESKY ? q0 : -1);
    cudaEventRecord(ctx->ev1, s);
    rc = cuda_check(ctx, cudaStreamSynchronize(s), "metric contraction");
    if (rc) { release(raw); return rc; }
    ms += elapsed(ctx->ev0, ctx->ev1);
  }
  release(raw);
  ctx->n = n;
  ctx->npad = npad;
  ctx->nt = nt;
  ctx->ntile = ntile;
  ctx->have_b = true;
  ctx->stats.ms_setup_3c = ms;
  ctx->stats.n = n;
  ctx->stats.npad = npad;
  ctx->stats.ntile = ntile;
  ctx->stats.bytes_b = nq * ntile * TILE2 * static_cast<long>(sizeof(double));
  ctx->stats.bytes_b_mixed = 0;
  return RIJK_OK;
}
}  // namespace rijk

namespace rijk {
// Reads and clears the device error word the kernels raise instead of trapping.
int check_device_error(rijk_ctx* ctx) {
  int h = 0;
  int rc = cuda_check(ctx, cudaMemcpy(&h, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost), "error word");
  if (rc) return rc;
  if (h == 0) return RIJK_OK;
  cudaMemsetAsync(ctx->err.p, 0, sizeof(int), ctx->stream);  // ordered before the next launch
  if (h & DEVERR_TIMEOUT) return set_err(ctx, RIJK_ERR_TIMEOUT, "a device-side wait ran out (error bits 0x%x)", h);
  if (h & DEVERR_NAN) return set_err(ctx, RIJK_ERR_NUMERIC, "non-finite value detected (error bits 0x%x)", h);
  return set_err(ctx, RIJK_ERR_CUDA, "device error bits 0x%x", h);
}
}  // namespace rijk

RIJK_API int rijk_sync(rijk_ctx* ctx) {
  if (!ctx) return RIJK_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "rijk_sync");
  if (rc) return rc;
  rc = check_device_error(ctx);
  if (rc) return rc;
  ctx->stats.ms_coulomb = elapsed(ctx->ev0, ctx->ev1);
  ctx->stats.ms_exchange = elapsed(ctx->ev1, ctx->ev2);
  ctx->stats.ms_last_fock = elapsed(ctx->ev0, ctx->ev2);
  if (ctx->log_pending) {
    ctx->log_pending = false;
    log_build(ctx, "rijk_fock_device", ctx->log_nocc, ctx->log_precision);
  }
  return RIJK_OK;
}

namespace rijk {
int check_fock_args(rijk_ctx* ctx, long nocc, int precision) {
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "Fock build before rijk_set_3c");
  if (nocc < 0 || nocc > round_up(ctx->n, 16))
    return set_err(ctx, RIJK_ERR_ARG, "n_c = %ld outside [0, n_ao = %ld]", nocc, ctx->n);
  if (precision != RIJK_PREC_FP64 && precision != RIJK_PREC_MIXED && precision != RIJK_PREC_FP64_TC)
    return set_err(ctx, RIJK_ERR_ARG, "unknown precision %d", precision);
  return RIJK_OK;
}
}  // namespace rijk

RIJK_API int rijk_fock_device(rijk_ctx* ctx, const double* dD, const double* dMO, long nocc, double* dJ, double* dK,
                              int precision) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!dD || !dJ || !dK || (nocc > 0 && !dMO)) return set_err(ctx, RIJK_ERR_ARG, "rijk_fock_device: null pointer");
  int rc = check_fock_args(ctx, nocc, precision);
  if (rc) return rc;
  NvtxRange range("rijk_fock_device");
  cudaSetDevice(ctx->device);
  rc = fock_device_impl(ctx, dD, dMO, nocc, dJ, dK, precision);
  if (!rc) {
    ctx->log_pending = true;
    ctx->log_nocc = nocc;
    ctx->log_precision = precision;
  }
  return rc;
}

RIJK_API int rijk_fock(rijk_ctx* ctx, const double* D, const double* MO, long nocc, double* J, double* K,
                       int precision) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!D || !J || !K || (nocc > 0 && !MO)) return set_err(ctx, RIJK_ERR_ARG, "rijk_fock: null pointer");
  int rc = check_fock_args(ctx, nocc, precision);
  if (rc) return rc;
  NvtxRange range("rijk_fock");
  cudaSetDevice(ctx->device);
  const long n = ctx->n;
  const size_t nn = static_cast<size_t>(n) * n * sizeof(double);
  if ((rc = ensure(ctx, ctx->stageD, nn, "stage D")) || (rc = ensure(ctx, ctx->stageJ, nn, "stage J")) ||
      (rc = ensure(ctx, ctx->stageK, nn, "stage K")) ||
      (rc = ensure(ctx, ctx->stageMO, std::max<size_t>(1, nocc * n * sizeof(double)), "stage MO")))
    return rc;
  cudaStream_t s = ctx->stream, c = ctx->copy_stream;
  // D on the build's stream; the orbitals on the copy stream (the Coulomb passes do not need
  // them); J comes down on the copy stream while the exchange runs; K on the build's stream.
  // Both staging areas are free: the previous call ended with both streams synchronised.
  rc = cuda_check(ctx, cudaMemcpyAsync(ctx->stageD.p, D, nn, cudaMemcpyHostToDevice, s), "H2D D");
  if (!rc && nocc > 0) {
    rc = cuda_check(ctx, cudaMemcpyAsync(ctx->stageMO.p, MO, nocc * n * sizeof(double), cudaMemcpyHostToDevice, c),
                    "H2D MO");
    if (!rc) cudaEventRecord(ctx->ev_mo, c);
  }
  if (rc) return rc;
  rc = fock_device_impl(ctx, static_cast<const double*>(ctx->stageD.p), static_cast<const double*>(ctx->stageMO.p),
                        nocc, static_cast<double*>(ctx->stageJ.p), static_cast<double*>(ctx->stageK.p), precision,
                        nocc > 0 ? ctx->ev_mo : nullptr, ctx->ev_j);
  if (rc) {
    cudaStreamSynchronize(c);
    return rc;
  }
  cudaStreamWaitEvent(c, ctx->ev_j, 0);
  rc = cuda_check(ctx, cudaMemcpyAsync(J, ctx->stageJ.p, nn, cudaMemcpyDeviceToHost, c), "D2H J");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(K, ctx->stageK.p, nn, cudaMemcpyDeviceToHost, s), "D2H K");
  const int rc_c = cuda_check(ctx, cudaStreamSynchronize(c), "rijk_fock copies");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_fock");
  if (!rc) rc = rc_c;
  if (!rc) rc = check_device_error(ctx);
  if (rc) return rc;
  ctx->stats.ms_coulomb = elapsed(ctx->ev0, ctx->ev1);
  ctx->stats.ms_exchange = elapsed(ctx->ev1, ctx->ev2);
  ctx->stats.ms_last_fock = elapsed(ctx->ev0, ctx->ev2);
  ctx->log_pending = false;
  log_build(ctx, "rijk_fock", nocc, precision);
  return RIJK_OK;
}

RIJK_API int rijk_fock_energy(rijk_ctx* ctx, const double* H, const double* DM, const double* J, const double* K,
                              double c, int mc, double e_nuc, double* F, double* E) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!H || !J || !K || (E && !DM)) return set_err(ctx, RIJK_ERR_ARG, "rijk_fock_energy: null pointer");
  if (mc < 0 || mc > 2) return set_err(ctx, RIJK_ERR_ARG, "rijk_fock_energy: mc must be 0, 1 or 2");
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "rijk_fock_energy before rijk_set_3c");
  cudaSetDevice(ctx->device);
  const long n = ctx->n;
  const size_t nn = static_cast<size_t>(n) * n * sizeof(double);
  int rc;
  DeviceBuf dH, dJ, dK, dF;
  auto cleanup = [&]() { release(dH); release(dJ); release(dK); release(dF); };
  if ((rc = ensure(ctx, dH, nn, "H")) || (rc = ensure(ctx, dJ, nn, "J")) || (rc = ensure(ctx, dK, nn, "K")) ||
      (rc = ensure(ctx, dF, nn, "F"))) {
    cleanup();
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaMemcpyAsync(dH.p, H, nn, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dJ.p, J, nn, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dK.p, K, nn, cudaMemcpyHostToDevice, s);
  // mc = 0, 2: F = H + (2J - K) c ;  mc = 1: F = H + (J - K) 2c
  const double cj = 2.0 * c, ck = (mc == 1) ? 2.0 * c : c;
  k_fock_matrix<<<grid1d(n * n), 256, 0, s>>>(static_cast<const double*>(dH.p), static_cast<const double*>(dJ.p),
                                              static_cast<const double*>(dK.p), cj, ck, n * n,
                                              static_cast<double*>(dF.p));
  std::vector<double> Fh(static_cast<size_t>(n) * n);
  rc = cuda_check(ctx, cudaMemcpyAsync(Fh.data(), dF.p, nn, cudaMemcpyDeviceToHost, s), "D2H F");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_fock_energy");
  cleanup();
  if (rc) return rc;
  if (F) std::memcpy(F, Fh.data(), nn);
  if (E) {
    // E_1el_calc(X, D) = sum_ij D[i + n j] X[i n + j]  (src/doCI_matr.cpp:38-47)
    double e = e_nuc;
    for (long i = 0; i < n; ++i)
      for (long j = 0; j < n; ++j) e += DM[i + n * j] * (Fh[i * n + j] + H[i * n + j]);
    *E = e;
  }
  return RIJK_OK;
}
