// rijk_stream3c.cu — the fitted tensor from three-centre integrals handed over in blocks of orbital rows
// (rijk_begin_3c / rijk_add_3c_block), for callers whose (mu nu|P) does not fit in host memory at once.
//
// The reference holds the whole raw tensor RI_AA (n^2 naux doubles) in host memory
// (src/RI.cpp:34-79, filled by calc_2el_AO_INTS_RI, src/libint_link.cpp:2261-2350); at (H2O)32 cc-pVTZ
// that is 123 GB.  Here the caller computes (mu nu|P) for a range of orbital rows mu at a time (the
// outer shell loop of calc_2el_AO_INTS_RI) and passes each range as it is done.  The blocks fill the
// same device staging that rijk_set_3c fills, one chunk of whole 64-row tile rows at a time; each
// completed chunk goes through the metric contraction K1 at once.  The chunks and their arithmetic
// are those of rijk_set_3c, so the fitted tensor is bit-identical to the one rijk_set_3c gives.
#include <cuda_runtime.h>

#include <algorithm>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {

void stream3c_cancel(rijk_ctx* ctx) {
  if (!ctx->s3.active && !ctx->s3.raw.p) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  release(ctx->s3.raw);
  ctx->s3.active = false;
}

namespace {

int fail(rijk_ctx* ctx, int rc) {
  stream3c_cancel(ctx);
  ctx->have_b = false;
  return rc;
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_begin_3c(rijk_ctx* ctx, long n, long naux, int layout) {
  if (!ctx) return RIJK_ERR_ARG;
  if (n <= 0 || naux <= 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_begin_3c: bad sizes");
  if (layout != RIJK_LAYOUT_NOPT_FULL && layout != RIJK_LAYOUT_PACKED)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_begin_3c: unknown layout %d", layout);
  if (!ctx->have_metric) return set_err(ctx, RIJK_ERR_STATE, "rijk_begin_3c: call rijk_set_metric first");
  if (naux != ctx->naux)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_begin_3c: naux %ld differs from the metric's %ld", naux, ctx->naux);
  cudaSetDevice(ctx->device);
  stream3c_cancel(ctx);
  cudaStream_t s = ctx->stream;
  const long npad = round_up(n, TILE), nt = npad / TILE, ntile = nt * (nt + 1) / 2;
  const long nauxp = round_up(naux, KC);
  const long nq = ctx->nq;
  ctx->have_b = false;
  ctx->have_bmix = false;
  release(ctx->Bmix);
  int rc;
  if ((rc = ensure(ctx, ctx->B, static_cast<size_t>(nq) * ntile * TILE2 * sizeof(double), "fitted tensor B")))
    return fail(ctx, rc);
  const long rows_per = rows_per_chunk(n, nauxp, layout);
  long maxcount = 0;
  for (long I0 = 0; I0 < nt; I0 += rows_per) {
    long f, c;
    pair_rows(layout, n, I0 * TILE, std::min(std::min(nt, I0 + rows_per) * TILE, n), &f, &c);
    maxcount = std::max(maxcount, c);
  }
  if ((rc = ensure(ctx, ctx->s3.raw, static_cast<size_t>(std::max<long>(maxcount, 1)) * nauxp * sizeof(double),
                   "raw 3c block")))
    return fail(ctx, rc);
  cudaMemsetAsync(ctx->s3.raw.p, 0, ctx->s3.raw.bytes, s);
  cudaMemsetAsync(ctx->B.p, 0, static_cast<size_t>(nq) * ntile * TILE2 * sizeof(double), s);
  ctx->s3.active = true;
  ctx->s3.n = n;
  ctx->s3.naux = naux;
  ctx->s3.layout = layout;
  ctx->s3.rows_per = rows_per;
  ctx->s3.next_mu = 0;
  ctx->s3.chunk_I0 = 0;
  ctx->s3.ms = 0.0;
  return cuda_check(ctx, cudaGetLastError(), "rijk_begin_3c");
}

RIJK_API int rijk_add_3c_block(rijk_ctx* ctx, long mu0, long mu1, const double* block) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!ctx->s3.active) return set_err(ctx, RIJK_ERR_STATE, "rijk_add_3c_block without rijk_begin_3c");
  const long n = ctx->s3.n, naux = ctx->s3.naux;
  const int layout = ctx->s3.layout;
  if (!block) return set_err(ctx, RIJK_ERR_ARG, "rijk_add_3c_block: null block");
  NvtxRange range("rijk_add_3c_block");
  if (mu0 != ctx->s3.next_mu || mu1 <= mu0 || mu1 > n)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_add_3c_block: rows [%ld, %ld) do not continue at row %ld (n_ao = %ld)", mu0,
                   mu1, ctx->s3.next_mu, n);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const long npad = round_up(n, TILE), nt = npad / TILE, ntile = nt * (nt + 1) / 2;
  const long nauxp = round_up(naux, KC);
  const long nq = ctx->nq, q0 = ctx->q0;
  long blk_first, blk_count;
  pair_rows(layout, n, mu0, mu1, &blk_first, &blk_count);
  int rc;
  long r0 = mu0;
  while (r0 < mu1) {
    const long I0 = ctx->s3.chunk_I0, I1 = std::min(nt, I0 + ctx->s3.rows_per);
    const long cmu0 = I0 * TILE, cmu1 = std::min(I1 * TILE, n);
    const long r1 = std::min(mu1, cmu1);
    long cfirst, ccount, f, c;
    pair_rows(layout, n, cmu0, cmu1, &cfirst, &ccount);
    pair_rows(layout, n, r0, r1, &f, &c);
    // pair rows [f, f + c) of the block land at row f - cfirst of the chunk's staging
    rc = cuda_check(ctx,
                    cudaMemcpy2DAsync(static_cast<double*>(ctx->s3.raw.p) + (f - cfirst) * nauxp, nauxp * sizeof(double),
                                      block + (f - blk_first) * naux, naux * sizeof(double), naux * sizeof(double),
                                      static_cast<size_t>(c), cudaMemcpyHostToDevice, s),
                    "H2D three-centre block");
    if (rc) return fail(ctx, rc);
    if (r1 == cmu1) {  // the chunk is complete: contract it with the metric factor
      cudaEventRecord(ctx->ev0, s);
      launch_metric_contract_chunk(static_cast<const double*>(ctx->M.p) + q0 * nauxp, nauxp, nauxp - q0,
                                   static_cast<const double*>(ctx->s3.raw.p), layout, n, nq, nt, I0, I1,
                                   static_cast<double*>(ctx->B.p), s,
                                 ctx->metric_form == RIJK_METRIC_CHOLESKY ? q0 : -1);
      cudaEventRecord(ctx->ev1, s);
      rc = cuda_check(ctx, cudaStreamSynchronize(s), "metric contraction");
      if (rc) return fail(ctx, rc);
      ctx->s3.ms += elapsed(ctx->ev0, ctx->ev1);
      ctx->s3.chunk_I0 = I1;
    }
    r0 = r1;
  }
  // the copies out of the caller's block have landed (pinned blocks included) before the call returns
  rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_add_3c_block");
  if (rc) return fail(ctx, rc);
  ctx->s3.next_mu = mu1;
  if (mu1 < n) return RIJK_OK;
  // the last row: the fitted tensor is complete
  release(ctx->s3.raw);
  ctx->s3.active = false;
  ctx->n = n;
  ctx->npad = npad;
  ctx->nt = nt;
  ctx->ntile = ntile;
  ctx->have_b = true;
  ctx->stats.ms_setup_3c = ctx->s3.ms;
  ctx->stats.n = n;
  ctx->stats.npad = npad;
  ctx->stats.ntile = ntile;
  ctx->stats.bytes_b = nq * ntile * TILE2 * static_cast<long>(sizeof(double));
  ctx->stats.bytes_b_mixed = 0;
  return RIJK_OK;
}
