// k_moints.cu — active-space MO integrals from the fitted tensor (rijk_mo_ints), the drop-in for
// calc_2el_MO_INTS_RI (src/RI.cpp:178-292), which the CASSCF engine calls each macro-iteration
// (src/CAS.cpp:461) and the CDAS/XMC perturbation codes call once (src/CDAS_PT.cpp:246).
//
// The reference forms RI_aA = C1 (mu nu|P), applies V^-1/2, transposes, contracts with C2 and
// takes MO_INTS = RI_aa RI_aa^T over the aux index.  With B already fitted:
//     Y^Q = C1 B^Q C2^T  (n_a x n_a),   MO_INTS[(b n_a + a) n_a^2 + d n_a + c] = sum_Q Y^Q_ab Y^Q_cd
// (a, c from MO_VEC1; b, d from MO_VEC2, as the reference's RI_aa index order (b, a)).
// Device work: the FP64 half-transform kernel (C1 as the orbital block), a batched DMMA GEMM
// (k_gemm.cu) with one product per aux function for Y^Q, one GEMM Z Z^T over Q, and a gather into
// the reference's order.
// The core J and K come from the ordinary FP64 Fock build with D_core and the first n_c rows of
// MO_VEC, exactly the reference's tail (src/RI.cpp:235-287).
#include <vector>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

// rows[i][mu] = C[i][mu] (t = 0, C is n_a x n) or C[mu][i] (t = 1, C is n x n_a); zero padded to
// noccp x npad.
__global__ void k_rows_from(const double* __restrict__ C, int t, long na, long n, long noccp, long npad,
                            double* __restrict__ rows) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < noccp * npad; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long i = idx / npad, mu = idx % npad;
    double v = 0.0;
    if (i < na && mu < n) v = t ? C[mu * na + i] : C[i * n + mu];
    rows[idx] = v;
  }
}

// out[(b na + a) na^2 + d na + c] = G[(a + b p) + (c + d p) * p^2], p = noccp (column-major G)
__global__ void k_gather_moints(const double* __restrict__ G, long na, long p, double* __restrict__ out) {
  const long na2 = na * na, p2 = p * p;
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < na2 * na2; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long r = idx / na2, c2 = idx % na2;
    long b = r / na, a = r % na, d = c2 / na, c = c2 % na;
    out[idx] = G[(a + b * p) + (c + d * p) * p2];
  }
}

unsigned grid_of(long total) {
  long blocks = (total + 255) / 256;
  if (blocks > 148L * 16) blocks = 148L * 16;
  return static_cast<unsigned>(blocks < 1 ? 1 : blocks);
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_mo_ints(rijk_ctx* ctx, const double* DM_D, double* J, double* K, double* MO_INTS,
                          const double* MO_VEC, const double* MO_VEC1, const double* MO_VEC2, long n_c, long n_a,
                          long t) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!MO_INTS || !MO_VEC1 || !MO_VEC2 || n_a < 1) return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_ints: bad arguments");
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "rijk_mo_ints before rijk_set_3c");
  if (n_a > ctx->n) return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_ints: n_a = %ld exceeds n_ao", n_a);
  const bool want_jk = (J != nullptr && K != nullptr);
  if (want_jk && (!DM_D || (n_c > 0 && !MO_VEC))) return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_ints: D or MO missing");
  if (want_jk) {
    int rc0 = check_fock_args(ctx, n_c, RIJK_PREC_FP64);
    if (rc0) return rc0;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const long n = ctx->n, naux = ctx->nq, npad = ctx->npad, nt = ctx->nt;
  const long p = round_up(n_a, 16), kdim = naux * p, p2 = p * p;
  const size_t cbytes = static_cast<size_t>(n_a) * n * sizeof(double);
  int rc;
  DeviceBuf dC1, dC2, R1, R2, XTa, Y, G, out;
  auto cleanup = [&]() {
    DeviceBuf* all[] = {&dC1, &dC2, &R1, &R2, &XTa, &Y, &G, &out};
    for (DeviceBuf* b : all) release(*b);
  };
  auto chk = [&](int r) {
    if (r) cleanup();
    return r;
  };
  if ((rc = chk(ensure(ctx, dC1, cbytes, "mo_ints C1"))) || (rc = chk(ensure(ctx, dC2, cbytes, "mo_ints C2"))) ||
      (rc = chk(ensure(ctx, R1, p * npad * sizeof(double), "mo_ints rows1"))) ||
      (rc = chk(ensure(ctx, R2, p * npad * sizeof(double), "mo_ints rows2"))) ||
      (rc = chk(ensure(ctx, XTa, static_cast<size_t>(npad) * kdim * sizeof(double), "mo_ints XT"))) ||
      (rc = chk(ensure(ctx, Y, static_cast<size_t>(naux) * p2 * sizeof(double), "mo_ints Y"))) ||
      (rc = chk(ensure(ctx, G, static_cast<size_t>(p2) * p2 * sizeof(double), "mo_ints G"))) ||
      (rc = chk(ensure(ctx, out, static_cast<size_t>(n_a * n_a) * n_a * n_a * sizeof(double), "mo_ints out"))))
    return rc;
  cudaMemcpyAsync(dC1.p, MO_VEC1, cbytes, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dC2.p, MO_VEC2, cbytes, cudaMemcpyHostToDevice, s);
  k_rows_from<<<grid_of(p * npad), 256, 0, s>>>(static_cast<const double*>(dC1.p), t ? 1 : 0, n_a, n, p, npad,
                                                 static_cast<double*>(R1.p));
  k_rows_from<<<grid_of(p * npad), 256, 0, s>>>(static_cast<const double*>(dC2.p), t ? 1 : 0, n_a, n, p, npad,
                                                 static_cast<double*>(R2.p));
  // X1^Q: XT[nu][Q p + a] = sum_mu B^Q_{nu mu} C1_{a mu}
  launch_xform_f64(static_cast<const double*>(ctx->B.p), static_cast<const double*>(R1.p), naux, nt, p,
                   static_cast<double*>(XTa.p), s);
  {  // Y^Q[b][a] = sum_nu C2_{b nu} X1^Q_{a nu}  (p x p per aux function)
    GemmF64Args g;
    g.M = p, g.N = p, g.K = npad;
    g.A = static_cast<const double*>(R2.p), g.lda = npad, g.sA = 0, g.a_kmajor = true;
    g.B = static_cast<const double*>(XTa.p), g.ldb = kdim, g.sB = p, g.b_kmajor = false;
    g.C = static_cast<double*>(Y.p), g.ldc = p, g.sC = p2;
    gemm_f64(g, naux, s);
  }
  {  // G[x][y] = sum_Q Y^Q[x] Y^Q[y] over the flattened p^2 entries
    GemmF64Args g;
    g.M = p2, g.N = p2, g.K = naux;
    g.A = static_cast<const double*>(Y.p), g.lda = p2, g.a_kmajor = false;
    g.B = static_cast<const double*>(Y.p), g.ldb = p2, g.b_kmajor = false;
    g.C = static_cast<double*>(G.p), g.ldc = p2;
    gemm_f64(g, 1, s);
  }
  k_gather_moints<<<grid_of(n_a * n_a * n_a * n_a), 256, 0, s>>>(static_cast<const double*>(G.p), n_a, p,
                                                                   static_cast<double*>(out.p));
  cudaMemcpyAsync(MO_INTS, out.p, static_cast<size_t>(n_a * n_a) * n_a * n_a * sizeof(double), cudaMemcpyDeviceToHost,
                  s);
  if ((rc = chk(cuda_check(ctx, cudaStreamSynchronize(s), "rijk_mo_ints")))) return rc;
  cleanup();
  if (!want_jk) return RIJK_OK;  // the reference returns here when J or K is NULL (src/RI.cpp:229-232)
  // core J and K: the ordinary Fock build (rijk_fock: D_core, the first n_c rows of MO_VEC)
  return rijk_fock(ctx, DM_D, MO_VEC, n_c, J, K, RIJK_PREC_FP64);
}
