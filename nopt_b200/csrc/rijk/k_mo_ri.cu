// k_mo_ri.cu — MO-basis fitted tensors from the resident fitted tensor B, the drop-ins for the
// reference's post-SCF RI routines:
//   rijk_mo_tensor        (p a|Q) = sum_{mu nu} C1[p][mu] C2[a][nu] B^Q_{mu nu}, stored [(p n2 + a)][Q]
//   rijk_mo_calc          RI_data::MO_calc (src/RI.cpp:469-587): CC, VC, AA, CA, VA blocks
//   rijk_mo_ints_aaag     calc_2el_MO_INTS_AAAG_RI (src/RI.cpp:294-346): (tu|vx), x over all orbitals
//   rijk_soscf_hess_ints  calc_SOSCF_hess_INTS_RI (src/RI.cpp:348-450): sum_Q (pp|Q)(tu|Q), sum_Q (pt|Q)(pu|Q)
// The reference forms each as C1 (mu nu|P), a product with V^-1/2 over P, a transpose and a
// second product with C2.  Here B (metric already applied, kept in HBM) is half-transformed by
// the FP64 DMMA kernel of the Fock build (X^Q = C2 B^Q, all aux functions per launch), the
// second orbital index comes from one DMMA GEMM over the AO index (k_gemm.cu), and a gather writes the
// reference's index order.  With RIJK_METRIC_INVSQRT the tensors equal the reference's; with the
// Cholesky form they differ by an orthogonal rotation of Q, and every contraction over Q agrees.
#include <algorithm>
#include <vector>

#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

unsigned grid_of(long total) {
  long blocks = (total + 255) / 256;
  if (blocks > 148L * 16) blocks = 148L * 16;
  return static_cast<unsigned>(blocks < 1 ? 1 : blocks);
}

// out[(r n2 + a) naux + Q] = R[r][Q p2 + a], r < nb, a < n2 (order 0);
// out[(a nb + r) naux + Q] = R[r][Q p2 + a] (order 1).
__global__ void k_gather_pa(const double* __restrict__ R, long nb, long n2, long p2, long naux, int order,
                            double* __restrict__ out) {
  const long kdim = naux * p2, total = nb * n2 * naux;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<long>(gridDim.x) * blockDim.x) {
    const long Q = idx % naux, rest = idx / naux;
    long r, a;
    if (order == 0) {
      a = rest % n2;
      r = rest / n2;
    } else {
      r = rest % nb;
      a = rest / nb;
    }
    out[idx] = R[r * kdim + Q * p2 + a];
  }
}

// out[r][Q] = sum_nu XT[nu][Q p2 + r] C[r][nu] for r < nr: the diagonal (rr|Q) of a batch of rows.
__global__ void k_diag_pair(const double* __restrict__ XT, const double* __restrict__ C, long nr, long p2, long naux,
                            long npad, double* __restrict__ out) {
  const long kdim = naux * p2, total = naux * p2;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<long>(gridDim.x) * blockDim.x) {
    const long Q = idx / p2, r = idx % p2;
    if (r >= nr) continue;
    const double* c = C + r * npad;
    double s = 0.0;
    for (long nu = 0; nu < npad; ++nu) s += XT[nu * kdim + Q * p2 + r] * c[nu];
    out[r * naux + Q] = s;
  }
}

// Device scratch of one call; released on every exit.
struct Scratch {
  std::vector<DeviceBuf> bufs;
  ~Scratch() {
    for (DeviceBuf& b : bufs) release(b);
  }
  double* get(rijk_ctx* ctx, size_t doubles, const char* what, int* rc) {
    bufs.emplace_back();
    *rc = ensure(ctx, bufs.back(), std::max<size_t>(doubles, 1) * sizeof(double), what);
    return static_cast<double*>(bufs.back().p);
  }
};

// Orbital rows (host, nr x n) -> device, zero padded to rows x npad.
double* upload_rows(rijk_ctx* ctx, Scratch& sc, const double* C, long nr, long rows, int* rc) {
  const long n = ctx->n, npad = ctx->npad;
  double* raw = sc.get(ctx, static_cast<size_t>(nr) * n, "orbital rows", rc);
  if (*rc) return nullptr;
  double* pad = sc.get(ctx, static_cast<size_t>(rows) * npad, "padded orbital rows", rc);
  if (*rc) return nullptr;
  if (nr > 0) {
    *rc = cuda_check(ctx, cudaMemcpyAsync(raw, C, static_cast<size_t>(nr) * n * sizeof(double), cudaMemcpyHostToDevice,
                                          ctx->stream), "H2D orbitals");
    if (*rc) return nullptr;
  }
  launch_pack_mo(raw, nr, n, rows, npad, pad, ctx->stream);
  return pad;
}

// XT[nu][Q p2 + a] = (C2 B^Q)[a][nu] for the padded rows (p2 x npad) of C2.
double* half_xform(rijk_ctx* ctx, Scratch& sc, const double* rows2, long p2, int* rc) {
  const long npad = ctx->npad, naux = ctx->nq;
  double* XT = sc.get(ctx, static_cast<size_t>(npad) * naux * p2, "half-transformed tensor", rc);
  if (*rc) return nullptr;
  launch_xform_f64(static_cast<const double*>(ctx->B.p), rows2, naux, ctx->nt, p2, XT, ctx->stream);
  return XT;
}

// R[r][Q p2 + a] = sum_nu rows1[r0 + r][nu] XT[nu][Q p2 + a], r < nb.
int second_xform(rijk_ctx* ctx, const double* XT, long p2, const double* rows1, long r0, long nb, double* R) {
  const long npad = ctx->npad, kdim = ctx->nq * p2;
  GemmF64Args g;
  g.M = nb, g.N = kdim, g.K = npad;
  g.A = rows1 + r0 * npad, g.lda = npad, g.a_kmajor = true;
  g.B = XT, g.ldb = kdim, g.b_kmajor = false;
  g.C = R, g.ldc = kdim;
  gemm_f64(g, 1, ctx->stream);
  return cuda_check(ctx, cudaGetLastError(), "second transform");
}

// out (host) [(p n2 + a)][Q] for all rows p of rows1 (n1 of them), in row blocks of <= ~1 GiB.
int tensor_to_host(rijk_ctx* ctx, Scratch& sc, const double* XT, long p2, long n2, const double* rows1, long n1,
                   double* out) {
  if (n1 == 0 || n2 == 0) return RIJK_OK;
  const long naux = ctx->nq, kdim = naux * p2;
  const long per_row = std::max(kdim, n2 * naux);
  long nb = std::max<long>(1, std::min<long>(n1, (1L << 27) / per_row));
  int rc = 0;
  double* R = sc.get(ctx, static_cast<size_t>(nb) * kdim, "second transform", &rc);
  if (rc) return rc;
  double* G = sc.get(ctx, static_cast<size_t>(nb) * n2 * naux, "gathered block", &rc);
  if (rc) return rc;
  for (long r0 = 0; r0 < n1; r0 += nb) {
    const long b = std::min(nb, n1 - r0);
    if ((rc = second_xform(ctx, XT, p2, rows1, r0, b, R))) return rc;
    k_gather_pa<<<grid_of(b * n2 * naux), 256, 0, ctx->stream>>>(R, b, n2, p2, naux, 0, G);
    rc = cuda_check(ctx, cudaMemcpyAsync(out + r0 * n2 * naux, G, static_cast<size_t>(b) * n2 * naux * sizeof(double),
                                         cudaMemcpyDeviceToHost, ctx->stream), "D2H MO tensor");
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "MO tensor block");
    if (rc) return rc;
  }
  return RIJK_OK;
}

int check_ready(rijk_ctx* ctx, const char* who) {
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "%s before rijk_set_3c / rijk_set_basis", who);
  cudaSetDevice(ctx->device);
  return RIJK_OK;
}

// The active-orbital intermediates shared by the AAAG and SOSCF integrals: R_all[x][Q p2 + v] =
// (x v|Q) for every orbital row x of MO (n_mo rows), v active (rows n_c .. n_c+n_a-1), and
// Yt[(t n_a + u)][Q] = (t u|Q).
struct ActiveParts {
  double* rows_all = nullptr;  // round_up(n_mo, 16) x npad
  double* R_all = nullptr;     // n_mo x naux p2
  double* Yt = nullptr;        // n_a^2 x naux
  long p2 = 0;
};

int active_parts(rijk_ctx* ctx, Scratch& sc, const double* MO, long n_c, long n_a, long n_mo, ActiveParts& ap) {
  int rc = 0;
  const long naux = ctx->nq;
  ap.p2 = round_up(n_a, 16);
  ap.rows_all = upload_rows(ctx, sc, MO, n_mo, round_up(n_mo, 16), &rc);  // zero rows up to a multiple of 16
  if (rc) return rc;
  double* rows_a = upload_rows(ctx, sc, MO + n_c * ctx->n, n_a, ap.p2, &rc);
  if (rc) return rc;
  double* XT = half_xform(ctx, sc, rows_a, ap.p2, &rc);
  if (rc) return rc;
  ap.R_all = sc.get(ctx, static_cast<size_t>(n_mo) * naux * ap.p2, "(x v|Q)", &rc);
  if (rc) return rc;
  if ((rc = second_xform(ctx, XT, ap.p2, ap.rows_all, 0, n_mo, ap.R_all))) return rc;
  ap.Yt = sc.get(ctx, static_cast<size_t>(n_a) * n_a * naux, "(t u|Q)", &rc);
  if (rc) return rc;
  k_gather_pa<<<grid_of(n_a * n_a * naux), 256, 0, ctx->stream>>>(ap.R_all + n_c * naux * ap.p2, n_a, n_a, ap.p2, naux,
                                                                   0, ap.Yt);
  return RIJK_OK;
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_mo_tensor(rijk_ctx* ctx, const double* C1, long n1, const double* C2, long n2, double* out) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!out || n1 < 0 || n2 < 0 || (n1 > 0 && !C1) || (n2 > 0 && !C2))
    return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_tensor: bad arguments");
  int rc = check_ready(ctx, "rijk_mo_tensor");
  if (rc || n1 == 0 || n2 == 0) return rc;
  Scratch sc;
  const long p2 = round_up(n2, 16);
  double* rows2 = upload_rows(ctx, sc, C2, n2, p2, &rc);
  if (rc) return rc;
  double* rows1 = upload_rows(ctx, sc, C1, n1, n1, &rc);
  if (rc) return rc;
  double* XT = half_xform(ctx, sc, rows2, p2, &rc);
  if (rc) return rc;
  return tensor_to_host(ctx, sc, XT, p2, n2, rows1, n1, out);
}

RIJK_API int rijk_mo_calc(rijk_ctx* ctx, const double* VEC, long n_cor, long n_act, long n_vac, double* CC, double* VC,
                          double* AA, double* CA, double* VA) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!VEC || n_cor < 0 || n_act < 0 || n_vac < 0)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_calc: bad arguments");
  int rc = check_ready(ctx, "rijk_mo_calc");
  if (rc) return rc;
  const long n = ctx->n;
  const double* COR = VEC;
  const double* ACT = VEC + n_cor * n;
  const double* VAC = VEC + (n_cor + n_act) * n;
  Scratch sc;
  // core half-transform: CC (core x core), VC (virtual x core)
  if (n_cor > 0 && (CC || VC)) {
    const long p2 = round_up(n_cor, 16);
    double* rows2 = upload_rows(ctx, sc, COR, n_cor, p2, &rc);
    if (rc) return rc;
    double* XT = half_xform(ctx, sc, rows2, p2, &rc);
    if (rc) return rc;
    if (CC && (rc = tensor_to_host(ctx, sc, XT, p2, n_cor, rows2, n_cor, CC))) return rc;
    if (VC && n_vac > 0) {
      double* rows1 = upload_rows(ctx, sc, VAC, n_vac, n_vac, &rc);
      if (rc) return rc;
      if ((rc = tensor_to_host(ctx, sc, XT, p2, n_cor, rows1, n_vac, VC))) return rc;
    }
  }
  // active half-transform: AA, CA (core x active), VA (virtual x active)
  if (n_act > 0 && (AA || CA || VA)) {
    Scratch sa;
    const long p2 = round_up(n_act, 16);
    double* rows2 = upload_rows(ctx, sa, ACT, n_act, p2, &rc);
    if (rc) return rc;
    double* XT = half_xform(ctx, sa, rows2, p2, &rc);
    if (rc) return rc;
    if (AA && (rc = tensor_to_host(ctx, sa, XT, p2, n_act, rows2, n_act, AA))) return rc;
    if (CA && n_cor > 0) {
      double* rows1 = upload_rows(ctx, sa, COR, n_cor, n_cor, &rc);
      if (rc) return rc;
      if ((rc = tensor_to_host(ctx, sa, XT, p2, n_act, rows1, n_cor, CA))) return rc;
    }
    if (VA && n_vac > 0) {
      double* rows1 = upload_rows(ctx, sa, VAC, n_vac, n_vac, &rc);
      if (rc) return rc;
      if ((rc = tensor_to_host(ctx, sa, XT, p2, n_act, rows1, n_vac, VA))) return rc;
    }
  }
  return RIJK_OK;
}

RIJK_API int rijk_mo_ints_aaag(rijk_ctx* ctx, double* MO_INTS, const double* MO_VEC, long n_c, long n_a, long n_mo) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!MO_INTS || !MO_VEC || n_c < 0 || n_a < 1 || n_mo < n_c + n_a)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_mo_ints_aaag: bad arguments");
  int rc = check_ready(ctx, "rijk_mo_ints_aaag");
  if (rc) return rc;
  const long naux = ctx->nq;
  Scratch sc;
  ActiveParts ap;
  if ((rc = active_parts(ctx, sc, MO_VEC, n_c, n_a, n_mo, ap))) return rc;
  // Z[(v n_mo + x)][Q] = (x v|Q);  MO_INTS[(t u)][(v x)] = sum_Q Yt[(t u)][Q] Z[(v x)][Q]
  double* Z = sc.get(ctx, static_cast<size_t>(n_a) * n_mo * naux, "(v x|Q)", &rc);
  if (rc) return rc;
  k_gather_pa<<<grid_of(n_mo * n_a * naux), 256, 0, ctx->stream>>>(ap.R_all, n_mo, n_a, ap.p2, naux, 1, Z);
  const long m = n_a * n_mo, nn = n_a * n_a;
  double* M = sc.get(ctx, static_cast<size_t>(m) * nn, "AAAG integrals", &rc);
  if (rc) return rc;
  {  // M[(t u)][(v x)] = sum_Q Yt[(t u)][Q] Z[(v x)][Q]
    GemmF64Args g;
    g.M = nn, g.N = m, g.K = naux;
    g.A = ap.Yt, g.lda = naux, g.a_kmajor = true;
    g.B = Z, g.ldb = naux, g.b_kmajor = true;
    g.C = M, g.ldc = m;
    gemm_f64(g, 1, ctx->stream);
  }
  rc = cuda_check(ctx, cudaMemcpyAsync(MO_INTS, M, static_cast<size_t>(m) * nn * sizeof(double), cudaMemcpyDeviceToHost,
                                       ctx->stream), "D2H AAAG integrals");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "rijk_mo_ints_aaag");
  return rc;
}

RIJK_API int rijk_soscf_hess_ints(rijk_ctx* ctx, double* aa_J, double* aa_K, const double* MO_VEC, long n_c, long n_a,
                                  long n_mo) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!aa_J || !aa_K || !MO_VEC || n_c < 0 || n_a < 1 || n_mo < n_c + n_a)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_soscf_hess_ints: bad arguments");
  int rc = check_ready(ctx, "rijk_soscf_hess_ints");
  if (rc) return rc;
  const long naux = ctx->nq, npad = ctx->npad;
  Scratch sc;
  ActiveParts ap;
  if ((rc = active_parts(ctx, sc, MO_VEC, n_c, n_a, n_mo, ap))) return rc;
  // aa_K[p][t][u] = sum_Q (p t|Q)(p u|Q): one n_a x n_a product per orbital p
  double* dK = sc.get(ctx, static_cast<size_t>(n_mo) * n_a * n_a, "aa_K", &rc);
  if (rc) return rc;
  const long kdim = naux * ap.p2;
  {
    GemmF64Args g;
    g.M = n_a, g.N = n_a, g.K = naux;
    g.A = ap.R_all, g.lda = ap.p2, g.sA = kdim, g.a_kmajor = false;
    g.B = ap.R_all, g.ldb = ap.p2, g.sB = kdim, g.b_kmajor = false;
    g.C = dK, g.ldc = n_a, g.sC = n_a * n_a;
    gemm_f64(g, n_mo, ctx->stream);
  }
  // (pp|Q) for every orbital, by half-transforms of batches of rows
  double* Rpp = sc.get(ctx, static_cast<size_t>(n_mo) * naux, "(pp|Q)", &rc);
  if (rc) return rc;
  const long batch = 96;
  {
    Scratch sb;
    double* XT = sb.get(ctx, static_cast<size_t>(npad) * naux * batch, "batch half-transform", &rc);
    if (rc) return rc;
    for (long p0 = 0; p0 < n_mo; p0 += batch) {
      const long nr = std::min(batch, n_mo - p0), pb = round_up(nr, 16);
      const double* rows = ap.rows_all + p0 * npad;
      launch_xform_f64(static_cast<const double*>(ctx->B.p), rows, naux, ctx->nt, pb, XT, ctx->stream);
      k_diag_pair<<<grid_of(naux * pb), 256, 0, ctx->stream>>>(XT, rows, nr, pb, naux, npad, Rpp + p0 * naux);
    }
    // p0 + pb <= round_up(n_mo, 16): the last batch's padding rows are the zero rows of rows_all
    if ((rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "(pp|Q)"))) return rc;
  }
  // aa_J[p][(t u)] = sum_Q (pp|Q)(t u|Q)
  double* dJ = sc.get(ctx, static_cast<size_t>(n_mo) * n_a * n_a, "aa_J", &rc);
  if (rc) return rc;
  {
    GemmF64Args g;
    g.M = n_mo, g.N = n_a * n_a, g.K = naux;
    g.A = Rpp, g.lda = naux, g.a_kmajor = true;
    g.B = ap.Yt, g.ldb = naux, g.b_kmajor = true;
    g.C = dJ, g.ldc = n_a * n_a;
    gemm_f64(g, 1, ctx->stream);
  }
  const size_t bytes = static_cast<size_t>(n_mo) * n_a * n_a * sizeof(double);
  rc = cuda_check(ctx, cudaMemcpyAsync(aa_J, dJ, bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H aa_J");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(aa_K, dK, bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H aa_K");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "rijk_soscf_hess_ints");
  return rc;
}
