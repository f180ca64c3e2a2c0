// k_adjoint.cu — the adjoint of the Fock build (rijk_grad).  No reference counterpart: the
// reference has no analytic gradient and differentiates by finite differences
// (src/QM_calc.cpp:142).
//
// With D = C^T C over the n_c occupied rows of MO (src/SCF.cpp:63-73), the fitted tensor
// B^Q = sum_P M_QP (P|.), w_Q = <B^Q, D> and Y^Q = C B^Q C^T (n_c x n_c), the energy of the
// reference's RHF (src/SCF.cpp:134) is
//     E = 2 tr(H D) + 2 sum_Q w_Q^2 - sum_Q |Y^Q|^2 + e_nuc ,
// and its derivatives are
//     dE/dC        = 4 C F,  F = H + 2J - K                          (orbital gradient)
//     Gamma^Q      = dE/dB^Q = 4 w_Q D - 2 C^T Y^Q C                 (full-square derivative)
//     dE/d(P|mu nu) = sum_Q M_QP Gamma^Q_{mu nu}                    (times 2 for mu != nu when the
//                                                                      pair is stored once)
//     dE/d(P|Q)    = -(M^T G M)_PQ,  G_QR = (1/2) sum_{mu nu} Gamma^Q_{mu nu} B^R_{mu nu}
// (E depends on the metric only through V^-1 = M^T M, for either metric form).
//
// Device work, FP64 throughout, every contraction on hand-written DMMA kernels: one FP64 Fock build
// (which leaves w and the half-transformed XT in the context), then, over chunks of aux functions,
// the products Y^Q = X^Q C^T and T^Q = Y^Q C for every Q of the chunk at once (k_gemm_f64), k_gamma_f64
// forming the packed Gamma tiles Gamma^Q_tile = 4 w_Q D_tile - 2 T^Q_rows Ct_cols^T, and two contractions of
// the chunk of Gamma: with M, written straight into the packed pair layout of dE/d(P|mu nu)
// (accumulated over chunks), and with B, the chunk's rows of G (diagonal tiles weighted 1/2).  When
// HBM cannot hold Gamma for every aux function at once, each chunk's X^Q is recomputed in tiles
// from B instead of read from the stored tensor.
#include <algorithm>
#include <cmath>
#include <vector>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

constexpr int G_THREADS = 128;

// Gamma[Q][t][r][c] = 4 w_Q D[mu][nu] - 2 sum_i T^Q[mu][i] Ct[nu][i], tile t = (I, J), I >= J.
// Tt: [(Q, i)][npad] = T^Q transposed (row (Q, i), mu contiguous); Ct: [npad][noccp]; D: n x n.
constexpr int G_ASTAGE = (64 * LDK > KC * LDM) ? 64 * LDK : KC * LDM;
__global__ void __launch_bounds__(G_THREADS)
    k_gamma_f64(const double* __restrict__ Tt, const double* __restrict__ Ct, const double* __restrict__ D,
                const double* __restrict__ w, long n, long npad, long noccp, long tile_elems,
                double* __restrict__ Gamma) {
  extern __shared__ __align__(16) double smem_g[];
  double* sA[2] = {smem_g, smem_g + G_ASTAGE};
  double* sB[2] = {smem_g + 2 * G_ASTAGE, smem_g + 2 * G_ASTAGE + 64 * LDK};
  const long t = blockIdx.x, Q = blockIdx.y;
  long I, J;
  tri_decode(t, I, J);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const double* Ar = Tt + Q * noccp * npad + I * TILE;  // A(mu, i) = Ar[i * npad + mu]: staged [i][mu]
  const double* Br = Ct + J * TILE * noccp;
  auto load = [&](int stage, long k0) {
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      int idx = tid + it * G_THREADS;
      int ka = idx >> 5, pa = idx & 31;  // A: k row (i) 0..31, mu pair 0..31
      bool oka = k0 + ka < noccp;
      cp_async16(&sA[stage][ka * LDM + pa * 2], oka ? Ar + (k0 + ka) * npad + pa * 2 : Tt, oka);
      int row = idx >> 4, seg = idx & 15;  // B: row nu 0..63, i pair 0..15
      long k = k0 + seg * 2;
      bool ok = k < noccp;
      cp_async16(&sB[stage][row * LDK + seg * 2], ok ? Br + row * noccp + k : Ct, ok);
    }
  };
  double acc[4][4][2];
  zero_acc(acc);
  const long nk = (noccp + KC - 1) / KC;
  load(0, 0);
  cp_async_commit();
  for (long kc = 0; kc < nk; ++kc) {
    if (kc + 1 < nk) {
      load(static_cast<int>((kc + 1) & 1), (kc + 1) * KC);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    warp_mma_chunk<4, 4, false>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * 32, lane);
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3;
  const double wq4 = 4.0 * w[Q];
  double* out = Gamma + Q * tile_elems + t * TILE2;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = wm * 32 + i * 8 + g;
    const long mu = I * TILE + r;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = wn * 32 + j * 8 + 2 * tq;
      const long nu = J * TILE + c;
      double d0 = (mu < n && nu < n) ? D[mu * n + nu] : 0.0;
      double d1 = (mu < n && nu + 1 < n) ? D[mu * n + nu + 1] : 0.0;
      *reinterpret_cast<double2*>(out + r * TILE + c) =
          make_double2(wq4 * d0 - 2.0 * acc[i][j][0], wq4 * d1 - 2.0 * acc[i][j][1]);
    }
  }
}

// Ct[nu][i] = C_{i nu} from the padded MOp[i][nu]
__global__ void k_transpose_mo(const double* __restrict__ MOp, long noccp, long npad, double* __restrict__ Ct) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < noccp * npad; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long nu = idx / noccp, i = idx % noccp;
    Ct[idx] = MOp[i * npad + nu];
  }
}

__global__ void k_fock_sym(const double* __restrict__ H, const double* __restrict__ J, const double* __restrict__ K,
                           long nn, double* __restrict__ F) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < nn; idx += static_cast<long>(gridDim.x) * blockDim.x) F[idx] = H[idx] + 2.0 * J[idx] - K[idx];
}

// partial[b], partial[512 + b]: compensated sum of D (F + H) over a grid-stride slice
__global__ void k_energy_partial(const double* __restrict__ D, const double* __restrict__ F,
                                 const double* __restrict__ H, long nn, double* __restrict__ partial) {
  double s = 0.0, c = 0.0;
  for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < nn; i += static_cast<long>(gridDim.x) * blockDim.x)
    neumaier_add(s, c, D[i] * (F[i] + H[i]));
  warp_sum_comp(s, c);
  __shared__ double sh[2][8];
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = s;
    sh[1][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0, u = 0.0;
    for (int i = 0; i < 8; ++i) {
      neumaier_add(t, u, sh[0][i]);
      u += sh[1][i];
    }
    partial[blockIdx.x] = t;
    partial[512 + blockIdx.x] = u;
  }
}

// Device time per stage of rijk_grad when profiling is on: mark(k) records an event on the stream,
// and the interval since the previous mark counts for stage k (k < 0: not counted).
struct GradTimer {
  bool on = false;
  cudaStream_t s = nullptr;
  std::vector<std::pair<int, cudaEvent_t>> ev;
  void mark(int stage) {
    if (!on) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    ev.emplace_back(stage, e);
  }
  // after the stream has drained
  void collect(rijk_stats_t& st) {
    for (double& v : st.ms_grad_stage) v = 0.0;
    st.ms_grad_total = 0.0;
    for (size_t i = 1; i < ev.size(); ++i) {
      if (ev[i].first < 0) continue;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev[i - 1].second, ev[i].second);
      st.ms_grad_stage[ev[i].first] += ms;
      st.ms_grad_total += ms;
    }
  }
  ~GradTimer() {
    for (auto& e : ev) cudaEventDestroy(e.second);
  }
};

unsigned grid_of(long total) {
  long b = (total + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_set_grad_chunk(rijk_ctx* ctx, long q_per_chunk) {
  if (!ctx) return RIJK_ERR_ARG;
  if (q_per_chunk < 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_grad_chunk: negative chunk");
  ctx->grad_qchunk = q_per_chunk;
  return RIJK_OK;
}

RIJK_API int rijk_grad(rijk_ctx* ctx, const double* MO, long nocc, const double* H, double e_nuc, double* E,
                       double* dEdC, double* dEdI3, double* dEdPQ) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!MO || !H || !E || !dEdC) return set_err(ctx, RIJK_ERR_ARG, "rijk_grad: null pointer");
  int rc = check_fock_args(ctx, nocc, RIJK_PREC_FP64);
  if (rc) return rc;
  if (nocc < 1) return set_err(ctx, RIJK_ERR_ARG, "rijk_grad: n_c must be at least 1");
  NvtxRange range("rijk_grad");
  if (ctx->nq != ctx->naux)
    return set_err(ctx, RIJK_ERR_STATE, "rijk_grad needs all aux functions in one context (no aux range)");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const long n = ctx->n, naux = ctx->naux, npad = ctx->npad, nt = ctx->nt, ntile = ctx->ntile;
  const long nn = n * n, te = ntile * TILE2, noccp = round_up(nocc, 16), nauxp = round_up(naux, KC);
  const size_t b_nn = nn * sizeof(double);
  DeviceBuf dMO, dH, dD, dJ, dK, dF, dG, red, Y, Tb, Ct, Gam, Gm, T1, out;
  auto cleanup = [&]() {
    DeviceBuf* all[] = {&dMO, &dH, &dD, &dJ, &dK, &dF, &dG, &red, &Y, &Tb, &Ct, &Gam, &Gm, &T1, &out};
    for (DeviceBuf* b : all) release(*b);
  };
  auto chk = [&](int r) {
    if (r) cleanup();
    return r;
  };
  if ((rc = chk(ensure(ctx, dMO, nocc * n * sizeof(double), "grad MO"))) || (rc = chk(ensure(ctx, dH, b_nn, "grad H"))) ||
      (rc = chk(ensure(ctx, dD, b_nn, "grad D"))) || (rc = chk(ensure(ctx, dJ, b_nn, "grad J"))) ||
      (rc = chk(ensure(ctx, dK, b_nn, "grad K"))) || (rc = chk(ensure(ctx, dF, b_nn, "grad F"))) ||
      (rc = chk(ensure(ctx, dG, nocc * n * sizeof(double), "grad dEdC"))) ||
      (rc = chk(ensure(ctx, red, 1024 * sizeof(double), "grad reduce"))))
    return rc;
  double* pMO = static_cast<double*>(dMO.p);
  double* pD = static_cast<double*>(dD.p);
  double* pF = static_cast<double*>(dF.p);
  cudaMemcpyAsync(pMO, MO, nocc * n * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dH.p, H, b_nn, cudaMemcpyHostToDevice, s);
  GradTimer tm;
  tm.on = ctx->profiling;
  tm.s = s;
  tm.mark(-1);
  {  // D[mu][nu] = sum_i C[i][mu] C[i][nu]
    GemmF64Args g;
    g.M = n, g.N = n, g.K = nocc;
    g.A = pMO, g.lda = n, g.a_kmajor = false;
    g.B = pMO, g.ldb = n, g.b_kmajor = false;
    g.C = pD, g.ldc = n;
    gemm_f64(g, 1, s);
  }
  if ((rc = chk(fock_device_impl(ctx, pD, pMO, nocc, static_cast<double*>(dJ.p), static_cast<double*>(dK.p),
                                 RIJK_PREC_FP64))))
    return rc;
  k_fock_sym<<<grid_of(nn), 256, 0, s>>>(static_cast<const double*>(dH.p), static_cast<const double*>(dJ.p),
                                         static_cast<const double*>(dK.p), nn, pF);
  k_energy_partial<<<512, 256, 0, s>>>(pD, pF, static_cast<const double*>(dH.p), nn, static_cast<double*>(red.p));
  {  // dE/dC[i][mu] = 4 sum_nu C[i][nu] F[nu][mu]
    GemmF64Args g;
    g.M = nocc, g.N = n, g.K = n;
    g.A = pMO, g.lda = n, g.a_kmajor = true;
    g.B = pF, g.ldb = n, g.b_kmajor = false;
    g.C = static_cast<double*>(dG.p), g.ldc = n;
    g.alpha = 4.0;
    gemm_f64(g, 1, s);
  }
  tm.mark(0);
  std::vector<double> part(1024);
  cudaMemcpyAsync(part.data(), red.p, 1024 * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(dEdC, dG.p, nocc * n * sizeof(double), cudaMemcpyDeviceToHost, s);
  tm.mark(-1);
  if ((rc = chk(cuda_check(ctx, cudaStreamSynchronize(s), "rijk_grad energy"))) || (rc = chk(check_device_error(ctx))))
    return rc;
  double es = 0.0, ec = 0.0;  // compensated: the 512 block sums, their compensations, then e_nuc
  for (int b = 0; b < 512; ++b) {
    neumaier_add(es, ec, part[b]);
    ec += part[512 + b];
  }
  neumaier_add(es, ec, e_nuc);
  *E = es + ec;
  if (!dEdI3 && !dEdPQ) {
    tm.collect(ctx->stats);
    cleanup();
    return RIJK_OK;
  }
  // Gamma and its contractions over chunks of aux functions [q0, q0 + qc).  X^Q comes from the
  // tensor the FP64 build left in HBM when every chunk fits at once; otherwise (HBM short, or a
  // chunk size set by rijk_set_grad_chunk) each chunk's X^Q is recomputed in tiles by the
  // half-transform kernel, and only one chunk of X, Y, T and Gamma exists at a time.
  const long kdim = naux * noccp;
  const long npair = n * (n + 1) / 2;
  const double* MOp = static_cast<const double*>(ctx->MOp.p);
  const double* pM = static_cast<const double*>(ctx->M.p);  // row-major [Q][P], ld nauxp
  if (dEdI3 && (rc = chk(ensure(ctx, out, static_cast<size_t>(npair) * naux * sizeof(double), "grad dI3"))))
    return rc;
  if (dEdPQ && ((rc = chk(ensure(ctx, Gm, static_cast<size_t>(naux) * naux * sizeof(double), "grad G"))) ||
                (rc = chk(ensure(ctx, T1, static_cast<size_t>(naux) * naux * sizeof(double), "grad T1")))))
    return rc;
  if ((rc = chk(ensure(ctx, Ct, static_cast<size_t>(npad) * noccp * sizeof(double), "grad Ct")))) return rc;
  k_transpose_mo<<<grid_of(noccp * npad), 256, 0, s>>>(MOp, noccp, npad, static_cast<double*>(Ct.p));
  // bytes per aux function of one chunk: Y, T, Gamma (and X when recomputed)
  const double per_q = 8.0 * (static_cast<double>(noccp) * noccp + static_cast<double>(npad) * noccp + te);
  const double per_q_x = per_q + 8.0 * npad * noccp;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const double room = 0.85 * static_cast<double>(free_b) - 64.0 * 1024 * 1024;
  long qc = ctx->grad_qchunk > 0 ? std::min(ctx->grad_qchunk, naux) : naux;
  if (ctx->grad_qchunk <= 0 && per_q * naux > room)
    qc = std::max<long>(1, std::min<long>(naux, static_cast<long>(room / per_q_x)));
  const bool recompute = qc < naux;
  if ((rc = chk(ensure(ctx, Y, static_cast<size_t>(qc) * noccp * noccp * sizeof(double), "grad Y"))) ||
      (rc = chk(ensure(ctx, Tb, static_cast<size_t>(qc) * npad * noccp * sizeof(double), "grad T"))) ||
      (rc = chk(ensure(ctx, Gam, static_cast<size_t>(qc) * te * sizeof(double), "grad Gamma"))))
    return rc;
  DeviceBuf Xc;
  if (recompute && (rc = chk(ensure(ctx, Xc, static_cast<size_t>(npad) * qc * noccp * sizeof(double), "grad X chunk")))) {
    release(Xc);
    return rc;
  }
  double* pGam = static_cast<double*>(Gam.p);
  double* pY = static_cast<double*>(Y.p);
  double* pT = static_cast<double*>(Tb.p);
  const size_t gsmem = (2 * G_ASTAGE + 2 * 64 * LDK) * sizeof(double);
  ensure_smem_limit(reinterpret_cast<const void*>(k_gamma_f64), gsmem);
  for (long q0 = 0; q0 < naux; q0 += qc) {
    const long nq = std::min(qc, naux - q0);
    const double* X;  // X^Q_{i nu} at X[nu * ldx + (Q - q0) * noccp + i]
    long ldx;
    if (recompute) {
      launch_xform_f64(static_cast<const double*>(ctx->B.p) + q0 * te, MOp, nq, nt, noccp, static_cast<double*>(Xc.p), s);
      X = static_cast<const double*>(Xc.p);
      ldx = nq * noccp;
      tm.mark(1);
    } else {
      X = static_cast<const double*>(ctx->XT.p) + q0 * noccp;
      ldx = kdim;
    }
    {  // Y^Q[i][j] = sum_nu X^Q_{i nu} C_{j nu} (= C B^Q C^T), every Q of the chunk in one product:
       // rows (Q, i) of X^T's columns are contiguous, so Y[(Q, i)][j] is one GEMM over nu
      GemmF64Args g;
      g.M = nq * noccp, g.N = noccp, g.K = npad;
      g.A = X, g.lda = ldx, g.a_kmajor = false;
      g.B = MOp, g.ldb = npad, g.b_kmajor = true;
      g.C = pY, g.ldc = noccp;
      gemm_f64(g, 1, s);
    }
    {  // T^Q transposed, Tt[(Q, i)][mu] = sum_j Y^Q[i][j] C_{j mu}: again one GEMM for the chunk
      GemmF64Args g;
      g.M = nq * noccp, g.N = npad, g.K = noccp;
      g.A = pY, g.lda = noccp, g.a_kmajor = true;
      g.B = MOp, g.ldb = npad, g.b_kmajor = false;
      g.C = pT, g.ldc = npad;
      gemm_f64(g, 1, s);
    }
    tm.mark(2);
    dim3 grid(static_cast<unsigned>(ntile), static_cast<unsigned>(nq));
    k_gamma_f64<<<grid, G_THREADS, gsmem, s>>>(pT, static_cast<const double*>(Ct.p), pD,
                                               static_cast<const double*>(ctx->w.p) + q0, n, npad, noccp, te, pGam);
    tm.mark(3);
    if (dEdI3) {
      // dE/d(P|mu nu) += sum_{Q in chunk} Gamma^Q_{mu nu} M_QP, straight into the packed pair rows
      GemmF64Args g;
      g.M = te, g.N = naux, g.K = nq;
      g.A = pGam, g.lda = te, g.a_kmajor = false;
      g.B = pM + q0 * nauxp, g.ldb = nauxp, g.b_kmajor = false;
      g.C = static_cast<double*>(out.p), g.ldc = naux;
      g.beta = q0 == 0 ? 0.0 : 1.0;
      g.mode = GEMM_PAIRS;
      g.n_ao = n;
      gemm_f64(g, 1, s);
    }
    tm.mark(4);
    if (dEdPQ) {
      // rows q0.. of G_QR = 1/2 sum_{mu nu} Gamma^Q B^R over the full squares: each stored element
      // of an off-diagonal tile once, of a diagonal tile one half
      GemmF64Args g;
      g.M = nq, g.N = naux, g.K = te;
      g.A = pGam, g.lda = te, g.a_kmajor = true;
      g.B = static_cast<const double*>(ctx->B.p), g.ldb = te, g.b_kmajor = true;
      g.C = static_cast<double*>(Gm.p) + q0 * naux, g.ldc = naux;
      g.kdiag = 1;
      gemm_f64(g, 1, s);
    }
    tm.mark(5);
  }
  release(Xc);
  release(Y);
  release(Tb);
  tm.mark(-1);  // the frees above wait on the host: that gap is not a stage
  if (dEdPQ) {
    // dE/dV = -M^T G M:  T1[Q][P'] = sum_R G[Q][R] M[R][P'];  out[P][P'] = -sum_Q M[Q][P] T1[Q][P']
    GemmF64Args g;
    g.M = naux, g.N = naux, g.K = naux;
    g.A = static_cast<const double*>(Gm.p), g.lda = naux, g.a_kmajor = true;
    g.B = pM, g.ldb = nauxp, g.b_kmajor = false;
    g.C = static_cast<double*>(T1.p), g.ldc = naux;
    gemm_f64(g, 1, s);
    GemmF64Args h;
    h.M = naux, h.N = naux, h.K = naux;
    h.A = pM, h.lda = nauxp, h.a_kmajor = false;
    h.B = static_cast<const double*>(T1.p), h.ldb = naux, h.b_kmajor = false;
    h.C = static_cast<double*>(Gm.p), h.ldc = naux;
    h.alpha = -1.0;
    gemm_f64(h, 1, s);
    tm.mark(6);
    cudaMemcpyAsync(dEdPQ, Gm.p, static_cast<size_t>(naux) * naux * sizeof(double), cudaMemcpyDeviceToHost, s);
  }
  if (dEdI3)
    cudaMemcpyAsync(dEdI3, out.p, static_cast<size_t>(npair) * naux * sizeof(double), cudaMemcpyDeviceToHost, s);
  ctx->stats.grad_qchunk = qc;
  rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_grad");
  if (!rc) tm.collect(ctx->stats);
  cleanup();
  (void)nt;
  return rc;
}
