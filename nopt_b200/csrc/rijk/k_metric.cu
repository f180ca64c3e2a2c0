// k_metric.cu — K1, the metric contraction B^Q_{mu nu} = sum_P M_QP (P|mu nu).
//
// Replaces the reference's per-iteration metric products (V^-1/2 applied to RI_J twice,
// src/RI.cpp:128-138, and to the half-transformed tensor, src/RI.cpp:152-156): the metric
// factor M (V^-1/2 or L^-1) is applied once per geometry and B is kept in HBM.
//
// GEMM: rows Q (64 per CTA), columns = one row r of one stored tile (64 pairs (mu, nu) =
// (I*64 + r, J*64 + c)), contraction over P in 32-wide chunks.  M is zero-padded to
// nauxp x nauxp and the raw integrals carry row pitch nauxp, so chunks never straddle.
// The raw integrals arrive in row-blocks of whole tile rows (I in [I0, I1)); pair rows are
// gathered per column (NOPT full-square layout or packed mu >= nu layout).
#include <algorithm>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

namespace rijk {

constexpr int K1_THREADS = 128;

__global__ void __launch_bounds__(K1_THREADS)
    k_metric_contract(const double* __restrict__ M, long nauxp, long mrows, const double* __restrict__ I3, int layout,
                      long n, long naux, long I0, long t0, long rows_in_chunk_base, double* __restrict__ B,
                      long tile_elems, long tri) {
  extern __shared__ __align__(16) double smem_k1[];
  double* sA[2] = {smem_k1, smem_k1 + 64 * LDK};
  double* sB[2] = {smem_k1 + 2 * 64 * LDK, smem_k1 + 3 * 64 * LDK};
  __shared__ long rowoff[64];

  const long q0 = static_cast<long>(blockIdx.y) * 64;
  const long trow = t0 * TILE + blockIdx.x;  // global tile-row index
  const long t = trow / TILE;
  const int r = static_cast<int>(trow % TILE);
  long I, J;
  tri_decode(t, I, J);
  const long mu = I * TILE + r;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  if (tid < 64) {
    long nu = J * TILE + tid;
    long off = -1;
    if (mu < n && nu < n) {
      if (layout == RIJK_LAYOUT_NOPT_FULL) {
        off = (mu - I0 * TILE) * n + nu;
      } else {
        long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
        off = hi * (hi + 1) / 2 + lo - rows_in_chunk_base;
      }
    }
    rowoff[tid] = off;
  }
  __syncthreads();

  auto load = [&](int stage, long p0) {
    // A: M rows q0..q0+63, cols p0..p0+31 ; B: raw rows rowoff[c], cols p0..p0+31
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      int idx = tid + it * K1_THREADS;  // 0..1023
      int row = idx >> 4, seg = idx & 15;
      long q = q0 + row;
      const double* src = M + q * nauxp + p0 + seg * 2;
      cp_async16(&sA[stage][row * LDK + seg * 2], q < mrows ? src : M, q < mrows);
      long ro = rowoff[row];
      const double* srcb = I3 + (ro >= 0 ? ro : 0) * nauxp + p0 + seg * 2;
      cp_async16(&sB[stage][row * LDK + seg * 2], srcb, ro >= 0);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  // tri >= 0: M is lower triangular (the Cholesky factor's inverse), its rows starting at global row
  // tri, so rows q0 .. q0 + 63 hold zeros past column tri + q0 + 63 and the chunks beyond add nothing
  const long nk = tri < 0 ? nauxp / KC : std::min(nauxp / KC, (tri + q0 + 64 + KC - 1) / KC);
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
    warp_mma_chunk<4, 4, true>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * 32, lane);
    __syncthreads();
  }

  const int g = lane >> 2, tq = lane & 3;
  double* Bt = B + t * TILE2 + static_cast<long>(r) * TILE;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    long q = q0 + wm * 32 + i * 8 + g;
    if (q >= naux) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int c = wn * 32 + j * 8 + 2 * tq;
      *reinterpret_cast<double2*>(Bt + q * tile_elems + c) = make_double2(acc[i][j][0], acc[i][j][1]);
    }
  }
}

// I3 holds the tile rows I in [I0, I1): full layout rows (mu - I0*64)*n + nu, packed layout
// pair rows starting at pair_base = (I0*64)(I0*64+1)/2.
void launch_metric_contract_chunk(const double* M, long nauxp, long mrows, const double* I3, int layout, long n,
                                  long naux, long nt, long I0, long I1, double* B, cudaStream_t s, long tri) {
  long t0 = tri_index(I0, 0);
  long t1 = tri_index(I1, 0);
  long ntile = nt * (nt + 1) / 2;
  long mu0 = I0 * TILE;
  long pair_base = mu0 * (mu0 + 1) / 2;
  dim3 grid(static_cast<unsigned>((t1 - t0) * TILE), static_cast<unsigned>((naux + 63) / 64));
  const size_t smem = 4 * 64 * LDK * sizeof(double);
  ensure_smem_limit(reinterpret_cast<const void*>(k_metric_contract), smem);
  k_metric_contract<<<grid, K1_THREADS, smem, s>>>(M, nauxp, mrows, I3, layout, n, naux, I0, t0, pair_base, B,
                                                   ntile * TILE2, tri);
}

}  // namespace rijk
