// k_coulomb.cu — the Coulomb pair of the RI Fock build, two bandwidth-bound passes over B.
//
// Reference (src/RI.cpp:122-144): RI_J = vec(D)^T RI_AA, then V^-1/2 twice, then
// J = RI_AA RI_J.  With the metric folded into B (B = M (P|mu nu), M^T M = V^-1) this is
//   w_Q  = sum_e B[Q][e] Dt[e]          (pass 1, one CTA per QB aux functions)
//   J[e] = sum_Q B[Q][e] w_Q            (pass 2, Q split into nsplit ranges, partials
//                                        summed while unpacking)
// Both passes stream B once with 128-bit loads that bypass L1; reductions are warp
// shuffles.  Algorithmic traffic: 2 * |B| bytes per build.
#include "dmma.cuh"
#include "rijk_internal.h"

namespace rijk {

constexpr int W_QB = 4;        // aux functions per CTA in pass 1 (reuses each Dt load)
constexpr int W_THREADS = 512;

__global__ void __launch_bounds__(W_THREADS) k_coulomb_w(const double* __restrict__ B, const double* __restrict__ Dt,
                                                          long naux, long tile_elems, double* __restrict__ w) {
  const long q0 = static_cast<long>(blockIdx.x) * W_QB;
  const long n2 = tile_elems / 2;
  const double2* D2 = reinterpret_cast<const double2*>(Dt);
  double acc[W_QB];
#pragma unroll
  for (int j = 0; j < W_QB; ++j) acc[j] = 0.0;
  const double2* Bq[W_QB];
#pragma unroll
  for (int j = 0; j < W_QB; ++j) {
    long q = q0 + j < naux ? q0 + j : naux - 1;
    Bq[j] = reinterpret_cast<const double2*>(B + q * tile_elems);
  }
  for (long e = threadIdx.x; e < n2; e += W_THREADS) {
    double2 d = D2[e];
#pragma unroll
    for (int j = 0; j < W_QB; ++j) {
      double2 b = ldg_stream(Bq[j] + e);
      acc[j] = fma(b.x, d.x, acc[j]);
      acc[j] = fma(b.y, d.y, acc[j]);
    }
  }
  __shared__ double red[W_QB][W_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < W_QB; ++j) {
    double v = warp_sum(acc[j]);
    if (lane == 0) red[j][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < W_QB; ++j) {
      double v = lane < W_THREADS / 32 ? red[j][lane] : 0.0;
      v = warp_sum(v);
      if (lane == 0 && q0 + j < naux) w[q0 + j] = v;
    }
  }
}

constexpr int J_THREADS = 256;
constexpr int J_UNROLL = 4;

// Jpart[s][e] = sum_{Q in split s} B[Q][e] w[Q]; each thread owns one double2 of e.
__global__ void __launch_bounds__(J_THREADS) k_coulomb_j(const double* __restrict__ B, const double* __restrict__ w,
                                                          long naux, long tile_elems, long qper,
                                                          double* __restrict__ Jpart) {
  const long e2 = static_cast<long>(blockIdx.x) * J_THREADS + threadIdx.x;
  const long s = blockIdx.y;
  const long qa = s * qper;
  const long qb = qa + qper < naux ? qa + qper : naux;
  if (e2 * 2 >= tile_elems) return;
  const double2* Bp = reinterpret_cast<const double2*>(B) + e2;
  const long stride2 = tile_elems / 2;
  double ax = 0.0, ay = 0.0;
  long q = qa;
  for (; q + J_UNROLL <= qb; q += J_UNROLL) {
    double2 b[J_UNROLL];
#pragma unroll
    for (int u = 0; u < J_UNROLL; ++u) b[u] = ldg_stream(Bp + (q + u) * stride2);
#pragma unroll
    for (int u = 0; u < J_UNROLL; ++u) {
      double wq = __ldg(w + q + u);
      ax = fma(b[u].x, wq, ax);
      ay = fma(b[u].y, wq, ay);
    }
  }
  for (; q < qb; ++q) {
    double2 b = ldg_stream(Bp + q * stride2);
    double wq = __ldg(w + q);
    ax = fma(b.x, wq, ax);
    ay = fma(b.y, wq, ay);
  }
  reinterpret_cast<double2*>(Jpart + s * tile_elems)[e2] = make_double2(ax, ay);
}

int coulomb_nsplit(long tile_elems, long naux) {
  long blocks = (tile_elems / 2 + J_THREADS - 1) / J_THREADS;
  long want = (148L * 8 + blocks - 1) / blocks;  // about 8 CTAs per SM in flight
  if (want < 1) want = 1;
  if (want > 32) want = 32;
  if (want > naux) want = naux;
  return static_cast<int>(want);
}

void launch_coulomb_w(const double* B, const double* Dt, long naux, long tile_elems, double* w, cudaStream_t s) {
  unsigned grid = static_cast<unsigned>((naux + W_QB - 1) / W_QB);
  k_coulomb_w<<<grid, W_THREADS, 0, s>>>(B, Dt, naux, tile_elems, w);
}

void launch_coulomb_j(const double* B, const double* w, long naux, long tile_elems, int nsplit, double* Jpart,
                      cudaStream_t s) {
  long qper = (naux + nsplit - 1) / nsplit;
  dim3 grid(static_cast<unsigned>((tile_elems / 2 + J_THREADS - 1) / J_THREADS), static_cast<unsigned>(nsplit));
  k_coulomb_j<<<grid, J_THREADS, 0, s>>>(B, w, naux, tile_elems, qper, Jpart);
}

}  // namespace rijk
