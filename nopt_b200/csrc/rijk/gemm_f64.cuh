// gemm_f64.cuh — the warp-level FP64 DMMA micro-kernel shared by the FP64 contractions.
//
// A CTA of 4 warps (2 x 2) owns a 64 x NT output tile; warp (wm, wn) owns rows
// wm*32 .. +32 and columns wn*NT/2 .. +NT/2, i.e. MF = 4 row fragments and NF = NT/16
// column fragments of 8 x 8.  The contraction runs over 32-wide chunks staged in shared
// memory:
//   A chunk  [m][k] with row stride LDK (= 36) when A_KMAJOR, else [k][m] with stride LDM (= 68)
//   B chunk  [n][k] with row stride LDK
#pragma once
#include "dmma.cuh"

namespace rijk {

constexpr int KC = 32;    // contraction chunk
constexpr int LDK = 36;   // stride of [row][k] chunks   (36 % 16 == 4)
constexpr int LDM = 68;   // stride of [k][row] chunks   (68 % 16 == 4)

template <int MF, int NF, bool A_KMAJOR>
__device__ __forceinline__ void warp_mma_chunk(double (&acc)[MF][NF][2], const double* __restrict__ sA,
                                               const double* __restrict__ sB, int m0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k = 0; k < KC; k += 4) {
    double a[MF], b[NF];
#pragma unroll
    for (int i = 0; i < MF; ++i)
      a[i] = A_KMAJOR ? sA[(m0 + i * 8 + g) * LDK + k + t] : sA[(k + t) * LDM + m0 + i * 8 + g];
#pragma unroll
    for (int j = 0; j < NF; ++j) b[j] = sB[(n0 + j * 8 + g) * LDK + k + t];
#pragma unroll
    for (int i = 0; i < MF; ++i)
#pragma unroll
      for (int j = 0; j < NF; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  }
}

template <int MF, int NF>
__device__ __forceinline__ void zero_acc(double (&acc)[MF][NF][2]) {
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
}

}  // namespace rijk
