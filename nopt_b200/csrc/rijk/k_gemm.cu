// k_gemm.cu — batched FP64 DMMA GEMM for the contractions around the Fock build (the adjoint, the
// MO-basis tensors): C_b = alpha op(A_b) op(B_b) + beta C_b, one 64 x 64 output tile per CTA.
//
// Layouts are given per operand, row-major with a leading dimension:
//   A K-major   A(m, k) = A[m lda + k]      A M-major   A(m, k) = A[k lda + m]
//   B K-major   B(k, n) = B[n ldb + k]      B N-major   B(k, n) = B[k ldb + n]
// (K-major is the [row][k] staging of gemm_f64.cuh; the M/N-major forms are staged [k][row]).
// Four warps (2 x 2) each own 32 x 32 of the tile; the contraction runs over 32-wide chunks
// double-buffered by cp.async, zero-filled past M, N and K.  With every leading dimension even and
// every base 16-byte aligned the copies move 16 bytes (two doubles), otherwise 8.
//
// Epilogues:
//   GEMM_STORE  C[m ldc + n] = alpha acc (+ beta C when beta != 0)
//   GEMM_PAIRS  the rows m are the elements of the packed lower block triangle (tile t = m / 4096,
//               row r and column c inside it, (mu, nu) = (64 I + r, 64 J + c)); each element with
//               mu >= nu, both below n_ao, goes to C[(mu (mu + 1) / 2 + nu) ldc + n] with weight 1 on
//               the diagonal and 2 off it (a stored pair stands for (mu nu) and (nu mu)).
// kdiag: the contraction index k runs over the packed triangle's elements, and products from a
// diagonal tile get weight 1/2 (each off-diagonal stored element then counts once, each element of
// a full-square sum over a diagonal tile once).
#include <algorithm>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

namespace rijk {
namespace {

constexpr int GM_THREADS = 128;
constexpr int GM_STAGE = (64 * LDK > KC * LDM) ? 64 * LDK : KC * LDM;  // doubles per operand stage

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  uint32_t s = smem_u32(smem);
  int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
// 16-byte copy of which the first `bytes` (0, 8 or 16) come from global memory, the rest zero.
__device__ __forceinline__ void cp_async16n(void* smem, const void* gmem, int bytes) {
  uint32_t s = smem_u32(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}

// One operand tile of 64 rows (m or n) x 32 k.  kmajor: global X[row * ld + k] staged [row][k]
// (stride LDK); else global X[k * ld + row] staged [k][row] (stride LDM).  `full`: every element of
// the tile is in bounds, so the copies skip the per-pair checks.
template <bool KMAJOR, bool VEC>
__device__ __forceinline__ void load_tile(double* sm, const double* __restrict__ X, long ld, long rows, long K,
                                          long r0, long k0, int tid, bool full) {
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int idx = tid + it * GM_THREADS;  // 1024 pairs of doubles
    int a, b;  // KMAJOR: a = row (0..63), b = k pair (0..15); else a = k (0..31), b = row pair (0..31)
    if (KMAJOR) {
      a = idx >> 4;
      b = idx & 15;
    } else {
      a = idx >> 5;
      b = idx & 31;
    }
    const long row = KMAJOR ? r0 + a : r0 + 2 * b;
    const long k = KMAJOR ? k0 + 2 * b : k0 + a;
    double* dst = KMAJOR ? sm + a * LDK + 2 * b : sm + a * LDM + 2 * b;
    const double* src = X + (KMAJOR ? row * ld + k : k * ld + row);
    if (full) {
      if (VEC) {
        cp_async16n(dst, src, 16);
      } else {
        cp_async8(dst, src, true);
        cp_async8(dst + 1, src + 1, true);
      }
      continue;
    }
    // valid doubles of the pair (the second runs along k for KMAJOR, along rows otherwise)
    int nv;
    if (KMAJOR)
      nv = row < rows ? static_cast<int>(min(2L, max(0L, K - k))) : 0;
    else
      nv = k < K ? static_cast<int>(min(2L, max(0L, rows - row))) : 0;
    if (VEC) {
      cp_async16n(dst, nv > 0 ? src : X, nv * 8);
    } else {
      cp_async8(dst, nv > 0 ? src : X, nv > 0);
      cp_async8(dst + 1, nv > 1 ? src + 1 : X, nv > 1);
    }
  }
}

template <bool AK, bool BK>
__device__ __forceinline__ void warp_mma_chunk_ab(double (&acc)[4][4][2], const double* __restrict__ sA,
                                                  const double* __restrict__ sB, int m0, int n0, int lane, double sc) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k = 0; k < KC; k += 4) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = AK ? sA[(m0 + i * 8 + g) * LDK + k + t] : sA[(k + t) * LDM + m0 + i * 8 + g];
    if (sc != 1.0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] *= sc;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = BK ? sB[(n0 + j * 8 + g) * LDK + k + t] : sB[(k + t) * LDM + n0 + j * 8 + g];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  }
}

template <bool AK, bool BK, bool VEC>
__global__ void __launch_bounds__(GM_THREADS) k_gemm_f64(GemmF64Args p, long ntn) {
  extern __shared__ __align__(16) double smem_gm[];
  double* sA[2] = {smem_gm, smem_gm + GM_STAGE};
  double* sB[2] = {smem_gm + 2 * GM_STAGE, smem_gm + 3 * GM_STAGE};
  // 1-D raster, N tiles fastest: the CTAs that share an A panel run together, so it is read from
  // HBM once and the (smaller) B operand is served from L2
  const long tile = blockIdx.x;
  const long m0 = (tile / ntn) * 64, n0 = (tile % ntn) * 64;
  const long bz = blockIdx.y;
  const double* A = p.A + bz * p.sA;
  const double* B = p.B + bz * p.sB;
  double* C = p.C + bz * p.sC;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const bool mfull = m0 + 64 <= p.M, nfull = n0 + 64 <= p.N;

  auto load = [&](int stage, long k0) {
    const bool kfull = k0 + KC <= p.K;
    load_tile<AK, VEC>(sA[stage], A, p.lda, p.M, p.K, m0, k0, tid, mfull && kfull);
    load_tile<BK, VEC>(sB[stage], B, p.ldb, p.N, p.K, n0, k0, tid, nfull && kfull);
  };
  double acc[4][4][2];
  zero_acc(acc);
  const long nk = (p.K + KC - 1) / KC;
  if (nk > 0) {  // K = 0 leaves acc at zero and issues no copy
    load(0, 0);
    cp_async_commit();
  }
  long diag_t = -1;  // kdiag: the packed tile of the current chunk and its weight
  double sc = 1.0;
  for (long kc = 0; kc < nk; ++kc) {
    if (kc + 1 < nk) {
      load(static_cast<int>((kc + 1) & 1), (kc + 1) * KC);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    if (p.kdiag && (kc * KC) / TILE2 != diag_t) {  // a 32-chunk lies inside one 64 x 64 tile
      diag_t = (kc * KC) / TILE2;
      long I, J;
      tri_decode(diag_t, I, J);
      sc = I == J ? 0.5 : 1.0;
    }
    __syncthreads();
    warp_mma_chunk_ab<AK, BK>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * 32, lane, sc);
    __syncthreads();
  }

  const int g = lane >> 2, tq = lane & 3;
  if (p.mode == GEMM_PAIRS) {
    // the CTA's 64 rows are one row r of one stored tile t: (mu, nu) = (64 I + r, 64 J + c)
    long I, J;
    tri_decode(m0 / TILE2, I, J);
    const long r = (m0 % TILE2) / TILE;
    const long mu = I * TILE + r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const long c = wm * 32 + i * 8 + g;
      const long nu = J * TILE + c;
      if (m0 + c >= p.M || mu >= p.n_ao || nu >= p.n_ao || (I == J && c > r)) continue;
      const double f = (mu == nu ? 1.0 : 2.0) * p.alpha;
      double* row = C + (mu * (mu + 1) / 2 + nu) * p.ldc;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const long n = n0 + wn * 32 + j * 8 + 2 * tq + h;
          if (n >= p.N) continue;
          double v = f * acc[i][j][h];
          if (p.beta != 0.0) v += p.beta * row[n];
          row[n] = v;
        }
      }
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long m = m0 + wm * 32 + i * 8 + g;
    if (m >= p.M) continue;
    double* row = C + m * p.ldc;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long n = n0 + wn * 32 + j * 8 + 2 * tq + h;
        if (n >= p.N) continue;
        double v = p.alpha * acc[i][j][h];
        if (p.beta != 0.0) v += p.beta * row[n];
        row[n] = v;
      }
    }
  }
}

template <bool AK, bool BK, bool VEC>
void launch_one(const GemmF64Args& p, long batch, cudaStream_t s) {
  const size_t smem = 4 * GM_STAGE * sizeof(double);
  ensure_smem_limit(reinterpret_cast<const void*>(k_gemm_f64<AK, BK, VEC>), smem);
  const long ntm = (p.M + 63) / 64, ntn = (p.N + 63) / 64;
  dim3 grid(static_cast<unsigned>(ntm * ntn), static_cast<unsigned>(batch));
  k_gemm_f64<AK, BK, VEC><<<grid, GM_THREADS, smem, s>>>(p, ntn);
}

bool aligned16(const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; }

}  // namespace

void gemm_f64(const GemmF64Args& p, long batch, cudaStream_t s) {
  if (p.M <= 0 || p.N <= 0 || batch <= 0) return;
  // grid limits: 2^31 - 1 tiles along x, 65535 batches along y (the callers stay far below both)
  // 16-byte copies need every row of both operands (and every batch) to start 16-byte aligned
  const bool vec = aligned16(p.A) && aligned16(p.B) && p.lda % 2 == 0 && p.ldb % 2 == 0 &&
                   (batch == 1 || (p.sA % 2 == 0 && p.sB % 2 == 0));
  const int key = (p.a_kmajor ? 4 : 0) | (p.b_kmajor ? 2 : 0) | (vec ? 1 : 0);
  switch (key) {
    case 0: launch_one<false, false, false>(p, batch, s); break;
    case 1: launch_one<false, false, true>(p, batch, s); break;
    case 2: launch_one<false, true, false>(p, batch, s); break;
    case 3: launch_one<false, true, true>(p, batch, s); break;
    case 4: launch_one<true, false, false>(p, batch, s); break;
    case 5: launch_one<true, false, true>(p, batch, s); break;
    case 6: launch_one<true, true, false>(p, batch, s); break;
    default: launch_one<true, true, true>(p, batch, s); break;
  }
}

}  // namespace rijk
