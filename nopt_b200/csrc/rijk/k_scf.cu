// k_scf.cu — restricted Hartree-Fock on the GPU around the Fock build (rijk_scf).
//
// The reference's RHF loop (src/SCF.cpp:78-223) builds D = sum_i C_i C_i^T (src/SCF.cpp:63-73),
// calls the RI Fock build, forms F = H + 2J - K and E = tr(F D) + tr(H D) + V_nuc
// (src/SCF.cpp:134) and takes an SOSCF/L-BFGS step.  Two convergers run here: Pulay DIIS on
// the commutator F D S - S D F in the orthogonal basis X = S^-1/2 (canonical, eigenvalues of S
// below `lindep` dropped), with diagonalisation of X^T F X; and the reference's SOSCF step
// (src/converger_2_1.cpp:55-125 with the L-BFGS of src/l-bfgs_2_1.cpp, built with
// LBFGS_RETURN_STEP): gradient g_ia = 4 F_ai and diagonal Hessian 4 (F_aa - F_ii) in the MO
// basis, a two-loop L-BFGS step capped at 0.1 per angle, the rotation I + X - X^T made
// orthonormal row by row (Gram-Schmidt, here as a QR factorisation with R's diagonal made
// positive, which gives the same rows) and applied to the orbitals.  The L-BFGS inner products
// stay on the device: each coefficient is read by the kernel that applies it.
// Everything n x n stays on the device in FP64: the small products are cuBLAS DGEMMs, the
// eigenproblems cuSOLVER syevd, the inner products deterministic two-stage reductions; only
// the DIIS coefficients ((m+1) x (m+1) system) are solved on the host.
//
// Matrices are column-major for cuBLAS.  H, S, F, D, J, K are symmetric, so their row-major
// and column-major forms coincide; the orbital matrix C (n x nmo, column i = orbital i) has
// the memory layout of the reference's MO_VEC (row i = orbital i), so its first n_c columns
// are passed to the Fock build as MO.
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "dmma.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

constexpr int kRedBlocks = 256;
constexpr int kRedThreads = 256;
constexpr int kOutSlots = 2 + 32 * 33 / 2;  // energy, error, lower triangle of a 32 x 32 Pulay matrix

// partial[b] (+ its compensation at partial[kRedBlocks + b]) = compensated sum over a grid-stride
// slice of f(i); the energy, DIIS inner products and norms all go through it.
template <typename F>
__global__ void k_reduce_partial(F f, long n, double* __restrict__ partial) {
  double s = 0.0, c = 0.0;
  for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * blockDim.x)
    neumaier_add(s, c, f(i));
  __shared__ double sh[2][kRedThreads / 32];
  warp_sum_comp(s, c);
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = s;
    sh[1][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kRedThreads / 32 ? sh[0][threadIdx.x] : 0.0;
    double w = threadIdx.x < kRedThreads / 32 ? sh[1][threadIdx.x] : 0.0;
    warp_sum_comp(v, w);
    if (threadIdx.x == 0) {
      partial[blockIdx.x] = v;
      partial[kRedBlocks + blockIdx.x] = w;
    }
  }
}

template <typename F>
__global__ void k_reduce_max_partial(F f, long n, double* __restrict__ partial) {
  double acc = 0.0;
  for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * blockDim.x)
    acc = fmax(acc, f(i));
  __shared__ double sh[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_xor_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kRedThreads / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// out[slot] = sum (compensated, partials and their compensations) or max of the kRedBlocks
// partials, in a fixed order: launched with kRedBlocks threads, thread b takes partial b, then a
// fixed shuffle tree per warp and the warps in order (deterministic).
__global__ void k_reduce_final(const double* __restrict__ partial, int is_max, double* __restrict__ out, int slot) {
  __shared__ double sh[2][kRedBlocks / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (is_max) {
    double m = partial[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) sh[0][warp] = m;
    __syncthreads();
    if (t == 0) {
      m = sh[0][0];
      for (int w = 1; w < kRedBlocks / 32; ++w) m = fmax(m, sh[0][w]);
      out[slot] = m;
    }
  } else {
    double v = partial[t], c = partial[kRedBlocks + t];
    warp_sum_comp(v, c);
    if (lane == 0) {
      sh[0][warp] = v;
      sh[1][warp] = c;
    }
    __syncthreads();
    if (t == 0) {
      v = sh[0][0];
      c = sh[1][0];
      for (int w = 1; w < kRedBlocks / 32; ++w) {
        neumaier_add(v, c, sh[0][w]);
        c += sh[1][w];
      }
      out[slot] = v + c;
    }
  }
}

struct DotF {
  const double* a;
  const double* b;
  __device__ double operator()(long i) const { return a[i] * b[i]; }
};
struct EnergyF {  // D (F + H)
  const double* d;
  const double* f;
  const double* h;
  __device__ double operator()(long i) const { return d[i] * (f[i] + h[i]); }
};
struct DiffSqF {
  const double* a;
  const double* b;
  __device__ double operator()(long i) const {
    double t = a[i] - b[i];
    return t * t;
  }
};
struct AbsF {
  const double* a;
  __device__ double operator()(long i) const { return fabs(a[i]); }
};

__global__ void k_scale_cols(const double* __restrict__ U, const double* __restrict__ w, long n, long first,
                             long nm, double* __restrict__ X) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < n * nm; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long col = idx / n, row = idx % n;
    X[idx] = U[row + (first + col) * n] / sqrt(w[first + col]);
  }
}

// F = H + 2J - K ; A = F - F^T style antisymmetrisation is done separately
__global__ void k_fock(const double* __restrict__ H, const double* __restrict__ J, const double* __restrict__ K,
                       long nn, double* __restrict__ F) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < nn; idx += static_cast<long>(gridDim.x) * blockDim.x) F[idx] = H[idx] + 2.0 * J[idx] - K[idx];
}

// E = A - A^T (column-major n x n)
__global__ void k_antisym(const double* __restrict__ A, long n, double* __restrict__ E) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < n * n; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long r = idx % n, c = idx / n;
    E[idx] = A[idx] - A[c + r * n];
  }
}

__global__ void k_axpy_set(double c, const double* __restrict__ x, long n, double* __restrict__ y, int first) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < n; idx += static_cast<long>(gridDim.x) * blockDim.x) y[idx] = first ? c * x[idx] : y[idx] + c * x[idx];
}

// ---- SOSCF (src/converger_2_1.cpp:55-125)
// g[i nv + a] = 4 F_MO[nocc + a][i], h[i nv + a] = 4 (F_MO[nocc + a][nocc + a] - F_MO[i][i])
__global__ void k_soscf_grad(const double* __restrict__ Fmo, long nm, long nocc, double* __restrict__ g,
                             double* __restrict__ h) {
  const long nv = nm - nocc;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < nocc * nv;
       idx += static_cast<long>(gridDim.x) * blockDim.x) {
    const long i = idx / nv, a = nocc + idx % nv;
    g[idx] = 4.0 * Fmo[a + i * nm];
    h[idx] = 4.0 * (Fmo[a * (nm + 1)] - Fmo[i * (nm + 1)]);
  }
}

__global__ void k_sub(const double* __restrict__ a, const double* __restrict__ b, long n, double* __restrict__ out) {
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n;
       idx += static_cast<long>(gridDim.x) * blockDim.x)
    out[idx] = a[idx] - b[idx];
}

// y += (ca dev[sa] + cb dev[sb]) x, a slot < 0 contributing nothing: the L-BFGS updates with
// their inner products taken from device memory.
__global__ void k_axpy_dev(double* __restrict__ y, const double* __restrict__ x, long n, const double* __restrict__ dev,
                           int sa, double ca, int sb, double cb) {
  const double c = (sa >= 0 ? ca * dev[sa] : 0.0) + (sb >= 0 ? cb * dev[sb] : 0.0);
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n;
       idx += static_cast<long>(gridDim.x) * blockDim.x)
    y[idx] += c * x[idx];
}

__global__ void k_div(const double* __restrict__ q, const double* __restrict__ h, long n, double* __restrict__ s) {
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n;
       idx += static_cast<long>(gridDim.x) * blockDim.x)
    s[idx] = q[idx] / h[idx];
}

// x = s zoom and x2 = s zoom, zoom = -min(1, xmax / max|s|) with max|s| at dev[smax]
// (src/l-bfgs_2_1.cpp:96-110, :118-121); the zoom is also stored at dev[szoom].
__global__ void k_zoom(const double* __restrict__ s, long n, double* __restrict__ dev, int smax, int szoom, double xmax,
                       double* __restrict__ x, double* __restrict__ x2) {
  const double m = dev[smax];
  const double zoom = (m > xmax) ? -xmax / m : -1.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) dev[szoom] = zoom;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n;
       idx += static_cast<long>(gridDim.x) * blockDim.x) {
    const double v = s[idx] * zoom;
    x[idx] = v;
    x2[idx] = v;
  }
}

// R[p][q] (row-major, nm x nm) = delta_pq + X_pq - X_qp with X[i][nocc + a] = x[i nv + a]
// (src/converger_2_1.cpp:107-113)
__global__ void k_rot_build(const double* __restrict__ x, long nm, long nocc, double* __restrict__ R) {
  const long nv = nm - nocc;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < nm * nm;
       idx += static_cast<long>(gridDim.x) * blockDim.x) {
    const long p = idx / nm, q = idx % nm;
    double v = p == q ? 1.0 : 0.0;
    if (p < nocc && q >= nocc) v = x[p * nv + (q - nocc)];
    if (q < nocc && p >= nocc) v = -x[q * nv + (p - nocc)];
    R[idx] = v;
  }
}

unsigned grid_of(long total) {
  long b = (total + 255) / 256;
  if (b > 148L * 8) b = 148L * 8;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

// ---- occupied projector by trace-correcting purification (TC2: A. M. N. Niklasson, Phys. Rev. B 66,
// 155115 (2002)).  The new density of a DIIS step is the projector on the n_c lowest eigenvectors of
// F' = X^T F X; purification reaches it with n' x n' products alone.  F' is mapped to
// P0 = (b I - F') / 2b, b = max_j sum_i |F'_ij| >= its spectral radius, so P0's eigenvalues lie in
// [0, 1] with the occupied ones highest; each step P <- P^2 or 2P - P^2, whichever trace is nearer
// n_c, drives them to 1 and the rest to 0 while keeping the eigenvectors.

// out[j] = sum_i |A_ij| (column-major n x n; for a symmetric A the absolute row sums): a warp per column
__global__ void k_col_abs_sum(const double* __restrict__ A, long n, double* __restrict__ out) {
  const long j = static_cast<long>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (j >= n) return;
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (long i = lane; i < n; i += 32) acc += fabs(A[i + j * n]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[j] = acc;
}

// One block: sc[slot] = the largest of v[0 .. n) (1 if that is 0).
__global__ void k_max_small(const double* __restrict__ v, long n, double* __restrict__ sc, int slot) {
  __shared__ double sh[32];
  double m = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, v[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x / 32); ++w) m = fmax(m, sh[w]);
    m = fmax(m, sh[0]);
    sc[slot] = m > 0.0 ? m : 1.0;
  }
}

// A <- (b I - A) / 2b in place, b = sc[0]
__global__ void k_purify_init(double* __restrict__ A, long n, const double* __restrict__ sc) {
  const double b = sc[0], h = 0.5 / b;
  for (long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n * n;
       idx += static_cast<long>(gridDim.x) * blockDim.x)
    A[idx] = ((idx % n == idx / n ? b : 0.0) - A[idx]) * h;
}

// One block: sc[1] = tr P, sc[2] = tr P2 (a fixed summation order)
__global__ void k_tc2_traces(const double* __restrict__ P, const double* __restrict__ P2, long n,
                             double* __restrict__ sc) {
  __shared__ double sh[2][32];
  double a = 0.0, c = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    a += P[i * (n + 1)];
    c += P2[i * (n + 1)];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a;
    sh[1][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = 0.0;
    c = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) {
      a += sh[0][w];
      c += sh[1][w];
    }
    sc[1] = a;
    sc[2] = c;
  }
}

// P <- P2 when tr P2 is nearer n_c than tr(2P - P2), else 2P - P2 (traces from sc), with P2 = P^T P
// given in its upper triangle (DSYRK, half the products of a GEMM): one 32 x 32 block per tile
// (ti, tj), ti <= tj, of the upper triangle; it updates that tile and its mirror, through shared
// memory so both accesses are coalesced.  P is symmetric and stays so.
__global__ void __launch_bounds__(256) k_tc2_update_sym(double* __restrict__ P, const double* __restrict__ P2,
                                                        long n, const double* __restrict__ sc, double nocc) {
  __shared__ double t[32][33];
  long ti = 0, rem = blockIdx.x;
  const long nb = (n + 31) / 32;
  while (rem >= nb - ti) {  // tile index -> (ti, tj), tj >= ti, row by row of the upper block triangle
    rem -= nb - ti;
    ++ti;
  }
  const long tj = ti + rem;
  const double t1 = sc[1], t2 = sc[2];
  const bool square = fabs(t2 - nocc) < fabs(2.0 * t1 - t2 - nocc);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  // t[c][r] = P2(ti*32 + r, tj*32 + c), from the upper triangle (within a diagonal tile, r <= c)
  for (int c = ty; c < 32; c += 8) {
    const long i = ti * 32 + tx, j = tj * 32 + c;
    t[c][tx] = (i < n && j < n) ? P2[i + j * n] : 0.0;
  }
  __syncthreads();
  for (int c = ty; c < 32; c += 8) {  // the tile itself: element (ti*32 + tx, tj*32 + c)
    const long i = ti * 32 + tx, j = tj * 32 + c;
    if (i < n && j < n && (ti != tj || tx <= c)) {
      const double p2 = t[c][tx];
      P[i + j * n] = square ? p2 : 2.0 * P[i + j * n] - p2;
    }
  }
  for (int r = ty; r < 32; r += 8) {  // its mirror: element (tj*32 + tx, ti*32 + r) = P2(ti*32 + r, tj*32 + tx)
    const long i = tj * 32 + tx, j = ti * 32 + r;
    if (i < n && j < n && (ti != tj || tx > r)) {
      const double p2 = t[tx][r];
      P[i + j * n] = square ? p2 : 2.0 * P[i + j * n] - p2;
    }
  }
}

// ---- one TC2 step in one kernel, for n' <= 512.  At n' = 384 a step of the form above (the library
// product, then the trace and update kernels) took about 23 us, most of it launch latency.  Here a CTA of
// 4 warps forms a 32 x 32 tile of P^2 on DMMA (warps 2 x 2, 16 x 16 each) over 32-wide chunks of k
// staged [k][row] (stride T2_LD, conflict-free as in dmma.cuh) through a three-stage cp.async pipeline.
// P is symmetric, so P(k, j) = P(j, k):
// both operands are columns of P, with the rows contiguous.  The choice between P^2 and 2P - P^2 needs
// tr P and tr P^2 = ||P||_F^2 of the input, which the previous step (or k_tc2_norms) left as partial sums,
// one pair per tile: lane 0 of warp 0 of every CTA adds them in the same fixed order, so every CTA, and
// every rank of a sharded SCF, takes the same branch.  The epilogue writes Pn and its tile's own partial
// sums; CTA (0, 0) also writes tr P and tr P^2 to sc[1], sc[2] for the host's convergence test.
constexpr int T2 = 32;
constexpr int T2_LD = 36;
constexpr int T2_THREADS = 128;

__device__ __forceinline__ void t2_cp8(double* smem, const double* gmem, bool valid) {
  const uint32_t d = smem_u32(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gmem), "r"(valid ? 8 : 0));
}

// this CTA's (sum of the diagonal, sum of squares) of v over its threads, in a fixed order
__device__ __forceinline__ void t2_tile_sums(double sdg, double ssq, double* __restrict__ part_out) {
  __shared__ double red[2][T2_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sdg += __shfl_down_sync(0xffffffffu, sdg, o);
    ssq += __shfl_down_sync(0xffffffffu, ssq, o);
  }
  if (lane == 0) {
    red[0][warp] = sdg;
    red[1][warp] = ssq;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const long blk = static_cast<long>(blockIdx.y) * gridDim.x + blockIdx.x;
    double a = 0.0, b = 0.0;
    for (int w = 0; w < T2_THREADS / 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    part_out[2 * blk] = a;
    part_out[2 * blk + 1] = b;
  }
}

// The partial sums of P0 (column-major n x n), one pair per 32 x 32 tile of the step's grid.
__global__ void __launch_bounds__(T2_THREADS) k_tc2_norms(const double* __restrict__ P, long n,
                                                          double* __restrict__ part_out) {
  const long r0 = static_cast<long>(blockIdx.y) * T2, c0 = static_cast<long>(blockIdx.x) * T2;
  double sdg = 0.0, ssq = 0.0;
  for (int e = threadIdx.x; e < T2 * T2; e += T2_THREADS) {
    const long r = r0 + (e & 31), c = c0 + (e >> 5);
    if (r < n && c < n) {
      const double v = P[r + c * n];
      ssq += v * v;
      if (r == c) sdg += v;
    }
  }
  t2_tile_sums(sdg, ssq, part_out);
}

constexpr int T2_STAGES = 3;
constexpr size_t T2_SMEM = static_cast<size_t>(T2_STAGES) * 2 * T2 * T2_LD * sizeof(double);

// 16-byte copy of which the first `bytes` (0, 8 or 16) come from global memory, the rest zero
__device__ __forceinline__ void t2_cp16(double* smem, const double* gmem, int bytes) {
  const uint32_t d = smem_u32(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem), "r"(bytes));
}

// PAIRS: n is even, so (row, k) pairs of rows start on 16-byte boundaries and move as one copy
template <bool PAIRS>
__global__ void __launch_bounds__(T2_THREADS) k_tc2_step(const double* __restrict__ P, double* __restrict__ Pn, long n,
                                                         const double* __restrict__ part_in,
                                                         double* __restrict__ part_out, double nocc,
                                                         double* __restrict__ sc) {
  extern __shared__ __align__(16) double t2s[];  // T2_STAGES x {A, B} chunks of [k][row]
  __shared__ double tr[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long r0 = static_cast<long>(blockIdx.y) * T2, c0 = static_cast<long>(blockIdx.x) * T2;
  const int nblk = gridDim.x * gridDim.y;
  if (warp == 0) {  // tr P and ||P||_F^2 from the input's partial sums, in a fixed order
    double a = 0.0, b = 0.0;
    for (int i = lane; i < nblk; i += 32) {
      a += part_in[2 * i];
      b += part_in[2 * i + 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      tr[0] = a;
      tr[1] = b;
      if (blockIdx.x == 0 && blockIdx.y == 0) {
        sc[1] = a;
        sc[2] = b;
      }
    }
  }
  auto stage_a = [&](int st) { return t2s + static_cast<size_t>(st) * 2 * T2 * T2_LD; };
  auto load = [&](int st, long k0) {  // element (row, k) of a column block: P[row + k n]
    double* sA = stage_a(st);
    double* sB = sA + T2 * T2_LD;
    if (PAIRS) {
      for (int e = tid; e < T2 * T2 / 2; e += T2_THREADS) {
        const int kk = e >> 4, rr = (e & 15) * 2;
        const long k = k0 + kk, ra = r0 + rr, rb = c0 + rr;
        const int ba = k < n ? static_cast<int>(8 * std::max<long>(0, std::min<long>(2, n - ra))) : 0;
        const int bb = k < n ? static_cast<int>(8 * std::max<long>(0, std::min<long>(2, n - rb))) : 0;
        t2_cp16(&sA[kk * T2_LD + rr], ba ? P + ra + k * n : P, ba);
        t2_cp16(&sB[kk * T2_LD + rr], bb ? P + rb + k * n : P, bb);
      }
    } else {
      for (int e = tid; e < T2 * T2; e += T2_THREADS) {
        const int kk = e >> 5, rr = e & 31;
        const long k = k0 + kk, ra = r0 + rr, rb = c0 + rr;
        const bool va = k < n && ra < n, vb = k < n && rb < n;
        t2_cp8(&sA[kk * T2_LD + rr], va ? P + ra + k * n : P, va);
        t2_cp8(&sB[kk * T2_LD + rr], vb ? P + rb + k * n : P, vb);
      }
    }
  };
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
  double acc[2][2][2] = {};
  const long nk = (n + T2 - 1) / T2;
  load(0, 0);
  cp_async_commit();
  if (nk > 1) {
    load(1, T2);
    cp_async_commit();
  }
  for (long kc = 0; kc < nk; ++kc) {
    if (kc + 2 < nk) {
      load(static_cast<int>((kc + 2) % T2_STAGES), (kc + 2) * T2);
      cp_async_commit();
      cp_async_wait<2>();
    } else if (kc + 1 < nk) {
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* a_ = stage_a(static_cast<int>(kc % T2_STAGES));
    const double* b_ = a_ + T2 * T2_LD;
#pragma unroll
    for (int k = 0; k < T2; k += 4) {
      double a[2], b[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) a[i] = a_[(k + t) * T2_LD + wm * 16 + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = b_[(k + t) * T2_LD + wn * 16 + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
  const double t1 = tr[0], t2 = tr[1];
  const bool square = fabs(t2 - nocc) < fabs(2.0 * t1 - t2 - nocc);
  double sdg = 0.0, ssq = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long r = r0 + wm * 16 + i * 8 + g, c = c0 + wn * 16 + j * 8 + 2 * t + h;
        if (r < n && c < n) {
          const double s2 = acc[i][j][h];
          const double v = square ? s2 : 2.0 * P[r + c * n] - s2;
          Pn[r + c * n] = v;
          ssq += v * v;
          if (r == c) sdg += v;
        }
      }
  t2_tile_sums(sdg, ssq, part_out);
}

// One fused step; the launch configuration for n' (even n': 16-byte copies).
void launch_tc2_step(const double* P, double* Pn, long n, const double* part_in, double* part_out, double nocc,
                     double* sc, cudaStream_t s) {
  const unsigned nb = static_cast<unsigned>((n + T2 - 1) / T2);
  if (n % 2 == 0) {
    ensure_smem_limit(reinterpret_cast<const void*>(k_tc2_step<true>), T2_SMEM);
    k_tc2_step<true><<<dim3(nb, nb), T2_THREADS, T2_SMEM, s>>>(P, Pn, n, part_in, part_out, nocc, sc);
  } else {
    ensure_smem_limit(reinterpret_cast<const void*>(k_tc2_step<false>), T2_SMEM);
    k_tc2_step<false><<<dim3(nb, nb), T2_THREADS, T2_SMEM, s>>>(P, Pn, n, part_in, part_out, nocc, sc);
  }
}

// One block: sc[slot] = min_i |R_ii| / max_i |R_ii| of a Cholesky factor (n x n, column-major)
__global__ void k_chol_ratio(const double* __restrict__ R, long n, double* __restrict__ sc, int slot) {
  __shared__ double sh[2][32];
  double lo = 1e300, hi = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = fabs(R[i * (n + 1)]);
    lo = fmin(lo, d);
    hi = fmax(hi, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = lo;
    sh[1][threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) {
      lo = fmin(lo, sh[0][w]);
      hi = fmax(hi, sh[1][w]);
    }
    sc[slot] = hi > 0.0 && lo == lo ? lo / hi : 0.0;
  }
}

// Solves the (m+1) x (m+1) Pulay system by Gaussian elimination with partial pivoting.
bool diis_coefficients(const std::vector<double>& Bm, int m, std::vector<double>& c) {
  const int N = m + 1;
  std::vector<double> A(static_cast<size_t>(N) * N), rhs(N, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) A[i * N + j] = Bm[i * m + j];
  for (int i = 0; i < m; ++i) A[i * N + m] = A[m * N + i] = -1.0;
  A[m * N + m] = 0.0;
  rhs[m] = -1.0;
  for (int k = 0; k < N; ++k) {
    int p = k;
    for (int i = k + 1; i < N; ++i)
      if (std::fabs(A[i * N + k]) > std::fabs(A[p * N + k])) p = i;
    if (std::fabs(A[p * N + k]) < 1e-300) return false;
    if (p != k) {
      for (int j = 0; j < N; ++j) std::swap(A[k * N + j], A[p * N + j]);
      std::swap(rhs[k], rhs[p]);
    }
    for (int i = k + 1; i < N; ++i) {
      double f = A[i * N + k] / A[k * N + k];
      for (int j = k; j < N; ++j) A[i * N + j] -= f * A[k * N + j];
      rhs[i] -= f * rhs[k];
    }
  }
  std::vector<double> x(N);
  for (int i = N - 1; i >= 0; --i) {
    double s = rhs[i];
    for (int j = i + 1; j < N; ++j) s -= A[i * N + j] * x[j];
    x[i] = s / A[i * N + i];
  }
  c.assign(x.begin(), x.begin() + m);
  for (double v : c)
    if (!std::isfinite(v)) return false;
  return true;
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_scf(rijk_ctx* ctx, const double* H, const double* S, long nocc, double e_nuc,
                      const rijk_scf_opts_t* opts, double* MO, rijk_scf_result_t* result) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!H || !S || !result) return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: null pointer");
  NvtxRange range("rijk_scf");
  rijk_scf_opts_t o{};
  if (opts) o = *opts;
  if (o.max_iter <= 0) o.max_iter = 100;
  if (o.conv_dm_rms <= 0) o.conv_dm_rms = 1e-10;
  if (o.switch_diis_err <= 0) o.switch_diis_err = 1e-5;
  if (o.diis_size <= 0) o.diis_size = 8;
  if (o.lindep <= 0) o.lindep = 1e-10;
  if (o.conv_grad <= 0) o.conv_grad = 1e-7;      // RHF_GR_CON_DEFAULT (include/defaults.h:7)
  if (o.conv_energy <= 0) o.conv_energy = 1e-10;  // RHF_EN_CON_DEFAULT (include/defaults.h:6)
  if (o.converger != RIJK_CONV_DIIS && o.converger != RIJK_CONV_SOSCF && o.converger != RIJK_CONV_DIIS_SOSCF)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: unknown converger %d", o.converger);
  if (o.lbfgs_vectors < 0 || o.lbfgs_vectors > 32)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: lbfgs_vectors outside 0 .. 32");
  const bool soscf = o.converger == RIJK_CONV_SOSCF;         // SOSCF from the start
  const bool hybrid = o.converger == RIJK_CONV_DIIS_SOSCF;   // DIIS, then SOSCF from the switch on
  int rc = check_fock_args(ctx, nocc, o.precision);
  if (rc) return rc;
  if (o.fp64_phase_precision != 0 && o.fp64_phase_precision != RIJK_PREC_FP64_TC)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: fp64_phase_precision must be 0 (FP64) or RIJK_PREC_FP64_TC");
  // the form of the FP64-accurate builds after a mixed phase, and of a closing build
  const int prec_fp64 = o.fp64_phase_precision == RIJK_PREC_FP64_TC ? RIJK_PREC_FP64_TC : RIJK_PREC_FP64;
  if (o.diis_size > 32) return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: diis_size above 32");
  if (o.guess_dm && (!o.guess_rows || o.guess_nrows <= 0 || o.guess_nrows > round_up(ctx->n, 16)))
    return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: guess needs factor rows (1 .. n_ao of them)");
  if (ctx->nq != ctx->naux && !o.reduce_jk)
    return set_err(ctx, RIJK_ERR_STATE,
                   "rijk_scf on an aux range [%ld, %ld) needs opts->reduce_jk to sum J and K over the ranks", ctx->q0,
                   ctx->q0 + ctx->nq);
  if (o.ao_projector && (o.n_proj < 1 || o.n_proj > ctx->n))
    return set_err(ctx, RIJK_ERR_ARG, "rijk_scf: n_proj = %ld outside [1, n_ao = %ld]", o.n_proj, ctx->n);
  cudaSetDevice(ctx->device);
  const auto t_start = std::chrono::steady_clock::now();
  const long n = ctx->n, nn = n * n;
  const int ni = static_cast<int>(n);
  cudaStream_t s = ctx->stream;
  cublasHandle_t cb = ctx->cublas;
  cusolverDnHandle_t cs = ctx->cusolver;
  const int m_max = o.diis_size;

  // Work buffers live in the context between calls (grown as needed, freed by rijk_destroy): an SCF
  // call then makes no cudaMalloc / cudaFree, whose frees synchronise the device.
  DeviceBuf* wb = ctx->scf;
  DeviceBuf &dH = wb[0], &dS = wb[1], &dX = wb[2], &dF = wb[3], &dFex = wb[4], &dD = wb[5], &dDn = wb[6],
            &dC = wb[7], &dJK = wb[8], &dT1 = wb[10], &dT2 = wb[11], &dE = wb[12], &dW = wb[13],
            &dU = wb[14], &work = wb[15], &info = wb[16], &red = wb[17], &out = wb[18], &ring_F = wb[19],
            &ring_E = wb[20];
  // occupied eigenvectors (X basis), purification scalars, Cholesky infos, the fused TC2 steps' partial sums
  DeviceBuf &dV = wb[21], &dPur = wb[22], &dInfo2 = wb[23], &dPart = wb[28];
  auto cleanup = [&]() {};  // nothing to free: the buffers stay with the context
  const size_t b_nn = nn * sizeof(double);
  if ((rc = ensure(ctx, dH, b_nn, "scf H")) || (rc = ensure(ctx, dS, b_nn, "scf S")) ||
      (rc = ensure(ctx, dX, b_nn, "scf X")) || (rc = ensure(ctx, dF, b_nn, "scf F")) ||
      (rc = ensure(ctx, dFex, b_nn, "scf Fex")) || (rc = ensure(ctx, dD, b_nn, "scf D")) ||
      (rc = ensure(ctx, dDn, b_nn, "scf Dn")) || (rc = ensure(ctx, dC, b_nn, "scf C")) ||
      (rc = ensure(ctx, dJK, 2 * b_nn, "scf J, K")) ||
      (rc = ensure(ctx, dT1, b_nn, "scf T1")) || (rc = ensure(ctx, dT2, b_nn, "scf T2")) ||
      (rc = ensure(ctx, dE, b_nn, "scf E")) || (rc = ensure(ctx, dU, b_nn, "scf U")) ||
      (rc = ensure(ctx, dW, n * sizeof(double), "scf w")) || (rc = ensure(ctx, info, sizeof(int), "scf info")) ||
      (rc = ensure(ctx, red, 2 * kRedBlocks * sizeof(double), "scf reduce")) ||
      (rc = ensure(ctx, out, kOutSlots * sizeof(double), "scf out")) ||
      (rc = ensure(ctx, ring_F, static_cast<size_t>(m_max) * b_nn, "scf DIIS F")) ||
      (rc = ensure(ctx, ring_E, static_cast<size_t>(m_max) * b_nn, "scf DIIS e")) ||
      (rc = ensure(ctx, dV, static_cast<size_t>(n) * std::max<long>(nocc, 1) * sizeof(double), "scf V")) ||
      (rc = ensure(ctx, dPur, 16 * sizeof(double), "scf purification")) ||
      (rc = ensure(ctx, dPart, 4 * 32 * 32 * sizeof(double), "scf purification partial sums")) ||
      (rc = ensure(ctx, dInfo2, 4 * sizeof(int), "scf Cholesky info"))) {
    cleanup();
    return rc;
  }
  double* pH = static_cast<double*>(dH.p);
  double* pS = static_cast<double*>(dS.p);
  double* pX = static_cast<double*>(dX.p);
  double* pF = static_cast<double*>(dF.p);
  double* pFex = static_cast<double*>(dFex.p);
  double* pD = static_cast<double*>(dD.p);
  double* pDn = static_cast<double*>(dDn.p);
  double* pC = static_cast<double*>(dC.p);
  double* pJ = static_cast<double*>(dJK.p);  // [J | K]: one array for the ranks' reduction
  double* pK = pJ + nn;
  double* pT1 = static_cast<double*>(dT1.p);
  double* pT2 = static_cast<double*>(dT2.p);
  double* pU = static_cast<double*>(dU.p);
  double* pW = static_cast<double*>(dW.p);
  double* pRed = static_cast<double*>(red.p);
  double* pOut = static_cast<double*>(out.p);
  double* rF = static_cast<double*>(ring_F.p);
  double* rE = static_cast<double*>(ring_E.p);
  double* pV = static_cast<double*>(dV.p);
  double* pPur = static_cast<double*>(dPur.p);
  int* pInfo2 = static_cast<int*>(dInfo2.p);
  int* pInfo = static_cast<int*>(info.p);
  const double one = 1.0, zero = 0.0;

  auto fail = [&](int code, const char* msg) {
    cleanup();
    return set_err(ctx, code, "rijk_scf: %s", msg);
  };
  // the sum of the ranks' partial J and K (aux-sharded SCF), by the caller's collective
  auto reduce_jk = [&]() -> int {
    if (!o.reduce_jk) return RIJK_OK;
    if (const int r = o.reduce_jk(pJ, 2 * nn, static_cast<void*>(s), o.reduce_user))
      return set_err(ctx, RIJK_ERR_REDUCE, "rijk_scf: reduce_jk returned %d", r);
    return cuda_check(ctx, cudaGetLastError(), "rijk_scf reduce_jk");
  };
  auto reduce = [&](auto f, long count, int is_max, int slot) {
    if (is_max)
      k_reduce_max_partial<<<kRedBlocks, kRedThreads, 0, s>>>(f, count, pRed);
    else
      k_reduce_partial<<<kRedBlocks, kRedThreads, 0, s>>>(f, count, pRed);
    k_reduce_final<<<1, kRedBlocks, 0, s>>>(pRed, is_max, pOut, slot);
  };

  cudaMemcpyAsync(pH, H, b_nn, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(pS, S, b_nn, cudaMemcpyHostToDevice, s);

  // eigensolver workspace: the larger of the S and F' problems (both n x n at most)
  int lwork = 0;
  if (cusolverDnDsyevd_bufferSize(cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, ni, pU, ni, pW, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(RIJK_ERR_SOLVER, "syevd buffer query failed");
  if ((rc = ensure(ctx, work, static_cast<size_t>(lwork) * sizeof(double), "scf syevd work"))) {
    cleanup();
    return rc;
  }
  double* pWork = static_cast<double*>(work.p);

  // X = U_k w_k^-1/2 over eigenvalues of S above lindep (ascending: drop the first ndrop).  With a
  // projector T (n x np), the same from S' = T^T S T, and X = T U'_k w'_k^-1/2: the orbitals then
  // lie in the span of T's columns (the reference's D5 treatment).
  const bool proj = o.ao_projector != nullptr;
  const long np = proj ? o.n_proj : n;
  const int npi = static_cast<int>(np);
  DeviceBuf& dP = wb[27];
  if (proj) {
    // T row-major (n x np) is, read column-major with ld np, T^T (np x n)
    if ((rc = ensure(ctx, dP, static_cast<size_t>(n) * np * sizeof(double), "scf projector"))) {
      cleanup();
      return rc;
    }
    cudaMemcpyAsync(dP.p, o.ao_projector, static_cast<size_t>(n) * np * sizeof(double), cudaMemcpyHostToDevice, s);
    const double* pP = static_cast<const double*>(dP.p);
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, ni, npi, ni, &one, pS, ni, pP, npi, &zero, pT1, ni);   // S T
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, npi, npi, ni, &one, pP, npi, pT1, ni, &zero, pU, npi);  // T^T S T
  } else {
    cudaMemcpyAsync(pU, pS, b_nn, cudaMemcpyDeviceToDevice, s);
  }
  if (cusolverDnDsyevd(cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, npi, pU, npi, pW, pWork, lwork, pInfo) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(RIJK_ERR_SOLVER, "syevd of S failed");
  std::vector<double> ws(np);
  int hinfo = 0;
  cudaMemcpyAsync(ws.data(), pW, np * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&hinfo, pInfo, sizeof(int), cudaMemcpyDeviceToHost, s);
  if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf overlap"))) {
    cleanup();
    return rc;
  }
  if (hinfo != 0) return fail(RIJK_ERR_SOLVER, "overlap eigendecomposition did not converge");
  long first = 0;
  while (first < np && ws[first] < o.lindep) ++first;
  const long nm = np - first;
  if (nm < nocc) return fail(RIJK_ERR_ARG, "fewer independent orbitals than n_c");
  const int nmi = static_cast<int>(nm);
  if (proj) {
    k_scale_cols<<<grid_of(np * nm), 256, 0, s>>>(pU, pW, np, first, nm, pT2);  // X' (np x nm)
    cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, ni, nmi, npi, &one, static_cast<const double*>(dP.p), npi, pT2, npi,
                &zero, pX, ni);  // X = T X'
  } else {
    k_scale_cols<<<grid_of(n * nm), 256, 0, s>>>(pU, pW, n, first, nm, pX);
  }

  // Inside the loop only the n_c occupied orbitals are needed: syevdx for the lowest n_c
  // eigenpairs (all of them, with syevd, for the final orbitals).
  const int nev = static_cast<int>(std::max<long>(nocc, 1));
  int lworkx = 0, meig = 0;
  if (cusolverDnDsyevdx_bufferSize(cs, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER, nmi,
                                   pU, nmi, 0.0, 0.0, 1, nev, &meig, pW, &lworkx) != CUSOLVER_STATUS_SUCCESS)
    return fail(RIJK_ERR_SOLVER, "syevdx buffer query failed");
  int lworkp = 0;  // Cholesky of the n_c x n_c Gram matrix in the purification step
  if (nocc > 0 && cusolverDnDpotrf_bufferSize(cs, CUBLAS_FILL_MODE_UPPER, static_cast<int>(nocc), pT2,
                                              static_cast<int>(nocc), &lworkp) != CUSOLVER_STATUS_SUCCESS)
    return fail(RIJK_ERR_SOLVER, "Cholesky buffer query failed");
  if (std::max(lworkx, lworkp) > lwork) {
    if ((rc = ensure(ctx, work, static_cast<size_t>(std::max(lworkx, lworkp)) * sizeof(double),
                     "scf syevdx work"))) {
      cleanup();
      return rc;
    }
    pWork = static_cast<double*>(work.p);
  }
  // diagonalise X^T F X -> C = X V (first nm columns of pC, or the first n_c when partial)
  auto diag = [&](const double* Fm, bool all = false) -> int {
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, nmi, ni, &one, Fm, ni, pX, ni, &zero, pT1, ni);    // F X
    cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, nmi, nmi, ni, &one, pX, ni, pT1, ni, &zero, pU, nmi);  // X^T F X
    int ncols = nmi;
    if (all) {
      if (cusolverDnDsyevd(cs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nmi, pU, nmi, pW, pWork, lwork,
                           pInfo) != CUSOLVER_STATUS_SUCCESS)
        return RIJK_ERR_SOLVER;
    } else {
      if (cusolverDnDsyevdx(cs, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER, nmi, pU, nmi,
                            0.0, 0.0, 1, nev, &meig, pW, pWork, std::max(lwork, lworkx), pInfo) !=
          CUSOLVER_STATUS_SUCCESS)
        return RIJK_ERR_SOLVER;
      ncols = nev;
    }
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, ncols, nmi, &one, pX, ni, pU, nmi, &zero, pC, ni);  // C = X V
    if (nocc > 0)  // the occupied eigenvectors start the next purification step's subspace
      cudaMemcpyAsync(pV, pU, static_cast<size_t>(nm) * nocc * sizeof(double), cudaMemcpyDeviceToDevice, s);
    return RIJK_OK;
  };
  // The occupied orbitals of a DIIS step without an eigensolver: the projector P on the n_c lowest
  // eigenvectors of F' = X^T F X by TC2 purification, then C = X Q with Q an orthonormal basis of
  // P V (V the previous step's occupied orbitals) from two Cholesky-QR passes.  D = C C^T and K
  // depend on C only through that projector, so the step is the eigenvector step's to rounding.
  // Returns 0, 1 when the caller should use the eigensolver (no convergence, a subspace too far
  // from the previous one), or a (negative) error code.
  int purified = 0;
  auto purify_occ = [&](const double* Fm) -> int {
    constexpr int kMaxSteps = 100;
    if (o.density_by_eigenvectors || nocc <= 0 || nocc >= nm) return 1;
    const int no = static_cast<int>(nocc);
    double sc[8];
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, nmi, ni, &one, Fm, ni, pX, ni, &zero, pT1, ni);    // F X
    cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, nmi, nmi, ni, &one, pX, ni, pT1, ni, &zero, pU, nmi);  // X^T F X
    double* P = pU;
    double* P2 = pT2;
    const long nb32 = (nm + 31) / 32, ntiles32 = nb32 * (nb32 + 1) / 2;
    k_col_abs_sum<<<static_cast<unsigned>((nm + 7) / 8), 256, 0, s>>>(P, nm, pW);
    k_max_small<<<1, 256, 0, s>>>(pW, nm, pPur, 0);
    k_purify_init<<<grid_of(nm * nm), 256, 0, s>>>(P, nm, pPur);
    int left = -1;  // steps still to take once the idempotency error is small
    bool done = false;
    // up to n' = 512 each step is one fused kernel, alternating between P and P2 (k_tc2_step).  Measured: the
    // fused steps won at n' = 144 and 384 (the SCF 24.5 -> 19.9 ms and 77 -> 72 ms), the library's DGEMM at
    // n' = 970 (1280 against 1289 ms), where the product, not the launches, sets a step's time.
    const bool fused = nm <= 512;
    const unsigned nb2 = static_cast<unsigned>((nm + T2 - 1) / T2);
    double* part = static_cast<double*>(dPart.p);
    const long pstride = 2L * nb2 * nb2;
    double* Pa = P;   // the current iterate of the fused steps
    double* Pb = P2;
    if (fused) k_tc2_norms<<<dim3(nb2, nb2), T2_THREADS, 0, s>>>(P, nm, part);
    for (int step = 1; step <= kMaxSteps && !done; ++step) {
      if (fused) {
        launch_tc2_step(Pa, Pb, nm, part + ((step - 1) & 1) * pstride, part + (step & 1) * pstride,
                        static_cast<double>(nocc), pPur, s);
        std::swap(Pa, Pb);
      } else {
        // P^2: its upper triangle is read.  DSYRK forms half the products; below n' = 1024 cuBLAS's DGEMM
        // was the faster of the two (21 against 25 ms of steps per SCF at n' = 384)
        if (nm >= 1024)
          cublasDsyrk(cb, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nmi, nmi, &one, P, nmi, &zero, P2, nmi);
        else
          cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, nmi, nmi, nmi, &one, P, nmi, P, nmi, &zero, P2, nmi);
        k_tc2_traces<<<1, 256, 0, s>>>(P, P2, nm, pPur);
        k_tc2_update_sym<<<static_cast<unsigned>(ntiles32), 256, 0, s>>>(P, P2, nm, pPur, static_cast<double>(nocc));
      }
      if (left > 0) {
        done = --left == 0;
      } else if (step >= 16 && step % 4 == 0) {
        // tr P - tr P^2 = sum lambda (1 - lambda) over P's eigenvalues, before this step
        cudaMemcpyAsync(sc, pPur, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (const cudaError_t e = cudaStreamSynchronize(s); e != cudaSuccess)
          return cuda_check(ctx, e, "rijk_scf purification");
        if (std::fabs(sc[1] - sc[2]) < 1e-8) left = 2;  // quadratic from here: two steps reach rounding
      }
    }
    if (fused && Pa != P) cudaMemcpyAsync(P, Pa, static_cast<size_t>(nm) * nm * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (!done) return 1;
    // W = P V, orthonormalised: W^T W = U^T U, W <- W U^-1, twice
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, nmi, no, nmi, &one, P, nmi, pV, nmi, &zero, pT1, nmi);
    for (int pass = 0; pass < 2; ++pass) {
      cublasDsyrk(cb, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, no, nmi, &one, pT1, nmi, &zero, P2, no);
      if (cusolverDnDpotrf(cs, CUBLAS_FILL_MODE_UPPER, no, P2, no, pWork, std::max(lworkp, 1), pInfo2 + pass) !=
          CUSOLVER_STATUS_SUCCESS)
        return 1;
      if (pass == 0) k_chol_ratio<<<1, 256, 0, s>>>(P2, no, pPur, 4);
      cublasDtrsm(cb, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nmi, no, &one, P2,
                  no, pT1, nmi);
    }
    int hinfo2[2] = {1, 1};
    cudaMemcpyAsync(sc, pPur, 5 * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hinfo2, pInfo2, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (const cudaError_t e = cudaStreamSynchronize(s); e != cudaSuccess)
      return cuda_check(ctx, e, "rijk_scf purification");
    // the last step's trace is n_c; the subspace step kept its rank (cond(P V) below 1e6)
    if (hinfo2[0] != 0 || hinfo2[1] != 0 || !(sc[4] > 1e-6) || !(std::fabs(sc[1] - nocc) < 1e-6)) return 1;
    cudaMemcpyAsync(pV, pT1, static_cast<size_t>(nm) * no * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, no, nmi, &one, pX, ni, pT1, nmi, &zero, pC, ni);  // C = X Q
    ++purified;
    return 0;
  };
  auto density = [&](double* Dm) {  // D = C_occ C_occ^T
    if (nocc > 0)
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, ni, ni, static_cast<int>(nocc), &one, pC, ni, pC, ni, &zero, Dm, ni);
    else
      cudaMemsetAsync(Dm, 0, b_nn, s);
  };

  if (o.guess_dm && o.guess_rows && o.guess_nrows > 0) {
    // start from the given density: one build with its factor rows, then diagonalise
    DeviceBuf& dR = wb[26];
    if ((rc = ensure(ctx, dR, static_cast<size_t>(o.guess_nrows) * n * sizeof(double), "scf guess rows"))) {
      cleanup();
      return rc;
    }
    cudaMemcpyAsync(pD, o.guess_dm, b_nn, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dR.p, o.guess_rows, static_cast<size_t>(o.guess_nrows) * n * sizeof(double),
                    cudaMemcpyHostToDevice, s);
    // The guess Fock matrix only seeds the first diagonalisation: a mixed run builds it in the
    // mixed form (the factor rows in orbital batches inside the build).
    rc = fock_device_impl(ctx, pD, static_cast<const double*>(dR.p), o.guess_nrows, pJ, pK, o.precision);
    if (!rc) rc = reduce_jk();
    if (!rc) {
      k_fock<<<grid_of(nn), 256, 0, s>>>(pH, pJ, pK, nn, pF);
      rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf guess");
    }
    if (rc) {
      cleanup();
      return rc;
    }
    if (diag(pF, soscf || hybrid) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the guess Fock matrix failed");
  } else {
    if (diag(pH, soscf || hybrid) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the core Hamiltonian failed");
  }
  density(pD);
  const auto t_loop0 = std::chrono::steady_clock::now();

  int prec = o.precision;
  int nmix = 0, nbuild = 0, m = 0, head = 0;
  double ms_fock = 0.0, E = 0.0, err = 1.0, rms = 1.0;
  double best_err = 1e300;
  int since_best = 0;
  result->history_len = 0;
  bool converged = false;
  std::vector<double> hout(8);
  int last_prec = -1;  // precision of the last build (pF, pJ, pK hold its result)
  auto build = [&](int p) -> int {
    int r = fock_device_impl(ctx, pD, pC, nocc, pJ, pK, p);
    if (!r) r = reduce_jk();
    if (r) return r;
    k_fock<<<grid_of(nn), 256, 0, s>>>(pH, pJ, pK, nn, pF);
    ++nbuild;
    if (p == RIJK_PREC_MIXED) ++nmix;
    last_prec = p;
    return RIJK_OK;
  };
  int it_used = 0;              // iterations taken by the DIIS phase of the hybrid converger
  bool run_soscf = soscf;       // the SOSCF loop runs (from the start, or after the DIIS phase)
  bool soscf_from_diis = false; // it starts from DIIS orbitals (all of them, eigenvectors of pFex)
  double t_build = 0.0, t_diis = 0.0, t_diag = 0.0;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto msec = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  if (!soscf) {
    bool have_fex = false;  // pFex holds the matrix whose eigenvectors gave pD
    std::vector<double> Bcache(32 * 32, 0.0);  // Pulay matrix entries by ring slot
    for (int it = 0; it < o.max_iter; ++it) {
      auto ta = now();
      if ((rc = build(prec))) {
        cleanup();
        return rc;
      }
      // energy and DIIS error X^T (F D S - S D F) X
      reduce(EnergyF{pD, pF, pH}, nn, 0, 0);
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, ni, ni, &one, pF, ni, pD, ni, &zero, pT1, ni);   // F D
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, ni, ni, &one, pT1, ni, pS, ni, &zero, pT2, ni);  // F D S
      k_antisym<<<grid_of(nn), 256, 0, s>>>(pT2, n, pT1);                                            // FDS - SDF
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, nmi, ni, &one, pT1, ni, pX, ni, &zero, pT2, ni);  // e X
      double* slotE = rE + static_cast<size_t>(head) * nn;
      double* slotF = rF + static_cast<size_t>(head) * nn;
      cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, nmi, nmi, ni, &one, pX, ni, pT2, ni, &zero, slotE, nmi);  // X^T e X
      cudaMemcpyAsync(slotF, pF, b_nn, cudaMemcpyDeviceToDevice, s);
      reduce(AbsF{slotE}, nm * nm, 1, 1);
      cudaEventRecord(ctx->ev3, s);
      cudaMemcpyAsync(hout.data(), pOut, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
      if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf iteration")) || (rc = check_device_error(ctx))) {
        cleanup();
        return rc;
      }
      ms_fock += elapsed(ctx->ev0, ctx->ev2);
      auto tb = now();
      t_build += msec(ta, tb);
      E = hout[0] + e_nuc;
      err = hout[1];
      if (result->history_len < 128) {
        result->history_energy[result->history_len] = E;
        result->history_diis_err[result->history_len] = err;
        result->history_mixed[result->history_len] = prec == RIJK_PREC_MIXED ? 1 : 0;
        ++result->history_len;
      }
      bool stalled = false;
      if (prec == RIJK_PREC_MIXED) {
        if (err < best_err * 0.9) {
          best_err = err;
          since_best = 0;
        } else {
          ++since_best;
        }
        // the split-BF16 rounding noise can put a floor under the DIIS error: stop waiting for it
        stalled = since_best >= 5 || nmix >= o.max_iter / 2;
      }
      if (prec == RIJK_PREC_MIXED && (err < o.switch_diis_err || stalled)) {
        prec = prec_fp64;
        if (hybrid) {
          // to the SOSCF loop, which rebuilds F in FP64 for this density.  It needs every
          // orbital: those of the extrapolated matrix this density came from (or, before the
          // first extrapolation, the full set of the start)
          if (have_fex) {
            auto tc = now();
            if (diag(pFex, true) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the Fock matrix failed");
            density(pD);
            t_diag += msec(tc, now());
          }
          soscf_from_diis = true;
          run_soscf = true;
          it_used = it;
          break;
        }
        // switch to the FP64 form: rebuild F for this same density and restart DIIS (unless the
        // caller keeps the mixed-phase vectors)
        if (!o.diis_keep_on_switch) {
          m = 0;
          head = 0;
        }
        --it;
        continue;
      }
      m = m < m_max ? m + 1 : m_max;
      head = (head + 1) % m_max;
      // Pulay B matrix over the stored error vectors.  Only the newest vector's row is new: the
      // other entries were formed when the later vector of each pair was stored, and are kept per
      // ring slot (each pair's dot product is formed once, by the same reduction).
      std::vector<double> Bm(static_cast<size_t>(m) * m);
      {
        int slots[32];
        for (int i = 0; i < m; ++i) slots[i] = (head - m + i + m_max) % m_max;
        const int knew = slots[m - 1];
        for (int i = 0; i < m; ++i)
          reduce(DotF{rE + static_cast<size_t>(knew) * nn, rE + static_cast<size_t>(slots[i]) * nn}, nm * nm, 0,
                 2 + i);
        std::vector<double> tmp(2 + m);
        cudaMemcpyAsync(tmp.data(), pOut, (2 + m) * sizeof(double), cudaMemcpyDeviceToHost, s);
        if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf DIIS"))) {
          cleanup();
          return rc;
        }
        for (int i = 0; i < m; ++i) Bcache[knew * 32 + slots[i]] = Bcache[slots[i] * 32 + knew] = tmp[2 + i];
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) Bm[i * m + j] = Bcache[slots[i] * 32 + slots[j]];
        std::vector<double> c;
        if (!diis_coefficients(Bm, m, c)) {
          c.assign(m, 0.0);
          c[m - 1] = 1.0;
        }
        for (int i = 0; i < m; ++i)
          k_axpy_set<<<grid_of(nn), 256, 0, s>>>(c[i], rF + static_cast<size_t>(slots[i]) * nn, nn, pFex, i == 0);
      }
      auto tc = now();
      t_diis += msec(tb, tc);
      const int pr = purify_occ(pFex);
      if (pr < 0) {  // the CUDA error is already recorded
        cleanup();
        return pr;
      }
      if (pr == 1 && diag(pFex) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the Fock matrix failed");
      have_fex = true;
      density(pDn);
      reduce(DiffSqF{pDn, pD}, nn, 0, 0);
      cudaMemcpyAsync(hout.data(), pOut, sizeof(double), cudaMemcpyDeviceToHost, s);
      if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf density"))) {
        cleanup();
        return rc;
      }
      rms = std::sqrt(hout[0] / static_cast<double>(nn));
      t_diag += msec(tc, now());
      std::swap(pD, pDn);
      if (rms < o.conv_dm_rms && prec != RIJK_PREC_MIXED) {  // FP64 results (RIJK_PREC_FP64 or _FP64_TC)
        converged = true;
        break;
      }
    }
  }
  if (run_soscf) {
    // the reference's RHF iteration (src/SCF.cpp:125-174) with its SOSCF engine
    const long nv = nm - nocc, dim = nocc * nv, dimc = std::max<long>(dim, 1);
    const int mvec = o.lbfgs_vectors > 0 ? o.lbfgs_vectors
                                         : static_cast<int>(std::min<long>(nm, std::min(20, o.max_iter)));
    const size_t nmm = static_cast<size_t>(nm) * nm;
    DeviceBuf &lb = wb[24], &qrw = wb[25];
    int lw_chol = 0;
    if ((rc = ensure(ctx, lb, ((2 * static_cast<size_t>(mvec) + 8) * dimc + 2 * nmm) * sizeof(double),
                     "scf L-BFGS"))) {
      cleanup();
      return rc;
    }
    double* g = static_cast<double*>(lb.p);  // gradient 4 F_ai, [i][a]
    double* hd = g + dimc;                    // diagonal Hessian 4 (F_aa - F_ii)
    double* q = hd + dimc;                    // two-loop work vector
    double* sv = q + dimc;                    // the step before scaling
    double* xs = sv + dimc;                   // the step applied
    double* gprev = xs + dimc;
    double* ysc = gprev + dimc;               // g - gprev
    double* Yv = ysc + dimc;                  // mvec gradient differences
    double* Sv = Yv + mvec * dimc;            // mvec steps, slot mvec = the last step taken
    double* Fmo = Sv + (mvec + 1) * dimc;     // C^T F C, then the Gram matrix of the rotation
    double* Rq = Fmo + nmm;                   // rotation, then its orthonormal columns
    cudaMemsetAsync(lb.p, 0, lb.bytes, s);
    if (cusolverDnDpotrf_bufferSize(cs, CUBLAS_FILL_MODE_UPPER, nmi, Fmo, nmi, &lw_chol) != CUSOLVER_STATUS_SUCCESS) {
      return fail(RIJK_ERR_SOLVER, "Cholesky buffer query failed");
    }
    const int lwq = std::max(lw_chol, 1);
    if ((rc = ensure(ctx, qrw, static_cast<size_t>(lwq) * sizeof(double), "scf QR work"))) {
      cleanup();
      return rc;
    }
    double* pQw = static_cast<double*>(qrw.p);
    const unsigned gd = grid_of(dim);
    // no first-iteration diagonalisation after a start from a Fock matrix's own orbitals
    const bool guess_diag = soscf_from_diis || (o.guess_dm && o.guess_rows && o.guess_nrows > 0);
    const double eps = std::numeric_limits<double>::epsilon();
    std::vector<double> rho(mvec, 0.0);
    double E_old = 1e15;
    int step_num = 0, pair_num = 0;
    bool have_rms = false;
    for (int it = 0; it < o.max_iter - it_used; ++it) {
      auto ta = now();
      if ((rc = build(prec))) {
        cleanup();
        return rc;
      }
      reduce(EnergyF{pD, pF, pH}, nn, 0, 0);
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, nmi, ni, &one, pF, ni, pC, ni, &zero, pT1, ni);     // F C
      cublasDgemm(cb, CUBLAS_OP_T, CUBLAS_OP_N, nmi, nmi, ni, &one, pC, ni, pT1, ni, &zero, Fmo, nmi);  // C^T F C
      k_soscf_grad<<<gd, 256, 0, s>>>(Fmo, nm, nocc, g, hd);
      reduce(AbsF{g}, dim, 1, 1);
      if (step_num > 0) {  // curvature pair candidate (src/l-bfgs_2_1.cpp:44-61)
        k_sub<<<gd, 256, 0, s>>>(g, gprev, dim, ysc);
        reduce(DotF{Sv + mvec * dimc, ysc}, dim, 0, 2);
        reduce(DotF{ysc, ysc}, dim, 0, 3);
      }
      cudaMemcpyAsync(hout.data(), pOut, 6 * sizeof(double), cudaMemcpyDeviceToHost, s);
      if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf iteration")) || (rc = check_device_error(ctx))) {
        cleanup();
        return rc;
      }
      ms_fock += elapsed(ctx->ev0, ctx->ev2);
      auto tb = now();
      t_build += msec(ta, tb);
      E = hout[0] + e_nuc;
      err = hout[1];
      if (have_rms) rms = std::sqrt(hout[5] / static_cast<double>(nn));
      if (result->history_len < 128) {
        result->history_energy[result->history_len] = E;
        result->history_diis_err[result->history_len] = err;
        result->history_mixed[result->history_len] = prec == RIJK_PREC_MIXED ? 1 : 0;
        ++result->history_len;
      }
      if (prec == RIJK_PREC_MIXED) {
        if (err < best_err * 0.9) {
          best_err = err;
          since_best = 0;
        } else {
          ++since_best;
        }
        if (err < o.switch_diis_err || since_best >= 5 || nmix >= o.max_iter / 2) {
          // to the FP64 form: rebuild F for the same orbitals, restart the L-BFGS history
          prec = prec_fp64;
          step_num = 0;
          E_old = 1e15;
          --it;
          continue;
        }
      } else if (err < o.conv_grad || std::fabs(E - E_old) < o.conv_energy) {  // src/SCF.cpp:145-156
        converged = true;
        break;
      }
      auto tc = now();
      if (it == 0 && !guess_diag) {  // first iteration: plain diagonalisation (src/SCF.cpp:160-166)
        if (diag(pF, true) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the Fock matrix failed");
        density(pDn);
        reduce(DiffSqF{pDn, pD}, nn, 0, 5);
        std::swap(pD, pDn);
        have_rms = true;
        E_old = E;
        t_diag += msec(tc, now());
        continue;
      }
      // L-BFGS two-loop step with the diagonal Hessian (src/l-bfgs_2_1.cpp:30-126)
      if (step_num == 0) pair_num = 0;
      if (step_num > 0) {
        const double sy = hout[2], yy = hout[3];
        if (sy > eps * yy) {
          const int slot = pair_num % mvec;
          cudaMemcpyAsync(Yv + slot * dimc, ysc, dim * sizeof(double), cudaMemcpyDeviceToDevice, s);
          cudaMemcpyAsync(Sv + slot * dimc, Sv + mvec * dimc, dim * sizeof(double), cudaMemcpyDeviceToDevice, s);
          rho[slot] = 1.0 / sy;
          ++pair_num;
        }
      }
      const int vec_num = std::min(pair_num, mvec);
      cudaMemcpyAsync(q, g, dim * sizeof(double), cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(gprev, g, dim * sizeof(double), cudaMemcpyDeviceToDevice, s);
      for (int i = 0; i < vec_num; ++i) {  // alpha_i = rho s_k . q ; q -= alpha_i y_k (newest first)
        const int k = (pair_num - i - 1) % mvec;
        reduce(DotF{Sv + k * dimc, q}, dim, 0, 10 + i);
        k_axpy_dev<<<gd, 256, 0, s>>>(q, Yv + k * dimc, dim, pOut, 10 + i, -rho[k], -1, 0.0);
      }
      k_div<<<gd, 256, 0, s>>>(q, hd, dim, sv);
      for (int i = 0; i < vec_num; ++i) {  // beta = rho y_k . s ; s += (alpha - beta) s_k (oldest first)
        const int k = (pair_num - vec_num + i) % mvec;
        reduce(DotF{Yv + k * dimc, sv}, dim, 0, 50 + i);
        k_axpy_dev<<<gd, 256, 0, s>>>(sv, Sv + k * dimc, dim, pOut, 10 + (vec_num - i - 1), rho[k], 50 + i, -rho[k]);
      }
      reduce(AbsF{sv}, dim, 1, 4);
      k_zoom<<<gd, 256, 0, s>>>(sv, dim, pOut, 4, 6, 0.1, xs, Sv + mvec * dimc);  // x_max_soscf = 0.1
      ++step_num;
      auto td = now();
      t_diis += msec(tc, td);
      // orbitals <- (orthonormalised I + X - X^T) orbitals (src/converger_2_1.cpp:105-123).  The
      // reference orthonormalises the columns in order (Gram-Schmidt): A = Q R with R's diagonal
      // positive, a unique factorisation.  Here Q comes from two Cholesky-QR passes, A^T A = U^T U and
      // A <- A U^-1: A = I + X - X^T has singular values in [1, sqrt(1 + |X|^2)], so A^T A is well
      // conditioned, and the second pass brings Q^T Q to I within rounding.
      k_rot_build<<<grid_of(nm * nm), 256, 0, s>>>(xs, nm, nocc, Rq);
      for (int pass = 0; pass < 2; ++pass) {
        cublasDsyrk(cb, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nmi, nmi, &one, Rq, nmi, &zero, Fmo, nmi);  // A^T A
        if (cusolverDnDpotrf(cs, CUBLAS_FILL_MODE_UPPER, nmi, Fmo, nmi, pQw, lwq, pInfo) != CUSOLVER_STATUS_SUCCESS)
          return fail(RIJK_ERR_SOLVER, "Cholesky factorisation of the rotation's Gram matrix failed");
        cublasDtrsm(cb, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nmi, nmi, &one,
                    Fmo, nmi, Rq, nmi);  // A U^-1
      }
      cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_N, ni, nmi, nmi, &one, pC, ni, Rq, nmi, &zero, pT1, ni);  // C Q
      cudaMemcpyAsync(pC, pT1, static_cast<size_t>(n) * nm * sizeof(double), cudaMemcpyDeviceToDevice, s);
      density(pDn);
      reduce(DiffSqF{pDn, pD}, nn, 0, 5);
      std::swap(pD, pDn);
      have_rms = true;
      E_old = E;
      t_diag += msec(td, now());
    }
  }
  const auto t_loop1 = std::chrono::steady_clock::now();
  // The energy is the last FP64 build's, as the reference reports it (src/SCF.cpp:134-156): a run
  // that ended in the mixed phase gets one FP64 build at its density for it.
  if (last_prec == RIJK_PREC_MIXED || last_prec < 0) {
    if ((rc = build(prec_fp64))) {
      cleanup();
      return rc;
    }
    reduce(EnergyF{pD, pF, pH}, nn, 0, 0);
    cudaMemcpyAsync(hout.data(), pOut, sizeof(double), cudaMemcpyDeviceToHost, s);
    if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf final")) || (rc = check_device_error(ctx))) {
      cleanup();
      return rc;
    }
    ms_fock += elapsed(ctx->ev0, ctx->ev2);
    E = hout[0] + e_nuc;
  }
  if (MO) {
    // every orbital of the last Fock matrix, as the reference's closing diagonalisation
    // (src/SCF.cpp:178)
    if (diag(pF, true) != RIJK_OK) return fail(RIJK_ERR_SOLVER, "syevd of the final Fock matrix failed");
    cudaMemcpyAsync(MO, pC, static_cast<size_t>(nm) * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if ((rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_scf orbitals"))) {
      cleanup();
      return rc;
    }
  }
  if (MO && nm < n) std::memset(MO + nm * n, 0, static_cast<size_t>(n - nm) * n * sizeof(double));
  result->energy = E;
  result->dm_rms = rms;
  result->diis_err = err;
  result->iterations = nbuild;
  result->iterations_mixed = nmix;
  result->converged = converged ? 1 : 0;
  result->nmo = static_cast<int>(nm);
  result->ms_fock = ms_fock;
  result->ms_build_phase = t_build;
  result->ms_diis_phase = t_diis;
  result->ms_diag_phase = t_diag;
  const auto t_end = std::chrono::steady_clock::now();
  result->ms_total = std::chrono::duration<double, std::milli>(t_end - t_start).count();
  result->ms_setup_phase = std::chrono::duration<double, std::milli>(t_loop0 - t_start).count();
  result->ms_final_phase = std::chrono::duration<double, std::milli>(t_end - t_loop1).count();
  result->purified = purified;
  cleanup();
  {
    char buf[384];
    std::snprintf(buf, sizeof(buf),
                  "{\"call\": \"rijk_scf\", \"device\": %d, \"n\": %ld, \"naux\": %ld, \"n_c\": %ld, "
                  "\"energy\": %.12f, \"iterations\": %d, \"iterations_mixed\": %d, \"converged\": %d, "
                  "\"ms_total\": %.6g, \"ms_fock\": %.6g}",
                  ctx->device, n, ctx->naux, nocc, E, nbuild, nmix, converged ? 1 : 0, result->ms_total, ms_fock);
    log_line(buf);
  }
  if (!converged) return set_err(ctx, RIJK_ERR_CONVERGE, "rijk_scf: not converged in %d iterations", o.max_iter);
  return RIJK_OK;
}
