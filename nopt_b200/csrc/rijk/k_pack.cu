// k_pack.cu — layout conversions around the Fock build.
//
//  pack_density   D (n x n, as given)  ->  Dt, the packed weights of the Coulomb contraction:
//                 w_Q = sum_{mu,nu} D_{mu nu} (Q|mu nu) over the full square, as
//                 DM_to_F_transform_RI does (src/RI.cpp:122-126), equals the sum over the
//                 stored lower tiles with off-diagonal tiles weighted by D_{mu nu} + D_{nu mu}.
//  pack_mo        MO rows 0..n_c-1 (n_c x n)  ->  zero-padded noccp x npad
//  unpack_sym     sum of split partials over the packed tiles  ->  full symmetric n x n
#include "dmma.cuh"
#include "rijk_internal.h"

namespace rijk {

__global__ void k_pack_density(const double* __restrict__ D, long n, long npad, double* __restrict__ Dt) {
  long t = blockIdx.x;
  long I, J;
  tri_decode(t, I, J);
  double* out = Dt + t * TILE2;
  for (int e = threadIdx.x; e < TILE2; e += blockDim.x) {
    int r = e / TILE, c = e % TILE;
    long mu = I * TILE + r, nu = J * TILE + c;
    double v = 0.0;
    if (mu < n && nu < n) {
      v = D[mu * n + nu];
      if (I != J) v += D[nu * n + mu];
    }
    out[e] = v;
  }
}

__global__ void k_pack_mo(const double* __restrict__ MO, long nocc, long n, long noccp, long npad,
                          double* __restrict__ MOp) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long total = noccp * npad;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long i = idx / npad, mu = idx % npad;
    MOp[idx] = (i < nocc && mu < n) ? MO[i * n + mu] : 0.0;
  }
}

// Two steps: (1) sum the split partials (fp64, or the fp32 tcgen05 accumulators) into an fp64
// packed buffer; (2) one CTA per 32 x 32 block of the full square copies the stored tile block,
// transposing it through shared memory for the upper triangle.
//
// Step 1: a CTA owns 128 consecutive elements (32 lanes x 4); its 8 warps take every 8th split
// each, four splits in flight, and the 8 warp sums are added in shared memory in warp order, so
// the result does not depend on timing.  With out == partial (fp64) the sum overwrites split 0
// after every warp has read it.
template <typename T>
__global__ void __launch_bounds__(256) k_sum_splits(const T* partial, int nsplit, long total, double* out) {
  __shared__ double red[8][32][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long e = (static_cast<long>(blockIdx.x) * 32 + lane) * 4;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  if (e < total) {
    int sp = warp;
    for (; sp + 24 < nsplit; sp += 32) {
      T v[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int k = 0; k < 4; ++k) v[u][k] = partial[static_cast<long>(sp + 8 * u) * total + e + k];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int k = 0; k < 4; ++k) a[k] += static_cast<double>(v[u][k]);
    }
    for (; sp < nsplit; sp += 8)
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] += static_cast<double>(partial[static_cast<long>(sp) * total + e + k]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) red[warp][lane][k] = a[k];
  __syncthreads();
  if (warp == 0 && e < total) {
    double r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      r[k] = red[0][lane][k];
      for (int w = 1; w < 8; ++w) r[k] += red[w][lane][k];
    }
    *reinterpret_cast<double4*>(out + e) = make_double4(r[0], r[1], r[2], r[3]);
  }
}

__global__ void __launch_bounds__(256) k_unpack_blocks(const double* __restrict__ packed, long n, long nb,
                                                      double* __restrict__ out) {
  __shared__ double blk[32][33];
  const long bi = blockIdx.x / nb, bj = blockIdx.x % nb;  // 32-blocks of the output
  const long I = bi / 2, J = bj / 2;                       // 64-tiles
  const bool lower = I >= J;
  // stored tile (max, min); sub-block of it that holds this output block
  const long a = lower ? I : J, b = lower ? J : I;
  const long rs = lower ? (bi & 1) * 32 : (bj & 1) * 32;  // row offset inside the stored tile
  const long cs = lower ? (bj & 1) * 32 : (bi & 1) * 32;
  const double* src = packed + tri_index(a, b) * TILE2;
  for (int e = threadIdx.x; e < 1024; e += 256) {
    const int r = e / 32, c = e % 32;
    blk[r][c] = src[(rs + r) * TILE + cs + c];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 1024; e += 256) {
    const int r = e / 32, c = e % 32;
    const long mu = bi * 32 + r, nu = bj * 32 + c;
    if (mu < n && nu < n) out[mu * n + nu] = lower ? blk[r][c] : blk[c][r];
  }
}

__global__ void k_scan_nonfinite(const double* __restrict__ x, long count, int* err) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool bad = false;
  for (; idx < count; idx += static_cast<long>(gridDim.x) * blockDim.x) bad |= !isfinite(x[idx]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, DEVERR_NAN);
}

static int grid_for(long total, int threads) {
  long b = (total + threads - 1) / threads;
  if (b > 148L * 16) b = 148L * 16;
  if (b < 1) b = 1;
  return static_cast<int>(b);
}

void launch_pack_density(const double* D, long n, long npad, long nt, double* Dt, cudaStream_t s) {
  long ntile = nt * (nt + 1) / 2;
  k_pack_density<<<static_cast<unsigned>(ntile), 256, 0, s>>>(D, n, npad, Dt);
}

cudaError_t preload_density_kernels() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_pack_density);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_sum_splits<double>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_unpack_blocks);
  return e;
}

// Ends after `cycles` SM clock cycles, whatever happens elsewhere: it waits on nothing.
__global__ void k_delay(long long cycles) {
  const long long t0 = clock64();
  while (clock64() - t0 < cycles) __nanosleep(500);
}

void launch_delay(long long cycles, cudaStream_t s) { k_delay<<<1, 32, 0, s>>>(cycles); }

void launch_pack_mo(const double* MO, long nocc, long n, long noccp, long npad, double* MOp, cudaStream_t s) {
  k_pack_mo<<<grid_for(noccp * npad, 256), 256, 0, s>>>(MO, nocc, n, noccp, npad, MOp);
}

// Sums the split partials in place (into split 0) and writes the full symmetric n x n matrix.
void launch_unpack_sym(double* partial, int nsplit, long ntile, long n, double* out, cudaStream_t s) {
  double* p = partial;
  const long total = ntile * TILE2;
  if (nsplit > 1) k_sum_splits<double><<<static_cast<unsigned>((total + 127) / 128), 256, 0, s>>>(p, nsplit, total, p);
  const long nb = (n + 31) / 32;
  k_unpack_blocks<<<static_cast<unsigned>(nb * nb), 256, 0, s>>>(p, n, nb, out);
}

// fp32 split partials -> their fp64 sum (into `sum`, ntile tiles) -> the full symmetric n x n matrix.
void launch_unpack_sym_f32(const float* partial, int nsplit, long ntile, long n, double* sum, double* out,
                           cudaStream_t s) {
  const long total = ntile * TILE2;
  k_sum_splits<float><<<static_cast<unsigned>((total + 127) / 128), 256, 0, s>>>(partial, nsplit, total, sum);
  const long nb = (n + 31) / 32;
  k_unpack_blocks<<<static_cast<unsigned>(nb * nb), 256, 0, s>>>(sum, n, nb, out);
}

void launch_scan_nonfinite(const double* x, long count, int* err, cudaStream_t s) {
  k_scan_nonfinite<<<grid_for(count, 256), 256, 0, s>>>(x, count, err);
}

}  // namespace rijk
