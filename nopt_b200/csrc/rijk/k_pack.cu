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

// Two steps: (1) sum the split partials into the first split's slot (each element read and
// written by one thread, coalesced); (2) one CTA per 32 x 32 block of the full square copies
// the stored tile block, transposing it through shared memory for the upper triangle.
__global__ void k_sum_splits(double* __restrict__ partial, int nsplit, long ntile) {
  const long total = ntile * TILE2;
  const long sstride = total;
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    double v = partial[idx];
    for (int s = 1; s < nsplit; ++s) v += partial[static_cast<long>(s) * sstride + idx];
    partial[idx] = v;
  }
}

// sum[idx] = sum_s partial[s][idx] for fp32 partials (the tcgen05 accumulators, exact in fp32),
// summed in fp64; four consecutive elements per thread, four splits in flight.
__global__ void k_sum_splits_f32(const float* __restrict__ partial, int nsplit, long ntile, double* __restrict__ sum) {
  const long total4 = ntile * TILE2 / 4;
  const float4* p4 = reinterpret_cast<const float4*>(partial);
  for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total4;
       i += static_cast<long>(gridDim.x) * blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int sp = 0;
    for (; sp + 4 <= nsplit; sp += 4) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = p4[static_cast<long>(sp + u) * total4 + i];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a0 += v[u].x;
        a1 += v[u].y;
        a2 += v[u].z;
        a3 += v[u].w;
      }
    }
    for (; sp < nsplit; ++sp) {
      const float4 v = p4[static_cast<long>(sp) * total4 + i];
      a0 += v.x;
      a1 += v.y;
      a2 += v.z;
      a3 += v.w;
    }
    reinterpret_cast<double4*>(sum)[i] = make_double4(a0, a1, a2, a3);
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

void launch_pack_mo(const double* MO, long nocc, long n, long noccp, long npad, double* MOp, cudaStream_t s) {
  k_pack_mo<<<grid_for(noccp * npad, 256), 256, 0, s>>>(MO, nocc, n, noccp, npad, MOp);
}

// Sums the split partials in place (into split 0) and writes the full symmetric n x n matrix.
void launch_unpack_sym(double* partial, int nsplit, long ntile, long n, double* out, cudaStream_t s) {
  double* p = partial;
  if (nsplit > 1) k_sum_splits<<<grid_for(ntile * TILE2, 256), 256, 0, s>>>(p, nsplit, ntile);
  const long nb = (n + 31) / 32;
  k_unpack_blocks<<<static_cast<unsigned>(nb * nb), 256, 0, s>>>(p, n, nb, out);
}

// fp32 split partials -> their fp64 sum (into `sum`, ntile tiles) -> the full symmetric n x n matrix.
void launch_unpack_sym_f32(const float* partial, int nsplit, long ntile, long n, double* sum, double* out,
                           cudaStream_t s) {
  k_sum_splits_f32<<<grid_for(ntile * TILE2 / 4, 256), 256, 0, s>>>(partial, nsplit, ntile, sum);
  const long nb = (n + 31) / 32;
  k_unpack_blocks<<<static_cast<unsigned>(nb * nb), 256, 0, s>>>(sum, n, nb, out);
}

void launch_scan_nonfinite(const double* x, long count, int* err, cudaStream_t s) {
  k_scan_nonfinite<<<grid_for(count, 256), 256, 0, s>>>(x, count, err);
}

}  // namespace rijk
