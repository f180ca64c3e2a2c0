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

// out[mu][nu] = sum_s partial[s][tile(max,min)][r][c] with (r, c) oriented to the stored tile.
__global__ void k_unpack_sym(const double* __restrict__ partial, int nsplit, long ntile, long n,
                             double* __restrict__ out) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long total = n * n;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long mu = idx / n, nu = idx % n;
    long I = mu / TILE, J = nu / TILE;
    long r = mu % TILE, c = nu % TILE;
    if (I < J) {
      long tmp = I; I = J; J = tmp;
      tmp = r; r = c; c = tmp;
    }
    const double* p = partial + tri_index(I, J) * TILE2 + r * TILE + c;
    double v = 0.0;
    for (int s = 0; s < nsplit; ++s) v += p[static_cast<long>(s) * ntile * TILE2];
    out[idx] = v;
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

void launch_unpack_sym(const double* partial, int nsplit, long ntile, long n, double* out, cudaStream_t s) {
  k_unpack_sym<<<grid_for(n * n, 256), 256, 0, s>>>(partial, nsplit, ntile, n, out);
}

void launch_scan_nonfinite(const double* x, long count, int* err, cudaStream_t s) {
  k_scan_nonfinite<<<grid_for(count, 256), 256, 0, s>>>(x, count, err);
}

}  // namespace rijk
