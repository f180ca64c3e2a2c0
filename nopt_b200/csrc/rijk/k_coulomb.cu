// k_coulomb.cu — the Coulomb pair of the RI Fock build, two bandwidth-bound passes over B.
//
// Reference (src/RI.cpp:122-144): RI_J = vec(D)^T RI_AA, then V^-1/2 twice, then
// J = RI_AA RI_J.  With the metric folded into B (B = M (P|mu nu), M^T M = V^-1) this is
//   w_Q  = sum_e B[Q][e] Dt[e]          (pass 1, one CTA per QB aux functions)
//   J[e] = sum_Q B[Q][e] w_Q            (pass 2, Q split into nsplit ranges, partials
//                                        summed while unpacking)
// Both passes stream B once with 128-bit loads that bypass L1; reductions are warp
// shuffles.  Algorithmic traffic: 2 * |B| bytes per build.  Both stride over their work, so a
// capped grid (one or two CTAs per SM, beside the half-transform) covers all of it.
#include <algorithm>

#include <cuda_bf16.h>

#include "dmma.cuh"
#include "rijk_internal.h"

namespace rijk {

constexpr int W_QB = 4;        // aux functions per CTA in pass 1 (reuses each Dt load)
constexpr int W_THREADS = 256;  // at most 16K registers a CTA: two fit beside two half-transform CTAs

// SIDE: the instantiation run beside the half-transform (its own shared-memory carveout); the same code
template <bool SIDE>
__global__ void __launch_bounds__(W_THREADS) k_coulomb_w(const double* __restrict__ B, const double* __restrict__ Dt,
                                                          long naux, long tile_elems, double* __restrict__ w) {
  const long n2 = tile_elems / 2;
  const double2* D2 = reinterpret_cast<const double2*>(Dt);
  __shared__ double red[W_QB][W_THREADS / 32];
  for (long q0 = static_cast<long>(blockIdx.x) * W_QB; q0 < naux; q0 += static_cast<long>(gridDim.x) * W_QB) {
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
    __syncthreads();  // red is refilled by the next group of aux functions
  }
}

constexpr int J_THREADS = 256;
constexpr int J_UNROLL = 4;

// Jpart[s][e] = sum_{Q in split s} B[Q][e] w[Q]; each thread owns one double2 of e.
template <bool SIDE>
__global__ void __launch_bounds__(J_THREADS) k_coulomb_j(const double* __restrict__ B, const double* __restrict__ w,
                                                          long naux, long tile_elems, long qper,
                                                          double* __restrict__ Jpart) {
  const long s = blockIdx.y;
  const long qa = s * qper;
  const long qb = qa + qper < naux ? qa + qper : naux;
  const long stride2 = tile_elems / 2;
  for (long e2 = static_cast<long>(blockIdx.x) * J_THREADS + threadIdx.x; e2 < stride2;
       e2 += static_cast<long>(gridDim.x) * J_THREADS) {
    const double2* Bp = reinterpret_cast<const double2*>(B) + e2;
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
}

int coulomb_nsplit(long tile_elems, long naux, int elems_per_thread) {
  long blocks = (tile_elems / elems_per_thread + J_THREADS - 1) / J_THREADS;
  long want = (148L * 8 + blocks - 1) / blocks;  // about 8 CTAs per SM in flight
  if (want < 1) want = 1;
  if (want > 32) want = 32;
  if (want > naux) want = naux;
  return static_cast<int>(want);
}

// The capped forms ask for the largest shared-memory carveout, the one the half-transform runs with, so that
// their CTAs can share its SMs.  The forms run alone keep the default (their L1 caches w and Dt).
static void prefer_shared_carveout() {
  prefer_max_shared(reinterpret_cast<const void*>(k_coulomb_w<true>));
  prefer_max_shared(reinterpret_cast<const void*>(k_coulomb_j<true>));
}

void launch_coulomb_w(const double* B, const double* Dt, long naux, long tile_elems, double* w, cudaStream_t s,
                      int max_ctas) {
  long grid = (naux + W_QB - 1) / W_QB;
  if (max_ctas > 0) {
    prefer_shared_carveout();
    if (grid > max_ctas) grid = max_ctas;
    k_coulomb_w<true><<<static_cast<unsigned>(grid), W_THREADS, 0, s>>>(B, Dt, naux, tile_elems, w);
    return;
  }
  k_coulomb_w<false><<<static_cast<unsigned>(grid), W_THREADS, 0, s>>>(B, Dt, naux, tile_elems, w);
}

cudaError_t preload_coulomb_kernels() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_coulomb_w<false>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_coulomb_j<false>);
  return e;
}

void launch_coulomb_j(const double* B, const double* w, long naux, long tile_elems, int nsplit, double* Jpart,
                      cudaStream_t s, int max_ctas) {
  if (max_ctas > 0) prefer_shared_carveout();
  long qper = (naux + nsplit - 1) / nsplit;
  long gx = (tile_elems / 2 + J_THREADS - 1) / J_THREADS;
  if (max_ctas > 0 && gx * nsplit > max_ctas) gx = std::max<long>(1, max_ctas / nsplit);
  dim3 grid(static_cast<unsigned>(gx), static_cast<unsigned>(nsplit));
  if (max_ctas > 0)
    k_coulomb_j<true><<<grid, J_THREADS, 0, s>>>(B, w, naux, tile_elems, qper, Jpart);
  else
    k_coulomb_j<false><<<grid, J_THREADS, 0, s>>>(B, w, naux, tile_elems, qper, Jpart);
}

// ---------------------------------------------------------------------------------
// The same two passes over the split-BF16 copy of B (mixed form): Bmix[Q][t][hl][64][64],
// hi and lo planes of a tile 4096 elements apart, tiles t < ntile (the padded tile row of an
// odd tile count is never read).  Each thread takes 8 consecutive elements (16-byte loads of
// each plane), forms b = hi + lo in fp32 (exact: the planes are 8 bits apart) and
// accumulates in fp64.  Half the bytes of the FP64 passes; B is represented to ~2^-17.

__device__ __forceinline__ void bf16x8_sum(const uint4 h, const uint4 l, float (&b)[8]) {
  const __nv_bfloat162* hp = reinterpret_cast<const __nv_bfloat162*>(&h);
  const __nv_bfloat162* lp = reinterpret_cast<const __nv_bfloat162*>(&l);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float2 a = __bfloat1622float2(hp[k]);
    float2 c = __bfloat1622float2(lp[k]);
    b[2 * k] = a.x + c.x;
    b[2 * k + 1] = a.y + c.y;
  }
}

__device__ __forceinline__ uint4 ldg_stream_u4(const void* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Element offset of packed element e (tile t = e / 4096) inside one aux function's Bmix block.
__device__ __forceinline__ long mix_off(long e) { return (e >> 12) * 8192 + (e & 4095); }

constexpr int WM_THREADS = 256;  // 8 warps; each warp reduces one aux function over the chunk at a time
constexpr int WM_OCT = 1024;     // octets (8 elements) per chunk: two tiles, 32 KB of fp32 Dt in shared memory
constexpr int WM_QR = 32;        // aux functions per CTA

int coulomb_w_mixed_chunks(long ntile) { return static_cast<int>((ntile * TILE2 / 8 + WM_OCT - 1) / WM_OCT); }

// wpart[c][q] = sum over octet chunk c (blockIdx.x) of Bmix[q][e] Dt[e], q in the WM_QR aux functions
// of blockIdx.y.  The chunk's Dt is staged once as fp32 in two planes (elements 0-3 and 4-7 of each
// octet), so a warp's 16-byte reads of it are conflict-free; each warp then streams one aux
// function's hi/lo planes over the chunk with four octets per lane in flight and reduces by shuffle.
__global__ void __launch_bounds__(WM_THREADS) k_coulomb_w_mixed(const __nv_bfloat16* __restrict__ Bmix,
                                                                 const double* __restrict__ Dt, long naux, long ntile,
                                                                 long ntile2, double* __restrict__ wpart) {
  __shared__ __align__(16) float sd[2][WM_OCT * 4];
  const long n8 = ntile * TILE2 / 8;
  const long c0 = static_cast<long>(blockIdx.x) * WM_OCT;
  const int cnt = static_cast<int>(n8 - c0 < WM_OCT ? n8 - c0 : WM_OCT);
  const double4* D4 = reinterpret_cast<const double4*>(Dt + c0 * 8);
  for (int i = threadIdx.x; i < 2 * cnt; i += WM_THREADS) {  // i = 2 * octet + half
    const double4 d = D4[i];
    reinterpret_cast<float4*>(sd[i & 1])[i >> 1] =
        make_float4(static_cast<float>(d.x), static_cast<float>(d.y), static_cast<float>(d.z), static_cast<float>(d.w));
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long qstride = ntile2 * 2 * TILE2;
  const long qa = static_cast<long>(blockIdx.y) * WM_QR;
  const float4* s0 = reinterpret_cast<const float4*>(sd[0]);
  const float4* s1 = reinterpret_cast<const float4*>(sd[1]);
  for (int j = warp; j < WM_QR; j += WM_THREADS / 32) {
    const long q = qa + j;
    if (q >= naux) break;
    const __nv_bfloat16* qb = Bmix + q * qstride;
    double acc = 0.0;  // each octet's 8 products are summed in fp32, the octets in fp64
    auto dot = [&](const uint4 h, const uint4 l, int o) {
      float b[8];
      bf16x8_sum(h, l, b);
      const float4 d0 = s0[o], d1 = s1[o];
      float t = b[0] * d0.x;
      t = fmaf(b[1], d0.y, t);
      t = fmaf(b[2], d0.z, t);
      t = fmaf(b[3], d0.w, t);
      t = fmaf(b[4], d1.x, t);
      t = fmaf(b[5], d1.y, t);
      t = fmaf(b[6], d1.z, t);
      t = fmaf(b[7], d1.w, t);
      acc += static_cast<double>(t);
    };
    int o = lane;
    for (; o + 96 < cnt; o += 128) {
      uint4 h[4], l[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const long off = mix_off((c0 + o + 32 * u) * 8);
        h[u] = ldg_stream_u4(qb + off);
        l[u] = ldg_stream_u4(qb + off + TILE2);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) dot(h[u], l[u], o + 32 * u);
    }
    for (; o < cnt; o += 32) {
      const long off = mix_off((c0 + o) * 8);
      dot(ldg_stream_u4(qb + off), ldg_stream_u4(qb + off + TILE2), o);
    }
    acc = warp_sum(acc);
    if (lane == 0) wpart[blockIdx.x * naux + q] = acc;
  }
}

// w[q] = sum_c wpart[c][q], in chunk order (deterministic)
__global__ void k_sum_chunks(const double* __restrict__ wpart, int nchunk, long naux, double* __restrict__ w) {
  for (long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; q < naux;
       q += static_cast<long>(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int c = 0; c < nchunk; ++c) v += wpart[c * naux + q];
    w[q] = v;
  }
}

__global__ void __launch_bounds__(J_THREADS) k_coulomb_j_mixed(const __nv_bfloat16* __restrict__ Bmix,
                                                                const double* __restrict__ w, long naux, long ntile,
                                                                long ntile2, long qper, double* __restrict__ Jpart) {
  const long e8 = static_cast<long>(blockIdx.x) * J_THREADS + threadIdx.x;
  const long s = blockIdx.y;
  const long tile_elems = ntile * TILE2;
  if (e8 * 8 >= tile_elems) return;
  const long qa = s * qper;
  const long qb = qa + qper < naux ? qa + qper : naux;
  const long qstride = ntile2 * 2 * TILE2;
  const __nv_bfloat16* base = Bmix + mix_off(e8 * 8);
  double acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc[k] = 0.0;
  long q = qa;
  for (; q + 4 <= qb; q += 4) {
    uint4 h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const __nv_bfloat16* p = base + (q + u) * qstride;
      h[u] = ldg_stream_u4(p);
      l[u] = ldg_stream_u4(p + TILE2);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float b[8];
      bf16x8_sum(h[u], l[u], b);
      const double wq = __ldg(w + q + u);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] = fma(static_cast<double>(b[k]), wq, acc[k]);
    }
  }
  for (; q < qb; ++q) {
    const __nv_bfloat16* p0 = base + q * qstride;
    float b0[8];
    bf16x8_sum(ldg_stream_u4(p0), ldg_stream_u4(p0 + TILE2), b0);
    const double w0 = __ldg(w + q);
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = fma(static_cast<double>(b0[k]), w0, acc[k]);
  }
  double* out = Jpart + s * tile_elems + e8 * 8;
  *reinterpret_cast<double4*>(out) = make_double4(acc[0], acc[1], acc[2], acc[3]);
  *reinterpret_cast<double4*>(out + 4) = make_double4(acc[4], acc[5], acc[6], acc[7]);
}

// w needs room for (1 + coulomb_w_mixed_chunks(ntile)) * naux doubles: w, then the chunk partials.
void launch_coulomb_w_mixed(const __nv_bfloat16* Bmix, const double* Dt, long naux, long ntile, long ntile2, double* w,
                            cudaStream_t s) {
  const int chunks = coulomb_w_mixed_chunks(ntile);
  dim3 grid(static_cast<unsigned>(chunks), static_cast<unsigned>((naux + WM_QR - 1) / WM_QR));
  k_coulomb_w_mixed<<<grid, WM_THREADS, 0, s>>>(Bmix, Dt, naux, ntile, ntile2, w + naux);
  k_sum_chunks<<<static_cast<unsigned>((naux + 255) / 256), 256, 0, s>>>(w + naux, chunks, naux, w);
}

void launch_coulomb_j_mixed(const __nv_bfloat16* Bmix, const double* w, long naux, long ntile, long ntile2,
                            int nsplit, double* Jpart, cudaStream_t s) {
  const long tile_elems = ntile * TILE2;
  long qper = (naux + nsplit - 1) / nsplit;
  dim3 grid(static_cast<unsigned>((tile_elems / 8 + J_THREADS - 1) / J_THREADS), static_cast<unsigned>(nsplit));
  k_coulomb_j_mixed<<<grid, J_THREADS, 0, s>>>(Bmix, w, naux, ntile, ntile2, qper, Jpart);
}

}  // namespace rijk
