// dmma.cuh — FP64 tensor-core (DMMA) and async-copy helpers shared by the FP64 kernels.
//
// tcgen05 has no f64 kind, so the FP64 contractions use the warp-level
// mma.sync.aligned.m8n8k4.row.col.f64 instruction.  Fragment ownership (PTX ISA, m8n8k4
// .f64): with g = lane / 4 and t = lane % 4,
//   A (8x4, row-major)  a = A[g][t]
//   B (4x8, column)     b = B[t][g]
//   C/D (8x8)           d0 = D[g][2t], d1 = D[g][2t+1]
//
// Shared-memory tiles are stored with the contraction index contiguous and a row stride
// LDS with LDS % 16 == 4 doubles: the 16 lanes of a half-warp then touch rows g = 0..3 at
// columns t = 0..3, i.e. 16 distinct 8-byte bank pairs (conflict-free).
#pragma once
#include <cstdint>

namespace rijk {

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte global -> shared copy; `valid` false zero-fills the destination.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  uint32_t s = smem_u32(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Streaming 128-bit load that does not allocate in L1 (B is read once per pass).
__device__ __forceinline__ double2 ldg_stream(const double2* p) {
  double2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Compensated (Neumaier) summation: the pair (s, c) carries the sum, c collecting the rounding
// error of every addition (Neumaier, Z. Angew. Math. Mech. 54 (1974) 39).  Used for the energy.
__host__ __device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
  const double t = s + x;
  c += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
  s = t;
}
__device__ __forceinline__ void warp_sum_comp(double& s, double& c) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double os = __shfl_xor_sync(0xffffffffu, s, o), oc = __shfl_xor_sync(0xffffffffu, c, o);
    neumaier_add(s, c, os);
    c += oc;
  }
}

// Tile (I, J), I >= J, of the lower block triangle.
__host__ __device__ __forceinline__ long tri_index(long I, long J) { return I * (I + 1) / 2 + J; }

__device__ __forceinline__ void tri_decode(long t, long& I, long& J) {
  long i = static_cast<long>((sqrt(8.0 * static_cast<double>(t) + 1.0) - 1.0) * 0.5);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  I = i;
  J = t - i * (i + 1) / 2;
}

}  // namespace rijk
