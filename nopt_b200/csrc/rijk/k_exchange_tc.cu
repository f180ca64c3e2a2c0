// k_exchange_tc.cu — mixed-precision exchange on tcgen05 tensor cores.
//
// Same contractions as the FP64 form (k_exchange_f64.cu; reference src/RI.cpp:146-171), with
// every operand split into two bf16 planes x = x_hi + x_lo (16 significant bits) and each
// product formed from three bf16 MMAs, a_hi b_hi + a_hi b_lo + a_lo b_hi, accumulated in fp32
// in TMEM ("split-BF16, 3-term").
//
//  split copy   Bmix[Q][t][hl][64][64] bf16: the packed tiles of B split once per geometry
//               (tile rows padded to an even count nt2 so that 128-row MMA blocks pair them)
//  K3 (mixed)   XT[nu][Q*noccp + i] (bf16 hi/lo planes) = sum_mu B^Q_{nu mu} C_{i mu}
//               persistent, warp-specialised: warp 0 issues TMA loads, one thread of warp 1
//               issues UMMA (M = 128 rows nu = two tile rows, N = noccp, K = 16), warps 2-5
//               drain TMEM.  For the block pair (J0, J1) and mu-tile I the A operand is the
//               tiles (J0, I), (J1, I) read K-major when I <= J0, otherwise the stored tiles
//               (I, J0), (I, J1) read MN-major (diagonal tiles are symmetric, so either view
//               of them is right): the packed triangle is consumed without unpacking.
//  K4 (mixed)   K = sum_k XT[mu][k] XT[nu][k] over 128 x 128 lower tiles, split over k;
//               fp32 accumulation per split, fp64 partial tiles summed by the unpack kernel.
// Every wait is bounded (about 1 s); on expiry a kernel raises an error bit, drains its
// in-flight copies and MMAs, frees TMEM and returns.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "rijk_internal.h"
#include "tc_util.cuh"

namespace rijk {

int set_err(rijk_ctx* ctx, int code, const char* fmt, ...);
int cuda_check(rijk_ctx* ctx, cudaError_t e, const char* what);
int ensure(rijk_ctx* ctx, DeviceBuf& b, size_t bytes, const char* what);
void release(DeviceBuf& b);

namespace {

constexpr uint32_t kTileBytes = 64 * 64 * 2;  // one 64 x 64 bf16 tile
constexpr int kTcThreads = 192;               // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kSmemBudget = 225 * 1024;
constexpr long kMixedMaxOcc = 192;  // orbitals of one half-transform batch (the MMA N of k_xform_tc)

__host__ __device__ inline int tri2(int I, int J) { return I * (I + 1) / 2 + J; }

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~static_cast<uintptr_t>(1023));
}

// ------------------------------------------------------------------ split copies ----
__global__ void k_split_b(const double* __restrict__ B, long nt, long ntile, long ntile2,
                          __nv_bfloat16* __restrict__ Bmix) {
  const long t2 = blockIdx.x, Q = blockIdx.y;
  long I, J;
  tri_decode(t2, I, J);
  const bool valid = I < nt && J < nt;
  const double* src = B + (Q * ntile + (valid ? tri_index(I, J) : 0)) * TILE2;
  __nv_bfloat16* hi = Bmix + (Q * ntile2 + t2) * 2 * TILE2;
  __nv_bfloat16* lo = hi + TILE2;
  for (int e = threadIdx.x; e < TILE2; e += blockDim.x) {
    double v = valid ? src[e] : 0.0;
    __nv_bfloat16 h = __float2bfloat16_rn(static_cast<float>(v));
    __nv_bfloat16 l = __float2bfloat16_rn(static_cast<float>(v - static_cast<double>(__bfloat162float(h))));
    hi[e] = h;
    lo[e] = l;
  }
}

__global__ void k_split_c(const double* __restrict__ MO, long nocc, long n, long noccp, long npad2,
                          __nv_bfloat16* __restrict__ Cmix) {
  long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long total = noccp * npad2;
  for (; idx < total; idx += static_cast<long>(gridDim.x) * blockDim.x) {
    long i = idx / npad2, mu = idx % npad2;
    double v = (i < nocc && mu < n) ? MO[i * n + mu] : 0.0;
    __nv_bfloat16 h = __float2bfloat16_rn(static_cast<float>(v));
    __nv_bfloat16 l = __float2bfloat16_rn(static_cast<float>(v - static_cast<double>(__bfloat162float(h))));
    Cmix[idx] = h;
    Cmix[total + idx] = l;
  }
}

// ---------------------------------------------------------- K3: half-transform ----
struct XformParams {
  int nt2, ntile2, naux, npairs, stages;
  int c_resident;  // 1: all of C is loaded into shared memory once; stages then carry the A tiles only
  long kdim;  // naux * noccp
  __nv_bfloat16* XTh;
  __nv_bfloat16* XTl;
  int* err;
};

template <int NOCCP>
struct XformCfg {
  static constexpr uint32_t kABytes = 4 * kTileBytes;      // A hi (2 tiles), A lo (2 tiles)
  static constexpr uint32_t kCBytes = NOCCP * 128;         // one bf16 plane of the C chunk
  static constexpr uint32_t kStage = kABytes + 2 * kCBytes;
  // two accumulator buffers, each at a power-of-two column offset
  static constexpr uint32_t kTmemCols = (2 * NOCCP <= 32) ? 32 : (2 * NOCCP <= 64) ? 64 : (2 * NOCCP <= 128) ? 128
                                        : (2 * NOCCP <= 256) ? 256 : 512;
  static constexpr uint32_t kAccCols = kTmemCols / 2;
  static int stages() { return std::min(6, static_cast<int>((kSmemBudget - 2048) / kStage)); }
  static size_t smem(int st) { return static_cast<size_t>(st) * kStage + 1024 + 256; }
  // resident C: nt2 chunks of (hi, lo) planes kept for the whole kernel, A-only stages
  __host__ __device__ static size_t c_bytes(int nt2) { return static_cast<size_t>(nt2) * 2 * kCBytes; }
  static int stages_resident(int nt2) {
    const long room = static_cast<long>(kSmemBudget) - 2048 - static_cast<long>(c_bytes(nt2));
    return room > 0 ? std::min(6, static_cast<int>(room / kABytes)) : 0;
  }
  static size_t smem_resident(int st, int nt2) { return static_cast<size_t>(st) * kABytes + c_bytes(nt2) + 1024 + 256; }
};

template <int NOCCP>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_xform_tc(const __grid_constant__ CUtensorMap mapB, const __grid_constant__ CUtensorMap mapC, XformParams p) {
  using Cfg = XformCfg<NOCCP>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int S = p.stages;
  const bool cres = p.c_resident != 0;
  const uint32_t stage_bytes = cres ? Cfg::kABytes : Cfg::kStage;
  uint8_t* cbase = smem + S * stage_bytes;  // resident C (cres only)
  uint64_t* full = reinterpret_cast<uint64_t*>(cbase + (cres ? Cfg::c_bytes(p.nt2) : 0));
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint64_t* cfull = drain + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cfull + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    mbar_init(drain, 1);
    mbar_init(cfull, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, Cfg::kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nitems = p.naux * p.npairs;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&mapB);
      tma_prefetch_desc(&mapC);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      if (cres) {  // every C chunk once: hi at + 0, lo at + kCBytes of chunk I
        mbar_expect_tx(cfull, static_cast<uint32_t>(Cfg::c_bytes(p.nt2)));
        for (int I = 0; I < p.nt2; ++I) {
          uint8_t* c = cbase + static_cast<size_t>(I) * 2 * Cfg::kCBytes;
          tma_load_2d(c, &mapC, cfull, I * 64, 0);
          tma_load_2d(c + Cfg::kCBytes, &mapC, cfull, I * 64, NOCCP);
        }
      }
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const int Q = item / p.npairs, jp = item - Q * p.npairs;
        const int J0 = 2 * jp, J1 = J0 + 1;
        const long qbase = static_cast<long>(Q) * p.ntile2;
        for (int I = 0; I < p.nt2; ++I) {
          if (!mbar_wait(&empty[stage], phase ^ 1, abort)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + stage * stage_bytes;
          mbar_expect_tx(&full[stage], stage_bytes);
          const int t0 = (I <= J0) ? tri2(J0, I) : tri2(I, J0);
          const int t1 = (I <= J0) ? tri2(J1, I) : tri2(I, J1);
          const int y0 = static_cast<int>((qbase + t0) * 128), y1 = static_cast<int>((qbase + t1) * 128);
          tma_load_2d(st + 0 * kTileBytes, &mapB, &full[stage], 0, y0);        // A hi, group 0
          tma_load_2d(st + 1 * kTileBytes, &mapB, &full[stage], 0, y1);        // A hi, group 1
          tma_load_2d(st + 2 * kTileBytes, &mapB, &full[stage], 0, y0 + 64);   // A lo, group 0
          tma_load_2d(st + 3 * kTileBytes, &mapB, &full[stage], 0, y1 + 64);   // A lo, group 1
          if (!cres) {
            tma_load_2d(st + Cfg::kABytes, &mapC, &full[stage], I * 64, 0);               // C hi
            tma_load_2d(st + Cfg::kABytes + Cfg::kCBytes, &mapC, &full[stage], I * 64, NOCCP);  // C lo
          }
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      // Drain: every stage's last issued load must have landed before the CTA exits.
      volatile int never = 0;
      for (int s = 0; s < S; ++s) {
        // stage s last used with parity (phase of its last fill); a stage never filled passes
        // immediately (fresh barrier, parity 1 = the phase before the first).
        uint32_t par = (s < stage) ? phase : (phase ^ 1);
        mbar_wait(&full[s], par, &never);
      }
      if (cres) mbar_wait(cfull, 0, &never);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint64_t kKdesc = sw128_desc_bits(16, 1024);
      constexpr uint64_t kMdesc = sw128_desc_bits(kTileBytes, 1024);  // LBO = 8 KB between the two nu groups
      constexpr uint32_t idK = idesc_bf16_f32(128, NOCCP, 0, 0);
      constexpr uint32_t idM = idesc_bf16_f32(128, NOCCP, 1, 0);
      int stage = 0;
      uint32_t phase = 0;
      uint32_t tph[2] = {0, 0};
      int buf = 0;
      bool ok = true;
      if (cres && !mbar_wait(cfull, 0, abort)) ok = false;
      for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const int Q = item / p.npairs, jp = item - Q * p.npairs;
        const int J0 = 2 * jp;
        if (!mbar_wait(&tempty[buf], tph[buf] ^ 1, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + buf * Cfg::kAccCols;
        for (int I = 0; I < p.nt2; ++I) {
          if (!mbar_wait(&full[stage], phase, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * stage_bytes);
          const uint32_t ahi = sa, alo = sa + 2 * kTileBytes;
          const uint32_t chi = cres ? smem_u32(cbase + static_cast<size_t>(I) * 2 * Cfg::kCBytes) : sa + Cfg::kABytes;
          const uint32_t clo = chi + Cfg::kCBytes;
          const bool mn = I > J0;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t a_h = mn ? sw128_desc(ahi + kk * 2048, kMdesc) : sw128_desc(ahi + kk * 32, kKdesc);
            const uint64_t a_l = mn ? sw128_desc(alo + kk * 2048, kMdesc) : sw128_desc(alo + kk * 32, kKdesc);
            const uint64_t b_h = sw128_desc(chi + kk * 32, kKdesc);
            const uint64_t b_l = sw128_desc(clo + kk * 32, kKdesc);
            const uint32_t id = mn ? idM : idK;
            umma_bf16(acc, a_h, b_h, id, (I | kk) != 0 ? 1u : 0u);
            umma_bf16(acc, a_h, b_l, id, 1u);
            umma_bf16(acc, a_l, b_h, id, 1u);
          }
          umma_commit(&empty[stage]);
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        umma_commit(&tfull[buf]);
        tph[buf] ^= 1;
        buf ^= 1;
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      // Drain: wait for every MMA issued by this thread before TMEM is released.
      umma_commit(drain);
      volatile int never = 0;
      if (!mbar_wait(drain, 0, &never)) atomicOr(p.err, DEVERR_TIMEOUT);
    }
  } else {
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    uint32_t tph[2] = {0, 0};
    int buf = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const int Q = item / p.npairs, jp = item - Q * p.npairs;
      if (!mbar_wait(&tfull[buf], tph[buf], abort)) {
        if (lane == 0) {
          *abort = 1;
          atomicOr(p.err, DEVERR_TIMEOUT);
        }
        break;
      }
      tc_fence_after();
      const long nu = static_cast<long>(jp) * 128 + q * 32 + lane;
      const uint32_t acc = tmem + buf * Cfg::kAccCols + (static_cast<uint32_t>(q * 32) << 16);
      __nv_bfloat16* dh = p.XTh + nu * p.kdim + static_cast<long>(Q) * NOCCP;
      __nv_bfloat16* dl = p.XTl + nu * p.kdim + static_cast<long>(Q) * NOCCP;
#pragma unroll 1
      for (int c0 = 0; c0 < NOCCP; c0 += 16) {
        float v[16];
        tmem_ld16(acc + c0, v);
        __align__(16) __nv_bfloat16 h[16], l[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) split_bf16(v[j], h[j], l[j]);
        uint4* oh = reinterpret_cast<uint4*>(dh + c0);
        uint4* ol = reinterpret_cast<uint4*>(dl + c0);
        oh[0] = reinterpret_cast<const uint4*>(h)[0];
        oh[1] = reinterpret_cast<const uint4*>(h)[1];
        ol[0] = reinterpret_cast<const uint4*>(l)[0];
        ol[1] = reinterpret_cast<const uint4*>(l)[1];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
      tph[buf] ^= 1;
      buf ^= 1;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, Cfg::kTmemCols);
  }
}

// ------------------------------------------------------------------ K4: SYRK ----
// K = X^T X over split-K ranges of kdim.  The contraction of one CTA runs in segments of `seg`
// 64-wide chunks (12 MMAs each: 4 k-steps x 3 split terms), alternating between two TMEM
// accumulators; the epilogue warps fold each finished segment into fp32 registers
// (accumulate_segment) while the next one is computed.  A TMEM accumulator thus never sums more
// than one segment, which keeps the tensor core's own fp32 accumulation error at the scale of a
// segment's partial sum instead of the whole range's.
struct SyrkParams {
  long kdim, kper;
  int npad2, ntile64, stages, seg;
  float* Kpart;  // fp32 partials, one 64 x 64 tile set per split
  int* err;
};

constexpr uint32_t kSyOpBytes = 128 * 128;  // 128 rows x 64 bf16
#ifndef RIJK_SYRK_SEG
#define RIJK_SYRK_SEG 4
#endif
constexpr int kSySeg = RIJK_SYRK_SEG;  // 64-wide chunks per TMEM accumulation segment
constexpr uint32_t kSyStage = 4 * kSyOpBytes;

__global__ void __launch_bounds__(kTcThreads, 1) k_syrk_tc(const __grid_constant__ CUtensorMap mapX, SyrkParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * kSyStage);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;   // [2] accumulator b holds a finished segment
  uint64_t* tempty = tfull + 2;  // [2] accumulator b has been folded into registers
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  long a, b;
  tri_decode(blockIdx.x, a, b);
  const bool diag = a == b;
  const long s = blockIdx.y;
  const long k0 = s * p.kper;
  const long k1 = std::min(k0 + p.kper, p.kdim);
  const int nch = static_cast<int>((k1 - k0 + 63) / 64);
  const int seg = p.seg;
  const int nseg = (nch + seg - 1) / seg;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 4);  // the four epilogue warps
    }
    mbar_init(drain, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&mapX);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      const uint32_t bytes = diag ? 2 * kSyOpBytes : 4 * kSyOpBytes;
      for (int c = 0; c < nch; ++c) {
        if (!mbar_wait(&empty[stage], phase ^ 1, abort)) {
          ok = false;
          break;
        }
        uint8_t* st = smem + stage * kSyStage;
        const int x = static_cast<int>(k0 + 64L * c);
        mbar_expect_tx(&full[stage], bytes);
        tma_load_2d(st, &mapX, &full[stage], x, static_cast<int>(a * 128));                          // A hi
        tma_load_2d(st + kSyOpBytes, &mapX, &full[stage], x, static_cast<int>(p.npad2 + a * 128));   // A lo
        if (!diag) {
          tma_load_2d(st + 2 * kSyOpBytes, &mapX, &full[stage], x, static_cast<int>(b * 128));              // B hi
          tma_load_2d(st + 3 * kSyOpBytes, &mapX, &full[stage], x, static_cast<int>(p.npad2 + b * 128));    // B lo
        }
        if (++stage == S) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      volatile int never = 0;
      for (int i = 0; i < S; ++i) {
        uint32_t par = (i < stage) ? phase : (phase ^ 1);
        mbar_wait(&full[i], par, &never);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint64_t kKdesc = sw128_desc_bits(16, 1024);
      constexpr uint32_t id = idesc_bf16_f32(128, 128, 0, 0);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int g = 0, kq = 0;  // segment of chunk c and its position in the segment
      for (int c = 0; c < nch; ++c) {
        const int buf = g & 1;
        if (kq == 0) {  // accumulator buf was last used by segment g - 2
          if (!mbar_wait(&tempty[buf], ((g >> 1) & 1) ^ 1, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        if (!mbar_wait(&full[stage], phase, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + buf * 128;
        const uint32_t sa = smem_u32(smem + stage * kSyStage);
        const uint32_t ah = sa, al = sa + kSyOpBytes;
        const uint32_t bh = diag ? ah : sa + 2 * kSyOpBytes, bl = diag ? al : sa + 3 * kSyOpBytes;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint64_t dah = sw128_desc(ah + kk * 32, kKdesc), dal = sw128_desc(al + kk * 32, kKdesc);
          const uint64_t dbh = sw128_desc(bh + kk * 32, kKdesc), dbl = sw128_desc(bl + kk * 32, kKdesc);
          umma_bf16(acc, dah, dbh, id, (kq | kk) != 0 ? 1u : 0u);
          umma_bf16(acc, dah, dbl, id, 1u);
          umma_bf16(acc, dal, dbh, id, 1u);
        }
        umma_commit(&empty[stage]);
        if (kq == seg - 1 || c == nch - 1) umma_commit(&tfull[buf]);
        if (++kq == seg) {
          kq = 0;
          ++g;
        }
        if (++stage == S) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      umma_commit(drain);
      volatile int never = 0;
      if (!mbar_wait(drain, 0, &never)) atomicOr(p.err, DEVERR_TIMEOUT);
    }
  } else {
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const long ra = 2 * a + row / 64;  // the same for the 32 lanes of a warp
    const int r = row % 64;
    float acc[128];
#pragma unroll
    for (int j = 0; j < 128; ++j) acc[j] = 0.f;
    bool ok = nseg > 0;
    for (int g = 0; g < nseg; ++g) {
      const int buf = g & 1;
      // warp-uniform outcome: the TMEM loads below are .sync.aligned
      if (!__all_sync(0xffffffffu, mbar_wait(&tfull[buf], (g >> 1) & 1, abort))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t t = tmem + buf * 128 + (static_cast<uint32_t>(q * 32) << 16);
      if (g + 1 < nseg) {
        accumulate_segment<32>(t, acc);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
        continue;
      }
      if (__any_sync(0xffffffffu, *abort)) {
        ok = false;
        break;
      }
      // last segment: fold and store 16 columns at a time, so the stores interleave with the loads
#pragma unroll
      for (int c0 = 0; c0 < 128; c0 += 16) {
        uint32_t v[16];
        tmem_ld16_nowait(t + c0, v);
        tmem_wait_ld();
        const long cb = 2 * b + c0 / 64;
        if (diag && ra < cb) continue;  // upper-right sub-tile of a diagonal tile: its mirror is stored
        float* out = p.Kpart + (s * p.ntile64 + tri_index(ra, cb)) * TILE2 + r * TILE + (c0 % 64);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(out + j) =
              make_float4(acc[c0 + j] + __uint_as_float(v[j]), acc[c0 + j + 1] + __uint_as_float(v[j + 1]),
                          acc[c0 + j + 2] + __uint_as_float(v[j + 2]), acc[c0 + j + 3] + __uint_as_float(v[j + 3]));
      }
    }
    if (!ok && lane == 0) {
      *abort = 1;
      atomicOr(p.err, DEVERR_TIMEOUT);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// --------------------------------------------------- K4 on CTA pairs: SYRK ----
// 256 x 256 output tiles on a pair of CTAs (cluster of 2) with tcgen05.mma.cta_group::2: CTA r
// holds rows 128 r .. 128 r + 127 of the tile's A panel and of its B panel (the same 64 KB
// stage layout as k_syrk_tc) and rows 128 r .. of the accumulator in its TMEM; the leader
// (rank 0) issues M = 256, N = 256 MMAs over both CTAs' shared memory.  Each operand byte
// crosses L2 -> SM once for twice the FLOPs of a 128 x 128 tile.  Both CTAs' TMA loads complete
// on the leader's stage barrier, which alone expects the pair's bytes; the leader's commits
// release the stage (and signal a finished accumulator) in both CTAs.  As in k_syrk_tc the
// contraction runs in segments over two TMEM accumulators (2 x 256 columns); eight epilogue
// warps per CTA fold them into registers (warp w reads TMEM lanes 32 (w % 4) .., columns
// 128 h .. 128 h + 127 with h = (w - 2) / 4) and report each fold to the leader's barrier.
// (Ten warps: the register file is split over four sub-partitions, so a thread may hold 168
// registers; more warps would leave too few for the 128 accumulators.)  A
// last 256-row panel that runs past npad2 computes rows and columns that are never stored.
constexpr int kPairThreads = 320;  // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue

struct SyrkPairParams {
  long kdim, kper;
  int npad2, nt2, ntile64, stages, seg;
  float* Kpart;
  int* err;
};

__global__ void __launch_bounds__(kPairThreads, 1)
    k_syrk_tc2(const __grid_constant__ CUtensorMap mapX, SyrkPairParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * kSyStage);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;   // [2]
  uint64_t* tempty = tfull + 2;  // [2] on the leader: 16 arrivals, 8 epilogue warps of each CTA
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  long a, b;
  tri_decode(blockIdx.x / 2, a, b);  // 256-row panels, b <= a
  const bool diag = a == b;
  const long s = blockIdx.y;
  const long k0 = s * p.kper;
  const long k1 = std::min(k0 + p.kper, p.kdim);
  const int nch = static_cast<int>((k1 - k0 + 63) / 64);
  const int seg = p.seg;
  const int nseg = (nch + seg - 1) / seg;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 16);
    }
    mbar_init(drain, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // both CTAs' barriers and TMEM exist before any traffic between them
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&mapX);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      const uint32_t cta_bytes = diag ? 2 * kSyOpBytes : 4 * kSyOpBytes;
      const int ra = static_cast<int>(a * 256 + rank * 128), rb = static_cast<int>(b * 256 + rank * 128);
      for (int c = 0; c < nch; ++c) {
        if (!mbar_wait(&empty[stage], phase ^ 1, abort)) {
          ok = false;
          break;
        }
        uint8_t* st = smem + stage * kSyStage;
        const int x = static_cast<int>(k0 + 64L * c);
        if (leader) mbar_expect_tx(&full[stage], 2 * cta_bytes);  // this CTA's bytes and the peer's
        tma_load_2d_pair(st, &mapX, &full[stage], x, ra);                                 // A hi
        tma_load_2d_pair(st + kSyOpBytes, &mapX, &full[stage], x, p.npad2 + ra);          // A lo
        if (!diag) {
          tma_load_2d_pair(st + 2 * kSyOpBytes, &mapX, &full[stage], x, rb);              // B hi
          tma_load_2d_pair(st + 3 * kSyOpBytes, &mapX, &full[stage], x, p.npad2 + rb);    // B lo
        }
        if (++stage == S) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      if (leader) {  // every issued load of the pair has landed before the pair may exit
        volatile int never = 0;
        for (int i = 0; i < S; ++i) {
          uint32_t par = (i < stage) ? phase : (phase ^ 1);
          mbar_wait(&full[i], par, &never);
        }
      }
    }
  } else if (warp == 1) {
    if (leader && lane == 0) {
      constexpr uint64_t kKdesc = sw128_desc_bits(16, 1024);
      constexpr uint32_t id = idesc_bf16_f32(256, 256, 0, 0);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int g = 0, kq = 0;  // segment of chunk c and its position in the segment
      for (int c = 0; c < nch; ++c) {
        const int buf = g & 1;
        if (kq == 0) {  // both CTAs have folded accumulator buf (segment g - 2)
          if (!mbar_wait(&tempty[buf], ((g >> 1) & 1) ^ 1, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        if (!mbar_wait(&full[stage], phase, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + buf * 256;
        const uint32_t sa = smem_u32(smem + stage * kSyStage);
        const uint32_t ah = sa, al = sa + kSyOpBytes;
        const uint32_t bh = diag ? ah : sa + 2 * kSyOpBytes, bl = diag ? al : sa + 3 * kSyOpBytes;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint64_t dah = sw128_desc(ah + kk * 32, kKdesc), dal = sw128_desc(al + kk * 32, kKdesc);
          const uint64_t dbh = sw128_desc(bh + kk * 32, kKdesc), dbl = sw128_desc(bl + kk * 32, kKdesc);
          umma_bf16_pair(acc, dah, dbh, id, (kq | kk) != 0 ? 1u : 0u);
          umma_bf16_pair(acc, dah, dbl, id, 1u);
          umma_bf16_pair(acc, dal, dbh, id, 1u);
        }
        umma_commit_pair(&empty[stage], 0x3);
        if (kq == seg - 1 || c == nch - 1) umma_commit_pair(&tfull[buf], 0x3);
        if (++kq == seg) {
          kq = 0;
          ++g;
        }
        if (++stage == S) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (!ok) {
        *abort = 1;
        atomicOr(p.err, DEVERR_TIMEOUT);
      }
      umma_commit_pair(drain, 0x3);
    }
  } else {
    const int q = warp & 3, h = (warp - 2) >> 2;
    const long row = a * 256 + rank * 128 + q * 32 + lane;  // row of K
    const long ra = row / 64;  // the same for the 32 lanes of a warp
    const int r = static_cast<int>(row % 64);
    float acc[128];
#pragma unroll
    for (int j = 0; j < 128; ++j) acc[j] = 0.f;
    bool ok = nseg > 0;
    for (int g = 0; g < nseg; ++g) {
      const int buf = g & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&tfull[buf], (g >> 1) & 1, abort))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t t = tmem + buf * 256 + h * 128 + (static_cast<uint32_t>(q * 32) << 16);
      if (g + 1 < nseg) {
        accumulate_segment<16>(t, acc);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(&tempty[buf], 0);
        continue;
      }
      if (__any_sync(0xffffffffu, *abort)) {
        ok = false;
        break;
      }
      // last segment: fold and store 16 columns at a time, so the stores interleave with the loads
#pragma unroll
      for (int c0 = 0; c0 < 128; c0 += 16) {
        uint32_t v[16];
        tmem_ld16_nowait(t + c0, v);
        tmem_wait_ld();
        const long cb = (b * 256 + h * 128 + c0) / 64;
        if (ra < cb || ra >= p.nt2 || cb >= p.nt2) continue;  // upper triangle, or past npad2
        float* out = p.Kpart + (s * p.ntile64 + tri_index(ra, cb)) * TILE2 + r * TILE + (c0 % 64);
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(out + j) =
              make_float4(acc[c0 + j] + __uint_as_float(v[j]), acc[c0 + j + 1] + __uint_as_float(v[j + 1]),
                          acc[c0 + j + 2] + __uint_as_float(v[j + 2]), acc[c0 + j + 3] + __uint_as_float(v[j + 3]));
      }
    }
    if (!ok && lane == 0) {
      *abort = 1;
      atomicOr(p.err, DEVERR_TIMEOUT);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1 && lane == 0) {  // no MMA of the pair still writes this CTA's TMEM
    volatile int never = 0;
    if (!mbar_wait(drain, 0, &never)) atomicOr(p.err, DEVERR_TIMEOUT);
  }
  __syncthreads();
  cluster_sync_all();  // neither CTA frees its TMEM or exits while the pair's work may touch it
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem, 512);
  }
}

// ------------------------------------------------------------- tensor maps ----
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  // looked up once (thread-safe static initialisation: contexts may live on several host threads)
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiledFn>(p);
    return static_cast<EncodeTiledFn>(nullptr);
  }();
  return fn;
}

// 2-D bf16 map of a row-major [rows][cols] array, box {64, box_rows}, 128-byte swizzle.
bool make_map(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int num_sms(int device) {
  static std::atomic<int> cached[64] = {};
  if (device >= 0 && device < 64 && cached[device]) return cached[device];
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  if (device >= 0 && device < 64) cached[device] = v;
  return v;
}

template <int NOCCP>
void launch_xform_tc(const CUtensorMap& mB, const CUtensorMap& mC, XformParams p, int device, cudaStream_t s) {
  using Cfg = XformCfg<NOCCP>;
  // keep C resident when it leaves room for at least 3 A stages
  const int sr = Cfg::stages_resident(p.nt2);
  p.c_resident = sr >= 3 ? 1 : 0;
  p.stages = p.c_resident ? sr : Cfg::stages();
  const size_t smem = p.c_resident ? Cfg::smem_resident(p.stages, p.nt2) : Cfg::smem(p.stages);
  ensure_smem_limit(reinterpret_cast<const void*>(k_xform_tc<NOCCP>), smem);
  int nitems = p.naux * p.npairs;
  int grid = std::min(nitems, num_sms(device));
  k_xform_tc<NOCCP><<<grid, kTcThreads, smem, s>>>(mB, mC, p);
}

using XformLaunch = void (*)(const CUtensorMap&, const CUtensorMap&, XformParams, int, cudaStream_t);
const XformLaunch kXformTable[13] = {nullptr,
                                     launch_xform_tc<16>,
                                     launch_xform_tc<32>,
                                     launch_xform_tc<48>,
                                     launch_xform_tc<64>,
                                     launch_xform_tc<80>,
                                     launch_xform_tc<96>,
                                     launch_xform_tc<112>,
                                     launch_xform_tc<128>,
                                     launch_xform_tc<144>,
                                     launch_xform_tc<160>,
                                     launch_xform_tc<176>,
                                     launch_xform_tc<192>};

}  // namespace

int mixed_prepare(rijk_ctx* ctx) {
  if (ctx->have_bmix) return RIJK_OK;
  if (!encode_fn()) return set_err(ctx, RIJK_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const long nt2 = round_up(ctx->nt, 2), ntile2 = nt2 * (nt2 + 1) / 2;
  const size_t bytes = static_cast<size_t>(ctx->nq) * ntile2 * 2 * TILE2 * sizeof(__nv_bfloat16);
  int rc = ensure(ctx, ctx->Bmix, bytes, "split-bf16 copy of B");
  if (rc) return rc;
  dim3 grid(static_cast<unsigned>(ntile2), static_cast<unsigned>(ctx->nq));
  k_split_b<<<grid, 256, 0, ctx->stream>>>(static_cast<const double*>(ctx->B.p), ctx->nt, ctx->ntile, ntile2,
                                           static_cast<__nv_bfloat16*>(ctx->Bmix.p));
  rc = cuda_check(ctx, cudaGetLastError(), "split copy of B");
  if (rc) return rc;
  ctx->have_bmix = true;
  ctx->stats.bytes_b_mixed = static_cast<long>(bytes);
  return RIJK_OK;
}

// Split-K plan of one SYRK launch: chunk-aligned ranges of `kper` columns, at least ~4 CTAs (or CTA
// pairs) per SM (pair) in total, every split non-empty; the split count is chosen in [want, 4 want] so
// that the CTAs fill whole waves.
struct SyrkPlan {
  long kper;
  int nsplit;
};
static SyrkPlan syrk_plan(long kdim, long tiles, long slots) {
  const long nchunks = (kdim + 63) / 64;
  const long want = std::max<long>(1, (4L * slots + tiles - 1) / tiles);
  long best = want;
  double best_eff = 0.0;
  for (long sp = want; sp <= 4 * want && sp <= std::max<long>(1, nchunks / 2); ++sp) {
    const long ctas = tiles * sp, waves = (ctas + slots - 1) / slots;
    const double eff = static_cast<double>(ctas) / static_cast<double>(waves * slots);
    if (eff > best_eff + 0.02) {  // prefer fewer splits unless the fill improves noticeably
      best_eff = eff;
      best = sp;
    }
  }
  const long kper = std::max<long>(2, (nchunks + best - 1) / best) * 64;
  return {kper, static_cast<int>((kdim + kper - 1) / kper)};
}

// Split-K plan of the single-CTA SYRK (one CTA per SM at a time): the fewest waves that are at least
// 90 % full, each CTA at most kMaxChunks 64-wide chunks (its fp32 register sum over the TMEM segments
// stays as short as the CTA-pair kernel's).  Few, long CTAs pay the pipeline fill and the epilogue once
// per wave instead of once per short range.
constexpr long kMaxChunks = 1024;
static SyrkPlan syrk_plan_waves(long kdim, long tiles, long slots) {
  const long nchunks = (kdim + 63) / 64;
  const long smin = std::max<long>(1, (nchunks + kMaxChunks - 1) / kMaxChunks);
  const long smax = std::max<long>(smin, nchunks / 2);
  long sp = smin;
  for (long w = 1; w <= 64; ++w) {
    const long cand = std::min(smax, (w * slots) / tiles);
    if (cand < smin) continue;
    if (static_cast<double>(tiles * cand) >= 0.9 * static_cast<double>(w * slots)) {
      sp = cand;
      break;
    }
  }
  const long kper = std::max<long>(2, (nchunks + sp - 1) / sp) * 64;
  return {kper, static_cast<int>((kdim + kper - 1) / kper)};
}

// K = sum over orbital batches of X_b^T X_b.  The half-transform holds all orbitals of one batch in
// the MMA's N dimension (at most 192), so n_c beyond that runs as several batches of equal size; each
// batch's split-K partials go to their own slots and one reduction sums them all.
int mixed_exchange(rijk_ctx* ctx, const double* dMO, long nocc, double* dK) {
  int rc = mixed_prepare(ctx);
  if (rc) return rc;
  const long n = ctx->n, naux = ctx->nq;
  const long nt2 = round_up(ctx->nt, 2), ntile2 = nt2 * (nt2 + 1) / 2, npad2 = nt2 * TILE;
  const long nb = nt2 / 2, ntile128 = nb * (nb + 1) / 2;
  const long sms = num_sms(ctx->device);
  // K on CTA pairs with 256 x 256 tiles once npad2 >= 1024 (at most one half-empty panel, <= 12.5 %
  // wasted); its split count fills whole waves of SM pairs the same way
  const bool pair_syrk = npad2 >= 1024;
  const long nb256 = (npad2 + 255) / 256, tiles256 = nb256 * (nb256 + 1) / 2;
  const long nbatch = (round_up(nocc, 16) + kMixedMaxOcc - 1) / kMixedMaxOcc;
  const long per_batch = round_up((nocc + nbatch - 1) / nbatch, 16);
  long noccp_max = 0;
  int nsplit_total = 0;
  for (long b0 = 0; b0 < nocc; b0 += per_batch) {
    const long noccp_b = round_up(std::min(per_batch, nocc - b0), 16);
    noccp_max = std::max(noccp_max, noccp_b);
    const SyrkPlan pl = pair_syrk ? syrk_plan(naux * noccp_b, tiles256, sms / 2) : syrk_plan_waves(naux * noccp_b, ntile128, sms);
    nsplit_total += pl.nsplit;
  }
  cudaStream_t s = ctx->stream;
  if ((rc = ensure(ctx, ctx->MOp, static_cast<size_t>(2 * noccp_max * npad2) * sizeof(__nv_bfloat16), "split C")) ||
      (rc = ensure(ctx, ctx->XT, static_cast<size_t>(2 * npad2) * naux * noccp_max * sizeof(__nv_bfloat16),
                   "split XT")) ||
      (rc = ensure(ctx, ctx->Kpart,
                   static_cast<size_t>(ntile2) * TILE2 * (sizeof(double) + nsplit_total * sizeof(float)), "Kpart")))
    return rc;  // fp64 sum area, then the fp32 split partials of every batch
  double* Ksum = static_cast<double*>(ctx->Kpart.p);
  float* Kpart32 = reinterpret_cast<float*>(Ksum + ntile2 * TILE2);
  __nv_bfloat16* Cmix = static_cast<__nv_bfloat16*>(ctx->MOp.p);
  __nv_bfloat16* XT = static_cast<__nv_bfloat16*>(ctx->XT.p);
  int launches = 0;
  int slot = 0;  // first split slot of the current batch
  for (long b0 = 0; b0 < nocc; b0 += per_batch) {
    const long nocc_b = std::min(per_batch, nocc - b0);
    const long noccp = round_up(nocc_b, 16);
    const long kdim = naux * noccp;
    {
      long total = noccp * npad2;
      unsigned g = static_cast<unsigned>(std::min<long>((total + 255) / 256, 148L * 16));
      k_split_c<<<g, 256, 0, s>>>(dMO + b0 * n, nocc_b, n, noccp, npad2, Cmix);
      ++launches;
      prof_mark(ctx, "split_c");
    }
    CUtensorMap mB, mC, mX;
    if (!make_map(&mB, ctx->Bmix.p, 64, static_cast<uint64_t>(naux) * ntile2 * 128, 64) ||
        !make_map(&mC, Cmix, static_cast<uint64_t>(npad2), static_cast<uint64_t>(2 * noccp), static_cast<uint32_t>(noccp)) ||
        !make_map(&mX, XT, static_cast<uint64_t>(kdim), static_cast<uint64_t>(2 * npad2), 128))
      return set_err(ctx, RIJK_ERR_CUDA, "tensor map encoding failed");
    XformParams xp{};
    xp.nt2 = static_cast<int>(nt2);
    xp.ntile2 = static_cast<int>(ntile2);
    xp.naux = static_cast<int>(naux);
    xp.npairs = static_cast<int>(nb);
    xp.kdim = kdim;
    xp.XTh = XT;
    xp.XTl = XT + npad2 * kdim;
    xp.err = static_cast<int*>(ctx->err.p);
    kXformTable[noccp / 16](mB, mC, xp, ctx->device, s);
    ++launches;
    prof_mark(ctx, "xform_tc");
    float* part = Kpart32 + static_cast<size_t>(slot) * ntile2 * TILE2;
    if (pair_syrk) {
      const SyrkPlan pl = syrk_plan(kdim, tiles256, sms / 2);
      SyrkPairParams pp{};
      pp.kdim = kdim;
      pp.kper = pl.kper;
      pp.npad2 = static_cast<int>(npad2);
      pp.nt2 = static_cast<int>(nt2);
      pp.ntile64 = static_cast<int>(ntile2);
      pp.Kpart = part;
      pp.err = static_cast<int*>(ctx->err.p);
      pp.seg = kSySeg;
      pp.stages = std::min(4, static_cast<int>((kSmemBudget - 2048) / kSyStage));
      const size_t smem2 = static_cast<size_t>(pp.stages) * kSyStage + 1024 + 256;
      ensure_smem_limit(reinterpret_cast<const void*>(k_syrk_tc2), smem2);
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(static_cast<unsigned>(2 * tiles256), static_cast<unsigned>(pl.nsplit));
      cfg.blockDim = dim3(kPairThreads);
      cfg.dynamicSmemBytes = smem2;
      cfg.stream = s;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 2;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      rc = cuda_check(ctx, cudaLaunchKernelEx(&cfg, k_syrk_tc2, mX, pp), "CTA-pair SYRK launch");
      if (rc) return rc;
      slot += pl.nsplit;
    } else {
      const SyrkPlan pl = syrk_plan_waves(kdim, ntile128, sms);
      SyrkParams sp{};
      sp.kdim = kdim;
      sp.kper = pl.kper;
      sp.npad2 = static_cast<int>(npad2);
      sp.ntile64 = static_cast<int>(ntile2);
      sp.Kpart = part;
      sp.err = static_cast<int*>(ctx->err.p);
      sp.seg = kSySeg;
      sp.stages = std::min(4, static_cast<int>((kSmemBudget - 2048) / kSyStage));
      size_t smem = static_cast<size_t>(sp.stages) * kSyStage + 1024 + 256;
      ensure_smem_limit(reinterpret_cast<const void*>(k_syrk_tc), smem);
      dim3 grid(static_cast<unsigned>(ntile128), static_cast<unsigned>(pl.nsplit));
      k_syrk_tc<<<grid, kTcThreads, smem, s>>>(mX, sp);
      slot += pl.nsplit;
    }
    ++launches;
    prof_mark(ctx, "syrk_tc");
  }
  launch_unpack_sym_f32(Kpart32, nsplit_total, ntile2, n, Ksum, dK, s);
  launches += 2;
  prof_mark(ctx, "unpack_k");
  ctx->stats.kernels_last_fock = launches;
  return cuda_check(ctx, cudaGetLastError(), "mixed exchange launch");
}

}  // namespace rijk
