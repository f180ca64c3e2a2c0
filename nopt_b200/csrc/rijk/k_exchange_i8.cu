// k_exchange_i8.cu — the exchange contraction K = X^T X of the FP64 form on tcgen05 tensor cores,
// with FP64 accuracy from exact int8 products (the Ozaki splitting scheme).
//
// tcgen05 has no FP64 kind.  Each row nu of X^T (the half-transformed tensor, k = Q n_c + i
// contiguous) is written, over the k range of one split-K part r, as
//     X[nu][k] = 2^e(r,nu) * sum_{s=0}^{7} d_s[nu][k] 2^{-7(s+1)},   d_s integer in [-64, 64],
// with e chosen so that max_k |X[nu][k]| / 2^e < 1/2 (k_slice_x).  The digits are exact: each
// step scales by 2^7, rounds to the nearest integer and keeps the exact remainder, so the value
// left after 8 digits is at most 2^-57 of 2^e, which is below 2^-55 of the row maximum.  Then
//     K_mu,nu = 2^(e_mu + e_nu) sum_g 2^{-7(g+2)} sum_{s+t=g} (d_s[mu] . d_t[nu]),
// where every (d_s . d_t) is an exact s32 tensor-core sum (|d_s d_t| <= 4096; a part spans at
// most 65504 k, and a group sums at most 8 pairs: 8 * 4096 * 65504 < 2^31 - 1).  The groups g < 8
// (36 digit pairs) are kept; the dropped ones are below 9 * 2^-58 of 2^(e_mu + e_nu) per k,
// the level of FP64 rounding in a sum of products.
//
// Digit layout: row nu of the planes is kdim/32 blocks of 256 bytes, block c holding the 8 digits
// of k in [32c, 32c + 32) as 8 runs of 32 bytes (digit-major).  A stage then moves two 128-byte
// halves per row (digits 0-3, 4-7) with 128-byte-swizzled TMA boxes, and the K-major descriptor
// of digit d points 32 (d mod 4) bytes into its half, as a 16-bit operand steps through K.
//
// k_syrk_i8: one CTA per (128 x 128 block (a, b), b <= a, split part r), in two passes over the
// part: groups 0-3 (10 products, digits 0-3 only) and groups 4-7 (26 products), each into 4 TMEM
// accumulators of 128 columns.  Every MMA is M 128, N 128, K 32: it reads 128 bytes of shared
// memory operands per tensor clock, which the SM sustains (N 64 would need 192).  The epilogue of
// pass 0 stores the scaled FP64 partial of its tiles, that of pass 1 adds to it (the same thread
// and elements); the partials have the layout of k_syrk_f64, summed and unpacked by
// launch_unpack_sym.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>

#include "rijk_internal.h"
#include "tc_util.cuh"

namespace rijk {

int set_err(rijk_ctx* ctx, int code, const char* fmt, ...);
int cuda_check(rijk_ctx* ctx, cudaError_t e, const char* what);
int ensure(rijk_ctx* ctx, DeviceBuf& b, size_t bytes, const char* what);

namespace {

constexpr int kDigits = 8;                     // digit planes per value
constexpr int kChunk = 32;                     // k per stage and per MMA (one 32-byte swizzle atom row)
constexpr int kI8Threads = 192;                // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kBlock = kDigits * kChunk;       // bytes per row and 32 k: 8 digits x 32 B
constexpr uint32_t kHalf = 128 * 128;          // 4 digits of a 128-row panel: 128 rows x 128 B
constexpr uint32_t kI8Stage = 4 * kHalf;       // A digits 0-3, A 4-7, B 0-3, B 4-7: 64 KB
constexpr long kMaxPart = 65504;               // k per split part: 8 * 4096 * 65504 < 2^31 - 1, every s32 sum exact
constexpr int kI8SmemBudget = 225 * 1024;

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~static_cast<uintptr_t>(1023));
}

// ------------------------------------------------------------------ digit planes ----
// One CTA per (row nu, part r), part length up to kMaxPart: a first sweep takes the row's maximum
// over the part (from HBM), a second one re-reads the part (now in L2) and writes each thread's
// 8 digits of 4 consecutive k as packed 4-byte words into the k's block.  Rows at or past npad
// (the padding of the 128-row blocks), and k from kdim to the end of the last block, get zero
// digits.
constexpr int kSliceThreads = 256;

__global__ void __launch_bounds__(kSliceThreads) k_slice_x(const double* __restrict__ XT, long npad, long npad2,
                                                           long kdim, long kper, int8_t* __restrict__ Xs,
                                                           int* __restrict__ E) {
  __shared__ double wmax[kSliceThreads / 32];
  const long row = blockIdx.x, part = blockIdx.y;
  const long k0 = part * kper, k1 = std::min(k0 + kper, kdim);
  const long kend = k1 == kdim ? (kdim + kChunk - 1) / kChunk * kChunk : k1;  // zero digits fill the last block
  const long nblk = (kdim + kChunk - 1) / kChunk;
  int8_t* out = Xs + static_cast<size_t>(row) * nblk * kBlock;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const bool live = row < npad;
  const double* x = XT + static_cast<size_t>(live ? row : 0) * kdim;
  double m = 0.0;
  if (live)
    for (long k = k0 + 4L * t; k < k1; k += 4L * kSliceThreads) {  // k1 and k are multiples of 4
      const double2 a = *reinterpret_cast<const double2*>(x + k);
      const double2 b = *reinterpret_cast<const double2*>(x + k + 2);
      m = fmax(m, fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y))));
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) wmax[warp] = m;
  __syncthreads();
  m = wmax[0];
#pragma unroll
  for (int w = 1; w < kSliceThreads / 32; ++w) m = fmax(m, wmax[w]);
  // m = f 2^(b+1) with f in [1/2, 1) (b = ilogb(m)); dividing by 2^(b+2) leaves |x| < 1/2
  const int e = m > 0.0 ? ilogb(m) + 2 : 0;
  if (t == 0) E[part * npad2 + row] = e;
  for (long k = k0 + 4L * t; k < kend; k += 4L * kSliceThreads) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (live && k < k1) {
      const double2 a = *reinterpret_cast<const double2*>(x + k);
      const double2 b = *reinterpret_cast<const double2*>(x + k + 2);
      v[0] = a.x;
      v[1] = a.y;
      v[2] = b.x;
      v[3] = b.y;
    }
    uint32_t packed[kDigits] = {};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double r = ldexp(v[q], -e);
#pragma unroll
      for (int d = 0; d < kDigits; ++d) {
        const double tt = r * 128.0;
        const double dg = rint(tt);
        r = tt - dg;
        packed[d] |= (static_cast<uint32_t>(static_cast<int>(dg)) & 0xFFu) << (8 * q);
      }
    }
    int8_t* blk = out + (k / kChunk) * kBlock + (k % kChunk);
#pragma unroll
    for (int d = 0; d < kDigits; ++d) *reinterpret_cast<uint32_t*>(blk + d * kChunk) = packed[d];
  }
}

// 2^e exactly for |e| <= 1000 (the exponent bits), else through ldexp.
__device__ __forceinline__ double pow2i(int e) {
  return (e >= -1000 && e <= 1000) ? __longlong_as_double(static_cast<long long>(e + 1023) << 52) : ldexp(1.0, e);
}

// ------------------------------------------------------------------ int8 SYRK ----
struct I8Params {
  long kdim, kper;
  int npad2, nt, stages;
  double* Kpart;  // FP64 partials [part][ntile][64][64]
  long ntile;
  const int* E;   // row exponents [part][npad2]
  int* err;
};

// One stage's MMAs of pass `pass` (groups 4 pass .. 4 pass + 3).  Digit d of a panel sits in half
// d / 4, 32 (d mod 4) bytes into each 128-byte swizzled row.  The first product of a group in a
// pass (digits (0, g), first chunk) starts its accumulator.
__device__ __forceinline__ void issue_chunk(uint32_t tmem, uint32_t sa, uint32_t sb, int pass, bool later) {
  constexpr uint64_t kDesc = sw128_desc_bits(16, 1024);
  constexpr uint32_t id = idesc_s8_s32(128, 128);
#pragma unroll
  for (int s = 0; s < kDigits; ++s) {
    const uint64_t da = sw128_desc(sa + (s / 4) * kHalf + (s % 4) * 32, kDesc);
#pragma unroll
    for (int t = 0; t < kDigits - s; ++t) {
      if ((s + t) / 4 != pass) continue;
      const uint64_t db = sw128_desc(sb + (t / 4) * kHalf + (t % 4) * 32, kDesc);
      umma_s8(tmem + ((s + t) % 4) * 128, da, db, id, (later || s != 0) ? 1u : 0u);
    }
  }
}

__global__ void __launch_bounds__(kI8Threads, 1)
    k_syrk_i8(const __grid_constant__ CUtensorMap mapX, I8Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = align1024(smem_raw);
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * kI8Stage);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;   // a pass's accumulators are final (phase = pass)
  uint64_t* tempty = tfull + 1;  // pass 0's accumulators have been read
  uint64_t* drain = tempty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  long a, b;
  tri_decode(blockIdx.x, a, b);  // 128-row blocks, b <= a
  const bool diag = a == b;
  const long part = blockIdx.y;
  const long k0 = part * p.kper;
  const long k1 = std::min(k0 + p.kper, p.kdim);
  const int nch = static_cast<int>((k1 - k0 + kChunk - 1) / kChunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, 4);
    mbar_init(drain, 1);
    *abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
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
      for (int pass = 0; pass < 2 && ok; ++pass) {
        const int halves = pass + 1;  // pass 0 needs digits 0-3 only
        const uint32_t bytes = (diag ? 1u : 2u) * halves * kHalf;
        for (int c = 0; c < nch; ++c) {
          if (!mbar_wait(&empty[stage], phase ^ 1, abort)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + stage * kI8Stage;
          const int x = static_cast<int>((k0 / kChunk + c) * kBlock);  // byte column of chunk c
          mbar_expect_tx(&full[stage], bytes);
          for (int h = 0; h < halves; ++h) {
            tma_load_2d(st + h * kHalf, &mapX, &full[stage], x + 128 * h, static_cast<int>(a * 128));
            if (!diag)
              tma_load_2d(st + (2 + h) * kHalf, &mapX, &full[stage], x + 128 * h, static_cast<int>(b * 128));
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
      volatile int never = 0;
      for (int i = 0; i < S; ++i) {
        uint32_t par = (i < stage) ? phase : (phase ^ 1);
        mbar_wait(&full[i], par, &never);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int pass = 0; pass < 2 && ok; ++pass) {
        if (pass == 1) {  // the epilogue has read pass 0's accumulators
          if (!mbar_wait(tempty, 0, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        for (int c = 0; c < nch; ++c) {
          if (!mbar_wait(&full[stage], phase, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * kI8Stage);
          issue_chunk(tmem, sa, diag ? sa : sa + 2 * kHalf, pass, c != 0);
          umma_commit(&empty[stage]);
          if (++stage == S) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (ok) umma_commit(tfull);
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
    const int row = q * 32 + lane;     // row of the 128-row block
    const long ra = 2 * a + row / 64;  // 64-row tile, the same for the warp's 32 lanes
    const int r = row % 64;
    const int* Ep = p.E + part * p.npad2;
    const double rs = pow2i(Ep[a * 128 + row]);  // row scale 2^e
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(q * 32) << 16);
    bool ok = true;
    for (int pass = 0; pass < 2; ++pass) {
      if (!__all_sync(0xffffffffu, mbar_wait(tfull, pass, abort)) || __any_sync(0xffffffffu, *abort)) {
        ok = false;
        break;
      }
      tc_fence_after();
      double gf[4];  // 2^-7(4 pass + g + 2)
#pragma unroll
      for (int g = 0; g < 4; ++g) gf[g] = pow2i(-7 * (4 * pass + g + 2));
#pragma unroll 1
      for (int c0 = 0; c0 < 128; c0 += 16) {
        const long cb = 2 * b + c0 / 64;
        // upper-right sub-tile of a diagonal block (its mirror is stored), or rows past npad
        if ((diag && ra < cb) || ra >= p.nt) continue;
        uint32_t v[4][16];
#pragma unroll
        for (int g = 0; g < 4; ++g) tmem_ld16_nowait(lane_base + g * 128 + c0, v[g]);
        tmem_wait_ld();
        double* out = p.Kpart + (part * p.ntile + tri_index(ra, cb)) * TILE2 + static_cast<long>(r) * TILE + (c0 % 64);
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          double w[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            double acc = 0.0;
#pragma unroll
            for (int g = 3; g >= 0; --g)  // smallest first; the group factors are exact powers of two
              acc = fma(static_cast<double>(static_cast<int32_t>(v[g][j + h])), gf[g], acc);
            w[h] = acc * (rs * pow2i(__ldg(Ep + b * 128 + c0 + j + h)));
          }
          double2* o = reinterpret_cast<double2*>(out + j);
          if (pass == 1) {
            const double2 prev = *o;
            w[0] += prev.x;
            w[1] += prev.y;
          }
          *o = make_double2(w[0], w[1]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (pass == 0 && lane == 0) mbar_arrive(tempty);
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
    tmem_dealloc(tmem, 512);
  }
}

// ------------------------------------------------------------------ tensor maps ----
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn_i8() {
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

// 2-D map of the digit rows [rows][cols bytes], box {128 bytes, box_rows}, 128-byte swizzle.
bool make_map_i8(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn_i8();
  if (!fn) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols};
  cuuint32_t box[2] = {128, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int sm_count(int device) {
  static std::atomic<int> cached[64] = {};
  if (device < 0 || device >= 64) return 148;
  if (!cached[device]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    cached[device] = v > 0 ? v : 148;
  }
  return cached[device];
}

}  // namespace

// Split-K parts of the int8 SYRK: chunk-aligned, at most kMaxPart k each, and enough CTAs for
// about two waves (one CTA per SM), chosen among [want, 4 want] so that the last wave is fullest.
int syrk_i8_parts(long nt, long kdim, int device, long* kper_out) {
  const long nb = (nt + 1) / 2, ctas_per_part = nb * (nb + 1) / 2;
  const long sms = sm_count(device);
  const long nchunks = (kdim + kChunk - 1) / kChunk;
  const long min_parts = (kdim + kMaxPart - 1) / kMaxPart;
  const long want = std::max(min_parts, (2 * sms + ctas_per_part - 1) / ctas_per_part);
  long best = want;
  double best_eff = 0.0;
  for (long sp = want; sp <= 4 * want && sp <= std::max<long>(1, nchunks); ++sp) {
    const long ctas = ctas_per_part * sp, waves = (ctas + sms - 1) / sms;
    const double eff = static_cast<double>(ctas) / static_cast<double>(waves * sms);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
      best = sp;
    }
  }
  long kper = round_up((kdim + best - 1) / best, kChunk);
  kper = std::min(kper, kMaxPart);
  *kper_out = kper;
  return static_cast<int>((kdim + kper - 1) / kper);
}

// K partials of the FP64 form from X^T (npad x kdim doubles) through the int8 digit planes.
int syrk_i8(rijk_ctx* ctx, const double* XT, long npad, long nt, long kdim, int nparts, long kper, double* Kpart,
            cudaStream_t s) {
  const long npad2 = round_up(npad, 128);
  const long nblk = (kdim + kChunk - 1) / kChunk;
  const size_t planes = static_cast<size_t>(npad2) * nblk * kBlock;
  int rc;
  if ((rc = ensure(ctx, ctx->Xs, planes, "int8 digit planes")) ||
      (rc = ensure(ctx, ctx->Xe, static_cast<size_t>(nparts) * npad2 * sizeof(int), "digit exponents")))
    return rc;
  int8_t* Xs = static_cast<int8_t*>(ctx->Xs.p);
  int* E = static_cast<int*>(ctx->Xe.p);
  k_slice_x<<<dim3(static_cast<unsigned>(npad2), static_cast<unsigned>(nparts)), kSliceThreads, 0, s>>>(
      XT, npad, npad2, kdim, kper, Xs, E);
  prof_mark(ctx, "slice_x");
  CUtensorMap mA;
  const uint64_t cols = static_cast<uint64_t>(nblk) * kBlock;
  if (!make_map_i8(&mA, Xs, cols, static_cast<uint64_t>(npad2), 128))
    return set_err(ctx, RIJK_ERR_CUDA, "tensor map encoding failed (int8 digits)");
  I8Params ip{};
  ip.kdim = kdim;
  ip.kper = kper;
  ip.npad2 = static_cast<int>(npad2);
  ip.nt = static_cast<int>(nt);
  ip.Kpart = Kpart;
  ip.ntile = nt * (nt + 1) / 2;
  ip.E = E;
  ip.err = static_cast<int*>(ctx->err.p);
  ip.stages = std::min(4, static_cast<int>((kI8SmemBudget - 2048) / kI8Stage));
  const size_t smem = static_cast<size_t>(ip.stages) * kI8Stage + 1024 + 256;
  ensure_smem_limit(reinterpret_cast<const void*>(k_syrk_i8), smem);
  const long nb = npad2 / 128;
  dim3 grid(static_cast<unsigned>(nb * (nb + 1) / 2), static_cast<unsigned>(nparts));
  k_syrk_i8<<<grid, kI8Threads, smem, s>>>(mA, ip);
  return cuda_check(ctx, cudaGetLastError(), "int8 SYRK launch");
}

}  // namespace rijk
