// k_exchange_f64.cu — FP64 exchange: half-transform (K3) and K contraction (K4).
//
// Reference (src/RI.cpp:146-171): RI_CA = MO . RI_AA (i, nu, P), RI_CA2 = RI_CA . V^-1/2,
// transpose to (nu, i, P), K = RI_CA RI_CA^T over (i, P).  With the metric folded into B:
//
//   K3  XT[nu][Q*noccp + i] = sum_mu B^Q_{nu mu} C_{i mu}
//       one CTA per (nu-block J, Q); the mu loop walks the stored tiles (J, I) for I <= J
//       and the transposes of (I, J) for I > J, so B's packed triangle is read as the full
//       symmetric matrix without unpacking.
//   K4  K[mu][nu] = sum_k XT[mu][k] XT[nu][k], k = (Q, i): only the lower tiles (a >= b)
//       are formed, split over k into nsplit ranges whose partial tiles are summed (and
//       mirrored) by the unpack kernel.  FLOPs n(n+1) noccp naux, the SYRK count.
#include <algorithm>
#include <atomic>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

namespace rijk {

constexpr int X_THREADS = 128;

// The half-transform's [row][k] chunks (the K-major tiles of B^Q and the orbitals) without padding: the
// 8-byte words of a row are XOR-swizzled, (row, k) at row * 32 + (k ^ 4 (row & 3)).  A half-warp reads
// rows g = 0..3 (or 4..7) at k + t, t = 0..3, and the swizzle spreads those over 16 distinct words mod 16,
// as the padded stride 36 did.  Every fragment row is g plus a multiple of 4, so the swizzle is one
// per-lane constant: (k + t) ^ 4 (g & 3) = (k ^ 4 (g & 3)) + t.  The XOR keeps pairs of words together,
// so each 16-byte copy stays whole and aligned.  The [k][row] chunks keep the padded stride 68.
// 74 KB of stages a CTA at 80 orbitals instead of 81 KB: three CTAs share an SM instead of two.
constexpr int XK = 32;  // [row][k] row length
__device__ __forceinline__ int swk(int row, int k) { return row * XK + (k ^ ((row & 3) << 2)); }

// warp_mma_chunk with the swizzled [row][k] chunks; m0 and n0 are multiples of 4
template <int MF, int NF, bool A_KMAJOR>
__device__ __forceinline__ void warp_mma_chunk_sw(double (&acc)[MF][NF][2], const double* __restrict__ sA,
                                                  const double* __restrict__ sB, int m0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int sg = (g & 3) << 2;
  const double* pa = A_KMAJOR ? sA + (m0 + g) * XK + t : sA + t * LDM + m0 + g;
  const double* pb = sB + (n0 + g) * XK + t;
#pragma unroll
  for (int k = 0; k < KC; k += 4) {
    const int kx = k ^ sg;
    double a[MF], b[NF];
#pragma unroll
    for (int i = 0; i < MF; ++i) a[i] = A_KMAJOR ? pa[i * 8 * XK + kx] : pa[k * LDM + i * 8];
#pragma unroll
    for (int j = 0; j < NF; ++j) b[j] = pb[j * 8 * XK + kx];
#pragma unroll
    for (int i = 0; i < MF; ++i)
#pragma unroll
      for (int j = 0; j < NF; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  }
}

// Grid (nb * nt, naux): block x = J nb + b handles orbital batch b (rows i0 + b NOCCP of MOp) of tile
// column J, so the nb batches of one (J, Q) run back to back and the later ones read the tiles of B^Q
// from L2.
template <int NF>
__global__ void __launch_bounds__(X_THREADS)
    k_xform_f64(const double* __restrict__ B, const double* __restrict__ MOp_all, long nt, long npad, long tile_elems,
                long kdim, long noccp_total, long i0_first, int nb, double* __restrict__ XT) {
  constexpr int NOCCP = NF * 16;
  constexpr int A_STAGE = (64 * XK > KC * LDM) ? 64 * XK : KC * LDM;
  constexpr int B_STAGE = NOCCP * XK;
  static_assert(KC == XK, "chunk shape");
  extern __shared__ __align__(16) double smem[];
  double* sA[2] = {smem, smem + A_STAGE};
  double* sB[2] = {smem + 2 * A_STAGE, smem + 2 * A_STAGE + B_STAGE};

  const long J = blockIdx.x / nb;
  const long i0 = i0_first + static_cast<long>(blockIdx.x % nb) * NOCCP;
  const double* MOp = MOp_all + i0 * npad;
  const long Q = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const double* BQ = B + Q * tile_elems;

  auto load = [&](int stage, long kc) {
    const long I = kc >> 1;
    const int half = static_cast<int>(kc & 1);
    if (J >= I) {  // tile (J, I): rows nu, cols mu -> [nu][mu-chunk]
      const double* tp = BQ + tri_index(J, I) * TILE2 + half * KC;
#pragma unroll
      for (int it = 0; it < 8; ++it) {
        int idx = tid + it * X_THREADS;
        int row = idx >> 4, seg = idx & 15;
        cp_async16(&sA[stage][swk(row, seg * 2)], tp + row * TILE + seg * 2, true);
      }
    } else {  // tile (I, J): rows mu, cols nu -> [mu-chunk][nu]
      const double* tp = BQ + tri_index(I, J) * TILE2 + half * KC * TILE;
#pragma unroll
      for (int it = 0; it < 8; ++it) {
        int idx = tid + it * X_THREADS;
        int row = idx >> 5, seg = idx & 31;
        cp_async16(&sA[stage][row * LDM + seg * 2], tp + row * TILE + seg * 2, true);
      }
    }
    const double* cp = MOp + I * TILE + half * KC;
    for (int idx = tid; idx < NOCCP * 16; idx += X_THREADS) {
      int row = idx >> 4, seg = idx & 15;
      cp_async16(&sB[stage][swk(row, seg * 2)], cp + row * npad + seg * 2, true);
    }
  };

  double acc[4][NF][2];
  zero_acc(acc);
  const long nk = nt * 2;
  load(0, 0);
  cp_async_commit();
  for (long kc = 0; kc < nk; ++kc) {
    if (kc + 1 < nk) {
      load(static_cast<int>((kc + 1) & 1), kc + 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (J >= (kc >> 1))
      warp_mma_chunk_sw<4, NF, true>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * (NOCCP / 2), lane);
    else
      warp_mma_chunk_sw<4, NF, false>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * (NOCCP / 2), lane);
    __syncthreads();
  }

  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    long nu = J * TILE + wm * 32 + i * 8 + g;
    double* row = XT + nu * kdim + Q * noccp_total + i0 + wn * (NOCCP / 2);
#pragma unroll
    for (int j = 0; j < NF; ++j)
      *reinterpret_cast<double2*>(row + j * 8 + 2 * tq) = make_double2(acc[i][j][0], acc[i][j][1]);
  }
}

// nb orbital batches of NF*16 rows from row i0 of MOp into columns Q*noccp_total + i0 + ... of XT.
template <int NF>
static void launch_xform_nf(const double* B, const double* MOp, long naux, long nt, long noccp_total, long i0, int nb,
                            double* XT, cudaStream_t s) {
  constexpr int NOCCP = NF * 16;
  constexpr int A_STAGE = (64 * XK > KC * LDM) ? 64 * XK : KC * LDM;
  size_t smem = (2 * A_STAGE + 2 * NOCCP * XK) * sizeof(double);
  ensure_smem_limit(reinterpret_cast<const void*>(k_xform_f64<NF>), smem);
  prefer_max_shared(reinterpret_cast<const void*>(k_xform_f64<NF>));  // room for three CTAs an SM
  long npad = nt * TILE;
  long tile_elems = nt * (nt + 1) / 2 * TILE2;
  dim3 grid(static_cast<unsigned>(nt * nb), static_cast<unsigned>(naux));
  k_xform_f64<NF><<<grid, X_THREADS, smem, s>>>(B, MOp, nt, npad, tile_elems, naux * noccp_total, noccp_total, i0, nb,
                                                 XT);
}

static void launch_xform_batches(int nf, const double* B, const double* MOp, long naux, long nt, long noccp, long i0,
                                 int nb, double* XT, cudaStream_t s) {
  switch (nf) {
    case 1: launch_xform_nf<1>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    case 2: launch_xform_nf<2>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    case 3: launch_xform_nf<3>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    case 4: launch_xform_nf<4>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    case 5: launch_xform_nf<5>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    case 6: launch_xform_nf<6>(B, MOp, naux, nt, noccp, i0, nb, XT, s); break;
    default: break;
  }
}

// The orbitals go in batches of at most 96 (NF <= 6 keeps the accumulators in registers).  The
// full-size batches run in one launch (each tile column's batches back to back, B^Q read once from
// HBM); a smaller last batch gets a launch of its own.
int launch_xform_f64(const double* B, const double* MOp, long naux, long nt, long noccp, double* XT, cudaStream_t s) {
  const long nbatch = (noccp + 95) / 96;
  const long per = round_up((noccp + nbatch - 1) / nbatch, 16);
  const long nfull = noccp / per, rest = noccp - nfull * per;
  if (nfull > 0) launch_xform_batches(static_cast<int>(per / 16), B, MOp, naux, nt, noccp, 0, static_cast<int>(nfull), XT, s);
  if (rest > 0) launch_xform_batches(static_cast<int>(rest / 16), B, MOp, naux, nt, noccp, nfull * per, 1, XT, s);
  return (nfull > 0 ? 1 : 0) + (rest > 0 ? 1 : 0);
}

constexpr int S_THREADS = 128;

__global__ void __launch_bounds__(S_THREADS)
    k_syrk_f64(const double* __restrict__ XT, long kdim, long kper, long ntile, double* __restrict__ Kpart) {
  extern __shared__ __align__(16) double smem_s[];
  double* sA[2] = {smem_s, smem_s + 64 * LDK};
  double* sB[2] = {smem_s + 2 * 64 * LDK, smem_s + 3 * 64 * LDK};
  const long t = blockIdx.x;
  const long s = blockIdx.y;
  long a, b;
  tri_decode(t, a, b);
  const long k0 = s * kper;
  const long k1 = k0 + kper < kdim ? k0 + kper : kdim;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const double* Ar = XT + a * TILE * kdim;
  const double* Br = XT + b * TILE * kdim;

  auto load = [&](int stage, long kk) {
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      int idx = tid + it * S_THREADS;
      int row = idx >> 4, seg = idx & 15;
      long k = kk + seg * 2;
      bool ok = k < k1;
      cp_async16(&sA[stage][row * LDK + seg * 2], ok ? Ar + row * kdim + k : XT, ok);
      cp_async16(&sB[stage][row * LDK + seg * 2], ok ? Br + row * kdim + k : XT, ok);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  const long nk = k1 > k0 ? (k1 - k0 + KC - 1) / KC : 0;
  if (nk > 0) {
    load(0, k0);
    cp_async_commit();
  }
  for (long kc = 0; kc < nk; ++kc) {
    if (kc + 1 < nk) {
      load(static_cast<int>((kc + 1) & 1), k0 + (kc + 1) * KC);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    warp_mma_chunk<4, 4, true>(acc, sA[kc & 1], sB[kc & 1], wm * 32, wn * 32, lane);
    __syncthreads();
  }
  const int g = lane >> 2, tq = lane & 3;
  double* out = Kpart + (s * ntile + t) * TILE2;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int r = wm * 32 + i * 8 + g;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int c = wn * 32 + j * 8 + 2 * tq;
      *reinterpret_cast<double2*>(out + r * TILE + c) = make_double2(acc[i][j][0], acc[i][j][1]);
    }
  }
}

namespace {
constexpr size_t kSyrkSmem = 4 * 64 * LDK * sizeof(double);

// CTAs of k_syrk_f64 resident per SM (registers and shared memory), from the runtime.
int syrk_ctas_per_sm() {
  static std::atomic<int> slots[64] = {};  // contexts on other host threads may ask at once
  int dev = 0;
  cudaGetDevice(&dev);
  ensure_smem_limit(reinterpret_cast<const void*>(k_syrk_f64), kSyrkSmem);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!slots[dev]) {
    int nb = 0, sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_syrk_f64, S_THREADS, kSyrkSmem) != cudaSuccess || nb < 1)
      nb = 2;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    slots[dev] = nb * sms;  // slots of one wave
  }
  return slots[dev];
}
}  // namespace

// Splits of the contraction range: enough CTAs for about two waves of the kernel's resident
// slots (CTAs per SM x SMs), chosen among [s_min, 4 s_min] so the last wave is fullest.
int syrk_nsplit(long nt, long kdim) {
  const long ntile = nt * (nt + 1) / 2;
  const long slots = syrk_ctas_per_sm();
  const long maxs = std::max<long>(1, kdim / (KC * 8));
  const long need = slots * 19 / 10;
  const long smin = std::min(maxs, std::max<long>(1, (need + ntile - 1) / ntile));
  long best = smin;
  double best_eff = 0.0;
  for (long sp = smin; sp <= std::min(maxs, 4 * smin); ++sp) {
    const long ctas = ntile * sp;
    const long waves = (ctas + slots - 1) / slots;
    const double eff = static_cast<double>(ctas) / static_cast<double>(waves * slots);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = sp;
    }
  }
  return static_cast<int>(best);
}

void launch_syrk_f64(const double* XT, long npad, long nt, long kdim, int nsplit, double* Kpart, cudaStream_t s) {
  (void)npad;
  long ntile = nt * (nt + 1) / 2;
  long kper = round_up((kdim + nsplit - 1) / nsplit, KC);
  dim3 grid(static_cast<unsigned>(ntile), static_cast<unsigned>(nsplit));
  syrk_ctas_per_sm();  // sets the shared-memory attribute once
  k_syrk_f64<<<grid, S_THREADS, kSyrkSmem, s>>>(XT, kdim, kper, ntile, Kpart);
}

}  // namespace rijk
