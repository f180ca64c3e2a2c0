// rijk_internal.h — context, device layout and kernel launchers of librijk.
//
// Device layout of the fitted tensor (the reference keeps the raw full square
// RI_AA[(mu*n+nu)*naux+P] in host RAM, src/RI.cpp:69-71; here B already carries the metric
// and only the lower triangle is stored):
//
//   n      orbital functions, npad = n rounded up to TILE (64), nt = npad / TILE
//   tiles  the lower block triangle, tile (I, J) with I >= J at index I(I+1)/2 + J,
//          each a dense TILE x TILE row-major block: element (r, c) is (mu, nu) =
//          (I*TILE + r, J*TILE + c).  Diagonal tiles hold both triangles; padding is zero.
//   B      double [naux][ntile][TILE][TILE]   (Q-major: one aux function's tensor is contiguous)
//
// Exchange intermediate (FP64 form): XT[nu][Q*noccp + i] = sum_mu C_{mu i} B^Q_{mu nu}, the
// half-transformed tensor with the contraction index k = (Q, i) contiguous.
#pragma once
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <functional>
#include <string>

#include "rijk.h"

namespace rijk {

constexpr int TILE = 64;
constexpr int TILE2 = TILE * TILE;

inline long round_up(long x, long m) { return (x + m - 1) / m * m; }

// Device-side error word bits (written by kernels instead of trapping).
constexpr int DEVERR_TIMEOUT = 1;
constexpr int DEVERR_NAN = 2;
constexpr int DEVERR_BOUNDS = 4;

struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// An NVTX range around one C-ABI call, for timeline tools (Nsight Systems); free when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace rijk

struct rijk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  // host-pointer builds (rijk_fock): the orbitals go up and J comes down on a second stream while
  // the Coulomb and exchange kernels run
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_mo = nullptr, ev_j = nullptr;
  // FP64 builds: the Coulomb pair runs on a high-priority stream beside the half-transform, in the
  // registers and shared memory its CTAs leave free on every SM (joined before the build ends)
  cudaStream_t j_stream = nullptr;
  cudaEvent_t ev_pk = nullptr, ev_jside = nullptr;
  int sms = 148;

  long n = 0, naux = 0, npad = 0, nt = 0, ntile = 0;
  long q0 = 0, nq = 0;  // aux functions [q0, q0 + nq) held in B (all of them unless rijk_set_aux_range)
  int metric_form = RIJK_METRIC_INVSQRT;
  bool have_metric = false, have_b = false;
  long grad_qchunk = 0;  // aux functions per chunk of rijk_grad (0: as many as HBM holds)

  rijk::DeviceBuf M;      // metric factor, naux x naux
  rijk::DeviceBuf B;      // fitted tensor, naux x ntile x TILE2 doubles
  rijk::DeviceBuf Bmix;   // split-BF16 copy of B for the mixed form (hi/lo planes)
  bool have_bmix = false;
  rijk::DeviceBuf stageD, stageMO, stageJ, stageK;  // n x n, n_c x n staging for host calls
  rijk::DeviceBuf Dt;     // packed density weights, ntile x TILE2
  rijk::DeviceBuf w;      // naux
  rijk::DeviceBuf Jpart;  // Coulomb partials, nsplit x ntile x TILE2
  rijk::DeviceBuf MOp;    // padded occupied coefficients, noccp x npad
  rijk::DeviceBuf XT;     // half-transformed tensor
  rijk::DeviceBuf Kpart;  // exchange split-K partials
  rijk::DeviceBuf err;    // int device error word
  rijk::DeviceBuf scratch;  // misc small
  rijk::DeviceBuf eri_tab;  // integral tables (Boys grid, harmonics, aux term lists)
  rijk::DeviceBuf Xs;       // int8 digits of X^T for the tensor-core FP64 exchange: npad2 rows of kdim/32
                            // blocks of 8 digits x 32 bytes
  rijk::DeviceBuf Xe;       // their row exponents, parts x npad2
  rijk::DeviceBuf scf[32];  // rijk_scf's work buffers, kept between calls
  double* noalloc_scratch = nullptr;  // device address of rijk_coulomb_noalloc's fixed scratch on `device`
  long fail_alloc_after = -1;  // rijk_selftest_alloc_failure: allocations left before one is refused (-1: off)
  // a device build queued by rijk_fock_device, written to the metrics log by the next rijk_sync
  bool log_pending = false;
  long log_nocc = 0;
  int log_precision = 0;
  // streaming three-centre input (rijk_begin_3c / rijk_add_3c_block) in progress
  struct {
    bool active = false;
    long n = 0, naux = 0;
    int layout = 0;
    long rows_per = 0;  // tile rows per metric-contraction chunk
    long next_mu = 0;   // first orbital row the next block must start at
    long chunk_I0 = 0;  // tile rows [chunk_I0, chunk_I0 + rows_per) fill the staging buffer
    double ms = 0.0;
    rijk::DeviceBuf raw;
  } s3;

  rijk_stats_t stats{};
  std::string last_error;

  // per-kernel timing (rijk_set_profiling)
  bool profiling = false;
  cudaEvent_t pev[13] = {};
  int npev = 0;
  const char* pname[12] = {};
};

namespace rijk {

// Marks the end of one kernel when profiling is on (first call marks the start).
void prof_mark(rijk_ctx* ctx, const char* name);

// ---- rijk_api.cu
int set_err(rijk_ctx* ctx, int code, const char* fmt, ...);
int cuda_check(rijk_ctx* ctx, cudaError_t e, const char* what);
int ensure(rijk_ctx* ctx, DeviceBuf& b, size_t bytes, const char* what);
void release(DeviceBuf& b);
float elapsed(cudaEvent_t a, cudaEvent_t b);
int check_device_error(rijk_ctx* ctx);
// Raises kernel `fn`'s dynamic shared-memory limit to at least `bytes` on the current device.  The
// attribute lives in each device's context, so it is set once per (kernel, device), not once per
// process: a process that drives several GPUs sets it on each.
cudaError_t ensure_smem_limit(const void* fn, size_t bytes);
// The largest shared-memory carveout for fn on the current device (a hint for co-resident CTAs), set
// once per (kernel, device) as above.
void prefer_max_shared(const void* fn);
int check_fock_args(rijk_ctx* ctx, long nocc, int precision);
// One JSON line per Fock build (and per rijk_scf) appended to the file named by the environment
// variable RIJK_LOG, when it is set: the call, sizes, precision, device times, algorithmic FLOPs and
// bytes and the rates they give.  Nothing is written when RIJK_LOG is unset.
void log_build(rijk_ctx* ctx, const char* call, long nocc, int precision);
void log_line(const std::string& json);
// One Fock build on device pointers (J into dJ, K into dK), asynchronous on ctx->stream.  With
// mo_ready the exchange waits for that event (dMO is written on another stream); with j_done the
// event is recorded once J is complete, before the exchange kernels.
int fock_device_impl(rijk_ctx* ctx, const double* dD, const double* dMO, long nocc, double* dJ, double* dK,
                     int precision, cudaEvent_t mo_ready = nullptr, cudaEvent_t j_done = nullptr);
// Metric factor from (P|Q) held in host memory (cudaMemcpyHostToDevice) or device memory.
int set_metric_impl(rijk_ctx* ctx, const double* PQ, cudaMemcpyKind kind, long naux, int form);
// Fitted tensor from three-centre integrals that `fill` writes, one block of tile rows at a time:
// fill(mu0, mu1, first, count, raw, ld) writes the `count` pair rows of functions mu in
// [mu0, mu1) (pair-row index minus `first`, in `layout`) with row pitch ld (>= naux, zero past
// naux) into the device buffer raw.
using ChunkFill = std::function<int(long mu0, long mu1, long first, long count, double* raw, long ld)>;
int set_3c_impl(rijk_ctx* ctx, long n, long naux, int layout, const ChunkFill& fill);
// Tile rows per metric-contraction chunk (raw blocks of at most ~2 GiB) and the pair rows of orbital
// rows [mu0, mu1) in a layout: first pair row and count.
long rows_per_chunk(long n, long nauxp, int layout);
void pair_rows(int layout, long n, long mu0, long mu1, long* first, long* count);
// Abandons a streaming three-centre input in progress (rijk_add_3c_block), freeing its staging.
void stream3c_cancel(rijk_ctx* ctx);

// ---- rijk_noalloc.cu
// Looks up the device address of rijk_coulomb_noalloc's fixed scratch array on ctx->device (which
// must be current) into ctx->noalloc_scratch, and loads the modules of the kernels that call launches.
// The lookup loads the module holding the array, and with it the array itself; a module load is a
// device allocation too.  rijk_create does both while allocating is still allowed.
int noalloc_resolve(rijk_ctx* ctx);

// ---- k_gemm.cu
// C_b = alpha op(A_b) op(B_b) + beta C_b for b < batch (FP64 DMMA, 64 x 64 tiles); see k_gemm.cu for
// the layouts and the GEMM_PAIRS epilogue.  K may be 0 (C = beta C).
constexpr int GEMM_STORE = 0;
constexpr int GEMM_PAIRS = 1;
struct GemmF64Args {
  long M = 0, N = 0, K = 0;
  const double* A = nullptr;
  long lda = 0, sA = 0;
  bool a_kmajor = true;  // A(m, k) = A[m lda + k]; false: A[k lda + m]
  const double* B = nullptr;
  long ldb = 0, sB = 0;
  bool b_kmajor = true;  // B(k, n) = B[n ldb + k]; false: B[k ldb + n]
  double* C = nullptr;
  long ldc = 0, sC = 0;
  double alpha = 1.0, beta = 0.0;
  int mode = GEMM_STORE;
  long n_ao = 0;       // GEMM_PAIRS: orbital functions
  int kdiag = 0;       // 1: k runs over packed-triangle elements, diagonal tiles weighted 1/2
};
void gemm_f64(const GemmF64Args& p, long batch, cudaStream_t s);

// ---- k_pack.cu
// Loads (CUDA loads modules lazily, on a kernel's first use) the density packing and symmetric unpacking
// kernels on the current device.
cudaError_t preload_density_kernels();
void launch_pack_density(const double* D, long n, long npad, long nt, double* Dt, cudaStream_t s);
void launch_pack_mo(const double* MO, long nocc, long n, long noccp, long npad, double* MOp, cudaStream_t s);
// One warp that sleeps for `cycles` SM clock cycles and exits (a fixed delay on a stream).
void launch_delay(long long cycles, cudaStream_t s);
void launch_unpack_sym(double* partial, int nsplit, long ntile, long n, double* out, cudaStream_t s);
void launch_unpack_sym_f32(const float* partial, int nsplit, long ntile, long n, double* sum, double* out,
                           cudaStream_t s);
void launch_scan_nonfinite(const double* x, long count, int* err, cudaStream_t s);

// ---- k_metric.cu
// B[Q][tile-packed e] = sum_P M[Q][P] * I3(pair(e), P) for the raw rows of tile rows [I0, I1).
// M may start at a row offset q0 (mrows = rows left after it); B receives naux rows.  tri >= 0 declares
// M lower triangular with its first row at global row tri (the Cholesky form): the contraction then
// stops at each row block's last nonzero column, half the products, the same result.
void launch_metric_contract_chunk(const double* M, long nauxp, long mrows, const double* I3, int layout, long n,
                                  long naux, long nt, long I0, long I1, double* B, cudaStream_t s, long tri = -1);

// ---- k_coulomb.cu
// Loads the FP64 Coulomb kernels' module on the current device (see preload_density_kernels).
cudaError_t preload_coulomb_kernels();
// Q splits of the J pass: elems_per_thread = 2 (FP64 B, double2) or 8 (split-BF16 copy).
int coulomb_nsplit(long tile_elems, long naux, int elems_per_thread);
// Octet chunks of the mixed w pass; its w buffer holds (1 + chunks) * naux doubles.
int coulomb_w_mixed_chunks(long ntile);
// max_ctas > 0 caps the grid (the kernels stride over the rest), for the pair run beside the half-transform
void launch_coulomb_w(const double* B, const double* Dt, long naux, long tile_elems, double* w, cudaStream_t s,
                      int max_ctas = 0);
void launch_coulomb_j(const double* B, const double* w, long naux, long tile_elems, int nsplit, double* Jpart,
                      cudaStream_t s, int max_ctas = 0);

// Mixed form: the same passes over the split-BF16 copy (Bmix[Q][t][hl][64][64], ntile2 tiles per Q).
void launch_coulomb_w_mixed(const __nv_bfloat16* Bmix, const double* Dt, long naux, long ntile, long ntile2, double* w,
                            cudaStream_t s);
void launch_coulomb_j_mixed(const __nv_bfloat16* Bmix, const double* w, long naux, long ntile, long ntile2,
                            int nsplit, double* Jpart, cudaStream_t s);

// ---- k_exchange_f64.cu
// Returns the number of kernel launches it made (one, or two when a smaller last orbital batch remains).
int launch_xform_f64(const double* B, const double* MOp, long naux, long nt, long noccp, double* XT, cudaStream_t s);
int syrk_nsplit(long nt, long kdim);
void launch_syrk_f64(const double* XT, long npad, long nt, long kdim, int nsplit, double* Kpart, cudaStream_t s);

// ---- k_exchange_i8.cu (RIJK_PREC_FP64_TC): K partials from int8 digit planes on tcgen05
int syrk_i8_parts(long nt, long kdim, int device, long* kper);
int syrk_i8(rijk_ctx* ctx, const double* XT, long npad, long nt, long kdim, int nparts, long kper, double* Kpart,
            cudaStream_t s);

}  // namespace rijk
