// rijk_noalloc.cu — the Coulomb build with a fixed, library-owned device scratch.
//
// Some callers cannot let the library call cudaMalloc once their iterations are running:
//  - an SCF or CASSCF program that hands all of its GPU memory to its own pool or arena up front;
//  - a program that must not add a device allocation, and the device synchronisation cudaMalloc may
//    bring, inside its iteration loop.
// rijk_coulomb_noalloc serves them.  It computes the Coulomb matrix J from the fitted tensor
// the context already holds (set up earlier, when allocating was still allowed). The caller
// passes the density and the output in device memory. The working space (packed density
// weights, the fitted-coefficient vector w, and the Q-split partial sums) lives in
// g_rijk_noalloc_scratch, a file-scope device array of fixed size.
//
// The scratch array:
//  - holds RIJK_NOALLOC_SCRATCH_BYTES (32 MiB). Every GPU that loads librijk keeps its own copy
//    until the process exits.
//  - is shared by every call on that GPU and keeps the contents of the last call. Every word a
//    call reads is first written by the same call, so nothing needs clearing.
//  - makes two calls that overlap on one GPU (on different streams) race.
//
// Host code cannot pass the array's name to a kernel: on the host it is only a stand-in, not a
// device address.  rijk_create looks the address up with cudaGetSymbolAddress (with the context's
// device current) and keeps it in the context.  With CUDA's lazy module loading that lookup is what
// loads this file's module and allocates the array on the device; the modules of the kernels the call
// launches (density packing, the Coulomb passes, the unpacking) would likewise load, and allocate, on
// their first launch, so rijk_create loads them too.  Both happen at set-up, while allocating is still
// allowed, and never inside rijk_coulomb_noalloc.  A context created after a device reset repeats them.
#include <cuda_runtime.h>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

static constexpr long kNoallocScratchDoubles = RIJK_NOALLOC_SCRATCH_BYTES / static_cast<long>(sizeof(double));

static __device__ __align__(256) double g_rijk_noalloc_scratch[kNoallocScratchDoubles];

namespace rijk {

int noalloc_resolve(rijk_ctx* ctx) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_rijk_noalloc_scratch);
  if (e == cudaSuccess) e = preload_density_kernels();
  if (e == cudaSuccess) e = preload_coulomb_kernels();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? RIJK_ERR_ALLOC : RIJK_ERR_CUDA;
  }
  ctx->noalloc_scratch = static_cast<double*>(p);
  return RIJK_OK;
}

}  // namespace rijk

RIJK_API int rijk_coulomb_noalloc(rijk_ctx* ctx, const double* dDM, double* dJ) {
  using namespace rijk;
  if (!ctx) return RIJK_ERR_ARG;
  if (!dDM || !dJ) return set_err(ctx, RIJK_ERR_ARG, "rijk_coulomb_noalloc: null pointer");
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "rijk_coulomb_noalloc before rijk_set_3c");
  if (!ctx->noalloc_scratch) return set_err(ctx, RIJK_ERR_STATE, "rijk_coulomb_noalloc: no scratch address");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_check(ctx, e, "rijk_coulomb_noalloc: cudaSetDevice");

  const long n = ctx->n, naux = ctx->nq, nt = ctx->nt, npad = ctx->npad, ntile = ctx->ntile;
  const long tile_elems = ntile * TILE2;
  const long nauxr = round_up(naux, 32);  // keeps the partial sums 256-byte aligned
  // scratch = [packed density weights | w | nsplit partial J tiles]
  const long need_min = tile_elems + nauxr + tile_elems;
  if (need_min > kNoallocScratchDoubles)
    return set_err(ctx, RIJK_ERR_ARG,
                   "rijk_coulomb_noalloc: n_ao = %ld, naux = %ld need %ld bytes of scratch; the fixed scratch holds "
                   "%ld bytes (use rijk_fock_device for this size)",
                   n, naux, need_min * static_cast<long>(sizeof(double)), static_cast<long>(RIJK_NOALLOC_SCRATCH_BYTES));
  int nsplit = coulomb_nsplit(tile_elems, naux, 2);
  const long fit = (kNoallocScratchDoubles - tile_elems - nauxr) / tile_elems;
  if (nsplit > fit) nsplit = static_cast<int>(fit);

  double* Dt = ctx->noalloc_scratch;
  double* w = Dt + tile_elems;
  double* Jpart = w + nauxr;

  cudaStream_t s = ctx->stream;
  launch_pack_density(dDM, n, npad, nt, Dt, s);
  launch_coulomb_w(static_cast<const double*>(ctx->B.p), Dt, naux, tile_elems, w, s);
  launch_coulomb_j(static_cast<const double*>(ctx->B.p), w, naux, tile_elems, nsplit, Jpart, s);
  launch_unpack_sym(Jpart, nsplit, ntile, n, dJ, s);
  return cuda_check(ctx, cudaGetLastError(), "rijk_coulomb_noalloc launch");
}
