// rijk_cache.cu — the fitted tensor on disk (rijk_save / rijk_load).
//
// The reference rebuilds RI_AA from libint for every run (gen_RI_AA, src/RI.cpp:34-79) and has no
// cache; this keeps the result of rijk_set_basis / rijk_set_3c (the metric factor M and the
// packed fitted tensor B, or an aux slice of it) in one file, so a later process starts its
// Fock builds without integrals or the metric contraction.
//
// File: a fixed header (magic, version, sizes, metric form, aux slice, checksum), then M
// (nauxp x nauxp doubles) and B (nq x ntile x 64 x 64 doubles), little-endian as in memory.
// Device <-> file goes through a pinned 64 MiB staging buffer in two halves, so the copy of one
// half overlaps the file I/O of the other.  The checksum is a 64-bit FNV-1a over the 8-byte words
// of M and B, checked on load before the context is changed.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "gemm_f64.cuh"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

constexpr char kMagic[8] = {'R', 'I', 'J', 'K', 'B', 'C', 'H', '1'};
constexpr int kVersion = 1;
constexpr size_t kStage = 64ull << 20;  // bytes of pinned staging (two halves)

struct Header {
  char magic[8];
  int version;
  int metric_form;
  long n, naux, q0, nq, npad, nt, ntile, nauxp;
  unsigned long long checksum;
  long reserved[6];
};

inline unsigned long long fnv_words(const unsigned long long* w, size_t count, unsigned long long h) {
  for (size_t i = 0; i < count; ++i) {
    h ^= w[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

// Streams `bytes` of device memory at src to the file, folding them into the checksum.  While
// one staging half is written to the file, the other receives the next device copy.
int stream_out(rijk_ctx* ctx, const char* src, size_t bytes, char* stage, FILE* f, unsigned long long& h) {
  const size_t half = kStage / 2;
  cudaStream_t s = ctx->stream;
  size_t done = 0, prev = 0;  // prev: bytes of the completed copy in half (buf ^ 1)
  int buf = 0;
  for (;;) {
    const size_t take = std::min(half, bytes - done);
    if (take) cudaMemcpyAsync(stage + buf * half, src + done, take, cudaMemcpyDeviceToHost, s);
    if (prev) {
      const char* q = stage + (buf ^ 1) * half;
      h = fnv_words(reinterpret_cast<const unsigned long long*>(q), prev / 8, h);
      if (fwrite(q, 1, prev, f) != prev) return set_err(ctx, RIJK_ERR_ARG, "rijk_save: write failed");
    }
    int rc = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_save copy");
    if (rc) return rc;
    if (!take) return RIJK_OK;
    prev = take;
    done += take;
    buf ^= 1;
  }
}

// Reads `bytes` from the file into device memory at dst (dst null: checksum only).  A staging
// half is refilled only after the copy that last read from it has completed (its event).
int stream_in(rijk_ctx* ctx, char* dst, size_t bytes, char* stage, FILE* f, unsigned long long& h) {
  const size_t half = kStage / 2;
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev[2];
  cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  bool used[2] = {false, false};
  int rc = RIJK_OK;
  size_t done = 0;
  int buf = 0;
  while (done < bytes && !rc) {
    const size_t take = std::min(half, bytes - done);
    char* p = stage + buf * half;
    if (used[buf]) rc = cuda_check(ctx, cudaEventSynchronize(ev[buf]), "rijk_load copy");
    if (rc) break;
    if (fread(p, 1, take, f) != take) {
      rc = set_err(ctx, RIJK_ERR_ARG, "rijk_load: file is truncated");
      break;
    }
    h = fnv_words(reinterpret_cast<const unsigned long long*>(p), take / 8, h);
    if (dst) {
      cudaMemcpyAsync(dst + done, p, take, cudaMemcpyHostToDevice, s);
      cudaEventRecord(ev[buf], s);
      used[buf] = true;
    }
    done += take;
    buf ^= 1;
  }
  int rs = cuda_check(ctx, cudaStreamSynchronize(s), "rijk_load copy");
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return rc ? rc : rs;
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_save(rijk_ctx* ctx, const char* path) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!path) return set_err(ctx, RIJK_ERR_ARG, "rijk_save: null path");
  if (!ctx->have_b) return set_err(ctx, RIJK_ERR_STATE, "rijk_save before rijk_set_basis / rijk_set_3c");
  cudaSetDevice(ctx->device);
  Header hd{};
  std::memcpy(hd.magic, kMagic, 8);
  hd.version = kVersion;
  hd.metric_form = ctx->metric_form;
  hd.n = ctx->n;
  hd.naux = ctx->naux;
  hd.q0 = ctx->q0;
  hd.nq = ctx->nq;
  hd.npad = ctx->npad;
  hd.nt = ctx->nt;
  hd.ntile = ctx->ntile;
  hd.nauxp = round_up(ctx->naux, KC);
  const size_t bM = static_cast<size_t>(hd.nauxp) * hd.nauxp * sizeof(double);
  const size_t bB = static_cast<size_t>(hd.nq) * hd.ntile * TILE2 * sizeof(double);
  File f;
  f.f = fopen(path, "wb");
  if (!f.f) return set_err(ctx, RIJK_ERR_ARG, "rijk_save: cannot open %s for writing", path);
  Pinned st;
  int rc = cuda_check(ctx, cudaMallocHost(&st.p, kStage), "rijk_save staging");
  if (rc) return rc;
  if (fwrite(&hd, sizeof hd, 1, f.f) != 1) return set_err(ctx, RIJK_ERR_ARG, "rijk_save: write failed");
  unsigned long long h = 1469598103934665603ull;
  if ((rc = stream_out(ctx, static_cast<const char*>(ctx->M.p), bM, static_cast<char*>(st.p), f.f, h))) return rc;
  if ((rc = stream_out(ctx, static_cast<const char*>(ctx->B.p), bB, static_cast<char*>(st.p), f.f, h))) return rc;
  hd.checksum = h;
  if (fseek(f.f, 0, SEEK_SET) != 0 || fwrite(&hd, sizeof hd, 1, f.f) != 1)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_save: header rewrite failed");
  if (fclose(f.f) != 0) {
    f.f = nullptr;
    return set_err(ctx, RIJK_ERR_ARG, "rijk_save: close failed");
  }
  f.f = nullptr;
  return RIJK_OK;
}

RIJK_API int rijk_load(rijk_ctx* ctx, const char* path) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!path) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: null path");
  cudaSetDevice(ctx->device);
  File f;
  f.f = fopen(path, "rb");
  if (!f.f) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: cannot open %s", path);
  Header hd{};
  if (fread(&hd, sizeof hd, 1, f.f) != 1) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: no header");
  if (std::memcmp(hd.magic, kMagic, 8) != 0 || hd.version != kVersion)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_load: %s is not a fitted-tensor file of this version", path);
  const long npad = round_up(hd.n, TILE), nt = npad / TILE;
  if (hd.n <= 0 || hd.naux <= 0 || hd.naux > 65535 || hd.q0 < 0 || hd.nq <= 0 || hd.q0 + hd.nq > hd.naux ||
      hd.npad != npad || hd.nt != nt || hd.ntile != nt * (nt + 1) / 2 || hd.nauxp != round_up(hd.naux, KC) ||
      (hd.metric_form != RIJK_METRIC_INVSQRT && hd.metric_form != RIJK_METRIC_CHOLESKY))
    return set_err(ctx, RIJK_ERR_ARG, "rijk_load: inconsistent header in %s", path);
  const size_t bM = static_cast<size_t>(hd.nauxp) * hd.nauxp * sizeof(double);
  const size_t bB = static_cast<size_t>(hd.nq) * hd.ntile * TILE2 * sizeof(double);
  Pinned st;
  int rc = cuda_check(ctx, cudaMallocHost(&st.p, kStage), "rijk_load staging");
  if (rc) return rc;
  // first pass: checksum only, so a damaged file leaves the context as it was
  unsigned long long h = 1469598103934665603ull;
  if ((rc = stream_in(ctx, nullptr, bM + bB, static_cast<char*>(st.p), f.f, h))) return rc;
  if (h != hd.checksum) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: checksum mismatch in %s", path);
  if (fseek(f.f, sizeof hd, SEEK_SET) != 0) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: seek failed");
  ctx->have_metric = ctx->have_b = ctx->have_bmix = false;
  release(ctx->Bmix);
  if ((rc = ensure(ctx, ctx->M, bM, "metric M")) || (rc = ensure(ctx, ctx->B, bB, "fitted tensor B"))) return rc;
  h = 1469598103934665603ull;
  if ((rc = stream_in(ctx, static_cast<char*>(ctx->M.p), bM, static_cast<char*>(st.p), f.f, h))) return rc;
  if ((rc = stream_in(ctx, static_cast<char*>(ctx->B.p), bB, static_cast<char*>(st.p), f.f, h))) return rc;
  if (h != hd.checksum) return set_err(ctx, RIJK_ERR_ARG, "rijk_load: %s changed while it was read", path);
  ctx->n = hd.n;
  ctx->naux = hd.naux;
  ctx->q0 = hd.q0;
  ctx->nq = hd.nq;
  ctx->npad = hd.npad;
  ctx->nt = hd.nt;
  ctx->ntile = hd.ntile;
  ctx->metric_form = hd.metric_form;
  ctx->have_metric = ctx->have_b = true;
  ctx->stats.n = hd.n;
  ctx->stats.naux = hd.naux;
  ctx->stats.npad = hd.npad;
  ctx->stats.ntile = hd.ntile;
  ctx->stats.bytes_b = static_cast<long>(bB);
  ctx->stats.bytes_b_mixed = 0;
  return RIJK_OK;
}
