// Device-resident copies of the blocks the library writes into caller
// memory.
//
// A sweep hands every block that tj_get_hamiltonian returns straight back to
// the library: as the system or environment of the next Lanczos calls and as
// the old block of a later renormalisation.  Each of those calls uploads the
// block's operators from the caller's (pageable) arrays -- tens of MB per
// step at m = 2000, more than the GEMMs of the step take.  With residency on
// (tj_set_residency), tj_get_hamiltonian keeps the device copy of the block
// it has just written, keyed by the caller's array, and every later upload
// whose source lies inside a kept array is a device-to-device copy instead.
//
// The caller's side of the contract: an array the library filled is not
// modified while it is kept (tj_residency_forget drops it first; freeing and
// reusing the memory for other data needs the same).  As a guard, each entry
// remembers a fingerprint of 64 values spread over the array, checked at
// every use; an entry whose fingerprint no longer matches is dropped and the
// upload goes to the host array.  Entries beyond the byte budget are dropped
// least recently used first.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "ctx.h"

namespace tjb {

namespace {

uint64_t fingerprint(const double *p, int64_t n) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)n;
  const int64_t k = n < 64 ? n : 64;
  for (int64_t i = 0; i < k; ++i) {
    const int64_t at = k > 1 ? i * (n - 1) / (k - 1) : 0;
    uint64_t u;
    std::memcpy(&u, p + at, 8);
    h = (h ^ u) * 1099511628211ull;
  }
  return h;
}

void drop(tj_ctx *ctx, size_t i) {
  ResEntry &e = ctx->resident[i];
  if (e.dev) cudaFree(e.dev);
  ctx->res_bytes -= (size_t)e.n * 8;
  ctx->resident.erase(ctx->resident.begin() + (long)i);
}

}  // namespace

const double *res_find(tj_ctx *ctx, const double *p, int64_t n) {
  if (ctx->res_budget == 0 || n <= 0) return nullptr;
  for (size_t i = 0; i < ctx->resident.size(); ++i) {
    ResEntry &e = ctx->resident[i];
    if (p < e.host || p + n > e.host + e.n) continue;
    if (fingerprint(e.host, e.n) != e.sample) {
      drop(ctx, i);
      return nullptr;
    }
    e.stamp = ++ctx->res_clock;
    ++ctx->res_hits;
    ctx->res_hit_bytes += 8.0 * (double)n;
    return e.dev + (p - e.host);
  }
  return nullptr;
}

int res_keep(tj_ctx *ctx, const double *host, int64_t n, const double *dev_src, cudaStream_t st) {
  if (ctx->res_budget == 0 || n <= 0) return TJ_OK;
  const size_t bytes = (size_t)n * 8;
  if (bytes > ctx->res_budget) return TJ_OK;
  for (size_t i = 0; i < ctx->resident.size();) {   // entries the new array overlaps are stale
    const ResEntry &e = ctx->resident[i];
    if (e.host < host + n && host < e.host + e.n)
      drop(ctx, i);
    else
      ++i;
  }
  while (ctx->res_bytes + bytes > ctx->res_budget && !ctx->resident.empty()) {
    size_t lru = 0;
    for (size_t i = 1; i < ctx->resident.size(); ++i)
      if (ctx->resident[i].stamp < ctx->resident[lru].stamp) lru = i;
    drop(ctx, lru);
  }
  ResEntry e;
  e.host = host;
  e.n = n;
  if (cudaMalloc((void **)&e.dev, bytes) != cudaSuccess) {
    cudaGetLastError();
    return TJ_OK;   // no room: the block stays host-only
  }
  cudaError_t rc = cudaMemcpyAsync(e.dev, dev_src, bytes, cudaMemcpyDeviceToDevice, st);
  if (rc != cudaSuccess) {
    cudaFree(e.dev);
    return set_err(TJ_ERR_CUDA, std::string("residency copy: ") + cudaGetErrorString(rc));
  }
  e.sample = fingerprint(host, n);
  e.stamp = ++ctx->res_clock;
  ctx->resident.push_back(e);
  ctx->res_bytes += bytes;
  return TJ_OK;
}

void res_clear(tj_ctx *ctx) {
  while (!ctx->resident.empty()) drop(ctx, ctx->resident.size() - 1);
}

cudaError_t upload(tj_ctx *ctx, double *dst, const double *src, int64_t n, cudaStream_t st) {
  const double *d = res_find(ctx, src, n);
  return cudaMemcpyAsync(dst, d ? d : src, sizeof(double) * n, d ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         st);
}

}  // namespace tjb

extern "C" int tj_set_residency(tj_ctx *ctx, double gigabytes) {
  if (!ctx) return tjb::set_err(TJ_ERR_ARG, "tj_set_residency: null context");
  if (!(gigabytes >= 0.0)) return tjb::set_err(TJ_ERR_ARG, "tj_set_residency: negative budget");
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->res_budget = (size_t)(gigabytes * 1e9);
  if (ctx->res_bytes > ctx->res_budget) tjb::res_clear(ctx);
  return TJ_OK;
}

extern "C" int tj_residency_forget(tj_ctx *ctx, const void *host) {
  if (!ctx) return tjb::set_err(TJ_ERR_ARG, "tj_residency_forget: null context");
  const double *p = (const double *)host;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (size_t i = 0; i < ctx->resident.size();) {
    const tjb::ResEntry &e = ctx->resident[i];
    if (p >= e.host && p < e.host + e.n) {
      if (e.dev) cudaFree(e.dev);
      ctx->res_bytes -= (size_t)e.n * 8;
      ctx->resident.erase(ctx->resident.begin() + (long)i);
    } else {
      ++i;
    }
  }
  return TJ_OK;
}
