// Device-resident copies of the blocks the library writes into caller
// memory.
//
// A sweep hands every block that tj_get_hamiltonian returns straight back to
// the library: as the system or environment of the next Lanczos calls and as
// the old block of a later renormalisation.  Each of those calls uploads the
// block's operators from the caller's (pageable) arrays -- tens of MB per
// step at m = 2000, more than the GEMMs of the step take.  With residency on
// (tj_set_residency), tj_get_hamiltonian keeps the device copy of the block
// it has just written, keyed by the caller's array (and tj_lanczos_memo_new
// and tj_wave_trans their wavefunctions, which the next truncation,
// prediction and Lanczos read, and tj_truncation its operator, which the
// step's renormalisation and the next step's prediction read), and every
// later upload whose source lies inside a kept array is a device-to-device
// copy instead.
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
#include <iterator>
#include <string>
#include <thread>
#include <vector>

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

// Kept arrays are carved out of large device slabs (4 GB, or the array's
// size if larger) by a first-fit allocator with coalescing free lists:
// cudaMalloc runs once per slab, not once per block (growing a memory pool
// per block cost more than the step's GEMMs).  All uses of kept memory are on
// the context's stream, so memory freed here and handed out again is only
// written after the earlier reads have run.
constexpr size_t SLAB = (size_t)4 << 30;

double *arena_alloc(tj_ctx *ctx, size_t bytes) {
  bytes = (bytes + 255) / 256 * 256;
  ResArena &A = ctx->arena;
  for (auto it = A.free.begin(); it != A.free.end(); ++it) {
    if (it->second.size < bytes) continue;
    char *p = it->first;
    const ResArena::Free f = it->second;
    A.free.erase(it);
    if (f.size > bytes) A.free[p + bytes] = ResArena::Free{f.size - bytes, f.slab};
    A.owner[p] = ResArena::Free{bytes, f.slab};
    return (double *)p;
  }
  const size_t sz = bytes > SLAB ? bytes : SLAB;
  char *slab = nullptr;
  if (cudaMalloc((void **)&slab, sz) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const int id = (int)A.slabs.size();
  A.slabs.push_back(slab);
  if (sz > bytes) A.free[slab + bytes] = ResArena::Free{sz - bytes, id};
  A.owner[slab] = ResArena::Free{bytes, id};
  return (double *)slab;
}

void arena_free(tj_ctx *ctx, double *ptr) {
  ResArena &A = ctx->arena;
  auto o = A.owner.find((char *)ptr);
  if (o == A.owner.end()) return;
  char *p = o->first;
  ResArena::Free f = o->second;
  A.owner.erase(o);
  auto next = A.free.lower_bound(p);
  if (next != A.free.end() && next->first == p + f.size && next->second.slab == f.slab) {
    f.size += next->second.size;
    next = A.free.erase(next);
  }
  if (next != A.free.begin()) {
    auto prev = std::prev(next);
    if (prev->first + prev->second.size == p && prev->second.slab == f.slab) {
      prev->second.size += f.size;
      return;
    }
  }
  A.free[p] = f;
}

void arena_release(tj_ctx *ctx) {
  ResArena &A = ctx->arena;
  if (A.slabs.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (char *s : A.slabs) cudaFree(s);
  A.slabs.clear();
  A.free.clear();
  A.owner.clear();
}

void drop(tj_ctx *ctx, size_t i) {
  ResEntry &e = ctx->resident[i];
  if (e.dev) arena_free(ctx, e.dev);
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
  e.dev = arena_alloc(ctx, bytes);
  if (!e.dev) return TJ_OK;   // no room: the block stays host-only
  cudaError_t rc = cudaMemcpyAsync(e.dev, dev_src, bytes, cudaMemcpyDeviceToDevice, st);
  if (rc != cudaSuccess) {
    arena_free(ctx, e.dev);
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
  arena_release(ctx);
}

cudaError_t upload(tj_ctx *ctx, double *dst, const double *src, int64_t n, cudaStream_t st) {
  const double *d = res_find(ctx, src, n);
  return cudaMemcpyAsync(dst, d ? d : src, sizeof(double) * n, d ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         st);
}

// Device-to-host copy into caller (pageable) memory through two page-locked
// staging chunks: the DMA of chunk c runs while chunk c - 1 is copied out on
// the host by several threads.  A copy straight into pageable memory runs
// at a fraction of the DMA rate, and slower still into pages never touched
// (each first touch is a page fault inside the copy); a page-locked
// destination is written directly.  Returns when dst is filled.
int download(tj_ctx *ctx, double *dst, const double *src, int64_t n, cudaStream_t st) {
  const size_t chunk = (size_t)8 << 20;
  const size_t bytes = (size_t)n * 8;
  cudaPointerAttributes pa;
  const bool locked = cudaPointerGetAttributes(&pa, dst) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (locked || bytes <= ((size_t)1 << 20)) {   // page-locked memory takes the DMA directly
    if (n > 0 && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return set_err(TJ_ERR_CUDA, "download: copy failed");
    if (cudaStreamSynchronize(st) != cudaSuccess) return set_err(TJ_ERR_CUDA, "download: stream failed");
    return TJ_OK;
  }
  if (!ctx->stage) {
    if (cudaMallocHost((void **)&ctx->stage, 2 * chunk) != cudaSuccess) {
      ctx->stage = nullptr;
      return set_err(TJ_ERR_CUDA, "download: no page-locked staging memory");
    }
    for (auto &e : ctx->sev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        return set_err(TJ_ERR_CUDA, "download: event creation failed");
  }
  char *stage = (char *)ctx->stage;
  const char *s = (const char *)src;
  char *d = (char *)dst;
  const size_t nch = (bytes + chunk - 1) / chunk;
  auto host_copy = [&](char *to, const char *from, size_t len) {
    const size_t T = len >= ((size_t)4 << 20) ? 4 : 1;
    if (T == 1) {
      std::memcpy(to, from, len);
      return;
    }
    std::vector<std::thread> th;
    const size_t part = (len / T + 4095) / 4096 * 4096;
    for (size_t t = 1; t < T; ++t) {
      const size_t a = t * part;
      if (a >= len) break;
      th.emplace_back([=] { std::memcpy(to + a, from + a, std::min(part, len - a)); });
    }
    std::memcpy(to, from, std::min(part, len));
    for (auto &x : th) x.join();
  };
  for (size_t c = 0; c <= nch; ++c) {
    if (c < nch) {
      const size_t off = c * chunk, len = std::min(chunk, bytes - off);
      if (cudaMemcpyAsync(stage + (c & 1) * chunk, s + off, len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaEventRecord(ctx->sev[c & 1], st) != cudaSuccess)
        return set_err(TJ_ERR_CUDA, "download: copy failed");
    }
    if (c > 0) {
      const size_t p = c - 1, off = p * chunk, len = std::min(chunk, bytes - off);
      if (cudaEventSynchronize(ctx->sev[p & 1]) != cudaSuccess) return set_err(TJ_ERR_CUDA, "download: copy failed");
      host_copy(d + off, stage + (p & 1) * chunk, len);
    }
  }
  return TJ_OK;
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
  for (size_t i = 0; i < ctx->resident.size();) {
    const tjb::ResEntry &e = ctx->resident[i];
    if (p >= e.host && p < e.host + e.n) {
      if (e.dev) tjb::arena_free(ctx, e.dev);
      ctx->res_bytes -= (size_t)e.n * 8;
      ctx->resident.erase(ctx->resident.begin() + (long)i);
    } else {
      ++i;
    }
  }
  return TJ_OK;
}
