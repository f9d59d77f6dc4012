// H*psi for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc while they run: a
// Fortran sweep driver whose device memory is owned by its own pool (an
// OpenACC or CUDA-Fortran runtime that hands out slices of one big
// allocation), or a host program that forbids allocation in the middle of a
// solve.  tj_model_wave_noalloc serves them: they pass the operators and both
// wavefunctions in device memory they already own, and every other buffer
// the computation needs -- the hmerge'd operator sums, the phase-1 products
// of the grouped GEMM and the work lists -- lives in one fixed array that
// this file declares in device global memory.  The array is
// TJ_NOALLOC_SCRATCH_BYTES (64 MiB) per GPU and stays resident on every GPU
// that loads the library until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.h"

namespace {

constexpr size_t kScratchDoubles = TJ_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current.  In host code the symbol itself is only a host-side stand-in
// and must never be passed to a kernel.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};

int scratch_address(int dev, double **out) {
  if (dev < 0 || dev >= kMaxDevices) return tjb::set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: device index too large");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return tjb::set_err(TJ_ERR_CUDA, std::string("tj_model_wave_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
    g_addr[dev] = (double *)p;
  }
  *out = g_addr[dev];
  return TJ_OK;
}

inline int64_t up256(int64_t doubles) { return (doubles + 31) / 32 * 32; }   // 256-byte granules

template <class T>
int put(cudaStream_t s, double *base, int64_t &cursor, const std::vector<T> &v, T **dev) {
  *dev = (T *)(base + cursor);
  if (!v.empty()) {
    cudaError_t e = cudaMemcpyAsync(*dev, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return tjb::set_err(TJ_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
  }
  cursor += up256((int64_t)((v.size() * sizeof(T) + sizeof(double) - 1) / sizeof(double)));
  return TJ_OK;
}

bool misaligned(const void *p) { return ((uintptr_t)p & 7u) != 0; }

}  // namespace

extern "C" int tj_model_wave_noalloc(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                                     const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *invec,
                                     tj_wave *outvec, void *stream) {
  using namespace tjb;
  if (!lat || !sys || !env || !sys_bs || !env_bs || !invec || !outvec)
    return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: null argument");
  int rc;
  if ((rc = check_wave(invec)) || (rc = check_wave(outvec))) return rc;
  if (!invec->data || !outvec->data || misaligned(invec->data) || misaligned(outvec->data))
    return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: wave data must be 8-byte aligned device pointers");
  if (!same_layout(invec, outvec))
    return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: outvec must have invec's sector layout");
  {
    // the second GEMM pass reads psi while other tiles already write H*psi:
    // the two vectors must not share memory
    const uintptr_t a0 = (uintptr_t)invec->data, a1 = a0 + sizeof(double) * (uintptr_t)invec->dim;
    const uintptr_t b0 = (uintptr_t)outvec->data, b1 = b0 + sizeof(double) * (uintptr_t)outvec->dim;
    if (invec->dim > 0 && a0 < b1 && b0 < a1)
      return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: invec and outvec data overlap (in-place H*psi is not supported)");
  }
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_err(TJ_ERR_NODEV, "tj_model_wave_noalloc: no CUDA device");
  double *base = nullptr;
  rc = scratch_address(dev, &base);
  if (rc) return rc;

  HpsiPlan P;
  std::string msg;
  rc = build_hpsi_plan(lat, sys, env, sys_bs, env_bs, invec, P, msg);
  if (rc) return set_err(rc, "tj_model_wave_noalloc: " + msg);

  // Operator offsets of the plan are virtual: input blocks first, merged
  // (hmerge) blocks after them.  Input blocks stay where the caller keeps
  // them; merged blocks go to the start of the scratch array.
  int64_t merged0 = P.ops_len;
  for (const auto &m : P.merges) merged0 = std::min(merged0, m.dst);
  // a block whose sub-blocks are all empty has an upload of length 0 at the
  // same offset as the next block's; it is dropped so that the offset search
  // below can only land on the block that holds the offset
  std::vector<HpsiPlan::Upload> ups;
  for (const auto &u : P.uploads)
    if (u.n > 0) {
      if (!u.src || misaligned(u.src))
        return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: operator data must be 8-byte aligned device pointers");
      ups.push_back(u);
    }
  std::sort(ups.begin(), ups.end(), [](const HpsiPlan::Upload &a, const HpsiPlan::Upload &b) { return a.dst < b.dst; });
  bool unmapped = false;
  auto remap = [&](int64_t v) -> int64_t {
    if (v >= merged0) return v - merged0;
    auto it = std::upper_bound(ups.begin(), ups.end(), v,
                               [](int64_t x, const HpsiPlan::Upload &u) { return x < u.dst; });
    if (it == ups.begin() || v >= (it - 1)->dst + (it - 1)->n) {
      unmapped = true;   // not inside any operator block the caller passed
      return 0;
    }
    const HpsiPlan::Upload &u = *(it - 1);
    return (int64_t)(((intptr_t)u.src - (intptr_t)base) / (intptr_t)sizeof(double)) + (v - u.dst);
  };
  for (auto *tv : {&P.tasks1, &P.tasks2})
    for (Task &t : *tv) {
      if (t.L.space == SP_OPS) t.L.off = remap(t.L.off);
      if (t.R.space == SP_OPS) t.R.off = remap(t.R.off);
    }
  std::vector<int64_t> mdst, mn, msrc(P.merge_src);
  std::vector<int32_t> msb, mse;
  for (const auto &m : P.merges) {
    mdst.push_back(remap(m.dst));
    mn.push_back(m.n);
    msb.push_back(m.s_begin);
    mse.push_back(m.s_end);
  }
  for (int64_t &x : msrc) x = remap(x);
  if (unmapped) return set_err(TJ_ERR_ARG, "tj_model_wave_noalloc: an operand lies outside every operator block");

  // scratch layout: merged operators | phase-1 products | partial tiles | work lists | counters
  int64_t cursor = up256(P.ops_len - merged0);
  const int64_t prod_off = cursor;
  cursor += up256(P.scratch_len);
  const int64_t slot_off = cursor;
  cursor += up256(std::max(P.nslots1, P.nslots2) * BM * BN);
  int64_t need = cursor;
  {
    auto b = [](size_t n, size_t sz) { return up256((int64_t)((n * sz + 7) / 8)); };
    need += b(P.cells1.size(), sizeof(Cell)) + b(P.cells2.size(), sizeof(Cell)) + b(P.tasks1.size(), sizeof(Task)) +
            b(P.tasks2.size(), sizeof(Task)) + b(P.tiles1.size(), sizeof(Tile)) + b(P.tiles2.size(), sizeof(Tile)) +
            b(mdst.size(), 8) + b(mn.size(), 8) + b(msb.size(), 4) + b(mse.size(), 4) + b(msrc.size(), 8) +
            b(P.merge_coef.size(), 8) + b(P.red1.size(), sizeof(Reduce)) + b(P.red2.size(), sizeof(Reduce)) + 32;
  }
  if (need > (int64_t)kScratchDoubles) {
    char b[256];
    std::snprintf(b, sizeof b,
                  "tj_model_wave_noalloc: this superblock needs %.1f MiB of scratch, above the fixed %llu MiB "
                  "(use tj_model_wave)",
                  need * 8.0 / (1 << 20), (unsigned long long)(TJ_NOALLOC_SCRATCH_BYTES >> 20));
    return set_err(TJ_ERR_LIMIT, b);
  }
  Cell *c1, *c2;
  Task *t1, *t2;
  Tile *l1, *l2;
  Reduce *r1, *r2;
  int64_t *d_mdst, *d_mn, *d_msrc;
  int32_t *d_msb, *d_mse;
  double *d_mcoef;
  if ((rc = put(s, base, cursor, P.cells1, &c1)) || (rc = put(s, base, cursor, P.cells2, &c2)) ||
      (rc = put(s, base, cursor, P.tasks1, &t1)) || (rc = put(s, base, cursor, P.tasks2, &t2)) ||
      (rc = put(s, base, cursor, P.tiles1, &l1)) || (rc = put(s, base, cursor, P.tiles2, &l2)) ||
      (rc = put(s, base, cursor, mdst, &d_mdst)) || (rc = put(s, base, cursor, mn, &d_mn)) ||
      (rc = put(s, base, cursor, msb, &d_msb)) || (rc = put(s, base, cursor, mse, &d_mse)) ||
      (rc = put(s, base, cursor, msrc, &d_msrc)) || (rc = put(s, base, cursor, P.merge_coef, &d_mcoef)) ||
      (rc = put(s, base, cursor, P.red1, &r1)) || (rc = put(s, base, cursor, P.red2, &r2)))
    return rc;
  // the tile counters must start at zero on every call
  unsigned int *cnt = (unsigned int *)(base + cursor);
  cudaError_t e = cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned int), s);
  if (e != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));

  launch_merge(base, d_mdst, d_mn, d_msb, d_mse, d_msrc, d_mcoef, (int)mdst.size(), s);
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = base;
  g.psi = invec->data;
  g.scr = base + prod_off;
  g.out = base + prod_off;
  g.cells = c1;
  g.tasks = t1;
  g.tiles = l1;
  g.ntiles = (int)P.tiles1.size();
  g.counter = cnt;
  g.slots = base + slot_off;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), s);
  launch_reduce(g, r1, (int)P.red1.size(), s);
  g.out = outvec->data;
  g.cells = c2;
  g.tasks = t2;
  g.tiles = l2;
  g.ntiles = (int)P.tiles2.size();
  g.counter = cnt + 1;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), s);
  launch_reduce(g, r2, (int)P.red2.size(), s);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string("tj_model_wave_noalloc: ") + cudaGetErrorString(e));
  return TJ_OK;
}
