// Autotuner of the grouped GEMMs: picks the tiling and schedule choices of
// TuneParams per block-size histogram of an H*psi plan by timing H*psi with
// each candidate on the device, and keeps the result in a process-wide table.
//
// Search: coordinate descent from the defaults over the knobs of the
// context's precision mode; a candidate replaces the current best when it is
// at least 2 % faster (so that timing noise does not move the choice).
//   FP64            items_per_cta {3, 6, 12}, min_ksteps {128, 256, 512},
//                   ctas_per_sm {2, 3, 4}
//   split precision oz_bn {48, 32} (5 slices), oz_item_cost {2, 4, 8}
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.h"

namespace tjb {

namespace {
std::mutex g_tune_mu;
std::map<uint64_t, TuneParams> g_tuned;

int ilog2(int64_t x) {
  int r = 0;
  while (x > 1) {
    x >>= 1;
    ++r;
  }
  return r;
}
}  // namespace

uint64_t plan_hist_key(const HpsiPlan &P, int prec_mode, int slices) {
  std::map<uint32_t, int64_t> hist;
  auto count = [&](const std::vector<Cell> &cells, const std::vector<Task> &tasks) {
    for (const Cell &c : cells)
      for (int t = c.t_begin; t < c.t_end; ++t) {
        if (tasks[t].R.space == SP_NONE) continue;
        const uint32_t b = (uint32_t)ilog2(c.M) | ((uint32_t)ilog2(c.N) << 8) | ((uint32_t)ilog2(tasks[t].K) << 16);
        ++hist[b];
      }
  };
  count(P.cells1, P.tasks1);
  count(P.cells2, P.tasks2);
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    for (int i = 0; i < 8; ++i) {
      h ^= (v >> (8 * i)) & 0xFF;
      h *= 1099511628211ull;
    }
  };
  mix((uint64_t)prec_mode);
  mix((uint64_t)(prec_mode == TJ_PREC_OZAKI ? slices : 0));
  for (const auto &kv : hist) {
    mix(kv.first);
    mix((uint64_t)kv.second);
  }
  return h;
}

bool tune_lookup(uint64_t key, TuneParams &tp) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tuned.find(key);
  if (it == g_tuned.end()) return false;
  tp = it->second;
  return true;
}

void tune_store(uint64_t key, const TuneParams &tp) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tuned[key] = tp;
}

bool tune_is_current(tj_ctx *ctx) {
  TuneParams want = ctx->tune;
  if (!ctx->tuning && ctx->autotune != TJ_TUNE_OFF) tune_lookup(ctx->hist_key, want);
  return want == ctx->plan_tune;
}

int autotune_plan(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                  const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, tj_tune_result *out) {
  struct Flag {
    tj_ctx *c;
    ~Flag() { c->tuning = false; }
  } flag{ctx};
  ctx->tuning = true;
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t D = wave->dim;
  int rc;
  if ((rc = ctx->vin.reserve(sizeof(double) * (D + 4))) || (rc = ctx->vout.reserve(sizeof(double) * (D + 4))))
    return rc;
  if (cudaMemcpyAsync(ctx->vin.d(), wave->data, sizeof(double) * D, cudaMemcpyHostToDevice, ctx->stream) !=
      cudaSuccess)
    return set_err(TJ_ERR_CUDA, "autotune: input upload failed");
  int evaluated = 0;
  // device time of one H*psi with the given choices (the plan is rebuilt with them)
  auto measure = [&](const TuneParams &tp, double &ms) -> int {
    ctx->tune = tp;
    ctx->plan_valid = false;
    int r = prepare_hpsi(ctx, lat, sys, env, sys_bs, env_bs, wave);
    if (r) return r;
    for (int i = 0; i < 2; ++i)
      if ((r = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), false))) return r;
    const int reps = 5;
    if (cudaEventRecord(ctx->ev[5], ctx->stream) != cudaSuccess) return set_err(TJ_ERR_CUDA, "autotune: event");
    for (int i = 0; i < reps; ++i)
      if ((r = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), false))) return r;
    if (cudaEventRecord(ctx->ev[0], ctx->stream) != cudaSuccess || cudaEventSynchronize(ctx->ev[0]) != cudaSuccess)
      return set_err(TJ_ERR_CUDA, "autotune: event");
    float t = 0;
    cudaEventElapsedTime(&t, ctx->ev[5], ctx->ev[0]);
    if ((r = check_device_flags(ctx))) return r;
    ms = t / reps;
    ++evaluated;
    return TJ_OK;
  };
  TuneParams best;   // the defaults
  double best_ms = 0;
  if ((rc = measure(best, best_ms))) return rc;
  const double default_ms = best_ms;
  struct Knob {
    int TuneParams::*field;
    std::vector<int> values;
  };
  std::vector<Knob> knobs;
  if (ctx->prec_mode == TJ_PREC_OZAKI) {
    if (ctx->slices == 5) knobs.push_back({&TuneParams::oz_bn, {48, 32}});
    knobs.push_back({&TuneParams::oz_item_cost, {2, 4, 8}});
  } else {
    knobs.push_back({&TuneParams::items_per_cta, {3, 6, 12}});
    knobs.push_back({&TuneParams::min_ksteps, {128, 256, 512}});
    knobs.push_back({&TuneParams::ctas_per_sm, {2, 3, 4}});
  }
  for (const Knob &k : knobs)
    for (int v : k.values) {
      if (best.*(k.field) == v || (k.field == &TuneParams::oz_bn && best.oz_bn == 0 && v == oz_bn(ctx->slices)))
        continue;
      TuneParams cand = best;
      cand.*(k.field) = v;
      double ms = 0;
      if ((rc = measure(cand, ms))) return rc;
      if (ms < 0.98 * best_ms) {
        best = cand;
        best_ms = ms;
      }
    }
  // the stored choice, and the plan rebuilt with it
  ctx->tune = best;
  ctx->plan_valid = false;
  if ((rc = prepare_hpsi(ctx, lat, sys, env, sys_bs, env_bs, wave))) return rc;
  tune_store(ctx->hist_key, best);
  if (out) {
    out->items_per_cta = best.items_per_cta;
    out->min_ksteps = best.min_ksteps;
    out->ctas_per_sm = best.ctas_per_sm;
    out->oz_bn = best.oz_bn ? best.oz_bn : (ctx->prec_mode == TJ_PREC_OZAKI ? oz_bn(ctx->slices) : 0);
    out->oz_item_cost = best.oz_item_cost;
    out->evaluated = evaluated;
    out->default_ms = default_ms;
    out->tuned_ms = best_ms;
    out->tuning_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out->hist_key = ctx->hist_key;
  }
  return TJ_OK;
}

}  // namespace tjb

using namespace tjb;

extern "C" int tj_set_autotune(tj_ctx *ctx, int mode) {
  if (!ctx) return set_err(TJ_ERR_ARG, "null context");
  if (mode != TJ_TUNE_OFF && mode != TJ_TUNE_CACHED && mode != TJ_TUNE_ON_MISS)
    return set_err(TJ_ERR_ARG, "unknown autotune mode");
  ctx->autotune = mode;
  if (mode == TJ_TUNE_OFF) ctx->tune = TuneParams();
  return TJ_OK;
}

extern "C" int tj_autotune(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                           const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, tj_tune_result *out) {
  if (!ctx || !wave || !wave->data) return set_err(TJ_ERR_ARG, "null argument");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(TJ_ERR_CUDA, "cudaSetDevice");
  return autotune_plan(ctx, lat, sys, env, sys_bs, env_bs, wave, out);
}
