// extern "C" entry points of include/tj_b200.h: context, H*psi and Lanczos.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ctx.h"

using namespace tjb;

static thread_local std::string g_err;
const char *tj_last_error(void) { return g_err.c_str(); }
int tjb::set_err(int code, const std::string &m) {
  g_err = m;
  return code;
}
int tjb_set_err(int code, const std::string &m) { return tjb::set_err(code, m); }

#define CK(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------ device arrays
int tjb::dev_reserve(void **p, size_t *cap, size_t bytes) {
  if (bytes <= *cap && *p) return TJ_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t want = bytes + bytes / 8 + 256;
  cudaError_t e = cudaMalloc(p, want);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_err(TJ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  *cap = want;
  return TJ_OK;
}

tj_ctx::~tj_ctx() {
  cudaSetDevice(device);
  tjb::res_clear(this);
  if (stage) cudaFreeHost(stage);
  for (auto &e : sev)
    if (e) cudaEventDestroy(e);
  for (DevBuf *b : all_bufs()) b->release();
  for (auto &e : ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : tev)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
  if (pinned) cudaFreeHost(pinned);
}

extern "C" int tj_ctx_create(tj_ctx **out, int device) {
  if (!out) return set_err(TJ_ERR_ARG, "tj_ctx_create: null output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return set_err(TJ_ERR_NODEV, "no CUDA device");
  if (device < 0 || device >= n) return set_err(TJ_ERR_ARG, "device index out of range");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return set_err(TJ_ERR_NODEV, "this library is built for sm_100a (B200) only");
  std::unique_ptr<tj_ctx> c(new tj_ctx());
  c->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaMallocHost((void **)&c->pinned, 32 * sizeof(double)));
  for (auto &e : c->ev) CK(cudaEventCreate(&e));
  for (auto &e : c->tev) CK(cudaEventCreate(&e));
  *out = c.release();
  return TJ_OK;
}

extern "C" int tj_ctx_destroy(tj_ctx *ctx) {
  delete ctx;
  return TJ_OK;
}

extern "C" int tj_set_precision(tj_ctx *ctx, int mode, int slices) {
  if (!ctx) return set_err(TJ_ERR_ARG, "null context");
  if (mode != TJ_PREC_FP64 && mode != TJ_PREC_OZAKI) return set_err(TJ_ERR_ARG, "unknown precision mode");
  if (mode == TJ_PREC_OZAKI && (slices < 3 || slices > 8)) return set_err(TJ_ERR_ARG, "slices must be 3..8");
  ctx->prec_mode = mode;
  ctx->slices = slices;
  ctx->plan_valid = false;
  return TJ_OK;
}

extern "C" int tj_set_wait_limit(tj_ctx *ctx, double seconds) {
  if (!ctx) return set_err(TJ_ERR_ARG, "null context");
  if (!(seconds >= 0.0) || seconds > 60.0) return set_err(TJ_ERR_ARG, "wait limit must be within [0, 60] seconds");
  ctx->wait_s = seconds;
  return TJ_OK;
}

extern "C" int tj_step_begin(tj_ctx *ctx) {
  if (!ctx) return set_err(TJ_ERR_ARG, "null context");
  ctx->plan_valid = false;
  return TJ_OK;
}

extern "C" int tj_host_register(void *p, size_t bytes) {
  if (!p || bytes == 0) return set_err(TJ_ERR_ARG, "tj_host_register: null pointer or zero size");
  CK(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
  return TJ_OK;
}

extern "C" int tj_host_unregister(void *p) {
  if (!p) return set_err(TJ_ERR_ARG, "tj_host_unregister: null pointer");
  CK(cudaHostUnregister(p));
  return TJ_OK;
}

extern "C" int tj_hpsi_stats_get(tj_ctx *ctx, tj_hpsi_stats *st) {
  if (!ctx || !st) return set_err(TJ_ERR_ARG, "null argument");
  *st = ctx->stats;
  st->res_hits = ctx->res_hits;
  st->res_hit_bytes = ctx->res_hit_bytes;
  return TJ_OK;
}

// ------------------------------------------------------------ plan upload
template <class T>
static int upload_vec(tj_ctx *ctx, DevBuf &b, const std::vector<T> &v) {
  int rc = b.reserve(v.size() * sizeof(T) + sizeof(T));
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return TJ_OK;
}

static uint64_t fnv(uint64_t h, const void *p, size_t n) {
  const unsigned char *c = (const unsigned char *)p;
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}
static uint64_t key_block(uint64_t h, const tj_block &b) {
  h = fnv(h, &b, sizeof b);
  if (b.num > 0 && b.sub) h = fnv(h, b.sub, sizeof(tj_block_sub) * b.num);
  return h;
}
static uint64_t key_model(uint64_t h, const tj_model *m) {
  h = fnv(h, m, sizeof *m);
  h = key_block(h, m->ham);
  for (int i = 0; i < m->nsub; ++i) {
    const tj_block_set &s = m->sub[i];
    h = key_block(key_block(key_block(key_block(key_block(h, s.elec_up), s.elec_down), s.spin_sd), s.spin_sz), s.num_sn);
  }
  return h;
}
static uint64_t key_basis(uint64_t h, const tj_basis *b) {
  h = fnv(h, b, sizeof *b);
  h = fnv(h, b->sub, sizeof(tj_basis_map) * b->num);
  int nm = 0;
  for (int i = 0; i < b->num; ++i) nm = std::max(nm, b->sub[i].first + b->sub[i].num);
  return fnv(h, b->maps, sizeof(tj_basis_sub) * nm);
}
static uint64_t key_lattice(uint64_t h, const tj_lattice *L) {
  const size_t ns1 = L->num_site + 1;
  h = fnv(h, L, sizeof *L);
  h = fnv(h, L->neib, sizeof(int32_t) * ns1 * L->neibt);
  h = fnv(h, L->neiba, sizeof(int32_t) * ns1 * ns1);
  h = fnv(h, L->inb1, sizeof(int32_t) * ns1 * ns1);
  h = fnv(h, L->nleg11, sizeof(int32_t) * L->num_site);
  h = fnv(h, L->nposi, sizeof(int32_t) * ns1);
  h = fnv(h, L->nposi_dm, sizeof(int32_t) * ns1);
  h = fnv(h, L->nposi_lat, sizeof(int32_t) * ns1);
  h = fnv(h, L->jt, sizeof(double) * ns1 * L->neibt);
  h = fnv(h, L->jz, sizeof(double) * ns1 * L->neibt);
  h = fnv(h, L->jd, sizeof(double) * ns1 * L->neibt);
  h = fnv(h, L->jn, sizeof(double) * L->neibt);
  return fnv(h, L->esite, sizeof(double) * ns1);
}

static uint64_t instance_key(uint64_t h, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                             const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave) {
  h = key_lattice(h, lat);
  h = key_model(h, sys);
  h = key_model(h, env);
  h = key_basis(h, sys_bs);
  h = key_basis(h, env_bs);
  return fnv(h, wave->sub, sizeof(tj_wave_sub) * wave->num);
}

// Compiles (or reuses) the plan of H*psi and uploads operators and work lists.
int tjb::prepare_hpsi(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                      const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave) {
  if (!ctx || !lat || !sys || !env || !sys_bs || !env_bs || !wave) return set_err(TJ_ERR_ARG, "null argument");
  if (!lat->neib || !lat->nleg11 || !lat->jt || !sys->sub || !env->sub || !sys_bs->sub || !env_bs->sub || !wave->sub)
    return set_err(TJ_ERR_ARG, "null table in the inputs");
  uint64_t h = instance_key(1469598103934665603ull, lat, sys, env, sys_bs, env_bs, wave);
  h = fnv(h, &ctx->prec_mode, sizeof ctx->prec_mode);
  h = fnv(h, &ctx->slices, sizeof ctx->slices);
  if (ctx->plan_valid && ctx->plan_key == h && tune_is_current(ctx)) return reset_device_flags(ctx);
  ctx->plan_valid = false;
  CK(cudaSetDevice(ctx->device));
  const auto t_start = std::chrono::steady_clock::now();
  std::unique_ptr<HpsiPlan> P(new HpsiPlan());
  std::string msg;
  // the FP64 work lists only for the FP64 path
  int rc = build_hpsi_plan(lat, sys, env, sys_bs, env_bs, wave, *P, msg, ctx->prec_mode == TJ_PREC_FP64);
  if (rc) return set_err(rc, "H*psi plan: " + msg);
  if ((rc = install_plan(ctx, std::move(P), h, t_start))) return rc;
  if (!ctx->tuning && ctx->autotune == TJ_TUNE_ON_MISS && !tune_lookup(ctx->hist_key, ctx->tune))
    if ((rc = autotune_plan(ctx, lat, sys, env, sys_bs, env_bs, wave, nullptr))) return rc;
  return reset_device_flags(ctx);
}

// Installs a compiled plan: tiling choices, operator upload and hmerge, work
// lists, and (split precision) the split-precision plan with the operator
// splits of this step.
int tjb::install_plan(tj_ctx *ctx, std::unique_ptr<HpsiPlan> P, uint64_t h,
                      std::chrono::steady_clock::time_point t_start) {
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
  int rc;
  // tiling choices: the autotuner's for this block-size histogram, when known
  ctx->hist_key = plan_hist_key(*P, ctx->prec_mode, ctx->slices);
  if (!ctx->tuning && ctx->autotune != TJ_TUNE_OFF) tune_lookup(ctx->hist_key, ctx->tune);
  if (!(ctx->tune == TuneParams()) && ctx->prec_mode == TJ_PREC_FP64) {
    split_tiles(P->cells1, P->tasks1, P->tiles1, P->red1, P->nslots1, false, ctx->tune);
    split_tiles(P->cells2, P->tasks2, P->tiles2, P->red2, P->nslots2, false, ctx->tune);
  }
  const double plan_ms = ms_since(t_start);
  const auto t_up = clk::now();
  // operators: one copy per input block, then the merged sums on the device
  if ((rc = ctx->ops.reserve(sizeof(double) * (P->ops_len + 4)))) return rc;
  for (const auto &u : P->uploads)
    if (u.n > 0)
      CK(upload(ctx, ctx->ops.d() + u.dst, u.src, u.n, ctx->stream));
  // the split-precision plan is built on the host while those copies run
  // (from page-locked memory they return at once; the table uploads below,
  // from pageable memory, wait for the stream to reach them)
  double ozplan_ms = 0;
  std::unique_ptr<OzPlan> oz;
  if (ctx->prec_mode == TJ_PREC_OZAKI) {
    const auto t_oz = clk::now();
    oz.reset(new OzPlan());
    try {
      int nsm = 148;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
      build_ozaki_plan(*P, ctx->slices, nsm, *oz, ctx->tune);
    } catch (const std::exception &e) {
      cudaStreamSynchronize(ctx->stream);   // the copies above still read the caller's buffers
      return set_err(TJ_ERR_ARG, std::string("split-precision plan: ") + e.what());
    }
    ozplan_ms = ms_since(t_oz);
  }
  {
    std::vector<int64_t> dst, n;
    std::vector<int32_t> sb, se;
    for (const auto &m : P->merges) {
      dst.push_back(m.dst);
      n.push_back(m.n);
      sb.push_back(m.s_begin);
      se.push_back(m.s_end);
    }
    if ((rc = upload_vec(ctx, ctx->m_dst, dst)) || (rc = upload_vec(ctx, ctx->m_n, n)) ||
        (rc = upload_vec(ctx, ctx->m_sb, sb)) || (rc = upload_vec(ctx, ctx->m_se, se)) ||
        (rc = upload_vec(ctx, ctx->m_src, P->merge_src)) || (rc = upload_vec(ctx, ctx->m_coef, P->merge_coef)))
      return rc;
    launch_merge(ctx->ops.d(), (const int64_t *)ctx->m_dst.p, (const int64_t *)ctx->m_n.p,
                 (const int32_t *)ctx->m_sb.p, (const int32_t *)ctx->m_se.p, (const int64_t *)ctx->m_src.p,
                 (const double *)ctx->m_coef.p, (int)P->merges.size(), ctx->stream);
    CK(cudaGetLastError());
  }
  if ((rc = upload_vec(ctx, ctx->cells1, P->cells1)) || (rc = upload_vec(ctx, ctx->cells2, P->cells2)) ||
      (rc = upload_vec(ctx, ctx->tasks1, P->tasks1)) || (rc = upload_vec(ctx, ctx->tasks2, P->tasks2)) ||
      (rc = upload_vec(ctx, ctx->tiles1, P->tiles1)) || (rc = upload_vec(ctx, ctx->tiles2, P->tiles2)) ||
      (rc = upload_vec(ctx, ctx->red1, P->red1)) || (rc = upload_vec(ctx, ctx->red2, P->red2)))
    return rc;
  if ((rc = ctx->slots.reserve(sizeof(double) * (std::max(P->nslots1, P->nslots2) * BM * BN + 4)))) return rc;
  if ((rc = ctx->scr.reserve(sizeof(double) * (P->scratch_len + 4)))) return rc;
  if ((rc = ctx->counters.reserve(64))) return rc;
  if ((rc = ctx->partials.reserve(sizeof(double) * (std::max(P->tiles2.size(), P->tiles1.size()) + 4096))))
    return rc;
  const double upload_ms = ms_since(t_up) - ozplan_ms;   // host time of the uploads themselves
  ctx->oz.reset();
  if (oz) {
    // split-precision form: its tables, then the operators' splits (once per step)
    if ((rc = upload_vec(ctx, ctx->ozStaJobs, oz->sta_jobs)) || (rc = upload_vec(ctx, ctx->ozPsiJobs, oz->psi_jobs)) ||
        (rc = upload_vec(ctx, ctx->ozProdJobs, oz->prod_jobs)) || (rc = upload_vec(ctx, ctx->ozSegs, oz->segs)) ||
        (rc = upload_vec(ctx, ctx->ozFams, oz->fams)) ||
        (rc = upload_vec(ctx, ctx->ozCells, oz->cells)) || (rc = upload_vec(ctx, ctx->ozProdRows, oz->prod_rows)) ||
        (rc = ctx->ozStackRows.reserve(sizeof(OzStackRow) * (oz->n_stack_rows + 1))) ||
        (rc = upload_vec(ctx, ctx->ozItems1, oz->items1)) ||
        (rc = upload_vec(ctx, ctx->ozItems2, oz->items2)) || (rc = upload_vec(ctx, ctx->ozCta1, oz->cta1)) ||
        (rc = upload_vec(ctx, ctx->ozCta2, oz->cta2)) || (rc = upload_vec(ctx, ctx->ozStaSpans, oz->sta_spans)) ||
        (rc = upload_vec(ctx, ctx->ozPsiSpans, oz->psi_spans)) || (rc = upload_vec(ctx, ctx->ozProdSpans, oz->prod_spans)) ||
        (rc = upload_vec(ctx, ctx->ozStaMSpans, oz->sta_mspans)) || (rc = upload_vec(ctx, ctx->ozPsiMSpans, oz->psi_mspans)) ||
        (rc = upload_vec(ctx, ctx->ozProdMSpans, oz->prod_mspans)) ||
        (rc = upload_vec(ctx, ctx->ozStaMJobs, oz->sta_mjobs)) || (rc = upload_vec(ctx, ctx->ozPsiMJobs, oz->psi_mjobs)) ||
        (rc = upload_vec(ctx, ctx->ozProdMJobs, oz->prod_mjobs)))
      return rc;
    if ((rc = ctx->ozPack.reserve(oz->sta_pack + oz->dyn_pack + 256)) ||
        (rc = ctx->ozScales.reserve(sizeof(double) * (oz->n_scales + 4))) || (rc = ctx->ozMisc.reserve(256)))
      return rc;
    CK(cudaMemsetAsync(ctx->ozMisc.p, 0, 256, ctx->stream));
    launch_oz_stack_rows((const OzCell *)ctx->ozCells.p, (int)oz->cells.size(), (const OzProdRow *)ctx->ozProdRows.p,
                         (OzStackRow *)ctx->ozStackRows.p, oz->n_stack_rows, ctx->stream);
    CK(cudaMemsetAsync(ctx->ozScales.p, 0, sizeof(double) * (oz->n_scales + 4), ctx->stream));
    // operator splits: once per step
    launch_oz_max((const OzJob *)ctx->ozStaMJobs.p, (int)oz->sta_mjobs.size(), (const OzSpan *)ctx->ozStaMSpans.p,
                  (int)oz->sta_mspans.size(), ctx->ops.d(), nullptr, nullptr, ctx->ozScales.d(),
                  (int *)((char *)ctx->ozMisc.p + 64), ctx->stream);
    launch_oz_split((const OzJob *)ctx->ozStaJobs.p, (int)oz->sta_jobs.size(), (const OzSpan *)ctx->ozStaSpans.p,
                    (int)oz->sta_spans.size(), ctx->ops.d(), nullptr, nullptr, ctx->ozScales.d(),
                    (uint8_t *)ctx->ozPack.p, oz->s, ctx->stream);
    CK(cudaGetLastError());
    ctx->oz = std::move(oz);
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->oz) {
    // the operators' own splits: a non-finite operator entry is reported now
    int flag = 0;
    CK(cudaMemcpy(&flag, (char *)ctx->ozMisc.p + 64, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag & 2) {
      ctx->oz.reset();
      return set_err(TJ_ERR_NUMERIC, "split-precision H*psi: an operator holds a NaN or an infinity");
    }
  }
  ctx->stats = tj_hpsi_stats();
  ctx->stats.prepare_ms = ms_since(t_start);
  ctx->stats.plan_ms = plan_ms;
  ctx->stats.upload_ms = upload_ms;
  ctx->stats.ozplan_ms = ozplan_ms;
  ctx->stats.flops = P->flops;
  ctx->stats.flops_ref = P->flops_ref;
  ctx->stats.bytes = P->bytes;
  ctx->stats.n_products = (int64_t)P->cells1.size();
  ctx->stats.n_tasks = (int64_t)P->tasks2.size();
  ctx->stats.n_tiles_p1 = (int64_t)P->tiles1.size();
  ctx->stats.n_tiles_p2 = (int64_t)P->tiles2.size();
  ctx->stats.scratch_doubles = P->scratch_len;
  ctx->stats.kernels_per_hpsi = 2 + (P->red1.empty() ? 0 : 1) + (P->red2.empty() ? 0 : 1);
  ctx->stats.flops_launch1 = 0;
  for (const Cell &c : P->cells1) ctx->stats.flops_launch1 += 2.0 * c.M * c.N * (double)P->tasks1[c.t_begin].K;
  ctx->stats.flops_launch2 = P->flops - ctx->stats.flops_launch1;
  if (ctx->oz) {
    const OzPlan &oz = *ctx->oz;
    ctx->stats.int8_ops = oz.mma_ops;
    ctx->stats.int8_ops_launch1 = oz.issued1;
    ctx->stats.int8_ops_launch2 = oz.issued2;
    ctx->stats.flops_launch1 = oz.flops1;
    ctx->stats.flops_launch2 = oz.flops2;
    ctx->stats.kernels_per_hpsi = (oz.psi_mspans.empty() ? 0 : 1) + (oz.psi_spans.empty() ? 0 : 1) +
                                  (oz.items1.empty() ? 0 : 1) + (oz.prod_mspans.empty() ? 0 : 1) +
                                  (oz.prod_spans.empty() ? 0 : 1) + (oz.items2.empty() ? 0 : 1);
  }
  ctx->plan = std::move(P);
  ctx->plan_key = h;
  ctx->plan_tune = ctx->tune;
  ctx->plan_valid = true;
  return TJ_OK;
}

// Split-precision H*psi: psi scales and splits, launch 1 (phase-1 products,
// left and right families), product splits, launch 2 (two-sided families).
static int run_hpsi_oz(tj_ctx *ctx, const double *in, double *out, bool timed) {
  const OzPlan &oz = *ctx->oz;
  cudaStream_t st = ctx->stream;
  int *err = (int *)((char *)ctx->ozMisc.p + 64);
  const uint64_t wait_ns = (uint64_t)(ctx->wait_s * 1e9);
  double *scales = ctx->ozScales.d();
  uint8_t *pack = (uint8_t *)ctx->ozPack.p;
  CK(cudaMemsetAsync(scales + oz.dyn_scale_begin, 0, sizeof(double) * (oz.n_scales - oz.dyn_scale_begin), st));
  if (timed) CK(cudaEventRecord(ctx->ev[0], st));
  launch_oz_max((const OzJob *)ctx->ozPsiMJobs.p, (int)oz.psi_mjobs.size(), (const OzSpan *)ctx->ozPsiMSpans.p,
                (int)oz.psi_mspans.size(), ctx->ops.d(), in, ctx->scr.d(), scales, err, st);
  launch_oz_split((const OzJob *)ctx->ozPsiJobs.p, (int)oz.psi_jobs.size(), (const OzSpan *)ctx->ozPsiSpans.p,
                  (int)oz.psi_spans.size(), ctx->ops.d(), in, ctx->scr.d(), scales, pack, oz.s, st);
  if (timed) CK(cudaEventRecord(ctx->ev[1], st));
  CK(launch_oz_gemm((const OzItem *)ctx->ozItems1.p, (const int32_t *)ctx->ozCta1.p, (int)oz.cta1.size() - 1,
                    (const OzSeg *)ctx->ozSegs.p,
                    (const OzFam *)ctx->ozFams.p, (const OzCell *)ctx->ozCells.p,
                    (const OzStackRow *)ctx->ozStackRows.p,
                    (const Task *)ctx->tasks2.p, pack, scales, in, ctx->scr.d(), out, err, oz.s, oz.bn, wait_ns, st));
  if (timed) CK(cudaEventRecord(ctx->ev[2], st));
  launch_oz_max((const OzJob *)ctx->ozProdMJobs.p, (int)oz.prod_mjobs.size(), (const OzSpan *)ctx->ozProdMSpans.p,
                (int)oz.prod_mspans.size(), ctx->ops.d(), in, ctx->scr.d(), scales, err, st);
  launch_oz_split((const OzJob *)ctx->ozProdJobs.p, (int)oz.prod_jobs.size(), (const OzSpan *)ctx->ozProdSpans.p,
                  (int)oz.prod_spans.size(), ctx->ops.d(), in, ctx->scr.d(), scales, pack, oz.s, st);
  if (timed) CK(cudaEventRecord(ctx->ev[3], st));
  CK(launch_oz_gemm((const OzItem *)ctx->ozItems2.p, (const int32_t *)ctx->ozCta2.p, (int)oz.cta2.size() - 1,
                    (const OzSeg *)ctx->ozSegs.p,
                    (const OzFam *)ctx->ozFams.p, (const OzCell *)ctx->ozCells.p,
                    (const OzStackRow *)ctx->ozStackRows.p,
                    (const Task *)ctx->tasks2.p, pack, scales, in, ctx->scr.d(), out, err, oz.s, oz.bn, wait_ns, st));
  if (timed) CK(cudaEventRecord(ctx->ev[4], st));
  CK(cudaGetLastError());
  ++ctx->n_hpsi;
  return TJ_OK;
}

// Reads the device error flag of the split-precision kernels (bounded waits).
int tjb::check_device_flags(tj_ctx *ctx) {
  if (!ctx->oz) return TJ_OK;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, (char *)ctx->ozMisc.p + 64, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (flag & 2)
    return set_err(TJ_ERR_NUMERIC, "split-precision H*psi: the input vector (or a product) holds a NaN or an infinity");
  if (flag & 1) return set_err(TJ_ERR_TIMEOUT, "split-precision GEMM: a bounded tensor-core wait timed out");
  return TJ_OK;
}

// Clears the split-precision kernels' error flags at the start of a call, so
// that each call reports its own failures.
int tjb::reset_device_flags(tj_ctx *ctx) {
  if (!ctx->oz) return TJ_OK;
  CK(cudaMemsetAsync((char *)ctx->ozMisc.p + 64, 0, sizeof(int), ctx->stream));
  return TJ_OK;
}

// out = H * in on the device (both device pointers in the plan's psi layout).
int tjb::run_hpsi(tj_ctx *ctx, const double *in, double *out, bool timed) {
  if (ctx->oz) return run_hpsi_oz(ctx, in, out, timed);
  const HpsiPlan &P = *ctx->plan;
  unsigned int *cnt = (unsigned int *)ctx->counters.p;
  CK(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned int), ctx->stream));
  if (timed) {
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
  }
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = ctx->ops.d();
  g.psi = in;
  g.scr = ctx->scr.d();
  g.out = ctx->scr.d();
  g.cells = (const Cell *)ctx->cells1.p;
  g.tasks = (const Task *)ctx->tasks1.p;
  g.tiles = (const Tile *)ctx->tiles1.p;
  g.ntiles = (int)P.tiles1.size();
  g.counter = cnt;
  g.slots = ctx->slots.d();
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles, ctx->tune.ctas_per_sm), ctx->stream);
  launch_reduce(g, (const Reduce *)ctx->red1.p, (int)P.red1.size(), ctx->stream);
  if (timed) {
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
  }
  g.out = out;
  g.cells = (const Cell *)ctx->cells2.p;
  g.tasks = (const Task *)ctx->tasks2.p;
  g.tiles = (const Tile *)ctx->tiles2.p;
  g.ntiles = (int)P.tiles2.size();
  g.counter = cnt + 1;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles, ctx->tune.ctas_per_sm), ctx->stream);
  launch_reduce(g, (const Reduce *)ctx->red2.p, (int)P.red2.size(), ctx->stream);
  if (timed) CK(cudaEventRecord(ctx->ev[4], ctx->stream));
  CK(cudaGetLastError());
  ++ctx->n_hpsi;
  return TJ_OK;
}

int tjb::check_wave(const tj_wave *w) {
  if (!w || w->num < 0 || (w->num > 0 && (!w->sub || !w->data)) || w->dim < 0)
    return set_err(TJ_ERR_ARG, "bad wavefunction");
  int64_t d = 0;
  for (int i = 0; i < w->num; ++i) {
    if (w->sub[i].sys_dim < 0 || w->sub[i].env_dim < 0 || w->sub[i].off < 0) return set_err(TJ_ERR_ARG, "bad sector");
    d = std::max(d, w->sub[i].off + (int64_t)w->sub[i].sys_dim * w->sub[i].env_dim);
  }
  if (d > w->dim) return set_err(TJ_ERR_ARG, "sector extends past wave->dim");
  return TJ_OK;
}
bool tjb::same_layout(const tj_wave *a, const tj_wave *b) {
  if (a->num != b->num || a->dim != b->dim) return false;
  return std::memcmp(a->sub, b->sub, sizeof(tj_wave_sub) * a->num) == 0;
}

// Device times of the last timed H*psi: splits, first GEMM launch, second
// GEMM launch (with its splits excluded), total.
static void read_phases(tj_ctx *ctx, double t[4]) {
  float e[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&e[i], ctx->ev[i], ctx->ev[i + 1]);
  t[0] = (double)e[0] + e[2];
  t[1] = e[1];
  t[2] = e[3];
  t[3] = (double)e[0] + e[1] + e[2] + e[3];
}

extern "C" int tj_model_wave(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                             const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *invec,
                             tj_wave *outvec) {
  int rc;
  if (!ctx) return set_err(TJ_ERR_ARG, "null context");
  if ((rc = check_wave(invec)) || (rc = check_wave(outvec))) return rc;
  if (!same_layout(invec, outvec)) return set_err(TJ_ERR_ARG, "outvec must have invec's sector layout");
  CK(cudaSetDevice(ctx->device));
  if ((rc = prepare_hpsi(ctx, lat, sys, env, sys_bs, env_bs, invec))) return rc;
  const int64_t D = invec->dim;
  if ((rc = ctx->vin.reserve(sizeof(double) * (D + 4))) || (rc = ctx->vout.reserve(sizeof(double) * (D + 4))))
    return rc;
  CK(cudaMemcpyAsync(ctx->vin.d(), invec->data, sizeof(double) * D, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), true))) return rc;
  CK(cudaMemcpyAsync(outvec->data, ctx->vout.d(), sizeof(double) * D, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((rc = check_device_flags(ctx))) return rc;
  double t[4];
  read_phases(ctx, t);
  ctx->stats.last_ms_split = t[0];
  ctx->stats.last_ms_phase1 = t[1];
  ctx->stats.last_ms_phase2 = t[2];
  ctx->stats.last_ms = t[3];
  return TJ_OK;
}

extern "C" int tj_model_wave_multi(tj_ctx *ctx, int n, const tj_lattice *const *lat, const tj_model *const *sys,
                                   const tj_model *const *env, const tj_basis *const *sys_bs,
                                   const tj_basis *const *env_bs, const tj_wave *const *invec,
                                   tj_wave *const *outvec, int reps, double *ms) {
  int rc;
  if (!ctx || n < 1 || !lat || !sys || !env || !sys_bs || !env_bs || !invec || !outvec)
    return set_err(TJ_ERR_ARG, "tj_model_wave_multi: null argument");
  if (reps < 0 || (reps > 0 && !ms)) return set_err(TJ_ERR_ARG, "tj_model_wave_multi: bad reps");
  uint64_t h = 1469598103934665603ull;
  for (int i = 0; i < n; ++i) {
    if (!lat[i] || !sys[i] || !env[i] || !sys_bs[i] || !env_bs[i]) return set_err(TJ_ERR_ARG, "null instance input");
    if (!lat[i]->neib || !lat[i]->nleg11 || !lat[i]->jt || !sys[i]->sub || !env[i]->sub || !sys_bs[i]->sub ||
        !env_bs[i]->sub)
      return set_err(TJ_ERR_ARG, "null table in the inputs");
    if ((rc = check_wave(invec[i])) || (rc = check_wave(outvec[i]))) return rc;
    if (!same_layout(invec[i], outvec[i])) return set_err(TJ_ERR_ARG, "outvec must have invec's sector layout");
    h = instance_key(h, lat[i], sys[i], env[i], sys_bs[i], env_bs[i], invec[i]);
  }
  h = fnv(h, &n, sizeof n);
  h = fnv(h, &ctx->prec_mode, sizeof ctx->prec_mode);
  h = fnv(h, &ctx->slices, sizeof ctx->slices);
  CK(cudaSetDevice(ctx->device));
  if (!(ctx->plan_valid && ctx->plan_key == h && tune_is_current(ctx) && (int)ctx->multi_off.size() == n)) {
    ctx->plan_valid = false;
    const auto t_start = std::chrono::steady_clock::now();
    std::vector<HpsiPlan> parts(n);
    std::vector<const HpsiPlan *> pp;
    for (int i = 0; i < n; ++i) {
      std::string msg;
      rc = build_hpsi_plan(lat[i], sys[i], env[i], sys_bs[i], env_bs[i], invec[i], parts[i], msg);
      if (rc) return set_err(rc, "H*psi plan of instance " + std::to_string(i) + ": " + msg);
      pp.push_back(&parts[i]);
    }
    std::unique_ptr<HpsiPlan> P(new HpsiPlan());
    merge_plans(pp, *P, ctx->multi_off);
    if ((rc = install_plan(ctx, std::move(P), h, t_start))) return rc;
  }
  if ((rc = reset_device_flags(ctx))) return rc;
  const int64_t D = ctx->plan->psi_len;
  if ((rc = ctx->vin.reserve(sizeof(double) * (D + 4))) || (rc = ctx->vout.reserve(sizeof(double) * (D + 4))))
    return rc;
  for (int i = 0; i < n; ++i)
    CK(cudaMemcpyAsync(ctx->vin.d() + ctx->multi_off[i], invec[i]->data, sizeof(double) * invec[i]->dim,
                       cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), true))) return rc;
  if (reps > 0) {
    CK(cudaEventRecord(ctx->ev[5], ctx->stream));
    for (int r = 0; r < reps; ++r)
      if ((rc = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), false))) return rc;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    CK(cudaEventSynchronize(ctx->ev[0]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, ctx->ev[5], ctx->ev[0]));
    *ms = t / reps;
  }
  for (int i = 0; i < n; ++i)
    CK(cudaMemcpyAsync(outvec[i]->data, ctx->vout.d() + ctx->multi_off[i], sizeof(double) * outvec[i]->dim,
                       cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_device_flags(ctx);
}

extern "C" int tj_model_wave_bench(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                                   const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *invec,
                                   tj_wave *outvec, int reps, double *ms) {
  int rc;
  if (!ctx || !ms || reps < 1) return set_err(TJ_ERR_ARG, "bad argument");
  if ((rc = check_wave(invec)) || (rc = check_wave(outvec))) return rc;
  if (!same_layout(invec, outvec)) return set_err(TJ_ERR_ARG, "outvec must have invec's sector layout");
  CK(cudaSetDevice(ctx->device));
  if ((rc = prepare_hpsi(ctx, lat, sys, env, sys_bs, env_bs, invec))) return rc;
  const int64_t D = invec->dim;
  if ((rc = ctx->vin.reserve(sizeof(double) * (D + 4))) || (rc = ctx->vout.reserve(sizeof(double) * (D + 4))))
    return rc;
  CK(cudaMemcpyAsync(ctx->vin.d(), invec->data, sizeof(double) * D, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), false))) return rc;   // warm-up
  CK(cudaStreamSynchronize(ctx->stream));
  double acc[4] = {0, 0, 0, 0};
  for (int r = 0; r < reps; ++r) {
    if ((rc = run_hpsi(ctx, ctx->vin.d(), ctx->vout.d(), true))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    double t[4];
    read_phases(ctx, t);
    for (int i = 0; i < 4; ++i) acc[i] += t[i];
  }
  *ms = acc[3] / reps;
  ctx->stats.last_ms_split = acc[0] / reps;
  ctx->stats.last_ms_phase1 = acc[1] / reps;
  ctx->stats.last_ms_phase2 = acc[2] / reps;
  ctx->stats.last_ms = *ms;
  CK(cudaMemcpyAsync(outvec->data, ctx->vout.d(), sizeof(double) * D, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_device_flags(ctx);
}

// ----------------------------------------------------------------- Lanczos
// lanczos_memo_new (code/tjsq/eigen.f90:2-175) with levels = 1: three-term
// recurrence, full classical Gram-Schmidt against all previous vectors, the
// lowest Ritz value of the tridiagonal matrix after every step, stop when it
// moves by <= lanzero (or when beta <= lanzero, or after 110 vectors), then
// the Ritz vector.  All vectors live on the device; the host reads two
// scalars per step (beta and the Ritz value) to take the stop decisions.
extern "C" int tj_lanczos_memo_new(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                                   const tj_basis *sys_bs, const tj_basis *env_bs, tj_wave *eigvec, int levels,
                                   double lanzero, double *energies, int *iters) {
  const int LOOP_IN = 110;
  int rc;
  if (!ctx || !energies || !iters) return set_err(TJ_ERR_ARG, "null argument");
  if (levels != 1) return set_err(TJ_ERR_ARG, "only levels = 1 is supported (main.f90 sets levels = 1)");
  if ((rc = check_wave(eigvec))) return rc;
  CK(cudaSetDevice(ctx->device));
  if ((rc = prepare_hpsi(ctx, lat, sys, env, sys_bs, env_bs, eigvec))) return rc;
  const int64_t D = eigvec->dim;
  const int64_t ld = (D + 31) / 32 * 32;
  if ((rc = ctx->lanV.reserve(sizeof(double) * ld * (LOOP_IN + 4)))) return rc;
  const int nblk = dot_blocks(D);
  const int mdb = (int)((D + 256 * 8 - 1) / (256 * 8));
  if ((rc = ctx->lanScal.reserve(sizeof(double) * 1024))) return rc;
  const int npart = std::max(nblk, lz_blocks(D));
  if ((rc = ctx->lanPart.reserve(sizeof(double) * ((size_t)std::max(npart, 1) + (size_t)std::max(mdb, 1) * 128 + 256))))
    return rc;
  double *V = ctx->lanV.d();
  double *S = ctx->lanScal.d();   // [0..127] alpha, [128..255] beta, [256..383] uu, [384..511] coef, [512] lam, [513] nrm, [600..727] dz
  double *alpha = S, *beta = S + 128, *uu = S + 256, *coef = S + 384, *lam = S + 512, *nrm = S + 513, *dz = S + 600;
  int *itd = (int *)(S + 1000);   // the iteration's step L, read by the captured kernels
  int *cnt = (int *)(S + 1002);   // block counter of the kernels that end in a grid-wide sum
  double *part = ctx->lanPart.d(), *mpart = part + npart;
  auto vec = [&](int j) { return V + (int64_t)(j - 1) * ld; };   // tempvec(j), 1-based
  double *X = vec(LOOP_IN + 3), *Y = vec(LOOP_IN + 4);         // H*psi input and output of an iteration
  auto norm_into = [&](const double *x, double *res) {
    launch_dot(x, x, D, part, nblk, ctx->stream);
    launch_sum(part, nblk, res, 1, ctx->stream);
  };
  auto dot_into = [&](const double *x, const double *y, double *res) {
    launch_dot(x, y, D, part, nblk, ctx->stream);
    launch_sum(part, nblk, res, 0, ctx->stream);
  };
  auto fetch = [&](const double *d, double *h) -> int {
    CK(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TJ_OK;
  };
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = ctx->stream;
  CK(cudaMemsetAsync(S, 0, sizeof(double) * 1024, st));
  CK(upload(ctx, vec(1), eigvec->data, D, st));
  norm_into(vec(1), nrm);
  launch_scale_inv(vec(1), nrm, D, st);
  dot_into(vec(1), vec(1), uu + 1);
  const int64_t h0 = ctx->n_hpsi;
  if ((rc = run_hpsi(ctx, vec(1), Y, false))) return rc;
  dot_into(vec(1), Y, alpha + 1);
  double ritzmin = 0, hb = 0, hl = 0;
  if ((rc = fetch(alpha + 1, &ritzmin))) return rc;
  int last = 1;
  const int one = 1;
  CK(cudaMemcpyAsync(itd, &one, sizeof(int), cudaMemcpyHostToDevice, st));
  // One iteration (block.f90:2515-2551 and eigen.f90:60-150), captured once
  // as a CUDA graph and launched per step; every kernel reads the step L from
  // *itd, and the last one publishes beta(L) and the Ritz value to page-locked
  // host memory and advances L.  The reference stops before normalising the
  // next vector when |beta| <= lanzero; here that vector and its H*psi are
  // computed speculatively and dropped, with `last` restored, so the result
  // is the same.
  auto ref = [&](int off) { return LzRef{V, ld, itd, off, nullptr}; };
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
  launch_lz_update_norm(ref(1), Y, ref(0), ref(-1), S, itd, D, part, cnt, st);   // vec(L+1), beta(L)
  launch_lz_gram_schmidt(V, ld, itd, ref(1), D, S, mpart, mdb, 128, uu + 1, coef, part, cnt, st);
  launch_lz_scale_norm(ref(1), X, D, S, itd, part, cnt, st);                    // X = vec(L+1), uu(L+1)
  rc = run_hpsi(ctx, X, Y, false);
  if (!rc) {
    launch_lz_dot(ref(1), Y, D, S, itd, part, cnt, st);                         // alpha(L+1)
    launch_lz_tridiag_publish(S, itd, ctx->pinned, st);
  }
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);
  --ctx->n_hpsi;   // the captured H*psi ran nothing
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string("Lanczos graph capture: ") + cudaGetErrorString(ce));
  cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string("Lanczos graph: ") + cudaGetErrorString(ie));
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { cudaGraphExecDestroy(e); }
  } guard{exec};
  while (last < LOOP_IN) {
    CK(cudaGraphLaunch(exec, st));
    CK(cudaStreamSynchronize(st));
    ++ctx->n_hpsi;
    hb = ctx->pinned[0];
    hl = ctx->pinned[1];
    ++last;
    if (!std::isfinite(hb)) return set_err(TJ_ERR_NUMERIC, "Lanczos: non-finite beta");
    if (std::fabs(hb) <= lanzero) {
      --last;
      break;
    }
    if (!std::isfinite(hl)) return set_err(TJ_ERR_NUMERIC, "Lanczos: non-finite Ritz value");
    if (std::fabs(hl - ritzmin) <= lanzero || last == LOOP_IN) {
      ritzmin = hl;
      break;
    }
    ritzmin = hl;
  }
  // label 411: dstev('V') and the Ritz vector
  launch_tridiag_min(alpha + 1, beta + 1, last, lam, dz, 1, ctx->stream);
  if ((rc = ctx->vout.reserve(sizeof(double) * (D + 4)))) return rc;
  launch_combine(V, ld, last, dz, ctx->vout.d(), D, 1, ctx->stream);
  norm_into(ctx->vout.d(), nrm);
  launch_scale_inv(ctx->vout.d(), nrm, D, ctx->stream);
  CK(cudaGetLastError());
  if ((rc = download(ctx, eigvec->data, ctx->vout.d(), D, ctx->stream))) return rc;
  if ((rc = res_keep(ctx, eigvec->data, D, ctx->vout.d(), ctx->stream))) return rc;
  if ((rc = fetch(lam, &hl))) return rc;
  if ((rc = check_device_flags(ctx))) return rc;
  energies[0] = hl;
  *iters = last;
  ctx->stats.lanczos_hpsi = ctx->n_hpsi - h0;
  ctx->stats.lanczos_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return TJ_OK;
}
