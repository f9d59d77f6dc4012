// Grouped block-GEMM benchmark: a synthetic batch of block GEMMs (the pattern
// of H*psi without its physics) run through the H*psi FP64 grouped kernel as
// one persistent launch, or as one launch per block GEMM.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

using namespace tjb;

#define CKG(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

// The batch in the kernel's task form: the terms, then one axpy task per
// cell that adds the cell's current value (read from the output, bound as the
// psi space), used by the per-block launches from a cell's second term on.
struct Batch {
  std::vector<Cell> cells;
  std::vector<Task> tasks;
  std::vector<Tile> tiles;   // grouped: the cells' split-K tiles
  std::vector<Reduce> red;
  int64_t nslots = 0;
};

}  // namespace

extern "C" int tj_grouped_gemm_bench(tj_ctx *ctx, const tj_gg_cell *cells, int ncells, const tj_gg_term *terms,
                                     int nterms, const double *pool, int64_t pool_len, int64_t out_len, int mode,
                                     int reps, double *out, double *ms, double *flops, tj_tune_result *tuned) {
  if (!ctx || !cells || !terms || !pool || !out || !ms || ncells < 1 || nterms < 1 || pool_len < 1 || out_len < 1)
    return set_err(TJ_ERR_ARG, "tj_grouped_gemm_bench: bad argument");
  if (mode < 0 || mode > 2 || reps < 1) return set_err(TJ_ERR_ARG, "tj_grouped_gemm_bench: bad mode or reps");
  // validate every window against the pool and every cell against the output
  double fl = 0;
  for (int c = 0; c < ncells; ++c) {
    const tj_gg_cell &g = cells[c];
    if (g.M < 1 || g.N < 1 || g.t_begin < 0 || g.t_end > nterms || g.t_begin >= g.t_end || g.out_off < 0 ||
        g.out_off + (int64_t)g.M * g.N > out_len)
      return set_err(TJ_ERR_ARG, "tj_grouped_gemm_bench: bad cell");
    for (int t = g.t_begin; t < g.t_end; ++t) {
      const tj_gg_term &x = terms[t];
      const int64_t lrows = x.l_trans ? x.K : g.M, lcols = x.l_trans ? g.M : x.K;
      const int64_t rrows = x.r_trans ? g.N : x.K, rcols = x.r_trans ? x.K : g.N;
      if (x.K < 1 || x.l_ld < lrows || x.r_ld < rrows || x.l_off < 0 || x.r_off < 0 ||
          x.l_off + (lcols - 1) * x.l_ld + lrows > pool_len || x.r_off + (rcols - 1) * x.r_ld + rrows > pool_len)
        return set_err(TJ_ERR_ARG, "tj_grouped_gemm_bench: operand window outside the pool");
      fl += 2.0 * g.M * g.N * (double)x.K;
    }
  }
  if (flops) *flops = fl;
  CKG(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = ctx->ggPool.reserve(sizeof(double) * pool_len)) || (rc = ctx->ggOut.reserve(sizeof(double) * out_len)))
    return rc;
  CKG(cudaMemcpyAsync(ctx->ggPool.d(), pool, sizeof(double) * pool_len, cudaMemcpyHostToDevice, st));
  CKG(cudaMemsetAsync(ctx->ggOut.d(), 0, sizeof(double) * out_len, st));

  Batch b;
  for (int c = 0; c < ncells; ++c) {
    Cell cl;
    std::memset(&cl, 0, sizeof cl);
    cl.off = cells[c].out_off;
    cl.ld = cells[c].M;
    cl.M = cells[c].M;
    cl.N = cells[c].N;
    cl.t_begin = cells[c].t_begin;
    cl.t_end = cells[c].t_end;
    cl.space = SP_PSI;
    b.cells.push_back(cl);
  }
  for (int t = 0; t < nterms; ++t) {
    Task k;
    std::memset(&k, 0, sizeof k);
    k.L.off = terms[t].l_off;
    k.L.ld = terms[t].l_ld;
    k.L.space = SP_OPS;
    k.L.trans = (int8_t)(terms[t].l_trans != 0);
    k.R.off = terms[t].r_off;
    k.R.ld = terms[t].r_ld;
    k.R.space = SP_OPS;
    k.R.trans = (int8_t)(terms[t].r_trans != 0);
    k.coef = terms[t].coef;
    k.K = terms[t].K;
    b.tasks.push_back(k);
  }
  const int self0 = (int)b.tasks.size();
  for (int c = 0; c < ncells; ++c) {
    Task k;
    std::memset(&k, 0, sizeof k);
    k.L.off = cells[c].out_off;
    k.L.ld = cells[c].M;
    k.L.space = SP_PSI;
    k.R.space = SP_NONE;
    k.coef = 1.0;
    b.tasks.push_back(k);
  }
  // per-block launch lists (built once; only mode 1 uses them)
  std::vector<Tile> ptiles;
  std::vector<int> pbegin;
  for (int c = 0; c < ncells; ++c)
    for (int t = cells[c].t_begin; t < cells[c].t_end; ++t) {
      pbegin.push_back((int)ptiles.size());
      for (int r = 0; r < cells[c].M; r += BM)
        for (int q = 0; q < cells[c].N; q += BN) {
          const bool add = t > cells[c].t_begin;
          ptiles.push_back(Tile{c, r, q, t, t + 1, add ? self0 + c : 0, add ? self0 + c + 1 : 0, -1});
        }
    }
  pbegin.push_back((int)ptiles.size());
  const int nlaunch = (int)pbegin.size() - 1;

  // tables: cells, tasks, per-block tiles, counters (one per launch), grouped tiles and reduce records
  auto upload_tables = [&](const TuneParams &tp, const Tile *&gtiles, int &ngt, const Reduce *&gred, int &ngred,
                           unsigned int *&counters, const Tile *&pt) -> int {
    split_tiles(b.cells, b.tasks, b.tiles, b.red, b.nslots, false, tp);
    const size_t sc = al256(b.cells.size() * sizeof(Cell)), stk = al256(b.tasks.size() * sizeof(Task));
    const size_t spt = al256(ptiles.size() * sizeof(Tile)), scn = al256(sizeof(unsigned int) * (nlaunch + 1));
    const size_t sgt = al256(b.tiles.size() * sizeof(Tile)), srd = al256(std::max<size_t>(1, b.red.size()) * sizeof(Reduce));
    int r = ctx->ggTab.reserve(sc + stk + spt + scn + sgt + srd);
    if (r) return r;
    char *base = (char *)ctx->ggTab.p;
    CKG(cudaMemcpyAsync(base, b.cells.data(), b.cells.size() * sizeof(Cell), cudaMemcpyHostToDevice, st));
    CKG(cudaMemcpyAsync(base + sc, b.tasks.data(), b.tasks.size() * sizeof(Task), cudaMemcpyHostToDevice, st));
    CKG(cudaMemcpyAsync(base + sc + stk, ptiles.data(), ptiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, st));
    CKG(cudaMemcpyAsync(base + sc + stk + spt + scn, b.tiles.data(), b.tiles.size() * sizeof(Tile),
                        cudaMemcpyHostToDevice, st));
    if (!b.red.empty())
      CKG(cudaMemcpyAsync(base + sc + stk + spt + scn + sgt, b.red.data(), b.red.size() * sizeof(Reduce),
                          cudaMemcpyHostToDevice, st));
    if ((r = ctx->ggSlots.reserve(sizeof(double) * (b.nslots * BM * BN + 4)))) return r;
    pt = (const Tile *)(base + sc + stk);
    counters = (unsigned int *)(base + sc + stk + spt);
    gtiles = (const Tile *)(base + sc + stk + spt + scn);
    ngt = (int)b.tiles.size();
    gred = (const Reduce *)(base + sc + stk + spt + scn + sgt);
    ngred = (int)b.red.size();
    return TJ_OK;
  };
  auto params = [&]() {
    GemmParams g;
    std::memset(&g, 0, sizeof g);
    g.ops = ctx->ggPool.d();
    g.psi = ctx->ggOut.d();
    g.out = ctx->ggOut.d();
    g.cells = (const Cell *)ctx->ggTab.p;
    g.tasks = (const Task *)((char *)ctx->ggTab.p + al256(b.cells.size() * sizeof(Cell)));
    g.slots = ctx->ggSlots.d();
    return g;
  };
  // one repetition of the chosen mode
  auto run_once = [&](int m, const TuneParams &tp, const Tile *gtiles, int ngt, const Reduce *gred, int ngred,
                      unsigned int *counters, const Tile *pt) -> int {
    CKG(cudaMemsetAsync(counters, 0, sizeof(unsigned int) * (nlaunch + 1), st));
    GemmParams g = params();
    if (m == 1) {
      for (int i = 0; i < nlaunch; ++i) {
        g.tiles = pt + pbegin[i];
        g.ntiles = pbegin[i + 1] - pbegin[i];
        g.counter = counters + i;
        launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
      }
    } else {
      g.tiles = gtiles;
      g.ntiles = ngt;
      g.counter = counters + nlaunch;
      launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles, tp.ctas_per_sm), st);
      launch_reduce(g, gred, ngred, st);
    }
    CKG(cudaGetLastError());
    return TJ_OK;
  };
  auto timed = [&](int m, const TuneParams &tp, int nrep, double &t_ms) -> int {
    const Tile *gt, *pt;
    const Reduce *gr;
    int ngt, ngr;
    unsigned int *cnt;
    int r = upload_tables(tp, gt, ngt, gr, ngr, cnt, pt);
    if (r) return r;
    if ((r = run_once(m, tp, gt, ngt, gr, ngr, cnt, pt))) return r;   // warm-up
    CKG(cudaEventRecord(ctx->ev[5], st));
    for (int i = 0; i < nrep; ++i)
      if ((r = run_once(m, tp, gt, ngt, gr, ngr, cnt, pt))) return r;
    CKG(cudaEventRecord(ctx->ev[0], st));
    CKG(cudaEventSynchronize(ctx->ev[0]));
    float f = 0;
    CKG(cudaEventElapsedTime(&f, ctx->ev[5], ctx->ev[0]));
    t_ms = f / nrep;
    return TJ_OK;
  };
  TuneParams tp = ctx->tune;
  if (mode == 2) {
    // coordinate descent over the FP64 tiling knobs (2 % threshold), from the defaults
    TuneParams best;
    double best_ms = 0;
    int evaluated = 0;
    if ((rc = timed(0, best, 3, best_ms))) return rc;
    ++evaluated;
    const double default_ms = best_ms;
    const std::pair<int TuneParams::*, std::vector<int>> knobs[] = {
        {&TuneParams::items_per_cta, {3, 6, 12}}, {&TuneParams::min_ksteps, {128, 256, 512}},
        {&TuneParams::ctas_per_sm, {2, 3, 4}}};
    for (const auto &k : knobs)
      for (int v : k.second) {
        if (best.*(k.first) == v) continue;
        TuneParams cand = best;
        cand.*(k.first) = v;
        double t = 0;
        if ((rc = timed(0, cand, 3, t))) return rc;
        ++evaluated;
        if (t < 0.98 * best_ms) {
          best = cand;
          best_ms = t;
        }
      }
    tp = best;
    if (tuned) {
      std::memset(tuned, 0, sizeof *tuned);
      tuned->items_per_cta = best.items_per_cta;
      tuned->min_ksteps = best.min_ksteps;
      tuned->ctas_per_sm = best.ctas_per_sm;
      tuned->evaluated = evaluated;
      tuned->default_ms = default_ms;
      tuned->tuned_ms = best_ms;
    }
  }
  CKG(cudaMemsetAsync(ctx->ggOut.d(), 0, sizeof(double) * out_len, st));
  if ((rc = timed(mode == 1 ? 1 : 0, tp, reps, *ms))) return rc;
  // the result of one clean repetition
  {
    const Tile *gt, *pt;
    const Reduce *gr;
    int ngt, ngr;
    unsigned int *cnt;
    if ((rc = upload_tables(tp, gt, ngt, gr, ngr, cnt, pt))) return rc;
    CKG(cudaMemsetAsync(ctx->ggOut.d(), 0, sizeof(double) * out_len, st));
    if ((rc = run_once(mode == 1 ? 1 : 0, tp, gt, ngt, gr, ngr, cnt, pt))) return rc;
  }
  CKG(cudaMemcpyAsync(out, ctx->ggOut.d(), sizeof(double) * out_len, cudaMemcpyDeviceToHost, st));
  CKG(cudaStreamSynchronize(st));
  return TJ_OK;
}
