// Correlator contractions <psi| O |psi> (code/tjsq/measure.f90) on the device.
//
// Each contraction is compiled like H*psi (one-directional terms, no
// Hermitian-conjugate part) and run through the same grouped GEMM; the
// epilogue dots every accumulated output tile with psi instead of storing it,
// writes one partial sum per tile, and a final reduction adds the partials in
// a fixed order.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

using namespace tjb;

#define CKC(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

template <class T>
int up(tj_ctx *ctx, DevBuf &b, const std::vector<T> &v) {
  int rc = b.reserve(v.size() * sizeof(T) + 256);
  if (rc) return rc;
  if (!v.empty()) CKC(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return TJ_OK;
}

int run_cor(tj_ctx *ctx, CorKind kind, const tj_block *a, const tj_block *b, const tj_basis *sbs, const tj_basis *ebs,
            const tj_wave *wave, char flag, double *value) {
  if (!ctx || !value || !wave) return set_err(TJ_ERR_ARG, "null argument");
  if (wave->num > 0 && (!wave->sub || !wave->data)) return set_err(TJ_ERR_ARG, "bad wavefunction");
  CKC(cudaSetDevice(ctx->device));
  HpsiPlan P;
  std::string msg;
  int rc = build_cor_plan(kind, a, b, sbs, ebs, wave, flag, P, msg);
  if (rc) return set_err(rc, "correlator plan: " + msg);
  *value = 0.0;
  if (P.tiles2.empty()) return TJ_OK;
  cudaStream_t st = ctx->stream;
  if ((rc = ctx->corOps.reserve(sizeof(double) * (P.ops_len + 4)))) return rc;
  for (const auto &u : P.uploads)
    if (u.n > 0)
      CKC(cudaMemcpyAsync(ctx->corOps.d() + u.dst, u.src, sizeof(double) * u.n, cudaMemcpyHostToDevice, st));
  if ((rc = ctx->corPsi.reserve(sizeof(double) * (wave->dim + 4)))) return rc;
  CKC(cudaMemcpyAsync(ctx->corPsi.d(), wave->data, sizeof(double) * wave->dim, cudaMemcpyHostToDevice, st));
  if ((rc = ctx->corScr.reserve(sizeof(double) * (P.scratch_len + 4)))) return rc;
  // work lists: phase 1 and phase 2 share one table buffer
  std::vector<char> tab;
  auto add = [&](const void *p, size_t n) {
    size_t at = (tab.size() + 255) / 256 * 256;
    tab.resize(at + n + 1);
    if (n && p) std::memcpy(tab.data() + at, p, n);
    return at;
  };
  const size_t o_c1 = add(P.cells1.data(), P.cells1.size() * sizeof(Cell));
  const size_t o_t1 = add(P.tasks1.data(), P.tasks1.size() * sizeof(Task));
  const size_t o_l1 = add(P.tiles1.data(), P.tiles1.size() * sizeof(Tile));
  const size_t o_c2 = add(P.cells2.data(), P.cells2.size() * sizeof(Cell));
  const size_t o_t2 = add(P.tasks2.data(), P.tasks2.size() * sizeof(Task));
  const size_t o_l2 = add(P.tiles2.data(), P.tiles2.size() * sizeof(Tile));
  const size_t o_cnt = add(nullptr, 16);
  std::memset(tab.data() + o_cnt, 0, 16);
  const size_t o_part = add(nullptr, sizeof(double) * (P.tiles2.size() + 1));
  const size_t o_val = add(nullptr, 16);
  if ((rc = up(ctx, ctx->corTiles, tab))) return rc;
  char *tb = (char *)ctx->corTiles.p;
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = ctx->corOps.d();
  g.psi = ctx->corPsi.d();
  g.scr = ctx->corScr.d();
  g.out = ctx->corScr.d();
  g.cells = (const Cell *)(tb + o_c1);
  g.tasks = (const Task *)(tb + o_t1);
  g.tiles = (const Tile *)(tb + o_l1);
  g.ntiles = (int)P.tiles1.size();
  g.counter = (unsigned int *)(tb + o_cnt);
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  g.out = nullptr;
  g.cells = (const Cell *)(tb + o_c2);
  g.tasks = (const Task *)(tb + o_t2);
  g.tiles = (const Tile *)(tb + o_l2);
  g.ntiles = (int)P.tiles2.size();
  g.counter = (unsigned int *)(tb + o_cnt) + 1;
  g.dot_mode = 1;
  g.dot_with = ctx->corPsi.d();
  g.partials = (double *)(tb + o_part);
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_sum((const double *)(tb + o_part), g.ntiles, (double *)(tb + o_val), 0, st);
  CKC(cudaGetLastError());
  CKC(cudaMemcpyAsync(value, tb + o_val, sizeof(double), cudaMemcpyDeviceToHost, st));
  CKC(cudaStreamSynchronize(st));
  return TJ_OK;
}

}  // namespace

extern "C" {

int tj_measure_sys_block(tj_ctx *ctx, const tj_block *sys_bl, const tj_basis *sys_bs, const tj_wave *wave,
                         double *value) {
  if (!sys_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_MEASURE_SYS_BLOCK, sys_bl, nullptr, sys_bs, nullptr, wave, 'B', value);
}
int tj_measure_env_block(tj_ctx *ctx, const tj_block *env_bl, const tj_basis *env_bs, const tj_wave *wave,
                         double *value) {
  if (!env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_MEASURE_ENV_BLOCK, env_bl, nullptr, nullptr, env_bs, wave, 'B', value);
}
int tj_sys_block_env_block_cor_dia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_bl, const tj_basis *sys_bs,
                                   const tj_basis *env_bs, const tj_wave *wave, double *value) {
  if (!sys_bs || !env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SBEB_DIA, sys_bl, env_bl, sys_bs, env_bs, wave, 'B', value);
}
int tj_sys_block_env_block_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_bl,
                                    const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, char flag,
                                    double *value) {
  if (!sys_bs || !env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SBEB_NDIA, sys_bl, env_bl, sys_bs, env_bs, wave, flag, value);
}
int tj_sys_block_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *sys_st, const tj_basis *sys_bs,
                               const tj_wave *wave, char flag, double *value) {
  if (!sys_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SB_SITE_NDIA, sys_bl, sys_st, sys_bs, nullptr, wave, flag, value);
}
int tj_env_block_site_cor_ndia(tj_ctx *ctx, const tj_block *env_bl, const tj_block *env_st, const tj_basis *env_bs,
                               const tj_wave *wave, char flag, double *value) {
  if (!env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_EB_SITE_NDIA, env_bl, env_st, nullptr, env_bs, wave, flag, value);
}
int tj_sys_block_env_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_st,
                                   const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, char flag,
                                   double *value) {
  if (!sys_bs || !env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SB_ESITE_NDIA, sys_bl, env_st, sys_bs, env_bs, wave, flag, value);
}
int tj_sys_site_env_block_cor_ndia(tj_ctx *ctx, const tj_block *sys_st, const tj_block *env_bl,
                                   const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, char flag,
                                   double *value) {
  if (!sys_bs || !env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SSITE_EB_NDIA, sys_st, env_bl, sys_bs, env_bs, wave, flag, value);
}
int tj_sys_site_env_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_st, const tj_block *env_st,
                                  const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, char flag,
                                  double *value) {
  if (!sys_bs || !env_bs) return set_err(TJ_ERR_ARG, "null basis");
  return run_cor(ctx, COR_SSITE_ESITE_NDIA, sys_st, env_st, sys_bs, env_bs, wave, flag, value);
}

}  // extern "C"
