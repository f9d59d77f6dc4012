// The context object behind tj_ctx*: one CUDA device, one stream, the compiled
// H*psi plan of the current DMRG step and the device buffers it uses.  Device
// buffers only grow; steady-state calls allocate nothing.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "ozaki.h"
#include "tj_internal.h"

namespace tjb {

int set_err(int code, const std::string &m);
int dev_reserve(void **p, size_t *cap, size_t bytes);

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int reserve(size_t bytes) { return dev_reserve(&p, &cap, bytes); }
  double *d() const { return (double *)p; }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace tjb

struct tj_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  double *pinned = nullptr;   // 32 doubles of page-locked host memory for scalar read-backs
  // H*psi timing: 0 start, 1 after the splits of psi, 2 after the first GEMM
  // launch, 3 after the product splits, 4 end (FP64: 1 = 0 and 3 = 2)
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int prec_mode = TJ_PREC_FP64, slices = 6;
  // compiled H*psi of the current step
  std::unique_ptr<tjb::HpsiPlan> plan;
  uint64_t plan_key = 0;
  bool plan_valid = false;
  int64_t n_hpsi = 0;
  tj_hpsi_stats stats{};
  // device buffers
  tjb::DevBuf ops, scr, vin, vout, counters, partials;
  tjb::DevBuf cells1, cells2, tasks1, tasks2, tiles1, tiles2, red1, red2, slots;
  tjb::DevBuf m_dst, m_n, m_sb, m_se, m_src, m_coef;
  tjb::DevBuf lanV, lanScal, lanPart;
  tjb::DevBuf trA, trB, trC, trD, trE;          // truncation
  tjb::DevBuf corCells, corTasks, corTiles, corOps, corScr, corPsi;   // correlators
  // split-precision H*psi
  std::unique_ptr<tjb::OzPlan> oz;
  tjb::DevBuf ozPack, ozScales, ozStaJobs, ozPsiJobs, ozProdJobs, ozSegs, ozFams, ozCells, ozItems1,
      ozItems2, ozCta1, ozCta2, ozStaSpans, ozPsiSpans, ozProdSpans, ozStaMSpans,
      ozPsiMSpans, ozProdMSpans, ozStaMJobs, ozPsiMJobs, ozProdMJobs, ozMisc;
  std::vector<tjb::DevBuf *> all_bufs() {
    return {&ops, &scr, &vin, &vout, &counters, &partials, &cells1, &cells2, &tasks1, &tasks2, &tiles1,
            &tiles2, &red1, &red2, &slots, &m_dst, &m_n, &m_sb, &m_se, &m_src, &m_coef, &lanV, &lanScal, &lanPart, &trA, &trB,
            &trC, &trD, &trE, &corCells, &corTasks, &corTiles, &corOps, &corScr, &corPsi, &ozPack, &ozScales,
            &ozStaJobs, &ozPsiJobs, &ozProdJobs, &ozSegs, &ozFams, &ozCells, &ozItems1, &ozItems2,
            &ozCta1, &ozCta2, &ozStaSpans, &ozPsiSpans, &ozProdSpans, &ozStaMSpans,
            &ozPsiMSpans, &ozProdMSpans, &ozStaMJobs, &ozPsiMJobs, &ozProdMJobs, &ozMisc};
  }
  ~tj_ctx();
};

namespace tjb {
int prepare_hpsi(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                 const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave);
int run_hpsi(tj_ctx *ctx, const double *in, double *out, bool timed);
int check_device_flags(tj_ctx *ctx);
}  // namespace tjb
