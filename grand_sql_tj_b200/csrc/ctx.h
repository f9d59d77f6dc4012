// The context object behind tj_ctx*: one CUDA device, one stream, the compiled
// H*psi plan of the current DMRG step and the device buffers it uses.  Device
// buffers only grow; steady-state calls allocate nothing.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <map>
#include <memory>
#include <unordered_map>
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

// a block kept on the device for the caller's array [host, host + n)
// (resident.cpp)
struct ResEntry {
  const double *host = nullptr;
  int64_t n = 0;
  double *dev = nullptr;
  uint64_t stamp = 0, sample = 0;
};

// device slabs the kept arrays are carved from (resident.cpp): free
// segments and handed-out segments by address, each with its slab
struct ResArena {
  struct Free {
    size_t size;
    int slab;
  };
  std::vector<char *> slabs;
  std::map<char *, Free> free, owner;
};

}  // namespace tjb

// compiled operator renormalisation of the last tj_get_hamiltonian call (renorm.cpp)
struct tj_renorm_state;
// device-resident result of the last measurement-operator call (renorm.cpp)
struct tj_meas_state;
namespace tjb {
std::shared_ptr<tj_renorm_state> new_renorm_state();
std::shared_ptr<tj_meas_state> new_meas_state();
}

struct tj_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  double *pinned = nullptr;   // 32 doubles of page-locked host memory for scalar read-backs
  // H*psi timing: 0 start, 1 after the splits of psi, 2 after the first GEMM
  // launch, 3 after the product splits, 4 end (FP64: 1 = 0 and 3 = 2)
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t tev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // truncation stages
  int prec_mode = TJ_PREC_FP64, slices = 6;
  double wait_s = 2.0;        // limit of the split-precision GEMM's pipeline waits (tj_set_wait_limit)
  // tiling / schedule choices in use, and how they are chosen (TJ_TUNE_*)
  tjb::TuneParams tune;
  int autotune = TJ_TUNE_CACHED;
  bool tuning = false;        // inside tj_autotune (prepare_hpsi must not recurse)
  uint64_t hist_key = 0;      // block-size histogram of the current plan
  tjb::TuneParams plan_tune;  // the choices the current plan was built with
  std::vector<int64_t> multi_off;   // shared-launch plan: offset of each instance's vector
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
  tjb::DevBuf ggPool, ggOut, ggTab, ggSlots;                          // grouped block-GEMM benchmark
  tjb::DevBuf rnOps, rnTrun, rnScr, rnOut, rnSlots, rnTab;             // operator renormalisation
  tjb::DevBuf wtOps, wtOld, wtNew, wtScr, wtSlots, wtTab;              // wavefunction prediction
  // device-resident blocks (tj_set_residency): budget in bytes (0: off)
  std::vector<tjb::ResEntry> resident;
  size_t res_budget = 0, res_bytes = 0;
  tjb::ResArena arena;
  uint64_t res_clock = 0;
  double *stage = nullptr;    // page-locked staging of large downloads (2 x 8 MB)
  cudaEvent_t sev[2] = {nullptr, nullptr};
  int64_t res_hits = 0;       // uploads served from kept copies since creation
  double res_hit_bytes = 0;
  uint64_t trunc_seq = 0;     // truncations computed (the device operator of the last one stays in trA)
  std::shared_ptr<tj_renorm_state> renorm;
  std::shared_ptr<tj_meas_state> meas;
  // split-precision H*psi
  std::unique_ptr<tjb::OzPlan> oz;
  tjb::DevBuf ozPack, ozScales, ozStaJobs, ozPsiJobs, ozProdJobs, ozSegs, ozFams, ozCells, ozProdRows, ozStackRows, ozItems1,
      ozItems2, ozCta1, ozCta2, ozStaSpans, ozPsiSpans, ozProdSpans, ozStaMSpans,
      ozPsiMSpans, ozProdMSpans, ozStaMJobs, ozPsiMJobs, ozProdMJobs, ozMisc;
  std::vector<tjb::DevBuf *> all_bufs() {
    return {&ops, &scr, &vin, &vout, &counters, &partials, &cells1, &cells2, &tasks1, &tasks2, &tiles1,
            &tiles2, &red1, &red2, &slots, &m_dst, &m_n, &m_sb, &m_se, &m_src, &m_coef, &lanV, &lanScal, &lanPart, &trA, &trB,
            &trC, &trD, &trE, &corCells, &corTasks, &corTiles, &corOps, &corScr, &corPsi, &ggPool, &ggOut, &ggTab,
            &ggSlots, &rnOps, &rnTrun, &rnScr, &rnOut, &rnSlots, &rnTab, &wtOps, &wtOld, &wtNew, &wtScr,
            &wtSlots, &wtTab, &ozPack, &ozScales,
            &ozStaJobs, &ozPsiJobs, &ozProdJobs, &ozSegs, &ozFams, &ozCells, &ozProdRows, &ozStackRows, &ozItems1, &ozItems2,
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
// residency (resident.cpp): the device copy of host [p, p + n) if kept, else
// null; keep the device copy dev_src of a host array the library filled;
// drop all; an upload that reads the kept copy when there is one
const double *res_find(tj_ctx *ctx, const double *p, int64_t n);
int res_keep(tj_ctx *ctx, const double *host, int64_t n, const double *dev_src, cudaStream_t st);
void res_clear(tj_ctx *ctx);
cudaError_t upload(tj_ctx *ctx, double *dst, const double *src, int64_t n, cudaStream_t st);
// device-to-host copy of n doubles into caller memory, through page-locked
// staging; returns when dst is filled (the stream is synchronised)
int download(tj_ctx *ctx, double *dst, const double *src, int64_t n, cudaStream_t st);
int reset_device_flags(tj_ctx *ctx);
// wavefunction table checks shared by every entry point that takes a tj_wave:
// null tables, negative sizes or offsets, a sector past wave->dim
int check_wave(const tj_wave *w);
// same sector table (outvec must have invec's layout)
bool same_layout(const tj_wave *a, const tj_wave *b);
int install_plan(tj_ctx *ctx, std::unique_ptr<HpsiPlan> P, uint64_t key, std::chrono::steady_clock::time_point t0);

// autotuning (tune.cpp)
// key of the plan's block-size histogram: GEMM tasks counted by
// (log2 M, log2 N, log2 K), with the precision mode and slice count
uint64_t plan_hist_key(const HpsiPlan &P, int prec_mode, int slices);
// process-wide table of tuned choices per histogram key
bool tune_lookup(uint64_t key, TuneParams &tp);
void tune_store(uint64_t key, const TuneParams &tp);
// whether the current plan was built with the choices that would be used now
bool tune_is_current(tj_ctx *ctx);
// searches the choices for the superblock by timing H*psi, stores them and
// leaves the plan prepared with the best
int autotune_plan(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                  const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, tj_tune_result *out);
}  // namespace tjb
