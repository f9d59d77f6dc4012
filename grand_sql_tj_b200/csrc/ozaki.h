// Split-precision H*psi: Ozaki-style int8 slicing on the tcgen05 tensor cores.
//
// Every GEMM task Y = coef * op(L) * op(R) of the compiled H*psi is recast as
// rows of one "group": a shared operand S (the operator sub-block the tasks
// have in common, N rows x K) and a stack of rows of varying operands L_i
// (each a length-K vector), so that a 128-row tcgen05 tile holds rows of many
// small tasks:
//
//   y_i[n] = coef_i * sum_k L_i[k] * S[n][k]
//
// Each L_i and each S row is scaled by a power of two so that |x| < 1 and cut
// into s int8 slices (truncating radix-128 digits), x = 2^e sum_p a_p 128^-p.
// The tensor cores form the exact int32 products of slice pairs with
// p + q <= s + 1, one TMEM accumulator per diagonal d = p + q; the epilogue
// adds the diagonals with weights 128^-d in FP64 and applies the scales.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "tj_internal.h"

namespace tjb {

constexpr int OZ_BM = 128;   // stacked rows per tile (tcgen05 M)
// shared-operand rows per tile (tcgen05 N): s diagonal accumulators of BN
// int32 columns must fit the 256 TMEM columns a CTA allocates
inline int oz_bn(int s) { return s <= 5 ? 48 : 32; }
constexpr int OZ_KC = 64;    // K bytes staged in shared memory per step (two k32 MMAs)
constexpr int OZ_MAX_S = 8;

// A matrix cut into row slices: element (r, k) = src[off + r*rs + k*ks].
struct OzSplit {
  int64_t src_off;
  int64_t pack_off;   // byte offset of slice 0, row 0 in the pack pool
  int64_t sig_off;    // index of row 0's scale in the scale pool
  int32_t rs, ks;
  int32_t nrows, K, K_pad;
  int8_t space;       // SP_OPS / SP_PSI / SP_SCR
  int8_t pad[3];
};

// A shared operand and its range of stacked rows in one GEMM launch.
struct OzGroup {
  int64_t s_pack_off;   // static pool: slice p, row n at s_pack_off + (p*N + n)*K_pad
  int64_t tau_off;      // static scale pool index of row 0
  int32_t N, K_pad;
  int32_t row_begin, row_end;
};

// One stacked row: a row of a dynamic split and where its output goes.
struct OzRow {
  int64_t pack_off;     // dynamic pool byte offset of this row's slice 0
  int64_t sig_idx;      // dynamic scale pool index
  int64_t dst_off;      // output element offset
  double coef;
  int32_t slice_stride; // bytes between slices of this row
  int32_t dst_stride;   // output element stride along n
  int32_t dst_space;    // 0: phase-1 products (scratch), 1: task slots
  int32_t pad;
};

struct OzItem {
  int32_t group, row0, n0, pad;
};

// Output cell = sum of its tasks' slots (in task order) + axpy terms.
struct OzCellSum {
  int64_t out_off;
  int32_t ld, M, N;
  int32_t s_begin, s_end;   // range in the slot-offset list
  int32_t a_begin, a_end;   // axpy tasks (indices into the H*psi phase-2 task list)
};

struct OzPlan {
  int s = 5;
  std::vector<OzSplit> sta;          // operator splits (once per DMRG step)
  std::vector<OzSplit> dyn_a;        // psi splits for launch A
  std::vector<OzSplit> dyn_b;        // product splits for launch B
  int64_t sta_pack = 0, sta_sig = 0, dyn_pack = 0, dyn_sig = 0;
  std::vector<OzGroup> groups_a, groups_b;
  std::vector<OzRow> rows_a, rows_b;
  std::vector<OzItem> items_a, items_b;
  std::vector<OzCellSum> sums;
  std::vector<int64_t> slot_offs;
  int64_t slots_len = 0;             // doubles of task slots
  double mma_ops = 0;                // int8 MACs * 2 per H*psi
};

// Builds the split-precision form of an H*psi plan (host).
void build_ozaki_plan(const HpsiPlan &hp, int s, OzPlan &oz);

// device launches (ozaki.cu)
void launch_oz_split(const OzSplit *jobs, int njobs, const double *ops, const double *psi, const double *scr,
                     int8_t *pack, double *sig, int s, cudaStream_t st);
cudaError_t launch_oz_gemm(const int8_t *dyn_pack, const double *dyn_sig, const int8_t *sta_pack,
                           const double *sta_sig, const OzGroup *groups, const OzRow *rows, const OzItem *items,
                           int nitems, double *out_scr, double *out_slots, unsigned int *counter, int *err, int s,
                           cudaStream_t st);
void launch_oz_sum(const OzCellSum *sums, int nsums, const int64_t *slot_offs, const double *slots,
                   const Task *tasks, const double *ops, const double *psi, const double *scr, double *out,
                   cudaStream_t st);

}  // namespace tjb
