// Split-precision H*psi: Ozaki-style int8 slicing on the tcgen05 tensor cores.
//
// Every matrix that enters a block GEMM is scaled row by row by a power of
// two, x = 2^e * sum_{p=1..s} a_p 128^-p + tail, with truncated radix-128
// digits a_p in [-127, 127] (the "slices").  The tensor cores form the exact
// int32 sums D_d = sum_{p+q=d} A_p B_q^T for d <= s + 1, one TMEM accumulator
// per diagonal d, and the epilogue forms 2^(e_row + e_col) sum_d 128^-d D_d
// in FP64.
//
// A sum of GEMMs sum_t L_t R_t becomes ONE integer accumulation over the
// concatenated inner dimension when every L_t shares the row scales and every
// R_t the column scales.  The tasks of an output cell fall into three
// families that allow this:
//
//   left   Y += sum_t coef_t op(A_t) X_t   A: per-cell concat of coef_t op(A_t)
//                                             (static, own row scales)
//                                          B: columns of the psi cells X_t, scaled
//                                             per env basis state (tau)
//   right  Y += sum_t X_t coef_t op(R_t)   A: rows of psi cells, scaled per sys
//                                             basis state (rho)
//                                          B: per-cell concat of coef_t op(R_t)
//   two    Y += sum_t P_t coef_t op(R_t)   A: rows of the phase-1 products P_t,
//                                             scaled per sys basis state (pi)
//                                          B: per-cell concat (static)
//
// Phase-1 products P_t = op(A_t) X_t are computed first, each as a family of
// one segment: A = the split of op(A_t) (static, own row scales, shared by
// every product of the operator), B = the column split of X_t (tau, shared
// with the left families); their epilogue stores P in FP64 and raises pi,
// the row maxima of P per sys basis state, with one atomic maximum per row.
//
// Split storage ("pack" pools, bytes): a split of `rows` x K is cut into
// tiles of R rows (R = 128 for an A operand, R = BN for a B operand) and
// ceil(K / 32) k-blocks.  Tile t holds G_t row groups of 8 rows (R/8 for all
// but the last; the last holds ceil(rem/8) for A, round16(rem)/8 for B, so a
// B tile is a whole number of 16-row MMA columns), laid out
//   [tile][kb][slice p][group g < G_t][c (2)][row r8 (8)][16 bytes]
// so that one k-block of one tile, all slices, is ONE contiguous block of
// s * G_t * 256 bytes: it lands in shared memory as s consecutive slices in
// the canonical UMMA K-major, no-swizzle layout (core matrices of 8 rows x
// 16 bytes, leading-byte offset 128 between the two K halves, stride-byte
// offset 256 between row groups).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "tj_internal.h"

namespace tjb {

constexpr int OZ_MAX_S = 8;
// N tile (shared-operand rows): s diagonal accumulators of <= 256 int32
// columns each, two TMEM buffers of 256 columns per CTA
inline int oz_bn(int s) { return s <= 5 ? 48 : 32; }

// One split job: rows [0, nrows) x k [0, K) of coef * M, M(r, k) =
// base[src_off + r*rs + k*ks], written as split rows row0 + r, k-blocks
// [kb0, kb0 + ceil(K/32)) of the split at pack offset `dst` (tiles of R
// rows, nkb k-blocks in all, ntiles tiles, the last of gt_last groups).  The
// job writes gtot groups (rows up to row0 + 8*gtot; rows past nrows and k
// past K as zero digits).  The row scale is scales[scale_idx + r] (max
// |value| of the row, made a power of two by the kernels); want_max: the job
// contributes to that maximum; want_split: the job writes digits (a job
// with only want_max computes a maximum shared by other jobs).
struct OzJob {
  int64_t src_off;
  int64_t dst;
  int64_t scale_idx;
  double coef;
  int32_t rs, ks, nrows, K;
  int32_t gtot, kb0;
  int32_t R, nkb, ntiles, gt_last, row0;
  int8_t space, want_max, want_split;
  int8_t pad;
};

// One k-range of an operand pair: k-blocks [a_kb0, a_kb0 + nkb) of the A
// split and [b_kb0, b_kb0 + nkb) of the B split.
struct OzSeg {
  int64_t a_base, b_base;   // pack offsets of the splits
  int32_t a_nkb, b_nkb;     // their k-block counts (tile strides)
  int32_t a_kb0, b_kb0, nkb;
  int32_t pad;
};

// A family: segments accumulated in one TMEM buffer, then scaled by
// scales[rs_idx + row] * scales[cs_idx + col].
struct OzFam {
  int32_t seg_begin, seg_end;
  int64_t rs_idx, cs_idx;
  int32_t nkb;              // k-blocks of all its segments
  int32_t pad;
};

// A work item: the output tile rows [row0, row0 + M) x cols [col0, col0 + N)
// of cell `cell` (an entry of the cell list), families [fam_begin, fam_end)
// (at most two):
//   kind 0 (H*psi cell):  init = 1: the tile is written (axpy terms or
//                         zero), then every family is added; init = 0: the
//                         families are added to the tile
//   kind 1 (products):    rows [row0, row0 + M) of a product stack (the
//                         phase-1 products P_t = op(A_t) X of one psi cell
//                         X, their operators' rows stacked): each tile row
//                         is stored to its product and its maximum |P|
//                         raises that product row's pi scale (OzProdRow)
struct OzItem {
  int32_t kind, cell;
  int32_t row0, col0;
  int32_t M, N;             // M in {64, 128}; N multiple of 16, <= oz_bn(s)
  int32_t mrows, ncols;     // valid rows / columns
  int32_t fam_begin, fam_end;
  int32_t pad1;
  int32_t init;
  int64_t pi_idx;           // unused (0): product rows carry their pi in OzProdRow
  int32_t nkb;              // k-blocks of all its families
  int32_t pad2;
  int64_t cost;             // issued int8 MACs (for ordering)
};

// Output cell of the items: a phase-2 cell of H*psi (in the output vector)
// with its axpy tasks [a_begin, a_end), or a product stack (M stacked rows,
// N columns) whose products are prod_rows [a_begin, a_end).
struct OzCell {
  int64_t off;
  int32_t ld, M, N;
  int32_t a_begin, a_end;
  int32_t pad;
};

// One product of a stack: stack rows [row_begin, row_begin + rows) are its
// rows 0..rows-1, stored at off + row + col * ld in the product space; the
// pi scale of its row r is scales[pi + r].  Products start on 8-row groups.
struct OzProdRow {
  int32_t row_begin, rows, ld, pad;
  int64_t off, pi;
};

// The same per stack row, for the GEMM (filled on the device from OzProdRow
// by launch_oz_stack_rows): the product-space offset of the row's column 0
// (-1: a padding row), its pi scale index and its column stride.  A stack's
// rows start at its cell's off.
struct OzStackRow {
  int64_t off, pi;
  int32_t ld, pad;
};

// Work split of a job list over 128-thread CTAs: CTA b starts at unit u0 of
// job `job`.  Split units: one row (rows padded to whole groups) x 16 k;
// maximum units: one row x OZ_MAX_CHUNK k.
struct OzSpan {
  int32_t job, u0;
};
constexpr int OZ_SPLIT_THREADS = 128;
constexpr int OZ_MAX_FAM = 3;   // families of one work item (a cell's left, right and two-sided sums)
constexpr int OZ_MAX_CHUNK = 16;

struct OzPlan {
  int s = 5;
  int bn = 48;
  // pools
  int64_t sta_pack = 0, dyn_pack = 0;      // bytes (static part first in one buffer)
  int64_t n_scales = 0;                    // doubles: static scales, then rho, tau, pi
  int64_t dyn_scale_begin = 0;             // first dynamic scale (zeroed per H*psi)
  int64_t rho0 = 0, tau0 = 0, pi0 = 0;
  // jobs
  std::vector<OzJob> sta_jobs;             // splits once per step
  std::vector<OzJob> psi_jobs;             // splits per H*psi, before launch 1
  std::vector<OzJob> prod_jobs;            // splits per H*psi, between the launches
  std::vector<OzSpan> sta_spans, psi_spans, prod_spans;            // split units
  std::vector<OzSpan> sta_mspans, psi_mspans, prod_mspans;         // maximum units
  // maximum jobs (the jobs with want_max, in their own lists)
  std::vector<OzJob> sta_mjobs, psi_mjobs, prod_mjobs;
  // GEMM tables
  std::vector<OzSeg> segs;
  std::vector<OzFam> fams;
  std::vector<OzCell> cells;
  std::vector<OzProdRow> prod_rows;        // products of the stacks (kind-1 cells)
  int64_t n_stack_rows = 0;                // rows of the stack-row table (kind-1 cell c: from cells[c].off)
  std::vector<OzItem> items1, items2;      // launch 1 (product stacks), launch 2 (cells: left, right, two-sided)
  // static schedule: CTA b of a launch runs items [cta[b], cta[b+1]) in order
  // (longest-processing-time-first assignment over nsm CTAs)
  std::vector<int32_t> cta1, cta2;
  int nsm = 148;
  double mma_ops = 0;                      // 2 x int8 MACs issued per H*psi
  double issued1 = 0, issued2 = 0;         // ... per launch
  double flops1 = 0, flops2 = 0;           // FP64-equivalent flops of each launch
};

// Builds the split-precision form of an H*psi plan (host); tp.oz_bn picks
// the N tile (0: oz_bn(s); 32 is also available for s = 5) and
// tp.oz_item_cost the per-item cost of the static schedule.
void build_ozaki_plan(const HpsiPlan &hp, int s, int nsm, OzPlan &oz, const TuneParams &tp = TuneParams());

// device launches (ozaki.cu)
// the stack-row table (n rows) from the stacks' products; padding rows get off = -1
void launch_oz_stack_rows(const OzCell *cells, int ncells, const OzProdRow *prows, OzStackRow *srows, int64_t n,
                          cudaStream_t st);
// raises bit 2 of *err when a value it reads is not finite
void launch_oz_max(const OzJob *jobs, int njobs, const OzSpan *spans, int nspans, const double *ops,
                   const double *psi, const double *scr, double *scales, int *err, cudaStream_t st);
void launch_oz_split(const OzJob *jobs, int njobs, const OzSpan *spans, int nspans, const double *ops,
                     const double *psi, const double *scr, const double *scales, uint8_t *pack, int s, cudaStream_t st);
cudaError_t launch_oz_gemm(const OzItem *items, const int32_t *cta, int ncta, const OzSeg *segs, const OzFam *fams,
                           const OzCell *cells, const OzStackRow *srows, const Task *tasks, const uint8_t *pack,
                           double *scales, const double *psi, double *scr, double *out, int *err, int s, int bn,
                           uint64_t wait_ns, cudaStream_t st);

}  // namespace tjb
