// Internal data structures of the B200 tjsq hot path.
//
// H*psi is compiled, once per DMRG step, into two grouped-GEMM work lists:
//
//   phase 1  (products)   P_p  = op(A_p) * X_p          one output per product
//   phase 2  (cells)      Y_c  = sum_t coef_t * L_t * R_t  (+ sum coef * X  axpy terms)
//
// where every X is a "cell" of psi -- the rectangle of one sector matrix
// spanned by one system sub-block (Sub_Basis_Map) and one environment
// sub-block -- every Y is a cell of the output vector, A/R are operator
// sub-blocks (possibly transposed), and L is a phase-1 product, an operator
// sub-block or a psi cell.  Each output cell is owned by exactly one set of
// CTAs, so accumulation needs no atomics and is deterministic.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/tj_b200.h"

namespace tjb {

// Memory space an operand lives in.
enum Space : int8_t { SP_NONE = 0, SP_OPS = 1, SP_PSI = 2, SP_SCR = 3 };

// A dense column-major matrix operand, used as op(M) (trans = 1 means M^T).
struct Operand {
  int64_t off;     // element offset into the space's base pointer
  int32_t ld;      // leading dimension of the stored matrix
  int8_t space;    // Space
  int8_t trans;    // 0: M, 1: M^T
  int16_t pad;
};

// One contribution to a cell: Y += coef * op(L) * op(R); R.space == SP_NONE is an axpy Y += coef * L.
struct Task {
  Operand L, R;
  double coef;
  int32_t K;       // inner dimension (ignored for axpy)
  int32_t pad;
};

// An output rectangle and the tasks that accumulate into it.
struct Cell {
  int64_t off;     // element offset of Y(0,0) in the output space
  int32_t ld, M, N;
  int32_t t_begin, t_end;  // range in the task array
  int8_t space;    // SP_SCR (phase 1) or SP_PSI (phase 2 output vector)
  int8_t pad[7];
};

// One CTA work item: a BM x BN tile of a cell and a contiguous range of the
// cell's GEMM tasks [tb, te).  The axpy tasks [ab, ae) are applied by the
// item that finishes the tile.  slot < 0: the item owns the whole tile and
// writes it; slot >= 0: the item writes a partial tile to partial slot
// `slot` and a Reduce record sums the slots of the tile in a fixed order.
struct Tile {
  int32_t cell, row0, col0, tb, te, ab, ae, slot;
};

// Sums the partial slots [slot0, slot0 + nslot) of one tile, adds its axpy
// tasks and stores it.
struct Reduce {
  int32_t cell, row0, col0, slot0, nslot, ab, ae, pad;
};

// The compiled H*psi of one superblock.
struct HpsiPlan {
  // operator storage: every input sub-block, then every merged sub-block
  int64_t ops_len = 0;                       // doubles
  struct Upload { const double *src; int64_t n; int64_t dst; };
  std::vector<Upload> uploads;               // host -> device op copies
  struct Merge { int64_t dst, n; int32_t s_begin, s_end; };
  std::vector<Merge> merges;                 // merged sub-blocks (hmerge)
  std::vector<int64_t> merge_src;            // source offsets
  std::vector<double> merge_coef;            // and coefficients
  std::vector<std::pair<int64_t, int64_t>> sub_extent;   // (offset, doubles) of every sub-block

  std::vector<Task> tasks1, tasks2;
  std::vector<Cell> cells1, cells2;
  std::vector<Tile> tiles1, tiles2;
  std::vector<Reduce> red1, red2;
  int64_t nslots1 = 0, nslots2 = 0;          // partial tiles of split cells
  int64_t scratch_len = 0;                   // doubles of phase-1 products
  int64_t psi_len = 0;

  // Block-state index (over all block sectors of the sys / env block, before
  // the site is added) of row 0 and column 0 of every phase-2 cell, and of
  // row 0 of every phase-1 product (its rows are states of the target sys
  // sub-block).
  std::vector<int32_t> cell2_row_state, cell2_col_state, cell1_row_state;
  int32_t n_sys_states = 0, n_env_states = 0;

  // accounting
  double flops = 0, flops_ref = 0, bytes = 0;
  std::string key;                           // structural fingerprint
};

// Tile shape of the grouped FP64 kernel.
constexpr int BM = 64, BN = 64, BK = 16;

// Tiling and scheduling choices the autotuner searches (defaults: the values
// set by hand for the 4x24 m = 2000 superblock).
struct TuneParams {
  int items_per_cta = 6;    // FP64: split-K aims at this many items per resident CTA ...
  int min_ksteps = 256;     // ... never cutting an item below this many inner-dimension steps
  int ctas_per_sm = 4;      // FP64: resident CTAs per SM of the grouped kernel (1..4)
  int oz_bn = 0;            // split precision: N tile (0: the default of the slice count)
  int oz_item_cost = 4;     // split precision: per-item cost, in k-blocks, of the static schedule
  bool operator==(const TuneParams &o) const {
    return items_per_cta == o.items_per_cta && min_ksteps == o.min_ksteps && ctas_per_sm == o.ctas_per_sm &&
           oz_bn == o.oz_bn && oz_item_cost == o.oz_item_cost;
  }
};

// Work items (and Reduce records) of one grouped-GEMM pass over `cells`.
void split_tiles(const std::vector<Cell> &cells, const std::vector<Task> &tasks, std::vector<Tile> &tiles,
                 std::vector<Reduce> &red, int64_t &nslots, bool dot_mode, const TuneParams &tp = TuneParams());

// Builds the plan (host).  Returns TJ_OK or an error code with msg set.
// tiles = false: the FP64 work lists (tiles, reduce records) are not made
// (the split-precision path runs its own)
int build_hpsi_plan(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                    const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave,
                    HpsiPlan &plan, std::string &msg, bool tiles = true);

// Independent superblocks in one plan (shared launches); psi_off[i]: offset of
// instance i's vector in the concatenated input / output vector.
void merge_plans(const std::vector<const HpsiPlan *> &parts, HpsiPlan &out, std::vector<int64_t> &psi_off,
                 const TuneParams &tp = TuneParams());

// Racah 6j symbol on doubled spins (host); same formula as the reference's W6JS.
double w6j(int j1, int j2, int j3, int l1, int l2, int l3);
// Wigner 3j symbol on doubled spins and projections (Racah's sum)
double w3j(int j1, int j2, int j3, int m1, int m2, int m3);

// Correlator plans: one cell list whose epilogue dots with psi instead of storing.
enum CorKind {
  COR_MEASURE_SYS_BLOCK, COR_MEASURE_ENV_BLOCK, COR_SBEB_DIA, COR_SBEB_NDIA, COR_SB_SITE_NDIA,
  COR_EB_SITE_NDIA, COR_SB_ESITE_NDIA, COR_SSITE_EB_NDIA, COR_SSITE_ESITE_NDIA
};
int build_cor_plan(CorKind kind, const tj_block *a, const tj_block *b, const tj_basis *sys_bs,
                   const tj_basis *env_bs, const tj_wave *wave, char flag, HpsiPlan &plan,
                   std::string &msg);

// Copies a plan into the caller's arrays of tj_plan_export (two-call pattern).
int export_hpsi_plan(const HpsiPlan &P, tj_plan_export *out);

}  // namespace tjb
