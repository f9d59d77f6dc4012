// Host side of the split-precision H*psi: turns the compiled FP64 task lists
// into split jobs, per-cell K-concatenated families and tcgen05 work items
// (the scheme and the storage layout are described in ozaki.h).
//
//   once per step   sta_jobs: operator splits (phase-1 operators, per-cell
//                   concatenations of coef * op(.)), with their own row scales
//   per H*psi       zero rho/tau/pi; psi_jobs (max, then split): psi column
//                   splits (tau) and row splits (rho), one of each per psi
//                   cell; launch 1 (products, left and right families; the
//                   product epilogue raises pi); prod_jobs: product row
//                   splits; launch 2 (two-sided families)
#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <queue>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "ozaki.h"
#include "tj_b200.h"

namespace tjb {

namespace {

inline int32_t cdiv(int64_t a, int64_t b) { return (int32_t)((a + b - 1) / b); }

// Which dynamic scale pool an index is relative to while building.
enum { REL_NONE = -1, REL_RHO = 0, REL_TAU = 1, REL_PI = 2 };

// Tiling of a split: tiles of R rows; the last one of gt_last groups.
struct Tiling {
  int32_t rows, R, nkb, ntiles, gt_last, gsum;
};

struct Builder {
  const HpsiPlan &hp;
  OzPlan &oz;
  int S;
  int64_t sta_bytes = 0, dyn_bytes = 0;
  std::vector<OzJob> dyn_psi, dyn_prod;
  std::vector<int> dyn_psi_rel;                 // REL_RHO / REL_TAU per psi job
  std::vector<int> row_job, col_job;            // per psi cell: its row / column split job in dyn_psi, or -1
  std::unordered_map<int64_t, int> psi_cell;    // psi offset -> phase-2 cell
  std::unordered_map<int64_t, int> prod_of;     // scratch offset -> product
  std::vector<int64_t> colsplit, rowsplit;      // per psi cell: dynamic pack offset or -1
  std::vector<int64_t> prodsplit;               // per product
  std::vector<int> seg_dyn_a, seg_dyn_b;        // segments with a dynamic A / B split
  struct FamRel { int fam, rs_rel, cs_rel; };
  std::vector<FamRel> famrel;

  int sched_item_cost = 4;   // fixed per-item cost of the schedule, in k-blocks
  Builder(const HpsiPlan &h, OzPlan &o, int s) : hp(h), oz(o), S(s) {}

  // A operands are tiled by 128 rows; B operands by the N tile, each tile a
  // whole number of 16-row MMA columns.
  Tiling tiling(int32_t rows, int32_t K, bool b_role) const {
    Tiling t;
    t.rows = rows;
    t.R = b_role ? oz.bn : 128;
    t.nkb = cdiv(K, 32);
    t.ntiles = cdiv(rows, t.R);
    const int32_t rem = rows - (t.ntiles - 1) * t.R;
    t.gt_last = b_role ? (rem + 15) / 16 * 2 : cdiv(rem, 8);
    t.gsum = (t.ntiles - 1) * (t.R / 8) + t.gt_last;
    return t;
  }
  int64_t split_bytes(const Tiling &t) const { return (int64_t)t.nkb * S * t.gsum * 256; }
  static int64_t align256(int64_t x) { return (x + 255) / 256 * 256; }
  int64_t alloc_sta(const Tiling &t) {
    const int64_t o = sta_bytes;
    sta_bytes = align256(sta_bytes + split_bytes(t));
    return o;
  }
  int64_t alloc_dyn(const Tiling &t) {
    const int64_t o = dyn_bytes;
    dyn_bytes = align256(dyn_bytes + split_bytes(t));
    return o;
  }
  int64_t alloc_scales(int64_t n) {
    const int64_t o = oz.n_scales;
    oz.n_scales += n;
    return o;
  }

  // A job writing rows [row0, row0 + 8*gtot) (gtot groups; the first nrows
  // from the source) and k-blocks from kb0 of the split at dst.
  static OzJob job(int8_t space, int64_t src_off, int32_t rs, int32_t ks, int32_t nrows, int32_t K, double coef,
                   int64_t dst, const Tiling &t, int32_t row0, int32_t gtot, int32_t kb0, int64_t scale_idx,
                   bool want_max) {
    if (nrows < 1 || K < 1 || gtot < 1) throw std::runtime_error("empty split");
    OzJob j;
    std::memset(&j, 0, sizeof j);
    j.src_off = src_off;
    j.dst = dst;
    j.scale_idx = scale_idx;
    j.coef = coef;
    j.rs = rs;
    j.ks = ks;
    j.nrows = nrows;
    j.K = K;
    j.gtot = gtot;
    j.kb0 = kb0;
    j.R = t.R;
    j.nkb = t.nkb;
    j.ntiles = t.ntiles;
    j.gt_last = t.gt_last;
    j.row0 = row0;
    j.space = space;
    j.want_max = want_max ? 1 : 0;
    j.want_split = 1;
    return j;
  }
  // Split rows of op(M) (role 0) or of op(M)^T (role 1): element (r, k) at
  // src + r*rs + k*ks.
  static void strides(const Operand &o, int role, int32_t &rs, int32_t &ks) {
    const bool t = (o.trans != 0) ^ (role == 1);
    rs = t ? o.ld : 1;
    ks = t ? 1 : o.ld;
  }

  int psi_index(const Operand &x) const {
    if (x.space != SP_PSI || x.trans) throw std::runtime_error("psi operand is not a plain cell");
    auto it = psi_cell.find(x.off);
    if (it == psi_cell.end()) throw std::runtime_error("psi operand is not a cell");
    return it->second;
  }
  // psi cell c as a B operand: rows = its columns (scale tau), K = its rows
  int64_t psi_col(int c) {
    if (colsplit[c] < 0) {
      const Cell &x = hp.cells2[c];
      const Tiling t = tiling(x.N, x.M, true);
      colsplit[c] = alloc_dyn(t);
      dyn_psi.push_back(job(SP_PSI, x.off, x.ld, 1, x.N, x.M, 1.0, colsplit[c], t, 0, t.gsum, 0,
                            hp.cell2_col_state[c], true));
      col_job[c] = (int)dyn_psi.size() - 1;
      dyn_psi_rel.push_back(REL_TAU);
    }
    return colsplit[c];
  }
  // psi cell c as an A operand: rows = its rows (scale rho), K = its columns
  int64_t psi_row(int c) {
    if (rowsplit[c] < 0) {
      const Cell &x = hp.cells2[c];
      const Tiling t = tiling(x.M, x.N, false);
      rowsplit[c] = alloc_dyn(t);
      dyn_psi.push_back(job(SP_PSI, x.off, 1, x.ld, x.M, x.N, 1.0, rowsplit[c], t, 0, t.gsum, 0,
                            hp.cell2_row_state[c], true));
      row_job[c] = (int)dyn_psi.size() - 1;
      dyn_psi_rel.push_back(REL_RHO);
    }
    return rowsplit[c];
  }
  // phase-1 product p as an A operand: rows = its rows (scale pi, raised by
  // the product's epilogue in launch 1), K = its columns
  int64_t prod_row(int p) {
    if (prodsplit[p] < 0) {
      const Cell &P = hp.cells1[p];
      const Tiling t = tiling(P.M, P.N, false);
      prodsplit[p] = alloc_dyn(t);
      dyn_prod.push_back(job(SP_SCR, P.off, 1, P.ld, P.M, P.N, 1.0, prodsplit[p], t, 0, t.gsum, 0,
                             hp.cell1_row_state[p], false));
    }
    return prodsplit[p];
  }

  int64_t item_cost(const OzItem &it, int64_t kbs) const {
    return (int64_t)it.M * it.N * 32 * kbs * (S * (S + 1) / 2);
  }

  // Phase-1 products P_t = op(A_t) X_t, stacked per psi cell X: the products
  // of one X share their B operand (the canonical column split of X, scale
  // tau) and their inner dimension, so their operators' rows are stacked
  // into one static split (A role, 128-row tiles, each product starting on
  // an 8-row group, row scales of their own) and the stack is one family of
  // one segment.  Its items are 128-row x N tiles of the stack; the epilogue
  // stores each row to its product (prod_rows) and raises that row's pi.
  void products() {
    const int BN = oz.bn;
    std::map<int, std::vector<int>> by_x;
    for (size_t p = 0; p < hp.cells1.size(); ++p) {
      const Cell &c = hp.cells1[p];
      if (c.t_end != c.t_begin + 1) throw std::runtime_error("phase-1 cell with more than one task");
      const Task &t = hp.tasks1[c.t_begin];
      if (t.L.space != SP_OPS || t.coef != 1.0) throw std::runtime_error("unexpected phase-1 task");
      by_x[psi_index(t.R)].push_back((int)p);
    }
    for (auto &kv : by_x) {
      const int x = kv.first;
      const std::vector<int> &prods = kv.second;
      const Cell &X = hp.cells2[x];
      const int32_t K = X.M;
      // the stack's rows: each product's rows from an 8-row boundary
      int32_t rows = 0;
      std::vector<int32_t> rb(prods.size());
      for (size_t i = 0; i < prods.size(); ++i) {
        const Cell &c = hp.cells1[prods[i]];
        const Task &t = hp.tasks1[c.t_begin];
        if (t.K != K || c.N != X.N) throw std::runtime_error("product operand shape");
        rb[i] = rows;
        rows += (c.M + 7) / 8 * 8;
      }
      const Tiling ta = tiling(rows, K, false);
      const int64_t pk = alloc_sta(ta);
      const int64_t sc = alloc_scales(rows);
      OzCell oc;
      std::memset(&oc, 0, sizeof oc);
      oc.M = rows;
      oc.N = X.N;
      oc.a_begin = (int32_t)oz.prod_rows.size();
      for (size_t i = 0; i < prods.size(); ++i) {
        const int p = prods[i];
        const Cell &c = hp.cells1[p];
        const Task &t = hp.tasks1[c.t_begin];
        int32_t rs, ks;
        strides(t.L, 0, rs, ks);
        oz.sta_jobs.push_back(job(SP_OPS, t.L.off, rs, ks, c.M, K, 1.0, pk, ta, rb[i], (c.M + 7) / 8, 0,
                                  sc + rb[i], true));
        OzProdRow pr;
        std::memset(&pr, 0, sizeof pr);
        pr.row_begin = rb[i];
        pr.rows = c.M;
        pr.ld = c.ld;
        pr.off = c.off;
        pr.pi = hp.cell1_row_state[p];   // made absolute in finish()
        oz.prod_rows.push_back(pr);
      }
      oc.a_end = (int32_t)oz.prod_rows.size();
      OzSeg sg;
      std::memset(&sg, 0, sizeof sg);
      sg.a_base = pk;
      sg.a_nkb = ta.nkb;
      sg.b_base = psi_col(x);
      sg.b_nkb = cdiv(K, 32);
      sg.nkb = cdiv(K, 32);
      OzFam f;
      std::memset(&f, 0, sizeof f);
      f.seg_begin = (int)oz.segs.size();
      seg_dyn_b.push_back((int)oz.segs.size());
      oz.segs.push_back(sg);
      f.seg_end = (int)oz.segs.size();
      f.rs_idx = sc;
      f.cs_idx = hp.cell2_col_state[x];
      const int fi = (int)oz.fams.size();
      famrel.push_back({fi, REL_NONE, REL_TAU});
      oz.fams.push_back(f);
      const int cell_idx = (int)oz.cells.size();
      oz.cells.push_back(oc);
      for (int32_t r0 = 0; r0 < rows; r0 += 128)
        for (int32_t n0 = 0; n0 < X.N; n0 += BN) {
          OzItem it;
          std::memset(&it, 0, sizeof it);
          it.kind = 1;
          it.cell = cell_idx;
          it.row0 = r0;
          it.col0 = n0;
          it.mrows = std::min(128, rows - r0);
          it.M = it.mrows <= 64 ? 64 : 128;
          it.ncols = std::min(BN, X.N - n0);
          it.N = std::min(BN, (it.ncols + 15) / 16 * 16);
          it.fam_begin = fi;
          it.fam_end = fi + 1;
          it.init = 0;
          it.pi_idx = 0;
          it.cost = item_cost(it, sg.nkb);
          oz.items1.push_back(it);
        }
    }
  }

  // A family of tasks that share the B side's concatenation (right: psi rows,
  // two-sided: product rows).
  int right_family(const Cell &c, int64_t ci, const std::vector<int> &tl, bool prods) {
    int32_t kbt = 0;
    for (int ti : tl) kbt += cdiv(hp.tasks2[ti].K, 32);
    const Tiling tb = tiling(c.N, 32 * kbt, true);
    const int64_t pk = alloc_sta(tb);
    const int64_t sc = alloc_scales(c.N);
    OzFam f;
    f.seg_begin = (int)oz.segs.size();
    int32_t kb = 0;
    for (int ti : tl) {
      const Task &t = hp.tasks2[ti];
      int32_t rs, ks;
      strides(t.R, 1, rs, ks);
      oz.sta_jobs.push_back(job(SP_OPS, t.R.off, rs, ks, c.N, t.K, t.coef, pk, tb, 0, tb.gsum, kb, sc, true));
      OzSeg sg;
      std::memset(&sg, 0, sizeof sg);
      if (!prods) {
        const int x = psi_index(t.L);
        const Cell &X = hp.cells2[x];
        if (X.M != c.M || X.N != t.K || hp.cell2_row_state[x] != hp.cell2_row_state[ci])
          throw std::runtime_error("right task operand shape");
        sg.a_base = psi_row(x);
      } else {
        if (t.L.trans || t.L.space != SP_SCR) throw std::runtime_error("product operand is not a plain product");
        auto it = prod_of.find(t.L.off);
        if (it == prod_of.end()) throw std::runtime_error("product operand is not a product");
        const int p = it->second;
        const Cell &P = hp.cells1[p];
        if (P.M != c.M || P.N != t.K || hp.cell1_row_state[p] != hp.cell2_row_state[ci])
          throw std::runtime_error("two-sided task operand shape");
        sg.a_base = prod_row(p);
      }
      sg.a_nkb = cdiv(t.K, 32);
      sg.a_kb0 = 0;
      sg.b_base = pk;
      sg.b_nkb = tb.nkb;
      sg.b_kb0 = kb;
      sg.nkb = cdiv(t.K, 32);
      seg_dyn_a.push_back((int)oz.segs.size());
      oz.segs.push_back(sg);
      kb += sg.nkb;
    }
    f.seg_end = (int)oz.segs.size();
    f.rs_idx = hp.cell2_row_state[ci];
    f.cs_idx = sc;
    const int fi = (int)oz.fams.size();
    famrel.push_back({fi, prods ? REL_PI : REL_RHO, REL_NONE});
    oz.fams.push_back(f);
    return fi;
  }

  int left_family(const Cell &c, int64_t ci, const std::vector<int> &tl) {
    int32_t kbt = 0;
    for (int ti : tl) kbt += cdiv(hp.tasks2[ti].K, 32);
    const Tiling ta = tiling(c.M, 32 * kbt, false);
    const int64_t pk = alloc_sta(ta);
    const int64_t sc = alloc_scales(c.M);
    OzFam f;
    f.seg_begin = (int)oz.segs.size();
    int32_t kb = 0;
    for (int ti : tl) {
      const Task &t = hp.tasks2[ti];
      int32_t rs, ks;
      strides(t.L, 0, rs, ks);
      oz.sta_jobs.push_back(job(SP_OPS, t.L.off, rs, ks, c.M, t.K, t.coef, pk, ta, 0, ta.gsum, kb, sc, true));
      const int x = psi_index(t.R);
      const Cell &X = hp.cells2[x];
      if (X.M != t.K || X.N != c.N || hp.cell2_col_state[x] != hp.cell2_col_state[ci])
        throw std::runtime_error("left task operand shape");
      OzSeg sg;
      std::memset(&sg, 0, sizeof sg);
      sg.a_base = pk;
      sg.a_nkb = ta.nkb;
      sg.a_kb0 = kb;
      sg.b_base = psi_col(x);
      sg.b_nkb = cdiv(t.K, 32);
      sg.b_kb0 = 0;
      sg.nkb = cdiv(t.K, 32);
      seg_dyn_b.push_back((int)oz.segs.size());
      oz.segs.push_back(sg);
      kb += sg.nkb;
    }
    f.seg_end = (int)oz.segs.size();
    f.rs_idx = sc;
    f.cs_idx = hp.cell2_col_state[ci];
    const int fi = (int)oz.fams.size();
    famrel.push_back({fi, REL_NONE, REL_TAU});
    oz.fams.push_back(f);
    return fi;
  }

  void add_items(std::vector<OzItem> &dst, const Cell &c, int cell_idx, int fb, int fe, int init) {
    const int BN = oz.bn;
    int64_t kbs = 0;
    for (int f = fb; f < fe; ++f)
      for (int sgi = oz.fams[f].seg_begin; sgi < oz.fams[f].seg_end; ++sgi) kbs += oz.segs[sgi].nkb;
    for (int32_t r0 = 0; r0 < c.M; r0 += 128)
      for (int32_t n0 = 0; n0 < c.N; n0 += BN) {
        OzItem it;
        std::memset(&it, 0, sizeof it);
        it.kind = 0;
        it.cell = cell_idx;
        it.row0 = r0;
        it.col0 = n0;
        it.mrows = std::min(128, c.M - r0);
        it.M = it.mrows <= 64 ? 64 : 128;
        it.ncols = std::min(BN, c.N - n0);
        it.N = std::min(BN, (it.ncols + 15) / 16 * 16);
        it.fam_begin = fb;
        it.fam_end = fe;
        it.pad1 = 0;
        it.init = init;
        it.cost = item_cost(it, kbs);
        dst.push_back(it);
      }
  }

  void cells() {
    const int64_t npsi = (int64_t)hp.cells2.size();
    std::vector<int> left, right, two;
    for (int64_t ci = 0; ci < npsi; ++ci) {
      const Cell &c = hp.cells2[ci];
      OzCell oc;
      std::memset(&oc, 0, sizeof oc);
      oc.off = c.off;
      oc.ld = c.ld;
      oc.M = c.M;
      oc.N = c.N;
      oc.a_begin = oc.a_end = c.t_end;
      left.clear();
      right.clear();
      two.clear();
      for (int ti = c.t_begin; ti < c.t_end; ++ti) {
        const Task &t = hp.tasks2[ti];
        if (t.R.space == SP_NONE) {
          if (t.L.trans || t.L.space != SP_PSI) throw std::runtime_error("axpy operand is not a psi cell");
          if (oc.a_begin == c.t_end) oc.a_begin = ti;
          continue;
        }
        if (t.L.space == SP_OPS) left.push_back(ti);
        else if (t.L.space == SP_PSI) right.push_back(ti);
        else if (t.L.space == SP_SCR) two.push_back(ti);
        else throw std::runtime_error("unknown task form");
      }
      if (oc.a_begin != c.t_end) oc.a_end = c.t_end;
      const int cell_idx = (int)oz.cells.size();
      oz.cells.push_back(oc);
      if (c.M <= 0 || c.N <= 0) continue;
      const int fl = left.empty() ? -1 : left_family(c, ci, left);
      const int fr = right.empty() ? -1 : right_family(c, ci, right, false);
      const int f2 = two.empty() ? -1 : right_family(c, ci, two, true);
      // launch 2 (after the products and their splits): one item per tile
      // with all of the cell's families (adjacent in the list: left, right,
      // two-sided), written once with its axpy terms
      int fb = 0, fe = 0;
      for (int f : {fl, fr, f2})
        if (f >= 0) {
          if (fe == 0) fb = f;
          fe = f + 1;
        }
      add_items(oz.items2, c, cell_idx, fb, fe, 1);
    }
  }

  void finish() {
    oz.sta_pack = sta_bytes;
    oz.dyn_pack = dyn_bytes;
    const int64_t dbase = sta_bytes;
    for (OzJob &j : dyn_psi) j.dst += dbase;
    for (OzJob &j : dyn_prod) j.dst += dbase;
    for (int i : seg_dyn_a) oz.segs[i].a_base += dbase;
    for (int i : seg_dyn_b) oz.segs[i].b_base += dbase;
    // scale pool: static scales, then rho, tau, pi
    oz.dyn_scale_begin = oz.n_scales;
    oz.rho0 = oz.n_scales;
    oz.tau0 = oz.rho0 + hp.n_sys_states;
    oz.pi0 = oz.tau0 + hp.n_env_states;
    oz.n_scales = oz.pi0 + hp.n_sys_states;
    const int64_t base[3] = {oz.rho0, oz.tau0, oz.pi0};
    for (size_t i = 0; i < dyn_psi.size(); ++i) dyn_psi[i].scale_idx += base[dyn_psi_rel[i]];
    for (OzJob &j : dyn_prod) j.scale_idx += oz.pi0;
    for (OzProdRow &pr : oz.prod_rows) pr.pi += oz.pi0;
    // the stacks' places in the per-row table the GEMM's metadata warp reads
    // (the table itself is filled on the device)
    oz.n_stack_rows = 0;
    for (OzCell &c : oz.cells) {
      if (c.a_end <= c.a_begin || c.ld != 0) continue;   // H*psi cells have ld > 0
      c.off = oz.n_stack_rows;
      oz.n_stack_rows += c.M;
    }
    for (const FamRel &fr : famrel) {
      OzFam &f = oz.fams[fr.fam];
      if (fr.rs_rel != REL_NONE) f.rs_idx += base[fr.rs_rel];
      if (fr.cs_rel != REL_NONE) f.cs_idx += base[fr.cs_rel];
    }
    // The GEMM's producer arms each stage with the bytes of the stage's
    // k-blocks, counted from the family totals below, and copies each
    // segment's k-blocks from its two splits: the totals are the sums of the
    // segments, and every segment's k-blocks must lie inside both splits, or
    // a stage would wait for bytes that never come (or copy past a split).
    for (const OzSeg &sg : oz.segs)
      if (sg.nkb < 1 || sg.a_kb0 < 0 || sg.b_kb0 < 0 || sg.a_kb0 + sg.nkb > sg.a_nkb || sg.b_kb0 + sg.nkb > sg.b_nkb)
        throw std::runtime_error("split-precision plan: a segment's k-blocks leave its splits");
    for (OzFam &f : oz.fams) {
      f.nkb = 0;
      f.pad = 0;
      for (int i = f.seg_begin; i < f.seg_end; ++i) f.nkb += oz.segs[i].nkb;
    }
    for (std::vector<OzItem> *v : {&oz.items1, &oz.items2})
      for (OzItem &it : *v) {
        it.nkb = 0;
        for (int f = it.fam_begin; f < it.fam_end; ++f) it.nkb += oz.fams[f].nkb;
      }
    // maximum jobs and split jobs in lists of their own, so that no kernel
    // walks over jobs it has nothing to do for
    auto part = [](std::vector<OzJob> &all, std::vector<OzJob> &mx) {
      size_t nm = 0;
      for (const OzJob &j : all) nm += j.want_max ? 1 : 0;
      mx.clear();
      mx.reserve(nm);
      size_t w = 0;
      for (size_t i = 0; i < all.size(); ++i) {
        if (all[i].want_max) mx.push_back(all[i]);
        if (all[i].want_split) all[w++] = all[i];
      }
      all.resize(w);
    };
    part(oz.sta_jobs, oz.sta_mjobs);
    // a psi cell split both ways gets one maximum job for its rows (rho) and
    // its columns (tau, base in the job's dst): want_max = 2, rows padded to
    // warps; those jobs go first, so that no warp of the maximum kernel
    // straddles two of them or a job of another kind
    {
      std::vector<OzJob> comb, rest;
      std::vector<char> merged(dyn_psi.size(), 0);
      for (size_t c = 0; c < row_job.size(); ++c)
        if (row_job[c] >= 0 && col_job[c] >= 0) {
          OzJob j = dyn_psi[row_job[c]];
          j.want_max = 2;
          j.dst = dyn_psi[col_job[c]].scale_idx;
          comb.push_back(j);
          merged[row_job[c]] = merged[col_job[c]] = 1;
        }
      for (size_t i = 0; i < dyn_psi.size(); ++i)
        if (!merged[i] && dyn_psi[i].want_max) rest.push_back(dyn_psi[i]);
      std::vector<OzJob> splits;
      part(dyn_psi, splits);   // the split list (want_split), in creation order
      oz.psi_mjobs = std::move(comb);
      oz.psi_mjobs.insert(oz.psi_mjobs.end(), rest.begin(), rest.end());
    }
    part(dyn_prod, oz.prod_mjobs);
    oz.psi_jobs = std::move(dyn_psi);
    oz.prod_jobs = std::move(dyn_prod);
    make_spans(oz.sta_jobs, oz.sta_spans, false);
    make_spans(oz.psi_jobs, oz.psi_spans, false);
    make_spans(oz.prod_jobs, oz.prod_spans, false);
    make_spans(oz.sta_mjobs, oz.sta_mspans, true);
    make_spans(oz.psi_mjobs, oz.psi_mspans, true);
    make_spans(oz.prod_mjobs, oz.prod_mspans, true);
    schedule(oz.items1, oz.cta1);
    schedule(oz.items2, oz.cta2);
    oz.mma_ops = 0;
    int64_t kmax = 0;
    for (const std::vector<OzItem> *v : {&oz.items1, &oz.items2})
      for (const OzItem &it : *v) {
        oz.mma_ops += 2.0 * it.cost;
        (v == &oz.items1 ? oz.issued1 : oz.issued2) += 2.0 * it.cost;
        kmax = std::max<int64_t>(kmax, it.cost / ((int64_t)it.M * it.N * (S * (S + 1) / 2)));
      }
    // FP64-equivalent work: the products in launch 1, the cells' tasks in launch 2
    oz.flops1 = oz.flops2 = 0;
    for (const Cell &c : hp.cells1) oz.flops1 += 2.0 * c.M * c.N * (double)hp.tasks1[c.t_begin].K;
    for (const Cell &c : hp.cells2)
      for (int ti = c.t_begin; ti < c.t_end; ++ti) {
        const Task &t = hp.tasks2[ti];
        if (t.R.space == SP_NONE) continue;
        oz.flops2 += 2.0 * c.M * c.N * (double)t.K;
      }
    // the epilogue stages at most two families of an item (an initialising
    // cell item may have none: it writes its axpy terms or zeros)
    for (const std::vector<OzItem> *v : {&oz.items1, &oz.items2})
      for (const OzItem &it : *v)
        if (it.fam_end - it.fam_begin > OZ_MAX_FAM || (it.fam_end <= it.fam_begin && !(it.kind == 0 && it.init)))
          throw std::runtime_error("work item with no family to add or with more than three");
    // exact int32 accumulation: the GEMM accumulates a family in pieces of
    // at most floor((2^31 - 1) / (32 s 127^2)) k-blocks, so only one k-block
    // has to fit (it always does: 32 s 127^2 < 2^31 for s <= 8)
    (void)kmax;
  }

  // CTA start points over the concatenated units of a job list: CTA b takes
  // global units [b*T, (b+1)*T), starting inside job `job` at unit u0.
  // Split units cover gtot*8 rows x K/16; maximum units nrows x K/OZ_MAX_CHUNK.
  static int64_t job_units(const OzJob &j, bool max_units) {
    if (max_units) return (int64_t)(j.want_max == 2 ? (j.nrows + 31) / 32 * 32 : j.nrows) * cdiv(j.K, OZ_MAX_CHUNK);
    return (int64_t)j.gtot * 8 * (cdiv(j.K, 32) * 2);
  }
  static void make_spans(const std::vector<OzJob> &jobs, std::vector<OzSpan> &spans, bool max_units) {
    spans.clear();
    std::vector<int64_t> st(jobs.size() + 1, 0);
    for (size_t j = 0; j < jobs.size(); ++j) st[j + 1] = st[j] + job_units(jobs[j], max_units);
    spans.reserve((size_t)((st.back() + OZ_SPLIT_THREADS - 1) / OZ_SPLIT_THREADS));
    size_t j = 0;
    for (int64_t g = 0; g < st.back(); g += OZ_SPLIT_THREADS) {
      while (st[j + 1] <= g) ++j;
      spans.push_back(OzSpan{(int32_t)j, (int32_t)(g - st[j])});
    }
  }

  // Longest-processing-time-first: items by decreasing estimated time, each
  // to the least loaded CTA; then each CTA's items are made contiguous.
  // Estimated time of an item: a fixed cost per k-block (the ring of stages is
  // latency-bound, not byte-bound: measured on the B200, an item takes about
  // 0.42 us per k-block whatever its tile size) plus about four k-blocks'
  // worth per item (pipeline hand-over and epilogue).
  void schedule(std::vector<OzItem> &v, std::vector<int32_t> &cta) {
    const int n = (int)v.size();
    if (n == 0) {
      cta.assign(1, 0);
      return;
    }
    const int nb = std::min(oz.nsm, n);
    const int64_t fixed = sched_item_cost;
    auto est = [fixed](const OzItem &it) { return (int64_t)it.nkb + fixed; };
    // items by decreasing estimate, ties in list order (a stable counting sort)
    int64_t emax = 0;
    for (const OzItem &it : v) emax = std::max(emax, est(it));
    std::vector<int32_t> start((size_t)emax + 2, 0), order(n);
    for (const OzItem &it : v) ++start[(size_t)(emax - est(it)) + 1];
    for (size_t e = 0; e + 1 < start.size(); ++e) start[e + 1] += start[e];
    for (int i = 0; i < n; ++i) order[start[(size_t)(emax - est(v[i]))]++] = i;
    // each to the least loaded CTA, the lowest-numbered among equals
    using Load = std::pair<int64_t, int32_t>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int b = 0; b < nb; ++b) heap.push({0, b});
    std::vector<int32_t> bin(n);
    cta.assign(nb + 1, 0);
    for (int i = 0; i < n; ++i) {
      Load l = heap.top();
      heap.pop();
      bin[i] = l.second;
      ++cta[l.second + 1];
      l.first += est(v[order[i]]);
      heap.push(l);
    }
    for (int b = 0; b < nb; ++b) cta[b + 1] += cta[b];
    std::vector<int32_t> fill(cta.begin(), cta.end() - 1);
    std::vector<OzItem> out(n);
    for (int i = 0; i < n; ++i) out[fill[bin[i]]++] = v[order[i]];
    v.swap(out);
  }

  void build() {
    const int64_t npsi = (int64_t)hp.cells2.size();
    if (hp.cell2_row_state.size() != hp.cells2.size() || hp.cell1_row_state.size() != hp.cells1.size())
      throw std::runtime_error("plan without basis-state tables");
    for (int64_t c = 0; c < npsi; ++c) psi_cell[hp.cells2[c].off] = (int)c;
    for (size_t p = 0; p < hp.cells1.size(); ++p) prod_of[hp.cells1[p].off] = (int)p;
    colsplit.assign(npsi, -1);
    rowsplit.assign(npsi, -1);
    row_job.assign(npsi, -1);
    col_job.assign(npsi, -1);
    prodsplit.assign(hp.cells1.size(), -1);
    // capacities: one static job and one segment per product and per phase-2
    // GEMM task, up to three families and one work-item row per tile
    const size_t n1 = hp.cells1.size(), n2 = (size_t)npsi, nt = hp.tasks2.size();
    size_t ntiles = 0;
    for (const Cell &c : hp.cells1) ntiles += (size_t)cdiv(c.M, 128) * cdiv(c.N, oz.bn);
    for (const Cell &c : hp.cells2) ntiles += (size_t)cdiv(c.M, 128) * cdiv(c.N, oz.bn);
    oz.sta_jobs.reserve(n1 + nt);
    oz.segs.reserve(n1 + nt);
    seg_dyn_a.reserve(nt);
    seg_dyn_b.reserve(n1 + nt);
    oz.fams.reserve(n1 + 3 * n2);
    famrel.reserve(n1 + 3 * n2);
    oz.cells.reserve(n1 + n2);
    oz.prod_rows.reserve(n1);
    oz.items1.reserve(ntiles);
    dyn_psi.reserve(2 * n2);
    dyn_psi_rel.reserve(2 * n2);
    dyn_prod.reserve(n1);
    products();
    cells();
    finish();
  }
};

}  // namespace

void build_ozaki_plan(const HpsiPlan &hp, int s, int nsm, OzPlan &oz, const TuneParams &tp) {
  if (s < 3 || s > OZ_MAX_S) throw std::runtime_error("slices must be in 3..8");
  if (tp.oz_bn != 0 && tp.oz_bn != oz_bn(s) && !(s == 5 && tp.oz_bn == 32))
    throw std::runtime_error("N tile not available for this slice count");
  oz = OzPlan();
  oz.s = s;
  oz.nsm = std::max(1, nsm);
  oz.bn = tp.oz_bn ? tp.oz_bn : oz_bn(s);
  Builder b(hp, oz, s);
  b.sched_item_cost = std::max(0, tp.oz_item_cost);
  b.build();
}

static_assert(sizeof(OzJob) == sizeof(tj_oz_job), "job layout");
static_assert(sizeof(OzSeg) == sizeof(tj_oz_seg), "segment layout");
static_assert(sizeof(OzFam) == sizeof(tj_oz_fam), "family layout");
static_assert(sizeof(OzItem) == sizeof(tj_oz_item), "item layout");
static_assert(sizeof(OzCell) == sizeof(tj_oz_cell), "cell layout");
static_assert(sizeof(OzProdRow) == sizeof(tj_oz_prow), "product row layout");

}  // namespace tjb

int tjb_set_err(int code, const std::string &m);

extern "C" int tj_ozaki_plan_export(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                                    const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, int slices,
                                    tj_ozaki_export *out) {
  if (!out) return tjb_set_err(TJ_ERR_ARG, "null output");
  tjb::HpsiPlan P;
  std::string msg;
  int rc = tjb::build_hpsi_plan(lat, sys, env, sys_bs, env_bs, wave, P, msg);
  if (rc) return tjb_set_err(rc, "H*psi plan: " + msg);
  tjb::OzPlan oz;
  try {
    tjb::build_ozaki_plan(P, slices, 148, oz);
  } catch (const std::exception &e) {
    return tjb_set_err(TJ_ERR_ARG, std::string("split-precision plan: ") + e.what());
  }
  out->slices = oz.s;
  out->tile_n = oz.bn;
  out->sta_pack = oz.sta_pack;
  out->dyn_pack = oz.dyn_pack;
  out->n_scales = oz.n_scales;
  out->rho0 = oz.rho0;
  out->tau0 = oz.tau0;
  out->pi0 = oz.pi0;
  out->int8_ops = oz.mma_ops;
  auto put = [](auto *dst, const auto &v, int64_t &n) {
    n = (int64_t)v.size();
    if (dst && !v.empty()) std::memcpy((void *)dst, v.data(), v.size() * sizeof(v[0]));
  };
  put(out->sta_jobs, oz.sta_jobs, out->n_sta_jobs);
  put(out->psi_jobs, oz.psi_jobs, out->n_psi_jobs);
  put(out->prod_jobs, oz.prod_jobs, out->n_prod_jobs);
  put(out->segs, oz.segs, out->n_segs);
  put(out->fams, oz.fams, out->n_fams);
  put(out->cells, oz.cells, out->n_cells);
  put(out->items1, oz.items1, out->n_items1);
  put(out->items2, oz.items2, out->n_items2);
  put(out->cta1, oz.cta1, out->n_cta1);
  put(out->cta2, oz.cta2, out->n_cta2);
  put(out->sta_mjobs, oz.sta_mjobs, out->n_sta_mjobs);
  put(out->psi_mjobs, oz.psi_mjobs, out->n_psi_mjobs);
  put(out->prod_mjobs, oz.prod_mjobs, out->n_prod_mjobs);
  put(out->prod_rows, oz.prod_rows, out->n_prod_rows);
  return TJ_OK;
}
