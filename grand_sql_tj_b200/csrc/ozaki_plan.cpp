// Host side of the split-precision H*psi: regroups the compiled tasks by the
// operator sub-block they share and lays out the int8 slice pools.
//
//   launch A  phase-1 products  P^T = X^T op(A)^T   rows: columns of X   S: rows of op(A)
//             left-only tasks   Y^T = X^T op(A)^T   rows: columns of X   S: rows of op(A)
//             right-only tasks  Y   = X op(R)       rows: rows of X      S: columns of op(R)
//   (split the products P)
//   launch B  two-sided tasks   Y   = P op(R)       rows: rows of P      S: columns of op(R)
//   reduce    out(cell) = sum of the cell's task outputs + axpy terms
#include <algorithm>
#include <map>
#include <stdexcept>
#include <tuple>

#include <cstring>
#include <string>

#include "ozaki.h"
#include "tj_b200.h"

namespace tjb {

namespace {

inline int32_t pad32(int32_t k) { return (k + 31) / 32 * 32; }

struct Builder {
  const HpsiPlan &hp;
  OzPlan &oz;
  std::map<std::tuple<int64_t, int, int>, int> sta_idx;   // (off, trans, role) -> static split
  std::map<std::pair<int64_t, int>, int> dyn_a_idx;       // (cell offset, kind) -> dynamic split
  std::map<int64_t, int> dyn_b_idx;                        // product offset -> dynamic split

  Builder(const HpsiPlan &h, OzPlan &o) : hp(h), oz(o) {}

  int add_split(std::vector<OzSplit> &v, int64_t &pack, int64_t &sig, int8_t space, int64_t off, int32_t rs,
                int32_t ks, int32_t nrows, int32_t K) {
    if (K < 1 || nrows < 1) throw std::runtime_error("empty split");
    OzSplit s;
    s.src_off = off;
    s.rs = rs;
    s.ks = ks;
    s.nrows = nrows;
    s.K = K;
    s.K_pad = pad32(K);
    s.space = space;
    s.pad[0] = s.pad[1] = s.pad[2] = 0;
    s.pack_off = pack;
    s.sig_off = sig;
    pack += (int64_t)oz.s * nrows * s.K_pad;
    sig += nrows;
    v.push_back(s);
    return (int)v.size() - 1;
  }
  // Shared operand from op(M): role 0 = rows of op(M), role 1 = columns of op(M).
  int static_split(const Operand &o, int rows, int cols, int role) {
    auto key = std::make_tuple(o.off, (int)o.trans, role);
    auto it = sta_idx.find(key);
    if (it != sta_idx.end()) return it->second;
    int32_t rs, ks, nr, K;
    if (role == 0) {   // row r of op(M), k along the row
      rs = o.trans ? o.ld : 1;
      ks = o.trans ? 1 : o.ld;
      nr = rows;
      K = cols;
    } else {           // column n of op(M), k down the column
      rs = o.trans ? 1 : o.ld;
      ks = o.trans ? o.ld : 1;
      nr = cols;
      K = rows;
    }
    int id = add_split(oz.sta, oz.sta_pack, oz.sta_sig, SP_OPS, o.off, rs, ks, nr, K);
    sta_idx[key] = id;
    return id;
  }
  // psi cell as the varying operand: kind 0 = its columns (X^T rows), kind 1 = its rows.
  int psi_split(const Operand &x, int M, int N, int kind) {
    if (x.space != SP_PSI || x.trans) throw std::runtime_error("psi operand is not a plain cell");
    auto key = std::make_pair(x.off, kind);
    auto it = dyn_a_idx.find(key);
    if (it != dyn_a_idx.end()) return it->second;
    int id = kind == 0 ? add_split(oz.dyn_a, oz.dyn_pack, oz.dyn_sig, SP_PSI, x.off, x.ld, 1, N, M)
                       : add_split(oz.dyn_a, oz.dyn_pack, oz.dyn_sig, SP_PSI, x.off, 1, x.ld, M, N);
    dyn_a_idx[key] = id;
    return id;
  }
  int prod_split(const Operand &p, int M, int N) {
    if (p.space != SP_SCR || p.trans) throw std::runtime_error("product operand is not a plain scratch cell");
    auto it = dyn_b_idx.find(p.off);
    if (it != dyn_b_idx.end()) return it->second;
    int id = add_split(oz.dyn_b, oz.dyn_pack, oz.dyn_sig, SP_SCR, p.off, 1, p.ld, M, N);
    dyn_b_idx[p.off] = id;
    return id;
  }

  // rows of one launch, grouped by their static split
  struct PendingRow {
    int dyn;          // dynamic split
    int row;          // row within it
    int64_t dst_off;
    int32_t dst_stride, dst_space;
    double coef;
  };
  std::map<int, std::vector<PendingRow>> pend_a, pend_b;

  void emit_rows(std::map<int, std::vector<PendingRow>> &pend, int sta, int dyn, int nrows, int64_t dst_base,
                 int32_t row_step, int32_t dst_stride, int32_t dst_space, double coef) {
    auto &v = pend[sta];
    for (int r = 0; r < nrows; ++r) v.push_back(PendingRow{dyn, r, dst_base + (int64_t)r * row_step, dst_stride, dst_space, coef});
  }

  void finish(std::map<int, std::vector<PendingRow>> &pend, const std::vector<OzSplit> &dyn, std::vector<OzGroup> &groups,
              std::vector<OzRow> &rows, std::vector<OzItem> &items) {
    for (auto &kv : pend) {
      const OzSplit &S = oz.sta[kv.first];
      OzGroup g;
      g.s_pack_off = S.pack_off;
      g.tau_off = S.sig_off;
      g.N = S.nrows;
      g.K_pad = S.K_pad;
      g.row_begin = (int32_t)rows.size();
      for (const PendingRow &p : kv.second) {
        const OzSplit &D = dyn[p.dyn];
        if (D.K_pad != S.K_pad) throw std::runtime_error("inner dimensions differ");
        // exact int32 accumulation: every diagonal sums at most s slice products of 127^2 per k
        if ((double)S.K_pad * oz.s * 127.0 * 127.0 >= 2147483647.0)
          throw std::runtime_error("inner dimension too large for int32 accumulation");
        OzRow r;
        r.pack_off = D.pack_off + (int64_t)p.row * D.K_pad;
        r.sig_idx = D.sig_off + p.row;
        r.dst_off = p.dst_off;
        r.coef = p.coef;
        r.slice_stride = D.nrows * D.K_pad;
        r.dst_stride = p.dst_stride;
        r.dst_space = p.dst_space;
        r.pad = 0;
        rows.push_back(r);
      }
      g.row_end = (int32_t)rows.size();
      const int gi = (int)groups.size();
      groups.push_back(g);
      const int bn = oz_bn(oz.s);
      for (int r0 = 0; r0 < g.row_end - g.row_begin; r0 += OZ_BM)
        for (int n0 = 0; n0 < g.N; n0 += bn) {
          items.push_back(OzItem{gi, r0, n0, 0});
          oz.mma_ops += 2.0 * OZ_BM * bn * (double)g.K_pad * (oz.s * (oz.s + 1) / 2);
        }
    }
  }

  void build() {
    // launch A: phase-1 products
    for (size_t p = 0; p < hp.cells1.size(); ++p) {
      const Cell &c = hp.cells1[p];
      if (c.t_end != c.t_begin + 1) throw std::runtime_error("phase-1 cell with more than one task");
      const Task &t = hp.tasks1[c.t_begin];
      if (t.L.space != SP_OPS) throw std::runtime_error("phase-1 task without an operator");
      const int sta = static_split(t.L, c.M, t.K, 0);       // rows of op(A): M x K
      const int dyn = psi_split(t.R, t.K, c.N, 0);          // columns of X (K x N)
      // row n of P^T (= column n of P) -> P(a, n) at off + n*ld + a
      emit_rows(pend_a, sta, dyn, c.N, c.off, c.ld, 1, 0, t.coef);
    }
    // phase-2 tasks: slots and rows
    for (size_t ci = 0; ci < hp.cells2.size(); ++ci) {
      const Cell &c = hp.cells2[ci];
      OzCellSum cs;
      cs.out_off = c.off;
      cs.ld = c.ld;
      cs.M = c.M;
      cs.N = c.N;
      cs.s_begin = (int32_t)oz.slot_offs.size();
      cs.a_begin = cs.a_end = c.t_end;
      for (int ti = c.t_begin; ti < c.t_end; ++ti) {
        const Task &t = hp.tasks2[ti];
        if (t.R.space == SP_NONE) {
          if (t.L.trans) throw std::runtime_error("transposed axpy operand");
          if (cs.a_begin == c.t_end) cs.a_begin = ti;
          continue;
        }
        const int64_t slot = oz.slots_len;
        oz.slots_len += ((int64_t)c.M * c.N + 3) / 4 * 4;
        oz.slot_offs.push_back(slot);
        if (t.L.space == SP_OPS) {            // op(A) X: Y^T = X^T op(A)^T
          const int sta = static_split(t.L, c.M, t.K, 0);
          const int dyn = psi_split(t.R, t.K, c.N, 0);
          emit_rows(pend_a, sta, dyn, c.N, slot, c.M, 1, 1, t.coef);
        } else if (t.L.space == SP_PSI) {     // X op(R)
          const int sta = static_split(t.R, t.K, c.N, 1);
          const int dyn = psi_split(t.L, c.M, t.K, 1);
          emit_rows(pend_a, sta, dyn, c.M, slot, 1, c.M, 1, t.coef);
        } else {                              // P op(R)
          const int sta = static_split(t.R, t.K, c.N, 1);
          const int dyn = prod_split(t.L, c.M, t.K);
          emit_rows(pend_b, sta, dyn, c.M, slot, 1, c.M, 1, t.coef);
        }
      }
      cs.s_end = (int32_t)oz.slot_offs.size();
      cs.a_end = c.t_end;
      oz.sums.push_back(cs);
    }
    finish(pend_a, oz.dyn_a, oz.groups_a, oz.rows_a, oz.items_a);
    finish(pend_b, oz.dyn_b, oz.groups_b, oz.rows_b, oz.items_b);
    auto by_k = [&](std::vector<OzItem> &items, const std::vector<OzGroup> &g) {
      std::stable_sort(items.begin(), items.end(),
                       [&](const OzItem &a, const OzItem &b) { return g[a.group].K_pad > g[b.group].K_pad; });
    };
    by_k(oz.items_a, oz.groups_a);
    by_k(oz.items_b, oz.groups_b);
  }
};

}  // namespace

void build_ozaki_plan(const HpsiPlan &hp, int s, OzPlan &oz) {
  if (s < 3 || s > OZ_MAX_S) throw std::runtime_error("slices must be in 3..8");
  oz = OzPlan();
  oz.s = s;
  Builder b(hp, oz);
  b.build();
}

static_assert(sizeof(OzSplit) == sizeof(tj_oz_split), "split layout");
static_assert(sizeof(OzGroup) == sizeof(tj_oz_group), "group layout");
static_assert(sizeof(OzRow) == sizeof(tj_oz_row), "row layout");
static_assert(sizeof(OzItem) == sizeof(tj_oz_item), "item layout");
static_assert(sizeof(OzCellSum) == sizeof(tj_oz_cell_sum), "cell-sum layout");

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
    tjb::build_ozaki_plan(P, slices, oz);
  } catch (const std::exception &e) {
    return tjb_set_err(TJ_ERR_ARG, std::string("split-precision plan: ") + e.what());
  }
  out->slices = oz.s;
  out->tile_m = tjb::OZ_BM;
  out->tile_n = tjb::oz_bn(oz.s);
  out->pad_ = 0;
  out->sta_pack = oz.sta_pack;
  out->sta_sig = oz.sta_sig;
  out->dyn_pack = oz.dyn_pack;
  out->dyn_sig = oz.dyn_sig;
  out->slots_len = oz.slots_len;
  out->int8_ops = oz.mma_ops;
  auto put = [](auto *dst, const auto &v, int64_t &n) {
    n = (int64_t)v.size();
    if (dst && !v.empty()) std::memcpy((void *)dst, v.data(), v.size() * sizeof(v[0]));
  };
  put(out->sta, oz.sta, out->n_sta);
  put(out->dyn_a, oz.dyn_a, out->n_dyn_a);
  put(out->dyn_b, oz.dyn_b, out->n_dyn_b);
  put(out->groups_a, oz.groups_a, out->n_groups_a);
  put(out->groups_b, oz.groups_b, out->n_groups_b);
  put(out->rows_a, oz.rows_a, out->n_rows_a);
  put(out->rows_b, oz.rows_b, out->n_rows_b);
  put(out->items_a, oz.items_a, out->n_items_a);
  put(out->items_b, oz.items_b, out->n_items_b);
  put(out->sums, oz.sums, out->n_sums);
  put(out->slot_offs, oz.slot_offs, out->n_slots);
  return TJ_OK;
}
