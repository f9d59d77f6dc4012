// Host-side compiler of H*psi (model_wave + hmerge) into grouped-GEMM work lists.
//
// For every term kernel that model_wave calls (code/tjsq/get_sys.f90:4127-4240,
// add_op = 1) this file walks the same loop nest over psi sectors, basis
// sub-blocks, spin-transfer channels and target total spins, applies the same
// look-up rules and the same recoupling coefficient (6j products, sqrt and
// sign factors), and records each surviving DGEMM pair as a task instead of
// executing it.  The operators that hmerge (get_sys.f90:4383-4593) pre-sums
// become "merged" sub-blocks computed on the device.  Transposed environment
// operators (block_transfer_trans, block.f90:1676-1706) are never copied: a
// transposed view only flips the operand's transpose flag.
#include <algorithm>
#include <functional>
#include <unordered_set>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <tuple>
#include <unordered_map>

#include "tj_internal.h"

int tjb_set_err(int code, const std::string &m);

namespace tjb {

// ----------------------------------------------------------------- 6j symbol
// Racah's single-sum formula for {j1 j2 j3; l1 l2 l3} with doubled spins, as
// in W6JS (block.f90:1564-1615): triangle and parity checks, then the
// alternating sum over w with factorial weights.  The factorial table holds
// 0!..142! like FACTRL (block.f90:1508-1516).
static double g_fact[302];
static bool g_fact_ready = false;
static inline double fct(int i) { return (i >= 0 && i <= 301) ? g_fact[i] : 0.0; }

static void fact_init() {
  if (g_fact_ready) return;
  std::fill(g_fact, g_fact + 302, 0.0);
  g_fact[0] = 1.0;
  for (int i = 1; i <= 142; ++i) g_fact[i] = g_fact[i - 1] * (double)(float)i;
  g_fact_ready = true;
}

// Wigner 3j symbol on doubled spins and projections, by the Racah sum:
// (j1 j2 j3; m1 m2 m3) = (-1)^(j1-j2-m3) sqrt(D(j1 j2 j3) prod (j_i+m_i)!(j_i-m_i)!)
//   sum_k (-1)^k / [k! (j3-j2+m1+k)! (j3-j1-m2+k)! (j1+j2-j3-k)! (j1-m1-k)! (j2+m2-k)!],
// D = (j1+j2-j3)!(j1-j2+j3)!(j2+j3-j1)!/(j1+j2+j3+1)!  (all arguments halved here).
double w3j(int j1, int j2, int j3, int m1, int m2, int m3) {
  fact_init();
  if (m1 + m2 + m3 != 0) return 0.0;
  if (j3 > j1 + j2 || j3 < std::abs(j1 - j2)) return 0.0;
  if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(m3) > j3) return 0.0;
  if (((j1 + j2 + j3) & 1) || ((j1 + m1) & 1) || ((j2 + m2) & 1) || ((j3 + m3) & 1)) return 0.0;
  const int a = j3 - j2 + m1, b = j3 - j1 - m2, c = j1 + j2 - j3, d = j1 - m1, e = j2 + m2;
  const int kmin = std::max(0, std::max(-a, -b)), kmax = std::min(c, std::min(d, e));
  double sum = 0.0;
  for (int k = kmin; k <= kmax; k += 2) {
    double den = fct(k / 2) * fct((a + k) / 2) * fct((b + k) / 2) * fct((c - k) / 2) * fct((d - k) / 2) *
                 fct((e - k) / 2);
    sum += ((k / 2) % 2 ? -1.0 : 1.0) / den;
  }
  const double tri = fct(c / 2) * fct((j1 - j2 + j3) / 2) * fct((j2 + j3 - j1) / 2) / fct((j1 + j2 + j3) / 2 + 1);
  const double mf = fct((j1 + m1) / 2) * fct((j1 - m1) / 2) * fct((j2 + m2) / 2) * fct((j2 - m2) / 2) *
                    fct((j3 + m3) / 2) * fct((j3 - m3) / 2);
  const int ph = (j1 - j2 - m3) / 2;
  return ((ph % 2) ? -1.0 : 1.0) * std::sqrt(tri * mf) * sum;
}

double w6j(int j1, int j2, int j3, int l1, int l2, int l3) {
  if (!g_fact_ready) {
    std::fill(g_fact, g_fact + 302, 0.0);
    g_fact[0] = 1.0;
    for (int i = 1; i <= 142; ++i) g_fact[i] = g_fact[i - 1] * (double)(float)i;
    g_fact_ready = true;
  }
  const int a = j1 + j2, b = j1 - j2, c = j1 + l2, d = j1 - l2;
  const int e = l1 + j2, f = l1 - j2, g = l1 + l2, h = l1 - l2;
  if (a < j3 || std::abs(b) > j3 || c < l3 || std::abs(d) > l3) return 0.0;
  if (e < l3 || std::abs(f) > l3 || g < j3 || std::abs(h) > j3) return 0.0;
  const int s1 = a + j3, s2 = c + l3, s3 = e + l3, s4 = g + j3;
  if ((s1 | s2 | s3 | s4) & 1) return 0.0;
  const int wmin = std::max(std::max(s1, s2), std::max(s3, s4));
  const int ii = a + g, ij = j2 + j3 + l2 + l3, ik = j3 + j1 + l3 + l1;
  const int wmax = std::min(ii, std::min(ij, ik));
  double omega = 0.0;
  for (int w = wmin; w <= wmax; w += 2) {
    double den = fct((w - s1) / 2) * fct((w - s2) / 2) * fct((w - s3) / 2) * fct((w - s4) / 2) *
                 fct((ii - w) / 2) * fct((ij - w) / 2) * fct((ik - w) / 2);
    if (w % 4 != 0) den = -den;
    omega += fct(w / 2 + 1) / den;
  }
  const double t1 = fct((a - j3) / 2) * fct((j3 + b) / 2) * fct((j3 - b) / 2) / fct(s1 / 2 + 1);
  const double t2 = fct((c - l3) / 2) * fct((l3 + d) / 2) * fct((l3 - d) / 2) / fct(s2 / 2 + 1);
  const double t3 = fct((e - l3) / 2) * fct((l3 + f) / 2) * fct((l3 - f) / 2) / fct(s3 / 2 + 1);
  const double t4 = fct((g - j3) / 2) * fct((j3 + h) / 2) * fct((j3 - h) / 2) / fct(s4 / 2 + 1);
  return omega * std::sqrt(t1 * t2 * t3 * t4);
}

namespace {

struct PlanError : std::runtime_error {
  int code;
  PlanError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ------------------------------------------------------------ operator view
struct OSub {
  int num_up, num_down, down_dif, row_dim, sdim;
  int64_t off;   // device offset of the stored matrix
  bool zero;     // structurally zero (merged sub-block without contributions)
  mutable bool touched = false;   // read by some task of the plan being built
  int32_t merge = -1;             // merged sub-blocks (hmerge): index of its merge record
};
struct OBlk {
  int len = 0, up_dif = 0, down_dif = 0;
  std::vector<OSub> sub;
};
// A block, or its transpose (block_transfer_trans) without copying.
struct OView {
  const OBlk *b;
  bool tr;
  int up_dif() const { return tr ? -b->up_dif : b->up_dif; }
  int down_dif() const { return b->down_dif; }
  int num() const { return (int)b->sub.size(); }
  // labels of sub-block k as seen through the view
  int nu(int k) const { const OSub &s = b->sub[k]; return tr ? s.num_up + b->up_dif : s.num_up; }
  int nd(int k) const { const OSub &s = b->sub[k]; return tr ? s.num_down + s.down_dif : s.num_down; }
  int dd(int k) const { const OSub &s = b->sub[k]; return tr ? -s.down_dif : s.down_dif; }
  int rows(int k) const { const OSub &s = b->sub[k]; return tr ? s.sdim : s.row_dim; }
  int cols(int k) const { const OSub &s = b->sub[k]; return tr ? s.row_dim : s.sdim; }
  bool zero(int k) const { return b->sub[k].zero; }
  // operand for (view matrix)^(extra ? T : N)
  Operand mat(int k, bool extra_t) const {
    const OSub &s = b->sub[k];
    Operand o;
    o.off = s.off;
    o.ld = s.row_dim;
    o.space = SP_OPS;
    o.trans = (int8_t)((tr ? 1 : 0) ^ (extra_t ? 1 : 0));
    o.pad = 0;
    return o;
  }
  // first sub-block with the labels (num_up, num_down[, down_dif])
  int find(int nu_, int nd_, int dd_, bool use_dd) const {
    for (int k = 0; k < num(); ++k)
      if (nu(k) == nu_ && nd(k) == nd_ && (!use_dd || dd(k) == dd_)) return k;
    return -1;
  }
};

// Site operators (Get_site_operator_su2_U0, dmrg_sub.f90:370-473) carry their
// 1x1 values on the host.
struct SiteOp {
  OBlk b;
  std::vector<double> val;
};

struct SiteOps {
  SiteOp eu, sd, ne, si;
};
static SiteOp make_site(int up_dif, int down_dif, std::vector<std::tuple<int, int, int, double>> subs) {
  SiteOp s;
  s.b.len = 1;
  s.b.up_dif = up_dif;
  s.b.down_dif = down_dif;
  for (auto &t : subs) {
    s.b.sub.push_back(OSub{std::get<0>(t), std::get<1>(t), std::get<2>(t), 1, 1, -1, false});
    s.val.push_back(std::get<3>(t));
  }
  return s;
}
static SiteOp site_from_block(const tj_block &b) {
  if (b.num < 1 || !b.sub || !b.data) throw PlanError(TJ_ERR_ARG, "site operator block is empty");
  SiteOp s;
  s.b.len = b.len;
  s.b.up_dif = b.up_dif;
  s.b.down_dif = b.down_dif;
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &q = b.sub[k];
    if (q.row_dim != 1 || q.sdim != 1) throw PlanError(TJ_ERR_ARG, "site operator sub-blocks must be 1x1");
    s.b.sub.push_back(OSub{q.num_up, q.num_down, q.down_dif, 1, 1, -1, false});
    s.val.push_back(b.data[q.off]);
  }
  return s;
}
static SiteOps make_site_ops(int ub) {
  SiteOps o;
  o.eu = make_site(ub, 1, {{0, 0, 1, -std::sqrt(2.0)}});                             // st_elec_up
  o.sd = make_site(0, 2, {{ub, 1, 0, std::sqrt(1.5)}});                              // st_sd
  o.ne = make_site(0, 0, {{0, 0, 0, 0.0}, {ub, 1, 0, std::sqrt(2.0)}});             // num_elec
  o.si = make_site(0, 0, {{0, 0, 0, 1.0}, {ub, 1, 0, std::sqrt(2.0)}});             // st_si
  return o;
}
static int site_find(const SiteOp &s, int nu, int nd, int dd, bool use_dd) {
  for (size_t k = 0; k < s.b.sub.size(); ++k) {
    const OSub &q = s.b.sub[k];
    if (q.num_up == nu && q.num_down == nd && (!use_dd || q.down_dif == dd)) return (int)k;
  }
  return -1;
}

static inline double sgn(char flag, int n) {
  if (flag == 'B') return 1.0;
  if (flag == 'F') return (n % 2 == 0) ? 1.0 : -1.0;
  return 0.0;
}
static inline double m1pow(int n) { return (n % 2) ? -1.0 : 1.0; }

}  // namespace

// Work items of one grouped-GEMM pass.  Every BM x BN tile of every cell
// becomes one or more items; a tile whose tasks carry more than `chunk`
// inner-dimension steps is cut at task boundaries into several items whose
// partial tiles a Reduce record adds up (dot mode needs no reduction: the
// partial dot products are simply summed).  Items are ordered by decreasing
// work so that the dynamic scheduler finishes with the small ones.
void split_tiles(const std::vector<Cell> &cells, const std::vector<Task> &tasks, std::vector<Tile> &tiles,
                 std::vector<Reduce> &red, int64_t &nslots, bool dot_mode, const TuneParams &tp) {
  tiles.clear();
  red.clear();
  nslots = 0;
  double total = 0;
  int64_t ntile = 0;
  for (const Cell &c : cells) {
    double k = 0;
    for (int t = c.t_begin; t < c.t_end; ++t) k += tasks[t].K;
    const int64_t nt = (int64_t)((c.M + BM - 1) / BM) * ((c.N + BN - 1) / BN);
    total += k * nt;
    ntile += nt;
  }
  // aim at tp.items_per_cta items per resident CTA (148 SMs x tp.ctas_per_sm),
  // never below tp.min_ksteps k-steps per item
  const double target =
      std::max((double)tp.min_ksteps, total / (148.0 * std::max(1, tp.ctas_per_sm) * std::max(1, tp.items_per_cta)));
  // tiles in emission order with their weights; sorted below by weight,
  // heaviest first, ties kept in emission order
  std::vector<Tile> all;
  std::vector<std::pair<double, int64_t>> w;
  all.reserve((size_t)ntile + cells.size());
  w.reserve((size_t)ntile + cells.size());
  std::vector<double> chunk_w;
  std::vector<std::pair<int, int>> chunks;
  for (int ci = 0; ci < (int)cells.size(); ++ci) {
    const Cell &c = cells[ci];
    int gb = c.t_begin, ge = c.t_begin;   // GEMM tasks [gb, ge), axpys [ge, t_end)
    while (ge < c.t_end && tasks[ge].R.space != SP_NONE) ++ge;
    chunks.clear();
    double acc = 0;
    int start = gb;
    for (int t = gb; t < ge; ++t) {
      acc += tasks[t].K;
      if (acc >= target && t + 1 < ge) {
        chunks.push_back({start, t + 1});
        start = t + 1;
        acc = 0;
      }
    }
    chunks.push_back({start, ge});
    const bool split = chunks.size() > 1 && !dot_mode;
    chunk_w.assign(chunks.size(), 1.0);
    for (size_t k = 0; k < chunks.size(); ++k)
      for (int t = chunks[k].first; t < chunks[k].second; ++t) chunk_w[k] += tasks[t].K;
    for (int r = 0; r < c.M; r += BM)
      for (int q = 0; q < c.N; q += BN) {
        int slot0 = -1;
        if (split) {
          slot0 = (int)nslots;
          nslots += (int64_t)chunks.size();
          red.push_back(Reduce{ci, r, q, slot0, (int)chunks.size(), ge, c.t_end, 0});
        }
        for (size_t k = 0; k < chunks.size(); ++k) {
          Tile t;
          t.cell = ci;
          t.row0 = r;
          t.col0 = q;
          t.tb = chunks[k].first;
          t.te = chunks[k].second;
          // axpys: by the single owner, or (dot mode) by the first chunk; split tiles get them in the Reduce
          t.ab = ge;
          t.ae = (!split && k == 0) ? c.t_end : ge;
          t.slot = split ? slot0 + (int)k : -1;
          w.push_back({chunk_w[k], (int64_t)all.size()});
          all.push_back(t);
        }
      }
  }
  // the weights take few distinct values: a stable counting sort over their
  // ranks (heaviest first) gives the order of a stable sort by weight
  std::unordered_set<double> distinct;
  for (auto &p : w) distinct.insert(p.first);
  std::vector<double> uniq(distinct.begin(), distinct.end());
  std::sort(uniq.begin(), uniq.end(), std::greater<double>());
  std::vector<int64_t> start(uniq.size() + 1, 0);
  std::vector<int32_t> rank(w.size());
  for (size_t j = 0; j < w.size(); ++j) {
    rank[j] = (int32_t)(std::lower_bound(uniq.begin(), uniq.end(), w[j].first, std::greater<double>()) - uniq.begin());
    ++start[rank[j] + 1];
  }
  for (size_t r = 0; r < uniq.size(); ++r) start[r + 1] += start[r];
  tiles.resize(all.size());
  for (size_t j = 0; j < w.size(); ++j) tiles[start[rank[j]]++] = all[w[j].second];
}

namespace {

// ------------------------------------------------------------------ builder
struct Builder {
  const tj_basis *sbs, *ebs;
  const tj_wave *wave;
  HpsiPlan &plan;
  // psi cells
  std::vector<int> sec_x, sec_y, cell_base;   // per sector: sys map, env map, first cell id
  std::vector<int64_t> cell_off;
  std::vector<int> cell_ld, cell_M, cell_N;
  std::vector<int32_t> cell_rs, cell_cs;       // basis-state index of row 0 / column 0
  int ncells = 0;
  std::map<std::tuple<int, int, int, int>, int> sec_of;   // first sector with the labels
  // tasks
  std::vector<Task> out_tasks;      // phase-2 tasks in emission order
  std::vector<int32_t> out_cell;    // and the output cell of each
  // phase-1 products op(A) * X already emitted: key (operator offset, transpose, psi cell)
  struct ProdKey {
    int64_t off;
    int32_t xc;
    int32_t trans;
    bool operator==(const ProdKey &o) const { return off == o.off && xc == o.xc && trans == o.trans; }
  };
  struct ProdKeyHash {
    size_t operator()(const ProdKey &k) const {
      uint64_t h = (uint64_t)k.off * 0x9e3779b97f4a7c15ull;
      h ^= ((uint64_t)(uint32_t)k.xc << 1 | (uint64_t)(k.trans & 1)) + 0x632be59bd9b4e019ull + (h << 6) + (h >> 2);
      return (size_t)h;
    }
  };
  std::unordered_map<ProdKey, int, ProdKeyHash> prod_id;
  bool dedup = true;
  bool cor_mode = false;   // correlators: keep only the cells that have tasks
  bool want_tiles = true;  // make the FP64 work lists

  Builder(const tj_basis *s, const tj_basis *e, const tj_wave *w, HpsiPlan &p) : sbs(s), ebs(e), wave(w), plan(p) {}

  const tj_basis_sub &SM(int x, int l) const { return sbs->maps[sbs->sub[x].first + l]; }
  const tj_basis_sub &EM(int y, int l) const { return ebs->maps[ebs->sub[y].first + l]; }

  static int find_map(const tj_basis *b, int nu, int nd) {
    for (int x = 0; x < b->num; ++x)
      if (b->sub[x].new_num_up == nu && b->sub[x].new_num_down == nd) return x;
    return -1;
  }

  void init_cells() {
    const int ns = wave->num;
    sec_x.assign(ns, -1);
    sec_y.assign(ns, -1);
    cell_base.assign(ns + 1, 0);
    for (int i = 0; i < ns; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      auto key = std::make_tuple(w.sys_num_up, w.sys_num_down, w.env_num_up, w.env_num_down);
      if (!sec_of.count(key)) sec_of[key] = i;
      int x = find_map(sbs, w.sys_num_up, w.sys_num_down);
      int y = find_map(ebs, w.env_num_up, w.env_num_down);
      if (x < 0 || y < 0) throw PlanError(TJ_ERR_QN, "wave sector without a matching basis sector");
      if (sbs->sub[x].dim != w.sys_dim || ebs->sub[y].dim != w.env_dim)
        throw PlanError(TJ_ERR_ARG, "wave sector dimensions differ from the basis");
      sec_x[i] = x;
      sec_y[i] = y;
      cell_base[i + 1] = cell_base[i] + sbs->sub[x].num * ebs->sub[y].num;
    }
    ncells = cell_base[ns];
    cell_off.resize(ncells);
    cell_ld.resize(ncells);
    cell_M.resize(ncells);
    cell_N.resize(ncells);
    cell_rs.resize(ncells);
    cell_cs.resize(ncells);
    // basis states of the (unenlarged) block: every sub-block (bl, st) of an
    // enlarged sector spans all states of its block sector bl (site sectors
    // are one-dimensional), so row i of any cell with block label bl is block
    // state first(bl) + i
    auto block_states = [](const tj_basis *b, std::map<std::pair<int, int>, int32_t> &first) {
      int32_t n = 0;
      for (int x = 0; x < b->num; ++x)
        for (int l = 0; l < b->sub[x].num; ++l) {
          const tj_basis_sub &m = b->maps[b->sub[x].first + l];
          auto key = std::make_pair(m.bl_num_up, m.bl_num_down);
          if (!first.count(key)) {
            first[key] = n;
            n += m.sdim;
          }
        }
      return n;
    };
    std::map<std::pair<int, int>, int32_t> sys_first, env_first;
    plan.n_sys_states = block_states(sbs, sys_first);
    plan.n_env_states = block_states(ebs, env_first);
    for (int i = 0; i < ns; ++i) {
      const int x = sec_x[i], y = sec_y[i], ny = ebs->sub[y].num;
      for (int m = 0; m < sbs->sub[x].num; ++m)
        for (int n = 0; n < ny; ++n) {
          const int c = cell_base[i] + m * ny + n;
          const tj_basis_sub &a = SM(x, m), &b = EM(y, n);
          cell_off[c] = wave->sub[i].off + (int64_t)b.spos * wave->sub[i].sys_dim + a.spos;
          cell_ld[c] = wave->sub[i].sys_dim;
          cell_M[c] = a.sdim;
          cell_rs[c] = sys_first[std::make_pair(a.bl_num_up, a.bl_num_down)];
          cell_cs[c] = env_first[std::make_pair(b.bl_num_up, b.bl_num_down)];
          cell_N[c] = b.sdim;
        }
    }
    out_tasks.clear();
    out_cell.clear();
    // capacities from the cell count (a cell has a few terms of each kind),
    // so that the lists are not regrown and rehashed while the terms are emitted
    out_tasks.reserve((size_t)ncells * 4);
    out_cell.reserve((size_t)ncells * 4);
    prod_id.reserve((size_t)ncells * 2);
    plan.cells1.reserve((size_t)ncells * 2);
    plan.tasks1.reserve((size_t)ncells * 2);
    plan.cell1_row_state.reserve((size_t)ncells * 2);
  }
  int cell(int i, int m, int n) const { return cell_base[i] + m * ebs->sub[sec_y[i]].num + n; }
  int find_sec(int su, int sd, int eu, int ed) const {
    auto it = sec_of.find(std::make_tuple(su, sd, eu, ed));
    return it == sec_of.end() ? -1 : it->second;
  }
  Operand xop(int c) const {
    Operand o;
    o.off = cell_off[c];
    o.ld = cell_ld[c];
    o.space = SP_PSI;
    o.trans = 0;
    o.pad = 0;
    return o;
  }
  static Operand none() {
    Operand o;
    std::memset(&o, 0, sizeof o);
    return o;
  }
  static void touch(const OView &V, int k) { V.b->sub[k].touched = true; }
  void add_task(int oc, const Task &t) {
    out_tasks.push_back(t);
    out_cell.push_back(oc);
  }

  // out(oc) += coef * op(A) * X(xc); op(A) is (rows x K)
  void emitL(int oc, const OView &A, int ka, bool at, int xc, double coef, double ref_extra = 0.0) {
    if (A.zero(ka) || coef == 0.0) return;
    const int rows = at ? A.cols(ka) : A.rows(ka), K = at ? A.rows(ka) : A.cols(ka);
    if (rows != cell_M[oc] || K != cell_M[xc] || cell_N[xc] != cell_N[oc])
      throw PlanError(TJ_ERR_ARG, "operator sub-block does not match the basis dimensions");
    Task t;
    t.L = A.mat(ka, at);
    t.R = xop(xc);
    t.coef = coef;
    t.K = K;
    t.pad = 0;
    touch(A, ka);
    add_task(oc, t);
    const double f = 2.0 * rows * cell_N[oc] * (double)K;
    plan.flops += f;
    plan.flops_ref += f + ref_extra;
  }
  // out(oc) += coef * X(xc) * op(B); op(B) is (K x cols)
  void emitR(int oc, int xc, const OView &B, int kb, bool bt, double coef) {
    if (B.zero(kb) || coef == 0.0) return;
    const int K = bt ? B.cols(kb) : B.rows(kb), cols = bt ? B.rows(kb) : B.cols(kb);
    if (cols != cell_N[oc] || K != cell_N[xc] || cell_M[xc] != cell_M[oc])
      throw PlanError(TJ_ERR_ARG, "operator sub-block does not match the basis dimensions");
    Task t;
    t.L = xop(xc);
    t.R = B.mat(kb, bt);
    t.coef = coef;
    t.K = K;
    t.pad = 0;
    touch(B, kb);
    add_task(oc, t);
    const double f = 2.0 * cell_M[oc] * cols * (double)K;
    plan.flops += f;
    plan.flops_ref += f;
  }
  // out(oc) += coef * X(xc)
  void emitAxpy(int oc, int xc, double coef) {
    if (coef == 0.0) return;
    if (cell_M[oc] != cell_M[xc] || cell_N[oc] != cell_N[xc])
      throw PlanError(TJ_ERR_ARG, "site term between cells of different size");
    Task t;
    t.L = xop(xc);
    t.R = none();
    t.coef = coef;
    t.K = 0;
    t.pad = 0;
    add_task(oc, t);
    plan.flops += 2.0 * cell_M[oc] * cell_N[oc];
    plan.flops_ref += 2.0 * cell_M[oc] * cell_N[oc];
  }
  // out(oc) += coef * [op(A) * X(xc)] * op(B)   (phase-1 product, then phase-2 task)
  void emit2(int oc, const OView &A, int ka, bool at, int xc, const OView &B, int kb, bool bt, double coef) {
    if (A.zero(ka) || B.zero(kb) || coef == 0.0) return;
    const int M = at ? A.cols(ka) : A.rows(ka), K1 = at ? A.rows(ka) : A.cols(ka);
    const int K2 = bt ? B.cols(kb) : B.rows(kb), N = bt ? B.rows(kb) : B.cols(kb);
    if (M != cell_M[oc] || N != cell_N[oc] || K1 != cell_M[xc] || K2 != cell_N[xc])
      throw PlanError(TJ_ERR_ARG, "operator sub-block does not match the basis dimensions");
    Operand a = A.mat(ka, at);
    const ProdKey key{a.off, xc, (int32_t)a.trans};
    int pid;
    auto it = dedup ? prod_id.find(key) : prod_id.end();
    if (it != prod_id.end()) {
      pid = it->second;
    } else {
      pid = (int)plan.cells1.size();
      if (dedup) prod_id[key] = pid;
      Cell c;
      std::memset(&c, 0, sizeof c);
      c.off = plan.scratch_len;
      c.ld = M;
      c.M = M;
      c.N = K2;
      c.space = SP_SCR;
      c.t_begin = (int)plan.tasks1.size();
      c.t_end = c.t_begin + 1;
      plan.scratch_len += ((int64_t)M * K2 + 3) / 4 * 4;
      plan.cells1.push_back(c);
      plan.cell1_row_state.push_back(cell_rs[oc]);
      Task t;
      t.L = a;
      t.R = xop(xc);
      t.coef = 1.0;
      t.K = K1;
      t.pad = 0;
      touch(A, ka);
      plan.tasks1.push_back(t);
      plan.flops += 2.0 * M * K2 * (double)K1;
    }
    Task t;
    t.L.off = plan.cells1[pid].off;
    t.L.ld = M;
    t.L.space = SP_SCR;
    t.L.trans = 0;
    t.L.pad = 0;
    t.R = B.mat(kb, bt);
    t.coef = coef;
    t.K = K2;
    t.pad = 0;
    touch(B, kb);
    add_task(oc, t);
    plan.flops += 2.0 * M * N * (double)K2;
    plan.flops_ref += 2.0 * M * K2 * (double)K1 + 2.0 * M * N * (double)K2;
  }

  // ============================================================ term kernels
  // block_vec_dia (get_sys.f90:1242-1289)
  void block_vec_dia(const OView &H, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &q = SM(x, m);
        const double c1 = coef / std::sqrt(1.0 + q.bl_num_down);
        const int k = H.find(q.bl_num_up, q.bl_num_down, 0, false);
        if (k < 0) continue;
        for (int n = 0; n < ebs->sub[y].num; ++n) emitL(cell(i, m, n), H, k, false, cell(i, m, n), c1);
      }
    }
  }
  // vec_block_dia (get_sys.f90:1293-1340)
  void vec_block_dia(const OView &H, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int n = 0; n < ebs->sub[y].num; ++n) {
        const tj_basis_sub &q = EM(y, n);
        const double c1 = coef / std::sqrt(1.0 + q.bl_num_down);
        const int k = H.find(q.bl_num_up, q.bl_num_down, 0, false);
        if (k < 0) continue;
        for (int m = 0; m < sbs->sub[x].num; ++m) emitR(cell(i, m, n), cell(i, m, n), H, k, true, c1);
      }
    }
  }
  // site_vec_site_dia (get_sys.f90:1609-1705)
  void site_vec_site_dia(const SiteOp &sst, const SiteOp &est, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &qs = SM(x, m);
        const int ks = site_find(sst, qs.st_num_up, qs.st_num_down, 0, false);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &qe = EM(y, n);
          const int ke = site_find(est, qe.st_num_up, qe.st_num_down, 0, false);
          if (ks < 0 || ke < 0) continue;
          double ct = coef * sst.val[ks] * est.val[ke];
          ct = ct / std::sqrt((1.0 + qs.st_num_down) * (1.0 + qe.st_num_down));
          emitAxpy(cell(i, m, n), cell(i, m, n), ct);
        }
      }
    }
  }
  // sectors of a basis with the labels (new_num_up, new_num_down), in index
  // order; built on first use
  struct SecIndex {
    std::unordered_map<uint64_t, std::vector<int>> by_lab;
    bool ready = false;
  };
  mutable SecIndex sys_idx, env_idx;
  static const std::vector<int> *sectors_with(const tj_basis *b, SecIndex &ix, int nu, int nd) {
    auto key = [](int u, int d) { return (uint64_t)(uint32_t)u << 32 | (uint32_t)d; };
    if (!ix.ready) {
      for (int k = 0; k < b->num; ++k) ix.by_lab[key(b->sub[k].new_num_up, b->sub[k].new_num_down)].push_back(k);
      ix.ready = true;
    }
    auto it = ix.by_lab.find(key(nu, nd));
    return it == ix.by_lab.end() ? nullptr : &it->second;
  }
  // locate the system sub-block of the sector with labels (nu, nd) satisfying pred
  template <class P>
  bool find_sys(int nu, int nd, P pred, int &xk, int &l) const {
    const std::vector<int> *ks = sectors_with(sbs, sys_idx, nu, nd);
    if (!ks) return false;
    for (int k : *ks)
      for (int q = 0; q < sbs->sub[k].num; ++q)
        if (pred(SM(k, q))) { xk = k; l = q; return true; }
    return false;
  }
  template <class P>
  bool find_env(int nu, int nd, P pred, int &yk, int &l) const {
    const std::vector<int> *ks = sectors_with(ebs, env_idx, nu, nd);
    if (!ks) return false;
    for (int k : *ks)
      for (int q = 0; q < ebs->sub[k].num; ++q)
        if (pred(EM(k, q))) { yk = k; l = q; return true; }
    return false;
  }
  // sub-block index l of map x, as a cell row/column index of sector ko
  int sys_index_in(int ko, int xk, int l) const {
    if (sec_x[ko] != xk) throw PlanError(TJ_ERR_QN, "basis sector mismatch");
    return l;
  }
  int env_index_in(int ko, int yk, int l) const {
    if (sec_y[ko] != yk) throw PlanError(TJ_ERR_QN, "basis sector mismatch");
    return l;
  }

  // site_vec_site_ndia (get_sys.f90:3761-4124, live 3794-3994)
  void site_vec_site_ndia(const SiteOp &sst, char fst, const SiteOp &est, char fet, double coef) {
    const int up = sst.b.up_dif, d1 = sst.b.down_dif;
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          for (int sdd1 = -sst.b.down_dif; sdd1 <= sst.b.down_dif; sdd1 += 2) {
            const int ks = site_find(sst, ms.st_num_up, ms.st_num_down, sdd1, true);
            const int nss_up = ms.st_num_up + up, nss_dn = ms.st_num_down + sdd1;
            for (int sdd2 = -est.b.down_dif; sdd2 <= est.b.down_dif; sdd2 += 2) {
              const int nes_up = me.st_num_up - up, nes_dn = me.st_num_down - sdd2;
              const int ke = site_find(est, nes_up, nes_dn, sdd2, true);
              if (ks < 0 || ke < 0) continue;
              const int nsu = su + up, neu = eu - up;
              for (int nsd = std::abs(sd - sst.b.down_dif); nsd <= sd + sst.b.down_dif; nsd += 2) {
                const int ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nss_up && q.st_num_down == nss_dn && q.bl_num_down == ms.bl_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nes_up && q.st_num_down == nes_dn && q.bl_num_down == me.bl_num_down; }, yk, le))
                  continue;
                const int ko = find_sec(nsu, nsd, neu, ned);
                if (ko < 0) continue;
                const double ct = sgn(fst, ms.bl_num_down) * sgn(fet, sd) * coef;
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.st_num_down, j5 = ms.bl_num_down, j6 = nss_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.st_num_down, j55 = me.bl_num_down, j66 = nes_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                const double c11 = w6j(j11, j22, j33, j44, j55, j66);
                if (c11 == 0.0) continue;
                c1 *= c11;
                if (c1 == 0.0) continue;
                c1 *= std::sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                if (((j55 + j44 + j11 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                c1 = ct * c1 * sst.val[ks] * est.val[ke];
                const int oc = cell(ko, sys_index_in(ko, xk, ls), env_index_in(ko, yk, le));
                emitAxpy(oc, cell(i, m, n), c1);
                if (d1 == 1) emitAxpy(cell(i, m, n), oc, c1);
              }
            }
          }
        }
      }
    }
  }
  // block_site_vec_ndia (get_sys.f90:2016-2265, live 2047-2170)
  void block_site_vec_ndia(const OView &bl, const SiteOp &st, char fst, double coef) {
    const int up = bl.up_dif(), d1 = bl.down_dif();
    if (up != st.b.up_dif || d1 != st.b.down_dif) throw PlanError(TJ_ERR_QN, "Quantum number error in block_site_vec");
    for (int i = 0; i < wave->num; ++i) {
      const int sd = wave->sub[i].sys_num_down;
      const int k = sec_x[i], y = sec_y[i];
      for (int x = 0; x < sbs->sub[k].num; ++x) {
        const tj_basis_sub &q = SM(k, x);
        for (int dd = -d1; dd <= d1; dd += 2)
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int kb = bl.find(q.bl_num_up, q.bl_num_down, dd, true);
            const int nst_up = q.st_num_up - up, nst_dn = q.st_num_down - sdd;
            const int ks = site_find(st, nst_up, nst_dn, sdd, true);
            const int nbl_up = q.bl_num_up + up, nbl_dn = q.bl_num_down + dd;
            if (kb < 0 || ks < 0) continue;
            int np = -1;
            for (int yy = 0; yy < sbs->sub[k].num; ++yy) {
              const tj_basis_sub &r = SM(k, yy);
              if (r.bl_num_up == nbl_up && r.bl_num_down == nbl_dn && r.st_num_up == nst_up && r.st_num_down == nst_dn) {
                np = yy;
                break;
              }
            }
            if (np < 0) continue;
            const int j1 = nbl_dn, j2 = q.bl_num_down, j3 = d1, j4 = q.st_num_down, j5 = nst_dn, j6 = sd;
            double c1 = w6j(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * m1pow((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + d1);
            const double ct = sgn(fst, q.bl_num_down) * c1 * coef * st.val[ks];
            for (int n = 0; n < ebs->sub[y].num; ++n) {
              emitL(cell(i, np, n), bl, kb, false, cell(i, x, n), ct);
              if (d1 == 1) emitL(cell(i, x, n), bl, kb, true, cell(i, np, n), ct);
            }
          }
      }
    }
  }
  // block_site_vec_dia (get_sys.f90:1460-1530)
  void block_site_vec_dia(const OView &bl, const SiteOp &st, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &q = SM(x, m);
        const int kb = bl.find(q.bl_num_up, q.bl_num_down, 0, false);
        const int ks = site_find(st, q.st_num_up, q.st_num_down, 0, false);
        if (kb < 0 || ks < 0) continue;
        double ct = coef * st.val[ks];
        ct = ct / std::sqrt((1.0 + q.bl_num_down) * (1.0 + q.st_num_down));
        for (int n = 0; n < ebs->sub[y].num; ++n) emitL(cell(i, m, n), bl, kb, false, cell(i, m, n), ct);
      }
    }
  }
  // vec_block_site_ndia (get_sys.f90:2269-2552, live 2301-2446)
  void vec_block_site_ndia(const OView &bl, char fbl, const SiteOp &st, char fst, double coef) {
    const int up = bl.up_dif(), d1 = bl.down_dif();
    if (up != st.b.up_dif || d1 != st.b.down_dif) throw PlanError(TJ_ERR_QN, "Quantum number error in vec_block_site");
    for (int i = 0; i < wave->num; ++i) {
      const int sd = wave->sub[i].sys_num_down, ed = wave->sub[i].env_num_down;
      const int xs = sec_x[i], k = sec_y[i];
      for (int x = 0; x < ebs->sub[k].num; ++x) {
        const tj_basis_sub &q = EM(k, x);
        for (int bdd = -d1; bdd <= d1; bdd += 2) {
          const int kb = bl.find(q.bl_num_up, q.bl_num_down, bdd, true);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int nst_up = q.st_num_up - up, nst_dn = q.st_num_down - sdd;
            const int ks = site_find(st, nst_up, nst_dn, sdd, true);
            const int nbl_up = q.bl_num_up + up, nbl_dn = q.bl_num_down + bdd;
            if (ks < 0 || kb < 0) continue;
            int np = -1;
            for (int yy = 0; yy < ebs->sub[k].num; ++yy) {
              const tj_basis_sub &r = EM(k, yy);
              if (r.bl_num_up == nbl_up && r.bl_num_down == nbl_dn && r.st_num_up == nst_up && r.st_num_down == nst_dn) {
                np = yy;
                break;
              }
            }
            if (np < 0) continue;
            const int j1 = nbl_dn, j2 = q.bl_num_down, j3 = d1, j4 = q.st_num_down, j5 = nst_dn, j6 = ed;
            double c1 = w6j(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * m1pow((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + d1);
            const double ct = sgn(fbl, sd + nst_dn) * sgn(fst, sd) * c1 * coef * st.val[ks];
            for (int m = 0; m < sbs->sub[xs].num; ++m) {
              emitR(cell(i, m, np), cell(i, m, x), bl, kb, true, ct);
              if (d1 == 1) emitR(cell(i, m, x), cell(i, m, np), bl, kb, false, ct);
            }
          }
        }
      }
    }
  }
  // vec_block_site_dia (get_sys.f90:1534-1605)
  void vec_block_site_dia(const OView &bl, const SiteOp &st, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int n = 0; n < ebs->sub[y].num; ++n) {
        const tj_basis_sub &q = EM(y, n);
        const int kb = bl.find(q.bl_num_up, q.bl_num_down, 0, false);
        const int ks = site_find(st, q.st_num_up, q.st_num_down, 0, false);
        if (kb < 0 || ks < 0) continue;
        double ct = coef * st.val[ks];
        ct = ct / std::sqrt((1.0 + q.bl_num_down) * (1.0 + q.st_num_down));
        for (int m = 0; m < sbs->sub[x].num; ++m) emitR(cell(i, m, n), cell(i, m, n), bl, kb, true, ct);
      }
    }
  }
  // block_vec_site_ndia (get_sys.f90:2984-3351, live 3021-3209)
  void block_vec_site_ndia(const OView &bl, const SiteOp &st, char fet, double coef) {
    const int up = bl.up_dif(), d1 = bl.down_dif();
    if (up != st.b.up_dif || d1 != st.b.down_dif) throw PlanError(TJ_ERR_QN, "Quantum number error in block_vec_site");
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          for (int bdd = -d1; bdd <= d1; bdd += 2) {
            const int nsb_up = ms.bl_num_up + up, nsb_dn = ms.bl_num_down + bdd;
            const int kb = bl.find(ms.bl_num_up, ms.bl_num_down, bdd, true);
            for (int sdd = -st.b.down_dif; sdd <= st.b.down_dif; sdd += 2) {
              const int nes_up = me.st_num_up - up, nes_dn = me.st_num_down - sdd;
              const int ks = site_find(st, nes_up, nes_dn, sdd, true);
              if (kb < 0 || ks < 0) continue;
              const int nsu = su + up, neu = eu - up;
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == nsb_up && q.bl_num_down == nsb_dn && q.st_num_down == ms.st_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nes_up && q.st_num_down == nes_dn && q.bl_num_down == me.bl_num_down; }, yk, le))
                  continue;
                const int ko = find_sec(nsu, nsd, neu, ned);
                if (ko < 0) continue;
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.bl_num_down, j5 = ms.st_num_down, j6 = nsb_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.st_num_down, j55 = me.bl_num_down, j66 = nes_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                const double c11 = w6j(j11, j22, j33, j44, j55, j66);
                if (c11 == 0.0) continue;
                c1 *= c11;
                if (c1 == 0.0) continue;
                c1 *= std::sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                if (((j6 + j5 + j3 + j2) / 2 + (j55 + j44 + j11 + j22) / 2) % 2 != 0) c1 = -c1;
                const double ct = sgn(fet, sd) * c1 * coef * st.val[ks];
                const int oc = cell(ko, sys_index_in(ko, xk, ls), env_index_in(ko, yk, le));
                emitL(oc, bl, kb, false, cell(i, m, n), ct);
                if (d1 == 1) emitL(cell(i, m, n), bl, kb, true, oc, ct);
              }
            }
          }
        }
      }
    }
  }
  // block_vec_site_dia (get_sys.f90:1709-1805)
  void block_vec_site_dia(const OView &bl, const SiteOp &st, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        const int kb = bl.find(ms.bl_num_up, ms.bl_num_down, 0, false);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          const int ks = site_find(st, me.st_num_up, me.st_num_down, 0, false);
          if (kb < 0 || ks < 0) continue;
          double ct = coef * st.val[ks];
          ct = ct / std::sqrt((1.0 + me.st_num_down) * (1.0 + ms.bl_num_down));
          emitL(cell(i, m, n), bl, kb, false, cell(i, m, n), ct);
        }
      }
    }
  }
  // site_vec_block_ndia (get_sys.f90:3355-3757, live 3391-3604); bl is a transposed view
  void site_vec_block_ndia(const SiteOp &st, char fst, const OView &bl, char fel, double coef) {
    const int up = st.b.up_dif, d1 = st.b.down_dif;
    if (up != bl.up_dif() || d1 != bl.down_dif()) throw PlanError(TJ_ERR_QN, "Quantum number error in site_vec_block");
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int nss_up = ms.st_num_up + up, nss_dn = ms.st_num_down + sdd;
            const int ks = site_find(st, ms.st_num_up, ms.st_num_down, sdd, true);
            for (int bdd = -bl.down_dif(); bdd <= bl.down_dif(); bdd += 2) {
              const int neb_up = me.bl_num_up - up, neb_dn = me.bl_num_down - bdd;
              const int kb = bl.find(neb_up, neb_dn, bdd, true);
              if (ks < 0 || kb < 0) continue;
              const int nsu = su + up, neu = eu - up;
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nss_up && q.st_num_down == nss_dn && q.bl_num_down == ms.bl_num_down &&
                             q.bl_num_up == ms.bl_num_up; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == neb_up && q.bl_num_down == neb_dn && q.st_num_up == me.st_num_up &&
                             q.st_num_down == me.st_num_down; }, yk, le))
                  continue;
                const int ko = find_sec(nsu, nsd, neu, ned);
                if (ko < 0) continue;
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.st_num_down, j5 = ms.bl_num_down, j6 = nss_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.bl_num_down, j55 = me.st_num_down, j66 = neb_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                const double c11 = w6j(j11, j22, j33, j44, j55, j66);
                if (c11 == 0.0) continue;
                c1 *= c11;
                if (c1 == 0.0) continue;
                c1 *= std::sqrt((1.0 + j11) * (j33 + 1.0) / (1.0 + d1));
                if (((j66 + j55 + j33 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                const double ct = sgn(fst, ms.bl_num_down) * sgn(fel, sd + me.st_num_down) * c1 * coef * st.val[ks];
                const int oc = cell(ko, sys_index_in(ko, xk, ls), env_index_in(ko, yk, le));
                emitR(oc, cell(i, m, n), bl, kb, false, ct);
                if (d1 == 1) emitR(cell(i, m, n), oc, bl, kb, true, ct);
              }
            }
          }
        }
      }
    }
  }
  // site_vec_block_dia (get_sys.f90:1809-1906)
  void site_vec_block_dia(const SiteOp &st, const OView &bl, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        const int ks = site_find(st, ms.st_num_up, ms.st_num_down, 0, false);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          const int kb = bl.find(me.bl_num_up, me.bl_num_down, 0, false);
          if (ks < 0 || kb < 0) continue;
          double ct = coef * st.val[ks];
          ct = ct / std::sqrt((1.0 + me.bl_num_down) * (1.0 + ms.st_num_down));
          emitR(cell(i, m, n), cell(i, m, n), bl, kb, true, ct);
        }
      }
    }
  }
  // block_vec_block_ndia (get_sys.f90:2555-2981, live 2595-2834); ebl is a transposed view
  void block_vec_block_ndia(const OView &sbl, const OView &ebl, char fel, double coef) {
    const int up = sbl.up_dif(), d1 = sbl.down_dif();
    if (up != ebl.up_dif() || d1 != ebl.down_dif()) throw PlanError(TJ_ERR_QN, "Quantum number error in block_vec_block");
    // The operator sub-block, the target basis sub-block and the 6j symbol of
    // each side depend on one side's sub-block, its spin step dd and the new
    // sector spin nsd only, so they are tabulated once per sector; the loops
    // below visit (m, n, dd, edd, nsd) in the order of the Fortran loops and
    // do the same floating-point operations.
    const int nq = d1 + 1;  // dd = -d1, -d1 + 2, ..., d1
    struct Half { int k, blk, l, hs; double w; };
    std::vector<Half> st, et;
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i], nm = sbs->sub[x].num, nn = ebs->sub[y].num;
      const int nsd0 = std::abs(sd - d1), nt = (sd + d1 - nsd0) / 2 + 1;
      const int nsu = su + up, neu = eu - up;
      int ko[8];
      if (nt > 8) throw PlanError(TJ_ERR_QN, "operator spin step too large in block_vec_block");
      for (int t = 0; t < nt; ++t) ko[t] = find_sec(nsu, nsd0 + 2 * t, neu, nsd0 + 2 * t);
      st.assign((size_t)nm * nq * nt, Half{-1, -1, -1, 0, 0.0});
      et.assign((size_t)nn * nq * nt, Half{-1, -1, -1, 0, 0.0});
      for (int m = 0; m < nm; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        for (int q = 0; q < nq; ++q) {
          const int dd = -d1 + 2 * q;
          const int ks = sbl.find(ms.bl_num_up, ms.bl_num_down, dd, true);
          const int nsb_up = ms.bl_num_up + up, nsb_dn = ms.bl_num_down + dd;
          for (int t = 0; t < nt; ++t) {
            Half &h = st[((size_t)m * nq + q) * nt + t];
            h.k = ks;
            if (ks < 0) continue;
            const int nsd = nsd0 + 2 * t;
            if (!find_sys(nsu, nsd, [&](const tj_basis_sub &b) {
                  return b.bl_num_up == nsb_up && b.bl_num_down == nsb_dn && b.st_num_down == ms.st_num_down &&
                         b.st_num_up == ms.st_num_up; }, h.blk, h.l))
              continue;
            h.w = w6j(nsd, d1, sd, ms.bl_num_down, ms.st_num_down, nsb_dn);
            h.hs = (nsb_dn + ms.st_num_down + sd + d1) / 2;
          }
        }
      }
      for (int n = 0; n < nn; ++n) {
        const tj_basis_sub &me = EM(y, n);
        for (int q = 0; q < nq; ++q) {
          const int edd = -d1 + 2 * q;
          const int neb_up = me.bl_num_up - up, neb_dn = me.bl_num_down - edd;
          const int ke = ebl.find(neb_up, neb_dn, edd, true);
          for (int t = 0; t < nt; ++t) {
            Half &h = et[((size_t)n * nq + q) * nt + t];
            h.k = ke;
            if (ke < 0) continue;
            const int ned = nsd0 + 2 * t;
            if (!find_env(neu, ned, [&](const tj_basis_sub &b) {
                  return b.bl_num_up == neb_up && b.bl_num_down == neb_dn && b.st_num_down == me.st_num_down &&
                         b.st_num_up == me.st_num_up; }, h.blk, h.l))
              continue;
            h.w = w6j(ned, d1, ed, me.bl_num_down, me.st_num_down, neb_dn);
            h.hs = (neb_dn + me.st_num_down + ed + d1) / 2;
          }
        }
      }
      for (int m = 0; m < nm; ++m)
        for (int n = 0; n < nn; ++n) {
          const tj_basis_sub &me = EM(y, n);
          const int xc = cell(i, m, n);
          const double sg = sgn(fel, sd + me.st_num_down);
          for (int q = 0; q < nq; ++q)
            for (int eq = 0; eq < nq; ++eq)
              for (int t = 0; t < nt; ++t) {
                const Half &hs = st[((size_t)m * nq + q) * nt + t], &he = et[((size_t)n * nq + eq) * nt + t];
                if (hs.k < 0 || he.k < 0 || hs.blk < 0 || he.blk < 0 || ko[t] < 0) continue;
                double c1 = hs.w;
                if (c1 == 0.0) continue;
                const double c11 = he.w;
                if (c11 == 0.0) continue;
                c1 *= c11;
                if (c1 == 0.0) continue;
                const int nsd = nsd0 + 2 * t;
                c1 *= std::sqrt((1.0 + nsd) * (1.0 + ed) / (1.0 + d1));
                if ((hs.hs + he.hs) % 2 == 1) c1 = -c1;
                const double ct = sg * coef * c1;
                const int oc = cell(ko[t], sys_index_in(ko[t], hs.blk, hs.l), env_index_in(ko[t], he.blk, he.l));
                emit2(oc, sbl, hs.k, false, xc, ebl, he.k, false, ct);
                if (d1 == 1) emit2(xc, sbl, hs.k, true, oc, ebl, he.k, true, ct);
              }
        }
    }
  }
  // block_vec_block_dia (get_sys.f90:1910-2012)
  void block_vec_block_dia(const OView &sbl, const OView &ebl, double coef) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        const int ks = sbl.find(ms.bl_num_up, ms.bl_num_down, 0, false);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          const int ke = ebl.find(me.bl_num_up, me.bl_num_down, 0, false);
          if (ks < 0 || ke < 0) continue;
          if (ms.sdim * me.sdim == 0) throw PlanError(TJ_ERR_ARG, "block_vec_block_dia: empty tile");
          const double c1 = coef / std::sqrt((1.0 + me.bl_num_down) * (1.0 + ms.bl_num_down));
          emit2(cell(i, m, n), sbl, ks, false, cell(i, m, n), ebl, ke, true, c1);
        }
      }
    }
  }

  // -------------------------------------------------------------- finalise
  void finalize() {
    // phase-2 cells: every cell of the output vector, its GEMM tasks first and
    // its axpy tasks last (the kernel applies axpys in its epilogue), each
    // group in emission order
    std::vector<int32_t> pg(ncells, 0), pa(ncells, 0);
    for (size_t j = 0; j < out_tasks.size(); ++j) ++(out_tasks[j].R.space != SP_NONE ? pg : pa)[out_cell[j]];
    plan.cells2.clear();
    plan.tasks2.clear();
    int32_t pos = 0;
    for (int c = 0; c < ncells; ++c) {
      const int32_t ng = pg[c], na = pa[c];
      if (cor_mode && ng + na == 0) continue;
      Cell cl;
      std::memset(&cl, 0, sizeof cl);
      cl.off = cell_off[c];
      cl.ld = cell_ld[c];
      cl.M = cell_M[c];
      cl.N = cell_N[c];
      cl.space = SP_PSI;
      cl.t_begin = pos;
      pg[c] = pos;
      pa[c] = pos + ng;
      pos += ng + na;
      cl.t_end = pos;
      plan.cells2.push_back(cl);
      plan.cell2_row_state.push_back(cell_rs[c]);
      plan.cell2_col_state.push_back(cell_cs[c]);
    }
    plan.tasks2.resize(pos);
    for (size_t j = 0; j < out_tasks.size(); ++j) {
      const Task &t = out_tasks[j];
      plan.tasks2[t.R.space != SP_NONE ? pg[out_cell[j]]++ : pa[out_cell[j]]++] = t;
    }
    auto make_tiles = [&](const std::vector<Cell> &cells, const std::vector<Task> &tasks,
                          std::vector<Tile> &tiles, std::vector<Reduce> &red, int64_t &nslots) {
      split_tiles(cells, tasks, tiles, red, nslots, cor_mode);
    };
    if (want_tiles) {
      make_tiles(plan.cells1, plan.tasks1, plan.tiles1, plan.red1, plan.nslots1);
      make_tiles(plan.cells2, plan.tasks2, plan.tiles2, plan.red2, plan.nslots2);
    }
  }
};

// ------------------------------------------------------------- model copy
struct Model {
  int len = 0;
  OBlk ham;
  std::vector<std::array<OBlk, 5>> sub;   // input slots
  std::array<OBlk, 5> snc[2];             // merged (hmerge)
  std::vector<std::array<OBlk, 5>> sub_s; // merged (hmerge)
};
enum { EU = 0, ED = 1, SD = 2, SZ = 3, SN = 4 };

static int64_t align4(int64_t x) { return (x + 3) / 4 * 4; }

static void load_block(const tj_block &b, OBlk &o, HpsiPlan &plan) {
  o.len = b.len;
  o.up_dif = b.up_dif;
  o.down_dif = b.down_dif;
  o.sub.clear();
  if (b.num < 0 || (b.num > 0 && (!b.sub || !b.data))) throw PlanError(TJ_ERR_ARG, "block with null sub/data");
  // one host-to-device copy per block: the span of its sub-block matrices
  int64_t lo = LLONG_MAX, hi = 0;
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &s = b.sub[k];
    if (s.row_dim < 0 || s.sdim < 0 || s.off < 0) throw PlanError(TJ_ERR_ARG, "negative sub-block size");
    lo = std::min(lo, (int64_t)s.off);
    hi = std::max(hi, (int64_t)s.off + (int64_t)s.row_dim * s.sdim);
  }
  if (b.num == 0) return;
  const int64_t base = plan.ops_len;
  plan.uploads.push_back({b.data + lo, hi - lo, base});
  plan.ops_len += align4(hi - lo);
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &s = b.sub[k];
    OSub q{s.num_up, s.num_down, s.down_dif, s.row_dim, s.sdim, base + (s.off - lo), false};
    plan.sub_extent.push_back({q.off, (int64_t)s.row_dim * s.sdim});
    o.sub.push_back(q);
  }
}
static void load_model(const tj_model *m, Model &o, HpsiPlan &plan) {
  if (!m || m->nsub < 1 || !m->sub) throw PlanError(TJ_ERR_ARG, "model needs sub(1:nsub), nsub >= 1");
  o.len = m->len;
  load_block(m->ham, o.ham, plan);
  o.sub.resize(m->nsub);
  for (int i = 0; i < m->nsub; ++i) {
    load_block(m->sub[i].elec_up, o.sub[i][EU], plan);
    load_block(m->sub[i].elec_down, o.sub[i][ED], plan);
    load_block(m->sub[i].spin_sd, o.sub[i][SD], plan);
    o.sub[i][SZ] = OBlk();
    load_block(m->sub[i].num_sn, o.sub[i][SN], plan);
  }
}
// block_pass_info (block.f90:1741-1768): zero block with the structure of `old`
static void pass_info(const OBlk &old, OBlk &nw, HpsiPlan &plan) {
  nw = old;
  for (OSub &s : nw.sub) {
    const int64_t n = (int64_t)s.row_dim * s.sdim;
    s.off = plan.ops_len;
    s.zero = true;
    plan.sub_extent.push_back({s.off, n});
    s.merge = (int32_t)plan.merges.size();
    plan.merges.push_back({s.off, n, (int32_t)plan.merge_src.size(), (int32_t)plan.merge_src.size()});
    plan.ops_len += align4(n);
  }
}
// block_add_block_two (block.f90:1786-1822): the search restarts after the last match
static void add_two(const OBlk &b1, double coef, OBlk &nw, HpsiPlan &plan) {
  size_t x1 = 0;
  for (OSub &s : nw.sub) {
    for (size_t x = x1; x < b1.sub.size(); ++x) {
      const OSub &q = b1.sub[x];
      if (q.num_up == s.num_up && q.num_down == s.num_down && q.down_dif == s.down_dif) {
        x1 = x + 1;
        if ((int64_t)q.row_dim * q.sdim != (int64_t)s.row_dim * s.sdim)
          throw PlanError(TJ_ERR_ARG, "hmerge: operator sub-blocks of different size");
        // the merge record of s (one per merged sub-block, made by pass_info)
        if (s.merge < 0 || plan.merges[s.merge].dst != s.off)
          throw PlanError(TJ_ERR_ARG, "hmerge: merged sub-block without its merge record");
        HpsiPlan::Merge &mr = plan.merges[s.merge];
        // sources of one destination are contiguous: append by moving them last
        const int32_t b = mr.s_begin, e = mr.s_end;
        mr.s_begin = (int32_t)plan.merge_src.size();
        for (int32_t k = b; k < e; ++k) {
          const int64_t src = plan.merge_src[k];
          const double cf = plan.merge_coef[k];
          plan.merge_src.push_back(src);
          plan.merge_coef.push_back(cf);
        }
        plan.merge_src.push_back(q.off);
        plan.merge_coef.push_back(coef);
        mr.s_end = (int32_t)plan.merge_src.size();
        s.zero = false;
        break;
      }
    }
  }
}

struct Geo {
  const tj_lattice *L;
  int ns1;
  std::vector<int> inb;   // inb(-4:num_site) at [i+4]
  int coup_bs[2][2] = {{0, 0}, {0, 0}}, coup_bb[2] = {0, 0};
  int neib(int i, int k) const { return L->neib[(size_t)(k - 1) * ns1 + i]; }
  int neiba(int i, int j) const { return L->neiba[(size_t)j * ns1 + i]; }
  int inb1(int i, int j) const { return L->inb1[(size_t)j * ns1 + i]; }
  int nleg11(int i) const { return L->nleg11[i - 1]; }
  int nposi(int i) const { return L->nposi[i]; }
  int nposi_dm(int i) const { return L->nposi_dm[i]; }
  int nposi_lat(int i) const { return L->nposi_lat[i]; }
  double jt(int k, int i) const { return L->jt[(size_t)i * L->neibt + k - 1]; }
  double jd(int k, int i) const { return L->jd[(size_t)i * L->neibt + k - 1]; }
  double jn(int k) const { return L->jn[k - 1]; }
  double esite(int i) const { return L->esite[i]; }
  int &INB(int i) { return inb[i + 4]; }
  int npd(int j) const {   // nposi(nposi_dm(j)) with range checks
    if (j < 0 || j >= ns1) throw PlanError(TJ_ERR_ARG, "lattice index out of range");
    int p = nposi_dm(j);
    if (p < 0 || p >= ns1) throw PlanError(TJ_ERR_ARG, "lattice index out of range");
    return nposi(p);
  }
};

static int slot(const Model &m, int i1) {
  if (i1 < 1 || i1 > (int)m.sub.size()) {
    char b[96];
    std::snprintf(b, sizeof b, "operator slot %d outside 1..%d", i1, (int)m.sub.size());
    throw PlanError(TJ_ERR_ARG, b);
  }
  return i1 - 1;
}

// hmerge (get_sys.f90:4383-4593)
static void hmerge(Geo &g, Model &sys, Model &env, HpsiPlan &plan) {
  const int neibt = g.L->neibt;
  const int syssite = sys.len + 1, dmsite = sys.len + env.len + 2;
  for (int k = 1; k <= neibt; ++k) {
    int j = g.neib(syssite, k);
    if (g.npd(j) == 3) g.coup_bs[1][0] = 1;
    if (g.npd(j) == 1) g.coup_bs[0][0] = 1;
    j = g.neib(g.nposi_lat(dmsite), k);
    if (g.npd(j) == 3) g.coup_bs[1][1] = 1;
    if (g.npd(j) == 1) g.coup_bs[0][1] = 1;
  }
  for (int ia = 0; ia < 2; ++ia) {
    if (g.coup_bs[0][ia] == 1)
      for (int op : {EU, SD, SN}) pass_info(sys.sub[0][op], sys.snc[ia][op], plan);
    if (g.coup_bs[1][ia] == 1)
      for (int op : {EU, ED, SD, SN}) pass_info(env.sub[0][op], env.snc[ia][op], plan);
  }
  for (int ia = 1; ia <= 2; ++ia) {
    const int j = sys.len + 1 + (env.len + 1) * (ia - 1);
    const int lj = g.nposi_lat(j);
    for (int k1 = 1; k1 <= neibt; ++k1) {
      const int ib = g.neib(lj, k1);
      if (g.npd(ib) == 3 && g.coup_bs[1][ia - 1] != 0) {
        const int s = slot(env, g.inb1(g.nposi_dm(ib) - sys.len - 1, env.len));
        const double jd1 = g.jd(k1, lj), jt1 = g.jt(k1, lj), jn1 = g.jn(k1);
        if (jt1 != 0.0) {
          add_two(env.sub[s][EU], jt1, env.snc[ia - 1][EU], plan);
          add_two(env.sub[s][ED], jt1, env.snc[ia - 1][ED], plan);
        }
        if (jd1 != 0.0) add_two(env.sub[s][SD], jd1, env.snc[ia - 1][SD], plan);
        if (jn1 != 0.0) add_two(env.sub[s][SN], jn1, env.snc[ia - 1][SN], plan);
      }
      if (g.npd(ib) == 1 && g.coup_bs[0][ia - 1] == 1) {
        const int s = slot(sys, g.inb1(g.nposi_dm(ib), sys.len));
        const double jd1 = g.jd(k1, lj), jt1 = g.jt(k1, lj), jn1 = g.jn(k1);
        if (jt1 != 0.0) add_two(sys.sub[s][EU], jt1, sys.snc[ia - 1][EU], plan);
        if (jd1 != 0.0) add_two(sys.sub[s][SD], jd1, sys.snc[ia - 1][SD], plan);
        if (jn1 != 0.0) add_two(sys.sub[s][SN], jn1, sys.snc[ia - 1][SN], plan);
      }
    }
  }
  int k11 = 0;
  for (int I = 1; I <= sys.len; ++I) {
    int k1 = 0;
    for (int k = 1; k <= neibt; ++k)
      if (g.npd(g.neib(I, k)) == 3) ++k1;
    g.INB(I) = k1;
    if (g.nleg11(env.len) < g.nleg11(sys.len)) g.INB(I) = 0;
    if (g.INB(I) != 0) ++k11;
  }
  g.coup_bb[0] = k11;
  g.INB(sys.len + 1) = 0;
  g.INB(sys.len + 1 + env.len + 1) = 0;
  for (int I = 1; I <= env.len; ++I) {
    int k1 = 0;
    g.INB(I + sys.len + 1) = 0;
    for (int k = 1; k <= neibt; ++k) {
      const int J = g.neib(g.nposi_lat(I + sys.len + 1), k);
      if (g.npd(J) == 1 && g.INB(J) == 0) ++k1;
    }
    g.INB(I + sys.len + 1) = k1;
    if (k1 != 0) ++k11;
  }
  g.coup_bb[1] = k11 - g.coup_bb[0];
  env.sub_s.assign(g.coup_bb[0], {});
  sys.sub_s.assign(g.coup_bb[1], {});
  for (int i = 0; i < g.coup_bb[0]; ++i)
    for (int op : {EU, ED, SD, SN}) pass_info(env.sub[0][op], env.sub_s[i][op], plan);
  for (int i = 0; i < g.coup_bb[1]; ++i)
    for (int op : {EU, SD, SN}) pass_info(sys.sub[0][op], sys.sub_s[i][op], plan);
  int jc = 0;
  for (int I = 1; I <= sys.len + env.len + 1; ++I) {
    if (g.INB(I) == 0) continue;
    const int Ia = g.nposi_lat(I);
    ++jc;
    for (int k1 = 1; k1 <= neibt; ++k1) {
      const int ib = g.neib(Ia, k1);
      if (g.npd(ib) == 3 && I <= sys.len) {
        const int s = slot(env, g.inb1(g.nposi_dm(ib) - sys.len - 1, env.len));
        const double jt1 = g.jt(k1, Ia), jd1 = g.jd(k1, Ia), jn1 = g.jn(k1);
        if (jt1 != 0.0) {
          add_two(env.sub[s][EU], jt1, env.sub_s[jc - 1][EU], plan);
          add_two(env.sub[s][ED], jt1, env.sub_s[jc - 1][ED], plan);
        }
        if (jd1 != 0.0) add_two(env.sub[s][SD], jd1, env.sub_s[jc - 1][SD], plan);
        if (jn1 != 0.0) add_two(env.sub[s][SN], jn1, env.sub_s[jc - 1][SN], plan);
      }
      if (g.npd(ib) == 1 && I > sys.len + 1 && g.INB(g.nposi_dm(ib)) == 0) {
        const int s = slot(sys, g.inb1(ib, sys.len));
        const int jc1 = jc - g.coup_bb[0];
        const double jt1 = g.jt(k1, Ia), jd1 = g.jd(k1, Ia), jn1 = g.jn(k1);
        if (jc1 < 1 || jc1 > (int)sys.sub_s.size()) throw PlanError(TJ_ERR_ARG, "hmerge: leg index out of range");
        if (jt1 != 0.0) add_two(sys.sub[s][EU], jt1, sys.sub_s[jc1 - 1][EU], plan);
        if (jd1 != 0.0) add_two(sys.sub[s][SD], jd1, sys.sub_s[jc1 - 1][SD], plan);
        if (jn1 != 0.0) add_two(sys.sub[s][SN], jn1, sys.sub_s[jc1 - 1][SN], plan);
      }
    }
  }
}

static void check_lattice(const tj_lattice *L) {
  if (!L || !L->neib || !L->neiba || !L->inb1 || !L->nleg11 || !L->nposi || !L->nposi_dm || !L->nposi_lat ||
      !L->jt || !L->jz || !L->jd || !L->jn || !L->esite)
    throw PlanError(TJ_ERR_ARG, "lattice tables missing");
  if (L->num_site < 2 || L->neibt < 1) throw PlanError(TJ_ERR_ARG, "bad lattice sizes");
}

}  // namespace

int build_hpsi_plan(const tj_lattice *lat, const tj_model *sysm, const tj_model *envm, const tj_basis *sys_bs,
                    const tj_basis *env_bs, const tj_wave *wave, HpsiPlan &plan, std::string &msg, bool tiles) {
  try {
    check_lattice(lat);
    if (!sys_bs || !env_bs || !wave || !sys_bs->sub || !env_bs->sub || (wave->num > 0 && !wave->sub))
      throw PlanError(TJ_ERR_ARG, "null basis or wave");
    plan = HpsiPlan();
    Model sys, env;
    load_model(sysm, sys, plan);
    load_model(envm, env, plan);
    if (sys.len + env.len + 2 > lat->num_site) throw PlanError(TJ_ERR_ARG, "sys_len + env_len + 2 exceeds num_site");
    Geo g;
    g.L = lat;
    g.ns1 = lat->num_site + 1;
    g.inb.assign(lat->num_site + 8, 0);
    hmerge(g, sys, env, plan);
    const SiteOps so = make_site_ops(lat->up_bias);
    Builder B(sys_bs, env_bs, wave, plan);
    B.want_tiles = tiles;
    B.init_cells();
    plan.psi_len = wave->dim;
    // model_wave, add_op = 1 (get_sys.f90:4157-4239)
    B.block_vec_dia(OView{&sys.ham, false}, 1.0);
    B.vec_block_dia(OView{&env.ham, false}, 1.0);
    const int is = g.nposi_lat(sys.len + 1), js = g.nposi_lat(sys.len + env.len + 2);
    if (g.esite(is) != 0.0) B.site_vec_site_dia(so.ne, so.si, g.esite(is));
    if (g.esite(js) != 0.0) B.site_vec_site_dia(so.si, so.ne, g.esite(js));
    const int ii = g.neiba(is, js);
    if (ii != 0) {
      const double jd1 = g.jd(ii, is), coefx = g.jt(ii, is), jn1 = g.jn(ii);
      if (coefx != 0.0) B.site_vec_site_ndia(so.eu, 'F', so.eu, 'F', coefx);
      if (jd1 != 0.0) B.site_vec_site_ndia(so.sd, 'B', so.sd, 'B', jd1);
      B.site_vec_site_dia(so.ne, so.ne, jn1);
    }
    if (g.coup_bs[0][0] == 1) {
      B.block_site_vec_ndia(OView{&sys.snc[0][EU], false}, so.eu, 'F', 1.0);
      B.block_site_vec_ndia(OView{&sys.snc[0][SD], false}, so.sd, 'B', 1.0);
      B.block_site_vec_dia(OView{&sys.snc[0][SN], false}, so.ne, 1.0);
    }
    if (g.coup_bs[0][1] == 1) {
      B.block_vec_site_ndia(OView{&sys.snc[1][EU], false}, so.eu, 'F', 1.0);
      B.block_vec_site_ndia(OView{&sys.snc[1][SD], false}, so.sd, 'B', 1.0);
      B.block_vec_site_dia(OView{&sys.snc[1][SN], false}, so.ne, 1.0);
    }
    if (g.coup_bs[1][0] == 1) {
      B.site_vec_block_ndia(so.eu, 'F', OView{&env.snc[0][ED], true}, 'F', 1.0);
      B.site_vec_block_ndia(so.sd, 'B', OView{&env.snc[0][SD], true}, 'B', 1.0);
      B.site_vec_block_dia(so.ne, OView{&env.snc[0][SN], false}, 1.0);
    }
    if (g.coup_bs[1][1] == 1) {
      B.vec_block_site_ndia(OView{&env.snc[1][EU], false}, 'F', so.eu, 'F', 1.0);
      B.vec_block_site_ndia(OView{&env.snc[1][SD], false}, 'B', so.sd, 'B', 1.0);
      B.vec_block_site_dia(OView{&env.snc[1][SN], false}, so.ne, 1.0);
    }
    int jc = 0;
    for (int i = 1; i <= sys.len + 1 + env.len; ++i) {
      if (g.INB(i) == 0) continue;
      ++jc;
      const std::array<OBlk, 5> *sa, *eb;
      if (i <= sys.len) {
        sa = &sys.sub[slot(sys, g.inb1(i, sys.len))];
        if (jc > (int)env.sub_s.size()) throw PlanError(TJ_ERR_ARG, "leg index out of range");
        eb = &env.sub_s[jc - 1];
      } else {
        eb = &env.sub[slot(env, g.inb1(i - sys.len - 1, env.len))];
        const int jc1 = jc - g.coup_bb[0];
        if (jc1 < 1 || jc1 > (int)sys.sub_s.size()) throw PlanError(TJ_ERR_ARG, "leg index out of range");
        sa = &sys.sub_s[jc1 - 1];
      }
      B.block_vec_block_ndia(OView{&(*sa)[EU], false}, OView{&(*eb)[ED], true}, 'F', 1.0);
      B.block_vec_block_ndia(OView{&(*sa)[SD], false}, OView{&(*eb)[SD], true}, 'B', 1.0);
      B.block_vec_block_dia(OView{&(*sa)[SN], false}, OView{&(*eb)[SN], false}, 1.0);
    }
    B.finalize();
    // algorithmic bytes: every operator sub-block touched once, psi read, output read-modify-write
    double opb = 0;
    auto add_touched = [&](const OBlk &b) {
      for (const OSub &s : b.sub)
        if (s.touched) opb += (double)s.row_dim * s.sdim;
    };
    for (const Model *m : {&sys, &env}) {
      add_touched(m->ham);
      for (const auto &a : m->sub) for (const OBlk &b : a) add_touched(b);
      for (const auto &a : m->snc) for (const OBlk &b : a) add_touched(b);
      for (const auto &a : m->sub_s) for (const OBlk &b : a) add_touched(b);
    }
    plan.bytes = 8.0 * (opb + 3.0 * (double)wave->dim);
    return TJ_OK;
  } catch (const PlanError &e) {
    msg = e.what();
    return e.code;
  } catch (const std::exception &e) {
    msg = e.what();
    return TJ_ERR_ARG;
  }
}


// ------------------------------------------------------------ correlators
namespace {
// A basis whose sectors are the wave's system (side 0) or environment labels,
// each one sub-block spanning the whole sector: used when a contraction has
// no operator on that side and the reference takes whole sector rows/columns.
struct TrivialBasis {
  std::vector<tj_basis_map> maps;
  std::vector<tj_basis_sub> subs;
  tj_basis b;
  TrivialBasis(const tj_wave *w, int side) {
    for (int i = 0; i < w->num; ++i) {
      const int nu = side == 0 ? w->sub[i].sys_num_up : w->sub[i].env_num_up;
      const int nd = side == 0 ? w->sub[i].sys_num_down : w->sub[i].env_num_down;
      const int dim = side == 0 ? w->sub[i].sys_dim : w->sub[i].env_dim;
      bool seen = false;
      for (auto &m : maps)
        if (m.new_num_up == nu && m.new_num_down == nd) seen = true;
      if (seen) continue;
      tj_basis_map m{0, 1, dim, nu, nd, (int32_t)subs.size()};
      maps.push_back(m);
      subs.push_back(tj_basis_sub{0, dim, -1000, -1000, -1000, -1000});
    }
    b.len = 0;
    b.num = (int32_t)maps.size();
    b.dim = 0;
    b.pad_ = 0;
    b.sub = maps.data();
    b.maps = subs.data();
  }
};

struct CorBuilder : Builder {
  using Builder::Builder;
  // measure_sys_block (measure.f90:1241-1295)
  void measure_sys_block(const OView &A) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &q = SM(x, m);
        const double c1 = 1.0 / std::sqrt(1.0 + q.bl_num_down);
        const int k = A.find(q.bl_num_up, q.bl_num_down, 0, false);
        if (k < 0) continue;
        for (int n = 0; n < ebs->sub[y].num; ++n) emitL(cell(i, m, n), A, k, false, cell(i, m, n), c1);
      }
    }
  }
  // measure_env_block (measure.f90:1359-1414)
  void measure_env_block(const OView &A) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int n = 0; n < ebs->sub[y].num; ++n) {
        const tj_basis_sub &q = EM(y, n);
        const int k = A.find(q.bl_num_up, q.bl_num_down, 0, false);
        if (k < 0) continue;
        const double c1 = 1.0 / std::sqrt(1.0 + q.bl_num_down);
        for (int m = 0; m < sbs->sub[x].num; ++m) emitR(cell(i, m, n), cell(i, m, n), A, k, false, c1);
      }
    }
  }
  // sys_block_env_block_cor_dia (measure.f90:1638-1732): <psi B, A psi> = <psi, A psi B^T>
  void sbeb_dia(const OView &A, const OView &B) {
    for (int i = 0; i < wave->num; ++i) {
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m) {
        const tj_basis_sub &ms = SM(x, m);
        const int ks = A.find(ms.bl_num_up, ms.bl_num_down, 0, false);
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &me = EM(y, n);
          const int ke = B.find(me.bl_num_up, me.bl_num_down, 0, false);
          if (ks < 0 || ke < 0) continue;
          const double c1 = 1.0 / std::sqrt((1.0 + me.bl_num_down) * (1.0 + ms.bl_num_down));
          emit2(cell(i, m, n), A, ks, false, cell(i, m, n), B, ke, true, c1);
        }
      }
    }
  }
  // sys_block_env_block_cor_ndia (measure.f90:5241-5480): <psi_k, c A psi_i B>
  void sbeb_ndia(const OView &A, const OView &B, char flag) {
    const int up = A.up_dif(), d1 = A.down_dif();
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m)
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &ms = SM(x, m), &me = EM(y, n);
          for (int dd = -d1; dd <= d1; dd += 2) {
            const int nsb_up = ms.bl_num_up + up, nsb_dn = ms.bl_num_down + dd;
            const int ks = A.find(ms.bl_num_up, ms.bl_num_down, dd, true);
            for (int edd = -d1; edd <= d1; edd += 2) {
              const int neb_up = me.bl_num_up - up, neb_dn = me.bl_num_down - edd;
              const int ke = B.find(neb_up, neb_dn, edd, true);
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int nsu = su + up, neu = eu - up, ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == nsb_up && q.bl_num_down == nsb_dn && q.st_num_up == ms.st_num_up &&
                             q.st_num_down == ms.st_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == neb_up && q.bl_num_down == neb_dn && q.st_num_up == me.st_num_up &&
                             q.st_num_down == me.st_num_down; }, yk, le))
                  continue;
                const int wid = find_sec(nsu, nsd, neu, ned);
                if (ks < 0 || ke < 0 || wid < 0) continue;
                const double signs = sgn(flag, sd + me.st_num_down);
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.bl_num_down, j5 = ms.st_num_down, j6 = nsb_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.bl_num_down, j55 = me.st_num_down, j66 = neb_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                c1 = c1 * w6j(j11, j22, j33, j44, j55, j66);
                if (c1 == 0.0) continue;
                c1 = c1 * std::sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                if (((j6 + j5 + j3 + j2) / 2 + (j66 + j55 + j33 + j22) / 2) % 2 == 1) c1 = -c1;
                emit2(cell(wid, sys_index_in(wid, xk, ls), env_index_in(wid, yk, le)), A, ks, false, cell(i, m, n), B,
                      ke, false, signs * c1);
              }
            }
          }
        }
    }
  }
  // sys_block_site_cor_ndia (measure.f90:4939-5083)
  void sb_site_ndia(const OView &A, const SiteOp &st, char flag) {
    const int up = A.up_dif(), d1 = A.down_dif();
    for (int i = 0; i < wave->num; ++i) {
      const int sd = wave->sub[i].sys_num_down;
      const int j = sec_x[i], y = sec_y[i];
      for (int k = 0; k < sbs->sub[j].num; ++k) {
        const tj_basis_sub &q = SM(j, k);
        for (int dd = -d1; dd <= d1; dd += 2)
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int nbl_up = q.bl_num_up + up, nbl_dn = q.bl_num_down + dd;
            const int nst_up = q.st_num_up - up, nst_dn = q.st_num_down - sdd;
            const int kb = A.find(q.bl_num_up, q.bl_num_down, dd, true);
            const int ks = site_find(st, nst_up, nst_dn, sdd, true);
            int np = -1;
            for (int x = 0; x < sbs->sub[j].num; ++x) {
              const tj_basis_sub &r = SM(j, x);
              if (r.bl_num_up == nbl_up && r.bl_num_down == nbl_dn && r.st_num_up == nst_up && r.st_num_down == nst_dn) {
                np = x;
                break;
              }
            }
            if (kb < 0 || ks < 0 || np < 0) continue;
            const double signs = sgn(flag, q.bl_num_down);
            const int j1 = nbl_dn, j2 = q.bl_num_down, j3 = d1, j4 = q.st_num_down, j5 = nst_dn, j6 = sd;
            double c1 = 1.0 / std::sqrt(1.0 + d1) * w6j(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * m1pow((j2 + j5 + j3 + j6) / 2);
            const double coef = signs * st.val[ks] * c1;
            for (int n = 0; n < ebs->sub[y].num; ++n) emitL(cell(i, np, n), A, kb, false, cell(i, k, n), coef);
          }
      }
    }
  }
  // env_block_site_cor_ndia (measure.f90:5085-5238)
  void eb_site_ndia(const OView &A, const SiteOp &st, char flag) {
    const int up = A.up_dif(), d1 = A.down_dif();
    for (int i = 0; i < wave->num; ++i) {
      const int sd = wave->sub[i].sys_num_down, ed = wave->sub[i].env_num_down;
      const int x0 = sec_x[i], j = sec_y[i];
      for (int k = 0; k < ebs->sub[j].num; ++k) {
        const tj_basis_sub &q = EM(j, k);
        for (int bdd = -d1; bdd <= d1; bdd += 2) {
          const int nbl_up = q.bl_num_up - up, nbl_dn = q.bl_num_down - bdd;
          const int kb = A.find(nbl_up, nbl_dn, bdd, true);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int nst_up = q.st_num_up + up, nst_dn = q.st_num_down + sdd;
            const int ks = site_find(st, q.st_num_up, q.st_num_down, sdd, true);
            int np = -1;
            for (int x = 0; x < ebs->sub[j].num; ++x) {
              const tj_basis_sub &r = EM(j, x);
              if (r.bl_num_up == nbl_up && r.bl_num_down == nbl_dn && r.st_num_up == nst_up && r.st_num_down == nst_dn) {
                np = x;
                break;
              }
            }
            if (kb < 0 || ks < 0 || np < 0) continue;
            const double signs = sgn(flag, sd + q.st_num_down + sd);
            const int j1 = nbl_dn, j2 = q.bl_num_down, j3 = d1, j4 = q.st_num_down, j5 = nst_dn, j6 = ed;
            double c1 = 1.0 / std::sqrt(1.0 + d1) * w6j(j1, j2, j3, j4, j5, j6);
            c1 = c1 * m1pow((j2 + j5 + j3 + j6) / 2);
            if (c1 == 0.0) continue;
            const double coef = signs * st.val[ks] * c1;
            for (int m = 0; m < sbs->sub[x0].num; ++m) emitR(cell(i, m, np), cell(i, m, k), A, kb, false, coef);
          }
        }
      }
    }
  }
  // sys_block_env_site_cor_ndia (measure.f90:5482-5706)
  void sb_esite_ndia(const OView &A, const SiteOp &st, char flag) {
    const int up = A.up_dif(), d1 = A.down_dif();
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m)
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &ms = SM(x, m), &me = EM(y, n);
          for (int bdd = -d1; bdd <= d1; bdd += 2) {
            const int nsb_up = ms.bl_num_up + up, nsb_dn = ms.bl_num_down + bdd;
            const int kb = A.find(ms.bl_num_up, ms.bl_num_down, bdd, true);
            for (int sdd = -st.b.down_dif; sdd <= st.b.down_dif; sdd += 2) {
              const int nes_up = me.st_num_up - up, nes_dn = me.st_num_down - sdd;
              const int ks = site_find(st, nes_up, nes_dn, sdd, true);
              if (kb < 0 || ks < 0) continue;
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int nsu = su + up, neu = eu - up, ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == nsb_up && q.bl_num_down == nsb_dn && q.st_num_up == ms.st_num_up &&
                             q.st_num_down == ms.st_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nes_up && q.st_num_down == nes_dn && q.bl_num_down == me.bl_num_down; }, yk, le))
                  continue;
                const int wid = find_sec(nsu, nsd, neu, ned);
                if (wid < 0) continue;
                const double signs = sgn(flag, sd);
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.bl_num_down, j5 = ms.st_num_down, j6 = nsb_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.st_num_down, j55 = me.bl_num_down, j66 = nes_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                c1 = c1 * w6j(j11, j22, j33, j44, j55, j66);
                if (c1 == 0.0) continue;
                c1 = c1 * std::sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                if (((j6 + j5 + j3 + j2) / 2 + (j55 + j44 + j11 + j22) / 2) % 2 != 0) c1 = -c1;
                const double coef = signs * st.val[ks] * c1;
                emitL(cell(wid, sys_index_in(wid, xk, ls), env_index_in(wid, yk, le)), A, kb, false, cell(i, m, n), coef);
              }
            }
          }
        }
    }
  }
  // sys_site_env_block_cor_ndia (measure.f90:5926-6154): <c psi_k B^T, psi_i>
  void ssite_eb_ndia(const SiteOp &st, const OView &B, char flag) {
    const int up = st.b.up_dif, d1 = st.b.down_dif;
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m)
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &ms = SM(x, m), &me = EM(y, n);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            const int nss_up = ms.st_num_up + up, nss_dn = ms.st_num_down + sdd;
            const int ks = site_find(st, ms.st_num_up, ms.st_num_down, sdd, true);
            for (int bdd = -B.down_dif(); bdd <= B.down_dif(); bdd += 2) {
              const int neb_up = me.bl_num_up - up, neb_dn = me.bl_num_down - bdd;
              const int kb = B.find(neb_up, neb_dn, bdd, true);
              if (ks < 0 || kb < 0) continue;
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int nsu = su + up, neu = eu - up, ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nss_up && q.st_num_down == nss_dn && q.bl_num_down == ms.bl_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.bl_num_up == neb_up && q.bl_num_down == neb_dn && q.st_num_down == me.st_num_down; }, yk, le))
                  continue;
                const int wid = find_sec(nsu, nsd, neu, ned);
                if (wid < 0) continue;
                const double signs = sgn(flag, sd + me.st_num_down + ms.bl_num_down);
                double coef = signs * st.val[ks];
                if (coef == 0.0) continue;
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.st_num_down, j5 = ms.bl_num_down, j6 = nss_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.bl_num_down, j55 = me.st_num_down, j66 = neb_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                c1 = c1 * w6j(j11, j22, j33, j44, j55, j66);
                if (c1 == 0.0) continue;
                c1 = c1 * std::sqrt((1.0 + j11) * (j33 + 1.0) / (1.0 + d1));
                if (((j66 + j55 + j33 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                coef = coef * c1;
                emitR(cell(i, m, n), cell(wid, sys_index_in(wid, xk, ls), env_index_in(wid, yk, le)), B, kb, true, coef);
              }
            }
          }
        }
    }
  }
  // sys_site_env_site_cor_ndia (measure.f90:5709-5924)
  void ssite_esite_ndia(const SiteOp &st, const SiteOp &et, char flag) {
    const int up = st.b.up_dif, d1 = st.b.down_dif;
    for (int i = 0; i < wave->num; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int su = w.sys_num_up, sd = w.sys_num_down, eu = w.env_num_up, ed = w.env_num_down;
      const int x = sec_x[i], y = sec_y[i];
      for (int m = 0; m < sbs->sub[x].num; ++m)
        for (int n = 0; n < ebs->sub[y].num; ++n) {
          const tj_basis_sub &ms = SM(x, m), &me = EM(y, n);
          for (int sdd1 = -d1; sdd1 <= d1; sdd1 += 2) {
            const int nss_up = ms.st_num_up + up, nss_dn = ms.st_num_down + sdd1;
            const int ks = site_find(st, ms.st_num_up, ms.st_num_down, sdd1, true);
            for (int sdd2 = -d1; sdd2 <= d1; sdd2 += 2) {
              const int nes_up = me.st_num_up - up, nes_dn = me.st_num_down - sdd2;
              const int ke = site_find(et, nes_up, nes_dn, sdd2, true);
              if (ks < 0 || ke < 0) continue;
              for (int nsd = std::abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                const int nsu = su + up, neu = eu - up, ned = nsd;
                int xk, ls, yk, le;
                if (!find_sys(nsu, nsd, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nss_up && q.st_num_down == nss_dn && q.bl_num_down == ms.bl_num_down; }, xk, ls))
                  continue;
                if (!find_env(neu, ned, [&](const tj_basis_sub &q) {
                      return q.st_num_up == nes_up && q.st_num_down == nes_dn && q.bl_num_down == me.bl_num_down; }, yk, le))
                  continue;
                const int wid = find_sec(nsu, nsd, neu, ned);
                if (wid < 0) continue;
                const double signs = sgn(flag, sd + ms.bl_num_down);
                double coef = signs * st.val[ks] * et.val[ke];
                if (coef == 0.0) continue;
                const int j1 = nsd, j2 = d1, j3 = sd, j4 = ms.st_num_down, j5 = ms.bl_num_down, j6 = nss_dn;
                const int j11 = ned, j22 = d1, j33 = ed, j44 = me.st_num_down, j55 = me.bl_num_down, j66 = nes_dn;
                double c1 = w6j(j1, j2, j3, j4, j5, j6);
                if (c1 == 0.0) continue;
                c1 = c1 * w6j(j11, j22, j33, j44, j55, j66);
                if (c1 == 0.0) continue;
                c1 = c1 * std::sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                if (((j55 + j44 + j11 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                coef = coef * c1;
                emitAxpy(cell(i, m, n), cell(wid, sys_index_in(wid, xk, ls), env_index_in(wid, yk, le)), coef);
              }
            }
          }
        }
    }
  }
};
}  // namespace

int build_cor_plan(CorKind kind, const tj_block *a, const tj_block *b, const tj_basis *sys_bs,
                   const tj_basis *env_bs, const tj_wave *wave, char flag, HpsiPlan &plan, std::string &msg) {
  try {
    if (!a || !wave || wave->num < 0 || (wave->num > 0 && !wave->sub)) throw PlanError(TJ_ERR_ARG, "null argument");
    if (flag != 'B' && flag != 'F') throw PlanError(TJ_ERR_ARG, "flag must be 'B' or 'F'");
    plan = HpsiPlan();
    TrivialBasis ts(wave, 0), te(wave, 1);
    const tj_basis *sb = sys_bs ? sys_bs : &ts.b, *eb = env_bs ? env_bs : &te.b;
    CorBuilder B(sb, eb, wave, plan);
    B.cor_mode = true;
    B.init_cells();
    plan.psi_len = wave->dim;
    OBlk ba, bb;
    switch (kind) {
      case COR_MEASURE_SYS_BLOCK:
        load_block(*a, ba, plan);
        B.measure_sys_block(OView{&ba, false});
        break;
      case COR_MEASURE_ENV_BLOCK:
        load_block(*a, ba, plan);
        B.measure_env_block(OView{&ba, false});
        break;
      case COR_SBEB_DIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*a, ba, plan);
        load_block(*b, bb, plan);
        B.sbeb_dia(OView{&ba, false}, OView{&bb, false});
        break;
      case COR_SBEB_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*a, ba, plan);
        load_block(*b, bb, plan);
        B.sbeb_ndia(OView{&ba, false}, OView{&bb, false}, flag);
        break;
      case COR_SB_SITE_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*a, ba, plan);
        B.sb_site_ndia(OView{&ba, false}, site_from_block(*b), flag);
        break;
      case COR_EB_SITE_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*a, ba, plan);
        B.eb_site_ndia(OView{&ba, false}, site_from_block(*b), flag);
        break;
      case COR_SB_ESITE_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*a, ba, plan);
        B.sb_esite_ndia(OView{&ba, false}, site_from_block(*b), flag);
        break;
      case COR_SSITE_EB_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        load_block(*b, bb, plan);
        B.ssite_eb_ndia(site_from_block(*a), OView{&bb, false}, flag);
        break;
      case COR_SSITE_ESITE_NDIA:
        if (!b) throw PlanError(TJ_ERR_ARG, "null operator");
        B.ssite_esite_ndia(site_from_block(*a), site_from_block(*b), flag);
        break;
    }
    B.finalize();
    return TJ_OK;
  } catch (const PlanError &e) {
    msg = e.what();
    return e.code;
  } catch (const std::exception &e) {
    msg = e.what();
    return TJ_ERR_ARG;
  }
}

static_assert(sizeof(Task) == sizeof(tj_plan_task), "task layout");
static_assert(sizeof(Cell) == sizeof(tj_plan_cell), "cell layout");
static_assert(sizeof(HpsiPlan::Upload) == sizeof(tj_plan_upload), "upload layout");
static_assert(sizeof(HpsiPlan::Merge) == sizeof(tj_plan_merge), "merge layout");
static_assert(sizeof(Tile) == sizeof(tj_plan_item), "item layout");
static_assert(sizeof(Reduce) == sizeof(tj_plan_reduce), "reduce layout");

}  // namespace tjb

int tjb::export_hpsi_plan(const tjb::HpsiPlan &P, tj_plan_export *out) {
  out->ops_len = P.ops_len;
  out->scratch_len = P.scratch_len;
  out->psi_len = P.psi_len;
  out->n_tasks1 = (int64_t)P.tasks1.size();
  out->n_tasks2 = (int64_t)P.tasks2.size();
  out->n_cells1 = (int64_t)P.cells1.size();
  out->n_cells2 = (int64_t)P.cells2.size();
  out->n_uploads = (int64_t)P.uploads.size();
  out->n_merges = (int64_t)P.merges.size();
  out->n_merge_src = (int64_t)P.merge_src.size();
  out->flops = P.flops;
  out->flops_ref = P.flops_ref;
  out->bytes = P.bytes;
  auto cp = [](void *dst, const void *src, size_t n) { if (dst && src && n) std::memcpy(dst, src, n); };
  cp(out->tasks1, P.tasks1.data(), P.tasks1.size() * sizeof(tjb::Task));
  cp(out->tasks2, P.tasks2.data(), P.tasks2.size() * sizeof(tjb::Task));
  cp(out->cells1, P.cells1.data(), P.cells1.size() * sizeof(tjb::Cell));
  cp(out->cells2, P.cells2.data(), P.cells2.size() * sizeof(tjb::Cell));
  cp(out->uploads, P.uploads.data(), P.uploads.size() * sizeof(tjb::HpsiPlan::Upload));
  cp(out->merges, P.merges.data(), P.merges.size() * sizeof(tjb::HpsiPlan::Merge));
  cp(out->merge_src, P.merge_src.data(), P.merge_src.size() * sizeof(int64_t));
  cp(out->merge_coef, P.merge_coef.data(), P.merge_coef.size() * sizeof(double));
  out->n_items1 = (int64_t)P.tiles1.size();
  out->n_items2 = (int64_t)P.tiles2.size();
  out->n_red1 = (int64_t)P.red1.size();
  out->n_red2 = (int64_t)P.red2.size();
  cp(out->items1, P.tiles1.data(), P.tiles1.size() * sizeof(tjb::Tile));
  cp(out->items2, P.tiles2.data(), P.tiles2.size() * sizeof(tjb::Tile));
  cp(out->red1, P.red1.data(), P.red1.size() * sizeof(tjb::Reduce));
  cp(out->red2, P.red2.data(), P.red2.size() * sizeof(tjb::Reduce));
  return TJ_OK;
}

extern "C" int tj_hpsi_plan_export(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                                   const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave,
                                   tj_plan_export *out) {
  if (!out) return tjb_set_err(TJ_ERR_ARG, "null output");
  tjb::HpsiPlan P;
  std::string msg;
  int rc = tjb::build_hpsi_plan(lat, sys, env, sys_bs, env_bs, wave, P, msg);
  if (rc) return tjb_set_err(rc, "H*psi plan: " + msg);
  return tjb::export_hpsi_plan(P, out);
}

extern "C" int tj_cor_plan_export(int kind, const tj_block *a, const tj_block *b, const tj_basis *sys_bs,
                                  const tj_basis *env_bs, const tj_wave *wave, char flag, tj_plan_export *out) {
  if (!out) return tjb_set_err(TJ_ERR_ARG, "null output");
  if (kind < 0 || kind > (int)tjb::COR_SSITE_ESITE_NDIA) return tjb_set_err(TJ_ERR_ARG, "unknown correlator kind");
  tjb::HpsiPlan P;
  std::string msg;
  int rc = tjb::build_cor_plan((tjb::CorKind)kind, a, b, sys_bs, env_bs, wave, flag, P, msg);
  if (rc) return tjb_set_err(rc, "correlator plan: " + msg);
  return tjb::export_hpsi_plan(P, out);
}

namespace tjb {

// Independent superblocks in one plan: instance i's operators, input and
// output vector, phase-1 products and basis-state indices are placed after
// those of the instances before it, and the work items are cut again over
// the union, so that one set of launches computes every instance's H*psi.
void merge_plans(const std::vector<const HpsiPlan *> &parts, HpsiPlan &out, std::vector<int64_t> &psi_off,
                 const TuneParams &tp) {
  out = HpsiPlan();
  psi_off.clear();
  for (const HpsiPlan *p : parts) {
    const int64_t ob = out.ops_len, pb = out.psi_len, sb = out.scratch_len;
    const int t1 = (int)out.tasks1.size(), t2 = (int)out.tasks2.size();
    const int mb = (int)out.merge_src.size();
    const int32_t ss = out.n_sys_states, es = out.n_env_states;
    psi_off.push_back(pb);
    auto shift = [&](Operand &o) {
      if (o.space == SP_OPS) o.off += ob;
      else if (o.space == SP_PSI) o.off += pb;
      else if (o.space == SP_SCR) o.off += sb;
    };
    for (HpsiPlan::Upload u : p->uploads) {
      u.dst += ob;
      out.uploads.push_back(u);
    }
    for (HpsiPlan::Merge m : p->merges) {
      m.dst += ob;
      m.s_begin += mb;
      m.s_end += mb;
      out.merges.push_back(m);
    }
    for (int64_t s : p->merge_src) out.merge_src.push_back(s + ob);
    out.merge_coef.insert(out.merge_coef.end(), p->merge_coef.begin(), p->merge_coef.end());
    for (auto e : p->sub_extent) out.sub_extent.push_back({e.first + ob, e.second});
    for (Task t : p->tasks1) {
      shift(t.L);
      shift(t.R);
      out.tasks1.push_back(t);
    }
    for (Task t : p->tasks2) {
      shift(t.L);
      shift(t.R);
      out.tasks2.push_back(t);
    }
    for (Cell c : p->cells1) {
      c.off += sb;
      c.t_begin += t1;
      c.t_end += t1;
      out.cells1.push_back(c);
    }
    for (Cell c : p->cells2) {
      c.off += pb;
      c.t_begin += t2;
      c.t_end += t2;
      out.cells2.push_back(c);
    }
    for (int32_t s : p->cell2_row_state) out.cell2_row_state.push_back(s + ss);
    for (int32_t s : p->cell2_col_state) out.cell2_col_state.push_back(s + es);
    for (int32_t s : p->cell1_row_state) out.cell1_row_state.push_back(s + ss);
    out.n_sys_states += p->n_sys_states;
    out.n_env_states += p->n_env_states;
    out.ops_len += p->ops_len;
    out.psi_len += p->psi_len;
    out.scratch_len += p->scratch_len;
    out.flops += p->flops;
    out.flops_ref += p->flops_ref;
    out.bytes += p->bytes;
    out.key += p->key;
  }
  split_tiles(out.cells1, out.tasks1, out.tiles1, out.red1, out.nslots1, false, tp);
  split_tiles(out.cells2, out.tasks2, out.tiles2, out.red2, out.nslots2, false, tp);
}

}  // namespace tjb

extern "C" double tj_w6js(int j1, int j2, int j3, int l1, int l2, int l3) { return tjb::w6j(j1, j2, j3, l1, l2, l3); }
extern "C" double tj_w3js(int j1, int j2, int j3, int m1, int m2, int m3) { return tjb::w3j(j1, j2, j3, m1, m2, m3); }
