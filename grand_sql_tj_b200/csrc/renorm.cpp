// Operator renormalisation on the device: Get_Hamiltonian_Sys / _Env
// (code/tjsq/get_sys.f90:4-480) with the block updates they call
// (code/tjsq/block.f90:382-1503).
//
// The reference enlarges every operator of a block by one site into dense
// sector matrices (update_block_*, update_site_*, Get_hamiltonian_*), then
// truncates each with two DGEMMs over the whole enlarged sector pair
// (update_trun_*).  Here no enlarged operator is ever formed.  An enlarged
// operator is a list of pieces -- coef * op(O) or coef * I placed at a (row
// window, column window) of a sector pair, O a sub-block of the old block's
// operator -- and its truncation U_l^T E U_r is the sum over its pieces of
// coef * U_l[rows]^T op(O) U_r[cols].  Each piece is a two-GEMM chain on the
// grouped FP64 GEMM of H*psi: phase 1 forms op(O) U_r[cols] or
// U_l[rows]^T op(O), whichever costs fewer flops (identical products are
// formed once), phase 2 accumulates all pieces of one output sub-block into
// it, which its CTAs own.  Structural zeros of the enlarged operators, which
// the reference multiplies through, cost nothing; every new operator of the
// step (Hamiltonian and all operator sets) is produced by the same two
// launches.
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "ctx.h"

using namespace tjb;

#define CKR(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace tjb {

namespace {

struct RenormError : std::runtime_error {
  int code;
  RenormError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// an operator sub-block of the old block, resident in the operator space
struct RSub {
  int num_up, num_down, down_dif, row_dim, sdim;
  int64_t off;
};
struct RBlk {
  int len = 0, up_dif = 0, down_dif = 0;
  std::vector<RSub> sub;
  int find(int nu, int nd, int dd, bool use_dd) const {
    for (size_t k = 0; k < sub.size(); ++k)
      if (sub[k].num_up == nu && sub[k].num_down == nd && (!use_dd || sub[k].down_dif == dd)) return (int)k;
    return -1;
  }
};
// a one-site operator: 1x1 sub-blocks with their values
struct SiteOp {
  int up_dif, down_dif;
  struct S { int num_up, num_down, down_dif; double v; };
  std::vector<S> sub;
  int find(int nu, int nd, int dd, bool use_dd) const {
    for (size_t k = 0; k < sub.size(); ++k)
      if (sub[k].num_up == nu && sub[k].num_down == nd && (!use_dd || sub[k].down_dif == dd)) return (int)k;
    return -1;
  }
};

// a piece of an enlarged operator: rows [lpos, lpos + ldim) x columns
// [rpos, rpos + rdim) of its sector pair hold coef * op(O) (ident: coef * I)
struct Piece {
  int lpos, ldim, rpos, rdim;
  int64_t off;
  int ld;
  int8_t trans, ident;
  double coef;
};
// a sub-block of an enlarged operator: sector (num_up, num_down) -> shifted by
// (up_dif, down_dif); lsec / rsec are its target / source sectors in the basis
struct ESub {
  int num_up, num_down, down_dif, lsec, rsec;
  std::vector<Piece> p;
};
struct EBlk {
  int len = 0, up_dif = 0, down_dif = 0;
  bool set = false;   // holds an operator (slots of the reference's next%sub)
  std::vector<ESub> sub;
  int find(int nu, int nd, int dd, bool use_dd) const {
    for (size_t k = 0; k < sub.size(); ++k)
      if (sub[k].num_up == nu && sub[k].num_down == nd && (!use_dd || sub[k].down_dif == dd)) return (int)k;
    return -1;
  }
};

inline double m1(int n) { return (n % 2) ? -1.0 : 1.0; }   // (-1)**n
inline double fsign(char flag, int n) { return flag == 'F' ? m1(n) : 1.0; }

struct Ctx {
  const tj_basis *bs;
  int find_bs(int nu, int nd) const {
    for (int x = 0; x < bs->num; ++x)
      if (bs->sub[x].new_num_up == nu && bs->sub[x].new_num_down == nd) return x;
    return -1;
  }
  const tj_basis_sub &M(int x, int m) const { return bs->maps[bs->sub[x].first + m]; }
};

// update_block_dia (block.f90:382-433) / update_site_dia (block.f90:439-494)
EBlk enl_dia(const Ctx &c, const RBlk *blk, const SiteOp *site) {
  EBlk e;
  e.len = c.bs->len;
  e.set = true;
  for (int k = 0; k < c.bs->num; ++k) {
    ESub s{c.bs->sub[k].new_num_up, c.bs->sub[k].new_num_down, 0, k, k, {}};
    for (int x = 0; x < c.bs->sub[k].num; ++x) {
      const tj_basis_sub &m = c.M(k, x);
      if (blk) {
        const int i = blk->find(m.bl_num_up, m.bl_num_down, 0, false);
        if (i < 0) continue;
        const RSub &o = blk->sub[i];
        if (o.row_dim != m.sdim || o.sdim != m.sdim)
          throw RenormError(TJ_ERR_QN, "operator sub-block dimension differs from the basis");
        s.p.push_back(Piece{m.spos, m.sdim, m.spos, m.sdim, o.off, o.row_dim, 0, 0,
                            std::sqrt((1.0 + s.num_down) / (1.0 + o.num_down))});
      } else {
        const int i = site->find(m.st_num_up, m.st_num_down, 0, false);
        if (i < 0) continue;
        const double v = site->sub[i].v * std::sqrt((1.0 + s.num_down) / (1.0 + site->sub[i].num_down));
        s.p.push_back(Piece{m.spos, m.sdim, m.spos, m.sdim, 0, 0, 0, 1, v});
      }
    }
    e.sub.push_back(std::move(s));
  }
  return e;
}

// update_block_ndia_sys/env (block.f90:497-881) when blk is given,
// update_site_ndia_sys/env (block.f90:888-1306) when site is given
EBlk enl_ndia(const Ctx &c, const RBlk *blk, const SiteOp *site, bool env_side, char flag) {
  EBlk e;
  e.len = c.bs->len;
  e.set = true;
  e.up_dif = blk ? blk->up_dif : site->up_dif;
  e.down_dif = blk ? blk->down_dif : site->down_dif;
  const int up_dif = e.up_dif, d1 = e.down_dif;
  for (int x = 0; x < c.bs->num; ++x)
    for (int dd = -d1; dd <= d1; dd += 2) {
      const int rnu = c.bs->sub[x].new_num_up, rnd = c.bs->sub[x].new_num_down;
      const int y = c.find_bs(rnu + up_dif, rnd + dd);
      if (y < 0) continue;
      ESub s{rnu, rnd, dd, y, x, {}};
      const int lnd = rnd + dd;
      for (int q = 0; q < c.bs->sub[x].num; ++q) {
        const tj_basis_sub &m = c.M(x, q);
        for (int sdd = -d1; sdd <= d1; sdd += 2) {
          const tj_basis_sub *ml = nullptr;
          if (blk) {
            const int bid = blk->find(m.bl_num_up, m.bl_num_down, sdd, true);
            if (bid < 0) continue;
            const int lsnu = m.bl_num_up + up_dif, lsnd = m.bl_num_down + sdd;
            for (int r = 0; r < c.bs->sub[y].num && !ml; ++r) {
              const tj_basis_sub &t = c.M(y, r);
              if (t.bl_num_up == lsnu && t.bl_num_down == lsnd && t.st_num_down == m.st_num_down) ml = &t;
            }
            if (!ml) continue;
            const int j1 = lnd, j2 = d1, j3 = rnd, j4 = m.bl_num_down, j5 = m.st_num_down, j6 = lsnd;
            double coef = w6j(j1, j2, j3, j4, j5, j6) * std::sqrt((1.0 + j1) * (1.0 + j3)) * m1((j6 + j5 + j3 + j2) / 2);
            if (coef == 0.0) continue;
            if (env_side) coef *= fsign(flag, m.st_num_down);
            const RSub &o = blk->sub[bid];
            if (o.row_dim != ml->sdim || o.sdim != m.sdim)
              throw RenormError(TJ_ERR_QN, "operator sub-block dimension differs from the basis");
            s.p.push_back(Piece{ml->spos, ml->sdim, m.spos, m.sdim, o.off, o.row_dim, 0, 0, coef});
          } else {
            const int sid = site->find(m.st_num_up, m.st_num_down, sdd, true);
            if (sid < 0) continue;
            const int lsnu = m.st_num_up + up_dif, lsnd = m.st_num_down + sdd;
            for (int r = 0; r < c.bs->sub[y].num && !ml; ++r) {
              const tj_basis_sub &t = c.M(y, r);
              if (t.st_num_up == lsnu && t.st_num_down == lsnd && t.bl_num_down == m.bl_num_down) ml = &t;
            }
            if (!ml) continue;
            const int j1 = lnd, j2 = d1, j3 = rnd, j4 = m.st_num_down, j5 = m.bl_num_down, j6 = lsnd;
            double coef = w6j(j1, j2, j3, j4, j5, j6) * m1((j5 + j4 + j1 + j2) / 2) * std::sqrt((1.0 + j1) * (1.0 + j3));
            if (coef == 0.0) continue;
            if (!env_side) coef *= fsign(flag, m.bl_num_down);
            if (ml->sdim != m.sdim) throw RenormError(TJ_ERR_QN, "site operator window sizes differ");
            s.p.push_back(Piece{ml->spos, m.sdim, m.spos, m.sdim, 0, 0, 0, 1, coef * site->sub[sid].v});
          }
        }
      }
      e.sub.push_back(std::move(s));
    }
  return e;
}

// Get_hamiltonian_ndia (get_sys.f90:578-759): coef [block x site^T + h.c.]
void ham_ndia(const Ctx &c, const RBlk &blk, const SiteOp &site, double coef, EBlk &ham, char flagsign, bool sys_side) {
  const int up_dif = blk.up_dif, d1 = blk.down_dif;
  for (ESub &h : ham.sub) {
    const int rnd = h.num_down;
    const int x = h.rsec, y = h.lsec;
    for (int q = 0; q < c.bs->sub[x].num; ++q) {
      const tj_basis_sub &m = c.M(x, q);
      for (int sdd = -d1; sdd <= d1; sdd += 2) {
        const int bid = blk.find(m.bl_num_up, m.bl_num_down, sdd, true);
        if (bid < 0) continue;
        const int lsnu = m.bl_num_up + up_dif, lsnd = m.bl_num_down + sdd;
        for (int nsd = std::abs(m.st_num_down - site.down_dif); nsd <= m.st_num_down + site.down_dif; nsd += 2) {
          const int sid = site.find(m.st_num_up - site.up_dif, nsd, m.st_num_down - nsd, true);
          const tj_basis_sub *ml = nullptr;
          for (int r = 0; r < c.bs->sub[y].num && !ml; ++r) {
            const tj_basis_sub &t = c.M(y, r);
            if (t.bl_num_up == lsnu && t.bl_num_down == lsnd && t.st_num_down == nsd) ml = &t;
          }
          if (!ml || sid < 0) continue;
          const int j1 = lsnd, j2 = m.bl_num_down, j3 = d1, j4 = m.st_num_down, j5 = nsd, j6 = rnd;
          double c1 = w6j(j1, j2, j3, j4, j5, j6) * std::sqrt((1.0 + j6) / (1.0 + j3)) * m1((j2 + j5 + j3 + j6) / 2) *
                      site.sub[sid].v;
          if (c1 == 0.0) continue;
          double sign = 1.0;
          if (sys_side && flagsign == 'F' && ((m.bl_num_up % 2 == 1) || (m.bl_num_down % 2 == 1))) sign = -1.0;
          c1 *= coef * sign;
          const RSub &o = blk.sub[bid];
          if (o.row_dim != ml->sdim || o.sdim != m.sdim)
            throw RenormError(TJ_ERR_QN, "operator sub-block dimension differs from the basis");
          h.p.push_back(Piece{ml->spos, ml->sdim, m.spos, m.sdim, o.off, o.row_dim, 0, 0, c1});
          if (site.down_dif == 1) h.p.push_back(Piece{m.spos, m.sdim, ml->spos, ml->sdim, o.off, o.row_dim, 1, 0, c1});
        }
      }
    }
  }
}

// Get_hamiltonian_dia (get_sys.f90:507-565) with Flag1 = Flag2 = 'N' and no
// conjugate part: coef / sqrt(1 + 2S) * o1 * o2, o1 a block operator and o2 a
// site operator enlarged by update_block_dia / update_site_dia (both
// block-diagonal over the basis's sub-sectors, o2 a multiple of I on each)
void ham_dia(const EBlk &o1, const EBlk &o2, double coef, EBlk &ham) {
  for (ESub &h : ham.sub) {
    const int a = o1.find(h.num_up, h.num_down, 0, false), b = o2.find(h.num_up, h.num_down, 0, false);
    if (a < 0 || b < 0) continue;
    const double c1 = coef / std::sqrt(1.0 + h.num_down);
    for (const Piece &p1 : o1.sub[a].p)
      for (const Piece &p2 : o2.sub[b].p) {
        if (!p2.ident || p2.lpos != p2.rpos) throw RenormError(TJ_ERR_ARG, "site operator is not diagonal");
        if (p2.lpos != p1.rpos) continue;
        Piece q = p1;
        q.coef = p1.coef * p2.coef * c1;
        h.p.push_back(q);
      }
  }
}

// block_add_block_two (block.f90:1786-1822): the search restarts after the last match
void add_two(const EBlk &b1, double coef, EBlk &nw) {
  size_t x1 = 0;
  for (ESub &s : nw.sub)
    for (size_t x = x1; x < b1.sub.size(); ++x) {
      const ESub &q = b1.sub[x];
      if (q.num_up == s.num_up && q.num_down == s.num_down && q.down_dif == s.down_dif) {
        for (Piece p : q.p) {
          p.coef *= coef;
          s.p.push_back(p);
        }
        x1 = x + 1;
        break;
      }
    }
}

// one sector of the truncation operator, in the trun space
struct TSec {
  int num_up, num_down, row_dim, kept;
  int64_t off;
};
struct TBlk {
  std::vector<TSec> sec;
  int find(int nu, int nd) const {
    for (size_t k = 0; k < sec.size(); ++k)
      if (sec[k].num_up == nu && sec[k].num_down == nd) return (int)k;
    return -1;
  }
};

// output sub-block records, in the order of the result
struct OutSub {
  tj_block_sub rec;
};
struct OutBlk {
  int len, up_dif, down_dif, dim;
  int first, num;   // records [first, first + num)
};

struct Builder {
  const tj_lattice *L;
  Ctx c;
  HpsiPlan &P;
  TBlk trun;
  int trun_dim = 0;   // trun%dim: the dimension update_trun_dia gives its result
  std::vector<tj_block_sub> recs;
  std::vector<OutBlk> blocks;
  int64_t out_len = 0;
  struct Key {
    int64_t a, b;
    int32_t m, n, k;
    int8_t ta, tb, assoc;
    bool operator==(const Key &o) const {
      return a == o.a && b == o.b && m == o.m && n == o.n && k == o.k && ta == o.ta && tb == o.tb && assoc == o.assoc;
    }
  };
  struct KeyHash {
    size_t operator()(const Key &k) const {
      uint64_t h = (uint64_t)k.a * 0x9e3779b97f4a7c15ull ^ ((uint64_t)k.b + 0x632be59bd9b4e019ull);
      h ^= ((uint64_t)(uint32_t)k.m << 32 | (uint32_t)k.n) * 0xbf58476d1ce4e5b9ull;
      h ^= (uint64_t)(uint32_t)k.k * 31 + (uint64_t)(k.ta * 4 + k.tb * 2 + k.assoc);
      return (size_t)h;
    }
  };
  std::unordered_map<Key, int64_t, KeyHash> prod;   // phase-1 product -> its scratch offset
  std::vector<Task> t2;
  std::vector<int32_t> t2cell;

  Builder(const tj_lattice *l, const tj_basis *b, HpsiPlan &p) : L(l), P(p) { c.bs = b; }

  int64_t product(const Operand &Lop, const Operand &Rop, int M, int N, int K, int8_t assoc) {
    Key key{Lop.space == SP_OPS ? Lop.off : Rop.off, Lop.space == SP_OPS ? Rop.off : Lop.off, M, N, K,
            Lop.trans, Rop.trans, assoc};
    auto it = prod.find(key);
    if (it != prod.end()) return it->second;
    const int64_t off = P.scratch_len;
    P.scratch_len += (int64_t)M * N;
    P.scratch_len = (P.scratch_len + 3) / 4 * 4;
    Cell cl;
    std::memset(&cl, 0, sizeof cl);
    cl.off = off;
    cl.ld = M;
    cl.M = M;
    cl.N = N;
    cl.t_begin = (int32_t)P.tasks1.size();
    cl.t_end = cl.t_begin + 1;
    cl.space = SP_SCR;
    Task t;
    std::memset(&t, 0, sizeof t);
    t.L = Lop;
    t.R = Rop;
    t.coef = 1.0;
    t.K = K;
    P.tasks1.push_back(t);
    P.cells1.push_back(cl);
    P.flops += 2.0 * M * N * (double)K;
    prod.emplace(key, off);
    return off;
  }

  static Operand opnd(int64_t off, int ld, int8_t space, int8_t trans) {
    Operand o;
    o.off = off;
    o.ld = ld;
    o.space = space;
    o.trans = trans;
    o.pad = 0;
    return o;
  }

  // tasks of output sub-block `cell` (kl x kr) from the pieces of `es`
  void emit(const ESub &es, const TSec &tl, const TSec &tr, int cell) {
    const int kl = tl.kept, kr = tr.kept;
    if (kl == 0 || kr == 0) return;
    for (const Piece &p : es.p) {
      if (p.ldim == 0 || p.rdim == 0 || p.coef == 0.0) continue;
      if (p.lpos + p.ldim > tl.row_dim || p.rpos + p.rdim > tr.row_dim)
        throw RenormError(TJ_ERR_QN, "truncation operator smaller than the enlarged sector");
      const Operand Ul = opnd(tl.off + p.lpos, tl.row_dim, SP_PSI, 1);   // U_l[rows]^T : kl x ldim
      const Operand Ur = opnd(tr.off + p.rpos, tr.row_dim, SP_PSI, 0);   // U_r[cols]   : rdim x kr
      Task t;
      std::memset(&t, 0, sizeof t);
      t.coef = p.coef;
      if (p.ident) {
        t.L = Ul;
        t.R = Ur;
        t.K = p.ldim;
        P.flops += 2.0 * kl * kr * (double)p.ldim;
      } else {
        const Operand O = opnd(p.off, p.ld, SP_OPS, p.trans);            // op(O) : ldim x rdim
        const double ca = (double)p.ldim * p.rdim * kr + (double)kl * p.ldim * kr;
        const double cb = (double)kl * p.ldim * p.rdim + (double)kl * p.rdim * kr;
        if (ca <= cb) {   // (op(O) U_r), then U_l^T (.)
          const int64_t off = product(O, Ur, p.ldim, kr, p.rdim, 0);
          t.L = Ul;
          t.R = opnd(off, p.ldim, SP_SCR, 0);
          t.K = p.ldim;
          P.flops += 2.0 * kl * kr * (double)p.ldim;
        } else {          // (U_l^T op(O)), then (.) U_r
          const int64_t off = product(Ul, O, kl, p.rdim, p.ldim, 1);
          t.L = opnd(off, kl, SP_SCR, 0);
          t.R = Ur;
          t.K = p.rdim;
          P.flops += 2.0 * kl * kr * (double)p.rdim;
        }
      }
      t2.push_back(t);
      t2cell.push_back(cell);
    }
  }

  // update_trun_dia (block.f90:1311-1362) / update_trun_ndia (block.f90:1365-
  // 1503) of the enlarged operator `e`: the output block's records and tasks
  void truncate(const EBlk &e, bool dia, int len) {
    OutBlk ob{len, e.up_dif, e.down_dif, 0, (int)recs.size(), 0};
    auto add = [&](const ESub *es, int li, int ri, int dd) {
      const TSec &tl = trun.sec[li], &tr = trun.sec[ri];
      tj_block_sub r;
      std::memset(&r, 0, sizeof r);
      r.num_up = tr.num_up;
      r.num_down = tr.num_down;
      r.down_dif = dd;
      r.row_dim = tl.kept;
      r.sdim = tr.kept;
      r.off = out_len;
      const int cell = (int)P.cells2.size();
      Cell cl;
      std::memset(&cl, 0, sizeof cl);
      cl.off = out_len;
      cl.ld = std::max(1, tl.kept);
      cl.M = tl.kept;
      cl.N = tr.kept;
      cl.space = SP_PSI;
      P.cells2.push_back(cl);
      if (es) emit(*es, tl, tr, cell);
      out_len += (int64_t)tl.kept * tr.kept;
      recs.push_back(r);
      ob.num++;
    };
    if (dia) {
      for (size_t i = 0; i < trun.sec.size(); ++i) {
        const int x = e.find(trun.sec[i].num_up, trun.sec[i].num_down, 0, false);
        add(x >= 0 ? &e.sub[x] : nullptr, (int)i, (int)i, 0);
      }
      ob.dim = trun_dim;
    } else {
      const int d1 = e.down_dif;
      for (size_t x = 0; x < trun.sec.size(); ++x)
        for (int dd = -d1; dd <= d1; dd += 2) {
          const int y = trun.find(trun.sec[x].num_up + e.up_dif, trun.sec[x].num_down + dd);
          if (y < 0) continue;
          const int o = e.find(trun.sec[x].num_up, trun.sec[x].num_down, dd, true);
          add(o >= 0 ? &e.sub[o] : nullptr, y, (int)x, dd);
          ob.dim += trun.sec[x].kept;
        }
    }
    blocks.push_back(ob);
  }

  void empty_block(int len) { blocks.push_back(OutBlk{len, 0, 0, 0, (int)recs.size(), 0}); }
};

int64_t align4(int64_t x) { return (x + 3) / 4 * 4; }

void load_block(const tj_block &b, RBlk &o, HpsiPlan &P) {
  o.len = b.len;
  o.up_dif = b.up_dif;
  o.down_dif = b.down_dif;
  o.sub.clear();
  if (b.num < 0 || (b.num > 0 && (!b.sub || !b.data))) throw RenormError(TJ_ERR_ARG, "block with null sub/data");
  int64_t lo = LLONG_MAX, hi = 0;
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &s = b.sub[k];
    if (s.row_dim < 0 || s.sdim < 0 || s.off < 0) throw RenormError(TJ_ERR_ARG, "negative sub-block size");
    lo = std::min(lo, (int64_t)s.off);
    hi = std::max(hi, (int64_t)s.off + (int64_t)s.row_dim * s.sdim);
  }
  if (b.num == 0) return;
  const int64_t base = P.ops_len;
  P.uploads.push_back({b.data + lo, hi - lo, base});
  P.ops_len += align4(hi - lo);
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &s = b.sub[k];
    o.sub.push_back(RSub{s.num_up, s.num_down, s.down_dif, s.row_dim, s.sdim, base + (s.off - lo)});
  }
}

}  // namespace

// The compiled renormalisation of one block.
struct RenormPlan {
  HpsiPlan P;                       // operator space = old block, psi space = trun, out = new operators
  std::vector<tj_block_sub> recs;   // output records (result order)
  std::vector<OutBlk> blocks;       // ham, then 5 per set
  int len = 0, nsub = 0;
  int64_t out_len = 0;
  uint64_t key = 0;
};

int build_renorm_plan(const tj_lattice *lat, int side, int mshift, const tj_model *pre, const tj_basis *basis,
                      const tj_block *trunb, RenormPlan &R, std::string &msg) {
  try {
    if (!lat || !pre || !basis || !trunb) throw RenormError(TJ_ERR_ARG, "null argument");
    if (!lat->neib || !lat->inb1 || !lat->nleg11 || !lat->jt || !lat->jd || !lat->jn || !lat->esite ||
        (side && (!lat->nposi_lat || !lat->nposi_dm)))
      throw RenormError(TJ_ERR_ARG, "null lattice table");
    if (side != 0 && side != 1) throw RenormError(TJ_ERR_ARG, "side must be 0 (system) or 1 (environment)");
    if (!basis->sub || !basis->maps || basis->num < 1) throw RenormError(TJ_ERR_ARG, "empty basis");
    if (pre->nsub < 0 || (pre->nsub > 0 && !pre->sub)) throw RenormError(TJ_ERR_ARG, "model without operator sets");
    const int len0 = pre->len, ns1 = lat->num_site + 1, neibt = lat->neibt;
    if (len0 < 1 || len0 + 1 > lat->num_site - 2 + 1) throw RenormError(TJ_ERR_ARG, "block length out of range");
    HpsiPlan &P = R.P;
    Builder B(lat, basis, P);
    // the truncation operator in the psi space
    {
      if (trunb->num < 1 || !trunb->sub || !trunb->data) throw RenormError(TJ_ERR_ARG, "empty truncation operator");
      int64_t lo = LLONG_MAX, hi = 0;
      for (int k = 0; k < trunb->num; ++k) {
        const tj_block_sub &s = trunb->sub[k];
        if (s.row_dim < 0 || s.sdim < 0 || s.off < 0) throw RenormError(TJ_ERR_ARG, "bad truncation sub-block");
        lo = std::min(lo, (int64_t)s.off);
        hi = std::max(hi, (int64_t)s.off + (int64_t)s.row_dim * s.sdim);
      }
      for (int k = 0; k < trunb->num; ++k) {
        const tj_block_sub &s = trunb->sub[k];
        const int x = B.c.find_bs(s.num_up, s.num_down);
        if (x < 0 || basis->sub[x].dim != s.row_dim)
          throw RenormError(TJ_ERR_QN, "truncation sector does not match the basis");
        B.trun.sec.push_back(TSec{s.num_up, s.num_down, s.row_dim, s.sdim, s.off - lo});
      }
      P.psi_len = hi - lo;   // the trun span, uploaded from its lowest sub-block offset
      B.trun_dim = trunb->dim;
    }
    const int nl0 = lat->nleg11[len0 - 1], nl1 = lat->nleg11[len0];
    if (pre->nsub < nl0) throw RenormError(TJ_ERR_ARG, "the block has fewer operator sets than nleg11(len)");
    RBlk ham;
    load_block(pre->ham, ham, P);
    std::vector<std::array<RBlk, 5>> ps(pre->nsub);
    for (int i = 0; i < pre->nsub; ++i) {
      load_block(pre->sub[i].elec_up, ps[i][0], P);
      load_block(pre->sub[i].elec_down, ps[i][1], P);
      load_block(pre->sub[i].spin_sd, ps[i][2], P);
      load_block(pre->sub[i].num_sn, ps[i][4], P);
    }
    const int ub = lat->up_bias;
    const SiteOp s_eu{ub, 1, {{0, 0, 1, -std::sqrt(2.0)}}};
    const SiteOp s_ed{-ub, 1, {{ub, 1, -1, -std::sqrt(2.0)}}};
    const SiteOp s_ne{0, 0, {{0, 0, 0, 0.0}, {ub, 1, 0, std::sqrt(2.0)}}};
    const SiteOp s_sd{0, 2, {{ub, 1, 0, std::sqrt(1.5)}}};
    auto NEIB = [&](int i, int k) { return lat->neib[(int64_t)(k - 1) * ns1 + i]; };
    auto INB1 = [&](int i, int j) { return lat->inb1[(int64_t)j * ns1 + i]; };
    const bool env = side == 1;
    const int J = env ? len0 + 1 + mshift : len0 + 1;
    if (J < 0 || J > lat->num_site) throw RenormError(TJ_ERR_ARG, "mshift puts the new site outside the lattice");
    const int jl = env ? lat->nposi_lat[J] : J;   // lattice index of the new site
    if (jl < 1 || jl > lat->num_site) throw RenormError(TJ_ERR_ARG, "new site outside the lattice");
    // block sites bonded to the new site: (operator slot, neighbour direction)
    std::vector<std::pair<int, int>> bonded;
    for (int k = 1; k <= neibt; ++k) {
      const int I = NEIB(jl, k);
      const int II = env ? ((I >= 0 && I <= lat->num_site) ? lat->nposi_dm[I] - mshift : 0) : I;
      if (!(II <= len0 && II > 0)) continue;
      const int i1 = INB1(II, len0);
      if (!(i1 > 0 && i1 <= nl0)) continue;
      bonded.push_back({i1, k});
    }
    auto JT = [&](int k) { return lat->jt[(int64_t)jl * neibt + k - 1]; };
    auto JD = [&](int k) { return lat->jd[(int64_t)jl * neibt + k - 1]; };
    auto JN = [&](int k) { return lat->jn[k - 1]; };
    EBlk nham = enl_dia(B.c, &ham, nullptr);
    const int nslot = std::max(nl0, nl1) + 1;
    std::vector<std::array<EBlk, 5>> next(nslot);
    R.len = len0 + 1;
    R.nsub = nl1;
    std::vector<std::array<EBlk, 5>> keep(nl1 + 1);   // enlarged operators of the new sets, by slot
    for (int ij = 1; ij <= 5; ij += 2) {
      for (auto &bk : bonded) {
        const int i1 = bk.first, k = bk.second;
        if (ij == 1 && JT(k) != 0.0) ham_ndia(B.c, ps[i1 - 1][0], s_eu, JT(k), nham, 'F', !env);
        if (ij == 3 && JD(k) != 0.0) ham_ndia(B.c, ps[i1 - 1][2], s_sd, JD(k), nham, 'B', !env);
      }
      const int kinds[2] = {ij == 1 ? 0 : ij == 3 ? 2 : 4, 1};
      const int nk = ij == 1 ? 2 : 1;
      for (int y = 1; y <= len0; ++y) {
        const int i1 = INB1(y, len0);
        if (i1 < 1 || i1 > nl0) continue;
        for (int q = 0; q < nk; ++q) {
          const int kd = kinds[q];
          next[i1][kd] = kd == 4 ? enl_dia(B.c, &ps[i1 - 1][4], nullptr)
                                 : enl_ndia(B.c, &ps[i1 - 1][kd], nullptr, env, kd == 2 ? 'B' : 'F');
        }
      }
      EBlk tmp, tmp1;
      if (ij == 1) {
        tmp = enl_ndia(B.c, nullptr, &s_eu, env, 'F');
        tmp1 = enl_ndia(B.c, nullptr, &s_ed, env, 'F');
      } else if (ij == 3) {
        tmp = enl_ndia(B.c, nullptr, &s_sd, env, 'B');
      } else {
        tmp = enl_dia(B.c, nullptr, &s_ne);
      }
      if (ij == 5) {
        for (auto &bk : bonded) ham_dia(next[bk.first][4], tmp, JN(bk.second), nham);
        const double es = lat->esite[jl];
        if (es != 0.0) add_two(tmp, es, nham);
      }
      // reorder (get_sys.f90:127-150): the sites that keep bonds move down, the new site last
      for (int I = 1; I <= len0; ++I) {
        const int i1 = INB1(I, len0), j = INB1(I, len0 + 1);
        if (j <= nl1 && j != i1) {
          if (i1 < 1 || i1 >= nslot || j < 1) throw RenormError(TJ_ERR_ARG, "operator slot table out of range");
          for (int q = 0; q < nk; ++q) next[j][kinds[q]] = next[i1][kinds[q]];
        }
      }
      const int jn = INB1(len0 + 1, len0 + 1);
      if (jn < 1 || jn >= nslot) throw RenormError(TJ_ERR_ARG, "new site has no operator slot");
      next[jn][kinds[0]] = tmp;
      if (ij == 1) next[jn][1] = tmp1;
      for (int ii = 1; ii <= nl1; ++ii)
        for (int q = 0; q < nk; ++q) keep[ii][kinds[q]] = next[ii][kinds[q]];
    }
    // truncated output, in result order: ham, then each set's five operators
    B.truncate(nham, true, len0 + 1);
    for (int ii = 1; ii <= nl1; ++ii) {
      B.truncate(keep[ii][0], false, len0 + 1);
      B.truncate(keep[ii][1], false, len0 + 1);
      B.truncate(keep[ii][2], false, len0 + 1);
      B.empty_block(len0 + 1);
      B.truncate(keep[ii][4], true, len0 + 1);
    }
    // tasks sorted by output cell (stable: emission order within a cell)
    {
      std::vector<int32_t> cnt(P.cells2.size() + 1, 0);
      for (int32_t c : B.t2cell) cnt[c + 1]++;
      for (size_t i = 0; i < P.cells2.size(); ++i) cnt[i + 1] += cnt[i];
      P.tasks2.resize(B.t2.size());
      std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
      for (size_t t = 0; t < B.t2.size(); ++t) P.tasks2[pos[B.t2cell[t]]++] = B.t2[t];
      std::vector<Cell> kept;
      for (size_t i = 0; i < P.cells2.size(); ++i) {
        if (cnt[i + 1] == cnt[i]) continue;   // zero sub-block: the output is cleared first
        Cell cl = P.cells2[i];
        cl.t_begin = cnt[i];
        cl.t_end = cnt[i + 1];
        kept.push_back(cl);
      }
      P.cells2.swap(kept);
    }
    R.recs = std::move(B.recs);
    R.blocks = std::move(B.blocks);
    R.out_len = B.out_len;
    double bytes = 0;
    for (const auto &u : P.uploads) bytes += 8.0 * u.n;
    P.bytes = bytes + 8.0 * (P.psi_len + R.out_len);
    split_tiles(P.cells1, P.tasks1, P.tiles1, P.red1, P.nslots1, false);
    split_tiles(P.cells2, P.tasks2, P.tiles2, P.red2, P.nslots2, false);
    return TJ_OK;
  } catch (const RenormError &e) {
    msg = e.what();
    return e.code;
  } catch (const std::exception &e) {
    msg = e.what();
    return TJ_ERR_ARG;
  }
}

// Fills the caller's result from the plan's records (and `data` when given).
static void fill_result(const RenormPlan &R, tj_model_result *out) {
  out->len = R.len;
  out->nsub = R.nsub;
  out->n_subs = (int32_t)R.recs.size();
  out->data_len = R.out_len;
  if (!(out->sets && out->subs && out->data)) return;
  std::memcpy(out->subs, R.recs.data(), R.recs.size() * sizeof(tj_block_sub));
  auto blk = [&](const OutBlk &b) {
    tj_block t;
    std::memset(&t, 0, sizeof t);
    t.len = b.len;
    t.num = b.num;
    t.dim = b.dim;
    t.up_dif = b.up_dif;
    t.down_dif = b.down_dif;
    t.sub = out->subs + b.first;
    t.data = out->data;
    return t;
  };
  out->model.len = R.len;
  out->model.nsub = R.nsub;
  out->model.ham = blk(R.blocks[0]);
  for (int i = 0; i < R.nsub; ++i) {
    const size_t b = 1 + 5 * (size_t)i;
    out->sets[i] = tj_block_set{blk(R.blocks[b]), blk(R.blocks[b + 1]), blk(R.blocks[b + 2]), blk(R.blocks[b + 3]),
                                blk(R.blocks[b + 4])};
  }
  out->model.sub = out->sets;
}

}  // namespace tjb

struct tj_renorm_state {
  tjb::RenormPlan plan;
  bool valid = false;
};
std::shared_ptr<tj_renorm_state> tjb::new_renorm_state() { return std::make_shared<tj_renorm_state>(); }

namespace {

uint64_t fnv(uint64_t h, const void *p, size_t n) {
  const unsigned char *c = (const unsigned char *)p;
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}
uint64_t key_block(uint64_t h, const tj_block &b) {
  h = fnv(h, &b, sizeof b);
  if (b.num > 0 && b.sub) h = fnv(h, b.sub, sizeof(tj_block_sub) * b.num);
  return h;
}
// structural key of a renormalisation call: tables and data pointers (the
// two calls of the result protocol must pass the same inputs)
uint64_t renorm_key(const tj_lattice *lat, int side, int mshift, const tj_model *pre, const tj_basis *basis,
                    const tj_block *trun) {
  uint64_t h = 1469598103934665603ull;
  h = fnv(h, lat, sizeof *lat);
  h = fnv(h, &side, sizeof side);
  h = fnv(h, &mshift, sizeof mshift);
  h = fnv(h, pre, sizeof *pre);
  h = key_block(h, pre->ham);
  for (int i = 0; i < pre->nsub && pre->sub; ++i) {
    const tj_block_set &s = pre->sub[i];
    h = key_block(key_block(key_block(key_block(h, s.elec_up), s.elec_down), s.spin_sd), s.num_sn);
  }
  h = fnv(h, basis, sizeof *basis);
  if (basis->sub) h = fnv(h, basis->sub, sizeof(tj_basis_map) * basis->num);
  return key_block(h, *trun);
}

}  // namespace

extern "C" int tj_get_hamiltonian(tj_ctx *ctx, const tj_lattice *lat, int side, int mshift, const tj_model *pre,
                                  const tj_basis *basis, const tj_block *trun, tj_model_result *out) {
  using namespace tjb;
  if (!ctx || !lat || !pre || !basis || !trun || !out) return set_err(TJ_ERR_ARG, "tj_get_hamiltonian: null argument");
  const uint64_t key = renorm_key(lat, side, mshift, pre, basis, trun);
  if (!ctx->renorm) ctx->renorm = new_renorm_state();
  tj_renorm_state &S = *ctx->renorm;
  if (!(S.valid && S.plan.key == key)) {
    S.valid = false;
    S.plan = RenormPlan();
    std::string msg;
    const auto t0 = std::chrono::steady_clock::now();
    int rc = build_renorm_plan(lat, side, mshift, pre, basis, trun, S.plan, msg);
    if (rc) return set_err(rc, "tj_get_hamiltonian: " + msg);
    S.plan.key = key;
    S.valid = true;
    ctx->stats.renorm_plan_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  const RenormPlan &R = S.plan;
  if (!(out->sets && out->subs && out->data)) {
    fill_result(R, out);
    return TJ_OK;
  }
  // second call: upload, two grouped-GEMM passes, download
  const auto h0 = std::chrono::steady_clock::now();
  const HpsiPlan &P = R.P;
  CKR(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = ctx->rnOps.reserve(sizeof(double) * (P.ops_len + 4))) ||
      (rc = ctx->rnTrun.reserve(sizeof(double) * (P.psi_len + 4))) ||
      (rc = ctx->rnScr.reserve(sizeof(double) * (P.scratch_len + 4))) ||
      (rc = ctx->rnOut.reserve(sizeof(double) * (R.out_len + 4))) ||
      (rc = ctx->rnSlots.reserve(sizeof(double) * (std::max(P.nslots1, P.nslots2) * BM * BN + 4))))
    return rc;
  const double pre_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
  CKR(cudaEventRecord(ctx->ev[5], st));
  for (const auto &u : P.uploads)
    if (u.n > 0) CKR(upload(ctx, ctx->rnOps.d() + u.dst, u.src, u.n, st));
  {
    int64_t lo = LLONG_MAX;
    for (int k = 0; k < trun->num; ++k) lo = std::min(lo, (int64_t)trun->sub[k].off);
    CKR(upload(ctx, ctx->rnTrun.d(), trun->data + lo, P.psi_len, st));
  }
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
  const size_t o_r1 = add(P.red1.data(), P.red1.size() * sizeof(Reduce));
  const size_t o_c2 = add(P.cells2.data(), P.cells2.size() * sizeof(Cell));
  const size_t o_t2 = add(P.tasks2.data(), P.tasks2.size() * sizeof(Task));
  const size_t o_l2 = add(P.tiles2.data(), P.tiles2.size() * sizeof(Tile));
  const size_t o_r2 = add(P.red2.data(), P.red2.size() * sizeof(Reduce));
  const size_t o_cnt = add(nullptr, 16);
  std::memset(tab.data() + o_cnt, 0, 16);
  if ((rc = ctx->rnTab.reserve(tab.size() + 256))) return rc;
  CKR(cudaMemcpyAsync(ctx->rnTab.p, tab.data(), tab.size(), cudaMemcpyHostToDevice, st));
  CKR(cudaMemsetAsync(ctx->rnOut.p, 0, sizeof(double) * (R.out_len + 4), st));
  char *tb = (char *)ctx->rnTab.p;
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = ctx->rnOps.d();
  g.psi = ctx->rnTrun.d();
  g.scr = ctx->rnScr.d();
  g.out = ctx->rnScr.d();
  g.cells = (const Cell *)(tb + o_c1);
  g.tasks = (const Task *)(tb + o_t1);
  g.tiles = (const Tile *)(tb + o_l1);
  g.ntiles = (int)P.tiles1.size();
  g.counter = (unsigned int *)(tb + o_cnt);
  g.slots = ctx->rnSlots.d();
  CKR(cudaEventRecord(ctx->ev[0], st));
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r1), (int)P.red1.size(), st);
  g.out = ctx->rnOut.d();
  g.cells = (const Cell *)(tb + o_c2);
  g.tasks = (const Task *)(tb + o_t2);
  g.tiles = (const Tile *)(tb + o_l2);
  g.ntiles = (int)P.tiles2.size();
  g.counter = (unsigned int *)(tb + o_cnt) + 1;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r2), (int)P.red2.size(), st);
  CKR(cudaEventRecord(ctx->ev[1], st));
  CKR(cudaGetLastError());
  if ((rc = download(ctx, out->data, ctx->rnOut.d(), R.out_len, st))) return rc;
  CKR(cudaEventRecord(ctx->ev[2], st));
  CKR(cudaStreamSynchronize(st));
  float gemm_ms = 0, all_ms = 0;
  cudaEventElapsedTime(&gemm_ms, ctx->ev[0], ctx->ev[1]);
  cudaEventElapsedTime(&all_ms, ctx->ev[5], ctx->ev[2]);
  ctx->stats.renorm_ms = gemm_ms;
  ctx->stats.renorm_e2e_ms = all_ms;
  ctx->stats.renorm_flops = P.flops;
  const auto h1 = std::chrono::steady_clock::now();
  fill_result(R, out);
  if ((rc = res_keep(ctx, out->data, R.out_len, ctx->rnOut.d(), st))) return rc;
  ctx->stats.renorm_pre_ms = pre_ms;
  ctx->stats.renorm_post_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h1).count();
  return TJ_OK;
}

// The compiled renormalisation, for checks on the CPU: operator space = the
// old block's blocks (uploads), input space = the truncation operator's data
// from its lowest sub-block offset, output space = the new operators in the
// result's order (psi_len of the export is the output length).  `res`
// (optional) receives the result's sizes and, with its arrays set, its
// records and blocks (its data is not written).
extern "C" int tj_renorm_plan_export(const tj_lattice *lat, int side, int mshift, const tj_model *pre,
                                     const tj_basis *basis, const tj_block *trun, tj_plan_export *out,
                                     tj_model_result *res) {
  using namespace tjb;
  if (!out) return set_err(TJ_ERR_ARG, "null output");
  RenormPlan R;
  std::string msg;
  int rc = build_renorm_plan(lat, side, mshift, pre, basis, trun, R, msg);
  if (rc) return set_err(rc, "renormalisation plan: " + msg);
  R.P.psi_len = R.out_len;
  if (res) fill_result(R, res);
  return export_hpsi_plan(R.P, out);
}

// ================================================= measurement operators
// Get_*_oper_* / Change_*_oper_* (code/tjsq/get_sys.f90:764-1238): an
// operator carried through the stored bases and truncations of one side,
// one step per block length -- each step the same enlarge-and-truncate pass
// as the renormalisation above, with the operator staying on the device
// between steps -- and block_mul_block_ndia / update_trun on their own.
namespace tjb {
namespace {

// a block operator resident on the device: structure on the host, matrices in buf
struct DevOp {
  RBlk b;
  int dim = 0;
  DevBuf buf;
  DevOp() = default;
  DevOp(const DevOp &) = delete;
  DevOp &operator=(const DevOp &) = delete;
  ~DevOp() { buf.release(); }
};

// the two grouped-GEMM passes of a plan whose operand spaces are on the device
int exec_passes(tj_ctx *ctx, const HpsiPlan &P, const double *ops, const double *psi, double *out) {
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = ctx->rnScr.reserve(sizeof(double) * (P.scratch_len + 4))) ||
      (rc = ctx->rnSlots.reserve(sizeof(double) * (std::max(P.nslots1, P.nslots2) * BM * BN + 4))))
    return rc;
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
  const size_t o_r1 = add(P.red1.data(), P.red1.size() * sizeof(Reduce));
  const size_t o_c2 = add(P.cells2.data(), P.cells2.size() * sizeof(Cell));
  const size_t o_t2 = add(P.tasks2.data(), P.tasks2.size() * sizeof(Task));
  const size_t o_l2 = add(P.tiles2.data(), P.tiles2.size() * sizeof(Tile));
  const size_t o_r2 = add(P.red2.data(), P.red2.size() * sizeof(Reduce));
  const size_t o_cnt = add(nullptr, 16);
  std::memset(tab.data() + o_cnt, 0, 16);
  if ((rc = ctx->rnTab.reserve(tab.size() + 256))) return rc;
  CKR(cudaMemcpyAsync(ctx->rnTab.p, tab.data(), tab.size(), cudaMemcpyHostToDevice, st));
  char *tb = (char *)ctx->rnTab.p;
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = ops;
  g.psi = psi;
  g.scr = ctx->rnScr.d();
  g.out = ctx->rnScr.d();
  g.cells = (const Cell *)(tb + o_c1);
  g.tasks = (const Task *)(tb + o_t1);
  g.tiles = (const Tile *)(tb + o_l1);
  g.ntiles = (int)P.tiles1.size();
  g.counter = (unsigned int *)(tb + o_cnt);
  g.slots = ctx->rnSlots.d();
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r1), (int)P.red1.size(), st);
  g.out = out;
  g.cells = (const Cell *)(tb + o_c2);
  g.tasks = (const Task *)(tb + o_t2);
  g.tiles = (const Tile *)(tb + o_l2);
  g.ntiles = (int)P.tiles2.size();
  g.counter = (unsigned int *)(tb + o_cnt) + 1;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r2), (int)P.red2.size(), st);
  CKR(cudaGetLastError());
  // the tables and the truncation buffer are rewritten by the next pass: wait for this one
  CKR(cudaStreamSynchronize(st));
  return TJ_OK;
}

// a host block uploaded into a device operator
int upload_op(tj_ctx *ctx, const tj_block &b, DevOp &d) {
  HpsiPlan P;
  load_block(b, d.b, P);
  d.dim = b.dim;
  int rc = d.buf.reserve(sizeof(double) * (P.ops_len + 4));
  if (rc) return rc;
  for (const auto &u : P.uploads)
    if (u.n > 0) CKR(upload(ctx, d.buf.d() + u.dst, u.src, u.n, ctx->stream));
  return TJ_OK;
}

// host storage of a truncation operator made of unit matrices (block_transfer_basis)
struct IdTrun {
  std::vector<tj_block_sub> subs;
  std::vector<double> data;
  tj_block blk;
  explicit IdTrun(const tj_basis *bs) {
    int64_t off = 0;
    for (int i = 0; i < bs->num; ++i) {
      const int d = bs->sub[i].dim;
      tj_block_sub s;
      std::memset(&s, 0, sizeof s);
      s.num_up = bs->sub[i].new_num_up;
      s.num_down = bs->sub[i].new_num_down;
      s.row_dim = d;
      s.sdim = d;
      s.off = off;
      subs.push_back(s);
      off += (int64_t)d * d;
    }
    data.assign(std::max<int64_t>(off, 1), 0.0);
    for (const auto &s : subs)
      for (int k = 0; k < s.row_dim; ++k) data[s.off + (int64_t)k * s.row_dim + k] = 1.0;
    std::memset(&blk, 0, sizeof blk);
    blk.len = bs->len;
    blk.num = (int32_t)subs.size();
    blk.dim = bs->dim;
    blk.sub = subs.data();
    blk.data = data.data();
  }
};

// U^T E U of an enlarged operator (pieces over the device operator `in_dev`):
// the truncation operator trun is uploaded, one plan, two passes -> out
int trunc_step(tj_ctx *ctx, const EBlk &e, bool dia, int len, const tj_block &trun, const tj_basis *basis,
               const double *in_dev, DevOp &out, std::string &msg) {
  if (trun.num < 1 || !trun.sub || !trun.data) {
    msg = "empty truncation operator";
    return TJ_ERR_ARG;
  }
  HpsiPlan P;
  Builder B(nullptr, basis, P);
  int64_t lo = LLONG_MAX, hi = 0;
  for (int k = 0; k < trun.num; ++k) {
    const tj_block_sub &s = trun.sub[k];
    if (s.row_dim < 0 || s.sdim < 0 || s.off < 0) {
      msg = "bad truncation sub-block";
      return TJ_ERR_ARG;
    }
    lo = std::min(lo, (int64_t)s.off);
    hi = std::max(hi, (int64_t)s.off + (int64_t)s.row_dim * s.sdim);
  }
  for (int k = 0; k < trun.num; ++k) {
    const tj_block_sub &s = trun.sub[k];
    B.trun.sec.push_back(TSec{s.num_up, s.num_down, s.row_dim, s.sdim, s.off - lo});
  }
  B.trun_dim = trun.dim;
  try {
    B.truncate(e, dia, len);
  } catch (const RenormError &er) {
    msg = er.what();
    return er.code;
  }
  {   // tasks sorted by cell (the cells were emitted in record order)
    std::vector<int32_t> cnt(P.cells2.size() + 1, 0);
    for (int32_t c : B.t2cell) cnt[c + 1]++;
    for (size_t i = 0; i < P.cells2.size(); ++i) cnt[i + 1] += cnt[i];
    P.tasks2.resize(B.t2.size());
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    for (size_t t = 0; t < B.t2.size(); ++t) P.tasks2[pos[B.t2cell[t]]++] = B.t2[t];
    std::vector<Cell> kept;
    for (size_t i = 0; i < P.cells2.size(); ++i) {
      if (cnt[i + 1] == cnt[i]) continue;
      Cell cl = P.cells2[i];
      cl.t_begin = cnt[i];
      cl.t_end = cnt[i + 1];
      kept.push_back(cl);
    }
    P.cells2.swap(kept);
  }
  split_tiles(P.cells1, P.tasks1, P.tiles1, P.red1, P.nslots1, false);
  split_tiles(P.cells2, P.tasks2, P.tiles2, P.red2, P.nslots2, false);
  int rc;
  if ((rc = ctx->rnTrun.reserve(sizeof(double) * (hi - lo + 4))) ||
      (rc = out.buf.reserve(sizeof(double) * (B.out_len + 4))))
    return rc;
  CKR(cudaMemcpyAsync(ctx->rnTrun.d(), trun.data + lo, sizeof(double) * (hi - lo), cudaMemcpyHostToDevice,
                      ctx->stream));
  CKR(cudaMemsetAsync(out.buf.p, 0, sizeof(double) * (B.out_len + 4), ctx->stream));
  if ((rc = exec_passes(ctx, P, in_dev, ctx->rnTrun.d(), out.buf.d()))) return rc;
  const OutBlk &ob = B.blocks[0];
  out.b.len = len;
  out.b.up_dif = ob.up_dif;
  out.b.down_dif = ob.down_dif;
  out.dim = ob.dim;
  out.b.sub.clear();
  for (int i = 0; i < ob.num; ++i) {
    const tj_block_sub &r = B.recs[ob.first + i];
    out.b.sub.push_back(RSub{r.num_up, r.num_down, r.down_dif, r.row_dim, r.sdim, r.off});
  }
  return TJ_OK;
}

// the enlargement of a device operator into a basis (update_block_dia /
// update_block_ndia_sys/env) or of a one-site operator (update_site_*)
EBlk enlarge(const tj_basis *bs, const RBlk *blk, const SiteOp *site, bool dia, int side, char types) {
  Ctx c;
  c.bs = bs;
  if (dia) return enl_dia(c, blk, site);
  return enl_ndia(c, blk, site, side == 1, types);
}

// a device operator whose pieces are its own sub-blocks (no enlargement), to be truncated
EBlk as_pieces(const DevOp &d) {
  EBlk e;
  e.len = d.b.len;
  e.up_dif = d.b.up_dif;
  e.down_dif = d.b.down_dif;
  e.set = true;
  for (const RSub &s : d.b.sub) {
    ESub q{s.num_up, s.num_down, s.down_dif, -1, -1, {}};
    q.p.push_back(Piece{0, s.row_dim, 0, s.sdim, s.off, s.row_dim, 0, 0, 1.0});
    e.sub.push_back(std::move(q));
  }
  return e;
}

SiteOp site_of(const tj_block &b) {
  SiteOp s;
  s.up_dif = b.up_dif;
  s.down_dif = b.down_dif;
  if (b.num > 0 && (!b.sub || !b.data)) throw RenormError(TJ_ERR_ARG, "site operator with null sub/data");
  for (int k = 0; k < b.num; ++k) {
    const tj_block_sub &q = b.sub[k];
    if (q.row_dim != 1 || q.sdim != 1) throw RenormError(TJ_ERR_ARG, "site operator sub-blocks must be 1x1");
    s.sub.push_back(SiteOp::S{q.num_up, q.num_down, q.down_dif, b.data[q.off]});
  }
  return s;
}

// result (two-call) of the last measurement-operator call, kept on the device
struct LastOp {
  uint64_t key = 0;
  bool valid = false;
  DevOp op;
};

int finish(tj_ctx *ctx, DevOp &d, tj_block_result *out) {
  int64_t n = 0;
  for (const RSub &s : d.b.sub) n = std::max(n, s.off + (int64_t)s.row_dim * s.sdim);
  out->num = (int32_t)d.b.sub.size();
  out->data_len = n;
  if (!out->subs || !out->data) return TJ_OK;
  for (size_t i = 0; i < d.b.sub.size(); ++i) {
    const RSub &s = d.b.sub[i];
    tj_block_sub r;
    std::memset(&r, 0, sizeof r);
    r.num_up = s.num_up;
    r.num_down = s.num_down;
    r.down_dif = s.down_dif;
    r.row_dim = s.row_dim;
    r.sdim = s.sdim;
    r.off = s.off;
    out->subs[i] = r;
  }
  if (n > 0) {
    const int rc = download(ctx, out->data, d.buf.d(), n, ctx->stream);
    if (rc) return rc;
  }
  CKR(cudaStreamSynchronize(ctx->stream));
  std::memset(&out->block, 0, sizeof out->block);
  out->block.len = d.b.len;
  out->block.num = out->num;
  out->block.dim = d.dim;
  out->block.up_dif = d.b.up_dif;
  out->block.down_dif = d.b.down_dif;
  out->block.sub = out->subs;
  out->block.data = out->data;
  return TJ_OK;
}

// The loop shared by Get_*_oper_* and Change_*_oper_* (get_sys.f90:764-1238):
// `cur` (block length idx) enlarged into bsm(idx+1) and truncated by its
// truncation, up to length idx_two - 1; then enlarged into bsm(idx_two), and
// truncated there when truns.
int carry_dev(tj_ctx *ctx, const tj_chain *ch, int side, bool dia, char types, DevOp &cur, int idx, int idx_two,
              bool truns, DevOp &res, std::string &msg) {
  DevOp tmp;
  auto chain_ok = [&](int i) { return i >= 1 && i <= ch->n; };
  while (idx + 1 <= idx_two - 1) {
    if (!chain_ok(idx + 1)) {
      msg = "chain index out of range";
      return TJ_ERR_ARG;
    }
    const tj_basis *bs = &ch->bsm[idx];
    EBlk e = enlarge(bs, &cur.b, nullptr, dia, side, types);
    ++idx;
    int rc;
    if (idx <= ch->trun_idx) {
      IdTrun id(bs);
      rc = trunc_step(ctx, e, dia, bs->len, id.blk, bs, cur.buf.d(), tmp, msg);
    } else {
      rc = trunc_step(ctx, e, dia, bs->len, ch->truns[idx - 1], bs, cur.buf.d(), tmp, msg);
    }
    if (rc) return rc;
    std::swap(cur.b, tmp.b);
    std::swap(cur.buf, tmp.buf);
    cur.dim = tmp.dim;
  }
  if (!chain_ok(idx + 1) || !chain_ok(idx_two)) {
    msg = "chain index out of range";
    return TJ_ERR_ARG;
  }
  const tj_basis *bs = &ch->bsm[idx];
  EBlk e = enlarge(bs, &cur.b, nullptr, dia, side, types);
  if (truns) return trunc_step(ctx, e, dia, bs->len, ch->truns[idx_two - 1], bs, cur.buf.d(), res, msg);
  IdTrun id(bs);
  return trunc_step(ctx, e, dia, bs->len, id.blk, bs, cur.buf.d(), res, msg);
}

uint64_t key_chain(uint64_t h, const tj_chain *ch) {
  h = fnv(h, ch, sizeof *ch);
  if (ch->bsm && ch->n > 0) h = fnv(h, ch->bsm, sizeof(tj_basis) * ch->n);
  if (ch->truns && ch->n > 0) h = fnv(h, ch->truns, sizeof(tj_block) * ch->n);
  return h;
}

}  // namespace
}  // namespace tjb

struct tj_meas_state {
  tjb::LastOp last;
};
std::shared_ptr<tj_meas_state> tjb::new_meas_state() { return std::make_shared<tj_meas_state>(); }

static int meas_call(tj_ctx *ctx, uint64_t key, tj_block_result *out,
                     const std::function<int(tjb::DevOp &, std::string &)> &compute, const char *what) {
  using namespace tjb;
  if (!ctx || !out) return set_err(TJ_ERR_ARG, std::string(what) + ": null argument");
  CKR(cudaSetDevice(ctx->device));
  if (!ctx->meas) ctx->meas = new_meas_state();
  LastOp &L = ctx->meas->last;
  if (!(L.valid && L.key == key)) {
    L.valid = false;
    std::string msg;
    int rc;
    try {
      rc = compute(L.op, msg);
    } catch (const std::exception &e) {
      rc = TJ_ERR_ARG;
      msg = e.what();
    }
    if (rc) return set_err(rc, std::string(what) + ": " + msg);
    L.key = key;
    L.valid = true;
  }
  return finish(ctx, L.op, out);
}

extern "C" int tj_get_oper(tj_ctx *ctx, int side, int dia, const tj_chain *chain, const tj_block *st_oper, int old_idx,
                           int new_idx, int truns, char types, tj_block_result *out) {
  using namespace tjb;
  if (!chain || !st_oper || (side != 0 && side != 1) || (chain->n > 0 && (!chain->bsm || !chain->truns)))
    return set_err(TJ_ERR_ARG, "tj_get_oper: bad argument");
  uint64_t h = 1469598103934665603ull;
  const int args[6] = {1, side, dia, old_idx, new_idx, truns};
  h = fnv(h, args, sizeof args);
  h = fnv(h, &types, 1);
  h = key_block(h, *st_oper);
  h = key_chain(h, chain);
  return meas_call(ctx, h, out, [&](DevOp &res, std::string &msg) -> int {
    const int i1 = std::min(old_idx, new_idx), i2 = std::max(old_idx, new_idx);
    const SiteOp site = site_of(*st_oper);
    auto chain_ok = [&](int i) { return i >= 1 && i <= chain->n; };
    DevOp cur;
    int rc;
    if (i1 <= i2 - 1) {
      if (i1 <= 1) {
        if ((rc = upload_op(ctx, *st_oper, cur))) return rc;
      } else {
        if (!chain_ok(i1)) {
          msg = "chain index out of range";
          return TJ_ERR_ARG;
        }
        const tj_basis *bs = &chain->bsm[i1 - 1];
        EBlk e = enlarge(bs, nullptr, &site, dia != 0, side, types);
        if (i1 <= chain->trun_idx) {
          IdTrun id(bs);
          rc = trunc_step(ctx, e, dia != 0, bs->len, id.blk, bs, nullptr, cur, msg);
        } else {
          rc = trunc_step(ctx, e, dia != 0, bs->len, chain->truns[i1 - 1], bs, nullptr, cur, msg);
        }
        if (rc) return rc;
      }
      return carry_dev(ctx, chain, side, dia != 0, types, cur, i1, i2, truns != 0, res, msg);
    }
    if (!chain_ok(i2) && !(i1 <= 1 && !truns)) {
      msg = "chain index out of range";
      return TJ_ERR_ARG;
    }
    if (i1 <= 1) {   // block_transfer(st_oper), then the optional truncation
      if (!truns) return upload_op(ctx, *st_oper, res);
      if ((rc = upload_op(ctx, *st_oper, cur))) return rc;
      return trunc_step(ctx, as_pieces(cur), dia != 0, cur.b.len, chain->truns[i2 - 1], &chain->bsm[i2 - 1],
                        cur.buf.d(), res, msg);
    }
    const tj_basis *bs = &chain->bsm[i2 - 1];
    EBlk e = enlarge(bs, nullptr, &site, dia != 0, side, types);
    if (truns) return trunc_step(ctx, e, dia != 0, bs->len, chain->truns[i2 - 1], bs, nullptr, res, msg);
    IdTrun id(bs);
    return trunc_step(ctx, e, dia != 0, bs->len, id.blk, bs, nullptr, res, msg);
  }, "tj_get_oper");
}

extern "C" int tj_change_oper(tj_ctx *ctx, int side, int dia, const tj_chain *chain, const tj_block *old_oper,
                              int old_idx, int new_idx, int truns, char types, tj_block_result *out) {
  using namespace tjb;
  if (!chain || !old_oper || (side != 0 && side != 1) || (chain->n > 0 && (!chain->bsm || !chain->truns)))
    return set_err(TJ_ERR_ARG, "tj_change_oper: bad argument");
  uint64_t h = 1469598103934665603ull;
  const int args[6] = {2, side, dia, old_idx, new_idx, truns};
  h = fnv(h, args, sizeof args);
  h = fnv(h, &types, 1);
  h = key_block(h, *old_oper);
  h = key_chain(h, chain);
  return meas_call(ctx, h, out, [&](DevOp &res, std::string &msg) -> int {
    const int i1 = std::min(old_idx, new_idx), i2 = std::max(old_idx, new_idx);
    int rc;
    if (i1 <= i2 - 1) {
      DevOp cur;
      if ((rc = upload_op(ctx, *old_oper, cur))) return rc;
      return carry_dev(ctx, chain, side, dia != 0, types, cur, i1, i2, truns != 0, res, msg);
    }
    return upload_op(ctx, *old_oper, res);
  }, "tj_change_oper");
}

extern "C" int tj_update_trun(tj_ctx *ctx, int dia, const tj_block *ori, const tj_block *trun, tj_block_result *out) {
  using namespace tjb;
  if (!ori || !trun) return set_err(TJ_ERR_ARG, "tj_update_trun: null argument");
  uint64_t h = 1469598103934665603ull;
  const int args[2] = {3, dia};
  h = fnv(h, args, sizeof args);
  h = key_block(key_block(h, *ori), *trun);
  return meas_call(ctx, h, out, [&](DevOp &res, std::string &msg) -> int {
    DevOp cur;
    int rc;
    if ((rc = upload_op(ctx, *ori, cur))) return rc;
    tj_basis none;   // the truncation reads trun's sectors only
    std::memset(&none, 0, sizeof none);
    return trunc_step(ctx, as_pieces(cur), dia != 0, ori->len, *trun, &none, cur.buf.d(), res, msg);
  }, "tj_update_trun");
}

extern "C" int tj_block_mul_block_ndia(tj_ctx *ctx, const tj_block *oper1, char flag1, const tj_block *oper2,
                                       char flag2, double coef, int down_dif, const tj_basis *basis,
                                       tj_block_result *out) {
  using namespace tjb;
  if (!oper1 || !oper2 || !basis || !basis->sub) return set_err(TJ_ERR_ARG, "tj_block_mul_block_ndia: null argument");
  if ((flag1 != 'N' && flag1 != 'T') || (flag2 != 'N' && flag2 != 'T'))
    return set_err(TJ_ERR_ARG, "tj_block_mul_block_ndia: flags must be 'N' or 'T'");
  uint64_t h = 1469598103934665603ull;
  const int args[2] = {4, down_dif};
  h = fnv(h, args, sizeof args);
  h = fnv(h, &flag1, 1);
  h = fnv(h, &flag2, 1);
  h = fnv(h, &coef, sizeof coef);
  h = key_block(key_block(h, *oper1), *oper2);
  h = fnv(h, basis, sizeof *basis);
  h = fnv(h, basis->sub, sizeof(tj_basis_map) * basis->num);
  return meas_call(ctx, h, out, [&](DevOp &res, std::string &msg) -> int {
    HpsiPlan P;
    RBlk a, b;
    load_block(*oper1, a, P);
    load_block(*oper2, b, P);
    int rc;
    DevOp src;
    if ((rc = src.buf.reserve(sizeof(double) * (P.ops_len + 4)))) return rc;
    for (const auto &u : P.uploads)
      if (u.n > 0)
        CKR(upload(ctx, src.buf.d() + u.dst, u.src, u.n, ctx->stream));
    auto find_bs = [&](int nu, int nd) {
      for (int x = 0; x < basis->num; ++x)
        if (basis->sub[x].new_num_up == nu && basis->sub[x].new_num_down == nd) return x;
      return -1;
    };
    const int up1 = flag1 == 'N' ? a.up_dif : -a.up_dif, up2 = flag2 == 'N' ? b.up_dif : -b.up_dif;
    const int up_dif = up1 + up2, d2 = b.down_dif;
    res.b.len = basis->len;
    res.b.up_dif = up_dif;
    res.b.down_dif = down_dif;
    res.b.sub.clear();
    res.dim = 0;
    int64_t out_len = 0;
    for (int i = 0; i < basis->num; ++i) {
      const int nu = basis->sub[i].new_num_up, nd = basis->sub[i].new_num_down, nnu = nu + up_dif;
      for (int nnd = std::abs(nd - down_dif); nnd <= nd + down_dif; nnd += 2) {
        const int x = find_bs(nnu, nnd);
        if (x < 0) continue;
        const int old_dim = basis->sub[i].dim, new_dim = basis->sub[x].dim;
        res.b.sub.push_back(RSub{nu, nd, nnd - nd, new_dim, old_dim, out_len});
        res.dim += old_dim;
        Cell cl;
        std::memset(&cl, 0, sizeof cl);
        cl.off = out_len;
        cl.ld = std::max(1, new_dim);
        cl.M = new_dim;
        cl.N = old_dim;
        cl.space = SP_PSI;
        cl.t_begin = (int32_t)P.tasks2.size();
        // the coupled product's 3j normalisation (block.f90:2138-2145), with the
        // operator's total transfer down_dif (new_oper%down_dif)
        const int kq = nnd - nd;
        const double c11 = w3j(nnd, down_dif, nd, -nnd, kq, nd);
        for (int mnd = std::abs(nd - d2); mnd <= nd + d2; mnd += 2) {
          const int m2u = flag2 == 'N' ? nu : nu + up2, m2d = flag2 == 'N' ? nd : mnd;
          const int dd22 = flag2 == 'N' ? mnd - nd : nd - mnd;
          const int m1u = flag1 == 'N' ? nu + up2 : nnu, m1d = flag1 == 'N' ? mnd : nnd;
          const int dd11 = flag1 == 'N' ? nnd - mnd : mnd - nnd;
          const int i2 = b.find(m2u, m2d, dd22, true), i1 = a.find(m1u, m1d, dd11, true);
          if (i1 < 0 || i2 < 0) continue;
          if (c11 == 0.0) {
            msg = "vanishing 3j normalisation";
            return TJ_ERR_NUMERIC;
          }
          double c1 = 0.0;
          for (int jj6 = -mnd; jj6 <= mnd; jj6 += 2) {
            const int a5 = nnd - jj6, b5 = jj6 - nd;
            double c12 = w3j(nnd, a.down_dif, mnd, -nnd, a5, jj6);
            c12 *= w3j(mnd, b.down_dif, nd, -jj6, b5, nd) * m1((mnd - jj6) / 2);
            c12 *= w3j(a.down_dif, b.down_dif, down_dif, a5, b5, -kq) * m1((-a.down_dif + b.down_dif + kq) / 2) *
                   std::sqrt(down_dif + 1.0);
            c1 += c12;
          }
          if (c1 == 0.0) continue;
          c1 = coef * c1 / c11;
          const RSub &A = a.sub[i1], &Bq = b.sub[i2];
          const int mid = flag1 == 'N' ? A.sdim : A.row_dim;
          if ((flag1 == 'N' ? A.row_dim : A.sdim) != new_dim || (flag2 == 'N' ? Bq.sdim : Bq.row_dim) != old_dim ||
              (flag2 == 'N' ? Bq.row_dim : Bq.sdim) != mid) {
            msg = "operator dimensions disagree with the basis";
            return TJ_ERR_QN;
          }
          Task t;
          std::memset(&t, 0, sizeof t);
          t.L.off = A.off;
          t.L.ld = std::max(1, A.row_dim);
          t.L.space = SP_OPS;
          t.L.trans = flag1 == 'T';
          t.R.off = Bq.off;
          t.R.ld = std::max(1, Bq.row_dim);
          t.R.space = SP_OPS;
          t.R.trans = flag2 == 'T';
          t.coef = c1;
          t.K = mid;
          P.tasks2.push_back(t);
          P.flops += 2.0 * new_dim * old_dim * (double)mid;
        }
        cl.t_end = (int32_t)P.tasks2.size();
        if (cl.t_end > cl.t_begin && new_dim > 0 && old_dim > 0) P.cells2.push_back(cl);
        out_len += (int64_t)new_dim * old_dim;
      }
    }
    split_tiles(P.cells2, P.tasks2, P.tiles2, P.red2, P.nslots2, false);
    if ((rc = res.buf.reserve(sizeof(double) * (out_len + 4)))) return rc;
    CKR(cudaMemsetAsync(res.buf.p, 0, sizeof(double) * (out_len + 4), ctx->stream));
    return exec_passes(ctx, P, src.buf.d(), nullptr, res.buf.d());
  }, "tj_block_mul_block_ndia");
}
