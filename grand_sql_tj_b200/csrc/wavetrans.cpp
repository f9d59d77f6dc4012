// Wavefunction prediction between DMRG steps on the device: wave_trans_LR /
// wave_trans_RL (code/tjsq/dmrg_sub.f90:1093-1384).
//
// When the sweep moves one site to the right, the converged psi of the last
// step, psi[(S s), (e E)], is carried to the next superblock
// psi'[(S' e), (E'' s'')]: the system block's truncation U (just computed)
// takes S s to S', and the truncation V that built the environment block E
// from E'' s'' is applied transposed; a closed-form 6j phase recouples the
// site e from the environment to the system side.  Every (old sector,
// environment sub-block, new system spin) triple is one two-GEMM chain
// coef * U^T psi_w V^T into a row window of a new sector (the mirror image
// for a move to the left).  The chains run on the grouped FP64 GEMM of H*psi
// -- the truncations in the operator space, the old psi as input, the new
// psi's windows as output cells owned by their CTAs -- and the result is
// normalised on the device.
#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "ctx.h"

using namespace tjb;

#define CKW(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace tjb {
namespace {

struct WtError : std::runtime_error {
  int code;
  WtError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

struct TSub {
  int num_up, num_down, rows, cols;
  int64_t off;   // in the operator space
};
struct TSet {
  std::vector<TSub> s;
  int find(int nu, int nd) const {
    for (size_t k = 0; k < s.size(); ++k)
      if (s[k].num_up == nu && s[k].num_down == nd) return (int)k;
    return -1;
  }
};

inline double m1(int n) { return (n % 2) ? -1.0 : 1.0; }

int find_map(const tj_basis *b, int nu, int nd) {
  for (int x = 0; x < b->num; ++x)
    if (b->sub[x].new_num_up == nu && b->sub[x].new_num_down == nd) return x;
  return -1;
}
const tj_basis_sub &BMap(const tj_basis *b, int x, int m) { return b->maps[b->sub[x].first + m]; }

int find_sector(const tj_wave *w, int su, int sd, int eu, int ed) {
  for (int k = 0; k < w->num; ++k)
    if (w->sub[k].sys_num_up == su && w->sub[k].sys_num_down == sd && w->sub[k].env_num_up == eu &&
        w->sub[k].env_num_down == ed)
      return k;
  return -1;
}

void load_trun(const tj_block *b, TSet &t, HpsiPlan &P) {
  if (!b || b->num < 1 || !b->sub || !b->data) throw WtError(TJ_ERR_ARG, "empty truncation operator");
  int64_t lo = LLONG_MAX, hi = 0;
  for (int k = 0; k < b->num; ++k) {
    const tj_block_sub &s = b->sub[k];
    if (s.row_dim < 0 || s.sdim < 0 || s.off < 0) throw WtError(TJ_ERR_ARG, "bad truncation sub-block");
    lo = std::min(lo, (int64_t)s.off);
    hi = std::max(hi, (int64_t)s.off + (int64_t)s.row_dim * s.sdim);
  }
  const int64_t base = P.ops_len;
  P.uploads.push_back({b->data + lo, hi - lo, base});
  P.ops_len += (hi - lo + 3) / 4 * 4;
  for (int k = 0; k < b->num; ++k) {
    const tj_block_sub &s = b->sub[k];
    t.s.push_back(TSub{s.num_up, s.num_down, s.row_dim, s.sdim, base + s.off - lo});
  }
}

Operand opnd(int64_t off, int ld, int8_t space, int8_t trans) {
  Operand o;
  o.off = off;
  o.ld = std::max(1, ld);
  o.space = space;
  o.trans = trans;
  o.pad = 0;
  return o;
}

struct WtBuilder {
  HpsiPlan &P;
  struct PKey {
    int64_t a, b;
    int32_t m, n, k;
    int8_t ta, tb, sa, sb;
    bool operator==(const PKey &o) const {
      return a == o.a && b == o.b && m == o.m && n == o.n && k == o.k && ta == o.ta && tb == o.tb && sa == o.sa &&
             sb == o.sb;
    }
  };
  struct PHash {
    size_t operator()(const PKey &k) const {
      uint64_t h = (uint64_t)k.a * 0x9e3779b97f4a7c15ull ^ ((uint64_t)k.b * 0xbf58476d1ce4e5b9ull);
      h ^= ((uint64_t)(uint32_t)k.m << 32 | (uint32_t)k.n) + (uint64_t)k.k * 131 + (uint64_t)(k.ta * 8 + k.tb * 4 + k.sa);
      return (size_t)h;
    }
  };
  std::unordered_map<PKey, int64_t, PHash> prod;
  std::unordered_map<int64_t, int> cell_of;   // output window offset -> cell
  std::vector<Task> t2;
  std::vector<int32_t> t2cell;
  explicit WtBuilder(HpsiPlan &p) : P(p) {}

  int64_t product(const Operand &L, const Operand &R, int M, int N, int K) {
    PKey key{L.off, R.off, M, N, K, L.trans, R.trans, L.space, R.space};
    auto it = prod.find(key);
    if (it != prod.end()) return it->second;
    const int64_t off = P.scratch_len;
    P.scratch_len += ((int64_t)M * N + 3) / 4 * 4;
    Cell c;
    std::memset(&c, 0, sizeof c);
    c.off = off;
    c.ld = std::max(1, M);
    c.M = M;
    c.N = N;
    c.t_begin = (int32_t)P.tasks1.size();
    c.t_end = c.t_begin + 1;
    c.space = SP_SCR;
    Task t;
    std::memset(&t, 0, sizeof t);
    t.L = L;
    t.R = R;
    t.coef = 1.0;
    t.K = K;
    P.tasks1.push_back(t);
    P.cells1.push_back(c);
    P.flops += 2.0 * M * N * (double)K;
    prod.emplace(key, off);
    return off;
  }
  int cell(int64_t off, int ld, int M, int N) {
    auto it = cell_of.find(off);
    if (it != cell_of.end()) {
      const Cell &c = P.cells2[it->second];
      if (c.M != M || c.N != N || c.ld != ld) throw WtError(TJ_ERR_QN, "overlapping output windows");
      return it->second;
    }
    Cell c;
    std::memset(&c, 0, sizeof c);
    c.off = off;
    c.ld = std::max(1, ld);
    c.M = M;
    c.N = N;
    c.space = SP_PSI;
    P.cells2.push_back(c);
    cell_of.emplace(off, (int)P.cells2.size() - 1);
    return (int)P.cells2.size() - 1;
  }
  // Y(cell) += coef * A * X * B, with op(A) M x K1, X K1 x K2, op(B) K2 x N
  void chain(int cl, double coef, const Operand &A, const Operand &X, const Operand &B, int M, int K1, int K2, int N) {
    if (M == 0 || N == 0 || K1 == 0 || K2 == 0) return;
    const double ca = (double)M * K1 * K2 + (double)M * K2 * N, cb = (double)K1 * K2 * N + (double)M * K1 * N;
    Task t;
    std::memset(&t, 0, sizeof t);
    t.coef = coef;
    if (ca <= cb) {   // (A X) then (.) B
      const int64_t off = product(A, X, M, K2, K1);
      t.L = opnd(off, M, SP_SCR, 0);
      t.R = B;
      t.K = K2;
    } else {          // (X B) then A (.)
      const int64_t off = product(X, B, K1, N, K2);
      t.L = A;
      t.R = opnd(off, K1, SP_SCR, 0);
      t.K = K1;
    }
    P.flops += 2.0 * M * N * (double)t.K;
    t2.push_back(t);
    t2cell.push_back(cl);
  }
};

}  // namespace

int build_wave_trans_plan(int direction, const tj_basis *sys_bs, const tj_basis *env_bs, const tj_block *sys_trun,
                          const tj_block *env_trun, const tj_wave *old, const tj_wave *nw, HpsiPlan &P,
                          std::string &msg) {
  try {
    if (direction != 0 && direction != 1) throw WtError(TJ_ERR_ARG, "direction must be 0 (left to right) or 1");
    if (!sys_bs || !env_bs || !sys_bs->sub || !env_bs->sub || !sys_bs->maps || !env_bs->maps)
      throw WtError(TJ_ERR_ARG, "null basis");
    TSet st, et;
    load_trun(sys_trun, st, P);
    load_trun(env_trun, et, P);
    WtBuilder B(P);
    for (int i = 0; i < old->num; ++i) {
      const tj_wave_sub &o = old->sub[i];
      const int snu = o.sys_num_up, snd = o.sys_num_down, enu = o.env_num_up, end = o.env_num_down;
      const int osd = o.sys_dim, oed = o.env_dim;
      if (direction == 0) {
        const int tid = st.find(snu, snd);
        if (tid < 0) continue;
        const TSub &U = st.s[tid];
        if (U.rows != osd) throw WtError(TJ_ERR_QN, "system truncation does not match the old sector");
        const int k = find_map(env_bs, enu, end);
        if (k < 0) continue;
        for (int x = 0; x < env_bs->sub[k].num; ++x) {
          const tj_basis_sub &m = BMap(env_bs, k, x);
          const int eid = et.find(m.bl_num_up, m.bl_num_down);
          for (int nsd = std::abs(snd - m.st_num_down); nsd <= snd + m.st_num_down; nsd += 2) {
            const int nsu = snu + m.st_num_up;
            const int y = find_map(sys_bs, nsu, nsd);
            const tj_basis_sub *q = nullptr;
            if (y >= 0)
              for (int z = 0; z < sys_bs->sub[y].num && !q; ++z) {
                const tj_basis_sub &t = BMap(sys_bs, y, z);
                if (t.bl_num_up == snu && t.bl_num_down == snd && t.st_num_up == m.st_num_up &&
                    t.st_num_down == m.st_num_down)
                  q = &t;
              }
            const int wid = find_sector(nw, nsu, nsd, m.bl_num_up, m.bl_num_down);
            if (eid < 0 || !q || wid < 0) continue;
            const TSub &V = et.s[eid];
            const int nedim = nw->sub[wid].env_dim, nsub = q->sdim;
            if (U.cols != nsub || V.rows != nedim || V.cols != m.sdim || q->spos + nsub > nw->sub[wid].sys_dim)
              throw WtError(TJ_ERR_QN, "truncation and basis dimensions disagree");
            const int j12 = snd, j3 = m.st_num_down, j4 = m.bl_num_down, j123 = nsd, j34 = end;
            double c1 = m1((j12 + j3 + j123) / 2) / std::sqrt((1.0 + j12) * (1.0 + j123));
            c1 *= std::sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j12 + j3 + j4) / 2) % 2 != 0) c1 = -c1;
            if (((j3 + j4 - j34) / 2) % 2 != 0) c1 = -c1;
            const int cl = B.cell(nw->sub[wid].off + q->spos, nw->sub[wid].sys_dim, nsub, nedim);
            B.chain(cl, c1, opnd(U.off, U.rows, SP_OPS, 1), opnd(o.off + (int64_t)m.spos * osd, osd, SP_PSI, 0),
                    opnd(V.off, V.rows, SP_OPS, 1), nsub, osd, m.sdim, nedim);
          }
        }
      } else {
        const int tid = et.find(enu, end);
        if (tid < 0) continue;
        const TSub &U = et.s[tid];
        if (U.rows != oed) throw WtError(TJ_ERR_QN, "environment truncation does not match the old sector");
        const int k = find_map(sys_bs, snu, snd);
        if (k < 0) continue;
        for (int x = 0; x < sys_bs->sub[k].num; ++x) {
          const tj_basis_sub &m = BMap(sys_bs, k, x);
          const int sid = st.find(m.bl_num_up, m.bl_num_down);
          for (int ned = std::abs(end - m.st_num_down); ned <= end + m.st_num_down; ned += 2) {
            const int neu = enu + m.st_num_up;
            const int y = find_map(env_bs, neu, ned);
            const tj_basis_sub *q = nullptr;
            if (y >= 0)
              for (int z = 0; z < env_bs->sub[y].num && !q; ++z) {
                const tj_basis_sub &t = BMap(env_bs, y, z);
                if (t.bl_num_up == enu && t.bl_num_down == end && t.st_num_up == m.st_num_up &&
                    t.st_num_down == m.st_num_down)
                  q = &t;
              }
            const int wid = find_sector(nw, m.bl_num_up, m.bl_num_down, neu, ned);
            if (sid < 0 || !q || wid < 0) continue;
            const TSub &W = st.s[sid];
            const int nsdim = nw->sub[wid].sys_dim, nsub = q->sdim;
            if (U.cols != nsub || W.rows != nsdim || W.cols != m.sdim || q->spos + nsub > nw->sub[wid].env_dim)
              throw WtError(TJ_ERR_QN, "truncation and basis dimensions disagree");
            const int j12 = end, j3 = m.st_num_down, j4 = m.bl_num_down, j123 = ned, j34 = snd;
            double c1 = m1((j34 + j4 + j3) / 2) / std::sqrt((1.0 + j12) * (1.0 + j4));
            c1 *= std::sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j4 + j3 + j12) / 2) % 2 != 0) c1 = -c1;
            if (((j12 + j3 - j123) / 2) % 2 != 0) c1 = -c1;
            const int cl = B.cell(nw->sub[wid].off + (int64_t)q->spos * nsdim, nsdim, nsdim, nsub);
            B.chain(cl, c1, opnd(W.off, W.rows, SP_OPS, 0), opnd(o.off + m.spos, osd, SP_PSI, 0),
                    opnd(U.off, U.rows, SP_OPS, 0), nsdim, m.sdim, oed, nsub);
          }
        }
      }
    }
    // tasks sorted by cell, emission order kept within a cell
    std::vector<int32_t> cnt(P.cells2.size() + 1, 0);
    for (int32_t c : B.t2cell) cnt[c + 1]++;
    for (size_t i = 0; i < P.cells2.size(); ++i) cnt[i + 1] += cnt[i];
    P.tasks2.resize(B.t2.size());
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    for (size_t t = 0; t < B.t2.size(); ++t) P.tasks2[pos[B.t2cell[t]]++] = B.t2[t];
    for (size_t i = 0; i < P.cells2.size(); ++i) {
      P.cells2[i].t_begin = cnt[i];
      P.cells2[i].t_end = cnt[i + 1];
    }
    P.psi_len = nw->dim;
    double bytes = 0;
    for (const auto &u : P.uploads) bytes += 8.0 * u.n;
    P.bytes = bytes + 8.0 * (old->dim + nw->dim);
    split_tiles(P.cells1, P.tasks1, P.tiles1, P.red1, P.nslots1, false);
    split_tiles(P.cells2, P.tasks2, P.tiles2, P.red2, P.nslots2, false);
    return TJ_OK;
  } catch (const WtError &e) {
    msg = e.what();
    return e.code;
  } catch (const std::exception &e) {
    msg = e.what();
    return TJ_ERR_ARG;
  }
}

}  // namespace tjb

extern "C" int tj_wave_trans(tj_ctx *ctx, int direction, const tj_basis *sys_bs, const tj_basis *env_bs,
                             const tj_block *sys_trun, const tj_block *env_trun, const tj_wave *old_wave,
                             tj_wave *new_wave) {
  using namespace tjb;
  int rc;
  if (!ctx) return set_err(TJ_ERR_ARG, "tj_wave_trans: null context");
  if ((rc = check_wave(old_wave)) || (rc = check_wave(new_wave))) return rc;
  HpsiPlan P;
  std::string msg;
  const auto t0 = std::chrono::steady_clock::now();
  if ((rc = build_wave_trans_plan(direction, sys_bs, env_bs, sys_trun, env_trun, old_wave, new_wave, P, msg)))
    return set_err(rc, "tj_wave_trans: " + msg);
  ctx->stats.wt_plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  CKW(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int64_t D = new_wave->dim;
  if ((rc = ctx->wtOps.reserve(sizeof(double) * (P.ops_len + 4))) ||
      (rc = ctx->wtOld.reserve(sizeof(double) * (old_wave->dim + 4))) ||
      (rc = ctx->wtNew.reserve(sizeof(double) * (D + 4))) ||
      (rc = ctx->wtScr.reserve(sizeof(double) * (P.scratch_len + 4))) ||
      (rc = ctx->wtSlots.reserve(sizeof(double) * (std::max(P.nslots1, P.nslots2) * BM * BN + 4))))
    return rc;
  CKW(cudaEventRecord(ctx->ev[5], st));
  for (const auto &u : P.uploads)
    if (u.n > 0) CKW(upload(ctx, ctx->wtOps.d() + u.dst, u.src, u.n, st));
  CKW(upload(ctx, ctx->wtOld.d(), old_wave->data, old_wave->dim, st));
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
  const int nblk = dot_blocks(D);
  const size_t o_part = add(nullptr, sizeof(double) * (nblk + 4));
  const size_t o_nrm = add(nullptr, 16);
  if ((rc = ctx->wtTab.reserve(tab.size() + 256))) return rc;
  CKW(cudaMemcpyAsync(ctx->wtTab.p, tab.data(), tab.size(), cudaMemcpyHostToDevice, st));
  CKW(cudaMemsetAsync(ctx->wtNew.p, 0, sizeof(double) * (D + 4), st));
  char *tb = (char *)ctx->wtTab.p;
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.ops = ctx->wtOps.d();
  g.psi = ctx->wtOld.d();
  g.scr = ctx->wtScr.d();
  g.out = ctx->wtScr.d();
  g.cells = (const Cell *)(tb + o_c1);
  g.tasks = (const Task *)(tb + o_t1);
  g.tiles = (const Tile *)(tb + o_l1);
  g.ntiles = (int)P.tiles1.size();
  g.counter = (unsigned int *)(tb + o_cnt);
  g.slots = ctx->wtSlots.d();
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r1), (int)P.red1.size(), st);
  g.out = ctx->wtNew.d();
  g.cells = (const Cell *)(tb + o_c2);
  g.tasks = (const Task *)(tb + o_t2);
  g.tiles = (const Tile *)(tb + o_l2);
  g.ntiles = (int)P.tiles2.size();
  g.counter = (unsigned int *)(tb + o_cnt) + 1;
  launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
  launch_reduce(g, (const Reduce *)(tb + o_r2), (int)P.red2.size(), st);
  // wave_normalize (block.f90:2419-2433)
  double *part = (double *)(tb + o_part), *nrm = (double *)(tb + o_nrm);
  launch_dot(ctx->wtNew.d(), ctx->wtNew.d(), D, part, nblk, st);
  launch_sum(part, nblk, nrm, 1, st);
  launch_scale_inv(ctx->wtNew.d(), nrm, D, st);
  CKW(cudaGetLastError());
  double h_nrm = 0;
  CKW(cudaMemcpyAsync(&h_nrm, nrm, sizeof(double), cudaMemcpyDeviceToHost, st));
  {
    int rc = download(ctx, new_wave->data, ctx->wtNew.d(), D, st);
    if (!rc) rc = res_keep(ctx, new_wave->data, D, ctx->wtNew.d(), st);
    if (rc) return rc;
    float ms = 0;
    if (cudaEventRecord(ctx->ev[2], st) == cudaSuccess && cudaEventSynchronize(ctx->ev[2]) == cudaSuccess &&
        cudaEventElapsedTime(&ms, ctx->ev[5], ctx->ev[2]) == cudaSuccess)
      ctx->stats.wt_ms = ms;
    cudaGetLastError();
  }
  if (!(h_nrm > 0.0) || !std::isfinite(h_nrm))
    return set_err(TJ_ERR_NUMERIC, "tj_wave_trans: the carried wavefunction is zero or not finite");
  return TJ_OK;
}

// The compiled form for checks on the CPU: space 1 = sys_trun's data span then
// env_trun's, space 2 = the old wave, output = the new wave before
// normalisation (psi_len = its dimension).
extern "C" int tj_wave_trans_plan_export(int direction, const tj_basis *sys_bs, const tj_basis *env_bs,
                                         const tj_block *sys_trun, const tj_block *env_trun,
                                         const tj_wave *old_wave, const tj_wave *new_wave, tj_plan_export *out) {
  using namespace tjb;
  int rc;
  if (!out) return set_err(TJ_ERR_ARG, "null output");
  if ((rc = check_wave(old_wave)) || (rc = check_wave(new_wave))) return rc;
  HpsiPlan P;
  std::string msg;
  if ((rc = build_wave_trans_plan(direction, sys_bs, env_bs, sys_trun, env_trun, old_wave, new_wave, P, msg)))
    return set_err(rc, "wave_trans plan: " + msg);
  return export_hpsi_plan(P, out);
}
