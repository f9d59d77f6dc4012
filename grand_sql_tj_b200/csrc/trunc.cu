// Reduced density matrices and the truncation operator on the device.
//
// Get_density_matrix_{sys,env}_new (code/tjsq/den_mat.f90:84-134) forms, per
// psi sector, rho = psi psi^T (system) or psi^T psi (environment) of the
// normalised wavefunction; Get_truncation_operator (den_mat.f90:141-383)
// diagonalises each rho (DSYEV), weighs the spectrum with the multiplet
// degeneracy 2S+1 for the entropies, sorts it, keeps kept_min..kept_max
// states by the discarded-weight rule and returns the kept eigenvectors.
//
// Here rho is one more grouped-GEMM pass (one cell per sector), the
// eigen-decomposition is a batched two-sided cyclic Jacobi (one CTA per
// sector, round-robin parallel ordering, FP64), and the selection -- a sort
// of at most a few 10^4 eigenvalues -- runs on the host in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "ctx.h"

namespace tjb {

constexpr int JAC_THREADS = 1024;
constexpr int JAC_MAX_N = 4096;

// Two-sided cyclic Jacobi on the symmetric matrix A (n x n, column-major).
// Each round applies n/2 disjoint plane rotations chosen by the circle
// method, so every pair (p, q) is visited once per sweep; a sweep that
// rotates nothing ends it.  On return the diagonal of A holds the eigenvalues
// and V the eigenvectors.  status[s] = 1 if max_sweeps were not enough.
__global__ void __launch_bounds__(JAC_THREADS) jacobi_kernel(double *Aall, double *Vall, const int64_t *off,
                                                            const int *dims, double *evals, const int64_t *eoff,
                                                            int max_sweeps, int *status) {
  extern __shared__ unsigned char sm_raw[];
  const int s = blockIdx.x, n = dims[s], tid = threadIdx.x;
  double *A = Aall + off[s], *V = Vall + off[s];
  const int m = n + (n & 1), half = m / 2;
  double *cs = (double *)sm_raw, *sn = cs + half;
  int *pp = (int *)(sn + half), *qq = pp + half;
  __shared__ int rotated;
  __shared__ double dmax_sh[JAC_THREADS / 32];
  for (int64_t i = tid; i < (int64_t)n * n; i += blockDim.x) V[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
  // sum of |diagonal| entries (the trace of a density matrix, a bound on its
  // norm): off-diagonal entries below 8 eps of it are at the rounding level of
  // the rotations themselves and are left alone (density matrices of
  // truncated states have many exactly-zero eigenvalues, whose block would
  // otherwise keep rotating on rounding noise)
  double dm = 0.0;
  for (int i = tid; i < n; i += blockDim.x) dm += fabs(A[(int64_t)i * n + i]);
  for (int k = 16; k > 0; k >>= 1) dm += __shfl_xor_sync(0xffffffffu, dm, k);
  if ((tid & 31) == 0) dmax_sh[tid >> 5] = dm;
  __syncthreads();
  double dsum = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) dsum += dmax_sh[w];
  const double floor_abs = fmax(8.0 * 2.220446049250313e-16 * dsum, 1e-300);
  int sweep = 0;
  bool converged = n <= 1;
  for (; sweep < max_sweeps && !converged; ++sweep) {
    // a sweep that needs no rotation ends the iteration: every off-diagonal
    // entry is below the FP64 rounding level of its diagonal pair,
    // |a_pq| <= 2^-53 sqrt(|a_pp a_qq|) (the classical relative threshold),
    // or below the absolute floor above
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < m - 1; ++r) {
      for (int i = tid; i < half; i += blockDim.x) {
        int p, q;
        if (i == 0) {
          p = m - 1;
          q = r;
        } else {
          p = (r + i) % (m - 1);
          q = (r - i + (m - 1)) % (m - 1);
        }
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, sv = 0.0;
        if (q < n) {
          const double apq = A[(int64_t)q * n + p];
          const double app = A[(int64_t)p * n + p], aqq = A[(int64_t)q * n + q];
          if (fabs(apq) > floor_abs && fabs(apq) > 1.1102230246251565e-16 * sqrt(fabs(app * aqq))) {
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            sv = t * c;
            rotated = 1;
          }
        } else {
          q = -1;   // pair with the padding index: no rotation
        }
        pp[i] = p;
        qq[i] = q;
        cs[i] = c;
        sn[i] = sv;
      }
      __syncthreads();
      // A <- A J (columns p, q) and V <- V J
      for (int64_t idx = tid; idx < (int64_t)half * n; idx += blockDim.x) {
        const int i = (int)(idx / n), k = (int)(idx % n);
        const int q = qq[i];
        if (q < 0 || sn[i] == 0.0) continue;
        const int p = pp[i];
        const double c = cs[i], sv = sn[i];
        double *ap = A + (int64_t)p * n, *aq = A + (int64_t)q * n;
        const double x = ap[k], y = aq[k];
        ap[k] = c * x - sv * y;
        aq[k] = sv * x + c * y;
        double *vp = V + (int64_t)p * n, *vq = V + (int64_t)q * n;
        const double vx = vp[k], vy = vq[k];
        vp[k] = c * vx - sv * vy;
        vq[k] = sv * vx + c * vy;
      }
      __syncthreads();
      // A <- J^T A (rows p, q): consecutive threads take consecutive pairs of
      // the same column, so a warp stays inside one column (8n bytes)
      for (int64_t idx = tid; idx < (int64_t)half * n; idx += blockDim.x) {
        const int i = (int)(idx % half), k = (int)(idx / half);
        const int q = qq[i];
        if (q < 0 || sn[i] == 0.0) continue;
        const int p = pp[i];
        const double c = cs[i], sv = sn[i];
        double *col = A + (int64_t)k * n;
        const double x = col[p], y = col[q];
        col[p] = c * x - sv * y;
        col[q] = sv * x + c * y;
      }
      __syncthreads();
    }
    converged = rotated == 0;
    __syncthreads();
  }
  if (tid == 0) status[s] = converged ? 0 : 1;
  for (int i = tid; i < n; i += blockDim.x) evals[eoff[s] + i] = A[(int64_t)i * n + i];
}

// out[j] gathers column src_col[j] (length rows[j]) of the matrix at src_off[j].
__global__ void gather_cols_kernel(const double *V, const int64_t *src_off, const int *rows, const int64_t *dst_off,
                                   double *out, int ncols) {
  const int j = blockIdx.x;
  if (j >= ncols) return;
  const double *s = V + src_off[j];
  double *d = out + dst_off[j];
  for (int i = threadIdx.x; i < rows[j]; i += blockDim.x) d[i] = s[i];
}

}  // namespace tjb

using namespace tjb;

#define CKT(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return set_err(TJ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

struct TruncCache {
  bool valid = false;
  const double *data = nullptr;
  int64_t dim = 0;
  int side = 0, kept_min = 0, kept_max = 0;
  double trun_err = 0;
  uint64_t hash = 0;
  tj_trunc_result res{};
  std::vector<tj_block_sub> sub;
  std::vector<double> mats;
};
thread_local TruncCache g_tc;

uint64_t hash_data(const double *p, int64_t n) {
  uint64_t h = 1469598103934665603ull;
  const uint64_t *u = (const uint64_t *)p;
  for (int64_t i = 0; i < n; ++i) {
    h ^= u[i];
    h *= 1099511628211ull;
  }
  return h;
}

}  // namespace

extern "C" int tj_truncation(tj_ctx *ctx, const tj_wave *wave, int side, int kept_min, int kept_max,
                             double trun_err, tj_trunc_result *out) {
  if (!ctx || !wave || !out) return set_err(TJ_ERR_ARG, "tj_truncation: null argument");
  if (side != 0 && side != 1) return set_err(TJ_ERR_ARG, "tj_truncation: side must be 0 (system) or 1 (environment)");
  if (wave->num < 1 || !wave->sub || !wave->data) return set_err(TJ_ERR_ARG, "tj_truncation: empty wavefunction");
  const int nsec = wave->num;
  const int64_t D = wave->dim;
  for (int i = 0; i < nsec; ++i) {
    const tj_wave_sub &w = wave->sub[i];
    if (w.sys_dim < 0 || w.env_dim < 0 || w.off < 0 || w.off + (int64_t)w.sys_dim * w.env_dim > D)
      return set_err(TJ_ERR_ARG, "tj_truncation: bad sector table");
    const int n = side == 0 ? w.sys_dim : w.env_dim;
    if (n > JAC_MAX_N) return set_err(TJ_ERR_LIMIT, "tj_truncation: a density-matrix sector exceeds 4096 states");
  }
  const uint64_t h = hash_data(wave->data, D);
  TruncCache &tc = g_tc;
  const bool hit = tc.valid && tc.data == wave->data && tc.dim == D && tc.side == side && tc.kept_min == kept_min &&
                   tc.kept_max == kept_max && tc.trun_err == trun_err && tc.hash == h;
  if (!hit) {
    CKT(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    // psi on the device and its norm
    int rc;
    if ((rc = ctx->trA.reserve(sizeof(double) * (D + 4)))) return rc;
    double *psi = ctx->trA.d();
    CKT(cudaMemcpyAsync(psi, wave->data, sizeof(double) * D, cudaMemcpyHostToDevice, st));
    double nrm2 = 0;
    for (int64_t i = 0; i < D; ++i) nrm2 += wave->data[i] * wave->data[i];
    if (!(nrm2 > 0) || !std::isfinite(nrm2)) return set_err(TJ_ERR_NUMERIC, "tj_truncation: zero or non-finite psi");
    // rho per sector as one grouped-GEMM pass
    std::vector<Cell> cells;
    std::vector<Task> tasks;
    std::vector<Tile> tiles;
    std::vector<int64_t> roff(nsec), eoff(nsec);
    std::vector<int> dims(nsec);
    int64_t rlen = 0, etot = 0;
    for (int i = 0; i < nsec; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int n = side == 0 ? w.sys_dim : w.env_dim, K = side == 0 ? w.env_dim : w.sys_dim;
      dims[i] = n;
      roff[i] = rlen;
      eoff[i] = etot;
      rlen += ((int64_t)n * n + 31) / 32 * 32;
      etot += n;
      Cell c;
      std::memset(&c, 0, sizeof c);
      c.off = roff[i];
      c.ld = n;
      c.M = n;
      c.N = n;
      c.space = SP_SCR;
      c.t_begin = (int)tasks.size();
      Task t;
      std::memset(&t, 0, sizeof t);
      t.L.off = w.off;
      t.L.ld = w.sys_dim;
      t.L.space = SP_PSI;
      t.L.trans = (int8_t)(side == 0 ? 0 : 1);
      t.R = t.L;
      t.R.trans = (int8_t)(side == 0 ? 1 : 0);
      t.coef = 1.0 / nrm2;
      t.K = K;
      if (n > 0 && K > 0) tasks.push_back(t);
      c.t_end = (int)tasks.size();
      const int ci = (int)cells.size();
      cells.push_back(c);
      for (int r0 = 0; r0 < n; r0 += BM)
        for (int c0 = 0; c0 < n; c0 += BN) tiles.push_back(Tile{ci, r0, c0, c.t_begin, c.t_end, c.t_end, c.t_end, -1});
    }
    if ((rc = ctx->trB.reserve(sizeof(double) * (rlen + 4))) || (rc = ctx->trC.reserve(sizeof(double) * (rlen + 4))) ||
        (rc = ctx->trD.reserve(sizeof(double) * (etot + 4))))
      return rc;
    // small tables packed into one buffer
    const size_t tb = cells.size() * sizeof(Cell), kb = tasks.size() * sizeof(Task), lb = tiles.size() * sizeof(Tile);
    const size_t ob = nsec * sizeof(int64_t), db = nsec * sizeof(int);
    size_t pos = 0;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t p_cells = pos; pos += al(tb);
    const size_t p_tasks = pos; pos += al(kb);
    const size_t p_tiles = pos; pos += al(lb);
    const size_t p_roff = pos; pos += al(ob);
    const size_t p_eoff = pos; pos += al(ob);
    const size_t p_dims = pos; pos += al(db);
    const size_t p_stat = pos; pos += al(db);
    const size_t p_cnt = pos; pos += 256;
    if ((rc = ctx->trE.reserve(pos))) return rc;
    char *tbase = (char *)ctx->trE.p;
    CKT(cudaMemcpyAsync(tbase + p_cells, cells.data(), tb, cudaMemcpyHostToDevice, st));
    if (kb) CKT(cudaMemcpyAsync(tbase + p_tasks, tasks.data(), kb, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_tiles, tiles.data(), lb, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_roff, roff.data(), ob, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_eoff, eoff.data(), ob, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_dims, dims.data(), db, cudaMemcpyHostToDevice, st));
    CKT(cudaMemsetAsync(tbase + p_cnt, 0, 16, st));
    GemmParams g;
    std::memset(&g, 0, sizeof g);
    g.psi = psi;
    g.scr = ctx->trB.d();
    g.out = ctx->trB.d();
    g.cells = (const Cell *)(tbase + p_cells);
    g.tasks = (const Task *)(tbase + p_tasks);
    g.tiles = (const Tile *)(tbase + p_tiles);
    g.ntiles = (int)tiles.size();
    g.counter = (unsigned int *)(tbase + p_cnt);
    launch_grouped_gemm(g, grouped_gemm_grid(g.ntiles), st);
    CKT(cudaGetLastError());
    // batched Jacobi
    int maxn = *std::max_element(dims.begin(), dims.end());
    const size_t smem = (size_t)((maxn + 1) / 2 + 1) * (2 * sizeof(double) + 2 * sizeof(int));
    jacobi_kernel<<<nsec, JAC_THREADS, smem, st>>>(ctx->trB.d(), ctx->trC.d(), (const int64_t *)(tbase + p_roff),
                                                  (const int *)(tbase + p_dims), ctx->trD.d(),
                                                  (const int64_t *)(tbase + p_eoff), 60, (int *)(tbase + p_stat));
    CKT(cudaGetLastError());
    std::vector<double> ev(etot);
    std::vector<int> status(nsec);
    CKT(cudaMemcpyAsync(ev.data(), ctx->trD.d(), sizeof(double) * etot, cudaMemcpyDeviceToHost, st));
    CKT(cudaMemcpyAsync(status.data(), tbase + p_stat, sizeof(int) * nsec, cudaMemcpyDeviceToHost, st));
    CKT(cudaStreamSynchronize(st));
    for (int i = 0; i < nsec; ++i)
      if (status[i]) return set_err(TJ_ERR_NUMERIC, "tj_truncation: Jacobi eigen-solver did not converge");

    // ---- selection (den_mat.f90:201-330) ----
    std::vector<int> qnu(nsec), qnd(nsec);
    for (int i = 0; i < nsec; ++i) {
      qnu[i] = side == 0 ? wave->sub[i].sys_num_up : wave->sub[i].env_num_up;
      qnd[i] = side == 0 ? wave->sub[i].sys_num_down : wave->sub[i].env_num_down;
    }
    // per sector, eigenvalue order (ascending, as DSYEV returns them)
    std::vector<std::vector<int>> asc(nsec);
    std::vector<double> val;
    std::vector<int> owner, mult;
    val.reserve(etot);
    for (int i = 0; i < nsec; ++i) {
      asc[i].resize(dims[i]);
      std::iota(asc[i].begin(), asc[i].end(), 0);
      const double *e = ev.data() + eoff[i];
      std::stable_sort(asc[i].begin(), asc[i].end(), [&](int a, int b) { return e[a] < e[b]; });
      for (int k = 0; k < dims[i]; ++k) {
        val.push_back(e[asc[i][k]]);
        owner.push_back(i);
        mult.push_back(qnd[i] + 1);
      }
    }
    const int total = (int)val.size();
    const double thr = (double)1.0e-15f;   // the reference compares against the literal 1.0E-15
    double tot_pm = 0;
    for (int i = 0; i < total; ++i) tot_pm += val[i] * mult[i];
    double ent1 = 0, ent2 = 0, ents = 0;
    for (int i = 0; i < total; ++i)
      if (val[i] >= thr) {
        const double v1 = val[i] / mult[i];
        ent1 -= v1 * std::log(v1) * mult[i];
      }
    for (int i = 0; i < total; ++i) {
      const double v = val[i] / tot_pm;
      if (v >= thr) ent2 -= v * std::log(v) * mult[i];
    }
    // descending order of the spectrum; ties keep the order of the sectors
    std::vector<int> ord(total);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return val[a] > val[b]; });
    double sum = 0;
    for (int i = 0; i < total; ++i) sum += val[ord[i]];
    std::vector<double> w(total);
    for (int i = 0; i < total; ++i) w[i] = val[ord[i]] / sum;
    int num_state;
    double err = 0;
    if (total <= kept_min) {
      num_state = total;
    } else {
      for (int i = kept_min; i < total; ++i) err += w[i];
      num_state = kept_min;
      while (err > trun_err && num_state < total) {
        ++num_state;
        err -= w[num_state - 1];
        if (err <= trun_err || num_state >= kept_max) break;
      }
    }
    for (int i = 0; i < total; ++i)
      if (w[i] >= thr) ents -= w[i] * std::log(w[i]);
    std::vector<int> cnt(nsec, 0);
    for (int k = 0; k < num_state; ++k) ++cnt[owner[ord[k]]];
    // kept eigenvectors: the cnt largest of each sector, in ascending order
    std::vector<int64_t> src_off, dst_off;
    std::vector<int> rows;
    tc.sub.clear();
    int64_t dpos = 0;
    for (int i = 0; i < nsec; ++i) {
      if (cnt[i] == 0) continue;
      int x = 0;   // the reference copies from the first sector with the same labels
      while (x < nsec && !(qnu[x] == qnu[i] && qnd[x] == qnd[i])) ++x;
      const int row = dims[i], col = cnt[i];
      tj_block_sub sb;
      std::memset(&sb, 0, sizeof sb);
      sb.num_up = qnu[i];
      sb.num_down = qnd[i];
      sb.down_dif = 0;
      sb.row_dim = row;
      sb.sdim = col;
      sb.off = dpos;
      tc.sub.push_back(sb);
      for (int c = 0; c < col; ++c) {
        const int k = asc[x][dims[x] - col + c];
        src_off.push_back(roff[x] + (int64_t)k * dims[x]);
        dst_off.push_back(dpos + (int64_t)c * row);
        rows.push_back(row);
      }
      dpos += (int64_t)row * col;
    }
    tc.mats.assign(dpos, 0.0);
    const int ncols = (int)rows.size();
    if (ncols > 0) {
      // gather tables and output reuse trD / trE (sized above for eigenvalues and tables)
      const size_t need = al(ncols * 8) * 2 + al(ncols * 4) + (size_t)dpos * 8 + 256;
      if ((rc = ctx->trA.reserve(std::max((size_t)(D + 4) * 8, need)))) return rc;
      char *gb = (char *)ctx->trA.p;   // psi is no longer needed
      int64_t *d_src = (int64_t *)gb, *d_dst = (int64_t *)(gb + al(ncols * 8));
      int *d_rows = (int *)(gb + 2 * al(ncols * 8));
      double *d_out = (double *)(gb + 2 * al(ncols * 8) + al(ncols * 4));
      CKT(cudaMemcpyAsync(d_src, src_off.data(), ncols * 8, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(d_dst, dst_off.data(), ncols * 8, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(d_rows, rows.data(), ncols * 4, cudaMemcpyHostToDevice, st));
      gather_cols_kernel<<<ncols, 128, 0, st>>>(ctx->trC.d(), d_src, d_rows, d_dst, d_out, ncols);
      CKT(cudaGetLastError());
      CKT(cudaMemcpyAsync(tc.mats.data(), d_out, sizeof(double) * dpos, cudaMemcpyDeviceToHost, st));
      CKT(cudaStreamSynchronize(st));
    }
    std::memset(&tc.res, 0, sizeof tc.res);
    tc.res.num_state = num_state;
    tc.res.num = (int32_t)tc.sub.size();
    tc.res.data_len = dpos;
    tc.res.trunc_err = err;
    tc.res.entropy1 = ent1;
    tc.res.entropy2 = ent2;
    tc.res.entropys = ents;
    tc.valid = true;
    tc.data = wave->data;
    tc.dim = D;
    tc.side = side;
    tc.kept_min = kept_min;
    tc.kept_max = kept_max;
    tc.trun_err = trun_err;
    tc.hash = h;
  }
  tj_block_sub *usub = out->sub;
  double *udata = out->data;
  *out = tc.res;
  out->sub = usub;
  out->data = udata;
  if (usub && udata) {
    std::memcpy(usub, tc.sub.data(), sizeof(tj_block_sub) * tc.sub.size());
    std::memcpy(udata, tc.mats.data(), sizeof(double) * tc.mats.size());
  }
  return TJ_OK;
}
