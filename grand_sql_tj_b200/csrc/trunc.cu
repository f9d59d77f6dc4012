// Reduced density matrices and the truncation operator on the device.
//
// Get_density_matrix_{sys,env}_new (code/tjsq/den_mat.f90:84-134) forms, per
// psi sector, rho = psi psi^T (system) or psi^T psi (environment) of the
// normalised wavefunction; Get_truncation_operator (den_mat.f90:141-383)
// diagonalises each rho (DSYEV), weighs the spectrum with the multiplet
// degeneracy 2S+1 for the entropies, sorts it, keeps kept_min..kept_max
// states by the discarded-weight rule and returns the kept eigenvectors.
//
// Here rho is one more grouped-GEMM pass (one cell per sector).  The
// eigen-decomposition follows the direct route of DSYEV's first stage and
// replaces its second: every sector is reduced to tridiagonal form by
// Householder reflections (one CTA per sector, or a thread-block cluster of
// 8-16 CTAs for sectors of 320 states and more), all eigenvalues come from
// Sturm-count multisection (one warp per eigenvalue), the host selects the
// kept states exactly as den_mat.f90 does, and only the kept eigenvectors
// are computed: inverse iteration on the tridiagonal matrix (one thread per
// vector), Gram-Schmidt orthonormalisation inside each kept block (one CTA,
// or a cluster for large blocks), and the back-transformation by the stored
// reflectors, written straight into the truncation operator's layout, which
// stays on the device until the second call of the two-call protocol copies
// it out.  Everything is FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "ctx.h"

namespace cg = cooperative_groups;

namespace tjb {

constexpr int EIG_THREADS = 512;
constexpr int EIG_MAX_N = 4096;
constexpr int TD_NX = (EIG_MAX_N + EIG_THREADS - 1) / EIG_THREADS;   // rows of a column per thread
constexpr double EIG_EPS = 2.220446049250313e-16;        // 2^-52
constexpr double EIG_SAFMIN = 2.2250738585072014e-308;   // smallest normal FP64
constexpr int ORTH_THREADS = 512;
constexpr int TD_BIG = 320;       // sectors of at least this many states are reduced by a whole cluster

// Sum of the warps' partial sums r[0..nw-1] by every warp: lane w takes
// r[w] and a shuffle tree adds them, in the same order in every warp (a
// serial sum would chain 32 dependent shared-memory loads and adds).
__device__ __forceinline__ double warp_sum_slots(const double *r) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double s = lane < nw ? r[lane] : 0.0;
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  return s;
}

// Sum of one value per thread over the block, in a fixed order; every thread
// receives it.  red holds 32 doubles of shared memory.
__device__ __forceinline__ double block_sum(double x, double *red) {
  for (int k = 16; k > 0; k >>= 1) x += __shfl_xor_sync(0xffffffffu, x, k);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  return warp_sum_slots(red);
}

// Householder reduction of one symmetric sector matrix A (n x n,
// column-major, both triangles) to tridiagonal form T = Q^T A Q with
// Q = H_0 H_1 ... H_{n-2}, H_k = I - tau_k v_k v_k^T acting on the indices
// k+1..n-1 and v_k(k+1) = 1 (the lower-triangle scheme of LAPACK's dsytd2).
// v_k overwrites A(k+1:n, k); d and e receive the diagonal and the
// off-diagonal of T, info[4s..4s+3] its Gershgorin interval, max row sum and
// the Sturm-count pivot floor.  The rank-2 update of step k,
// A <- A - v w^T - w v^T, is applied lazily inside the matrix-vector product
// p = A v of step k+1, so each step reads and writes the trailing block once.
// One CTA per sector (tridiag_one) or one cluster per large sector
// (tridiag_coop).
__device__ __forceinline__ void tridiag_info(int s, int n, const double *d, const double *e, double *info) {
  double gl = 1e308, gu = -1e308, emax2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double el = i > 0 ? fabs(e[i - 1]) : 0.0, er = i + 1 < n ? fabs(e[i]) : 0.0;
    gl = fmin(gl, d[i] - el - er);
    gu = fmax(gu, d[i] + el + er);
    if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
  }
  info[4 * s + 0] = gl;
  info[4 * s + 1] = gu;
  info[4 * s + 2] = fmax(fabs(gl), fabs(gu));
  info[4 * s + 3] = EIG_SAFMIN * fmax(1.0, emax2);
}

__device__ void tridiag_one(int s, double *Aall, const int64_t *off, const int *dims, const int64_t *eoff,
                            double *dall, double *eall, double *tauall, double *info, double *sm, double *red,
                            double &sh_tau, double &sh_scl) {
  const int n = dims[s], tid = threadIdx.x, nt = blockDim.x;
  double *A = Aall + off[s];
  double *d = dall + eoff[s], *e = eall + eoff[s], *tau = tauall + eoff[s];
  double *vp = sm, *wp = vp + n, *v = wp + n, *part = v + n;   // part: max(n, nt) entries
  if (n == 0) return;
  bool pending = false;
  for (int k = 0; k + 1 < n; ++k) {
    const int k1 = k + 1, m = n - k1;
    double *colk = A + (int64_t)k * n;
    // column k (rows k..n-1) with the pending update applied
    double ss = 0.0;
    for (int i = k + tid; i < n; i += nt) {
      double a = colk[i];
      if (pending) a -= vp[i] * wp[k] + wp[i] * vp[k];
      v[i] = a;
      if (i > k1) ss += a * a;
    }
    const double sigma2 = block_sum(ss, red);
    if (tid == 0) {
      d[k] = v[k];
      const double alpha = v[k1];
      double beta = alpha, t = 0.0, scl = 0.0;
      if (sigma2 > 0.0) {
        const double nr = sqrt(alpha * alpha + sigma2);
        beta = alpha >= 0.0 ? -nr : nr;
        t = (beta - alpha) / beta;
        scl = 1.0 / (alpha - beta);
      }
      e[k] = beta;
      tau[k] = t;
      sh_tau = t;
      sh_scl = scl;
    }
    __syncthreads();
    const double t = sh_tau, scl = sh_scl;
    for (int i = k1 + tid; i < n; i += nt) {
      const double x = i == k1 ? 1.0 : v[i] * scl;
      v[i] = x;
      colk[i] = x;
    }
    __syncthreads();
    // trailing block: apply the pending rank-2 update, p = A v
    const int R = min((m + 31) & ~31, nt), G = nt / R;
    const int g = tid / R, r = tid - g * R;
    if (g < G) {
      for (int ii = r; ii < m; ii += R) {
        const int i = k1 + ii;
        const double vpi = pending ? vp[i] : 0.0, wpi = pending ? wp[i] : 0.0;
        double acc = 0.0;
        double *a = A + (int64_t)(k1 + g) * n + i;
        const int64_t st = (int64_t)G * n;
        if (pending) {
          // eight loads issued before the eight stores: a store through a
          // may alias the next load, so loads and stores interleaved one
          // column at a time would wait out a full L2 round trip per column
          int jj = g;
          for (; jj + 7 * G < m; jj += 8 * G, a += 8 * st) {
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) x[u] = a[u * st];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int j = k1 + jj + u * G;
              x[u] -= vpi * wp[j] + wpi * vp[j];
              a[u * st] = x[u];
              acc += x[u] * v[j];
            }
          }
          for (; jj < m; jj += G, a += st) {
            const int j = k1 + jj;
            const double x = *a - (vpi * wp[j] + wpi * vp[j]);
            *a = x;
            acc += x * v[j];
          }
        } else {
#pragma unroll 4
          for (int jj = g; jj < m; jj += G, a += (int64_t)G * n) acc += *a * v[k1 + jj];
        }
        part[g * m + ii] = acc;
      }
    }
    __syncthreads();
    // p = tau A v, w = p - (tau/2)(p.v) v
    double pv = 0.0;
    for (int ii = tid; ii < m; ii += nt) {
      double p = 0.0;
      for (int q = 0; q < G; ++q) p += part[q * m + ii];
      p *= t;
      part[ii] = p;   // own entry only: q = 0 slot of the same ii
      pv += p * v[k1 + ii];
    }
    const double K = 0.5 * t * block_sum(pv, red);
    for (int ii = tid; ii < m; ii += nt) {
      const int i = k1 + ii;
      wp[i] = part[ii] - K * v[i];
      vp[i] = v[i];
    }
    pending = true;
    __syncthreads();
  }
  if (tid == 0) {
    d[n - 1] = A[(int64_t)(n - 1) * n + (n - 1)];
    if (n >= 1) tau[n - 1] = 0.0;
    tridiag_info(s, n, d, e, info);
  }
}

// Sum of one value per thread over the block with one barrier: each warp's
// sum goes to its slot of red[2][32] (the half selected by the caller's
// alternating flag, so that the next sum does not overwrite a half still
// being read) and every thread adds the slots in the same order.
__device__ __forceinline__ double block_sum1(double x, double *red, int &half) {
  for (int k = 16; k > 0; k >>= 1) x += __shfl_xor_sync(0xffffffffu, x, k);
  double *r = red + 32 * half;
  half ^= 1;
  if ((threadIdx.x & 31) == 0) r[threadIdx.x >> 5] = x;
  __syncthreads();
  return warp_sum_slots(r);
}

// The same reduction of one large sector by the CL CTAs of a thread-block
// cluster.  Every CTA forms column k itself (the pending update applied; the
// same arithmetic in the same order, so the same reflector everywhere, and
// every thread derives beta, tau and the scale from the same sum); CTA c
// owns the trailing columns j = c (mod CL), applies the pending rank-2 update
// to them and forms its part of p = A v, one thread per row, or, when the
// CTA's threads outnumber the rows, one per row in each of G groups that
// split the owned columns (the reflector is scaled where it is read).  The
// parts meet through distributed shared memory as a reduce-scatter and a
// broadcast, both by remote stores: each CTA stores the parts of rows
// [o ch, (o + 1) ch) into CTA o's shared memory; after the first cluster
// barrier CTA o sums them in rank order and stores the sums into every
// CTA's p; after the second, every CTA reads its own copy.  Per step: two
// cluster barriers (the first also orders the owners' column writes in
// global memory before they are read) and three CTA barriers (four with
// column groups).  Column k + 1, complete at the first barrier, is loaded
// into registers there for the next step.  The owner of column k stores its
// reflector there only after the first barrier, when no CTA reads the column
// any more.
template <int CL>
__device__ void tridiag_coop(cg::cluster_group &cl, int rank, int s, double *Aall, const int64_t *off,
                             const int *dims, const int64_t *eoff, double *dall, double *eall, double *tauall,
                             double *info, double *sm, int64_t smem_doubles, double *red2, double *pvs) {
  const int n = dims[s], tid = threadIdx.x, nt = blockDim.x;
  double *A = Aall + off[s];
  double *d = dall + eoff[s], *e = eall + eoff[s], *tau = tauall + eoff[s];
  // vp, wp, v: n each; cp: the bin of parts of A v sent to this CTA (CL x
  // ceil(m / CL) <= 2n); pp: p = tau A v, n
  // gp: the column groups' parts of A v when a CTA's threads outnumber the
  // trailing rows (G groups, G * m <= nt entries); sl: the CTA's slice of the
  // trailing block, the rest of the shared memory
  double *vp = sm, *wp = vp + n, *v = wp + n, *cp = v + n, *pp = cp + 2 * n, *gp = pp + n, *sl = gp + nt;
  // From step kres on, when the trailing block has mres = n - 1 - kres rows,
  // each CTA's owned columns (ceil(mres / CL) of them at most) live in its
  // slice: owned column j >= jr0(c), row i >= kres + 1 at
  // sl[(j - jr0(c)) / CL * mres + i - kres - 1].  Step kres reads them from
  // global memory and writes them there; later steps touch only the slice,
  // and the other CTAs read the next column from its owner's slice.
  const int64_t cap = smem_doubles - (6 * (int64_t)n + nt);
  int mres = 0;
  if (cap > 0) {
    mres = min(n - 1, (int)sqrt((double)cap * CL));
    while (mres > 0 && (int64_t)((mres + CL - 1) / CL) * mres > cap) --mres;
  }
  const int kres = n - 1 - mres, kr1 = kres + 1;
  auto jr0 = [&](int c) { return kr1 + ((c - kr1) % CL + CL) % CL; };
  const int myr0 = jr0(rank);
  int half = 0;
  bool pending = false;
  // rows k + tid + c nt of column k, loaded during step k - 1 (n <= TD_NX nt)
  double nx[TD_NX];
  for (int k = 0; k + 1 < n; ++k) {
    const int k1 = k + 1, m = n - k1;
    const bool owner = (k % CL) == rank;
    double *colk = A + (int64_t)k * n;
    double ss = 0.0;
#pragma unroll
    for (int c = 0; c < TD_NX; ++c) {
      const int i = k + tid + c * nt;
      if (i < n) {
        double a = k == 0 ? colk[i] : nx[c];
        if (pending) a -= vp[i] * wp[k] + wp[i] * vp[k];
        v[i] = a;
        if (i > k1) ss += a * a;
      }
    }
    const double sigma2 = block_sum1(ss, red2, half);   // also the barrier after v
    const double alpha = v[k1];
    double beta = alpha, t = 0.0, scl = 0.0;
    if (sigma2 > 0.0) {
      const double nr = sqrt(alpha * alpha + sigma2);
      beta = alpha >= 0.0 ? -nr : nr;
      t = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
    if (owner && tid == 0) {
      d[k] = v[k];
      e[k] = beta;
      tau[k] = t;
    }
    // the scaled reflector: 1 at k1, v[i] * scl below
    auto rv = [&](int i) { return i == k1 ? 1.0 : v[i] * scl; };
    // owned trailing columns j0, j0 + CL, ... (mloc of them): rows r, r + R,
    // ... by the R threads of each of G column groups, group g taking the
    // owned columns q = g, g + G, ...
    const int j0 = k1 + ((rank - k1) % CL + CL) % CL;
    const int mloc = j0 < n ? (n - 1 - j0) / CL + 1 : 0;
    const int R = min((m + 31) & ~31, nt), G = nt / R;
    const int g = tid / R, r = tid - g * R;
    // the parts of A v go to the CTA that sums their rows: rows [o ch, (o + 1)
    // ch) to CTA o, whose bin holds CL rows of ch slots (by sender)
    const int ch = (m + CL - 1) / CL;
    auto push = [&](int ii, double val) {
      const int o = ii / ch;
      cl.map_shared_rank(cp, o)[rank * ch + (ii - o * ch)] = val;
    };
    const bool s_in = k > kres, s_out = k >= kres;   // the owned columns are read / written in the slice
    if (g < G) {
      const int64_t gst = (int64_t)G * CL * n, sst = (int64_t)G * mres;
      const int64_t ist = s_in ? sst : gst, ost = s_out ? sst : gst;
      const int jg = j0 + g * CL;   // the group's first column
      const int64_t sbase = (int64_t)((jg - myr0) / CL) * mres - kr1;
      for (int ii = r; ii < m; ii += R) {
        const int i = k1 + ii;
        const double vpi = pending ? vp[i] : 0.0, wpi = pending ? wp[i] : 0.0;
        double acc = 0.0;
        const double *ia = s_in ? sl + sbase + i : A + (int64_t)jg * n + i;
        double *oa = s_out ? sl + sbase + i : A + (int64_t)jg * n + i;
        int q = g;
        if (pending || s_out != s_in) {
          // eight loads issued before the eight stores (a store through a
          // may alias the next load: interleaved, every column would wait
          // out a full L2 round trip)
          for (; q + 7 * G < mloc; q += 8 * G, ia += 8 * ist, oa += 8 * ost) {
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) x[u] = ia[u * ist];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int j = j0 + (q + u * G) * CL;
              if (pending) x[u] -= vpi * wp[j] + wpi * vp[j];
              oa[u * ost] = x[u];
              acc += x[u] * rv(j);
            }
          }
          for (; q < mloc; q += G, ia += ist, oa += ost) {
            const int j = j0 + q * CL;
            double x = *ia;
            if (pending) x -= vpi * wp[j] + wpi * vp[j];
            *oa = x;
            acc += x * rv(j);
          }
        } else {
          for (; q < mloc; q += G, ia += ist) acc += *ia * rv(j0 + q * CL);
        }
        if (G == 1)
          push(ii, acc);
        else
          gp[g * m + ii] = acc;
      }
    }
    if (G > 1) {
      __syncthreads();
      for (int ii = tid; ii < m; ii += nt) {
        double acc = 0.0;
        for (int c = 0; c < G; ++c) acc += gp[c * m + ii];
        push(ii, acc);
      }
    }
    // the cluster barrier's release / acquire order the column writes
    // (global memory) and the parts (shared memory) for the other CTAs
    cl.sync();
    // column k + 1 is complete now (its owner stored it before the barrier):
    // its loads for the next step overlap the sums below
    if (k + 2 < n) {
      const double *c1 = A + (int64_t)k1 * n;
      if (s_out) {   // in the slice of its owner
        const int ow = k1 % CL;
        c1 = cl.map_shared_rank(sl, ow) + (int64_t)((k1 - jr0(ow)) / CL) * mres - kr1;
      }
#pragma unroll
      for (int c = 0; c < TD_NX; ++c) {
        const int i = k1 + tid + c * nt;
        nx[c] = i < n ? c1[i] : 0.0;
      }
    }
    if (owner)
      for (int i = k1 + tid; i < n; i += nt) colk[i] = rv(i);
    // CTA c sums the parts of its rows from its bin (in sender order), and
    // stores the sums into every CTA's pp and its part of p.v into every
    // CTA's pvs[c]; after the second barrier each CTA reads only its own
    // shared memory.  Every exchange is a store to another CTA's shared
    // memory: a store does not wait for its reply as a remote load does.
    // A bin is written again in the next step's product, after its owner
    // has passed the second barrier; pp and pvs after the next step's first
    // barrier, which every reader passes after its reads.
    const int lo = min(m, rank * ch), hi = min(m, lo + ch);
    double pv = 0.0;
    for (int ii = lo + tid; ii < hi; ii += nt) {
      double p = 0.0;
#pragma unroll
      for (int c = 0; c < CL; ++c) p += cp[c * ch + (ii - lo)];
      p *= t;
      pv += p * rv(k1 + ii);
#pragma unroll
      for (int c = 0; c < CL; ++c) cl.map_shared_rank(pp, c)[ii] = p;
    }
    pv = block_sum1(pv, red2, half);
    if (tid < CL) cl.map_shared_rank(pvs, tid)[rank] = pv;
    cl.sync();
    double K = 0.0;
#pragma unroll
    for (int c = 0; c < CL; ++c) K += pvs[c];
    K *= 0.5 * t;
    for (int ii = tid; ii < m; ii += nt) {
      const int i = k1 + ii;
      const double vi = rv(i);
      wp[i] = pp[ii] - K * vi;
      vp[i] = vi;
    }
    pending = true;
    __syncthreads();
  }
  // the last diagonal entry, from its owner's slice when the last step
  // wrote it there
  const bool last_in_slice = n - 2 >= kres;
  if (last_in_slice && rank == (n - 1) % CL && tid == 0)
    d[n - 1] = sl[(int64_t)((n - 1 - myr0) / CL) * mres + (n - 1 - kr1)];
  __threadfence();
  cl.sync();   // the last parts are read; every owner's writes are visible
  if (rank == 0 && tid == 0) {
    if (!last_in_slice) d[n - 1] = A[(int64_t)(n - 1) * n + (n - 1)];
    tau[n - 1] = 0.0;
    tridiag_info(s, n, d, e, info);
  }
}

// One cluster of CL CTAs per entry of the cluster list: a large sector
// shared by all of them (tbig), or up to CL small sectors, one per CTA
// (tsec[cluster * CL + rank], -1 for none).  Sectors largest first.  CL is
// 16 where the GPU can schedule clusters of 16 such CTAs (a non-portable
// size), else 8.
template <int CL>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(EIG_THREADS)
    tridiag_kernel(double *Aall, const int64_t *off, const int *dims, const int64_t *eoff, const int *tsec,
                   const int *tbig, double *dall, double *eall, double *tauall, double *info, int64_t smem_doubles) {
  extern __shared__ double sm[];
  __shared__ double red[64];
  __shared__ double sh_tau, sh_scl, sh_pvs[16];
  cg::cluster_group cl = cg::this_cluster();
  const int b = blockIdx.x / CL, rank = (int)cl.block_rank();
  const int s = tsec[blockIdx.x];
  if (tbig[b]) {
    tridiag_coop<CL>(cl, rank, s, Aall, off, dims, eoff, dall, eall, tauall, info, sm, smem_doubles, red, sh_pvs);
  } else if (s >= 0 && dims[s] > 0) {
    tridiag_one(s, Aall, off, dims, eoff, dall, eall, tauall, info, sm, red, sh_tau, sh_scl);
  }
}

// Number of eigenvalues of T below x: the negative LDL^T pivots of T - x I
// (pivots below pivmin in size are replaced by -pivmin, as LAPACK's dstebz
// does).
__device__ __forceinline__ int sturm1(const double *d, const double *e, int n, double pivmin, double x) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - e[i - 1] * e[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

// Eigenvalue k (ascending) of every sector, one warp each: the interval
// [lo, hi) with count(lo) <= k < count(hi) starts at the Gershgorin bounds;
// per pass lane l counts the eigenvalues below lo + (l + 1) (hi - lo) / 33,
// and the interval becomes the 33rd between the last point at or below k
// and the first above it, until it is below 2 eps max(|lo|, |hi|) or
// eps ||T|| (the absolute accuracy of any backward-stable solver): about 11
// passes of one Sturm sequence per lane where bisection takes 52.
__global__ void bisect_kernel(const double *dall, const double *eall, const int64_t *eoff, const int *dims,
                              const double *info, const int *esec, int etot, double *evals) {
  const int idx = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (idx >= etot) return;   // uniform in a warp
  const int s = esec[idx], n = dims[s];
  const int k = (int)(idx - eoff[s]);
  const double *d = dall + eoff[s], *e = eall + eoff[s];
  const double tnorm = info[4 * s + 2], pivmin = info[4 * s + 3];
  const double pad = 2.0 * EIG_EPS * tnorm + 2.0 * pivmin;
  double lo = info[4 * s + 0] - pad, hi = info[4 * s + 1] + pad;
  for (int it = 0; it < 40; ++it) {
    const double tol = fmax(fmax(2.0 * EIG_EPS * fmax(fabs(lo), fabs(hi)), EIG_EPS * tnorm), pivmin);
    if (hi - lo <= tol) break;
    const double h = (hi - lo) / 33.0;
    const int c = sturm1(d, e, n, pivmin, lo + (lane + 1) * h);
    const unsigned above = __ballot_sync(0xffffffffu, c > k);
    const int f = above ? __ffs(above) - 1 : 32;   // first point above eigenvalue k
    const double nlo = f == 0 ? lo : lo + f * h, nhi = f == 32 ? hi : lo + (f + 1) * h;
    if (nlo == lo && nhi == hi) break;   // the interval no longer shrinks in FP64
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) evals[idx] = 0.5 * (lo + hi);
}

// Pseudo-random start vector entry in [-1, 1) (splitmix64 of the indices).
__device__ __forceinline__ double start_entry(int s, int k, int i) {
  uint64_t z = ((uint64_t)(uint32_t)s << 40) ^ ((uint64_t)(uint32_t)k << 20) ^ (uint64_t)(uint32_t)i;
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Eigenvector of T (sector job_sec[j]) for its eigenvalue job_k[j] by
// inverse iteration, one thread per vector: LU factorisation of T - lam I
// with partial pivoting (pivots below eps ||T|| raised to it, so that the
// nearly singular factor stays finite), three solves from a fixed
// pseudo-random start, each result rescaled.  The per-thread factors live in
// work[] with element i of job j at i * njobs + j (coalesced across a warp);
// the unit vector goes to Y[j * ldy + i].  status[0] bit 0: a non-finite
// value; the first such vector is described at status + 4 (six doubles).
__global__ void inverse_iter_kernel(const double *dall, const double *eall, const int64_t *eoff, const int *dims,
                                    const double *info, const double *evals, const int *job_sec, const int *job_k,
                                    int njobs, int nmax, double *work, unsigned char *piv, double *Y, int ldy,
                                    int *status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  const int s = job_sec[j], k = job_k[j], n = dims[s];
  const double *__restrict__ d = dall + eoff[s];
  const double *__restrict__ e = eall + eoff[s];
  const double lam = evals[eoff[s] + k];
  const double pert = fmax(EIG_EPS * info[4 * s + 2], 1e-290);
  const size_t st = (size_t)njobs, pl = (size_t)nmax * st;
  // disjoint regions: the loads of the factors may run ahead of the stores to X
  double *__restrict__ U = work;
  double *__restrict__ DU = work + pl;
  double *__restrict__ DU2 = work + 2 * pl;
  double *__restrict__ DL = work + 3 * pl;
  double *__restrict__ X = work + 4 * pl;
#define AT(arr, i) arr[(size_t)(i) * st + j]
  // LU = P (T - lam I): row i of U is (U_i, DU_i, DU2_i) at columns i, i+1, i+2
  double di = d[0] - lam, dui = n > 1 ? e[0] : 0.0;
  for (int i = 0; i + 1 < n; ++i) {
    const double sub = e[i];
    double dn = d[i + 1] - lam, dun = i + 2 < n ? e[i + 1] : 0.0;
    if (fabs(di) >= fabs(sub) || fabs(sub) < pert) {
      const double u = fabs(di) < pert ? copysign(pert, di) : di;
      const double l = sub / u;
      AT(U, i) = u;
      AT(DU, i) = dui;
      AT(DU2, i) = 0.0;
      AT(DL, i) = l;
      piv[(size_t)i * st + j] = 0;
      dn -= l * dui;
    } else {   // rows i and i+1 exchanged
      const double l = di / sub;
      AT(U, i) = sub;
      AT(DU, i) = dn;
      AT(DU2, i) = dun;
      AT(DL, i) = l;
      piv[(size_t)i * st + j] = 1;
      dn = dui - l * dn;
      dun = -l * dun;
    }
    di = dn;
    dui = dun;
  }
  AT(U, n - 1) = fabs(di) < pert ? copysign(pert, di) : di;
  AT(DU, n - 1) = 0.0;   // read (times zero) by the first back-substitution row
  AT(DU2, n - 1) = 0.0;
  if (n >= 2) AT(DU2, n - 2) = 0.0;
  for (int i = 0; i < n; ++i) AT(X, i) = start_entry(s, k, i);
  // Each sweep solves with X times `scale` (the previous sweep's rescale to
  // a largest entry of 1, applied where X is read) and keeps the largest
  // entry of its result as it goes.  Both passes read eight rows ahead of
  // their stores: X[i] is stored through the same pointer as the next row's
  // load, and a load the compiler must keep behind that store would wait out
  // an L2 round trip per row.
  bool bad = false;
  double scale = 1.0;
  for (int sweep = 0; sweep < 3; ++sweep) {
    // forward: P and L
    double cur = AT(X, 0) * scale;
    int i = 0;
    for (; i + 8 < n; i += 8) {   // rows i..i+7; their solves read X[i+1..i+8] as they were
      double l[8], nx[8];
      unsigned char pv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        l[u] = AT(DL, i + u);
        nx[u] = AT(X, i + u + 1) * scale;
        pv[u] = piv[(size_t)(i + u) * st + j];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (pv[u]) {   // rows i+u and i+u+1 exchanged
          AT(X, i + u) = nx[u];
          cur = cur - l[u] * nx[u];
        } else {
          AT(X, i + u) = cur;
          cur = nx[u] - l[u] * cur;
        }
      }
    }
    for (; i + 1 < n; ++i) {
      const double l = AT(DL, i), nxt = AT(X, i + 1) * scale;
      if (piv[(size_t)i * st + j]) {
        AT(X, i) = nxt;
        cur = cur - l * nxt;
      } else {
        AT(X, i) = cur;
        cur = nxt - l * cur;
      }
    }
    AT(X, n - 1) = cur;
    // backward: U, with a rescale of the whole vector if it nears overflow
    // (the rows loaded but not yet solved are rescaled in registers)
    double x1 = 0.0, x2 = 0.0, mx = 0.0;   // x_{i+1}, x_{i+2}, the largest |x| so far
    auto row = [&](double xv, double du, double du2, double uu, int at, double *ahead, int nahead) {
      double xi = (xv - du * x1 - du2 * x2) / uu;
      if (fabs(xi) > 1e250) {
        const double f = 1e-250;
        for (int q = 0; q < n; ++q) AT(X, q) *= f;
        for (int w = 0; w < nahead; ++w) ahead[w] *= f;
        xi *= f;
        x1 *= f;
        x2 *= f;
        mx *= f;
      }
      AT(X, at) = xi;
      mx = fmax(mx, fabs(xi));
      x2 = x1;
      x1 = xi;
    };
    i = n - 1;
    for (; i >= 7; i -= 8) {   // rows i, i-1, ..., i-7
      double xv[8], du[8], du2[8], uu[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        xv[u] = AT(X, i - u);
        du[u] = AT(DU, i - u);
        du2[u] = AT(DU2, i - u);
        uu[u] = AT(U, i - u);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) row(xv[u], du[u], du2[u], uu[u], i - u, xv + u + 1, 7 - u);
    }
    for (; i >= 0; --i) row(AT(X, i), AT(DU, i), AT(DU2, i), AT(U, i), i, nullptr, 0);
    if (!(mx > 0.0) || !isfinite(mx)) {
      bad = true;
      break;
    }
    scale = 1.0 / mx;
  }
  double nrm = 0.0;
  for (int i = 0; i < n; ++i) {
    const double x = AT(X, i) * scale;
    nrm += x * x;
  }
  if (bad || !(nrm > 0.0) || !isfinite(nrm)) {
    atomicOr(status, 1);
    // the first failing vector: sector, eigenvalue index, lam, pivot floor, n
    if (atomicCAS(status + 1, 0, j + 1) == 0) {
      double *diag = (double *)(status + 4);
      diag[0] = s;
      diag[1] = k;
      diag[2] = lam;
      diag[3] = pert;
      diag[4] = n;
      diag[5] = nrm;
    }
    nrm = 1.0;
    scale = 1.0;
  }
  const double inv = 1.0 / sqrt(nrm);
  double *y = Y + (size_t)j * ldy;
  for (int i = 0; i < n; ++i) y[i] = AT(X, i) * scale * inv;
  for (int i = n; i < nmax; ++i) y[i] = 0.0;
#undef AT
}

// Dots of y (rows 0..nr-1; shared or global memory) with the vectors zq(q),
// q = 0..nq-1, into out[q]: each warp takes eight vectors at a time so that
// their loads are in flight together (one vector at a time, every vector
// would wait out an L2 round trip: the store of a sum may alias the next
// vector's loads).  Each dot is summed as lane-strided parts and a shuffle
// tree, the same for every q.
template <class ZQ>
__device__ __forceinline__ void warp_dots8(ZQ zq, int nq, const double *y, int nr, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q0 = 8 * warp; q0 < nq; q0 += 8 * nw) {
    double acc[8];
    const double *z[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      acc[u] = 0.0;
      z[u] = zq(min(q0 + u, nq - 1));   // past nq: a repeat, discarded
    }
    for (int i = lane; i < nr; i += 32) {
      const double yi = y[i];
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] += z[u][i] * yi;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      double a = acc[u];
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0 && q0 + u < nq) out[q0 + u] = a;
    }
  }
}

// y <- y - sum_q h[q] zq(q) over rows 0..nr-1, returning the thread's part
// of the new squared norm.  When the block's threads outnumber the rows, G
// groups of R threads split the vectors (group g takes q = g, g + G, ...) and
// their parts (gp: G * nr <= blockDim.x entries) are summed in group order;
// otherwise one thread per row runs over all of them.  Ends with the block's
// writes to y complete only for the writing thread (the caller's barrier
// follows).
template <class ZQ>
__device__ __forceinline__ double project_off(ZQ zq, int t, const double *h, double *y, int nr, double *gp) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int R = min(max((nr + 31) & ~31, 32), nt), G = nt / R;
  double ss = 0.0;
  if (G == 1) {
    for (int i = tid; i < nr; i += nt) {
      double acc = y[i];
      for (int q = 0; q < t; ++q) acc -= h[q] * zq(q)[i];
      y[i] = acc;
      ss += acc * acc;
    }
    return ss;
  }
  const int g = tid / R, r = tid - g * R;
  if (g < G && r < nr) {
    double acc = 0.0;
#pragma unroll 4
    for (int q = g; q < t; q += G) acc += h[q] * zq(q)[r];
    gp[g * nr + r] = acc;
  }
  __syncthreads();
  for (int i = tid; i < nr; i += nt) {
    double acc = 0.0;
    for (int c = 0; c < G; ++c) acc += gp[c * nr + i];
    const double yv = y[i] - acc;
    y[i] = yv;
    ss += yv * yv;
  }
  return ss;
}

// One kept block (grp = {sector, first job, count}): classical Gram-Schmidt
// on its vectors in descending eigenvalue order, so that the dominant states
// are the least changed; inverse iteration leaves vectors of close
// eigenvalues only approximately orthogonal (to about eps ||T|| / gap).  The
// projection is repeated only when the first one removed more than half of
// the vector's squared norm ("twice is enough": after one pass that keeps
// the norm above 1/sqrt(2), the vector is orthogonal to working accuracy).
//
// A vector that loses more than 0.999 of its norm to the projection depends
// on the accepted ones.  That happens for a cluster of eigenvalues closer
// than the pivot floor eps ||T||, where inverse iteration amplifies one
// direction of the cluster far above the others -- in practice the null
// space of a rank-deficient density matrix (a sector with fewer environment
// than system states, or one of tiny weight), all of whose states the keep
// rule may keep.  When the vector's eigenvalue lies within 1e4 eps ||T|| of
// the sector's smallest, the cluster is the bottom of the spectrum, every
// eigenvector above it has been accepted (kept vectors are the largest of
// their sector), and the complement of the accepted vectors is the rest of
// the cluster: a pseudo-random vector projected off the accepted ones is then
// an eigenvector to working accuracy (residual <= the cluster's width), as
// good as any basis DSYEV returns for it.  Up to four such vectors are tried.
// status bit 1: a vector stayed dependent (or its cluster is not at the
// bottom of the spectrum).
__device__ void ortho_one(int blk, const int *grp, const int *dims, const int64_t *eoff, const double *evals,
                          const double *info, const int *job_k, double *Y, int ldy, int *status, double *h,
                          double *red) {
  const int s = grp[4 * blk], j0 = grp[4 * blk + 1], cnt = grp[4 * blk + 2];
  const int n = dims[s], tid = threadIdx.x;
  const double lam_min = evals[eoff[s]], cluster = 1e4 * EIG_EPS * info[4 * s + 2];
  double *gp = h + cnt;   // project_off's group parts
  auto vec = [&](int q) -> const double * { return Y + (size_t)(j0 + cnt - 1 - q) * ldy; };
  for (int t = 1; t < cnt; ++t) {
    const int jt = j0 + cnt - 1 - t;
    double *y = Y + (size_t)jt * ldy;
    bool ok = false;
    for (int attempt = 0; attempt < 5 && !ok; ++attempt) {
      if (attempt > 0) {   // a fresh pseudo-random unit vector (k + 4096 a never repeats a start)
        double ss = 0.0;
        for (int i = tid; i < n; i += blockDim.x) {
          const double v = start_entry(s, job_k[jt] + 4096 * attempt, i);
          y[i] = v;
          ss += v * v;
        }
        const double inv = 1.0 / sqrt(block_sum(ss, red));
        for (int i = tid; i < n; i += blockDim.x) y[i] *= inv;
        __syncthreads();
      }
      ok = true;
      for (int pass = 0; pass < 2; ++pass) {
        warp_dots8(vec, t, y, n, h);
        __syncthreads();
        const double ss = project_off(vec, t, h, y, n, gp);
        const double nrm = sqrt(block_sum(ss, red));   // the same value in every thread
        if (pass == 0 && !(nrm >= 1e-3)) {
          ok = false;
          break;
        }
        const double inv = 1.0 / nrm;
        for (int i = tid; i < n; i += blockDim.x) y[i] *= inv;
        __syncthreads();
        if (nrm > 0.7071067811865476) break;   // the vector entered with unit norm
      }
      if (!ok && attempt == 0 && !(evals[eoff[s] + job_k[jt]] - lam_min <= cluster)) break;
    }
    if (!ok && tid == 0) atomicOr(status, 2);
  }
}

// The same orthonormalisation of one large kept block by the CL CTAs of a
// cluster: CTA c owns a slice of rows of every vector.  Per projection pass
// each CTA forms its part of the dot products with the accepted vectors, the
// parts meet through distributed shared memory, every CTA sums them in rank
// order (so every CTA holds the same coefficients and takes the same
// decisions), subtracts on its own rows; the vector's squared norm travels
// with the dots, so that when the projection removes less than half of it
// (the common case: inverse iteration leaves the vectors nearly orthogonal)
// the new norm needs no second exchange; otherwise it is summed the same way
// after the subtraction.  Each exchange uses the buffer of its parity and ends with one
// cluster barrier; a buffer is written again only two exchanges later, after
// every CTA has passed the barrier that follows its reads.  A CTA reads and
// writes only its own rows of the vectors in global memory.
template <int CL>
__device__ void ortho_coop(cg::cluster_group &cl, int rank, int blk, const int *grp, const int *dims,
                           const int64_t *eoff, const double *evals, const double *info, const int *job_k, double *Y,
                           int ldy, int *status, double *sm, double *red) {
  const int s = grp[4 * blk], j0 = grp[4 * blk + 1], cnt = grp[4 * blk + 2];
  const int n = dims[s], tid = threadIdx.x, nt = blockDim.x;
  const double lam_min = evals[eoff[s]], cluster = 1e4 * EIG_EPS * info[4 * s + 2];
  const int per = (n + CL - 1) / CL, r0 = min(n, rank * per), r1 = min(n, r0 + per), nr = r1 - r0;
  // hp: parts of the dots (2 x cnt), h: the dots (cnt), ys: own rows of the
  // vector (per), sl: parts of the squared norm (2), gp: project_off's group
  // parts (nt)
  double *hp = sm, *h = hp + 2 * cnt, *ys = h + cnt, *sl = ys + per, *gp = sl + 2;
  unsigned xch = 0;   // exchanges so far (buffer parity)
  int half = 0;       // block_sum1's alternating half of red
  auto cluster_sum = [&](double x) -> double {   // x: the CTA's value, the same in all its threads
    double *slot = sl + (xch & 1);
    if (tid == 0) *slot = x;
    cl.sync();
    ++xch;
    double tot = 0.0;
    for (int c = 0; c < CL; ++c) tot += *cl.map_shared_rank(slot, c);
    return tot;
  };
  auto vec = [&](int q) { return Y + (size_t)(j0 + cnt - 1 - q) * ldy; };   // q-th vector in descending order
  for (int t = 1; t < cnt; ++t) {
    double *y = vec(t);
    const int jt = j0 + cnt - 1 - t;
    bool ok = false;
    for (int attempt = 0; attempt < 5 && !ok; ++attempt) {
      if (attempt == 0) {
        for (int i = tid; i < nr; i += nt) ys[i] = y[r0 + i];
        __syncthreads();
      } else {   // a fresh pseudo-random unit vector (see ortho_one)
        double ss = 0.0;
        for (int i = tid; i < nr; i += nt) {
          const double v = start_entry(s, job_k[jt] + 4096 * attempt, r0 + i);
          ys[i] = v;
          ss += v * v;
        }
        const double inv = 1.0 / sqrt(cluster_sum(block_sum1(ss, red, half)));
        for (int i = tid; i < nr; i += nt) ys[i] *= inv;
        __syncthreads();
      }
      ok = true;
      for (int pass = 0; pass < 2; ++pass) {
        // one exchange carries the dots with the accepted vectors and the
        // vector's own squared norm (slot t); when the projection removes
        // less than half of the squared norm, the new norm is yy - sum h^2
        // (accurate to rounding there), and no second exchange is needed
        double *hpw = hp + (xch & 1) * cnt;
        warp_dots8([&](int q) -> const double * { return q < t ? vec(q) + r0 : ys; }, t + 1, ys, nr, hpw);
        cl.sync();
        ++xch;
        double hh = 0.0;
        for (int q = tid; q <= t; q += nt) {
          double tot = 0.0;
          for (int c = 0; c < CL; ++c) tot += cl.map_shared_rank(hpw, c)[q];
          h[q] = tot;
          if (q < t) hh += tot * tot;
        }
        const double s2 = block_sum1(hh, red, half);   // also the barrier after h
        const double yy = h[t], rest = yy - s2;        // the same values in every CTA
        const bool fast = rest >= 0.5 * yy && rest > 0.0;
        const double ss = project_off([&](int q) -> const double * { return vec(q) + r0; }, t, h, ys, nr, gp);
        const double nrm = fast ? sqrt(rest) : sqrt(cluster_sum(block_sum1(ss, red, half)) / yy);
        if (pass == 0 && !(nrm >= 1e-3)) {
          ok = false;
          break;
        }
        const double inv = fast ? 1.0 / nrm : 1.0 / (nrm * sqrt(yy));
        for (int i = tid; i < nr; i += nt) ys[i] *= inv;
        __syncthreads();
        if (nrm > 0.7071067811865476) break;   // relative to the norm the vector entered with
      }
      if (!ok && attempt == 0 && !(evals[eoff[s] + job_k[jt]] - lam_min <= cluster)) break;
    }
    for (int i = tid; i < nr; i += nt) y[r0 + i] = ys[i];
    __syncthreads();
    if (!ok && rank == 0 && tid == 0) atomicOr(status, 2);
  }
  cl.sync();   // no CTA leaves while another may still read its buffers
}

// One cluster of CL CTAs per entry of the cluster list: a large kept block
// shared by all of them (obig), or up to CL small blocks, one per CTA
// (oblk[cluster * CL + rank], -1 for none); CL as for tridiag_kernel.
template <int CL>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(ORTH_THREADS, 1)
    orthonormalize_kernel(const int *oblk, const int *obig, const int *grp, const int *dims, const int64_t *eoff,
                          const double *evals, const double *info, const int *job_k, double *Y, int ldy,
                          int *status) {
  extern __shared__ double sm[];
  __shared__ double red[64];
  cg::cluster_group cl = cg::this_cluster();
  const int b = blockIdx.x / CL, rank = (int)cl.block_rank();
  const int blk = oblk[blockIdx.x];
  if (obig[b])
    ortho_coop<CL>(cl, rank, blk, grp, dims, eoff, evals, info, job_k, Y, ldy, status, sm, red);
  else if (blk >= 0)
    ortho_one(blk, grp, dims, eoff, evals, info, job_k, Y, ldy, status, sm, red);
}

// Back-transformation of the kept vectors, one warp per vector and the
// vector in shared memory: y <- H_0 (H_1 (... H_{n-2} y)), reflector k read
// from A(k+1:n, k) of its sector.  The sign is fixed so that the entry of
// largest magnitude (the first of equal ones) is positive, and the column is
// written to the truncation operator at job_dst[j].  slab[2b], slab[2b+1]:
// the block (grp index) and its first column handled by CTA b.
__global__ void backtransform_kernel(const double *Aall, const int64_t *off, const double *tauall,
                                     const int64_t *eoff, const int *dims, const int *grp, const int *slab,
                                     const double *Y, int ldy, const int64_t *job_dst, double *out) {
  extern __shared__ double colsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = slab[2 * blockIdx.x], c = slab[2 * blockIdx.x + 1] + warp;
  const int s = grp[4 * g], j0 = grp[4 * g + 1], cnt = grp[4 * g + 2];
  if (c >= cnt) return;
  const int n = dims[s], j = j0 + c;
  const double *A = Aall + off[s], *tau = tauall + eoff[s];
  double *col = colsm + (size_t)warp * ldy;
  for (int i = lane; i < n; i += 32) col[i] = Y[(size_t)j * ldy + i];
  __syncwarp();
  for (int k = n - 2; k >= 0; --k) {
    const double t = tau[k];
    if (t == 0.0) continue;
    const double *v = A + (int64_t)k * n;
    double acc = 0.0;
    for (int i = k + 1 + lane; i < n; i += 32) acc += v[i] * col[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const double f = t * acc;
    for (int i = k + 1 + lane; i < n; i += 32) col[i] -= f * v[i];
    __syncwarp();
  }
  double best = -1.0;
  int bi = 0;
  for (int i = lane; i < n; i += 32)
    if (fabs(col[i]) > best) {
      best = fabs(col[i]);
      bi = i;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  const double sg = col[bi] < 0.0 ? -1.0 : 1.0;
  double *dst = out + job_dst[j];
  for (int i = lane; i < n; i += 32) dst[i] = sg * col[i];
}

// The same back-transformation with each warp's vector in registers (lane l
// holds rows l + 32 r, r < RPL) for sectors of up to 32 RPL states: the CTA's
// BT_WARPS warps (vectors of one kept block, so of one sector) share the
// reflectors, staged kb at a time in shared memory by one coalesced load of
// the whole CTA, so that a step waits for no L2 load.  A lane's rows stay
// fixed (backtransform_kernel's shift with k), so the dot products are
// grouped differently: the two agree to rounding.  Warps past the block's
// last vector take part in the loads and barriers only.
constexpr int BT_WARPS = 8;
template <int RPL>
__global__ void __launch_bounds__(32 * BT_WARPS)
    backtransform_reg_kernel(const double *Aall, const int64_t *off, const double *tauall, const int64_t *eoff,
                             const int *dims, const int *grp, const int *slab, const double *Y, int ldy,
                             const int64_t *job_dst, double *out, int kb) {
  extern __shared__ double sv[];   // kb reflectors of n rows
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nt = blockDim.x;
  const int g = slab[2 * blockIdx.x], c = slab[2 * blockIdx.x + 1] + warp;
  const int s = grp[4 * g], j0 = grp[4 * g + 1], cnt = grp[4 * g + 2];
  const bool active = c < cnt;
  const int n = dims[s], j = j0 + c;
  const double *A = Aall + off[s], *tau = tauall + eoff[s];
  double col[RPL];
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int i = lane + 32 * r;
    col[r] = active && i < n ? Y[(size_t)j * ldy + i] : 0.0;
  }
  for (int k0 = n - 2; k0 >= 0; k0 -= kb) {
    const int nk = min(kb, k0 + 1);   // reflectors k0, k0 - 1, ..., k0 - nk + 1
    __syncthreads();                  // the previous chunk is read
    for (int u = 0; u < nk; ++u) {
      const int k = k0 - u;
      const double *v = A + (int64_t)k * n;
      for (int i = k + 1 + (int)threadIdx.x; i < n; i += nt) sv[(size_t)u * n + i] = v[i];
    }
    __syncthreads();
    if (!active) continue;
    for (int u = 0; u < nk; ++u) {
      const int k = k0 - u;
      const double t = tau[k];
      if (t == 0.0) continue;
      const double *v = sv + (size_t)u * n;
      // rows 32 r .. 32 r + 31 all at or above k are skipped by the whole
      // warp; two partial sums (even and odd r) shorten the chain of adds
      double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (32 * r + 31 > k && i > k && i < n) {
          if (r & 1)
            acc1 += v[i] * col[r];
          else
            acc0 += v[i] * col[r];
        }
      }
      double acc = acc0 + acc1;
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      const double f = t * acc;
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (32 * r + 31 > k && i > k && i < n) col[r] -= f * v[i];
      }
    }
  }
  if (!active) return;
  double best = -1.0;
  int bi = 0;
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int i = lane + 32 * r;
    if (i < n && fabs(col[r]) > best) {
      best = fabs(col[r]);
      bi = i;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  // the sign of the entry of largest magnitude: the lane holding row bi
  // broadcasts it
  double atbi = 0.0;
#pragma unroll
  for (int r = 0; r < RPL; ++r)
    if (lane + 32 * r == bi) atbi = col[r];
  atbi = __shfl_sync(0xffffffffu, atbi, bi & 31);
  const double sg = atbi < 0.0 ? -1.0 : 1.0;
  double *dst = out + job_dst[j];
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int i = lane + 32 * r;
    if (i < n) dst[i] = sg * col[r];
  }
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
  // the operator stays on the device (trA of ctx) until the second call
  // copies it out: valid while ctx has computed no other truncation
  int64_t len = 0;
  const tj_ctx *ctx = nullptr;
  uint64_t seq = 0;
  const double *dev = nullptr;
};
thread_local TruncCache g_tc;

// Fingerprint of psi for the two-call cache: 4096 values spread over it
// (the second call of the protocol passes the same, unchanged psi; a full
// pass over psi would cost more than the rest of the second call).
uint64_t hash_data(const double *p, int64_t n) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t)n;
  const int64_t k = n < 4096 ? n : 4096;
  for (int64_t i = 0; i < k; ++i) {
    const int64_t at = k > 1 ? i * (n - 1) / (k - 1) : 0;
    uint64_t u;
    std::memcpy(&u, p + at, 8);
    h = (h ^ u) * 1099511628211ull;
  }
  return h;
}

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

// Clusters of 16 CTAs (a non-portable size) where the GPU can schedule one
// with `threads` threads and `smem` bytes of dynamic shared memory per CTA;
// otherwise 8.  Asked once per kernel and shared-memory size.
template <typename K16>
int cluster_size(K16 kernel16, int threads, size_t smem) {
  static thread_local std::vector<std::pair<size_t, int>> seen;
  for (auto &x : seen)
    if (x.first == smem) return x.second;
  int cl = 8;
  if (cudaFuncSetAttribute(kernel16, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
      cudaFuncSetAttribute(kernel16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 16;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel16, &cfg) == cudaSuccess && n >= 1) cl = 16;
  }
  cudaGetLastError();
  seen.push_back({smem, cl});
  return cl;
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
    if (n > EIG_MAX_N) return set_err(TJ_ERR_LIMIT, "tj_truncation: a density-matrix sector exceeds 4096 states");
  }
  const uint64_t h = hash_data(wave->data, D);
  TruncCache &tc = g_tc;
  const bool hit = tc.valid && tc.data == wave->data && tc.dim == D && tc.side == side && tc.kept_min == kept_min &&
                   tc.kept_max == kept_max && tc.trun_err == trun_err && tc.hash == h && tc.ctx == ctx &&
                   tc.seq == ctx->trunc_seq;
  if (!hit) {
    CKT(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const auto wall0 = std::chrono::steady_clock::now();
    tc.valid = false;   // until this computation completes
    tc.ctx = ctx;
    tc.seq = ++ctx->trunc_seq;
    tc.dev = nullptr;
    tc.len = 0;
    CKT(cudaEventRecord(ctx->tev[0], st));
    // psi on the device and its norm
    int rc;
    if ((rc = ctx->trA.reserve(sizeof(double) * (D + 4)))) return rc;
    double *psi = ctx->trA.d();
    CKT(upload(ctx, psi, wave->data, D, st));
    double acc[4] = {0, 0, 0, 0};   // four independent sums, added at the end
    int64_t i = 0;
    for (; i + 4 <= D; i += 4)
      for (int q = 0; q < 4; ++q) acc[q] += wave->data[i + q] * wave->data[i + q];
    for (; i < D; ++i) acc[0] += wave->data[i] * wave->data[i];
    const double nrm2 = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    if (!(nrm2 > 0) || !std::isfinite(nrm2)) return set_err(TJ_ERR_NUMERIC, "tj_truncation: zero or non-finite psi");
    // rho per sector as one grouped-GEMM pass
    std::vector<Cell> cells;
    std::vector<Task> tasks;
    std::vector<Tile> tiles;
    std::vector<int64_t> roff(nsec), eoff(nsec);
    std::vector<int> dims(nsec), esec;
    int64_t rlen = 0, etot = 0;
    for (int i = 0; i < nsec; ++i) {
      const tj_wave_sub &w = wave->sub[i];
      const int n = side == 0 ? w.sys_dim : w.env_dim, K = side == 0 ? w.env_dim : w.sys_dim;
      dims[i] = n;
      roff[i] = rlen;
      eoff[i] = etot;
      rlen += ((int64_t)n * n + 31) / 32 * 32;
      etot += n;
      esec.insert(esec.end(), n, i);
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
    const int maxn = std::max(1, *std::max_element(dims.begin(), dims.end()));
    // sectors largest first for the one-CTA-per-sector reduction
    std::vector<int> order(nsec);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dims[a] > dims[b]; });
    // trD: d, e, tau, eigenvalues (etot each), then 4 per sector
    if ((rc = ctx->trB.reserve(sizeof(double) * (rlen + 4))) ||
        (rc = ctx->trD.reserve(sizeof(double) * (4 * etot + 4 * nsec + 8))))
      return rc;
    double *dd = ctx->trD.d(), *de = dd + etot, *dtau = de + etot, *dev = dtau + etot, *dinfo = dev + etot;
    // small tables packed into one buffer
    const size_t tb = cells.size() * sizeof(Cell), kb = tasks.size() * sizeof(Task), lb = tiles.size() * sizeof(Tile);
    const size_t ob = nsec * sizeof(int64_t), db = nsec * sizeof(int);
    size_t pos = 0;
    const size_t p_cells = pos; pos += al256(tb);
    const size_t p_tasks = pos; pos += al256(kb);
    const size_t p_tiles = pos; pos += al256(lb);
    const size_t p_roff = pos; pos += al256(ob);
    const size_t p_eoff = pos; pos += al256(ob);
    const size_t p_dims = pos; pos += al256(db);
    // clusters of the tridiagonal reduction: one per large sector, then the
    // small sectors tcl at a time (largest first)
    // shared memory: the per-sector vectors, and for a sector reduced by a
    // cluster as much more as a CTA may have (its slice of the trailing block)
    size_t tsm = sizeof(double) * (6 * (size_t)maxn + std::max(maxn, EIG_THREADS));
    if (maxn >= TD_BIG) {
      int optin = 0;
      cudaFuncAttributes fa;
      if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) == cudaSuccess &&
          cudaFuncGetAttributes(&fa, tridiag_kernel<16>) == cudaSuccess && optin > (int)fa.sharedSizeBytes + 1024)
        tsm = std::max(tsm, (size_t)(optin - (int)fa.sharedSizeBytes - 1024) / 256 * 256);
      cudaGetLastError();
    }
    const int tcl = cluster_size(tridiag_kernel<16>, EIG_THREADS, tsm);
    std::vector<int> tsec, tbig;
    {
      size_t q = 0;
      for (; q < order.size() && dims[order[q]] >= TD_BIG; ++q) {
        tsec.insert(tsec.end(), tcl, order[q]);
        tbig.push_back(1);
      }
      std::vector<int> small;
      for (; q < order.size(); ++q)
        if (dims[order[q]] > 0) small.push_back(order[q]);
      for (size_t i = 0; i < small.size(); i += tcl) {
        for (int r = 0; r < tcl; ++r) tsec.push_back(i + r < small.size() ? small[i + r] : -1);
        tbig.push_back(0);
      }
    }
    const int nclus = (int)tbig.size();
    const size_t p_tsec = pos; pos += al256(sizeof(int) * std::max<size_t>(tsec.size(), 1));
    const size_t p_tbig = pos; pos += al256(sizeof(int) * std::max<size_t>(tbig.size(), 1));
    const size_t p_esec = pos; pos += al256(sizeof(int) * (size_t)std::max<int64_t>(etot, 1));
    const size_t p_cnt = pos; pos += 256;
    if ((rc = ctx->trE.reserve(pos))) return rc;
    char *tbase = (char *)ctx->trE.p;
    CKT(cudaMemcpyAsync(tbase + p_cells, cells.data(), tb, cudaMemcpyHostToDevice, st));
    if (kb) CKT(cudaMemcpyAsync(tbase + p_tasks, tasks.data(), kb, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_tiles, tiles.data(), lb, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_roff, roff.data(), ob, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_eoff, eoff.data(), ob, cudaMemcpyHostToDevice, st));
    CKT(cudaMemcpyAsync(tbase + p_dims, dims.data(), db, cudaMemcpyHostToDevice, st));
    if (nclus) {
      CKT(cudaMemcpyAsync(tbase + p_tsec, tsec.data(), sizeof(int) * tsec.size(), cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(tbase + p_tbig, tbig.data(), sizeof(int) * tbig.size(), cudaMemcpyHostToDevice, st));
    }
    if (etot) CKT(cudaMemcpyAsync(tbase + p_esec, esec.data(), sizeof(int) * etot, cudaMemcpyHostToDevice, st));
    CKT(cudaMemsetAsync(tbase + p_cnt, 0, 256, st));
    const int64_t *d_roff = (const int64_t *)(tbase + p_roff), *d_eoff = (const int64_t *)(tbase + p_eoff);
    const int *d_dims = (const int *)(tbase + p_dims);
    int *d_status = (int *)(tbase + p_cnt + 16);
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
    CKT(cudaEventRecord(ctx->tev[1], st));
    // tridiagonal reduction, then all eigenvalues
    if (nclus) {
      const int *d_tsec = (const int *)(tbase + p_tsec), *d_tbig = (const int *)(tbase + p_tbig);
      if (tcl == 16) {
        CKT(cudaFuncSetAttribute(tridiag_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
        tridiag_kernel<16><<<nclus * 16, EIG_THREADS, tsm, st>>>(ctx->trB.d(), d_roff, d_dims, d_eoff, d_tsec, d_tbig,
                                                                 dd, de, dtau, dinfo, (int64_t)(tsm / 8));
      } else {
        CKT(cudaFuncSetAttribute(tridiag_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
        tridiag_kernel<8><<<nclus * 8, EIG_THREADS, tsm, st>>>(ctx->trB.d(), d_roff, d_dims, d_eoff, d_tsec, d_tbig,
                                                               dd, de, dtau, dinfo, (int64_t)(tsm / 8));
      }
      CKT(cudaGetLastError());
    }
    CKT(cudaEventRecord(ctx->tev[2], st));
    if (etot) {
      bisect_kernel<<<(unsigned)((etot + 3) / 4), 128, 0, st>>>(dd, de, d_eoff, d_dims, dinfo,
                                                                    (const int *)(tbase + p_esec), (int)etot, dev);
      CKT(cudaGetLastError());
    }
    std::vector<double> ev(etot);
    CKT(cudaMemcpyAsync(ev.data(), dev, sizeof(double) * etot, cudaMemcpyDeviceToHost, st));
    CKT(cudaEventRecord(ctx->tev[3], st));
    CKT(cudaStreamSynchronize(st));
    const auto sel0 = std::chrono::steady_clock::now();
    float stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 3; ++i) CKT(cudaEventElapsedTime(&stage_ms[i], ctx->tev[i], ctx->tev[i + 1]));
    double select_ms = 0;
    int max_kept = 0;

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
    std::vector<int> job_sec, job_k, grp, slab;
    std::vector<int64_t> job_dst;
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
      grp.insert(grp.end(), {x, (int)job_sec.size(), col, 0});
      for (int c = 0; c < col; ++c) {
        job_sec.push_back(x);
        job_k.push_back(asc[x][dims[x] - col + c]);
        job_dst.push_back(dpos + (int64_t)c * row);
      }
      dpos += (int64_t)row * col;
    }
    tc.len = dpos;
    const int njobs = (int)job_sec.size(), ngrp = (int)grp.size() / 4;
    if (njobs > 0) {
      // back-transformation: vectors in registers (BT_WARPS to a CTA) for
      // sectors of up to 32 * 48 states, else in shared memory (W warps)
      const bool bt_reg = maxn <= 32 * 48;
      const int W = bt_reg ? BT_WARPS : std::max(1, std::min(32, (int)(196608 / (sizeof(double) * maxn))));
      for (int b = 0; b < ngrp; ++b)
        for (int c0 = 0; c0 < grp[4 * b + 2]; c0 += W) slab.insert(slab.end(), {b, c0});
      const int nslab = (int)slab.size() / 2;
      const int ldy = (maxn + 3) / 4 * 4;
      // trC: inverse-iteration factors and vectors; trA: job tables and the operator
      const size_t wpl = (size_t)maxn * njobs;
      const size_t p_work = 0, p_y = p_work + al256(5 * wpl * 8), p_piv = p_y + al256((size_t)njobs * ldy * 8);
      if ((rc = ctx->trC.reserve(p_piv + al256(wpl)))) return rc;
      size_t q = 0;
      const size_t q_sec = q; q += al256((size_t)njobs * 4);
      const size_t q_k = q; q += al256((size_t)njobs * 4);
      const size_t q_dst = q; q += al256((size_t)njobs * 8);
      const size_t q_grp = q; q += al256(grp.size() * 4);
      const size_t q_slab = q; q += al256(slab.size() * 4);
      // clusters of the orthonormalisation: one per large kept block (cnt^2 n
      // above 3e7), then the other blocks ocl at a time, largest first
      const size_t osm = sizeof(double) * (3 * (size_t)maxn + (maxn + 7) / 8 + 8 + ORTH_THREADS);
      const int ocl = cluster_size(orthonormalize_kernel<16>, ORTH_THREADS, osm);
      std::vector<int> oblk, obig;
      {
        std::vector<int> bo(ngrp);
        std::iota(bo.begin(), bo.end(), 0);
        auto work = [&](int b) { return (double)grp[4 * b + 2] * grp[4 * b + 2] * dims[grp[4 * b]]; };
        std::stable_sort(bo.begin(), bo.end(), [&](int a, int b) { return work(a) > work(b); });
        size_t i = 0;
        for (; i < bo.size() && work(bo[i]) >= 3e7; ++i) {
          oblk.insert(oblk.end(), ocl, bo[i]);
          obig.push_back(1);
        }
        for (; i < bo.size(); i += ocl) {
          for (int r = 0; r < ocl; ++r) oblk.push_back(i + r < bo.size() ? bo[i + r] : -1);
          obig.push_back(0);
        }
      }
      const int nocl = (int)obig.size();
      const size_t q_oblk = q; q += al256(oblk.size() * 4);
      const size_t q_obig = q; q += al256(obig.size() * 4);
      const size_t q_out = q; q += al256((size_t)dpos * 8);
      if ((rc = ctx->trA.reserve(q))) return rc;   // psi is no longer needed
      char *ab = (char *)ctx->trA.p, *cb = (char *)ctx->trC.p;
      CKT(cudaMemcpyAsync(ab + q_sec, job_sec.data(), (size_t)njobs * 4, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_k, job_k.data(), (size_t)njobs * 4, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_dst, job_dst.data(), (size_t)njobs * 8, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_grp, grp.data(), grp.size() * 4, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_slab, slab.data(), slab.size() * 4, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_oblk, oblk.data(), oblk.size() * 4, cudaMemcpyHostToDevice, st));
      CKT(cudaMemcpyAsync(ab + q_obig, obig.data(), obig.size() * 4, cudaMemcpyHostToDevice, st));
      double *Y = (double *)(cb + p_y), *d_out = (double *)(ab + q_out);
      tc.dev = d_out;
      for (int b = 0; b < ngrp; ++b) max_kept = std::max(max_kept, grp[4 * b + 2]);
      select_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - sel0).count();
      CKT(cudaEventRecord(ctx->tev[4], st));
      inverse_iter_kernel<<<(njobs + 63) / 64, 64, 0, st>>>(dd, de, d_eoff, d_dims, dinfo, dev,
                                                            (const int *)(ab + q_sec), (const int *)(ab + q_k), njobs,
                                                            maxn, (double *)(cb + p_work),
                                                            (unsigned char *)(cb + p_piv), Y, ldy, d_status);
      CKT(cudaGetLastError());
      CKT(cudaEventRecord(ctx->tev[5], st));
      {
        const int *d_oblk = (const int *)(ab + q_oblk), *d_obig = (const int *)(ab + q_obig);
        const int *d_grp = (const int *)(ab + q_grp), *d_k = (const int *)(ab + q_k);
        if (ocl == 16) {
          CKT(cudaFuncSetAttribute(orthonormalize_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)osm));
          orthonormalize_kernel<16><<<nocl * 16, ORTH_THREADS, osm, st>>>(d_oblk, d_obig, d_grp, d_dims, d_eoff, dev,
                                                                          dinfo, d_k, Y, ldy, d_status);
        } else {
          CKT(cudaFuncSetAttribute(orthonormalize_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)osm));
          orthonormalize_kernel<8><<<nocl * 8, ORTH_THREADS, osm, st>>>(d_oblk, d_obig, d_grp, d_dims, d_eoff, dev,
                                                                        dinfo, d_k, Y, ldy, d_status);
        }
      }
      CKT(cudaGetLastError());
      CKT(cudaEventRecord(ctx->tev[6], st));
      if (bt_reg) {
        // eight reflectors per chunk: two CTAs fit an SM for sectors of up to 1536 states
        const int kb = 8;
        const size_t bsm = sizeof(double) * (size_t)kb * maxn;
        const int rpl = (maxn + 31) / 32;
        auto launch = [&](auto kern) -> cudaError_t {
          cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm);
          if (e != cudaSuccess) return e;
          kern<<<nslab, 32 * BT_WARPS, bsm, st>>>(ctx->trB.d(), d_roff, dtau, d_eoff, d_dims, (const int *)(ab + q_grp),
                                                 (const int *)(ab + q_slab), Y, ldy, (const int64_t *)(ab + q_dst),
                                                 d_out, kb);
          return cudaGetLastError();
        };
        if (rpl <= 8) CKT(launch(backtransform_reg_kernel<8>));
        else if (rpl <= 16) CKT(launch(backtransform_reg_kernel<16>));
        else if (rpl <= 24) CKT(launch(backtransform_reg_kernel<24>));
        else if (rpl <= 32) CKT(launch(backtransform_reg_kernel<32>));
        else if (rpl <= 40) CKT(launch(backtransform_reg_kernel<40>));
        else CKT(launch(backtransform_reg_kernel<48>));
      } else {
        const size_t bsm = sizeof(double) * (size_t)W * ldy;
        CKT(cudaFuncSetAttribute(backtransform_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
        backtransform_kernel<<<nslab, 32 * W, bsm, st>>>(ctx->trB.d(), d_roff, dtau, d_eoff, d_dims,
                                                         (const int *)(ab + q_grp), (const int *)(ab + q_slab), Y,
                                                         ldy, (const int64_t *)(ab + q_dst), d_out);
        CKT(cudaGetLastError());
      }
      int status[16] = {0};
      CKT(cudaMemcpyAsync(status, d_status, sizeof status, cudaMemcpyDeviceToHost, st));
      CKT(cudaEventRecord(ctx->tev[7], st));
      CKT(cudaStreamSynchronize(st));
      for (int i = 4; i < 7; ++i) CKT(cudaEventElapsedTime(&stage_ms[i - 1], ctx->tev[i], ctx->tev[i + 1]));
      if (status[0] & 1) {
        double dg[6];
        std::memcpy(dg, status + 4, sizeof dg);
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "tj_truncation: inverse iteration produced a non-finite vector (sector %d, eigenvalue %d of "
                      "%d, lambda %.17g, pivot floor %.3g, norm %g)",
                      (int)dg[0], (int)dg[1], (int)dg[4], dg[2], dg[3], dg[5]);
        return set_err(TJ_ERR_NUMERIC, buf);
      }
      if (status[0] & 2)
        return set_err(TJ_ERR_NUMERIC,
                       "tj_truncation: inverse iteration gave linearly dependent eigenvectors for a cluster of "
                       "eigenvalues above the bottom of its sector's spectrum");
    }
    {
      tj_hpsi_stats &S = ctx->stats;
      S.trunc_ms_rho = stage_ms[0];
      S.trunc_ms_tridiag = stage_ms[1];
      S.trunc_ms_eig = stage_ms[2];
      S.trunc_ms_select = select_ms;
      S.trunc_ms_vec = stage_ms[3];
      S.trunc_ms_orth = stage_ms[4];
      S.trunc_ms_back = stage_ms[5];
      S.trunc_ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
      S.trunc_max_n = maxn;
      S.trunc_max_kept = max_kept;
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
    if (tc.len > 0) {
      // straight from the device into the caller's array (the cache hit
      // above requires the device copy to be intact)
      CKT(cudaSetDevice(ctx->device));
      const int rc = download(ctx, udata, tc.dev, tc.len, ctx->stream);
      if (rc) return rc;
    }
    // the renormalisation of this step and the prediction of the next read
    // the operator again: with residency on, its device copy is kept (the
    // copy runs on the context's stream, ahead of anything that rewrites trA)
    if (tc.len > 0) {
      const int rc = res_keep(ctx, udata, tc.len, tc.dev, ctx->stream);
      if (rc) return rc;
    }
  }
  return TJ_OK;
}
