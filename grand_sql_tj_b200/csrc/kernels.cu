// Device kernels of the B200 tjsq hot path: grouped FP64 GEMM over psi cells,
// merged-operator sums (hmerge), and the Lanczos vector operations.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"

namespace tjb {

// ------------------------------------------------------------ grouped GEMM
// One persistent CTA (4 warps) repeatedly takes a 64x64 tile of a cell from a
// global counter and accumulates sum_t coef_t * op(L_t) * op(R_t) over the
// cell's tasks with FP64 DMMA (mma.sync m8n8k4).  Operand tiles are staged in
// shared memory in the layout that keeps the global reads coalesced:
// [k][m] when op(L) is stored m-contiguous, [m][k] when k-contiguous (same
// for R), each padded by 4 doubles so the fragment reads are conflict-free.
constexpr int LDS_KM = BM + 4;   // [k][m] leading dimension
constexpr int LDS_KN = BN + 4;   // [k][n]
constexpr int LDS_MK = BK + 4;   // [m][k] and [n][k]
constexpr int SMEM_L = (BM * LDS_MK > BK * LDS_KM) ? BM * LDS_MK : BK * LDS_KM;
constexpr int SMEM_R = (BN * LDS_MK > BK * LDS_KN) ? BN * LDS_MK : BK * LDS_KN;
constexpr int GEMM_THREADS = 128;

__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ const double *space_base(const GemmParams &p, int sp) {
  return sp == SP_OPS ? p.ops : (sp == SP_PSI ? p.psi : p.scr);
}

__global__ void __launch_bounds__(GEMM_THREADS, 4) grouped_gemm_f64(GemmParams p) {
  __shared__ __align__(16) double Ls[SMEM_L];
  __shared__ __align__(16) double Rs[SMEM_R];
  __shared__ int s_tile;
  __shared__ double s_red[GEMM_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp >> 1, wc = warp & 1;

  for (;;) {
    if (tid == 0) s_tile = (int)atomicAdd(p.counter, 1u);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if (t >= p.ntiles) return;
    const Tile tl = p.tiles[t];
    const Cell c = p.cells[tl.cell];

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    for (int ti = tl.tb; ti < tl.te; ++ti) {
      const Task tk = p.tasks[ti];
      const double *__restrict__ Lb = space_base(p, tk.L.space) + tk.L.off;
      const double *__restrict__ Rb = space_base(p, tk.R.space) + tk.R.off;
      const int ldl = tk.L.ld, ldr = tk.R.ld, K = tk.K;
      const bool lt = tk.L.trans != 0, rt = tk.R.trans != 0;
      const double coef = tk.coef;
      const int lsr = lt ? LDS_MK : 1, lsk = lt ? 1 : LDS_KM;
      const int rsn = rt ? 1 : LDS_MK, rsk = rt ? LDS_KN : 1;
      for (int k0 = 0; k0 < K; k0 += BK) {
        if (!lt) {
          const int r = tid & 63, kb = tid >> 6, gr = tl.row0 + r;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k = kb + 2 * j, gk = k0 + k;
            double v = 0.0;
            if (gr < c.M && gk < K) v = coef * Lb[(int64_t)gk * ldl + gr];
            Ls[k * LDS_KM + r] = v;
          }
        } else {
          const int k = tid & 15, rb = tid >> 4, gk = k0 + k;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int r = rb + 8 * j, gr = tl.row0 + r;
            double v = 0.0;
            if (gr < c.M && gk < K) v = coef * Lb[(int64_t)gr * ldl + gk];
            Ls[r * LDS_MK + k] = v;
          }
        }
        if (!rt) {
          const int k = tid & 15, nb = tid >> 4, gk = k0 + k;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int n = nb + 8 * j, gn = tl.col0 + n;
            double v = 0.0;
            if (gn < c.N && gk < K) v = Rb[(int64_t)gn * ldr + gk];
            Rs[n * LDS_MK + k] = v;
          }
        } else {
          const int n = tid & 63, kb = tid >> 6, gn = tl.col0 + n;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k = kb + 2 * j, gk = k0 + k;
            double v = 0.0;
            if (gn < c.N && gk < K) v = Rb[(int64_t)gk * ldr + gn];
            Rs[k * LDS_KN + n] = v;
          }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK / 4; ++kk) {
          const int k = kk * 4 + (lane & 3);
          double a[4], b[4];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) a[mi] = Ls[(wr * 32 + mi * 8 + (lane >> 2)) * lsr + k * lsk];
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) b[ni] = Rs[(wc * 32 + ni * 8 + (lane >> 2)) * rsn + k * rsk];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma_8x8x4(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
      }
    }

    double local = 0.0;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = tl.row0 + wr * 32 + mi * 8 + (lane >> 2);
          const int n = tl.col0 + wc * 32 + ni * 8 + 2 * (lane & 3) + e;
          if (r < c.M && n < c.N) {
            double v = acc[mi][ni][e];
            for (int tj = tl.ab; tj < tl.ae; ++tj) {
              const Task &ax = p.tasks[tj];
              v += ax.coef * space_base(p, ax.L.space)[ax.L.off + (int64_t)n * ax.L.ld + r];
            }
            const int64_t o = c.off + (int64_t)n * c.ld + r;
            if (p.dot_mode)
              local += v * p.dot_with[o];
            else if (tl.slot < 0)
              p.out[o] = v;
            else
              p.slots[(int64_t)tl.slot * (BM * BN) + (n - tl.col0) * BM + (r - tl.row0)] = v;
          }
        }
    if (p.dot_mode) {
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) local += __shfl_down_sync(0xffffffffu, local, s);
      if (lane == 0) s_red[warp] = local;
      __syncthreads();
      if (tid == 0) {
        double tot = 0.0;
        for (int w = 0; w < GEMM_THREADS / 32; ++w) tot += s_red[w];
        p.partials[t] = tot;
      }
      __syncthreads();
    }
  }
}

int grouped_gemm_grid(int ntiles, int ctas_per_sm) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int g = sms * std::min(4, std::max(1, ctas_per_sm));
  return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

void launch_grouped_gemm(const GemmParams &p, int grid, cudaStream_t s) {
  if (p.ntiles <= 0) return;
  grouped_gemm_f64<<<grid, GEMM_THREADS, 0, s>>>(p);
}

// One CTA per split tile: the slots are added in slot order, so the result
// does not depend on which items finished first.
__global__ void reduce_slots_kernel(GemmParams p, const Reduce *red) {
  const Reduce rd = red[blockIdx.x];
  const Cell c = p.cells[rd.cell];
  const int rows = min(BM, c.M - rd.row0), cols = min(BN, c.N - rd.col0);
  for (int idx = threadIdx.x; idx < rows * cols; idx += blockDim.x) {
    const int r = idx % rows, n = idx / rows;
    double v = 0.0;
    for (int k = 0; k < rd.nslot; ++k) v += p.slots[(int64_t)(rd.slot0 + k) * (BM * BN) + n * BM + r];
    const int gr = rd.row0 + r, gn = rd.col0 + n;
    for (int tj = rd.ab; tj < rd.ae; ++tj) {
      const Task &ax = p.tasks[tj];
      v += ax.coef * space_base(p, ax.L.space)[ax.L.off + (int64_t)gn * ax.L.ld + gr];
    }
    p.out[c.off + (int64_t)gn * c.ld + gr] = v;
  }
}

void launch_reduce(const GemmParams &p, const Reduce *red, int nred, cudaStream_t s) {
  if (nred > 0) reduce_slots_kernel<<<nred, 256, 0, s>>>(p, red);
}

// ------------------------------------------------------------------ merges
__global__ void merge_kernel(double *ops, const int64_t *dst, const int64_t *n, const int32_t *sb,
                             const int32_t *se, const int64_t *src, const double *coef) {
  const int r = blockIdx.x;
  const int64_t d = dst[r], len = n[r];
  const int b = sb[r], e = se[r];
  for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
    double acc = 0.0;
    for (int j = b; j < e; ++j) acc = acc + coef[j] * ops[src[j] + i];
    ops[d + i] = acc;
  }
}
void launch_merge(double *ops, const int64_t *dst, const int64_t *n, const int32_t *sb, const int32_t *se,
                  const int64_t *src, const double *coef, int nrec, cudaStream_t s) {
  if (nrec > 0) merge_kernel<<<nrec, 256, 0, s>>>(ops, dst, n, sb, se, src, coef);
}

// --------------------------------------------------------------- reductions
constexpr int VT = 256;   // threads of the vector kernels

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffu, v, s);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double tot = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += sh[i];
  __syncthreads();
  return tot;   // valid in thread 0
}

int dot_blocks(int64_t n) {
  int64_t b = (n + VT * 8 - 1) / (VT * 8);
  if (b < 1) b = 1;
  if (b > 2048) b = 2048;
  return (int)b;
}

__global__ void dot_kernel(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                           double *partials) {
  __shared__ double sh[VT / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
void launch_dot(const double *x, const double *y, int64_t n, double *partials, int nblk, cudaStream_t s) {
  dot_kernel<<<nblk, VT, 0, s>>>(x, y, n, partials);
}

__global__ void sum_kernel(const double *partials, int nblk, double *res, int sqrt_flag) {
  __shared__ double sh[VT / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += partials[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *res = sqrt_flag ? sqrt(s) : s;
}
void launch_sum(const double *partials, int nblk, double *res, int sqrt_flag, cudaStream_t s) {
  sum_kernel<<<1, VT, 0, s>>>(partials, nblk, res, sqrt_flag);
}

__global__ void lanczos_update_kernel(double *y, const double *x1, const double *x2, const double *a,
                                      const double *b, int64_t n) {
  const double av = *a, bv = x2 ? *b : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = y[i] - av * x1[i];
    if (x2) v = v - bv * x2[i];
    y[i] = v;
  }
}
static int vgrid(int64_t n) {
  int64_t g = (n + VT - 1) / VT;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}
void launch_lanczos_update(double *y, const double *x1, const double *x2, const double *a, const double *b,
                           int64_t n, cudaStream_t s) {
  lanczos_update_kernel<<<vgrid(n), VT, 0, s>>>(y, x1, x2, a, b, n);
}

__global__ void scale_inv_kernel(double *x, const double *nrm, int64_t n) {
  const double d = *nrm;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = x[i] / d;
}
void launch_scale_inv(double *x, const double *nrm, int64_t n, cudaStream_t s) {
  scale_inv_kernel<<<vgrid(n), VT, 0, s>>>(x, nrm, n);
}

// Gram-Schmidt projections: each block keeps its slice of w in registers and
// streams the k basis vectors past it.
constexpr int MD_PER = 8;
__global__ void multi_dot_kernel(const double *__restrict__ V, int64_t ld, int k, const double *__restrict__ w,
                                 int64_t n, double *partials, int kmax) {
  __shared__ double sh[VT / 32];
  const int64_t base = (int64_t)blockIdx.x * VT * MD_PER + threadIdx.x;
  double wr[MD_PER];
#pragma unroll
  for (int i = 0; i < MD_PER; ++i) {
    const int64_t e = base + (int64_t)i * VT;
    wr[i] = e < n ? w[e] : 0.0;
  }
  for (int j = 0; j < k; ++j) {
    const double *v = V + (int64_t)j * ld;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < MD_PER; ++i) {
      const int64_t e = base + (int64_t)i * VT;
      if (e < n) s += v[e] * wr[i];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[(int64_t)blockIdx.x * kmax + j] = s;
  }
}
void launch_multi_dot(const double *V, int64_t ld, int k, const double *w, int64_t n, double *partials, int nblk,
                      int kmax, cudaStream_t s) {
  multi_dot_kernel<<<nblk, VT, 0, s>>>(V, ld, k, w, n, partials, kmax);
}

__global__ void multi_sum_kernel(const double *partials, int nblk, int kmax, const double *uu, double *coef) {
  __shared__ double sh[VT / 32];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partials[(int64_t)b * kmax + j];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) coef[j] = uu ? s / uu[j] : s;
}
void launch_multi_sum(const double *partials, int nblk, int k, int kmax, const double *uu, double *coef,
                      cudaStream_t s) {
  if (k > 0) multi_sum_kernel<<<k, VT, 0, s>>>(partials, nblk, kmax, uu, coef);
}

__global__ void combine_kernel(const double *__restrict__ V, int64_t ld, int k, const double *__restrict__ coef,
                               double *w, int64_t n, int assign) {
  __shared__ double c[128];
  for (int j = threadIdx.x; j < k && j < 128; j += blockDim.x) c[j] = coef[j];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < k; ++j) t = t + c[j] * V[(int64_t)j * ld + i];
    w[i] = assign ? t : w[i] - t;
  }
}
void launch_combine(const double *V, int64_t ld, int k, const double *coef, double *w, int64_t n, int assign,
                    cudaStream_t s) {
  combine_kernel<<<vgrid(n), VT, 0, s>>>(V, ld, k, coef, w, n, assign);
}

// Number of eigenvalues of the tridiagonal (a, b) below x (Sturm count).
__device__ __forceinline__ int sturm_count(const double *a, const double *b, int n, double x) {
  const double tiny = 1e-300;
  int cnt = 0;
  double q = a[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    if (fabs(q) < tiny) q = -tiny;
    q = (a[i] - x) - b[i - 1] * b[i - 1] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}

// Lowest eigenpair of a symmetric tridiagonal matrix (n <= 128): the lowest
// eigenvalue to full precision -- the pair of adjacent doubles where the
// Sturm count turns from 0 to 1 -- by 32-point multisection (one warp, one
// point per lane: five bits per pass) finished by bisection, then inverse
// iteration with a pivoted tridiagonal solve on one thread.  n is at most the
// Lanczos depth.
__device__ void tridiag_min_body(const double *a, const double *b, int n, double *lam, double *vec, int want_vec) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  double lo = 0.0, hi = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < n - 1 ? fabs(b[i]) : 0.0);
    const double l = a[i] - r, h = a[i] + r;
    if (i == 0 || l < lo) lo = l;
    if (i == 0 || h > hi) hi = h;
  }
  // invariant: count(lo) = 0 < count(hi) (Gershgorin bounds)
  for (int pass = 0; pass < 64; ++pass) {
    const double x = lo + (hi - lo) * ((double)(lane + 1) / 33.0);
    const bool valid = x > lo && x < hi;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (vmask == 0) break;
    const int cnt = valid ? sturm_count(a, b, n, x) : 0;
    const unsigned up = __ballot_sync(0xffffffffu, valid && cnt >= 1);
    if (up == 0) {
      lo = __shfl_sync(0xffffffffu, x, 31 - __clz(vmask));   // the highest valid point
    } else {
      const int f = __ffs(up) - 1;
      const double xf = __shfl_sync(0xffffffffu, x, f);
      const double xp = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
      if (f > 0 && ((vmask >> (f - 1)) & 1u)) lo = xp;
      hi = xf;
    }
  }
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(a, b, n, mid) >= 1) hi = mid; else lo = mid;
  }
  const double l = 0.5 * (lo + hi);
  if (lane != 0) return;
  *lam = l;
  if (!want_vec) return;
  // inverse iteration on (T - l I) with partial pivoting
  double x[128], dd[128], du[128], du2[128], dl[128];
  int piv[128];
  double scale = fabs(hi) + fabs(lo) + 1.0;
  for (int i = 0; i < n; ++i) x[i] = 1.0;
  for (int iter = 0; iter < 3; ++iter) {
    for (int i = 0; i < n; ++i) {
      dd[i] = a[i] - l;
      du[i] = i < n - 1 ? b[i] : 0.0;
      dl[i] = i < n - 1 ? b[i] : 0.0;
      du2[i] = 0.0;
    }
    // LU with partial pivoting (dgttrf-like)
    for (int i = 0; i < n - 1; ++i) {
      if (fabs(dd[i]) >= fabs(dl[i])) {
        piv[i] = 0;
        if (dd[i] == 0.0) dd[i] = 1e-300 * scale + 1e-300;
        const double f = dl[i] / dd[i];
        dl[i] = f;
        dd[i + 1] -= f * du[i];
      } else {
        piv[i] = 1;
        const double f = dd[i] / dl[i];
        dd[i] = dl[i];
        dl[i] = f;
        const double t = du[i];
        du[i] = dd[i + 1];
        dd[i + 1] = t - f * dd[i + 1];
        if (i < n - 2) {
          du2[i] = du[i + 1];
          du[i + 1] = -f * du[i + 1];
        }
      }
    }
    if (dd[n - 1] == 0.0) dd[n - 1] = 1e-16 * scale;
    // solve L U y = x
    for (int i = 0; i < n - 1; ++i) {
      if (piv[i] == 0) {
        x[i + 1] -= dl[i] * x[i];
      } else {
        const double t = x[i];
        x[i] = x[i + 1];
        x[i + 1] = t - dl[i] * x[i + 1];
      }
    }
    x[n - 1] /= dd[n - 1];
    if (n > 1) x[n - 2] = (x[n - 2] - du[n - 2] * x[n - 1]) / dd[n - 2];
    for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - du[i] * x[i + 1] - du2[i] * x[i + 2]) / dd[i];
    double nr = 0.0;
    for (int i = 0; i < n; ++i) nr += x[i] * x[i];
    nr = sqrt(nr);
    for (int i = 0; i < n; ++i) x[i] /= nr;
  }
  // sign convention: first nonzero component positive
  double sgn = 1.0;
  for (int i = 0; i < n; ++i)
    if (x[i] != 0.0) { sgn = x[i] > 0 ? 1.0 : -1.0; break; }
  for (int i = 0; i < n; ++i) vec[i] = sgn * x[i];
}
__global__ void tridiag_min_kernel(const double *a, const double *b, int n, double *lam, double *vec, int want_vec) {
  tridiag_min_body(a, b, n, lam, vec, want_vec);
}
void launch_tridiag_min(const double *a, const double *b, int n, double *lam, double *vec, int want_vec,
                        cudaStream_t s) {
  tridiag_min_kernel<<<1, 32, 0, s>>>(a, b, n, lam, vec, want_vec);
}

// ---- one Lanczos iteration with its step read from device memory (*it), so
// that the same launches -- captured once as a CUDA graph -- serve every
// iteration.  S holds alpha (0..127), beta (128..255), uu (256..383), the
// Gram-Schmidt coefficients (384..511), the Ritz value (512) and a norm (513).
__device__ __forceinline__ double *lz_ptr(const LzRef &r) {
  return r.fixed ? r.fixed : r.V + (int64_t)(*r.it + r.off - 1) * r.ld;
}

__global__ void lz_update_kernel(LzRef dst, const double *__restrict__ src, LzRef x1, LzRef x2, const double *S,
                                 const int *it, int64_t n) {
  const int L = *it;
  const double av = S[L], bv = L >= 2 ? S[128 + L - 1] : 0.0;
  double *y = lz_ptr(dst);
  const double *p1 = lz_ptr(x1), *p2 = L >= 2 ? lz_ptr(x2) : nullptr;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = src[i] - av * p1[i];
    if (p2) v = v - bv * p2[i];
    y[i] = v;
  }
}

__global__ void lz_dot_kernel(LzRef x, LzRef y, int64_t n, double *partials) {
  __shared__ double sh[VT / 32];
  const double *__restrict__ px = lz_ptr(x), *__restrict__ py = lz_ptr(y);
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += px[i] * py[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void lz_sum_kernel(const double *partials, int nblk, double *S, const int *it, int idx, int sqrt_flag) {
  __shared__ double sh[VT / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += partials[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) S[idx + (it ? *it : 0)] = sqrt_flag ? sqrt(s) : s;
}

__global__ void lz_scale_kernel(LzRef x, const double *S, const int *it, int idx, double *copy, int64_t n) {
  const double d = S[idx + (it ? *it : 0)];
  double *px = lz_ptr(x);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = px[i] / d;
    px[i] = v;
    if (copy) copy[i] = v;
  }
}

__global__ void lz_multi_dot_kernel(const double *__restrict__ V, int64_t ld, const int *it, LzRef wr_, int64_t n,
                                    double *partials, int kmax) {
  __shared__ double sh[VT / 32];
  const int k = *it;
  const double *__restrict__ w = lz_ptr(wr_);
  const int64_t base = (int64_t)blockIdx.x * VT * MD_PER + threadIdx.x;
  double wr[MD_PER];
#pragma unroll
  for (int i = 0; i < MD_PER; ++i) {
    const int64_t e = base + (int64_t)i * VT;
    wr[i] = e < n ? w[e] : 0.0;
  }
  for (int j = 0; j < k; ++j) {
    const double *v = V + (int64_t)j * ld;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < MD_PER; ++i) {
      const int64_t e = base + (int64_t)i * VT;
      if (e < n) s += v[e] * wr[i];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partials[(int64_t)blockIdx.x * kmax + j] = s;
  }
}

__global__ void lz_multi_sum_kernel(const double *partials, int nblk, int kmax, const double *uu, double *coef,
                                    const int *it) {
  __shared__ double sh[VT / 32];
  const int j = blockIdx.x;
  if (j >= *it) return;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partials[(int64_t)b * kmax + j];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) coef[j] = s / uu[j];
}

__global__ void lz_combine_kernel(const double *__restrict__ V, int64_t ld, const int *it,
                                  const double *__restrict__ coef, LzRef wr_, int64_t n) {
  __shared__ double c[128];
  const int k = *it;
  double *w = lz_ptr(wr_);
  for (int j = threadIdx.x; j < k && j < 128; j += blockDim.x) c[j] = coef[j];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < k; ++j) t = t + c[j] * V[(int64_t)j * ld + i];
    w[i] = w[i] - t;
  }
}

__global__ void lz_tridiag_kernel(const double *a, const double *b, const int *it, int noff, double *lam) {
  tridiag_min_body(a, b, *it + noff, lam, nullptr, 0);
}

// beta(L) and the Ritz value to page-locked host memory; the step advances
__global__ void lz_publish_kernel(const double *S, int *it, double *host) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int L = *it;
  host[0] = S[128 + L];
  host[1] = S[512];
  __threadfence_system();
  *it = L + 1;
}

void launch_lz_update(LzRef dst, const double *src, LzRef x1, LzRef x2, const double *S, const int *it, int64_t n,
                      cudaStream_t s) {
  lz_update_kernel<<<vgrid(n), VT, 0, s>>>(dst, src, x1, x2, S, it, n);
}
void launch_lz_norm(LzRef x, int64_t n, double *partials, int nblk, double *S, const int *it, int idx, int sqrt_flag,
                    cudaStream_t s) {
  lz_dot_kernel<<<nblk, VT, 0, s>>>(x, x, n, partials);
  lz_sum_kernel<<<1, VT, 0, s>>>(partials, nblk, S, it, idx, sqrt_flag);
}
void launch_lz_dot(LzRef x, LzRef y, int64_t n, double *partials, int nblk, double *S, const int *it, int idx,
                   cudaStream_t s) {
  lz_dot_kernel<<<nblk, VT, 0, s>>>(x, y, n, partials);
  lz_sum_kernel<<<1, VT, 0, s>>>(partials, nblk, S, it, idx, 0);
}
void launch_lz_scale(LzRef x, const double *S, const int *it, int idx, double *copy, int64_t n, cudaStream_t s) {
  lz_scale_kernel<<<vgrid(n), VT, 0, s>>>(x, S, it, idx, copy, n);
}
void launch_lz_gram_schmidt(const double *V, int64_t ld, const int *it, LzRef w, int64_t n, double *partials,
                            int nblk, int kmax, const double *uu, double *coef, cudaStream_t s) {
  lz_multi_dot_kernel<<<nblk, VT, 0, s>>>(V, ld, it, w, n, partials, kmax);
  lz_multi_sum_kernel<<<kmax, VT, 0, s>>>(partials, nblk, kmax, uu, coef, it);
  lz_combine_kernel<<<vgrid(n), VT, 0, s>>>(V, ld, it, coef, w, n);
}
void launch_lz_tridiag(const double *a, const double *b, const int *it, int noff, double *lam, cudaStream_t s) {
  lz_tridiag_kernel<<<1, 32, 0, s>>>(a, b, it, noff, lam);
}
void launch_lz_publish(const double *S, int *it, double *host, cudaStream_t s) {
  lz_publish_kernel<<<1, 32, 0, s>>>(S, it, host);
}

__global__ void copy_kernel(double *dst, const double *src, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}
void launch_copy(double *dst, const double *src, int64_t n, cudaStream_t s) {
  copy_kernel<<<vgrid(n), VT, 0, s>>>(dst, src, n);
}

}  // namespace tjb
