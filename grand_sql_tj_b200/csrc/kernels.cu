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

// Number of eigenvalues of the tridiagonal (a, b2 = b*b) below x (Sturm count).
__device__ __forceinline__ int sturm_count(const double *a, const double *b2, int n, double x) {
  const double tiny = 1e-300;
  int cnt = 0;
  double q = a[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < n; ++i) {
    if (fabs(q) < tiny) q = -tiny;
    q = (a[i] - x) - b2[i - 1] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}

// Ordered integer image of a double: monotone in the value, with +0 and -0
// both at 0, so that consecutive integers are adjacent doubles.
__device__ __forceinline__ int64_t ord_of(double x) {
  const int64_t bits = __double_as_longlong(x);
  return bits >= 0 ? bits : -(bits & 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double val_of(int64_t k) {
  return k >= 0 ? __longlong_as_double(k) : __longlong_as_double((-k) | (int64_t)0x8000000000000000ULL);
}

constexpr int TRI_THREADS = 256;   // threads (multisection points) of the tridiagonal eigenvalue kernels

// Lowest eigenpair of a symmetric tridiagonal matrix (n <= 128): the lowest
// eigenvalue to full precision -- the pair of adjacent doubles where the
// Sturm count turns from 0 to 1 -- by multisection over the ordered integer
// images of the doubles (TRI_THREADS points per pass, one per thread, about
// eight bits per pass; the last pass places its points on consecutive
// doubles), then inverse iteration with a pivoted tridiagonal solve on one
// thread.  n is at most the Lanczos depth.  Runs on one block of TRI_THREADS
// threads; every thread returns the same bracket [lo, hi] of adjacent doubles.
// hint (if finite): an upper estimate of the eigenvalue, such as the lowest
// eigenvalue of the leading (n-1) x (n-1) matrix, which is never below it
// (Cauchy interlacing).  The first pass then places its points at
// geometrically growing distances below the hint (and one just above it), so
// that the bracket it leaves is a fraction of the eigenvalue's distance from
// the hint wide; the bracket at the end is the same either way.
__device__ void tridiag_min_bracket(const double *a, const double *b, int n, double hint, double &lo_out,
                                    double &hi_out) {
  __shared__ double sa[128], sb2[128], slo[TRI_THREADS / 32], shi[TRI_THREADS / 32];
  __shared__ unsigned sv[TRI_THREADS / 32], su[TRI_THREADS / 32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  // the matrix to shared memory, and its Gershgorin bounds (a block-wide min
  // and max of a[i] -+ (|b[i-1]| + |b[i]|), exact in any order)
  double lo = INFINITY, hi = -INFINITY;
  for (int i = t; i < n; i += blockDim.x) {
    sa[i] = a[i];
    sb2[i] = i < n - 1 ? b[i] * b[i] : 0.0;
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < n - 1 ? fabs(b[i]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (lane == 0) {
    slo[w] = lo;
    shi[w] = hi;
  }
  __syncthreads();
  lo = slo[0];
  hi = shi[0];
  for (int q = 1; q < TRI_THREADS / 32; ++q) {
    lo = fmin(lo, slo[q]);
    hi = fmax(hi, shi[q]);
  }
  // invariant: count(lo) = 0 < count(hi) (Gershgorin bounds)
  // images lie in (-2^63, 2^63), so their distance can exceed the int64
  // range: spans and offsets are taken modulo 2^64, where they are exact
  int64_t klo = ord_of(lo), khi = ord_of(hi);
  auto dist = [](int64_t kl, int64_t kh) -> uint64_t { return (uint64_t)kh - (uint64_t)kl; };
  auto point = [&](int j, int64_t kl, int64_t kh) -> int64_t {
    const uint64_t span = dist(kl, kh);
    if (span <= (uint64_t)TRI_THREADS + 1) return (int64_t)((uint64_t)kl + (uint64_t)(j + 1));
    return (int64_t)((uint64_t)kl +
                     (uint64_t)((double)span * ((double)(j + 1) / (double)(TRI_THREADS + 1))));
  };
  // first-pass points from the hint: point j = khint + 1 - (g - 1) with
  // g = below^((T-1-j)/(T-1)), below = khint + 1 - klo; non-decreasing in j,
  // the last one just above the hint
  const bool use_hint = isfinite(hint) && hint > lo && hint < hi;
  const int64_t khint = use_hint ? ord_of(hint) : 0;
  auto hint_point = [&](int j, int64_t kl) -> int64_t {
    const double below = (double)(dist(kl, khint) + 1);
    const double g = exp2((double)(TRI_THREADS - 1 - j) * log2(below) / (double)(TRI_THREADS - 1));
    const uint64_t off = g >= below ? dist(kl, khint) + 1 : (uint64_t)g;   // 1 .. below
    return (int64_t)((uint64_t)khint + 1 - (off - 1));
  };
  for (int pass = 0; pass < 64 && khi > klo && dist(klo, khi) > 1; ++pass) {
    const bool geo = use_hint && pass == 0;
    auto pt = [&](int j) { return geo ? hint_point(j, klo) : point(j, klo, khi); };
    const int64_t kx = pt(t);
    const bool valid = kx > klo && kx < khi;
    const bool up = valid && sturm_count(sa, sb2, n, val_of(kx)) >= 1;
    const unsigned vm = __ballot_sync(0xffffffffu, valid), um = __ballot_sync(0xffffffffu, up);
    if (lane == 0) {
      sv[w] = vm;
      su[w] = um;
    }
    __syncthreads();
    // f: the first point with a count of at least one; the new lo is the
    // highest valid point below it (all of them have a count of zero)
    int f = -1, g = -1;
    for (int q = 0; q < TRI_THREADS / 32 && f < 0; ++q)
      if (su[q]) f = q * 32 + __ffs(su[q]) - 1;
    const int lim = f < 0 ? TRI_THREADS : f;
    for (int q = (lim - 1) >> 5; q >= 0 && g < 0 && lim > 0; --q) {
      unsigned m = sv[q];
      const int top = lim - q * 32;
      if (top < 32) m &= (1u << top) - 1u;
      if (m) g = q * 32 + 31 - __clz(m);
    }
    const int64_t nlo = g >= 0 ? pt(g) : klo, nhi = f >= 0 ? pt(f) : khi;
    __syncthreads();
    if (nlo == klo && nhi == khi) break;   // no valid point: lo and hi are adjacent
    klo = nlo;
    khi = nhi;
  }
  lo_out = val_of(klo);
  hi_out = val_of(khi);
}

__device__ void tridiag_min_body(const double *a, const double *b, int n, double *lam, double *vec, int want_vec) {
  if (blockIdx.x != 0) return;
  double lo, hi;
  tridiag_min_bracket(a, b, n, __longlong_as_double(0x7FF8000000000000LL), lo, hi);
  const double l = 0.5 * (lo + hi);
  if (threadIdx.x != 0) return;
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
  tridiag_min_kernel<<<1, TRI_THREADS, 0, s>>>(a, b, n, lam, vec, want_vec);
}

// ---- one Lanczos iteration with its step read from device memory (*it), so
// that the same launches -- captured once as a CUDA graph -- serve every
// iteration.  S holds alpha (0..127), beta (128..255), uu (256..383), the
// Gram-Schmidt coefficients (384..511), the Ritz value (512) and a norm (513).
// Each norm or dot product is folded into the kernel that produces its
// vector (one pass over the vector instead of two, one launch instead of
// three): every block reduces its share of the squares or products, and the
// last block to finish adds the block partials in a fixed order, so the
// result does not depend on the order the blocks run in.
__device__ __forceinline__ double *lz_ptr(const LzRef &r) {
  return r.fixed ? r.fixed : r.V + (int64_t)(*r.it + r.off - 1) * r.ld;
}

// The block partial s (valid in thread 0) to partials[blockIdx.x]; the last
// block to arrive (counted on *cnt, which it resets for the next kernel) adds
// the partials, thread i taking i, i + blockDim.x, ..., then the block tree,
// and stores the total (or its square root) at *res.
__device__ void lz_grid_sum(double s, double *partials, int *cnt, double *res, int sqrt_flag, double *sh) {
  __shared__ int last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(cnt, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += __ldcg(partials + i);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    *res = sqrt_flag ? sqrt(t) : t;
    *cnt = 0;
  }
}

// vec(L+1) = H vec(L) - alpha(L) vec(L) - beta(L-1) vec(L-1); beta(L) = |vec(L+1)|
__global__ void lz_update_norm_kernel(LzRef dst, const double *__restrict__ src, LzRef x1, LzRef x2, double *S,
                                      const int *it, int64_t n, double *partials, int *cnt) {
  __shared__ double sh[VT / 32];
  const int L = *it;
  const double av = S[L], bv = L >= 2 ? S[128 + L - 1] : 0.0;
  double *__restrict__ y = lz_ptr(dst);
  const double *__restrict__ p1 = lz_ptr(x1);
  const double *__restrict__ p2 = L >= 2 ? lz_ptr(x2) : nullptr;
  double s = 0.0;
#pragma unroll 4
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = src[i] - av * p1[i];
    if (p2) v = v - bv * p2[i];
    y[i] = v;
    s += v * v;
  }
  s = block_sum(s, sh);
  lz_grid_sum(s, partials, cnt, S + 128 + L, 1, sh);
}

// Projections of w / beta(L) on vec(1..L), with w scaled in place: each block
// keeps its slice of w in registers and streams the L vectors past it (the
// kernel is bound by those reads: L vectors of n doubles).  Five resident
// blocks per SM put the grid (one block per VT * MD_PER elements: 685 for
// 1.4M) in one wave on 148 SMs.
__global__ void __launch_bounds__(VT, 5) lz_multi_dot_kernel(const double *__restrict__ V, int64_t ld, const int *it, LzRef wr_, int64_t n,
                                    const double *S, double *partials, int kmax) {
  __shared__ double sh[VT / 32];
  const int L = *it;
  const int k = min(L, kmax);
  const double d = S[128 + L];
  double *__restrict__ w = lz_ptr(wr_);
  const int64_t base = (int64_t)blockIdx.x * VT * MD_PER + threadIdx.x;
  double wr[MD_PER];
#pragma unroll
  for (int i = 0; i < MD_PER; ++i) {
    const int64_t e = base + (int64_t)i * VT;
    wr[i] = 0.0;
    if (e < n) {
      wr[i] = w[e] / d;
      w[e] = wr[i];
    }
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

// coef(j) = (sum of the block projections) / uu(j), one block per vector
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

// w -= sum_j coef(j) vec(j); S[513] = |w|
constexpr int LZ_KMAX = 128;
__global__ void lz_combine_norm_kernel(const double *__restrict__ V, int64_t ld, const int *it,
                                       const double *__restrict__ coef, LzRef wr_, int64_t n, double *S,
                                       double *partials, int *cnt) {
  __shared__ double c[LZ_KMAX];
  __shared__ double sh[VT / 32];
  const int k = min(*it, LZ_KMAX);
  double *__restrict__ w = lz_ptr(wr_);
  for (int j = threadIdx.x; j < k; j += blockDim.x) c[j] = coef[j];
  __syncthreads();
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int j = 0; j < k; ++j) t = t + c[j] * V[(int64_t)j * ld + i];
    const double v = w[i] - t;
    w[i] = v;
    s += v * v;
  }
  s = block_sum(s, sh);
  lz_grid_sum(s, partials, cnt, S + 513, 1, sh);
}

// w /= S[513], copied to x; uu(L+1) = w . w
__global__ void lz_scale_norm_kernel(LzRef wr_, double *__restrict__ x, int64_t n, double *S, const int *it,
                                     double *partials, int *cnt) {
  __shared__ double sh[VT / 32];
  const int L = *it;
  const double d = S[513];
  double *__restrict__ w = lz_ptr(wr_);
  double s = 0.0;
#pragma unroll 4
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = w[i] / d;
    w[i] = v;
    x[i] = v;
    s += v * v;
  }
  s = block_sum(s, sh);
  lz_grid_sum(s, partials, cnt, S + 257 + L, 0, sh);
}

// alpha(L+1) = vec(L+1) . y
__global__ void lz_dot_kernel(LzRef xr, const double *__restrict__ y, int64_t n, double *S, const int *it,
                              double *partials, int *cnt) {
  __shared__ double sh[VT / 32];
  const int L = *it;
  const double *__restrict__ x = lz_ptr(xr);
  double s = 0.0;
#pragma unroll 4
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  s = block_sum(s, sh);
  lz_grid_sum(s, partials, cnt, S + 1 + L, 0, sh);
}

// The Ritz value of T(L+1); beta(L) and the Ritz value to page-locked host
// memory; the step advances.
__global__ void lz_tridiag_publish_kernel(double *S, int *it, double *host) {
  const int L = *it;
  double lo, hi;
  // from the second step on, S[512] holds the Ritz value of the step before
  tridiag_min_bracket(S + 1, S + 129, L + 1, L >= 2 ? S[512] : __longlong_as_double(0x7FF8000000000000LL), lo, hi);
  if (threadIdx.x != 0) return;
  S[512] = 0.5 * (lo + hi);
  host[0] = S[128 + L];
  host[1] = S[512];
  __threadfence_system();
  *it = L + 1;
}

// the elementwise kernels with a fused norm run on the grid of a dot product
// (fewer partials for the last block to add); the Gram-Schmidt combination,
// which streams L vectors per element, on the wider vector grid
int lz_blocks(int64_t n) { return std::max(vgrid(n), dot_blocks(n)); }
void launch_lz_update_norm(LzRef dst, const double *src, LzRef x1, LzRef x2, double *S, const int *it, int64_t n,
                           double *partials, int *cnt, cudaStream_t s) {
  lz_update_norm_kernel<<<dot_blocks(n), VT, 0, s>>>(dst, src, x1, x2, S, it, n, partials, cnt);
}
void launch_lz_gram_schmidt(const double *V, int64_t ld, const int *it, LzRef w, int64_t n, double *S,
                            double *mpartials, int mdb, int kmax, const double *uu, double *coef, double *partials,
                            int *cnt, cudaStream_t s) {
  lz_multi_dot_kernel<<<mdb, VT, 0, s>>>(V, ld, it, w, n, S, mpartials, kmax);
  lz_multi_sum_kernel<<<kmax, VT, 0, s>>>(mpartials, mdb, kmax, uu, coef, it);
  lz_combine_norm_kernel<<<vgrid(n), VT, 0, s>>>(V, ld, it, coef, w, n, S, partials, cnt);
}
void launch_lz_scale_norm(LzRef w, double *x, int64_t n, double *S, const int *it, double *partials, int *cnt,
                          cudaStream_t s) {
  lz_scale_norm_kernel<<<dot_blocks(n), VT, 0, s>>>(w, x, n, S, it, partials, cnt);
}
void launch_lz_dot(LzRef x, const double *y, int64_t n, double *S, const int *it, double *partials, int *cnt,
                   cudaStream_t s) {
  lz_dot_kernel<<<dot_blocks(n), VT, 0, s>>>(x, y, n, S, it, partials, cnt);
}
void launch_lz_tridiag_publish(double *S, int *it, double *host, cudaStream_t s) {
  lz_tridiag_publish_kernel<<<1, TRI_THREADS, 0, s>>>(S, it, host);
}

__global__ void copy_kernel(double *dst, const double *src, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}
void launch_copy(double *dst, const double *src, int64_t n, cudaStream_t s) {
  copy_kernel<<<vgrid(n), VT, 0, s>>>(dst, src, n);
}

}  // namespace tjb
