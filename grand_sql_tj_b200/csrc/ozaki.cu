// Device side of the split-precision H*psi (see ozaki.h for the scheme).
//
// oz_split:  one warp per row: row max -> power-of-two scale 2^e with
//            |x| / 2^e < 1 -> s truncated radix-128 digits, each in [-127, 127].
// oz_gemm:   persistent CTAs (4 warps).  Per work item (group, 128 stacked
//            rows, BN shared-operand rows) the A slices (gathered rows) and B
//            slices are staged in shared memory in the UMMA K-major,
//            no-swizzle layout (8-row x 16-byte core matrices), one thread
//            issues tcgen05.mma kind::i8 for every slice pair (p, q) with
//            p + q <= s + 1 into the TMEM accumulator of diagonal p + q, a
//            tcgen05.commit arrives on an mbarrier, and all four warps read
//            the diagonals back (tcgen05.ld 32x32b), weight them by 128^-d in
//            FP64 and store the scaled rows.  Every wait is bounded: on
//            timeout the kernel raises an error flag, frees its TMEM and
//            returns.
// oz_sum:    output cell = sum of its tasks' results + axpy terms.
#include <cuda_runtime.h>

#include <cstdint>

#include <cute/arch/mma_sm100_desc.hpp>

#include "kernels.cuh"
#include "ozaki.h"

namespace tjb {

struct OzSplitParams {
  const OzSplit *jobs;
  const double *ops, *psi, *scr;
  int8_t *pack;
  double *sig;
  int s;
};

__global__ void __launch_bounds__(256) oz_split_kernel(OzSplitParams p) {
  const OzSplit J = p.jobs[blockIdx.x];
  const double *base = J.space == SP_OPS ? p.ops : (J.space == SP_PSI ? p.psi : p.scr);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < J.nrows; r += nw) {
    const double *row = base + J.src_off + (int64_t)r * J.rs;
    double mx = 0.0;
    for (int k = lane; k < J.K; k += 32) mx = fmax(mx, fabs(row[(int64_t)k * J.ks]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);   // mx = f 2^e, f in [0.5, 1): |x| 2^-e < 1
    if (lane == 0) p.sig[J.sig_off + r] = mx > 0.0 ? ldexp(1.0, e) : 0.0;
    int8_t *dst = p.pack + J.pack_off + (int64_t)r * J.K_pad;
    const int64_t sstride = (int64_t)J.nrows * J.K_pad;
    for (int k = lane; k < J.K_pad; k += 32) {
      double t = (k < J.K && mx > 0.0) ? ldexp(row[(int64_t)k * J.ks], -e) : 0.0;
      for (int q = 0; q < p.s; ++q) {
        t *= 128.0;
        const double a = trunc(t);
        t -= a;
        dst[q * sstride + k] = (int8_t)(int)a;
      }
    }
  }
}

// ------------------------------------------------------------ tcgen05 GEMM
struct OzGemmParams {
  const int8_t *dyn_pack;
  const double *dyn_sig;
  const int8_t *sta_pack;
  const double *sta_sig;
  const OzGroup *groups;
  const OzRow *rows;
  const OzItem *items;
  int nitems;
  double *out_scr, *out_slots;
  unsigned int *counter;
  int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no-swizzle UMMA shared-memory descriptor: core matrices of 8 rows
// x 16 bytes stored contiguously; lbo = bytes between the two 16-byte halves
// of a k32 step, sbo = bytes between consecutive 8-row groups.
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  cute::UMMA::SmemDescriptor d;
  d.desc_ = 0;
  d.start_address_ = (uint16_t)((saddr >> 4) & 0x3FFF);
  d.leading_byte_offset_ = (uint16_t)((lbo >> 4) & 0x3FFF);
  d.stride_byte_offset_ = (uint16_t)((sbo >> 4) & 0x3FFF);
  d.version_ = 1;
  d.base_offset_ = 0;
  d.lbo_mode_ = 0;
  d.layout_type_ = (uint8_t)cute::UMMA::LayoutType::SWIZZLE_NONE;
  return d.desc_;
}

template <int BN>
__host__ __device__ constexpr uint32_t oz_idesc() {
  // kind::i8: signed int8 A and B (K-major), int32 accumulator, M = 128, N = BN
  return (uint32_t)cute::UMMA::make_instr_desc<int8_t, int8_t, int32_t, OZ_BM, BN, cute::UMMA::Major::K,
                                               cute::UMMA::Major::K>();
}

__device__ __forceinline__ uint64_t oz_now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the mbarrier phase with the given parity; gives up after about
// two seconds of wall time (true: the phase completed).
__device__ __forceinline__ bool oz_wait(uint32_t mbar, uint32_t parity) {
  const uint64_t t0 = oz_now_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (oz_now_ns() - t0 > 2000000000ull) return false;
  }
}

template <int S, int BN>
__global__ void __launch_bounds__(128, 1) oz_gemm_kernel(OzGemmParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int A_CHUNK = OZ_BM * 16;          // bytes of one 16-byte K column of A (128 rows)
  constexpr int B_CHUNK = BN * 16;
  constexpr int A_SLICE = A_CHUNK * (OZ_KC / 16);
  constexpr int B_SLICE = B_CHUNK * (OZ_KC / 16);
  constexpr int TMEM_COLS = 256;
  static_assert(S * BN <= TMEM_COLS, "diagonal accumulators exceed the TMEM allocation");
  uint8_t *As = smem;
  uint8_t *Bs = smem + S * A_SLICE;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_sh;
  __shared__ int item_sh, bad_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
    bad_sh = 0;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_sh;
  const uint32_t mb = smem_u32(&mbar);
  const uint32_t idesc = oz_idesc<BN>();
  uint32_t phase = 0;

  for (;;) {
    if (tid == 0) item_sh = (int)atomicAdd(p.counter, 1u);
    __syncthreads();
    const int it = item_sh;
    if (it >= p.nitems || bad_sh) break;
    const OzItem item = p.items[it];
    const OzGroup g = p.groups[item.group];
    const int nrows = min(OZ_BM, g.row_end - g.row_begin - item.row0);
    const int ncols = min(BN, g.N - item.n0);
    for (int kc = 0; kc < g.K_pad; kc += OZ_KC) {
      const int kb = min(OZ_KC, g.K_pad - kc), nch = kb / 16;
      for (int idx = tid; idx < S * OZ_BM * nch; idx += blockDim.x) {
        const int c = idx % nch, r = (idx / nch) % OZ_BM, sl = idx / (nch * OZ_BM);
        const uint32_t dst = smem_u32(As) + sl * A_SLICE + c * A_CHUNK + (r >> 3) * 128 + (r & 7) * 16;
        const int8_t *src = p.dyn_pack;
        uint32_t bytes = 0;
        if (r < nrows) {
          const OzRow &R = p.rows[g.row_begin + item.row0 + r];
          src = p.dyn_pack + R.pack_off + (int64_t)sl * R.slice_stride + kc + c * 16;
          bytes = 16;
        }
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
      }
      for (int idx = tid; idx < S * BN * nch; idx += blockDim.x) {
        const int c = idx % nch, n = (idx / nch) % BN, sl = idx / (nch * BN);
        const uint32_t dst = smem_u32(Bs) + sl * B_SLICE + c * B_CHUNK + (n >> 3) * 128 + (n & 7) * 16;
        const int8_t *src = p.sta_pack;
        uint32_t bytes = 0;
        if (n < ncols) {
          src = p.sta_pack + g.s_pack_off + ((int64_t)sl * g.N + item.n0 + n) * g.K_pad + kc + c * 16;
          bytes = 16;
        }
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
      }
      asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        for (int ks = 0; ks < kb / 32; ++ks) {
#pragma unroll
          for (int pa = 1; pa <= S; ++pa)
#pragma unroll
            for (int qb = 1; pa + qb <= S + 1; ++qb) {
              const int d = pa + qb;
              const uint64_t da = oz_desc(smem_u32(As) + (pa - 1) * A_SLICE + ks * 2 * A_CHUNK, A_CHUNK, 128);
              const uint64_t db = oz_desc(smem_u32(Bs) + (qb - 1) * B_SLICE + ks * 2 * B_CHUNK, B_CHUNK, 128);
              const uint32_t dt = tmem + (uint32_t)((d - 2) * BN);
              // the first product of each diagonal in an item overwrites the accumulator
              const uint32_t acc = (kc > 0 || ks > 0 || pa > 1) ? 1u : 0u;
              asm volatile(
                  "{\n\t.reg .pred p;\n\t"
                  "setp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                  :
                  : "r"(dt), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                     : "memory");
      }
      if (!oz_wait(mb, phase)) {
        if (tid == 0) {
          bad_sh = 1;
          atomicExch(p.err, 1);
        }
        oz_wait(mb, phase);   // give the MMAs in flight one more bounded chance before TMEM is freed
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
      __syncthreads();
      if (bad_sh) break;
    }
    if (bad_sh) break;
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = stacked rows 32w..32w+31
    const int r = warp * 32 + lane;
    const bool rv = r < nrows;
    double rscale = 0.0;
    double *dst = nullptr;
    int32_t dstride = 0;
    if (rv) {
      const OzRow &R = p.rows[g.row_begin + item.row0 + r];
      rscale = R.coef * p.dyn_sig[R.sig_idx];
      dst = (R.dst_space == 0 ? p.out_scr : p.out_slots) + R.dst_off;
      dstride = R.dst_stride;
    }
#pragma unroll
    for (int j0 = 0; j0 < BN; j0 += 16) {
      uint32_t v[S][16];
#pragma unroll
      for (int d = 0; d < S; ++d) {
        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * BN + j0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[d][0]), "=r"(v[d][1]), "=r"(v[d][2]), "=r"(v[d][3]), "=r"(v[d][4]), "=r"(v[d][5]),
              "=r"(v[d][6]), "=r"(v[d][7]), "=r"(v[d][8]), "=r"(v[d][9]), "=r"(v[d][10]), "=r"(v[d][11]),
              "=r"(v[d][12]), "=r"(v[d][13]), "=r"(v[d][14]), "=r"(v[d][15])
            : "r"(ta));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (rv) {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const int n = j0 + jj;
          if (n < ncols) {
            double acc = 0.0;
#pragma unroll
            for (int d = S - 1; d >= 0; --d) acc = acc + ldexp((double)(int32_t)v[d][jj], -7 * (d + 2));
            dst[(int64_t)(item.n0 + n) * dstride] = acc * rscale * p.sta_sig[g.tau_off + item.n0 + n];
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// output cell = sum of task slots (in task order) + axpy terms
struct OzSumParams {
  const OzCellSum *sums;
  const int64_t *slot_offs;
  const double *slots;
  const Task *tasks;
  const double *ops, *psi, *scr;
  double *out;
};
__global__ void oz_sum_kernel(OzSumParams p) {
  const OzCellSum c = p.sums[blockIdx.x];
  for (int idx = threadIdx.x; idx < c.M * c.N; idx += blockDim.x) {
    const int i = idx % c.M, n = idx / c.M;
    double v = 0.0;
    for (int s = c.s_begin; s < c.s_end; ++s) v += p.slots[p.slot_offs[s] + (int64_t)n * c.M + i];
    for (int a = c.a_begin; a < c.a_end; ++a) {
      const Task &t = p.tasks[a];
      const double *b = t.L.space == SP_OPS ? p.ops : (t.L.space == SP_PSI ? p.psi : p.scr);
      v += t.coef * b[t.L.off + (int64_t)n * t.L.ld + i];
    }
    p.out[c.out_off + (int64_t)n * c.ld + i] = v;
  }
}

// ------------------------------------------------------------ host launches
void launch_oz_split(const OzSplit *jobs, int njobs, const double *ops, const double *psi, const double *scr,
                     int8_t *pack, double *sig, int s, cudaStream_t st) {
  if (njobs <= 0) return;
  OzSplitParams p{jobs, ops, psi, scr, pack, sig, s};
  oz_split_kernel<<<njobs, 256, 0, st>>>(p);
}

template <int S, int BN>
static cudaError_t launch_gemm_t(const OzGemmParams &p, int grid, cudaStream_t st) {
  // at least 100 KB per CTA keeps two CTAs per SM, so their 2 x 256 TMEM
  // columns never exceed the SM's 512 and no allocation has to wait
  size_t smem = (size_t)S * (OZ_BM + BN) * OZ_KC;
  if (smem < (100u << 10)) smem = 100u << 10;
  cudaError_t e = cudaFuncSetAttribute(oz_gemm_kernel<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  oz_gemm_kernel<S, BN><<<grid, 128, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_oz_gemm(const int8_t *dyn_pack, const double *dyn_sig, const int8_t *sta_pack,
                           const double *sta_sig, const OzGroup *groups, const OzRow *rows, const OzItem *items,
                           int nitems, double *out_scr, double *out_slots, unsigned int *counter, int *err, int s,
                           cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  OzGemmParams p{dyn_pack, dyn_sig, sta_pack, sta_sig, groups, rows, items, nitems, out_scr, out_slots, counter, err};
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nitems < 2 * sms ? nitems : 2 * sms;
  switch (s) {
    case 3: return launch_gemm_t<3, 48>(p, grid, st);
    case 4: return launch_gemm_t<4, 48>(p, grid, st);
    case 5: return launch_gemm_t<5, 48>(p, grid, st);
    case 6: return launch_gemm_t<6, 32>(p, grid, st);
    case 7: return launch_gemm_t<7, 32>(p, grid, st);
    case 8: return launch_gemm_t<8, 32>(p, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

void launch_oz_sum(const OzCellSum *sums, int nsums, const int64_t *slot_offs, const double *slots,
                   const Task *tasks, const double *ops, const double *psi, const double *scr, double *out,
                   cudaStream_t st) {
  if (nsums <= 0) return;
  OzSumParams p{sums, slot_offs, slots, tasks, ops, psi, scr, out};
  oz_sum_kernel<<<nsums, 256, 0, st>>>(p);
}

}  // namespace tjb
