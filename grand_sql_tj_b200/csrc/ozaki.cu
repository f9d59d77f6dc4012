// Device side of the split-precision H*psi (the scheme and the split layout
// are described in ozaki.h).
//
// oz_max_kernel    row maxima of the split jobs (atomic max on the scale pool)
// oz_split_kernel  scaled, truncated radix-128 digits in the tile-ready layout
// oz_gemm_kernel   persistent, warp-specialised tcgen05 kind::i8 GEMM:
//                    warp 4 (one lane)  bulk-copies the A and B digit blocks of
//                                       each k-block into a ring of smem stages
//                    warp 5 (one lane)  issues, per stage, the MMAs of every slice
//                                       pair p + q <= s + 1 into the TMEM
//                                       accumulator of diagonal p + q (two TMEM
//                                       buffers, one family each)
//                    warp 10            stages each item's scales and output
//                                       addresses in shared memory ahead of it
//                    warps 0-7          read the diagonals back (tcgen05.ld),
//                                       weight them by 128^-d, scale by the row
//                                       and column scales and add into the FP64
//                                       output tile (products: store P and raise
//                                       the pi scales)
//                  Every wait is bounded by wall time: on timeout the kernel
//                  raises *err, lets the other roles drop out, waits (bounded)
//                  for its copies and MMAs in flight, frees TMEM and returns.
//                  Where all lanes of a warp wait, the warp decides together.
#include <cuda_runtime.h>

#include <cstdint>

#include <cute/arch/mma_sm100_desc.hpp>

#include "kernels.cuh"
#include "ozaki.h"

namespace tjb {

// The power of two just above the row maximum m: 2^(E+1) for m = 1.f * 2^E
// (so every |x| <= m has |x| / 2^(E+1) < 1); 0 for m = 0.  Read off the
// exponent bits; m is finite and non-negative.
__device__ __forceinline__ double oz_pow2_of(double m) {
  if (!(m > 0.0)) return 0.0;
  const unsigned long long e = ((unsigned long long)__double_as_longlong(m) >> 52) & 0x7FFull;
  return __longlong_as_double((long long)((e == 0 ? 1ull : e + 1ull) << 52));
}

__device__ __forceinline__ const double *oz_space(int8_t sp, const double *ops, const double *psi,
                                                  const double *scr) {
  return sp == SP_OPS ? ops : (sp == SP_PSI ? psi : scr);
}

// ------------------------------------------------------------ split jobs
// The units of a job list (one unit = one row x 16 consecutive k of a job,
// rows padded to whole groups) are laid end to end and cut into CTAs of
// OZ_SPLIT_THREADS threads, one unit per thread.  Within a job consecutive
// threads take consecutive rows.
struct OzUnit {
  int job, r, c16;
};

__device__ __forceinline__ bool oz_unit(const OzJob *jobs, int njobs, const OzSpan *spans, OzUnit &u, OzJob &J) {
  const OzSpan sp = spans[blockIdx.x];
  int j = sp.job;
  int64_t k = (int64_t)sp.u0 + threadIdx.x;
  for (; j < njobs; ++j) {
    J = jobs[j];
    const int rows = J.gtot * 8, nk16 = (J.K + 31) / 32 * 2;
    const int64_t units = (int64_t)rows * nk16;
    if (k < units) {
      // consecutive threads: consecutive rows, so that the 16-byte digit rows
      // of a group land as whole 128-byte lines
      u.job = j;
      u.r = (int)(k % rows);
      u.c16 = (int)(k / rows);
      return true;
    }
    k -= units;
  }
  return false;
}

// Row maxima of |coef * M| (a list of maximum jobs): one unit = one row x
// OZ_MAX_CHUNK k, consecutive threads on consecutive rows, one atomic max
// per unit.  Jobs with want_max = 2 (a psi cell split both ways) also raise
// the column maxima, scales[dst + k]: their rows are padded to whole warps
// and they come first in the list, so a warp holds 32 rows of one job and
// one chunk, and each column's maximum is reduced across the warp and
// raised by one lane.
__global__ void __launch_bounds__(OZ_SPLIT_THREADS) oz_max_kernel(const OzJob *jobs, int njobs, const OzSpan *spans,
                                                                  const double *ops, const double *psi,
                                                                  const double *scr, double *scales, int *err) {
  const OzSpan sp = spans[blockIdx.x];
  int64_t k = (int64_t)sp.u0 + threadIdx.x;
  OzJob J;
  int r = -1, c = 0;
  for (int j = sp.job; j < njobs; ++j) {
    J = jobs[j];
    const int nc = (J.K + OZ_MAX_CHUNK - 1) / OZ_MAX_CHUNK;
    const int rows = J.want_max == 2 ? (J.nrows + 31) / 32 * 32 : J.nrows;
    const int64_t units = (int64_t)rows * nc;
    if (k < units) {
      r = (int)(k % rows);
      c = (int)(k / rows);
      break;
    }
    k -= units;
  }
  if (r < 0) return;
  const bool valid = r < J.nrows;
  const double *row = oz_space(J.space, ops, psi, scr) + J.src_off + (int64_t)(valid ? r : 0) * J.rs;
  // all OZ_MAX_CHUNK loads of the unit in flight at once (the kernel is bound
  // by the loads in flight, not by the instructions)
  const int k0 = c * OZ_MAX_CHUNK;
  double x[OZ_MAX_CHUNK];
#pragma unroll
  for (int q = 0; q < OZ_MAX_CHUNK; ++q) x[q] = valid && k0 + q < J.K ? fabs(row[(int64_t)(k0 + q) * J.ks]) : 0.0;
  // a NaN or an infinity cannot be split (its scale and digits are undefined):
  // the host reports it instead of returning a silently wrong product
  bool bad = false;
#pragma unroll
  for (int q = 0; q < OZ_MAX_CHUNK; ++q) bad |= !isfinite(x[q]);
  if (bad) atomicOr(err, 2);
  if (J.want_max == 2) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < OZ_MAX_CHUNK; ++q) {
      double cm = x[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, o));
      cm *= fabs(J.coef);
      if (lane == q && k0 + q < J.K && cm > 0.0)
        atomicMax((unsigned long long *)&scales[J.dst + k0 + q], (unsigned long long)__double_as_longlong(cm));
    }
  }
#pragma unroll
  for (int w = OZ_MAX_CHUNK / 2; w > 0; w >>= 1)
#pragma unroll
    for (int q = 0; q < w; ++q) x[q] = fmax(x[q], x[q + w]);
  const double m = fabs(J.coef) * x[0];
  if (valid && m > 0.0)
    atomicMax((unsigned long long *)&scales[J.scale_idx + r], (unsigned long long)__double_as_longlong(m));
}

// The radix-128 digits of y (|y| < 1) truncated toward zero -- digit q is
// sign(y) * (floor(|y| * 128^(q+1)) mod 128), what S rounds of "multiply by
// 128, truncate, subtract" give (every step of those is exact) -- are the
// 7-bit groups of F = floor(|y| * 2^(7S)) with the sign of y.  F comes from
// one truncating conversion (|y| * 2^(7S) is exact: a power-of-two scaling),
// the groups are packed four elements to a word per slice, and the words of
// negative elements are negated bytewise at the end: (w ^ m) - m per byte,
// m = 0xFF in the bytes of negative elements.  Non-finite inputs give 0.
// Scaled, truncated radix-128 digits: s 16-byte digit rows per unit.
template <int S>
__global__ void __launch_bounds__(OZ_SPLIT_THREADS) oz_split_kernel(const OzJob *jobs, int njobs, const OzSpan *spans,
                                                                    const double *ops, const double *psi,
                                                                    const double *scr, const double *scales,
                                                                    uint8_t *pack) {
  OzUnit u;
  OzJob J;
  if (!oz_unit(jobs, njobs, spans, u, J)) return;
  const int r = u.r, c16 = u.c16;
  uint32_t dig[S][4];
#pragma unroll
  for (int q = 0; q < S; ++q) dig[q][0] = dig[q][1] = dig[q][2] = dig[q][3] = 0u;
  if (r < J.nrows) {
    const double sc = oz_pow2_of(scales[J.scale_idx + r]);
    if (sc > 0.0) {
      const double inv = 1.0 / sc;   // exact: sc is a power of two
      const double *row = oz_space(J.space, ops, psi, scr) + J.src_off + (int64_t)r * J.rs;
      double x[16];
#pragma unroll
      for (int kk = 0; kk < 16; ++kk) {
        const int k = c16 * 16 + kk;
        x[kk] = k < J.K ? row[(int64_t)k * J.ks] : 0.0;
      }
      constexpr double P2 = (double)(1ull << (7 * S));
      uint32_t negm[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int kk = 0; kk < 16; ++kk) {
        const double t = (J.coef * x[kk]) * inv;
        const double a = fabs(t);
        const uint64_t f = a < 1.0 ? __double2ull_rz(a * P2) : 0ull;
        if (__double_as_longlong(t) < 0) negm[kk >> 2] |= 0xFFu << (8 * (kk & 3));
#pragma unroll
        for (int q = 0; q < S; ++q)
          dig[q][kk >> 2] |= ((uint32_t)(f >> (7 * (S - 1 - q))) & 127u) << (8 * (kk & 3));
      }
#pragma unroll
      for (int q = 0; q < S; ++q)
#pragma unroll
        for (int w = 0; w < 4; ++w) dig[q][w] = __vsub4(dig[q][w] ^ negm[w], negm[w]);
    }
  }
  // split row -> tile, group within the tile
  const int sr = J.row0 + r;
  const int t = sr / J.R, rl = sr - t * J.R;
  const int gt = t < J.ntiles - 1 ? J.R / 8 : J.gt_last;
  const int kb = c16 >> 1, c = c16 & 1, g = rl >> 3, r8 = rl & 7;
  const int64_t plane = (int64_t)gt * 256;   // bytes of one slice of one k-block of the tile
  uint8_t *dst = pack + J.dst + (int64_t)t * J.nkb * S * (J.R / 8) * 256 + ((int64_t)(J.kb0 + kb) * S * gt + g) * 256 +
                 c * 128 + r8 * 16;
#pragma unroll
  for (int q = 0; q < S; ++q)
    *reinterpret_cast<uint4 *>(dst + q * plane) = make_uint4(dig[q][0], dig[q][1], dig[q][2], dig[q][3]);
}

// ------------------------------------------------------------ tcgen05 GEMM
struct OzGemmParams {
  const OzItem *items;
  const int32_t *cta;   // CTA b runs items [cta[b], cta[b+1])
  const OzSeg *segs;
  const OzFam *fams;
  const OzCell *cells;
  const OzStackRow *srows;
  const Task *tasks;
  const uint8_t *pack;
  double *scales;
  const double *psi;
  double *scr, *out;
  int *err;
  uint64_t wait_ns;   // limit of the pipeline's waits
};

__device__ __forceinline__ uint32_t oz_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t oz_now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr uint64_t OZ_WAIT_NS = 2000000000ull;

__device__ __forceinline__ bool oz_try(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of the given parity; false after limit_ns or when
// another role has aborted (*abort != 0).  The clock is read only once the
// first try has failed (a phase that has already completed costs one try).
// The pipeline's waits use the caller's limit (OzGemmParams::wait_ns); the
// drain waits before the CTA exits always use OZ_WAIT_NS, so that no CTA
// leaves with bulk copies or MMAs in flight.
__device__ __forceinline__ bool oz_wait(uint32_t mbar, uint32_t parity, volatile int *abort,
                                        uint64_t limit_ns = OZ_WAIT_NS) {
  if (oz_try(mbar, parity)) return true;
  const uint64_t t0 = oz_now_ns();
  for (;;) {
    if (oz_try(mbar, parity)) return true;
    if (abort && *abort) return false;
    if (oz_now_ns() - t0 > limit_ns) return false;
  }
}

// *err bits: 1 a bounded wait gave up, 2 a non-finite value entered a split
__device__ __forceinline__ void oz_fail(volatile int *abort, int *err) {
  *abort = 1;
  atomicOr(err, 1);
}

// K-major, no-swizzle UMMA shared-memory descriptor (core matrices of 8 rows x
// 16 bytes; lbo = bytes between the two K halves, sbo = bytes between groups).
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

// kind::i8 instruction descriptor: signed int8 A and B (K-major), int32 D, M x N.
__device__ __forceinline__ uint32_t oz_idesc(int M, int N) {
  cute::UMMA::InstrDescriptor d =
      cute::UMMA::make_instr_desc<int8_t, int8_t, int32_t, 128, 64, cute::UMMA::Major::K, cute::UMMA::Major::K>();
  d.m_dim_ = (uint8_t)(M >> 4);
  d.n_dim_ = (uint8_t)(N >> 3);
  return (uint32_t)d;
}

__device__ __forceinline__ void oz_bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

__device__ __forceinline__ void oz_arrive_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void oz_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void oz_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// k-blocks per pipeline stage (up to 5 slices) and the shared memory given to
// the stages
// (build-time settings; the defaults are the measured best)
#ifndef OZ_KPS
#define OZ_KPS 2
#endif
#ifndef OZ_STAGE_CAP
#define OZ_STAGE_CAP (192 * 1024)
#endif

template <int S, int BN>
struct OzCfg {
  // a stage holds KPS consecutive k-blocks of an item's family: the cost of a
  // stage (barriers, copies, MMA issue) is nearly fixed, so fewer, larger
  // stages go faster
  static constexpr int KPS = S <= 5 ? OZ_KPS : 2;
  static constexpr int A_KB = S * 16 * 256;             // one k-block: 128 rows x 32 k, s slices
  static constexpr int B_KB = S * (BN / 8) * 256;
  static constexpr int A_BYTES = KPS * A_KB;
  static constexpr int B_BYTES = KPS * B_KB;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int STAGES_RAW = (OZ_STAGE_CAP) / STAGE;
  static constexpr int STAGES = STAGES_RAW > 8 ? 8 : STAGES_RAW;
  static constexpr int SMEM = STAGES * STAGE;
  static_assert(S * BN <= 256, "diagonal accumulators exceed one TMEM buffer");
  // k-blocks one TMEM accumulation may take: a diagonal sums at most S slice
  // products of 127^2 per k, and must stay below 2^31; longer families are
  // accumulated in pieces and the pieces added in FP64
  static constexpr int KB_PIECE = (int)(2147483647LL / (32LL * S * 127 * 127)) / KPS * KPS;
  static_assert(STAGES >= 2, "too few pipeline stages");
};

// Per-item data of the epilogue, staged in shared memory by the metadata warp
// ahead of the item's accumulators: power-of-two column scales and row scales
// of each family (at most two per item), the output tile and the axpy terms.
constexpr int OZ_META = 4;       // ring slots
constexpr int OZ_META_AX = 4;    // axpy terms held per cell (more are read from global memory)
template <int BN>
struct OzMeta {
  double cs[OZ_MAX_FAM][BN];
  double rs[OZ_MAX_FAM][128];
  int32_t npiece[OZ_MAX_FAM];    // accumulations of each family (pieces of at most OzCfg::KB_PIECE k-blocks)
  int64_t c_off;                 // offset of the tile's (row0, col0) in out (cells) or scr (products)
  int32_t c_ld, na;              // cells: leading dimension; axpy terms (init items)
  double ax_coef[OZ_META_AX];
  int64_t ax_off[OZ_META_AX];    // psi offset of the axpy operand's (row0, col0)
  int32_t ax_ld[OZ_META_AX];
  // product stacks (kind 1): per tile row, the product-space offset of its
  // column 0 (-1: a padding row of the stack), its column stride and its pi
  int64_t row_off[128];
  int64_t row_pi[128];
  int32_t row_ld[128];
};

// 8 epilogue warps (two column halves of the tile x four TMEM lane quarters),
// then the producer warp, the MMA warp and the metadata warp
constexpr int OZ_EPI_THREADS = 256, OZ_GEMM_THREADS = OZ_EPI_THREADS + 96;

template <int S, int BN>
__global__ void __launch_bounds__(OZ_GEMM_THREADS, 1) oz_gemm_kernel(OzGemmParams p) {
  using C = OzCfg<S, BN>;
  constexpr int ST = C::STAGES;
  constexpr uint32_t GB = S * 256;   // bytes of one row group (all slices) of one k-block
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t full_bar[ST], empty_bar[ST], tfull_bar[2], tempty_bar[2], drain_bar;
  __shared__ uint32_t tmem_sh;
  __shared__ volatile int abort_sh;
  __shared__ volatile int tfull_ok_sh;
  // this CTA's first OZ_ICACHE items (and the segment of each product item),
  // so that no role waits on a global load at an item boundary
  constexpr int OZ_ICACHE = 64;
  __shared__ OzItem item_sh[OZ_ICACHE];
  __shared__ OzMeta<BN> meta[OZ_META];
  __shared__ __align__(8) uint64_t meta_full[OZ_META], meta_empty[OZ_META];
  static_assert(C::SMEM + sizeof(OzMeta<BN>) * OZ_META + OZ_ICACHE * sizeof(OzItem) + 2048 <=
                    232448,
                "shared memory above 227 KB");
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int i = 0; i < ST; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&full_bar[i])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&empty_bar[i])), "r"(1));
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&tfull_bar[i])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&tempty_bar[i])), "r"(OZ_EPI_THREADS));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&drain_bar)), "r"(1));
    for (int i = 0; i < OZ_META; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&meta_full[i])), "r"(32));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(&meta_empty[i])), "r"(OZ_EPI_THREADS));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_sh = 0;
  }
  const int ib = p.cta[blockIdx.x], ie_cta = p.cta[blockIdx.x + 1];
  for (int i = tid; i < min(ie_cta - ib, OZ_ICACHE); i += blockDim.x) item_sh[i] = p.items[ib + i];
  auto get_item = [&](int ii) -> OzItem { return ii - ib < OZ_ICACHE ? item_sh[ii - ib] : p.items[ii]; };
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tmem_sh)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_sh;
  const uint32_t smem0 = oz_smem(smem);

  if (warp == OZ_EPI_THREADS / 32) {
    // ------------------------------------------------ producer (whole warp; lane 0 owns the barriers)
    int stage = 0;
    uint32_t ph = 0;
    uint32_t armed = 0, armed_ph = 0;   // bit i: stage i armed, and the parity of its last arming
    bool ok = true;
    // lane 0 waits for a free stage and arms it with `bytes`; every lane learns the outcome
    auto acquire = [&](uint32_t bytes) -> bool {
      int good = 1;
      if (lane == 0) {
        if (!oz_wait(oz_smem(&empty_bar[stage]), ph ^ 1u, &abort_sh, p.wait_ns)) {
          if (!abort_sh) oz_fail(&abort_sh, p.err);
          good = 0;
        } else {
          oz_arrive_expect(oz_smem(&full_bar[stage]), bytes);
        }
      }
      good = __shfl_sync(0xffffffffu, good, 0);
      if (good) {
        armed |= 1u << stage;
        armed_ph = (armed_ph & ~(1u << stage)) | (ph << stage);
      }
      __syncwarp();
      return good != 0;
    };
    for (int ii = p.cta[blockIdx.x], ie = p.cta[blockIdx.x + 1]; ii < ie && ok; ++ii) {
      const OzItem it = get_item(ii);
      // tiles of this item: A row tile ta (ga groups), B column tile tb (gb groups)
      const uint32_t ga = (uint32_t)((it.mrows + 7) >> 3), gb = (uint32_t)(it.N >> 3);
      const int64_t ta = it.row0 / 128, tb = it.col0 / BN;
      const uint32_t bytes1 = (ga + gb) * GB;   // one k-block of both operands
      for (int f = it.fam_begin; f < it.fam_end && ok; ++f) {
        const OzFam fm = p.fams[f];
        const int sb = fm.seg_begin, se = fm.seg_end;
        // the family's k-blocks, segment after segment, fill stages of up to
        // KPS k-blocks (a stage may hold the end of one segment and the start
        // of the next; stage boundaries fall every KPS k-blocks of the family)
        int done = 0, in_stage = 0;
        uint32_t sa = 0, sbb = 0, fbar = 0;
        for (int s0 = sb; s0 < se && ok; s0 += 32) {
          // the next <= 32 segments, one per lane
          OzSeg mine;
          if (s0 + lane < se) mine = p.segs[s0 + lane];
          const int cnt = min(32, se - s0);
          for (int j = 0; j < cnt && ok; ++j) {
            const int64_t a_base = __shfl_sync(0xffffffffu, mine.a_base, j);
            const int64_t b_base = __shfl_sync(0xffffffffu, mine.b_base, j);
            const int32_t a_nkb = __shfl_sync(0xffffffffu, mine.a_nkb, j);
            const int32_t b_nkb = __shfl_sync(0xffffffffu, mine.b_nkb, j);
            const int32_t a_kb0 = __shfl_sync(0xffffffffu, mine.a_kb0, j);
            const int32_t b_kb0 = __shfl_sync(0xffffffffu, mine.b_kb0, j);
            const int32_t nkb = __shfl_sync(0xffffffffu, mine.nkb, j);
            const uint8_t *asrc = p.pack + a_base + ta * a_nkb * (int64_t)(16 * GB) + (int64_t)a_kb0 * ga * GB;
            const uint8_t *bsrc = p.pack + b_base + tb * b_nkb * (int64_t)((BN / 8) * GB) + (int64_t)b_kb0 * gb * GB;
            for (int kb = 0; kb < nkb;) {
              if (in_stage == 0) {
                const int n = min(C::KPS, fm.nkb - done);
                if (!acquire((uint32_t)n * bytes1)) {
                  ok = false;
                  break;
                }
                sa = smem0 + (uint32_t)(stage * C::STAGE);
                sbb = sa + C::A_BYTES;
                fbar = oz_smem(&full_bar[stage]);
              }
              // the k-blocks of this segment that go into the current stage are
              // contiguous in the split and in the stage: one copy per operand
              const int take = min(nkb - kb, C::KPS - in_stage);
              if (lane == 0)
                oz_bulk_g2s(sa + in_stage * ga * GB, asrc + (int64_t)kb * ga * GB, (uint32_t)take * ga * GB, fbar);
              if (lane == 1)
                oz_bulk_g2s(sbb + in_stage * gb * GB, bsrc + (int64_t)kb * gb * GB, (uint32_t)take * gb * GB, fbar);
              kb += take;
              done += take;
              in_stage += take;
              if (in_stage == C::KPS || done == fm.nkb) {
                in_stage = 0;
                if (++stage == ST) stage = 0, ph ^= 1u;
              }
            }
          }
        }
      }
    }
    // copies still in flight land before the CTA exits
    if (lane == 0)
      for (int i = 0; i < ST; ++i)
        if (armed & (1u << i)) oz_wait(oz_smem(&full_bar[i]), (armed_ph >> i) & 1u, nullptr);
    __syncwarp();
  } else if (warp == OZ_EPI_THREADS / 32 + 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      int stage = 0;
      uint32_t ph = 0;
      uint32_t famc = 0;
      bool ok = true, issued = false;
      const uint64_t dbase = oz_desc(0u, 128u, 256u);   // start address added per stage
      for (int ii = p.cta[blockIdx.x], ie = p.cta[blockIdx.x + 1]; ii < ie && ok; ++ii) {
        const OzItem it = get_item(ii);
        // MMA pa multiplies A slice pa with B slices 1..S+1-pa (N' = (S+1-pa) N):
        // its column block q lands on the accumulator of diagonal pa+q at column (pa+q-2) N
        uint32_t idesc[S];
#pragma unroll
        for (int pa = 1; pa <= S; ++pa) idesc[pa - 1] = oz_idesc(it.M, (S + 1 - pa) * it.N);
        const uint32_t aslice16 = (uint32_t)((it.mrows + 7) >> 3) * 16u;   // A slice stride in 16-byte units
        const uint32_t ga_gb = (uint32_t)((it.mrows + 7) >> 3) * GB;       // bytes of one A k-block
        const uint32_t gb_gb = (uint32_t)(it.N >> 3) * GB;                 // bytes of one B k-block
        const int nf = it.fam_end - it.fam_begin;
        for (int f = 0; f < nf && ok; ++f) {
          const int nkb_f = p.fams[it.fam_begin + f].nkb;
          for (int k0 = 0; k0 < nkb_f && ok; k0 += C::KB_PIECE) {
          const int nkb = min(C::KB_PIECE, nkb_f - k0);
          const uint32_t buf = famc & 1u, use = famc >> 1;
          if (!oz_wait(oz_smem(&tempty_bar[buf]), (use & 1u) ^ 1u, &abort_sh, p.wait_ns)) {
            if (!abort_sh) oz_fail(&abort_sh, p.err);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t dt = tmem + buf * 256u;
          for (int kb = 0; kb < nkb; kb += C::KPS) {
            if (!oz_wait(oz_smem(&full_bar[stage]), ph, &abort_sh, p.wait_ns)) {
              if (!abort_sh) oz_fail(&abort_sh, p.err);
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t sa = smem0 + (uint32_t)(stage * C::STAGE);
            const int n = min(C::KPS, nkb - kb);   // k-blocks in this stage
            for (int j = 0; j < n; ++j) {
              // k-block j of the stage: A at sa + j ga GB, B at sa + A_BYTES + j gb GB
              const uint64_t da0 = dbase + (uint64_t)((sa + (uint32_t)j * ga_gb) >> 4);
              const uint64_t db = dbase + (uint64_t)((sa + C::A_BYTES + (uint32_t)j * gb_gb) >> 4);
#pragma unroll
              for (int pa = 1; pa <= S; ++pa) {
                const uint64_t da = da0 + (uint64_t)((pa - 1) * aslice16);   // A slices ga groups apart
                const uint32_t d = dt + (uint32_t)((pa - 1) * it.N);
                const uint32_t acc = (kb == 0 && j == 0 && pa == 1) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :
                    : "r"(d), "l"(da), "l"(db), "r"(idesc[pa - 1]), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
              }
            }
            issued = true;
            oz_commit(oz_smem(&empty_bar[stage]));   // frees the stage when these MMAs finish
            if (++stage == ST) stage = 0, ph ^= 1u;
          }
          if (!ok) break;
          oz_commit(oz_smem(&tfull_bar[buf]));
          ++famc;
          }
        }
      }
      if (issued) {
        // every MMA issued so far has finished before TMEM is released
        oz_commit(oz_smem(&drain_bar));
        oz_wait(oz_smem(&drain_bar), 0u, nullptr);
      }
    }
    __syncwarp();
  } else if (warp == OZ_EPI_THREADS / 32 + 2) {
    // ------------------------------------------------ metadata (whole warp): one ring slot per item
    // An item's static records (its families, its cell) are loaded one item
    // ahead, and all of its own loads (the families' scales, the stack rows
    // or the axpy terms) are issued before its ring slot is waited for, so
    // that an item costs about one round of global loads, not a chain.
    constexpr int CQ = (BN + 31) / 32, RQ = 128 / 32;   // loads per lane: columns, rows
    struct FamS { int64_t rs, cs; int32_t nkb; };
    struct CellS { int64_t off; int32_t ld, a_begin, a_end; };
    FamS fn[OZ_MAX_FAM];
    CellS cn;
    auto load_static = [&](int ii) {
      const OzItem it = get_item(ii);
      const int nf = it.fam_end - it.fam_begin;
#pragma unroll
      for (int f = 0; f < OZ_MAX_FAM; ++f)
        if (f < nf) {
          const OzFam fm = p.fams[it.fam_begin + f];
          fn[f] = FamS{fm.rs_idx, fm.cs_idx, fm.nkb};
        }
      const OzCell c = p.cells[it.cell];
      cn = CellS{c.off, c.ld, c.a_begin, c.a_end};
    };
    if (ib < ie_cta) load_static(ib);
    uint32_t icount = 0;
    for (int ii = ib; ii < ie_cta; ++ii, ++icount) {
      const OzItem it = get_item(ii);
      FamS fc[OZ_MAX_FAM];
#pragma unroll
      for (int f = 0; f < OZ_MAX_FAM; ++f) fc[f] = fn[f];
      const CellS c = cn;
      if (ii + 1 < ie_cta) load_static(ii + 1);
      const int nf = it.fam_end - it.fam_begin;   // at most OZ_MAX_FAM (checked by the plan)
      const int na = it.init ? c.a_end - c.a_begin : 0;
      double csv[OZ_MAX_FAM][CQ], rsv[OZ_MAX_FAM][RQ];
#pragma unroll
      for (int f = 0; f < OZ_MAX_FAM; ++f) {
#pragma unroll
        for (int q = 0; q < CQ; ++q) {
          const int j = lane + 32 * q;
          csv[f][q] = f < nf && j < it.ncols ? p.scales[fc[f].cs + it.col0 + j] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
          const int r = lane + 32 * q;
          rsv[f][q] = f < nf && r < it.mrows ? p.scales[fc[f].rs + it.row0 + r] : 0.0;
        }
      }
      Task tk;
      if (lane < min(na, OZ_META_AX)) tk = p.tasks[c.a_begin + lane];
      OzStackRow sr[RQ];
#pragma unroll
      for (int q = 0; q < RQ; ++q) {
        const int r = lane + 32 * q;
        sr[q] = OzStackRow{-1, 0, 0, 0};
        if (it.kind == 1 && r < it.mrows) sr[q] = p.srows[c.off + it.row0 + r];
      }
      const int slot = (int)(icount % OZ_META);
      int good = 1;
      if (lane == 0 && !oz_wait(oz_smem(&meta_empty[slot]), ((icount / OZ_META) & 1u) ^ 1u, &abort_sh, p.wait_ns)) {
        if (!abort_sh) oz_fail(&abort_sh, p.err);
        good = 0;
      }
      if (!__shfl_sync(0xffffffffu, good, 0)) break;
      OzMeta<BN> &m = meta[slot];
#pragma unroll
      for (int f = 0; f < OZ_MAX_FAM; ++f) {
        if (f < nf) {
          if (lane == 0) m.npiece[f] = (fc[f].nkb + C::KB_PIECE - 1) / C::KB_PIECE;
#pragma unroll
          for (int q = 0; q < CQ; ++q)
            if (lane + 32 * q < it.ncols) m.cs[f][lane + 32 * q] = oz_pow2_of(csv[f][q]);
#pragma unroll
          for (int q = 0; q < RQ; ++q)
            if (lane + 32 * q < it.mrows) m.rs[f][lane + 32 * q] = oz_pow2_of(rsv[f][q]);
        }
      }
      if (lane == 0) {
        m.c_off = c.off + it.row0 + (int64_t)it.col0 * c.ld;
        m.c_ld = c.ld;
        m.na = na;
      }
      if (lane < min(na, OZ_META_AX)) {
        m.ax_coef[lane] = tk.coef;
        m.ax_off[lane] = tk.L.off + (int64_t)it.col0 * tk.L.ld + it.row0;
        m.ax_ld[lane] = tk.L.ld;
      }
      if (it.kind == 1) {
        // a product stack: tile row r is stack row row0 + r, whose product
        // the stack-row table names
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
          const int r = lane + 32 * q;
          m.row_off[r] = sr[q].off >= 0 ? sr[q].off + (int64_t)it.col0 * sr[q].ld : -1;
          m.row_pi[r] = sr[q].pi;
          m.row_ld[r] = sr[q].ld;
        }
      }
      oz_arrive(oz_smem(&meta_full[slot]));   // every lane: release of its own writes
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ epilogue (warps 0-7, named barrier 1)
    uint32_t famc = 0, icount = 0;
    // diagonal d carries weight 128^-(d+2).  The diagonals are combined
    // exactly in 64-bit integers, in groups of at most five (|D_d| < 2^31, so
    // a group sum_d D_d 128^(g1-1-d) stays below 2^59), and each group is
    // converted once: weight of the group ending at g1 is 128^-(g1+1)
    constexpr int NG = (S + 4) / 5;
    double wg[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      const int g1 = min(S, 5 * g + 5);
      double x = 1.0;
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (i <= g1) x *= 1.0 / 128.0;
      wg[g] = x;
    }
    bool ok = true;
    constexpr int HCH = (BN / 8 + 1) / 2;   // most 8-column chunks of a half
    for (int ii = ib; ii < ie_cta && ok; ++ii, ++icount) {
      const OzItem it = get_item(ii);
      // warp w reads TMEM lane quarter q = w % 4 (lanes 32q..32q+31) and
      // column half h = w / 4 of the tile; the tile row it holds:
      //   M = 128: row = 32q + lane; M = 64: rows 16q..16q+15 in lanes 32q..32q+15
      const int quarter = warp & 3, half = warp >> 2;
      int r;
      bool rv;
      if (it.M == 128) {
        r = quarter * 32 + lane;
        rv = r < it.mrows;
      } else {
        r = quarter * 16 + lane;
        rv = lane < 16 && r < it.mrows;
      }
      // this half's 8-column chunks: [c0, c0 + nchh)
      const int nch = it.N >> 3, hch = (nch + 1) >> 1;
      const int c0 = half * hch, nchh = min(hch, nch - c0);
      const int nf = it.fam_end - it.fam_begin;
      const int slot = (int)(icount % OZ_META);
      // every lane waits (acquiring the slot's data) and the warp decides
      // together, so that the warp-collective TMEM reads below are never
      // reached by part of a warp
      if (!__all_sync(0xffffffffu, oz_wait(oz_smem(&meta_full[slot]), (icount / OZ_META) & 1u, &abort_sh,
                                           p.wait_ns))) {
        if (!abort_sh) oz_fail(&abort_sh, p.err);
        ok = false;
        break;
      }
      const OzMeta<BN> &m = meta[slot];
      // the tile row's destination: an H*psi cell, or (product stacks) the
      // product the row belongs to (none for the stack's padding rows)
      double *dst;
      int64_t cstride, pi_r = 0;
      if (it.kind == 1) {
        const int64_t ro = rv ? m.row_off[r] : -1;
        rv = ro >= 0;
        dst = p.scr + (rv ? ro : 0);
        cstride = rv ? m.row_ld[r] : 0;
        pi_r = rv ? m.row_pi[r] : 0;
      } else {
        dst = p.out + m.c_off + r;
        cstride = m.c_ld;
      }
      // the values the tile is added to, loaded before the accumulators are
      // waited for: the old H*psi (cells of launch 2) or the axpy terms (init)
      double old[HCH * 8];
#pragma unroll
      for (int j = 0; j < HCH * 8; ++j) old[j] = 0.0;
      if (it.kind == 0) {
        const int na = m.na;
        if (rv) {
#pragma unroll
          for (int cl = 0; cl < HCH; ++cl) {
            const int col = (c0 + cl) * 8;
            if (cl < nchh) {
#pragma unroll
              for (int jj = 0; jj < 8; ++jj) {
                const int n = col + jj;
                if (n < it.ncols) {
                  if (!it.init) {
                    old[cl * 8 + jj] = dst[(int64_t)n * cstride];
                  } else {
                    double a0 = 0.0;
                    for (int a = 0; a < min(na, OZ_META_AX); ++a)
                      a0 += m.ax_coef[a] * p.psi[m.ax_off[a] + (int64_t)n * m.ax_ld[a] + r];
                    old[cl * 8 + jj] = a0;
                  }
                }
              }
            }
          }
          if (it.init && na > OZ_META_AX) {
            const OzCell c = p.cells[it.cell];
            for (int a = c.a_begin + OZ_META_AX; a < c.a_end; ++a) {
              const Task t = p.tasks[a];
#pragma unroll
              for (int cl = 0; cl < HCH; ++cl) {
                const int col = (c0 + cl) * 8;
                if (cl < nchh)
#pragma unroll
                  for (int jj = 0; jj < 8; ++jj)
                    if (col + jj < it.ncols)
                      old[cl * 8 + jj] +=
                          t.coef * p.psi[t.L.off + (int64_t)(it.col0 + col + jj) * t.L.ld + it.row0 + r];
              }
            }
          }
        }
      }
      // this half of the tile row, summed over the item's families
      double accv[HCH * 8];
#pragma unroll
      for (int j = 0; j < HCH * 8; ++j) accv[j] = 0.0;
      for (int f = 0; f < nf && ok; ++f)
      for (int pc = 0; pc < m.npiece[f]; ++pc) {
        const uint32_t buf = famc & 1u, use = famc >> 1;
        const double rscale = rv ? m.rs[f][r] : 0.0;
        if (!__all_sync(0xffffffffu, oz_wait(oz_smem(&tfull_bar[buf]), use & 1u, &abort_sh, p.wait_ns))) {
          if (!abort_sh) oz_fail(&abort_sh, p.err);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
        for (int cl = 0; cl < HCH; ++cl) {
          if (cl < nchh) {
            const int col = (c0 + cl) * 8;
            uint32_t v[S][8];
#pragma unroll
            for (int d = 0; d < S; ++d) {
              const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + buf * 256u + (uint32_t)(d * it.N + col);
              asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                           : "=r"(v[d][0]), "=r"(v[d][1]), "=r"(v[d][2]), "=r"(v[d][3]), "=r"(v[d][4]),
                             "=r"(v[d][5]), "=r"(v[d][6]), "=r"(v[d][7])
                           : "r"(ta));
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              double acc = 0.0;
#pragma unroll
              for (int g = 0; g < NG; ++g) {
                long long q = 0;
#pragma unroll
                for (int d = 5 * g; d < min(S, 5 * g + 5); ++d) q = q * 128 + (long long)(int32_t)v[d][jj];
                acc += (double)q * wg[g];
              }
              accv[cl * 8 + jj] += acc * rscale * m.cs[f][min(col + jj, BN - 1)];
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        oz_arrive(oz_smem(&tempty_bar[buf]));
        ++famc;
      }
      if (!ok) break;
      oz_arrive(oz_smem(&meta_empty[slot]));   // the slot's data is in registers now
      // store this half of the tile row (products: and raise pi with the row's maximum)
      double rmax = 0.0;
#pragma unroll
      for (int cl = 0; cl < HCH; ++cl) {
        const int col = (c0 + cl) * 8;
        if (rv && cl < nchh) {
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int n = col + jj;
            if (n < it.ncols) {
              const double v = old[cl * 8 + jj] + accv[cl * 8 + jj];
              dst[(int64_t)n * cstride] = v;
              rmax = fmax(rmax, fabs(v));
            }
          }
        }
      }
      if (it.kind == 1 && rv && rmax > 0.0)
        atomicMax((unsigned long long *)&p.scales[pi_r], (unsigned long long)__double_as_longlong(rmax));
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

// The stack-row table: one CTA per cell; a product stack's products write
// their rows (the table was set to 0xFF bytes, off = -1, for padding rows).
__global__ void oz_stack_rows_kernel(const OzCell *cells, const OzProdRow *prows, OzStackRow *srows) {
  const OzCell c = cells[blockIdx.x];
  if (c.ld != 0 || c.a_end <= c.a_begin) return;   // not a product stack
  for (int k = c.a_begin; k < c.a_end; ++k) {
    const OzProdRow pr = prows[k];
    for (int r = threadIdx.x; r < pr.rows; r += blockDim.x)
      srows[c.off + pr.row_begin + r] = OzStackRow{pr.off + r, pr.pi + r, pr.ld, 0};
  }
}

// ------------------------------------------------------------ host launches
void launch_oz_stack_rows(const OzCell *cells, int ncells, const OzProdRow *prows, OzStackRow *srows, int64_t n,
                          cudaStream_t st) {
  if (ncells <= 0 || n <= 0) return;
  cudaMemsetAsync(srows, 0xFF, sizeof(OzStackRow) * (size_t)n, st);
  oz_stack_rows_kernel<<<ncells, 128, 0, st>>>(cells, prows, srows);
}

void launch_oz_max(const OzJob *jobs, int njobs, const OzSpan *spans, int nspans, const double *ops,
                   const double *psi, const double *scr, double *scales, int *err, cudaStream_t st) {
  if (njobs <= 0 || nspans <= 0) return;
  oz_max_kernel<<<nspans, OZ_SPLIT_THREADS, 0, st>>>(jobs, njobs, spans, ops, psi, scr, scales, err);
}

void launch_oz_split(const OzJob *jobs, int njobs, const OzSpan *spans, int nspans, const double *ops,
                     const double *psi, const double *scr, const double *scales, uint8_t *pack, int s, cudaStream_t st) {
  if (njobs <= 0 || nspans <= 0) return;
#define OZ_SPLIT(SS) oz_split_kernel<SS><<<nspans, OZ_SPLIT_THREADS, 0, st>>>(jobs, njobs, spans, ops, psi, scr, scales, pack)
  switch (s) {
    case 3: OZ_SPLIT(3); break;
    case 4: OZ_SPLIT(4); break;
    case 5: OZ_SPLIT(5); break;
    case 6: OZ_SPLIT(6); break;
    case 7: OZ_SPLIT(7); break;
    case 8: OZ_SPLIT(8); break;
    default: break;
  }
#undef OZ_SPLIT
}

template <int S, int BN>
static cudaError_t launch_gemm_t(const OzGemmParams &p, int ncta, cudaStream_t st) {
  using Cf = OzCfg<S, BN>;
  cudaError_t e = cudaFuncSetAttribute(oz_gemm_kernel<S, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cf::SMEM);
  if (e != cudaSuccess) return e;
  oz_gemm_kernel<S, BN><<<ncta, OZ_GEMM_THREADS, Cf::SMEM, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_oz_gemm(const OzItem *items, const int32_t *cta, int ncta, const OzSeg *segs, const OzFam *fams,
                           const OzCell *cells, const OzStackRow *srows, const Task *tasks, const uint8_t *pack,
                           double *scales, const double *psi, double *scr, double *out, int *err, int s, int bn,
                           uint64_t wait_ns, cudaStream_t st) {
  if (ncta <= 0) return cudaSuccess;
  const OzGemmParams p{items, cta, segs, fams, cells, srows, tasks, pack, scales, psi, scr, out, err, wait_ns};
  if (s == 5 && bn == 32) return launch_gemm_t<5, 32>(p, ncta, st);
  if (bn != oz_bn(s)) return cudaErrorInvalidValue;
  switch (s) {
    case 3: return launch_gemm_t<3, 48>(p, ncta, st);
    case 4: return launch_gemm_t<4, 48>(p, ncta, st);
    case 5: return launch_gemm_t<5, 48>(p, ncta, st);
    case 6: return launch_gemm_t<6, 32>(p, ncta, st);
    case 7: return launch_gemm_t<7, 32>(p, ncta, st);
    case 8: return launch_gemm_t<8, 32>(p, ncta, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tjb
