// Device kernels of the B200 tjsq hot path (declarations shared by the host code).
#pragma once
#include <cuda_runtime.h>

#include "tj_internal.h"

namespace tjb {

// Parameters of one grouped-GEMM pass over a cell list.
struct GemmParams {
  const double *ops;    // SP_OPS base
  const double *psi;    // SP_PSI base (input vector)
  const double *scr;    // SP_SCR base (phase-1 products)
  double *out;          // base of the cells' output space
  const Cell *cells;
  const Task *tasks;
  const Tile *tiles;
  int ntiles;
  unsigned int *counter;   // dynamic tile counter (zeroed before launch)
  double *partials;        // dot mode: one partial sum per work item
  double *slots;           // partial tiles of split cells, BM*BN doubles per slot
  const double *dot_with;  // dot mode: vector the result is dotted with (same layout as out)
  int dot_mode;            // 0: store the tile, 1: write <dot_with, tile> to partials[tile]
};

void launch_grouped_gemm(const GemmParams &p, int grid, cudaStream_t s);
// out tile = sum of its partial slots (in slot order) + its axpy tasks
void launch_reduce(const GemmParams &p, const Reduce *red, int nred, cudaStream_t s);
int grouped_gemm_grid(int ntiles, int ctas_per_sm = 4);

// merged operators: dst[e] = sum_j coef_j * src_j[e]
void launch_merge(double *ops, const int64_t *dst, const int64_t *n, const int32_t *sb, const int32_t *se,
                  const int64_t *src, const double *coef, int nrec, cudaStream_t s);

// ---- vector kernels (length n) ----
// partial sums of x.y per block -> partials[gridDim]; finalize with launch_sum
void launch_dot(const double *x, const double *y, int64_t n, double *partials, int nblk, cudaStream_t s);
void launch_sum(const double *partials, int nblk, double *res, int sqrt_flag, cudaStream_t s);
int dot_blocks(int64_t n);
// y = y - a[ia]*x1 (- b[ib]*x2 if x2)   (a, b device scalars)
void launch_lanczos_update(double *y, const double *x1, const double *x2, const double *a, const double *b,
                           int64_t n, cudaStream_t s);
// x = x / (*nrm)
void launch_scale_inv(double *x, const double *nrm, int64_t n, cudaStream_t s);
// Gram-Schmidt: partial dots of w with V[0..k-1] (vectors of stride ld) -> partials[blk*kmax + j]
void launch_multi_dot(const double *V, int64_t ld, int k, const double *w, int64_t n, double *partials, int nblk,
                      int kmax, cudaStream_t s);
// coef[j] = (sum over blocks of partials[:, j]) / uu[j] ; uu == nullptr -> divide by 1
void launch_multi_sum(const double *partials, int nblk, int k, int kmax, const double *uu, double *coef,
                      cudaStream_t s);
// w = w - sum_j coef[j] * V[j]    (or w = sum_j coef[j] V[j] when assign)
void launch_combine(const double *V, int64_t ld, int k, const double *coef, double *w, int64_t n, int assign,
                    cudaStream_t s);
// lowest eigenvalue (and its eigenvector if vec) of the symmetric tridiagonal (a[0..n-1], b[0..n-2])
void launch_tridiag_min(const double *a, const double *b, int n, double *lam, double *vec, int want_vec,
                        cudaStream_t s);
// out = sum of a device array of n doubles into res (deterministic)
void launch_copy(double *dst, const double *src, int64_t n, cudaStream_t s);

// ---- Lanczos iteration with the step L read from device memory (*it) ----
// A vector chosen when the kernel runs: vec(*it + off) = V + (*it + off - 1) * ld, or `fixed`.
struct LzRef {
  double *V;
  int64_t ld;
  const int *it;
  int off;
  double *fixed;
};
// S: alpha(j) at S[j], beta(j) at S[128 + j], uu(j) at S[256 + j], the Ritz
// value at S[512], a norm at S[513]; cnt: a zeroed int the kernels that end in
// a grid-wide sum count their blocks on (the last block resets it); partials:
// lz_blocks(n) doubles.
int lz_blocks(int64_t n);
// dst = src - alpha(L) x1 - beta(L-1) x2 (x2 only for L >= 2); beta(L) = |dst|
void launch_lz_update_norm(LzRef dst, const double *src, LzRef x1, LzRef x2, double *S, const int *it, int64_t n,
                           double *partials, int *cnt, cudaStream_t s);
// w /= beta(L); w -= sum_{j < L} (V_j . w / uu[j]) V_j (classical Gram-Schmidt
// against the first L vectors); S[513] = |w|.  mpartials: mdb * kmax doubles.
void launch_lz_gram_schmidt(const double *V, int64_t ld, const int *it, LzRef w, int64_t n, double *S,
                            double *mpartials, int mdb, int kmax, const double *uu, double *coef, double *partials,
                            int *cnt, cudaStream_t s);
// w /= S[513], copied to x; uu(L + 1) = w . w
void launch_lz_scale_norm(LzRef w, double *x, int64_t n, double *S, const int *it, double *partials, int *cnt,
                          cudaStream_t s);
// alpha(L + 1) = x . y
void launch_lz_dot(LzRef x, const double *y, int64_t n, double *S, const int *it, double *partials, int *cnt,
                   cudaStream_t s);
// S[512] = lowest eigenvalue of the leading (L + 1) x (L + 1) tridiagonal;
// host[0] = beta(L), host[1] = S[512] (page-locked host memory); then L += 1
void launch_lz_tridiag_publish(double *S, int *it, double *host, cudaStream_t s);

}  // namespace tjb
