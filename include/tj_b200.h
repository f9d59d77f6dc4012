/*
 * tj_b200.h -- C ABI of the B200 implementation of the tjsq SU(2) t-J DMRG hot path.
 *
 * The reference (DongNingSheng/Grand_SQL_tJ, code/tjsq, Fortran 90) keeps its
 * block-sparse tensors in derived types with allocatable components, which are
 * not C-interoperable.  This header gives flat mirrors of those types and one
 * entry point per reference routine on the hot path.  A Fortran caller fills
 * the structs from its derived types through an ISO_C_BINDING shim module
 * and calls these functions in place of the Fortran ones.
 *
 * Conventions shared by every struct below:
 *   - quantum numbers are the reference's integer labels: num_up (particle
 *     number, or 0 when up_bias = 0) and num_down (twice the total spin, 2S);
 *   - every dense matrix is column-major (Fortran order) and addressed as
 *     data + off, with off counted in doubles;
 *   - all pointers are host pointers owned by the caller;
 *   - every function returns 0 on success or a TJ_ERR_* code; the message of
 *     the last error on the calling thread is returned by tj_last_error().
 */
#ifndef TJ_B200_H
#define TJ_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ errors */
enum {
  TJ_OK = 0,
  TJ_ERR_ARG = 1,         /* null pointer, negative or inconsistent size            */
  TJ_ERR_QN = 2,          /* quantum-number mismatch (the reference calls `stop`)   */
  TJ_ERR_CUDA = 3,        /* a CUDA runtime call failed                             */
  TJ_ERR_NOMEM = 4,       /* device allocation failed                               */
  TJ_ERR_NODEV = 5,       /* no CUDA device, or the device is not sm_100            */
  TJ_ERR_TIMEOUT = 6,     /* a bounded device-side wait gave up                     */
  TJ_ERR_NUMERIC = 7,     /* NaN/Inf met, or an eigen-solver did not converge       */
  TJ_ERR_LIMIT = 8        /* a size exceeds a documented fixed limit                */
};

/* -------------------------------------------------------------- data types */

/* Sub_Block + its mat(row_dim, sdim)  (code/tjsq/common.f90:114-117).
 * The sub-block maps the sector (num_up, num_down) to
 * (num_up + up_dif, num_down + down_dif); mat has row_dim rows (the target
 * sector's dimension) and sdim columns (the source sector's dimension). */
typedef struct tj_block_sub {
  int32_t num_up, num_down, down_dif, row_dim, sdim, pad_;
  int64_t off;
} tj_block_sub;

/* Total_Block  (code/tjsq/common.f90:119-122).  sub(1:num) = sub[0..num-1]. */
typedef struct tj_block {
  int32_t len, num, dim, up_dif, down_dif, pad_;
  const tj_block_sub *sub;
  const double *data;
} tj_block;

/* Block_Set  (code/tjsq/common.f90:139-141). */
typedef struct tj_block_set {
  tj_block elec_up, elec_down, spin_sd, spin_sz, num_sn;
} tj_block_set;

/* Total_Model  (code/tjsq/common.f90:144-149).  Only ham and sub(1:nsub) are
 * inputs; snc(2) and sub_s(nxx) are produced by hmerge inside the library
 * (code/tjsq/get_sys.f90:4383-4593). */
typedef struct tj_model {
  int32_t len, nsub;
  tj_block ham;
  const tj_block_set *sub;       /* sub(1:nsub) */
} tj_model;

/* Sub_Basis_Map  (code/tjsq/common.f90:65-69). */
typedef struct tj_basis_sub {
  int32_t spos, sdim, bl_num_up, bl_num_down, st_num_up, st_num_down;
} tj_basis_sub;

/* Basis_Map  (code/tjsq/common.f90:72-76); sub(1:num) = maps[first .. first+num-1]. */
typedef struct tj_basis_map {
  int32_t idx, num, dim, new_num_up, new_num_down, first;
} tj_basis_map;

/* Total_Basis  (code/tjsq/common.f90:79-82). */
typedef struct tj_basis {
  int32_t len, num, dim, pad_;
  const tj_basis_map *sub;
  const tj_basis_sub *maps;
} tj_basis;

/* Sub_Wave  (code/tjsq/common.f90:100-105); vec(sys_dim, env_dim) at data + off. */
typedef struct tj_wave_sub {
  int32_t sys_num_up, sys_num_down, env_num_up, env_num_down, sys_dim, env_dim;
  int64_t off;
} tj_wave_sub;

/* Wavefunction  (code/tjsq/common.f90:107-110).  dim = sum sys_dim*env_dim. */
typedef struct tj_wave {
  int32_t sys_len, env_len, num, pad_;
  int64_t dim;
  const tj_wave_sub *sub;
  double *data;
} tj_wave;

/* Module pubdata globals read on the hot path (code/tjsq/common.f90:10-45),
 * passed with their Fortran shapes and lower bounds:
 *   neib (0:num_site, neibt)      neib [(k-1)*(num_site+1) + i]
 *   neiba(0:num_site, 0:num_site) neiba[j*(num_site+1) + i]
 *   inb1 (0:num_site, 0:num_site) inb1 [j*(num_site+1) + i]
 *   nleg11(1:num_site)            nleg11[i-1]
 *   nposi, nposi_dm, nposi_lat (0:num_site)  x[i]
 *   jt, jz, jd (neibt, 0:num_site)           x[i*neibt + (k-1)]
 *   jn (neibt)                                jn[k-1]
 *   esite (0:num_site)                        esite[i]
 * up_bias is the parameter of common.f90:12 (0: grand-canonical labels).
 * The site operators st_elec_up, st_sd, num_elec, st_si of
 * Get_site_operator_su2_U0 (code/tjsq/dmrg_sub.f90:370-473) are rebuilt
 * from up_bias inside the library. */
typedef struct tj_lattice {
  int32_t num_site, neibt, up_bias, pad_;
  const int32_t *neib, *neiba, *inb1, *nleg11, *nposi, *nposi_dm, *nposi_lat;
  const double *jt, *jz, *jd, *jn, *esite;
} tj_lattice;

/* Output of Get_truncation_operator (code/tjsq/den_mat.f90:141-383).
 * Two-call pattern: call tj_truncation with data == NULL to learn num and
 * the total number of doubles (data_len); allocate sub[num] and
 * data[data_len]; call again to fill them.  trun_op sub-blocks have
 * down_dif = 0, row_dim = sector dimension, sdim = kept columns.  The first
 * call leaves the operator on the device and the second copies it from
 * there into data (at the DMA rate when data is page-locked); when another
 * truncation ran on the same context in between, the second call computes
 * it again. */
typedef struct tj_trunc_result {
  int32_t num_state;         /* kept states (Num_state)                             */
  int32_t num;               /* kept sectors (trun_op%num)                          */
  int64_t data_len;          /* doubles needed for all trun_op mats                 */
  double trunc_err;          /* discarded weight of the renormalised spectrum       */
  double entropy1, entropy2, entropys;  /* entropies of den_mat.f90:222-297         */
  tj_block_sub *sub;         /* caller-allocated, num entries (or NULL)             */
  double *data;              /* caller-allocated, data_len doubles (or NULL)        */
} tj_trunc_result;

/* -------------------------------------------------------------- context */
typedef struct tj_ctx tj_ctx;

enum { TJ_PREC_FP64 = 0, TJ_PREC_OZAKI = 1 };

/* Creates a context bound to one CUDA device (one context per host thread). */
int tj_ctx_create(tj_ctx **ctx, int device);
int tj_ctx_destroy(tj_ctx *ctx);
/* Arithmetic of the block GEMMs of H*psi: TJ_PREC_FP64, or TJ_PREC_OZAKI with
 * `slices` int8 slices per operand (3..8). */
int tj_set_precision(tj_ctx *ctx, int mode, int slices);
/* No counterpart in the reference.  Every wait inside the split-precision
 * GEMM's pipeline (a stage's copies, the MMAs of a family, an item's
 * metadata) gives up after `seconds` (default 2): the kernel then lets its
 * other roles stop, waits for its copies and MMAs in flight (with their own
 * 2 s bound), releases its tensor memory and returns, and the call returns
 * TJ_ERR_TIMEOUT; the context stays usable.  seconds in [0, 60]. */
int tj_set_wait_limit(tj_ctx *ctx, double seconds);
/* Invalidates the operators and task lists cached for the current DMRG step. */
int tj_step_begin(tj_ctx *ctx);
/* No counterpart in the reference.  Keeps on the device, within a budget of
 * `gigabytes` (0, the default: off), the arrays the library writes into
 * caller memory -- the blocks of tj_get_hamiltonian, the Ritz vector of
 * tj_lanczos_memo_new, the truncation operator of tj_truncation, the
 * predicted wavefunction of tj_wave_trans; later
 * uploads from inside such an array (tj_model_wave, tj_lanczos_memo_new,
 * tj_truncation, tj_wave_trans, tj_get_hamiltonian, the measurement
 * operators) copy the kept device data instead.  The caller must not modify a filled array
 * while it is kept: tj_residency_forget(ctx, p) drops the array containing
 * p (do so before freeing or reusing it).  A fingerprint of 64 values of
 * each array, checked at every use, drops an entry whose array changed
 * there; least recently used entries go first when the budget is full. */
int tj_set_residency(tj_ctx *ctx, double gigabytes);
int tj_residency_forget(tj_ctx *ctx, const void *host);
const char *tj_last_error(void);
/* No counterpart in the reference.  Page-locks (pins) `bytes` of the caller's
 * host memory at `p` for the lifetime of the registration, so that the
 * per-step operator upload of tj_model_wave / tj_lanczos_memo_new runs as
 * asynchronous DMA that overlaps the plan compilation on the host.  Optional:
 * unpinned memory works, with the upload copied through the driver's staging
 * buffers.  tj_host_unregister releases a registration made here. */
int tj_host_register(void *p, size_t bytes);
int tj_host_unregister(void *p);

/* W6JS / W3JS (code/tjsq/block.f90:1564-1615, 1522-1561): the Wigner 6j and
 * 3j symbols on doubled spins (and doubled projections), as the library's
 * coefficient tables compute them on the host. */
double tj_w6js(int j1, int j2, int j3, int l1, int l2, int l3);
double tj_w3js(int j1, int j2, int j3, int m1, int m2, int m3);

/* ------------------------------------------------------- hot-path calls */

/* model_wave(sys,env,sys_bs,env_bs,invec,outvec)  (code/tjsq/get_sys.f90:4127-4381),
 * add_op = 1 branch, preceded by hmerge(sys,env,sys_bs,env_bs)
 * (code/tjsq/get_sys.f90:4383-4593) as lanczos_memo_new does
 * (code/tjsq/eigen.f90:53-56).  outvec must have invec's sector layout; it
 * is overwritten. */
int tj_model_wave(tj_ctx *ctx, const tj_lattice *lat,
                  const tj_model *sys, const tj_model *env,
                  const tj_basis *sys_bs, const tj_basis *env_bs,
                  const tj_wave *invec, tj_wave *outvec);

/* lanczos_memo_new(sys,env,sys_bs,env_bs,super,eigvec,levels,num_idx)
 * (code/tjsq/eigen.f90:2-175) for levels = 1: eigvec is the start vector on
 * entry and the normalised Ritz vector on return; energies[0] = Energys(1);
 * iters = Lanczos vectors used.  lanzero is the module global Lanzero. */
int tj_lanczos_memo_new(tj_ctx *ctx, const tj_lattice *lat,
                        const tj_model *sys, const tj_model *env,
                        const tj_basis *sys_bs, const tj_basis *env_bs,
                        tj_wave *eigvec, int levels, double lanzero,
                        double *energies, int *iters);

/* Get_density_matrix_{sys,env}_new + Get_truncation_operator
 * (code/tjsq/den_mat.f90:84-134, 141-383) for levels = 1.
 * side = 0: system block (rho = psi psi^T), side = 1: environment block
 * (rho = psi^T psi).  The block length written to the result's sub-blocks is
 * wave->sys_len or wave->env_len. */
int tj_truncation(tj_ctx *ctx, const tj_wave *wave, int side,
                  int kept_min, int kept_max, double trun_err,
                  tj_trunc_result *out);

/* Correlator contractions value = <psi| O |psi> (code/tjsq/measure.f90).
 * flag is 'B' (boson) or 'F' (fermion) as FlagSign in the reference. */
int tj_measure_sys_block(tj_ctx *ctx, const tj_block *sys_bl, const tj_basis *sys_bs,
                         const tj_wave *wave, double *value);              /* :1241-1295 */
int tj_measure_env_block(tj_ctx *ctx, const tj_block *env_bl, const tj_basis *env_bs,
                         const tj_wave *wave, double *value);              /* :1359-1414 */
int tj_sys_block_env_block_cor_dia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_bl,
                                   const tj_basis *sys_bs, const tj_basis *env_bs,
                                   const tj_wave *wave, double *value);    /* :1638-1732 */
int tj_sys_block_env_block_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_bl,
                                    const tj_basis *sys_bs, const tj_basis *env_bs,
                                    const tj_wave *wave, char flag, double *value); /* :5241-5480 */
int tj_sys_block_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *sys_st,
                               const tj_basis *sys_bs, const tj_wave *wave,
                               char flag, double *value);                  /* :4939-5083 */
int tj_env_block_site_cor_ndia(tj_ctx *ctx, const tj_block *env_bl, const tj_block *env_st,
                               const tj_basis *env_bs, const tj_wave *wave,
                               char flag, double *value);                  /* :5085-5238 */
int tj_sys_block_env_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_bl, const tj_block *env_st,
                                   const tj_basis *sys_bs, const tj_basis *env_bs,
                                   const tj_wave *wave, char flag, double *value); /* :5482-5706 */
int tj_sys_site_env_block_cor_ndia(tj_ctx *ctx, const tj_block *sys_st, const tj_block *env_bl,
                                   const tj_basis *sys_bs, const tj_basis *env_bs,
                                   const tj_wave *wave, char flag, double *value); /* :5926-6154 */
int tj_sys_site_env_site_cor_ndia(tj_ctx *ctx, const tj_block *sys_st, const tj_block *env_st,
                                  const tj_basis *sys_bs, const tj_basis *env_bs,
                                  const tj_wave *wave, char flag, double *value); /* :5709-5924 */

/* ------------------------------------------------ operator renormalisation */

/* A block model written by the library: Total_Model (code/tjsq/common.f90:
 * 144-149) with ham and sub(1:nsub).  Two-call pattern, as tj_trunc_result:
 * with sets, subs or data NULL only the sizes are filled; then the caller
 * allocates sets[nsub], subs[n_subs] and data[data_len] and calls again, and
 * `model` is filled with blocks that point into those arrays (every block's
 * data pointer is `data`; its sub-blocks' offsets are counted from there).
 * Sub-block records follow the order ham, then sets 1..nsub, each set in the
 * order elec_up, elec_down, spin_sd, spin_sz, num_sn; a block's records are
 * in the order the reference's update_trun_dia / update_trun_ndia create
 * them (code/tjsq/block.f90:1311-1503), their matrices back to back. */
typedef struct tj_model_result {
  int32_t len, nsub;            /* new block length, operator sets nleg11(len)          */
  int32_t n_subs, pad_;         /* sub-block records of ham and every operator           */
  int64_t data_len;             /* doubles of all their matrices                         */
  tj_block_set *sets;           /* caller-allocated, nsub entries (or NULL)              */
  tj_block_sub *subs;           /* caller-allocated, n_subs entries (or NULL)            */
  double *data;                 /* caller-allocated, data_len doubles (or NULL)          */
  tj_model model;               /* second call: the new model                            */
} tj_model_result;

/* Get_Hamiltonian_Sys(pre,next,basis,trun)  (code/tjsq/get_sys.f90:4-239)
 * for side = 0, Get_Hamiltonian_Env  (code/tjsq/get_sys.f90:245-480) for
 * side = 1: the block `pre` (length L) is enlarged by one site into the
 * basis `basis` (Get_basis of pre, length L + 1) -- its Hamiltonian with the
 * new bonds (update_block_dia, Get_hamiltonian_ndia, Get_hamiltonian_dia,
 * the site's chemical potential) and the operator sets of the sites that
 * still have bonds outside the block (update_block_ndia_sys/env,
 * update_site_ndia_sys/env, update_block_dia, update_site_dia;
 * code/tjsq/block.f90:382-1306), reordered as the reference reorders them
 * -- and every operator is truncated with `trun`: U^T O U per sector pair
 * (update_trun_dia / update_trun_ndia, code/tjsq/block.f90:1311-1503).  trun
 * is the truncation operator of tj_truncation (sub-block (num_up, num_down),
 * row_dim = the sector's dimension in `basis`, sdim = kept states); the
 * reference's untruncated steps pass the identity (block_transfer_basis with
 * unit matrices, code/tjsq/dmrg_sub.f90:659-667, 678-686).  mshift is the reference's global
 * of the same name, read by the environment side only (the superblock's
 * system-block length + 1).  The new model (length L + 1, spin_sz left
 * empty as in the reference, whose loop over operator kinds skips it) is
 * returned through `out`. */
int tj_get_hamiltonian(tj_ctx *ctx, const tj_lattice *lat, int side, int mshift, const tj_model *pre,
                       const tj_basis *basis, const tj_block *trun, tj_model_result *out);


/* ------------------------------------------------- measurement operators */

/* A block operator written by the library, two-call pattern as above: with
 * subs or data NULL only num and data_len are filled; then the caller
 * allocates subs[num] and data[data_len] and calls again, and `block` is
 * filled (its sub points to subs, its data to data). */
typedef struct tj_block_result {
  int32_t num, pad_;
  int64_t data_len;
  tj_block_sub *subs;          /* caller-allocated, num entries (or NULL)  */
  double *data;                /* caller-allocated, data_len doubles       */
  tj_block block;              /* second call: the operator                */
} tj_block_result;

/* The measurement chain of one side: the module arrays sys_bsm(:) /
 * systruns(:) (or env_bsm / envtruns) that the reference's Measurement reads
 * from disk (code/tjsq/main.f90:225-240).  bsm[i - 1] is the enlarged basis
 * of block length i (i = 2..n; bsm[0] is not read) and truns[i - 1] its
 * truncation operator (read for i > trun_idx; lengths <= trun_idx are kept
 * untruncated, as the reference's trun_idx). */
typedef struct tj_chain {
  int32_t n, trun_idx;
  const tj_basis *bsm;
  const tj_block *truns;
} tj_chain;

/* Get_sys_oper_dia / Get_env_oper_dia / Get_sys_oper_ndia / Get_env_oper_ndia
 * (code/tjsq/get_sys.f90:764-891, 998-1130): the one-site operator st_oper
 * placed at site old_idx (counted from the block's open end) and carried
 * through the chain to a block of length new_idx (the enlarged basis of
 * length new_idx; with truns != 0 truncated by its truncation operator).
 * side 0: system chain, 1: environment chain; dia != 0: the _dia routines
 * (down_dif = 0 operators), else the _ndia routines with types 'F' or 'B'.
 * Each step of the chain (enlarge by one site, truncate) is one pair of
 * grouped-GEMM launches; the operator stays on the device between steps. */
int tj_get_oper(tj_ctx *ctx, int side, int dia, const tj_chain *chain, const tj_block *st_oper, int old_idx,
                int new_idx, int truns, char types, tj_block_result *out);
/* Change_sys_oper_dia / Change_env_oper_dia / Change_sys_oper_ndia /
 * Change_env_oper_ndia (code/tjsq/get_sys.f90:893-996, 1134-1238): a block
 * operator of block length old_idx carried to block length new_idx. */
int tj_change_oper(tj_ctx *ctx, int side, int dia, const tj_chain *chain, const tj_block *old_oper, int old_idx,
                   int new_idx, int truns, char types, tj_block_result *out);
/* block_mul_block_ndia(oper1,Flag1,oper2,Flag2,coef,new_oper,basis)
 * (code/tjsq/block.f90:1956-2197): the product of two operators of one block
 * coupled to total spin transfer down_dif (the caller's new_oper%down_dif),
 * with the Wigner 3j recoupling; flag 'N' or 'T' per operand. */
int tj_block_mul_block_ndia(tj_ctx *ctx, const tj_block *oper1, char flag1, const tj_block *oper2, char flag2,
                            double coef, int down_dif, const tj_basis *basis, tj_block_result *out);
/* update_trun_dia (dia != 0) / update_trun_ndia (code/tjsq/block.f90:1311-
 * 1503): U^T O U of a block operator by a truncation operator. */
int tj_update_trun(tj_ctx *ctx, int dia, const tj_block *ori, const tj_block *trun, tj_block_result *out);

/* ------------------------------------------------ wavefunction prediction */

/* wave_trans_LR(sys_bs,env_bs,sys_trun,env_trun,old_wave,new_wave)
 * (code/tjsq/dmrg_sub.f90:1093-1238) for direction = 0 and wave_trans_RL
 * (code/tjsq/dmrg_sub.f90:1242-1384) for direction = 1: the converged
 * wavefunction of the last DMRG step carried to the next superblock of a
 * sweep, as the reference's left_to_right / right_to_left call them
 * (dmrg_sub.f90:778, 845, 960, 1026).  Arguments as in the reference:
 * direction 0 -- sys_bs is the new system block's enlarged basis, env_bs the
 * environment basis of the last step, sys_trun the truncation just computed,
 * env_trun the one that built the last step's environment block; direction
 * 1 -- the mirror image.  new_wave's sector table is the caller's
 * (allocate_wave of the new super basis); its data is overwritten by the
 * carried vector, normalised (wave_normalize).  TJ_ERR_NUMERIC if the
 * carried vector is zero. */
int tj_wave_trans(tj_ctx *ctx, int direction, const tj_basis *sys_bs, const tj_basis *env_bs,
                  const tj_block *sys_trun, const tj_block *env_trun, const tj_wave *old_wave,
                  tj_wave *new_wave);

/* ------------------------------------------------------- checkpoint files */

/* The reference's files (code/tjsq/block.f90:2760-3097), read and written on
 * the host.  Binary files are Fortran sequential unformatted files as
 * gfortran and ifort write them: each WRITE statement is one record framed by
 * its byte length as a 4-byte little-endian integer before and after (a
 * record above 2^31 - 9 bytes as subrecords with negative markers), default
 * integers of 4 bytes, REAL(8) of 8, matrices column-major.  Basis files are
 * the formatted text of basis_to_disk.  The reference names them sysblocks<i>,
 * systruns<i>, sysbs<i> (and env...) and eigvec<i> (Get_model_name,
 * Get_wave_name, code/tjsq/dmrg_sub.f90:294-346); tj_disk_name builds them:
 * kind 0 sysblocks, 1 systruns, 2 sysbs, 3 envblocks, 4 envtruns, 5 envbs,
 * 6 eigvec. */
int tj_disk_name(int kind, int idx, char *buf, int buflen);
/* wave_to_disk (block.f90:2760-2787) */
int tj_wave_to_disk(const char *path, const tj_wave *wave);
/* wave_from_disk (block.f90:2791-2821), two-call: with subs or data NULL
 * only hdr's sys_len, env_len, num and dim are filled; then the caller
 * allocates subs[num] and data[dim] and calls again (hdr->sub and hdr->data
 * are set to them, sectors back to back from offset 0). */
int tj_wave_from_disk(const char *path, tj_wave *hdr, tj_wave_sub *subs, double *data);
/* truns_to_disk / truns_from_disk (block_to_disk / block_from_disk;
 * block.f90:2826-2870, 2956-2996): one block per file; two-call result. */
int tj_block_to_disk(const char *path, const tj_block *block);
int tj_block_from_disk(const char *path, tj_block_result *out);
/* model_to_disk (block.f90:2873-2906): len, ham, then per operator set (the
 * caller's nsub = nleg11(len)) elec_up, elec_down, spin_sd, num_sn.
 * model_from_disk (block.f90:2910-2952), two-call as tj_model_result, nsub
 * from the number of blocks stored, spin_sz empty (it is not stored); the
 * reference's deletion of the next block file is left to the caller. */
int tj_model_to_disk(const char *path, const tj_model *model);
int tj_model_from_disk(const char *path, tj_model_result *out);
/* basis_to_disk / basis_from_disk (block.f90:3000-3097), formatted text.
 * Two-call: with sub or maps NULL the sizes are filled; then the caller
 * allocates sub[num] and maps[nmaps] and calls again. */
typedef struct tj_basis_result {
  int32_t len, num, dim, nmaps;
  tj_basis_map *sub;           /* caller-allocated, num entries (or NULL)   */
  tj_basis_sub *maps;          /* caller-allocated, nmaps entries (or NULL) */
  tj_basis basis;              /* second call: the basis                    */
} tj_basis_result;
int tj_basis_to_disk(const char *path, const tj_basis *basis);
int tj_basis_from_disk(const char *path, tj_basis_result *out);

/* --------------------------------------------------- measurement support */

/* Statistics of the H*psi task list compiled for the last tj_model_wave /
 * tj_lanczos_memo_new call: flops and bytes per H*psi (the algorithmic work
 * used for the roofline), task and tile counts, and the device time of the
 * last H*psi in milliseconds (CUDA events on the context's stream). */
typedef struct tj_hpsi_stats {
  double flops;            /* executed FP64-equivalent flops per H*psi           */
  double flops_ref;        /* flops of the reference's DGEMM sequence           */
  double bytes;            /* algorithmic HBM bytes per H*psi                    */
  int64_t n_products, n_tasks, n_tiles_p1, n_tiles_p2, scratch_doubles;
  double last_ms;          /* device time of the last H*psi                      */
  double last_ms_phase1, last_ms_phase2;  /* its first / second GEMM launch          */
  int64_t lanczos_hpsi;    /* H*psi products of the last tj_lanczos_memo_new      */
  double int8_ops;         /* split precision: 2 x int8 MACs issued per H*psi     */
  int64_t kernels_per_hpsi; /* kernel launches of one H*psi                        */
  double last_ms_split;    /* split precision: its max/split kernels             */
  double flops_launch1, flops_launch2;  /* FP64-equivalent flops of each launch    */
  double int8_ops_launch1, int8_ops_launch2;  /* split precision: issued per launch */
  /* host wall time (ms) of the last plan preparation: all of it, the H*psi
   * plan compile, operator upload + hmerge + work-list upload, the
   * split-precision plan, and the last tj_lanczos_memo_new after it */
  double prepare_ms, plan_ms, upload_ms, ozplan_ms, lanczos_ms;
  /* the last tj_get_hamiltonian: host time of its plan (ms), device time of
   * its two GEMM launches (ms), the whole call from the first upload to the
   * end of the download (ms), and its FP64 flops */
  double renorm_plan_ms, renorm_ms, renorm_e2e_ms, renorm_flops;
  /* the last tj_truncation that computed (not the cached second call):
   * device time (ms) of psi's upload and the density matrices, the
   * tridiagonal reductions, the eigenvalues (with their download), the host
   * keep rule, inverse iteration of the kept vectors, their
   * orthonormalisation, the back-transformation and download; the whole
   * call (host wall time); the largest density-matrix sector and the largest
   * kept block */
  double trunc_ms_rho, trunc_ms_tridiag, trunc_ms_eig, trunc_ms_select, trunc_ms_vec, trunc_ms_orth,
      trunc_ms_back, trunc_ms_total;
  int64_t trunc_max_n, trunc_max_kept;
  /* residency (tj_set_residency): uploads served from kept device copies
   * since the context was created, and their bytes */
  int64_t res_hits;
  double res_hit_bytes;
  /* the last tj_get_hamiltonian's second call: host time (ms) before its
   * first upload and after its download (result tables, residency) */
  double renorm_pre_ms, renorm_post_ms;
  /* the last tj_wave_trans: host time (ms) of its plan, and device time
   * from its first upload to the end of its download */
  double wt_plan_ms, wt_ms;
} tj_hpsi_stats;
int tj_hpsi_stats_get(tj_ctx *ctx, tj_hpsi_stats *st);

/* ---------------------------------------------- independent instances */
/* No counterpart in the reference.  model_wave (with hmerge) of n
 * independent superblocks -- several DMRG runs at different dopings or J/t,
 * each with its own lattice, models, bases and wavefunction -- in shared
 * launches: the instances' plans are merged into one (operators, vectors,
 * products and basis-state scales placed one after another) so that one set
 * of kernels computes every outvec[i] = H_i invec[i].  The merged plan is
 * cached like the single one.  reps > 0: after the product, `reps` more
 * products of all instances are timed on the device and *ms receives the
 * mean time of one. */
int tj_model_wave_multi(tj_ctx *ctx, int n, const tj_lattice *const *lat, const tj_model *const *sys,
                        const tj_model *const *env, const tj_basis *const *sys_bs, const tj_basis *const *env_bs,
                        const tj_wave *const *invec, tj_wave *const *outvec, int reps, double *ms);

/* ------------------------------------------------------------ autotuning */
/* No counterpart in the reference.  The tiling of the grouped FP64 GEMM
 * (split-K granularity: items per resident CTA and minimum inner-dimension
 * steps per item; resident CTAs per SM) and of the split-precision GEMM (N
 * tile, per-item cost of its static schedule) is chosen per block-size
 * histogram of the H*psi plan -- its GEMM tasks counted by (log2 M, log2 N,
 * log2 K) -- by timing H*psi with each candidate (coordinate descent from the
 * defaults; a change is kept when it is at least 2 % faster).  The choices
 * are kept in a process-wide table; TJ_TUNE_CACHED (default) uses a stored
 * choice when the histogram matches, TJ_TUNE_ON_MISS also runs the search
 * the first time a histogram is seen, TJ_TUNE_OFF always uses the defaults. */
enum { TJ_TUNE_OFF = 0, TJ_TUNE_CACHED = 1, TJ_TUNE_ON_MISS = 2 };
typedef struct tj_tune_result {
  int32_t items_per_cta, min_ksteps, ctas_per_sm, oz_bn, oz_item_cost;
  int32_t evaluated;            /* candidates timed                                   */
  double default_ms, tuned_ms;  /* device time of one H*psi with the defaults / chosen */
  double tuning_ms;             /* host wall time of the search                       */
  uint64_t hist_key;
} tj_tune_result;
int tj_set_autotune(tj_ctx *ctx, int mode);
/* Runs the search for this superblock (in the context's precision mode)
 * whatever the mode, stores the choice and leaves the plan prepared with it. */
int tj_autotune(tj_ctx *ctx, const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, tj_tune_result *out);

/* ------------------------------------------- grouped block-GEMM benchmark */
/* No counterpart in the reference.  The batched block-GEMM pattern of H*psi
 * on synthetic data: output cell c (M x N, column-major, ld = M, at
 * out[out_off]) = sum over its terms t in [t_begin, t_end) of
 * coef * op(L) op(R), op(L) M x K, op(R) K x N, both windows of one operand
 * pool (l_off / r_off, leading dimensions l_ld / r_ld, transposed when
 * l_trans / r_trans).  mode 0: one persistent grouped launch (the H*psi FP64
 * kernel, split-K tiling from the context's choices); mode 1: one launch per
 * term (block GEMM), each adding to its cell; mode 2: mode 0 after the
 * autotuner's search of the tiling for this batch (reported in *tuned when
 * not NULL; the context's own choices are left as they were).  The pool is
 * uploaded once; `reps` timed repetitions (CUDA events) after one warm-up
 * give *ms per repetition; out (out_len doubles) receives the result and
 * *flops the algorithmic 2 M N K sum. */
typedef struct tj_gg_cell { int64_t out_off; int32_t M, N, t_begin, t_end; } tj_gg_cell;
typedef struct tj_gg_term {
  int64_t l_off, r_off;
  int32_t l_ld, r_ld, K, l_trans, r_trans, pad_;
  double coef;
} tj_gg_term;
int tj_grouped_gemm_bench(tj_ctx *ctx, const tj_gg_cell *cells, int ncells, const tj_gg_term *terms, int nterms,
                          const double *pool, int64_t pool_len, int64_t out_len, int mode, int reps,
                          double *out, double *ms, double *flops, tj_tune_result *tuned);

/* Device-resident benchmarking helper: uploads invec once, then runs `reps`
 * H*psi products back to back on the device (inputs resident in HBM), with
 * CUDA events around the whole loop; *ms is the mean device time per H*psi.
 * The result of the last product is copied to outvec. */
int tj_model_wave_bench(tj_ctx *ctx, const tj_lattice *lat,
                        const tj_model *sys, const tj_model *env,
                        const tj_basis *sys_bs, const tj_basis *env_bs,
                        const tj_wave *invec, tj_wave *outvec, int reps, double *ms);

/* ------------------------------------------------ allocation-free H*psi */
/* No counterpart in the reference.  model_wave (with hmerge) for callers that
 * cannot allocate device memory while they run -- for example a Fortran sweep
 * driver whose device memory belongs to its own pool, or a host program that
 * forbids allocation inside a solve.  The caller passes every operator
 * block's data and both wavefunctions' data as DEVICE pointers (8-byte
 * aligned; the sector and sub-block tables stay in host memory).  Everything
 * else -- hmerge'd operator sums, phase-1 products, work lists -- is placed
 * in one fixed array of TJ_NOALLOC_SCRATCH_BYTES in device global memory
 * that the library declares; every GPU that loads the library holds it until
 * the process exits.  The call allocates nothing (no cudaMalloc/cudaFree),
 * runs on `stream` (a cudaStream_t, NULL for the default stream) and returns
 * after the stream has synchronised.  It always computes in FP64 (the grouped
 * FP64 GEMM): the split-precision mode of a tj_ctx does not apply to it.
 * invec and outvec must not share memory (TJ_ERR_ARG otherwise).  A
 * superblock needing more scratch than the array holds is rejected with
 * TJ_ERR_LIMIT.  The first call on a device looks up the array's device
 * address and keeps it for the life of the process, so make that first call
 * before any stream capture, and do not call this entry point on a device
 * after resetting it (cudaDeviceReset): the kept address would be stale.  All
 * calls share the one array: calls that overlap on the GPU (other threads,
 * other streams) race and must not be issued. */
#define TJ_NOALLOC_SCRATCH_BYTES (64ull << 20)
int tj_model_wave_noalloc(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                          const tj_basis *sys_bs, const tj_basis *env_bs,
                          const tj_wave *invec, tj_wave *outvec, void *stream);

/* ------------------------------------------------------ plan introspection */
/* The compiled form of one H*psi (hmerge + model_wave): phase-1 products
 * P = op(A) * X and phase-2 cells Y = sum coef * op(L) * op(R) (R.space == 0:
 * Y += coef * L).  Spaces: 1 operators, 2 input vector, 3 phase-1 products.
 * op(M) = M (trans 0) or M^T (trans 1) of the column-major matrix at
 * base + off with leading dimension ld.  This call needs no GPU and does no
 * arithmetic; the test-suite uses it to check the compiler on the CPU.
 * Two-call pattern: with every array pointer NULL the counts are filled. */
typedef struct tj_plan_operand { int64_t off; int32_t ld; int8_t space, trans; int16_t pad_; } tj_plan_operand;
typedef struct tj_plan_task { tj_plan_operand L, R; double coef; int32_t K, pad_; } tj_plan_task;
typedef struct tj_plan_cell { int64_t off; int32_t ld, M, N, t_begin, t_end; int8_t space, pad_[7]; } tj_plan_cell;
typedef struct tj_plan_upload { const double *src; int64_t n, dst; } tj_plan_upload;
typedef struct tj_plan_merge { int64_t dst, n; int32_t s_begin, s_end; } tj_plan_merge;
/* A work item: BM x BN tile (row0, col0) of `cell`, GEMM tasks [tb, te), axpy
 * tasks [ab, ae); slot < 0 stores the tile, slot >= 0 writes partial slot
 * `slot`.  A reduce record sums slots [slot0, slot0 + nslot) of a tile and
 * adds the axpy tasks [ab, ae).  Tile size: 64 x 64. */
typedef struct tj_plan_item { int32_t cell, row0, col0, tb, te, ab, ae, slot; } tj_plan_item;
typedef struct tj_plan_reduce { int32_t cell, row0, col0, slot0, nslot, ab, ae, pad_; } tj_plan_reduce;
typedef struct tj_plan_export {
  int64_t ops_len, scratch_len, psi_len;
  int64_t n_tasks1, n_tasks2, n_cells1, n_cells2, n_uploads, n_merges, n_merge_src;
  double flops, flops_ref, bytes;
  tj_plan_task *tasks1, *tasks2;
  tj_plan_cell *cells1, *cells2;
  tj_plan_upload *uploads;
  tj_plan_merge *merges;
  int64_t *merge_src;
  double *merge_coef;
  int64_t n_items1, n_items2, n_red1, n_red2;
  tj_plan_item *items1, *items2;
  tj_plan_reduce *red1, *red2;
} tj_plan_export;
int tj_hpsi_plan_export(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                        const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave,
                        tj_plan_export *out);
/* The same for one correlator contraction: kind 0..8 in the order of the
 * tj_measure_* / tj_*_cor_* declarations above (measure_sys_block = 0, ...,
 * sys_site_env_site_cor_ndia = 8); the epilogue dots every phase-2 cell with
 * psi, so value = sum over cells <psi_cell, Y_cell>.  Arguments as in the
 * matching entry point (NULL for a basis or operator it does not take). */
int tj_cor_plan_export(int kind, const tj_block *a, const tj_block *b, const tj_basis *sys_bs,
                       const tj_basis *env_bs, const tj_wave *wave, char flag, tj_plan_export *out);
/* The compiled form of tj_get_hamiltonian for checks on the CPU (no GPU, no
 * arithmetic): the two grouped-GEMM passes as in tj_hpsi_plan_export, with
 * space 1 = the blocks of `pre`, space 2 = trun's data from its lowest
 * sub-block offset, and the cells of the second pass writing the new
 * operators in the result's layout (psi_len = the result's data_len).  `res`
 * (optional) receives the result's sizes, and with its arrays set its
 * records and blocks, as tj_get_hamiltonian would give them (data left
 * unwritten). */
int tj_renorm_plan_export(const tj_lattice *lat, int side, int mshift, const tj_model *pre,
                          const tj_basis *basis, const tj_block *trun, tj_plan_export *out,
                          tj_model_result *res);
/* The compiled form of tj_wave_trans for checks on the CPU: space 1 = the
 * data of sys_trun then of env_trun (each from its lowest sub-block offset,
 * as the uploads say), space 2 = old_wave's data, the cells of the second
 * pass writing new_wave's layout before the normalisation (psi_len =
 * new_wave->dim). */
int tj_wave_trans_plan_export(int direction, const tj_basis *sys_bs, const tj_basis *env_bs,
                              const tj_block *sys_trun, const tj_block *env_trun, const tj_wave *old_wave,
                              const tj_wave *new_wave, tj_plan_export *out);

/* The split-precision form of the same H*psi (TJ_PREC_OZAKI with `slices`
 * int8 slices), for CPU checks of its tables.  A split stores `rows` x K of
 * a matrix in tiles of R rows (R = 128 for an A operand, the N tile for a B
 * operand) and ceil(K/32) k-blocks of `slices` int8 digit planes; tile t
 * (G_t row groups of 8: R/8, the last one gt_last) holds byte
 * (kb, p, g, c, r8, b) at
 *   base + t*nkb*slices*(R/8)*256 + ((kb*slices + p)*G_t + g)*256 + c*128 + r8*16 + b
 * for tile row 8g + r8 and k = 32kb + 16c + b.  A job writes coef*M(r, k) =
 * coef*src[src_off + r*rs + k*ks] (space 1 operators, 2 input vector, 3
 * phase-1 products) for r < nrows, k < K to split rows row0 + r, k-blocks
 * kb0.., with the row scale held in scales[scale_idx + r] (the row's max
 * |value|; want_max: the job raises it).  A segment pairs k-blocks of an A
 * split and a B split; a family sums its segments and scales by
 * scales[rs_idx + row] * scales[cs_idx + col]; an item is one output tile
 * of cell `cell` with families [fam_begin, fam_end) (kind 0: a cell of H*psi,
 * added to; kind 1: a tile of a product stack -- the phase-1 products of one
 * input cell, their operators' rows stacked -- whose rows are stored to their
 * products and raise their pi scales as prod_rows say; pi_idx is unused).
 * The plan schedules the items of each launch statically over 148
 * CTAs (the export's device-independent choice).  Two-call pattern as
 * above. */
typedef struct tj_oz_job {
  int64_t src_off, dst, scale_idx;
  double coef;
  int32_t rs, ks, nrows, K, gtot, kb0, R, nkb, ntiles, gt_last, row0;
  int8_t space, want_max, want_split, pad_;
} tj_oz_job;
typedef struct tj_oz_seg { int64_t a_base, b_base; int32_t a_nkb, b_nkb, a_kb0, b_kb0, nkb, pad_; } tj_oz_seg;
typedef struct tj_oz_fam { int32_t seg_begin, seg_end; int64_t rs_idx, cs_idx; int32_t nkb, pad_; } tj_oz_fam;
typedef struct tj_oz_item {
  int32_t kind, cell, row0, col0, M, N, mrows, ncols, fam_begin, fam_end, pad1_, init;
  int64_t pi_idx;
  int32_t nkb, pad2_;
  int64_t cost;
} tj_oz_item;
typedef struct tj_oz_cell { int64_t off; int32_t ld, M, N, a_begin, a_end, pad_; } tj_oz_cell;
/* a product of a product stack (kind-1 cell): stack rows [row_begin, row_begin + rows) are stored at
   off + row + col * ld of the product space; pi scale of its row r: pi + r */
typedef struct tj_oz_prow { int32_t row_begin, rows, ld, pad_; int64_t off, pi; } tj_oz_prow;
typedef struct tj_ozaki_export {
  int32_t slices, tile_n;
  int64_t sta_pack, dyn_pack, n_scales, rho0, tau0, pi0;
  double int8_ops;
  int64_t n_sta_jobs, n_psi_jobs, n_prod_jobs, n_segs, n_fams, n_cells, n_items1, n_items2;
  tj_oz_job *sta_jobs, *psi_jobs, *prod_jobs;
  tj_oz_seg *segs;
  tj_oz_fam *fams;
  tj_oz_cell *cells;
  tj_oz_item *items1, *items2;
  int64_t n_cta1, n_cta2;     /* CTA b of launch k runs items [cta_k[b], cta_k[b+1]) */
  int32_t *cta1, *cta2;
  /* the maximum jobs (row scales) of the three lists, run before their splits */
  int64_t n_sta_mjobs, n_psi_mjobs, n_prod_mjobs;
  tj_oz_job *sta_mjobs, *psi_mjobs, *prod_mjobs;
  /* the products of the product stacks (cells of kind-1 items: prod_rows[a_begin, a_end)) */
  int64_t n_prod_rows;
  tj_oz_prow *prod_rows;
} tj_ozaki_export;
int tj_ozaki_plan_export(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                         const tj_basis *sys_bs, const tj_basis *env_bs, const tj_wave *wave, int slices,
                         tj_ozaki_export *out);

#ifdef __cplusplus
}
#endif
#endif /* TJ_B200_H */
