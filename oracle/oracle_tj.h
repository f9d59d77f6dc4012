/*
 * oracle_tj.h -- CPU restatement of the tjsq hot path (TEST INFRASTRUCTURE).
 *
 * This library is the oracle of the test-suite and the CPU baseline of the
 * benchmark.  It is never linked into, loaded by or called from the product
 * library (grand_sql_tj_b200).  It restates, in FP64 C, the Fortran routines
 * of DongNingSheng/Grand_SQL_tJ code/tjsq named beside each function below,
 * following their loop order, look-up rules and DGEMM call sequence (live
 * code only).  BLAS/LAPACK (dgemm, dsyev, dstev) come from the OpenBLAS that
 * ships inside scipy, loaded with dlopen as a stand-in for the reference's
 * Intel MKL.
 *
 * Parity status: unpinned.  The reference is Fortran, no Fortran compiler
 * exists in this image, and the reference ships no test vectors for these
 * routines; the oracle is checked against mathematical identities instead
 * (6j closed forms and orthogonality, symmetry of H*psi, exact
 * diagonalisation of small clusters -- see tests/).
 */
#ifndef ORACLE_TJ_H
#define ORACLE_TJ_H
#include "../include/tj_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Loads dgemm/dsyev/dstev from the OpenBLAS at `libpath`; threads <= 0 keeps
 * the library default.  Returns 0 on success. */
int ora_init(const char *libpath, int threads);
int ora_set_threads(int threads);

/* FACTRL + W6JS (code/tjsq/block.f90:1508-1516, 1564-1615) and W3JS
 * (block.f90:1522-1561); spins are doubled integers. */
double ora_w6js(int j1, int j2, int j3, int l1, int l2, int l3);
double ora_w3js(int j1, int j2, int j3, int m1, int m2, int m3);

/* hmerge + model_wave (code/tjsq/get_sys.f90:4383-4593, 4127-4381). */
int ora_model_wave(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                   const tj_basis *sys_bs, const tj_basis *env_bs,
                   const tj_wave *invec, tj_wave *outvec);

/* lanczos_memo_new for levels = 1 (code/tjsq/eigen.f90:2-175). */
int ora_lanczos(const tj_lattice *lat, const tj_model *sys, const tj_model *env,
                const tj_basis *sys_bs, const tj_basis *env_bs,
                tj_wave *eigvec, double lanzero, double *energy, int *iters);

/* Get_density_matrix_{sys,env} + Get_truncation_operator
 * (code/tjsq/den_mat.f90:4-78, 141-383); same two-call protocol as
 * tj_truncation.  eigval_out (optional, length = sum of sector dims) receives
 * the per-sector eigenvalues in DSYEV's ascending order, sector by sector. */
int ora_truncation(const tj_wave *wave, int side, int kept_min, int kept_max,
                   double trun_err, tj_trunc_result *out, double *eigval_out);

/* Correlator contractions (code/tjsq/measure.f90, lines in tj_b200.h). */
int ora_measure_sys_block(const tj_block *sys_bl, const tj_basis *sys_bs, const tj_wave *w, double *v);
int ora_measure_env_block(const tj_block *env_bl, const tj_basis *env_bs, const tj_wave *w, double *v);
int ora_sys_block_env_block_cor_dia(const tj_block *a, const tj_block *b, const tj_basis *sbs,
                                    const tj_basis *ebs, const tj_wave *w, double *v);
int ora_sys_block_env_block_cor_ndia(const tj_block *a, const tj_block *b, const tj_basis *sbs,
                                     const tj_basis *ebs, const tj_wave *w, char flag, double *v);
int ora_sys_block_site_cor_ndia(const tj_block *a, const tj_block *st, const tj_basis *sbs,
                                const tj_wave *w, char flag, double *v);
int ora_env_block_site_cor_ndia(const tj_block *b, const tj_block *st, const tj_basis *ebs,
                                const tj_wave *w, char flag, double *v);
int ora_sys_block_env_site_cor_ndia(const tj_block *a, const tj_block *st, const tj_basis *sbs,
                                    const tj_basis *ebs, const tj_wave *w, char flag, double *v);
int ora_sys_site_env_block_cor_ndia(const tj_block *st, const tj_block *b, const tj_basis *sbs,
                                    const tj_basis *ebs, const tj_wave *w, char flag, double *v);
int ora_sys_site_env_site_cor_ndia(const tj_block *st, const tj_block *st2, const tj_basis *sbs,
                                   const tj_basis *ebs, const tj_wave *w, char flag, double *v);

/* Get_Hamiltonian_Sys (side 0, code/tjsq/get_sys.f90:4-239) and
 * Get_Hamiltonian_Env (side 1, get_sys.f90:245-480) with update_block_dia,
 * update_site_dia, update_block_ndia_sys/env, update_site_ndia_sys/env,
 * Get_hamiltonian_ndia, Get_hamiltonian_dia and update_trun_dia/ndia
 * (block.f90:382-1503, get_sys.f90:507-759); same arguments and two-call
 * result as tj_get_hamiltonian. */
int ora_get_hamiltonian(const tj_lattice *lat, int side, int mshift, const tj_model *pre, const tj_basis *basis,
                        const tj_block *trun, tj_model_result *out);

/* wave_trans_LR (direction 0, code/tjsq/dmrg_sub.f90:1093-1238) and
 * wave_trans_RL (direction 1, dmrg_sub.f90:1242-1384): the wavefunction of
 * the last step carried to the next superblock; new_wave's sectors are set
 * by the caller (allocate_wave), its data is overwritten and normalised. */
int ora_wave_trans(int direction, const tj_basis *sys_bs, const tj_basis *env_bs, const tj_block *sys_trun,
                   const tj_block *env_trun, const tj_wave *old_wave, tj_wave *new_wave);

/* Get_{sys,env}_oper_{dia,ndia} (code/tjsq/get_sys.f90:764-891, 998-1130),
 * Change_{sys,env}_oper_{dia,ndia} (get_sys.f90:893-996, 1134-1238),
 * block_mul_block_ndia (block.f90:1956-2197) and update_trun_dia / ndia
 * (block.f90:1311-1503); arguments and two-call results as tj_get_oper,
 * tj_change_oper, tj_block_mul_block_ndia and tj_update_trun. */
int ora_get_oper(int side, int dia, const tj_chain *ch, const tj_block *st_oper, int old_idx, int new_idx,
                 int truns, char types, tj_block_result *out);
int ora_change_oper(int side, int dia, const tj_chain *ch, const tj_block *old_oper, int old_idx, int new_idx,
                    int truns, char types, tj_block_result *out);
int ora_block_mul_block_ndia(const tj_block *o1, char f1, const tj_block *o2, char f2, double coef, int down_dif,
                             const tj_basis *basis, tj_block_result *out);
int ora_update_trun(int dia, const tj_block *ori, const tj_block *trun, tj_block_result *out);

/* Site operators of Get_site_operator_su2_U0 (code/tjsq/dmrg_sub.f90:370-473):
 * which = 0 st_elec_up, 1 st_elec_down, 2 num_elec, 3 st_sd, 4 st_si.
 * Writes at most 2 sub-blocks and 2 doubles; returns the sub count. */
int ora_site_operator(int which, int up_bias, tj_block *blk, tj_block_sub *subs, double *vals);

const char *ora_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
