/*
 * oracle_tj.c -- CPU restatement of the tjsq hot path (TEST INFRASTRUCTURE).
 *
 * Only the test-suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * use this file; the product library never links it.  Each function names the
 * Fortran routine of DongNingSheng/Grand_SQL_tJ (code/tjsq) it restates and
 * follows that routine's loop nest, look-up order, coefficient formula and
 * DGEMM sequence; unreachable code of the reference (the blocks after an
 * unconditional `go to`) is not restated.  Parity is unpinned: the reference
 * cannot be compiled here (no Fortran compiler) and ships no golden vectors.
 *
 * Arrays are 0-based here; comments use the reference's 1-based names.
 */
#define _GNU_SOURCE
#include "oracle_tj.h"

#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ errors */
static __thread char g_err[512];
static int fail(int code, const char *msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}
const char *ora_last_error(void) { return g_err; }

/* ------------------------------------------------------- BLAS/LAPACK */
typedef void (*dgemm_fn)(const char *, const char *, const int *, const int *, const int *,
                         const double *, const double *, const int *, const double *,
                         const int *, const double *, double *, const int *, size_t, size_t);
typedef void (*dsyev_fn)(const char *, const char *, const int *, double *, const int *,
                         double *, double *, const int *, int *, size_t, size_t);
typedef void (*dstev_fn)(const char *, const int *, double *, double *, double *, const int *,
                         double *, int *, size_t);
typedef void (*setthr_fn)(int);
static dgemm_fn p_dgemm;
static dsyev_fn p_dsyev;
static dstev_fn p_dstev;
static setthr_fn p_setthr;

int ora_init(const char *libpath, int threads) {
  void *h = dlopen(libpath, RTLD_NOW | RTLD_LOCAL);
  if (!h) return fail(TJ_ERR_ARG, "ora_init: dlopen failed");
  p_dgemm = (dgemm_fn)dlsym(h, "scipy_dgemm_");
  p_dsyev = (dsyev_fn)dlsym(h, "scipy_dsyev_");
  p_dstev = (dstev_fn)dlsym(h, "scipy_dstev_");
  p_setthr = (setthr_fn)dlsym(h, "scipy_openblas_set_num_threads");
  if (!p_dgemm || !p_dsyev || !p_dstev) return fail(TJ_ERR_ARG, "ora_init: symbols missing");
  if (threads > 0 && p_setthr) p_setthr(threads);
  return 0;
}
int ora_set_threads(int threads) {
  if (!p_setthr) return fail(TJ_ERR_ARG, "ora_set_threads: not initialised");
  p_setthr(threads);
  return 0;
}

/* column-major DGEMM; zero-sized calls are no-ops as in reference BLAS */
static void dg(char ta, char tb, int m, int n, int k, double alpha, const double *a, int lda,
               const double *b, int ldb, double beta, double *c, int ldc) {
  if (m <= 0 || n <= 0) return;
  if (lda < 1) lda = 1;
  if (ldb < 1) ldb = 1;
  if (ldc < 1) ldc = 1;
  p_dgemm(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc, 1, 1);
}

/* ------------------------------------------------- FACTRL, W3JS, W6JS */
/* FACTRL (block.f90:1508-1516) fills fact(0:142); the rest of fact(0:301) stays 0. */
static double fact[302];
static int fact_ready;
static void factrl(void) {
  if (fact_ready) return;
  memset(fact, 0, sizeof fact);
  fact[0] = 1.0;
  for (int i = 1; i <= 142; i++) fact[i] = fact[i - 1] * (double)(float)i;
  fact_ready = 1;
}
static double F(int i) { return (i >= 0 && i <= 301) ? fact[i] : 0.0; }

/* W3JS (block.f90:1522-1561) */
double ora_w3js(int j1, int j2, int j3, int m1, int m2, int m3) {
  factrl();
  if (m1 + m2 + m3 != 0) return 0.0;
  int ia = j1 + j2;
  if (j3 > ia) return 0.0;
  int ib = j1 - j2;
  if (j3 < abs(ib)) return 0.0;
  int jsum = j3 + ia, ic = j1 - m1, id = j2 - m2;
  if (jsum % 2 || ic % 2 || id % 2) return 0.0;
  if (abs(m1) > j1 || abs(m2) > j2 || abs(m3) > j3) return 0.0;
  int ie = j3 - j2 + m1, iff = j3 - j1 - m2;
  int zmin = 0;
  if (-ie > zmin) zmin = -ie;
  if (-iff > zmin) zmin = -iff;
  int ig = ia - j3, ih = j2 + m2;
  int zmax = ig;
  if (ih < zmax) zmax = ih;
  if (ic < zmax) zmax = ic;
  double cc = 0.0;
  for (int z = zmin; z <= zmax; z += 2) {
    double denom = F(z / 2) * F((ig - z) / 2) * F((ic - z) / 2) * F((ih - z) / 2) *
                   F((ie + z) / 2) * F((iff + z) / 2);
    if (z % 4 != 0) denom = -denom;
    cc += 1.0 / denom;
  }
  double cc1 = F(ig / 2) * F((j3 + ib) / 2) * F((j3 - ib) / 2) / F((jsum + 2) / 2);
  double cc2 = F((j1 + m1) / 2) * F(ic / 2) * F(ih / 2) * F(id / 2) * F((j3 - m3) / 2) *
               F((j3 + m3) / 2);
  cc = cc * sqrt(cc1 * cc2);
  if ((ib - m3) % 4 != 0) cc = -cc;
  return cc;
}

/* W6JS (block.f90:1564-1615): Racah's formula on doubled spins. */
double ora_w6js(int j1, int j2, int j3, int l1, int l2, int l3) {
  factrl();
  int ia = j1 + j2;
  if (ia < j3) return 0.0;
  int ib = j1 - j2;
  if (abs(ib) > j3) return 0.0;
  int ic = j1 + l2;
  if (ic < l3) return 0.0;
  int id = j1 - l2;
  if (abs(id) > l3) return 0.0;
  int ie = l1 + j2;
  if (ie < l3) return 0.0;
  int iff = l1 - j2;
  if (abs(iff) > l3) return 0.0;
  int ig = l1 + l2;
  if (ig < j3) return 0.0;
  int ih = l1 - l2;
  if (abs(ih) > j3) return 0.0;
  int s1 = ia + j3, s2 = ic + l3, s3 = ie + l3, s4 = ig + j3;
  if (s1 % 2 || s2 % 2 || s3 % 2 || s4 % 2) return 0.0;
  int wmin = s1;
  if (s2 > wmin) wmin = s2;
  if (s3 > wmin) wmin = s3;
  if (s4 > wmin) wmin = s4;
  int ii = ia + ig, ij = j2 + j3 + l2 + l3, ik = j3 + j1 + l3 + l1;
  int wmax = ii;
  if (ij < wmax) wmax = ij;
  if (ik < wmax) wmax = ik;
  double omega = 0.0;
  for (int w = wmin; w <= wmax; w += 2) {
    double denom = F((w - s1) / 2) * F((w - s2) / 2) * F((w - s3) / 2) * F((w - s4) / 2) *
                   F((ii - w) / 2) * F((ij - w) / 2) * F((ik - w) / 2);
    if (w % 4 != 0) denom = -denom;
    omega += F(w / 2 + 1) / denom;
  }
  double t1 = F((ia - j3) / 2) * F((j3 + ib) / 2) * F((j3 - ib) / 2) / F(s1 / 2 + 1);
  double t2 = F((ic - l3) / 2) * F((l3 + id) / 2) * F((l3 - id) / 2) / F(s2 / 2 + 1);
  double t3 = F((ie - l3) / 2) * F((l3 + iff) / 2) * F((l3 - iff) / 2) / F(s3 / 2 + 1);
  double t4 = F((ig - j3) / 2) * F((j3 + ih) / 2) * F((j3 - ih) / 2) / F(s4 / 2 + 1);
  return omega * sqrt(t1 * t2 * t3 * t4);
}
#define W6 ora_w6js
static double ipow_m1(int n) { return (n % 2) ? -1.0 : 1.0; } /* (-1)**n, n >= 0 */

/* ---------------------------------------------------- block storage */
/* Mutable mirror of Total_Block for the operators hmerge builds and the
 * transposes model_wave makes. */
typedef struct {
  int num_up, num_down, down_dif, row_dim, sdim;
  double *mat;
} OSub;
typedef struct {
  int len, num, dim, up_dif, down_dif;
  OSub *sub;
  int owns;
} OBlk;
enum { EU = 0, ED = 1, SD = 2, SZ = 3, SN = 4 };
typedef struct { OBlk op[5]; } OSet;

static void blk_view(const tj_block *b, OBlk *o) {
  memset(o, 0, sizeof *o);
  o->len = b->len; o->num = b->num; o->dim = b->dim; o->up_dif = b->up_dif; o->down_dif = b->down_dif;
  o->sub = (OSub *)calloc(b->num > 0 ? b->num : 1, sizeof(OSub));
  for (int i = 0; i < b->num; i++) {
    o->sub[i].num_up = b->sub[i].num_up; o->sub[i].num_down = b->sub[i].num_down;
    o->sub[i].down_dif = b->sub[i].down_dif; o->sub[i].row_dim = b->sub[i].row_dim;
    o->sub[i].sdim = b->sub[i].sdim; o->sub[i].mat = (double *)(b->data + b->sub[i].off);
  }
  o->owns = 0;
}
static void blk_free(OBlk *o) {
  if (!o->sub) return;
  if (o->owns)
    for (int i = 0; i < o->num; i++) free(o->sub[i].mat);
  free(o->sub);
  o->sub = NULL;
  o->num = 0;
}
/* block_pass_info (block.f90:1741-1768): same structure, zero matrices. */
static void blk_pass_info(const OBlk *old, OBlk *nw) {
  blk_free(nw);
  *nw = *old;
  nw->owns = 1;
  nw->sub = (OSub *)calloc(old->num > 0 ? old->num : 1, sizeof(OSub));
  for (int i = 0; i < old->num; i++) {
    nw->sub[i] = old->sub[i];
    nw->sub[i].mat = (double *)calloc((size_t)old->sub[i].row_dim * old->sub[i].sdim + 1, sizeof(double));
  }
}
/* block_transfer_trans (block.f90:1676-1706). */
static void blk_trans(const OBlk *in, OBlk *out) {
  memset(out, 0, sizeof *out);
  out->len = in->len; out->num = in->num; out->dim = 0;
  out->up_dif = -in->up_dif; out->down_dif = in->down_dif;
  out->owns = 1;
  out->sub = (OSub *)calloc(in->num > 0 ? in->num : 1, sizeof(OSub));
  for (int i = 0; i < in->num; i++) {
    const OSub *s = &in->sub[i];
    OSub *t = &out->sub[i];
    t->num_up = s->num_up + in->up_dif;
    t->num_down = s->num_down + s->down_dif;
    t->down_dif = -s->down_dif;
    t->row_dim = s->sdim;
    t->sdim = s->row_dim;
    out->dim += t->sdim;
    t->mat = (double *)malloc(((size_t)t->row_dim * t->sdim + 1) * sizeof(double));
    for (int c = 0; c < t->sdim; c++)
      for (int r = 0; r < t->row_dim; r++) t->mat[(size_t)c * t->row_dim + r] = s->mat[(size_t)r * s->row_dim + c];
  }
}
/* block_add_block_two (block.f90:1786-1822): the search for the next
 * matching sub-block restarts after the previous match. */
static void blk_add_two(const OBlk *b1, double coef, OBlk *nw) {
  int x1 = 0;
  for (int i = 0; i < nw->num; i++) {
    int found = -1;
    for (int x = x1; x < b1->num; x++) {
      if (b1->sub[x].num_up == nw->sub[i].num_up && b1->sub[x].num_down == nw->sub[i].num_down &&
          b1->sub[x].down_dif == nw->sub[i].down_dif) {
        found = x;
        x1 = x + 1;
        break;
      }
    }
    if (found >= 0) {
      size_t n = (size_t)nw->sub[i].row_dim * nw->sub[i].sdim;
      for (size_t e = 0; e < n; e++) nw->sub[i].mat[e] += coef * b1->sub[found].mat[e];
    }
  }
}

/* ------------------------------------------------ basis / wave access */
static inline const tj_basis_sub *BM(const tj_basis *b, int x, int m) { return &b->maps[b->sub[x].first + m]; }
static inline double *WV(const tj_wave *w, int i) { return w->data + w->sub[i].off; }
static inline int LD(const tj_wave *w, int i) { return w->sub[i].sys_dim; }
/* element (r, c) of sector i (0-based row r, column c) */
static inline double *WP(const tj_wave *w, int i, int r, int c) {
  return w->data + w->sub[i].off + (size_t)c * w->sub[i].sys_dim + r;
}
static int find_out(const tj_wave *w, int su, int sd, int eu, int ed) {
  for (int k = 0; k < w->num; k++)
    if (w->sub[k].sys_num_up == su && w->sub[k].sys_num_down == sd && w->sub[k].env_num_up == eu &&
        w->sub[k].env_num_down == ed)
      return k;
  return -1;
}
/* first sub-block of `b` with (num_up, num_down[, down_dif]) */
static int find_sub(const OBlk *b, int nu, int nd, int dd, int use_dd) {
  for (int k = 0; k < b->num; k++)
    if (b->sub[k].num_up == nu && b->sub[k].num_down == nd && (!use_dd || b->sub[k].down_dif == dd)) return k;
  return -1;
}
static int find_bs(const tj_basis *b, int nu, int nd) {
  for (int x = 0; x < b->num; x++)
    if (b->sub[x].new_num_up == nu && b->sub[x].new_num_down == nd) return x;
  return -1;
}
static double sgn_flag(char flag, int n) {
  if (flag == 'B') return 1.0;
  if (flag == 'F') return (n % 2 == 0) ? 1.0 : -1.0;
  return 0.0;
}

/* axpy on a sub-matrix: dst(r0.., c0..) += a * src(r1.., c1..), nr x nc */
static void sub_axpy(double a, const tj_wave *src, int is, int r1, int c1, tj_wave *dst, int id, int r0,
                     int c0, int nr, int nc) {
  for (int c = 0; c < nc; c++) {
    const double *s = WP(src, is, r1, c1 + c);
    double *d = WP(dst, id, r0, c0 + c);
    for (int r = 0; r < nr; r++) d[r] += a * s[r];
  }
}

/* ===================================================== term kernels */
/* block_vec_dia (get_sys.f90:1242-1289) */
static void block_vec_dia(const OBlk *bl, const tj_basis *sbs, const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down, ed = in->sub[i].env_dim;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < sbs->sub[x].num; y++) {
        const tj_basis_sub *m = BM(sbs, x, y);
        double c1 = coef / sqrt(1.0 + m->bl_num_down);
        int k = find_sub(bl, m->bl_num_up, m->bl_num_down, 0, 0);
        if (k < 0) continue;
        dg('N', 'N', m->sdim, ed, m->sdim, c1, bl->sub[k].mat, m->sdim, WP(in, i, m->spos, 0), LD(in, i), 1.0,
           WP(out, i, m->spos, 0), LD(out, i));
      }
    }
  }
}
/* vec_block_dia (get_sys.f90:1293-1340) */
static void vec_block_dia(const OBlk *bl, const tj_basis *ebs, const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down, sdm = in->sub[i].sys_dim;
    for (int x = 0; x < ebs->num; x++) {
      if (ebs->sub[x].new_num_up != eu || ebs->sub[x].new_num_down != edn) continue;
      for (int y = 0; y < ebs->sub[x].num; y++) {
        const tj_basis_sub *m = BM(ebs, x, y);
        double c1 = coef / sqrt(1.0 + m->bl_num_down);
        int k = find_sub(bl, m->bl_num_up, m->bl_num_down, 0, 0);
        if (k < 0) continue;
        dg('N', 'T', sdm, m->sdim, m->sdim, c1, WP(in, i, 0, m->spos), LD(in, i), bl->sub[k].mat, m->sdim, 1.0,
           WP(out, i, 0, m->spos), LD(out, i));
      }
    }
  }
}
/* site_vec_site_dia (get_sys.f90:1609-1705) */
static void site_vec_site_dia(const OBlk *sst, const OBlk *est, const tj_basis *sbs, const tj_basis *ebs,
                              const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int xs = find_bs(sbs, in->sub[i].sys_num_up, in->sub[i].sys_num_down);
    int xe = find_bs(ebs, in->sub[i].env_num_up, in->sub[i].env_num_down);
    if (xs < 0 || xe < 0) continue;
    for (int x = 0; x < sbs->sub[xs].num; x++) {
      const tj_basis_sub *ms = BM(sbs, xs, x);
      int ks = find_sub(sst, ms->st_num_up, ms->st_num_down, 0, 0);
      for (int y = 0; y < ebs->sub[xe].num; y++) {
        const tj_basis_sub *me = BM(ebs, xe, y);
        int ke = find_sub(est, me->st_num_up, me->st_num_down, 0, 0);
        if (ks < 0 || ke < 0) continue;
        double ct = coef * sst->sub[ks].mat[0] * est->sub[ke].mat[0];
        ct = ct / sqrt((1.0 + ms->st_num_down) * (1.0 + me->st_num_down));
        sub_axpy(ct, in, i, ms->spos, me->spos, out, i, ms->spos, me->spos, ms->sdim, me->sdim);
      }
    }
  }
}
/* site_vec_site_ndia (get_sys.f90:3761-4124, live 3794-3994) */
static void site_vec_site_ndia(const OBlk *sst, char fst, const OBlk *est, char fet, const tj_basis *sbs,
                               const tj_basis *ebs, const tj_wave *in, tj_wave *out, double coef) {
  int up_dif = sst->up_dif, d1 = sst->down_dif;
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down;
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < ebs->num; y++) {
        if (ebs->sub[y].new_num_up != eu || ebs->sub[y].new_num_down != edn) continue;
        for (int m = 0; m < sbs->sub[x].num; m++) {
          const tj_basis_sub *ms = BM(sbs, x, m);
          for (int n = 0; n < ebs->sub[y].num; n++) {
            const tj_basis_sub *me = BM(ebs, y, n);
            int nss_up = 0, nss_dn = 0;
            for (int sdd1 = -sst->down_dif; sdd1 <= sst->down_dif; sdd1 += 2) {
              int ks = -1;
              for (int k = 0; k < sst->num; k++)
                if (sst->sub[k].num_up == ms->st_num_up && sst->sub[k].num_down == ms->st_num_down &&
                    sst->sub[k].down_dif == sdd1) {
                  ks = k;
                  nss_up = ms->st_num_up + up_dif;
                  nss_dn = ms->st_num_down + sdd1;
                  break;
                }
              for (int sdd2 = -est->down_dif; sdd2 <= est->down_dif; sdd2 += 2) {
                int nes_up = me->st_num_up - up_dif, nes_dn = me->st_num_down - sdd2;
                int ke = find_sub(est, nes_up, nes_dn, sdd2, 1);
                int nsu = su + up_dif, neu = eu - up_dif;
                if (ks < 0 || ke < 0) continue;
                for (int nsd = abs(sd - sst->down_dif); nsd <= sd + sst->down_dif; nsd += 2) {
                  int ned = nsd;
                  int nsp = -1, nep = -1;
                  for (int k = 0; k < sbs->num && nsp < 0; k++) {
                    if (sbs->sub[k].new_num_up != nsu || sbs->sub[k].new_num_down != nsd) continue;
                    for (int l = 0; l < sbs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(sbs, k, l);
                      if (q->st_num_up == nss_up && q->st_num_down == nss_dn && q->bl_num_down == ms->bl_num_down) {
                        nsp = q->spos;
                        break;
                      }
                    }
                  }
                  for (int k = 0; k < ebs->num && nep < 0; k++) {
                    if (ebs->sub[k].new_num_up != neu || ebs->sub[k].new_num_down != ned) continue;
                    for (int l = 0; l < ebs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(ebs, k, l);
                      if (q->st_num_up == nes_up && q->st_num_down == nes_dn && q->bl_num_down == me->bl_num_down) {
                        nep = q->spos;
                        break;
                      }
                    }
                  }
                  if (nsp < 0 || nep < 0) continue;
                  int ko = find_out(out, nsu, nsd, neu, ned);
                  if (ko < 0) continue;
                  double ss = sgn_flag(fst, ms->bl_num_down), se = sgn_flag(fet, sd);
                  double ct = ss * se * coef;
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->st_num_down, j5 = ms->bl_num_down, j6 = nss_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->st_num_down, j55 = me->bl_num_down, j66 = nes_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  double c11 = W6(j11, j22, j33, j44, j55, j66);
                  if (c11 == 0.0) continue;
                  c1 *= c11;
                  if (c1 != 0.0) {
                    c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                    if (((j55 + j44 + j11 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                    c1 = ct * c1 * sst->sub[ks].mat[0] * est->sub[ke].mat[0];
                    sub_axpy(c1, in, i, ms->spos, me->spos, out, ko, nsp, nep, ms->sdim, me->sdim);
                    if (d1 == 1) sub_axpy(c1, in, ko, nsp, nep, out, i, ms->spos, me->spos, ms->sdim, me->sdim);
                  }
                }
              }
            }
          }
        }
      }
    }
  }
}
/* block_site_vec_ndia (get_sys.f90:2016-2265, live 2047-2170) */
static int block_site_vec_ndia(const OBlk *bl, char fbl, const OBlk *st, char fst, const tj_basis *sbs,
                               const tj_wave *in, tj_wave *out, double coef) {
  (void)fbl;
  int up_dif = bl->up_dif, d1 = bl->down_dif;
  if (up_dif != st->up_dif || d1 != st->down_dif) return fail(TJ_ERR_QN, "Quantum number error in block_site_vec!");
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down, ed = in->sub[i].env_dim;
    for (int k = 0; k < sbs->num; k++) {
      if (sbs->sub[k].new_num_up != su || sbs->sub[k].new_num_down != sd) continue;
      for (int x = 0; x < sbs->sub[k].num; x++) {
        const tj_basis_sub *m = BM(sbs, k, x);
        for (int dd = -d1; dd <= d1; dd += 2) {
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            int kb = find_sub(bl, m->bl_num_up, m->bl_num_down, dd, 1);
            int nst_up = m->st_num_up - up_dif, nst_dn = m->st_num_down - sdd;
            int ks = find_sub(st, nst_up, nst_dn, sdd, 1);
            int nbl_up = m->bl_num_up + up_dif, nbl_dn = m->bl_num_down + dd;
            if (kb < 0 || ks < 0) continue;
            int np = -1, nd = 0;
            for (int y = 0; y < sbs->sub[k].num; y++) {
              const tj_basis_sub *q = BM(sbs, k, y);
              if (q->bl_num_up == nbl_up && q->bl_num_down == nbl_dn && q->st_num_up == nst_up &&
                  q->st_num_down == nst_dn) {
                np = q->spos;
                nd = q->sdim;
                break;
              }
            }
            if (np < 0) continue;
            double sst = sgn_flag(fst, m->bl_num_down);
            int j1 = nbl_dn, j2 = m->bl_num_down, j3 = d1, j4 = m->st_num_down, j5 = nst_dn, j6 = sd;
            double c1 = W6(j1, j2, j3, j4, j5, j6);
            if (c1 != 0.0) {
              c1 = c1 * ipow_m1((j2 + j5 + j3 + j6) / 2) / sqrt(1.0 + d1);
              double ct = sst * c1 * coef * st->sub[ks].mat[0];
              dg('N', 'N', nd, ed, m->sdim, ct, bl->sub[kb].mat, nd, WP(in, i, m->spos, 0), LD(in, i), 1.0,
                 WP(out, i, np, 0), LD(out, i));
              if (d1 == 1)
                dg('T', 'N', m->sdim, ed, nd, ct, bl->sub[kb].mat, nd, WP(in, i, np, 0), LD(in, i), 1.0,
                   WP(out, i, m->spos, 0), LD(out, i));
            }
          }
        }
      }
    }
  }
  return 0;
}
/* block_site_vec_dia (get_sys.f90:1460-1530) */
static void block_site_vec_dia(const OBlk *bl, const OBlk *st, const tj_basis *sbs, const tj_wave *in, tj_wave *out,
                               double coef) {
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down, ed = in->sub[i].env_dim;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < sbs->sub[x].num; y++) {
        const tj_basis_sub *m = BM(sbs, x, y);
        int kb = find_sub(bl, m->bl_num_up, m->bl_num_down, 0, 0);
        int ks = find_sub(st, m->st_num_up, m->st_num_down, 0, 0);
        if (kb < 0 || ks < 0) continue;
        double ct = coef * st->sub[ks].mat[0];
        ct = ct / sqrt((1.0 + m->bl_num_down) * (1.0 + m->st_num_down));
        dg('N', 'N', m->sdim, ed, m->sdim, ct, bl->sub[kb].mat, m->sdim, WP(in, i, m->spos, 0), LD(in, i), 1.0,
           WP(out, i, m->spos, 0), LD(out, i));
      }
    }
  }
}
/* vec_block_site_ndia (get_sys.f90:2269-2552, live 2301-2446) */
static int vec_block_site_ndia(const OBlk *bl, char fbl, const OBlk *st, char fst, const tj_basis *ebs,
                               const tj_wave *in, tj_wave *out, double coef) {
  int up_dif = bl->up_dif, d1 = bl->down_dif;
  if (up_dif != st->up_dif || d1 != st->down_dif) return fail(TJ_ERR_QN, "Quantum number error in vec_block_site!");
  for (int i = 0; i < in->num; i++) {
    int sd = in->sub[i].sys_num_down, eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down;
    int sdm = in->sub[i].sys_dim;
    for (int k = 0; k < ebs->num; k++) {
      if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
      for (int x = 0; x < ebs->sub[k].num; x++) {
        const tj_basis_sub *m = BM(ebs, k, x);
        for (int bdd = -d1; bdd <= d1; bdd += 2) {
          int kb = find_sub(bl, m->bl_num_up, m->bl_num_down, bdd, 1);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            int nst_up = m->st_num_up - up_dif, nst_dn = m->st_num_down - sdd;
            int ks = find_sub(st, nst_up, nst_dn, sdd, 1);
            int nbl_up = m->bl_num_up + up_dif, nbl_dn = m->bl_num_down + bdd;
            if (ks < 0 || kb < 0) continue;
            int np = -1, nd = 0;
            for (int y = 0; y < ebs->sub[k].num; y++) {
              const tj_basis_sub *q = BM(ebs, k, y);
              if (q->bl_num_up == nbl_up && q->bl_num_down == nbl_dn && q->st_num_up == nst_up &&
                  q->st_num_down == nst_dn) {
                np = q->spos;
                nd = q->sdim;
                break;
              }
            }
            if (np < 0) continue;
            double sbl = sgn_flag(fbl, sd + nst_dn), sst = sgn_flag(fst, sd);
            int j1 = nbl_dn, j2 = m->bl_num_down, j3 = d1, j4 = m->st_num_down, j5 = nst_dn, j6 = edn;
            double c1 = W6(j1, j2, j3, j4, j5, j6);
            if (c1 != 0.0) {
              c1 = c1 * ipow_m1((j2 + j5 + j3 + j6) / 2) / sqrt(1.0 + d1);
              double ct = sbl * sst * c1 * coef * st->sub[ks].mat[0];
              dg('N', 'T', sdm, nd, m->sdim, ct, WP(in, i, 0, m->spos), LD(in, i), bl->sub[kb].mat, nd, 1.0,
                 WP(out, i, 0, np), LD(out, i));
              if (d1 == 1)
                dg('N', 'N', sdm, m->sdim, nd, ct, WP(in, i, 0, np), LD(in, i), bl->sub[kb].mat, nd, 1.0,
                   WP(out, i, 0, m->spos), LD(out, i));
            }
          }
        }
      }
    }
  }
  return 0;
}
/* vec_block_site_dia (get_sys.f90:1534-1605) */
static void vec_block_site_dia(const OBlk *bl, const OBlk *st, const tj_basis *ebs, const tj_wave *in, tj_wave *out,
                               double coef) {
  for (int i = 0; i < in->num; i++) {
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down, sdm = in->sub[i].sys_dim;
    for (int x = 0; x < ebs->num; x++) {
      if (ebs->sub[x].new_num_up != eu || ebs->sub[x].new_num_down != edn) continue;
      for (int y = 0; y < ebs->sub[x].num; y++) {
        const tj_basis_sub *m = BM(ebs, x, y);
        int kb = find_sub(bl, m->bl_num_up, m->bl_num_down, 0, 0);
        int ks = find_sub(st, m->st_num_up, m->st_num_down, 0, 0);
        if (kb < 0 || ks < 0) continue;
        double ct = coef * st->sub[ks].mat[0];
        ct = ct / sqrt((1.0 + m->bl_num_down) * (1.0 + m->st_num_down));
        dg('N', 'T', sdm, m->sdim, m->sdim, ct, WP(in, i, 0, m->spos), LD(in, i), bl->sub[kb].mat, m->sdim, 1.0,
           WP(out, i, 0, m->spos), LD(out, i));
      }
    }
  }
}
/* block_vec_site_ndia (get_sys.f90:2984-3351, live 3021-3209) */
static int block_vec_site_ndia(const OBlk *bl, char fsl, const OBlk *st, char fet, const tj_basis *sbs,
                               const tj_basis *ebs, const tj_wave *in, tj_wave *out, double coef) {
  (void)fsl;
  int up_dif = bl->up_dif, d1 = bl->down_dif;
  if (up_dif != st->up_dif || d1 != st->down_dif) return fail(TJ_ERR_QN, "Quantum number error in block_vec_site!");
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down;
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < ebs->num; y++) {
        if (ebs->sub[y].new_num_up != eu || ebs->sub[y].new_num_down != edn) continue;
        for (int m = 0; m < sbs->sub[x].num; m++) {
          const tj_basis_sub *ms = BM(sbs, x, m);
          for (int n = 0; n < ebs->sub[y].num; n++) {
            const tj_basis_sub *me = BM(ebs, y, n);
            for (int bdd = -bl->down_dif; bdd <= bl->down_dif; bdd += 2) {
              int nbl_up = ms->bl_num_up + up_dif, nbl_dn = ms->bl_num_down + bdd;
              int kb = find_sub(bl, ms->bl_num_up, ms->bl_num_down, bdd, 1);
              for (int sdd = -st->down_dif; sdd <= st->down_dif; sdd += 2) {
                int nes_up = me->st_num_up - up_dif, nes_dn = me->st_num_down - sdd;
                int ks = find_sub(st, nes_up, nes_dn, sdd, 1);
                int nsu = su + up_dif, neu = eu - up_dif;
                if (kb < 0 || ks < 0) continue;
                for (int nsd = abs(sd - bl->down_dif); nsd <= sd + bl->down_dif; nsd += 2) {
                  int ned = nsd, nsp = -1, nsdim = 0, nep = -1;
                  for (int k = 0; k < sbs->num && nsp < 0; k++) {
                    if (sbs->sub[k].new_num_up != nsu || sbs->sub[k].new_num_down != nsd) continue;
                    for (int l = 0; l < sbs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(sbs, k, l);
                      if (q->bl_num_up == nbl_up && q->bl_num_down == nbl_dn && q->st_num_down == ms->st_num_down) {
                        nsp = q->spos;
                        nsdim = q->sdim;
                        break;
                      }
                    }
                  }
                  for (int k = 0; k < ebs->num && nep < 0; k++) {
                    if (ebs->sub[k].new_num_up != neu || ebs->sub[k].new_num_down != ned) continue;
                    for (int l = 0; l < ebs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(ebs, k, l);
                      if (q->st_num_up == nes_up && q->st_num_down == nes_dn && q->bl_num_down == me->bl_num_down) {
                        nep = q->spos;
                        break;
                      }
                    }
                  }
                  if (nsp < 0 || nep < 0) continue;
                  int ko = find_out(out, nsu, nsd, neu, ned);
                  if (ko < 0) continue;
                  double set = sgn_flag(fet, sd);
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->bl_num_down, j5 = ms->st_num_down, j6 = nbl_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->st_num_down, j55 = me->bl_num_down, j66 = nes_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  double c11 = W6(j11, j22, j33, j44, j55, j66);
                  if (c11 == 0.0) continue;
                  c1 *= c11;
                  if (c1 != 0.0) {
                    c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                    if (((j6 + j5 + j3 + j2) / 2 + (j55 + j44 + j11 + j22) / 2) % 2 != 0) c1 = -c1;
                    double ct = set * c1 * coef * st->sub[ks].mat[0];
                    dg('N', 'N', nsdim, me->sdim, ms->sdim, ct, bl->sub[kb].mat, nsdim,
                       WP(in, i, ms->spos, me->spos), LD(in, i), 1.0, WP(out, ko, nsp, nep), LD(out, ko));
                    if (d1 == 1)
                      dg('T', 'N', ms->sdim, me->sdim, nsdim, ct, bl->sub[kb].mat, nsdim, WP(in, ko, nsp, nep),
                         LD(in, ko), 1.0, WP(out, i, ms->spos, me->spos), LD(out, i));
                  }
                }
              }
            }
          }
        }
      }
    }
  }
  return 0;
}
/* block_vec_site_dia (get_sys.f90:1709-1805) */
static void block_vec_site_dia(const OBlk *bl, const OBlk *st, const tj_basis *sbs, const tj_basis *ebs,
                               const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int xs = find_bs(sbs, in->sub[i].sys_num_up, in->sub[i].sys_num_down);
    int xe = find_bs(ebs, in->sub[i].env_num_up, in->sub[i].env_num_down);
    if (xs < 0 || xe < 0) continue;
    for (int x = 0; x < sbs->sub[xs].num; x++) {
      const tj_basis_sub *ms = BM(sbs, xs, x);
      int kb = find_sub(bl, ms->bl_num_up, ms->bl_num_down, 0, 0);
      for (int y = 0; y < ebs->sub[xe].num; y++) {
        const tj_basis_sub *me = BM(ebs, xe, y);
        int ks = find_sub(st, me->st_num_up, me->st_num_down, 0, 0);
        if (kb < 0 || ks < 0) continue;
        double ct = coef * st->sub[ks].mat[0];
        ct = ct / sqrt((1.0 + me->st_num_down) * (1.0 + ms->bl_num_down));
        dg('N', 'N', ms->sdim, me->sdim, ms->sdim, ct, bl->sub[kb].mat, ms->sdim, WP(in, i, ms->spos, me->spos),
           LD(in, i), 1.0, WP(out, i, ms->spos, me->spos), LD(out, i));
      }
    }
  }
}
/* site_vec_block_ndia (get_sys.f90:3355-3757, live 3391-3604) */
static int site_vec_block_ndia(const OBlk *st, char fst, const OBlk *bl, char fel, const tj_basis *sbs,
                               const tj_basis *ebs, const tj_wave *in, tj_wave *out, double coef) {
  int up_dif = st->up_dif, d1 = st->down_dif;
  if (up_dif != bl->up_dif || d1 != bl->down_dif) return fail(TJ_ERR_QN, "Quantum number error in site_vec_block!");
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down;
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < ebs->num; y++) {
        if (ebs->sub[y].new_num_up != eu || ebs->sub[y].new_num_down != edn) continue;
        for (int m = 0; m < sbs->sub[x].num; m++) {
          const tj_basis_sub *ms = BM(sbs, x, m);
          for (int n = 0; n < ebs->sub[y].num; n++) {
            const tj_basis_sub *me = BM(ebs, y, n);
            for (int sdd = -st->down_dif; sdd <= st->down_dif; sdd += 2) {
              int nss_up = ms->st_num_up + up_dif, nss_dn = ms->st_num_down + sdd;
              int ks = find_sub(st, ms->st_num_up, ms->st_num_down, sdd, 1);
              for (int bdd = -bl->down_dif; bdd <= bl->down_dif; bdd += 2) {
                int neb_up = me->bl_num_up - up_dif, neb_dn = me->bl_num_down - bdd;
                int kb = find_sub(bl, neb_up, neb_dn, bdd, 1);
                int nsu = su + up_dif, neu = eu - up_dif;
                if (ks < 0 || kb < 0) continue;
                for (int nsd = abs(sd - st->down_dif); nsd <= sd + st->down_dif; nsd += 2) {
                  int ned = nsd, nsp = -1, nep = -1, nedim = 0;
                  for (int k = 0; k < sbs->num && nsp < 0; k++) {
                    if (sbs->sub[k].new_num_up != nsu || sbs->sub[k].new_num_down != nsd) continue;
                    for (int l = 0; l < sbs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(sbs, k, l);
                      if (q->st_num_up == nss_up && q->st_num_down == nss_dn && q->bl_num_down == ms->bl_num_down &&
                          q->bl_num_up == ms->bl_num_up) {
                        nsp = q->spos;
                        break;
                      }
                    }
                  }
                  for (int k = 0; k < ebs->num && nep < 0; k++) {
                    if (ebs->sub[k].new_num_up != neu || ebs->sub[k].new_num_down != ned) continue;
                    for (int l = 0; l < ebs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(ebs, k, l);
                      if (q->bl_num_up == neb_up && q->bl_num_down == neb_dn && q->st_num_up == me->st_num_up &&
                          q->st_num_down == me->st_num_down) {
                        nep = q->spos;
                        nedim = q->sdim;
                        break;
                      }
                    }
                  }
                  if (nsp < 0 || nep < 0) continue;
                  int ko = find_out(out, nsu, nsd, neu, ned);
                  if (ko < 0) continue;
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->st_num_down, j5 = ms->bl_num_down, j6 = nss_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->bl_num_down, j55 = me->st_num_down, j66 = neb_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  double c11 = W6(j11, j22, j33, j44, j55, j66);
                  if (c11 == 0.0) continue;
                  c1 *= c11;
                  if (c1 != 0.0) {
                    c1 *= sqrt((1.0 + j11) * (j33 + 1.0) / (1.0 + d1));
                    if (((j66 + j55 + j33 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                    double sst = sgn_flag(fst, ms->bl_num_down);
                    double sel = sgn_flag(fel, sd + me->st_num_down);
                    double ct = sst * sel * c1 * coef * st->sub[ks].mat[0];
                    dg('N', 'N', ms->sdim, nedim, me->sdim, ct, WP(in, i, ms->spos, me->spos), LD(in, i),
                       bl->sub[kb].mat, me->sdim, 1.0, WP(out, ko, nsp, nep), LD(out, ko));
                    if (d1 == 1)
                      dg('N', 'T', ms->sdim, me->sdim, nedim, ct, WP(in, ko, nsp, nep), LD(in, ko), bl->sub[kb].mat,
                         me->sdim, 1.0, WP(out, i, ms->spos, me->spos), LD(out, i));
                  }
                }
              }
            }
          }
        }
      }
    }
  }
  return 0;
}
/* site_vec_block_dia (get_sys.f90:1809-1906) */
static void site_vec_block_dia(const OBlk *st, const OBlk *bl, const tj_basis *sbs, const tj_basis *ebs,
                               const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int xs = find_bs(sbs, in->sub[i].sys_num_up, in->sub[i].sys_num_down);
    int xe = find_bs(ebs, in->sub[i].env_num_up, in->sub[i].env_num_down);
    if (xs < 0 || xe < 0) continue;
    for (int x = 0; x < sbs->sub[xs].num; x++) {
      const tj_basis_sub *ms = BM(sbs, xs, x);
      int ks = find_sub(st, ms->st_num_up, ms->st_num_down, 0, 0);
      for (int y = 0; y < ebs->sub[xe].num; y++) {
        const tj_basis_sub *me = BM(ebs, xe, y);
        int kb = find_sub(bl, me->bl_num_up, me->bl_num_down, 0, 0);
        if (ks < 0 || kb < 0) continue;
        double ct = coef * st->sub[ks].mat[0];
        ct = ct / sqrt((1.0 + me->bl_num_down) * (1.0 + ms->st_num_down));
        dg('N', 'T', ms->sdim, me->sdim, me->sdim, ct, WP(in, i, ms->spos, me->spos), LD(in, i), bl->sub[kb].mat,
           me->sdim, 1.0, WP(out, i, ms->spos, me->spos), LD(out, i));
      }
    }
  }
}
/* block_vec_block_ndia (get_sys.f90:2555-2981, live 2595-2834 with 2800-2823) */
static int block_vec_block_ndia(const OBlk *sbl, char fsl, const OBlk *ebl, char fel, const tj_basis *sbs,
                                const tj_basis *ebs, const tj_wave *in, tj_wave *out, double coef) {
  (void)fsl;
  int up_dif = sbl->up_dif, d1 = sbl->down_dif;
  if (up_dif != ebl->up_dif || d1 != ebl->down_dif) return fail(TJ_ERR_QN, "Quantum number error in block_vec_block!");
  for (int i = 0; i < in->num; i++) {
    int su = in->sub[i].sys_num_up, sd = in->sub[i].sys_num_down;
    int eu = in->sub[i].env_num_up, edn = in->sub[i].env_num_down;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < ebs->num; y++) {
        if (ebs->sub[y].new_num_up != eu || ebs->sub[y].new_num_down != edn) continue;
        for (int m = 0; m < sbs->sub[x].num; m++) {
          for (int n = 0; n < ebs->sub[y].num; n++) {
            const tj_basis_sub *ms = BM(sbs, x, m), *me = BM(ebs, y, n);
            for (int dd = -d1; dd <= d1; dd += 2) {
              int ks = find_sub(sbl, ms->bl_num_up, ms->bl_num_down, dd, 1);
              int nsb_up = ms->bl_num_up + up_dif, nsb_dn = ms->bl_num_down + dd;
              for (int edd = -d1; edd <= d1; edd += 2) {
                int neb_up = me->bl_num_up - up_dif, neb_dn = me->bl_num_down - edd;
                int ke = find_sub(ebl, neb_up, neb_dn, edd, 1);
                if (ks < 0 || ke < 0) continue;
                for (int nsd = abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                  int nsu = su + up_dif, neu = eu - up_dif, ned = nsd;
                  int nsp = -1, nsdim = 0, nep = -1, nedim = 0;
                  for (int k = 0; k < sbs->num && nsp < 0; k++) {
                    if (sbs->sub[k].new_num_up != nsu || sbs->sub[k].new_num_down != nsd) continue;
                    for (int l = 0; l < sbs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(sbs, k, l);
                      if (q->bl_num_up == nsb_up && q->bl_num_down == nsb_dn && q->st_num_down == ms->st_num_down &&
                          q->st_num_up == ms->st_num_up) {
                        nsp = q->spos;
                        nsdim = q->sdim;
                        break;
                      }
                    }
                  }
                  for (int k = 0; k < ebs->num && nep < 0; k++) {
                    if (ebs->sub[k].new_num_up != neu || ebs->sub[k].new_num_down != ned) continue;
                    for (int l = 0; l < ebs->sub[k].num; l++) {
                      const tj_basis_sub *q = BM(ebs, k, l);
                      if (q->bl_num_up == neb_up && q->bl_num_down == neb_dn && q->st_num_down == me->st_num_down &&
                          q->st_num_up == me->st_num_up) {
                        nep = q->spos;
                        nedim = q->sdim;
                        break;
                      }
                    }
                  }
                  if (nsp < 0 || nep < 0) continue;
                  int ko = find_out(out, nsu, nsd, neu, ned);
                  if (ko < 0) continue;
                  double sel = sgn_flag(fel, sd + me->st_num_down);
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->bl_num_down, j5 = ms->st_num_down, j6 = nsb_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->bl_num_down, j55 = me->st_num_down, j66 = neb_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  double c11 = W6(j11, j22, j33, j44, j55, j66);
                  if (c11 == 0.0) continue;
                  c1 *= c11;
                  if (c1 == 0.0) continue;
                  c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                  if (((j6 + j5 + j3 + j2) / 2 + (j66 + j55 + j33 + j22) / 2) % 2 == 1) c1 = -c1;
                  double ct = sel * coef * c1;
                  int od = ms->sdim, oe = me->sdim;
                  double *tmp = (double *)malloc(((size_t)nsdim * oe + 1) * sizeof(double));
                  dg('N', 'N', nsdim, oe, od, 1.0, sbl->sub[ks].mat, nsdim, WP(in, i, ms->spos, me->spos), LD(in, i),
                     0.0, tmp, nsdim);
                  dg('N', 'N', nsdim, nedim, oe, ct, tmp, nsdim, ebl->sub[ke].mat, oe, 1.0, WP(out, ko, nsp, nep),
                     LD(out, ko));
                  free(tmp);
                  if (d1 == 1) {
                    tmp = (double *)malloc(((size_t)od * nedim + 1) * sizeof(double));
                    dg('T', 'N', od, nedim, nsdim, 1.0, sbl->sub[ks].mat, nsdim, WP(in, ko, nsp, nep), LD(in, ko), 0.0,
                       tmp, od);
                    dg('N', 'T', od, oe, nedim, ct, tmp, od, ebl->sub[ke].mat, oe, 1.0, WP(out, i, ms->spos, me->spos),
                       LD(out, i));
                    free(tmp);
                  }
                }
              }
            }
          }
        }
      }
    }
  }
  return 0;
}
/* block_vec_block_dia (get_sys.f90:1910-2012) */
static int block_vec_block_dia(const OBlk *sbl, const OBlk *ebl, const tj_basis *sbs, const tj_basis *ebs,
                               const tj_wave *in, tj_wave *out, double coef) {
  for (int i = 0; i < in->num; i++) {
    int xs = find_bs(sbs, in->sub[i].sys_num_up, in->sub[i].sys_num_down);
    int xe = find_bs(ebs, in->sub[i].env_num_up, in->sub[i].env_num_down);
    if (xs < 0 || xe < 0) continue;
    for (int x = 0; x < sbs->sub[xs].num; x++) {
      const tj_basis_sub *ms = BM(sbs, xs, x);
      int ks = find_sub(sbl, ms->bl_num_up, ms->bl_num_down, 0, 0);
      for (int y = 0; y < ebs->sub[xe].num; y++) {
        const tj_basis_sub *me = BM(ebs, xe, y);
        int ke = find_sub(ebl, me->bl_num_up, me->bl_num_down, 0, 0);
        if (ks < 0 || ke < 0) continue;
        if (ms->sdim * me->sdim == 0) return fail(TJ_ERR_ARG, "block_vec_block_dia: empty tile");
        double c1 = coef / sqrt((1.0 + me->bl_num_down) * (1.0 + ms->bl_num_down));
        double *tmp = (double *)malloc(((size_t)ms->sdim * me->sdim + 1) * sizeof(double));
        dg('N', 'N', ms->sdim, me->sdim, ms->sdim, 1.0, sbl->sub[ks].mat, ms->sdim, WP(in, i, ms->spos, me->spos),
           LD(in, i), 0.0, tmp, ms->sdim);
        dg('N', 'T', ms->sdim, me->sdim, me->sdim, c1, tmp, ms->sdim, ebl->sub[ke].mat, me->sdim, 1.0,
           WP(out, i, ms->spos, me->spos), LD(out, i));
        free(tmp);
      }
    }
  }
  return 0;
}

/* ============================================== site operators */
/* Get_site_operator_su2_U0 (dmrg_sub.f90:370-473). */
typedef struct {
  OBlk eu, ed, ne, sd, si;
  OSub s_eu[1], s_ed[1], s_ne[2], s_sd[1], s_si[2];
  double v_eu[1], v_ed[1], v_ne[2], v_sd[1], v_si[2];
} SiteOps;
static void site_ops_build(int up_bias, SiteOps *o) {
  memset(o, 0, sizeof *o);
  o->v_eu[0] = -sqrt(2.0);
  o->s_eu[0] = (OSub){0, 0, 1, 1, 1, o->v_eu};
  o->eu = (OBlk){1, 1, 1, up_bias, 1, o->s_eu, 0};
  o->v_ed[0] = -sqrt(2.0);
  o->s_ed[0] = (OSub){up_bias, 1, -1, 1, 1, o->v_ed};
  o->ed = (OBlk){1, 1, 1, -up_bias, 1, o->s_ed, 0};
  o->v_ne[0] = 0.0;
  o->v_ne[1] = sqrt(2.0);
  o->s_ne[0] = (OSub){0, 0, 0, 1, 1, &o->v_ne[0]};
  o->s_ne[1] = (OSub){up_bias, 1, 0, 1, 1, &o->v_ne[1]};
  o->ne = (OBlk){1, 2, 2, 0, 0, o->s_ne, 0};
  o->v_sd[0] = sqrt(1.5);
  o->s_sd[0] = (OSub){up_bias, 1, 0, 1, 1, o->v_sd};
  o->sd = (OBlk){1, 1, 1, 0, 2, o->s_sd, 0};
  o->v_si[0] = 1.0;
  o->v_si[1] = sqrt(2.0);
  o->s_si[0] = (OSub){0, 0, 0, 1, 1, &o->v_si[0]};
  o->s_si[1] = (OSub){up_bias, 1, 0, 1, 1, &o->v_si[1]};
  o->si = (OBlk){1, 2, 2, 0, 0, o->s_si, 0};
}
int ora_site_operator(int which, int up_bias, tj_block *blk, tj_block_sub *subs, double *vals) {
  SiteOps o;
  site_ops_build(up_bias, &o);
  const OBlk *b = which == 0 ? &o.eu : which == 1 ? &o.ed : which == 2 ? &o.ne : which == 3 ? &o.sd : &o.si;
  memset(blk, 0, sizeof *blk);
  blk->len = b->len; blk->num = b->num; blk->dim = b->dim; blk->up_dif = b->up_dif; blk->down_dif = b->down_dif;
  for (int i = 0; i < b->num; i++) {
    subs[i].num_up = b->sub[i].num_up; subs[i].num_down = b->sub[i].num_down;
    subs[i].down_dif = b->sub[i].down_dif; subs[i].row_dim = 1; subs[i].sdim = 1; subs[i].off = i;
    vals[i] = b->sub[i].mat[0];
  }
  blk->sub = subs;
  blk->data = vals;
  return b->num;
}

/* ======================================================== hmerge */
typedef struct {
  int len;
  OBlk ham;
  int nsub;
  OSet *sub;     /* views of the caller's sub(1:nsub) */
  OSet snc[2];   /* owned, built by hmerge */
  OSet *sub_s;   /* owned, built by hmerge */
  int nsub_s;
} OModel;

static void model_view(const tj_model *m, OModel *o, int nxx) {
  memset(o, 0, sizeof *o);
  o->len = m->len;
  blk_view(&m->ham, &o->ham);
  o->nsub = m->nsub;
  o->sub = (OSet *)calloc(m->nsub > 0 ? m->nsub : 1, sizeof(OSet));
  for (int i = 0; i < m->nsub; i++) {
    blk_view(&m->sub[i].elec_up, &o->sub[i].op[EU]);
    blk_view(&m->sub[i].elec_down, &o->sub[i].op[ED]);
    blk_view(&m->sub[i].spin_sd, &o->sub[i].op[SD]);
    blk_view(&m->sub[i].spin_sz, &o->sub[i].op[SZ]);
    blk_view(&m->sub[i].num_sn, &o->sub[i].op[SN]);
  }
  o->nsub_s = nxx;
  o->sub_s = (OSet *)calloc(nxx, sizeof(OSet));
}
static void model_free(OModel *o) {
  blk_free(&o->ham);
  for (int i = 0; i < o->nsub; i++)
    for (int k = 0; k < 5; k++) blk_free(&o->sub[i].op[k]);
  free(o->sub);
  for (int a = 0; a < 2; a++)
    for (int k = 0; k < 5; k++) blk_free(&o->snc[a].op[k]);
  for (int i = 0; i < o->nsub_s; i++)
    for (int k = 0; k < 5; k++) blk_free(&o->sub_s[i].op[k]);
  free(o->sub_s);
}

typedef struct {
  const tj_lattice *L;
  int ns1; /* num_site + 1 */
  int *inb; /* inb(-4:num_site) stored at inb[i+4] */
  int coup_bs[2][2], coup_bb[2];
} Geo;
#define NEIB(g, i, k) ((g)->L->neib[((k)-1) * (g)->ns1 + (i)])
#define NEIBA(g, i, j) ((g)->L->neiba[(j) * (g)->ns1 + (i)])
#define INB1(g, i, j) ((g)->L->inb1[(j) * (g)->ns1 + (i)])
#define NLEG11(g, i) ((g)->L->nleg11[(i)-1])
#define NPOSI(g, i) ((g)->L->nposi[i])
#define NPOSI_DM(g, i) ((g)->L->nposi_dm[i])
#define NPOSI_LAT(g, i) ((g)->L->nposi_lat[i])
#define JT(g, k, i) ((g)->L->jt[(i) * (g)->L->neibt + (k)-1])
#define JZ(g, k, i) ((g)->L->jz[(i) * (g)->L->neibt + (k)-1])
#define JD(g, k, i) ((g)->L->jd[(i) * (g)->L->neibt + (k)-1])
#define JN(g, k) ((g)->L->jn[(k)-1])
#define ESITE(g, i) ((g)->L->esite[i])
#define INB(g, i) ((g)->inb[(i) + 4])

static int sub_slot(const OModel *m, int i1, const char *what) {
  if (i1 < 1 || i1 > m->nsub) {
    snprintf(g_err, sizeof g_err, "%s: operator slot %d outside 1..%d", what, i1, m->nsub);
    return -1;
  }
  return i1 - 1;
}

/* hmerge (get_sys.f90:4383-4593) */
static int hmerge(Geo *g, OModel *sys, OModel *env) {
  const int neibt = g->L->neibt;
  int syssite = sys->len + 1, dmsite = sys->len + env->len + 2;
  memset(g->coup_bs, 0, sizeof g->coup_bs);
  for (int k = 1; k <= neibt; k++) {
    int j = NEIB(g, syssite, k);
    if (NPOSI(g, NPOSI_DM(g, j)) == 3) g->coup_bs[1][0] = 1;
    if (NPOSI(g, NPOSI_DM(g, j)) == 1) g->coup_bs[0][0] = 1;
    j = NEIB(g, NPOSI_LAT(g, dmsite), k);
    if (NPOSI(g, NPOSI_DM(g, j)) == 3) g->coup_bs[1][1] = 1;
    if (NPOSI(g, NPOSI_DM(g, j)) == 1) g->coup_bs[0][1] = 1;
  }
  if (sys->nsub < 1 || env->nsub < 1) return fail(TJ_ERR_ARG, "hmerge: models need sub(1)");
  for (int ia = 0; ia < 2; ia++) {
    if (g->coup_bs[0][ia] == 1) {
      blk_pass_info(&sys->sub[0].op[EU], &sys->snc[ia].op[EU]);
      blk_pass_info(&sys->sub[0].op[SD], &sys->snc[ia].op[SD]);
      blk_pass_info(&sys->sub[0].op[SN], &sys->snc[ia].op[SN]);
    }
    if (g->coup_bs[1][ia] == 1) {
      blk_pass_info(&env->sub[0].op[EU], &env->snc[ia].op[EU]);
      blk_pass_info(&env->sub[0].op[ED], &env->snc[ia].op[ED]);
      blk_pass_info(&env->sub[0].op[SD], &env->snc[ia].op[SD]);
      blk_pass_info(&env->sub[0].op[SN], &env->snc[ia].op[SN]);
    }
  }
  for (int ia = 1; ia <= 2; ia++) {
    int j = sys->len + 1 + (env->len + 1) * (ia - 1);
    int lj = NPOSI_LAT(g, j);
    for (int k1 = 1; k1 <= neibt; k1++) {
      int ib = NEIB(g, lj, k1);
      if (NPOSI(g, NPOSI_DM(g, ib)) == 3) {
        int ib1 = NPOSI_DM(g, ib) - sys->len - 1;
        ib1 = INB1(g, ib1, env->len);
        if (g->coup_bs[1][ia - 1] != 0) {
          double jd1 = JD(g, k1, lj), jt1 = JT(g, k1, lj), jn1 = JN(g, k1);
          int s = sub_slot(env, ib1, "hmerge");
          if (s < 0) return TJ_ERR_ARG;
          if (jt1 != 0.0) {
            blk_add_two(&env->sub[s].op[EU], jt1, &env->snc[ia - 1].op[EU]);
            blk_add_two(&env->sub[s].op[ED], jt1, &env->snc[ia - 1].op[ED]);
          }
          if (jd1 != 0.0) blk_add_two(&env->sub[s].op[SD], jd1, &env->snc[ia - 1].op[SD]);
          if (jn1 != 0.0) blk_add_two(&env->sub[s].op[SN], jn1, &env->snc[ia - 1].op[SN]);
        }
      }
      if (NPOSI(g, NPOSI_DM(g, ib)) == 1) {
        int ib1 = NPOSI_DM(g, ib);
        ib1 = INB1(g, ib1, sys->len);
        if (g->coup_bs[0][ia - 1] == 1) {
          double jd1 = JD(g, k1, lj), jt1 = JT(g, k1, lj), jn1 = JN(g, k1);
          int s = sub_slot(sys, ib1, "hmerge");
          if (s < 0) return TJ_ERR_ARG;
          if (jt1 != 0.0) blk_add_two(&sys->sub[s].op[EU], jt1, &sys->snc[ia - 1].op[EU]);
          if (jd1 != 0.0) blk_add_two(&sys->sub[s].op[SD], jd1, &sys->snc[ia - 1].op[SD]);
          if (jn1 != 0.0) blk_add_two(&sys->sub[s].op[SN], jn1, &sys->snc[ia - 1].op[SN]);
        }
      }
    }
  }
  g->coup_bb[0] = g->coup_bb[1] = 0;
  int k11 = 0;
  for (int I = 1; I <= sys->len; I++) {
    int k1 = 0;
    INB(g, I) = 0;
    for (int k = 1; k <= neibt; k++) {
      int J = NEIB(g, I, k);
      if (NPOSI(g, NPOSI_DM(g, J)) == 3) k1++;
    }
    INB(g, I) = k1;
    if (NLEG11(g, env->len) < NLEG11(g, sys->len)) INB(g, I) = 0;
    if (INB(g, I) != 0) k11++;
  }
  g->coup_bb[0] = k11;
  INB(g, sys->len + 1) = 0;
  INB(g, sys->len + 1 + env->len + 1) = 0;
  for (int I = 1; I <= env->len; I++) {
    int k1 = 0;
    INB(g, I + sys->len + 1) = 0;
    for (int k = 1; k <= neibt; k++) {
      int J = NEIB(g, NPOSI_LAT(g, I + sys->len + 1), k);
      if (NPOSI(g, NPOSI_DM(g, J)) == 1)
        if (INB(g, J) == 0) k1++;
    }
    INB(g, I + sys->len + 1) = k1;
    if (k1 != 0) k11++;
  }
  g->coup_bb[1] = k11 - g->coup_bb[0];
  if (g->coup_bb[0] > env->nsub_s || g->coup_bb[1] > sys->nsub_s) return fail(TJ_ERR_LIMIT, "hmerge: too many legs");
  for (int i = 0; i < g->coup_bb[0]; i++) {
    blk_pass_info(&env->sub[0].op[EU], &env->sub_s[i].op[EU]);
    blk_pass_info(&env->sub[0].op[ED], &env->sub_s[i].op[ED]);
    blk_pass_info(&env->sub[0].op[SD], &env->sub_s[i].op[SD]);
    blk_pass_info(&env->sub[0].op[SN], &env->sub_s[i].op[SN]);
  }
  for (int i = 0; i < g->coup_bb[1]; i++) {
    blk_pass_info(&sys->sub[0].op[EU], &sys->sub_s[i].op[EU]);
    blk_pass_info(&sys->sub[0].op[SD], &sys->sub_s[i].op[SD]);
    blk_pass_info(&sys->sub[0].op[SN], &sys->sub_s[i].op[SN]);
  }
  int jc = 0;
  for (int I = 1; I <= sys->len + env->len + 1; I++) {
    if (INB(g, I) == 0) continue;
    int Ia = NPOSI_LAT(g, I);
    jc++;
    for (int k1 = 1; k1 <= neibt; k1++) {
      int ib = NEIB(g, Ia, k1);
      if (NPOSI(g, NPOSI_DM(g, ib)) == 3 && I <= sys->len) {
        int ib1 = INB1(g, NPOSI_DM(g, ib) - sys->len - 1, env->len);
        double jt1 = JT(g, k1, Ia), jd1 = JD(g, k1, Ia), jn1 = JN(g, k1);
        int s = sub_slot(env, ib1, "hmerge");
        if (s < 0) return TJ_ERR_ARG;
        if (jt1 != 0.0) {
          blk_add_two(&env->sub[s].op[EU], jt1, &env->sub_s[jc - 1].op[EU]);
          blk_add_two(&env->sub[s].op[ED], jt1, &env->sub_s[jc - 1].op[ED]);
        }
        if (jd1 != 0.0) blk_add_two(&env->sub[s].op[SD], jd1, &env->sub_s[jc - 1].op[SD]);
        if (jn1 != 0.0) blk_add_two(&env->sub[s].op[SN], jn1, &env->sub_s[jc - 1].op[SN]);
      }
      if (NPOSI(g, NPOSI_DM(g, ib)) == 1 && I > sys->len + 1) {
        if (INB(g, NPOSI_DM(g, ib)) == 0) {
          int ib1 = INB1(g, ib, sys->len);
          int jc1 = jc - g->coup_bb[0];
          double jt1 = JT(g, k1, Ia), jd1 = JD(g, k1, Ia), jn1 = JN(g, k1);
          int s = sub_slot(sys, ib1, "hmerge");
          if (s < 0) return TJ_ERR_ARG;
          if (jt1 != 0.0) blk_add_two(&sys->sub[s].op[EU], jt1, &sys->sub_s[jc1 - 1].op[EU]);
          if (jd1 != 0.0) blk_add_two(&sys->sub[s].op[SD], jd1, &sys->sub_s[jc1 - 1].op[SD]);
          if (jn1 != 0.0) blk_add_two(&sys->sub[s].op[SN], jn1, &sys->sub_s[jc1 - 1].op[SN]);
        }
      }
    }
  }
  return 0;
}

/* model_wave, add_op = 1 branch (get_sys.f90:4127-4240) */
static int model_wave_core(Geo *g, OModel *sys, OModel *env, const tj_basis *sbs, const tj_basis *ebs,
                           const SiteOps *so, const tj_wave *in, tj_wave *out) {
  int rc = 0;
  memset(out->data, 0, (size_t)out->dim * sizeof(double));
  block_vec_dia(&sys->ham, sbs, in, out, 1.0);
  vec_block_dia(&env->ham, ebs, in, out, 1.0);
  int is = NPOSI_LAT(g, sys->len + 1), js = NPOSI_LAT(g, sys->len + env->len + 2);
  if (ESITE(g, is) != 0.0) site_vec_site_dia(&so->ne, &so->si, sbs, ebs, in, out, ESITE(g, is));
  if (ESITE(g, js) != 0.0) site_vec_site_dia(&so->si, &so->ne, sbs, ebs, in, out, ESITE(g, js));
  int ii = NEIBA(g, is, js);
  if (ii != 0) {
    double jd1 = JD(g, ii, is), coefx = JT(g, ii, is), jn1 = JN(g, ii);
    if (coefx != 0.0) site_vec_site_ndia(&so->eu, 'F', &so->eu, 'F', sbs, ebs, in, out, coefx);
    if (jd1 != 0.0) site_vec_site_ndia(&so->sd, 'B', &so->sd, 'B', sbs, ebs, in, out, jd1);
    site_vec_site_dia(&so->ne, &so->ne, sbs, ebs, in, out, jn1);
  }
  if (g->coup_bs[0][0] == 1) {
    if ((rc = block_site_vec_ndia(&sys->snc[0].op[EU], 'F', &so->eu, 'F', sbs, in, out, 1.0))) return rc;
    if ((rc = block_site_vec_ndia(&sys->snc[0].op[SD], 'B', &so->sd, 'B', sbs, in, out, 1.0))) return rc;
    block_site_vec_dia(&sys->snc[0].op[SN], &so->ne, sbs, in, out, 1.0);
  }
  if (g->coup_bs[0][1] == 1) {
    if ((rc = block_vec_site_ndia(&sys->snc[1].op[EU], 'F', &so->eu, 'F', sbs, ebs, in, out, 1.0))) return rc;
    if ((rc = block_vec_site_ndia(&sys->snc[1].op[SD], 'B', &so->sd, 'B', sbs, ebs, in, out, 1.0))) return rc;
    block_vec_site_dia(&sys->snc[1].op[SN], &so->ne, sbs, ebs, in, out, 1.0);
  }
  if (g->coup_bs[1][0] == 1) {
    OBlk t1, t;
    blk_trans(&env->snc[0].op[ED], &t1);
    rc = site_vec_block_ndia(&so->eu, 'F', &t1, 'F', sbs, ebs, in, out, 1.0);
    blk_trans(&env->snc[0].op[SD], &t);
    if (!rc) rc = site_vec_block_ndia(&so->sd, 'B', &t, 'B', sbs, ebs, in, out, 1.0);
    if (!rc) site_vec_block_dia(&so->ne, &env->snc[0].op[SN], sbs, ebs, in, out, 1.0);
    blk_free(&t);
    blk_free(&t1);
    if (rc) return rc;
  }
  if (g->coup_bs[1][1] == 1) {
    if ((rc = vec_block_site_ndia(&env->snc[1].op[EU], 'F', &so->eu, 'F', ebs, in, out, 1.0))) return rc;
    if ((rc = vec_block_site_ndia(&env->snc[1].op[SD], 'B', &so->sd, 'B', ebs, in, out, 1.0))) return rc;
    vec_block_site_dia(&env->snc[1].op[SN], &so->ne, ebs, in, out, 1.0);
  }
  int jc = 0;
  for (int i = 1; i <= sys->len + 1 + env->len; i++) {
    if (INB(g, i) == 0) continue;
    jc++;
    OBlk t1, t;
    const OSet *sa, *eb;
    if (i <= sys->len) {
      int s = sub_slot(sys, INB1(g, i, sys->len), "model_wave");
      if (s < 0) return TJ_ERR_ARG;
      sa = &sys->sub[s];
      eb = &env->sub_s[jc - 1];
    } else {
      int s = sub_slot(env, INB1(g, i - sys->len - 1, env->len), "model_wave");
      if (s < 0) return TJ_ERR_ARG;
      int jc1 = jc - g->coup_bb[0];
      sa = &sys->sub_s[jc1 - 1];
      eb = &env->sub[s];
    }
    blk_trans(&eb->op[ED], &t1);
    rc = block_vec_block_ndia(&sa->op[EU], 'F', &t1, 'F', sbs, ebs, in, out, 1.0);
    blk_trans(&eb->op[SD], &t);
    if (!rc) rc = block_vec_block_ndia(&sa->op[SD], 'B', &t, 'B', sbs, ebs, in, out, 1.0);
    if (!rc) rc = block_vec_block_dia(&sa->op[SN], &eb->op[SN], sbs, ebs, in, out, 1.0);
    blk_free(&t);
    blk_free(&t1);
    if (rc) return rc;
  }
  return 0;
}

typedef struct {
  Geo g;
  OModel sys, env;
  SiteOps so;
} MVState;

static int mv_setup(MVState *st, const tj_lattice *lat, const tj_model *sys, const tj_model *env) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  memset(st, 0, sizeof *st);
  st->g.L = lat;
  st->g.ns1 = lat->num_site + 1;
  st->g.inb = (int *)calloc((size_t)lat->num_site + 5, sizeof(int));
  int nxx = lat->num_site + 1;
  model_view(sys, &st->sys, nxx);
  model_view(env, &st->env, nxx);
  site_ops_build(lat->up_bias, &st->so);
  return hmerge(&st->g, &st->sys, &st->env);
}
static void mv_free(MVState *st) {
  model_free(&st->sys);
  model_free(&st->env);
  free(st->g.inb);
}

int ora_model_wave(const tj_lattice *lat, const tj_model *sys, const tj_model *env, const tj_basis *sys_bs,
                   const tj_basis *env_bs, const tj_wave *invec, tj_wave *outvec) {
  MVState st;
  int rc = mv_setup(&st, lat, sys, env);
  if (!rc) rc = model_wave_core(&st.g, &st.sys, &st.env, sys_bs, env_bs, &st.so, invec, outvec);
  mv_free(&st);
  return rc;
}

/* ================================================== wave algebra */
/* wave_product / wave_norm (block.f90:2377-2414): per sector, per column dots */
static double wave_product(const tj_wave *a, const double *x, const double *y) {
  double s = 0.0;
  for (int i = 0; i < a->num; i++) {
    int sd = a->sub[i].sys_dim, ed = a->sub[i].env_dim;
    for (int c = 0; c < ed; c++) {
      const double *p = x + a->sub[i].off + (size_t)c * sd, *q = y + a->sub[i].off + (size_t)c * sd;
      double d = 0.0;
      for (int r = 0; r < sd; r++) d += p[r] * q[r];
      s += d;
    }
  }
  return s;
}
static void wave_scale(int64_t n, double *x, double a) {
  for (int64_t e = 0; e < n; e++) x[e] /= a;
}

/* lanczos_memo_new, levels = 1 (eigen.f90:2-175) */
int ora_lanczos(const tj_lattice *lat, const tj_model *sys, const tj_model *env, const tj_basis *sys_bs,
                const tj_basis *env_bs, tj_wave *eigvec, double lanzero, double *energy, int *iters) {
  enum { LOOP_IN = 110 };
  const int64_t D = eigvec->dim;
  MVState st;
  int rc = mv_setup(&st, lat, sys, env);
  if (rc) {
    mv_free(&st);
    return rc;
  }
  double *V = (double *)malloc(((size_t)(LOOP_IN + 1) * D + 1) * sizeof(double));
  double alpha[LOOP_IN + 1], beta[LOOP_IN + 1];
  memset(alpha, 0, sizeof alpha);
  memset(beta, 0, sizeof beta);
  tj_wave wa = *eigvec, wb = *eigvec;
#define VEC(j) (V + (size_t)((j)-1) * D)
  int last = 1;
  double ritzmin = 1024.0;
  memcpy(VEC(1), eigvec->data, (size_t)D * sizeof(double));
  wave_scale(D, VEC(1), sqrt(wave_product(eigvec, VEC(1), VEC(1))));
  wa.data = VEC(1);
  wb.data = VEC(2);
  rc = model_wave_core(&st.g, &st.sys, &st.env, sys_bs, env_bs, &st.so, &wa, &wb);
  alpha[1] = wave_product(eigvec, VEC(1), VEC(2));
  ritzmin = alpha[1];
  while (!rc && last < LOOP_IN) {
    double *w = VEC(last + 1), *v = VEC(last);
    if (last < 2) {
      for (int64_t e = 0; e < D; e++) w[e] = w[e] - alpha[last] * v[e];
    } else {
      double *u = VEC(last - 1);
      for (int64_t e = 0; e < D; e++) w[e] = w[e] - alpha[last] * v[e] - beta[last - 1] * u[e];
    }
    beta[last] = sqrt(wave_product(eigvec, w, w));
    if (fabs(beta[last]) <= lanzero) break;
    wave_scale(D, w, sqrt(wave_product(eigvec, w, w)));
    /* Gram_Schmidt_process (block.f90:2515-2551): classical Gram-Schmidt */
    {
      double uv[LOOP_IN + 1], uu[LOOP_IN + 1];
      for (int j = 1; j <= last; j++) {
        uv[j] = wave_product(eigvec, VEC(j), w);
        uu[j] = wave_product(eigvec, VEC(j), VEC(j));
      }
      double *tmp = (double *)calloc((size_t)D + 1, sizeof(double));
      for (int j = 1; j <= last; j++) {
        double f = uv[j] / uu[j];
        const double *p = VEC(j);
        for (int64_t e = 0; e < D; e++) tmp[e] = tmp[e] + f * p[e];
      }
      for (int64_t e = 0; e < D; e++) w[e] = w[e] - tmp[e];
      free(tmp);
      wave_scale(D, w, sqrt(wave_product(eigvec, w, w)));
    }
    last++;
    wa.data = VEC(last);
    wb.data = VEC(last + 1);
    rc = model_wave_core(&st.g, &st.sys, &st.env, sys_bs, env_bs, &st.so, &wa, &wb);
    if (rc) break;
    alpha[last] = wave_product(eigvec, VEC(last), VEC(last + 1));
    double dia[LOOP_IN + 1], ndia[LOOP_IN + 1], dz[1];
    int n = last, ldz = 1, info = 0;
    memcpy(dia, &alpha[1], sizeof(double) * n);
    memcpy(ndia, &beta[1], sizeof(double) * n);
    char jobz = 'N';
    p_dstev(&jobz, &n, dia, ndia, dz, &ldz, NULL, &info, 1);
    if (fabs(dia[0] - ritzmin) <= lanzero || last == LOOP_IN) {
      ritzmin = dia[0];
      break;
    }
    ritzmin = dia[0];
  }
  if (!rc) {
    /* label 411: dstev('V') and the Ritz vector */
    int n = last, ldz = last, info = 0;
    double *dz = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *work = (double *)malloc(sizeof(double) * (size_t)(2 * n + 2));
    double dia[LOOP_IN + 1], ndia[LOOP_IN + 1];
    memcpy(dia, &alpha[1], sizeof(double) * n);
    memcpy(ndia, &beta[1], sizeof(double) * n);
    char jobz = 'V';
    p_dstev(&jobz, &n, dia, ndia, dz, &ldz, work, &info, 1);
    if (info != 0) rc = fail(TJ_ERR_NUMERIC, "dstev failed");
    *energy = dia[0];
    memset(eigvec->data, 0, (size_t)D * sizeof(double));
    for (int i = 1; i <= last; i++) {
      double f = dz[i - 1];
      const double *p = VEC(i);
      for (int64_t e = 0; e < D; e++) eigvec->data[e] += f * p[e];
    }
    wave_scale(D, eigvec->data, sqrt(wave_product(eigvec, eigvec->data, eigvec->data)));
    *iters = last;
    free(dz);
    free(work);
  }
#undef VEC
  free(V);
  mv_free(&st);
  return rc;
}

/* ==================================================== truncation */
/* QuickSort_Double (block.f90:288-332): descending, carries an index array. */
static void quicksort_double(double *arr, int *idx, int lower, int upper) {
  int i = lower, j = upper;
  int index = (int)((lower + upper) / 2.0);
  double mn = arr[index];
  while (i <= j) {
    while (arr[i] > mn) i++;
    while (arr[j] < mn) j--;
    if (i <= j) {
      double t = arr[i];
      arr[i] = arr[j];
      arr[j] = t;
      int ti = idx[i];
      idx[i] = idx[j];
      idx[j] = ti;
      i++;
      j--;
    }
  }
  if (lower < j) quicksort_double(arr, idx, lower, j);
  if (i < upper) quicksort_double(arr, idx, i, upper);
}

int ora_truncation(const tj_wave *wave, int side, int kept_min, int kept_max, double trun_err, tj_trunc_result *out,
                   double *eigval_out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  const int nsec = wave->num;
  const int64_t D = wave->dim;
  /* Get_density_matrix_*_new (den_mat.f90:84-134): normalised copy of psi */
  double *psi = (double *)malloc(((size_t)D + 1) * sizeof(double));
  memcpy(psi, wave->data, (size_t)D * sizeof(double));
  wave_scale(D, psi, sqrt(wave_product(wave, psi, psi)));
  int *dims = (int *)malloc(sizeof(int) * (nsec + 1)), *qnu = (int *)malloc(sizeof(int) * (nsec + 1)),
      *qnd = (int *)malloc(sizeof(int) * (nsec + 1));
  double **ev = (double **)calloc(nsec + 1, sizeof(double *)), **eval = (double **)calloc(nsec + 1, sizeof(double *));
  int total = 0, rc = 0;
  for (int i = 0; i < nsec; i++) {
    int sd = wave->sub[i].sys_dim, ed = wave->sub[i].env_dim;
    int n = side == 0 ? sd : ed;
    dims[i] = n;
    qnu[i] = side == 0 ? wave->sub[i].sys_num_up : wave->sub[i].env_num_up;
    qnd[i] = side == 0 ? wave->sub[i].sys_num_down : wave->sub[i].env_num_down;
    ev[i] = (double *)malloc(((size_t)n * n + 1) * sizeof(double));
    eval[i] = (double *)malloc(((size_t)n + 1) * sizeof(double));
    const double *p = psi + wave->sub[i].off;
    if (side == 0)
      dg('N', 'T', sd, sd, ed, 1.0, p, sd, p, sd, 0.0, ev[i], sd);
    else
      dg('T', 'N', ed, ed, sd, 1.0, p, sd, p, sd, 0.0, ev[i], ed);
    int lwork = 3 * n - 1 > 1 ? 3 * n - 1 : 1, info = 0, lda = n > 0 ? n : 1;
    double *work = (double *)malloc(sizeof(double) * (size_t)lwork);
    char jobz = 'V', uplo = 'U';
    if (n > 0) p_dsyev(&jobz, &uplo, &n, ev[i], &lda, eval[i], work, &lwork, &info, 1, 1);
    free(work);
    if (info != 0) rc = fail(TJ_ERR_NUMERIC, "dsyev failed");
    total += n;
  }
  int *idx = (int *)malloc(sizeof(int) * (total + 1)), *eigs = (int *)malloc(sizeof(int) * (total + 1));
  int *owner = (int *)malloc(sizeof(int) * (total + 1));
  double *eigvalue = (double *)malloc(sizeof(double) * (total + 1));
  {
    int t = 0;
    for (int k = 0; k < nsec; k++)
      for (int i = 0; i < dims[k]; i++) {
        idx[t] = t + 1;
        owner[t] = k;
        eigvalue[t] = eval[k][i];
        eigs[t] = qnd[k] + 1;
        if (eigval_out) eigval_out[t] = eval[k][i];
        t++;
      }
  }
  const double thr = (double)1.0e-15f; /* the reference's single-precision literal 1.0E-15 */
  double tot_pm = 0.0;
  for (int i = 0; i < total; i++) tot_pm += eigvalue[i] * eigs[i];
  double entropy1 = 0.0, entropy2 = 0.0, entropys = 0.0;
  for (int i = 0; i < total; i++)
    if (eigvalue[i] >= thr) {
      double v1 = eigvalue[i] / eigs[i];
      entropy1 = entropy1 - v1 * log(v1) * eigs[i];
    }
  for (int i = 0; i < total; i++) eigvalue[i] = eigvalue[i] / tot_pm;
  for (int i = 0; i < total; i++)
    if (eigvalue[i] >= thr) entropy2 = entropy2 - eigvalue[i] * log(eigvalue[i]) * eigs[i];
  for (int i = 0; i < total; i++) eigvalue[i] = eigvalue[i] * tot_pm;
  if (total > 0) quicksort_double(eigvalue, idx, 0, total - 1);
  tot_pm = 0.0;
  for (int i = 0; i < total; i++) tot_pm += eigvalue[i];
  for (int i = 0; i < total; i++) eigvalue[i] = eigvalue[i] / tot_pm;
  int num_state;
  double tmp_err = 0.0;
  if (total <= kept_min) {
    num_state = total;
  } else {
    for (int i = kept_min; i < total; i++) tmp_err += eigvalue[i];
    num_state = kept_min;
    while (tmp_err > trun_err && num_state < total) {
      num_state++;
      tmp_err -= eigvalue[num_state - 1];
      if (tmp_err <= trun_err || num_state >= kept_max) break;
    }
  }
  for (int i = 0; i < total; i++)
    if (eigvalue[i] >= thr) entropys = entropys - eigvalue[i] * log(eigvalue[i]);
  int *cnt = (int *)calloc(nsec + 1, sizeof(int));
  for (int k = 0; k < num_state; k++) cnt[owner[idx[k] - 1]]++;
  int nkept = 0;
  int64_t need = 0;
  for (int i = 0; i < nsec; i++)
    if (cnt[i] > 0) {
      nkept++;
      need += (int64_t)dims[i] * cnt[i];
    }
  out->num_state = num_state;
  out->num = nkept;
  out->data_len = need;
  out->trunc_err = tmp_err;
  out->entropy1 = entropy1;
  out->entropy2 = entropy2;
  out->entropys = entropys;
  if (out->sub && out->data) {
    int t = 0;
    int64_t off = 0;
    for (int i = 0; i < nsec; i++) {
      if (cnt[i] == 0) continue;
      /* the reference copies from the first sector with the same labels */
      int x = 0;
      while (x < nsec && !(qnu[x] == qnu[i] && qnd[x] == qnd[i])) x++;
      int row = dims[i], col = cnt[i];
      tj_block_sub *s = &out->sub[t++];
      s->num_up = qnu[i]; s->num_down = qnd[i]; s->down_dif = 0; s->row_dim = row; s->sdim = col; s->off = off;
      for (int c = 0; c < col; c++)
        memcpy(out->data + off + (size_t)c * row, ev[x] + (size_t)(row - col + c) * row, sizeof(double) * row);
      off += (int64_t)row * col;
    }
  }
  for (int i = 0; i < nsec; i++) {
    free(ev[i]);
    free(eval[i]);
  }
  free(ev); free(eval); free(dims); free(qnu); free(qnd); free(idx); free(eigs); free(owner);
  free(eigvalue); free(cnt); free(psi);
  return rc;
}

/* ================================================== correlators */
/* measure_sys_block (measure.f90:1241-1295) */
int ora_measure_sys_block(const tj_block *sys_bl, const tj_basis *sbs, const tj_wave *w, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk bl;
  blk_view(sys_bl, &bl);
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, ed = w->sub[i].env_dim;
    for (int k = 0; k < sbs->num; k++) {
      if (sbs->sub[k].new_num_up != su || sbs->sub[k].new_num_down != sd) continue;
      for (int x = 0; x < sbs->sub[k].num; x++) {
        const tj_basis_sub *m = BM(sbs, k, x);
        double c1 = 1.0 / sqrt(1.0 + m->bl_num_down);
        int y = find_sub(&bl, m->bl_num_up, m->bl_num_down, 0, 0);
        if (y < 0) continue;
        double *mid = (double *)malloc(((size_t)m->sdim * ed + 1) * sizeof(double));
        dg('N', 'N', m->sdim, ed, m->sdim, c1, bl.sub[y].mat, m->sdim, WP(w, i, m->spos, 0), LD(w, i), 0.0, mid,
           m->sdim);
        for (int z = 0; z < ed; z++) {
          double d = 0.0;
          const double *p = WP(w, i, m->spos, z);
          for (int r = 0; r < m->sdim; r++) d += p[r] * mid[(size_t)z * m->sdim + r];
          v += d;
        }
        free(mid);
      }
    }
  }
  blk_free(&bl);
  *value = v;
  return 0;
}
/* measure_env_block (measure.f90:1359-1414) */
int ora_measure_env_block(const tj_block *env_bl, const tj_basis *ebs, const tj_wave *w, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk bl;
  blk_view(env_bl, &bl);
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int eu = w->sub[i].env_num_up, edn = w->sub[i].env_num_down, sdm = w->sub[i].sys_dim;
    for (int k = 0; k < ebs->num; k++) {
      if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
      for (int x = 0; x < ebs->sub[k].num; x++) {
        const tj_basis_sub *m = BM(ebs, k, x);
        int y = find_sub(&bl, m->bl_num_up, m->bl_num_down, 0, 0);
        if (y < 0) continue;
        double c1 = 1.0 / sqrt(1.0 + m->bl_num_down);
        double *mid = (double *)malloc(((size_t)sdm * m->sdim + 1) * sizeof(double));
        dg('N', 'N', sdm, m->sdim, m->sdim, 1.0, WP(w, i, 0, m->spos), LD(w, i), bl.sub[y].mat, m->sdim, 0.0, mid,
           sdm);
        for (int z = 0; z < m->sdim; z++) {
          double d = 0.0;
          const double *p = WP(w, i, 0, m->spos + z);
          for (int r = 0; r < sdm; r++) d += mid[(size_t)z * sdm + r] * p[r];
          v += d * c1;
        }
        free(mid);
      }
    }
  }
  blk_free(&bl);
  *value = v;
  return 0;
}
static double dot_cols(const double *a, int lda, const double *b, int ldb, int nr, int nc) {
  double v = 0.0;
  for (int c = 0; c < nc; c++) {
    double d = 0.0;
    for (int r = 0; r < nr; r++) d += a[(size_t)c * lda + r] * b[(size_t)c * ldb + r];
    v += d;
  }
  return v;
}
/* sys_block_env_block_cor_dia (measure.f90:1638-1732) */
int ora_sys_block_env_block_cor_dia(const tj_block *a, const tj_block *b, const tj_basis *sbs, const tj_basis *ebs,
                                    const tj_wave *w, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk sb, eb;
  blk_view(a, &sb);
  blk_view(b, &eb);
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up,
        edn = w->sub[i].env_num_down;
    for (int x = 0; x < sbs->num; x++) {
      if (sbs->sub[x].new_num_up != su || sbs->sub[x].new_num_down != sd) continue;
      for (int y = 0; y < sbs->sub[x].num; y++) {
        const tj_basis_sub *ms = BM(sbs, x, y);
        int ks = find_sub(&sb, ms->bl_num_up, ms->bl_num_down, 0, 0);
        for (int m = 0; m < ebs->num; m++) {
          if (ebs->sub[m].new_num_up != eu || ebs->sub[m].new_num_down != edn) continue;
          for (int n = 0; n < ebs->sub[m].num; n++) {
            const tj_basis_sub *me = BM(ebs, m, n);
            int ke = find_sub(&eb, me->bl_num_up, me->bl_num_down, 0, 0);
            if (ks < 0 || ke < 0) continue;
            int sdim = ms->sdim, edim = me->sdim;
            double *m1 = (double *)malloc(((size_t)sdim * edim + 1) * sizeof(double));
            double *m2 = (double *)malloc(((size_t)sdim * edim + 1) * sizeof(double));
            double c1 = 1.0 / sqrt((1.0 + me->bl_num_down) * (1.0 + ms->bl_num_down));
            dg('N', 'N', sdim, edim, edim, 1.0, WP(w, i, ms->spos, me->spos), LD(w, i), eb.sub[ke].mat, edim, 0.0, m1,
               sdim);
            dg('N', 'N', sdim, edim, sdim, 1.0, sb.sub[ks].mat, sdim, WP(w, i, ms->spos, me->spos), LD(w, i), 0.0, m2,
               sdim);
            for (int z = 0; z < edim; z++) v += dot_cols(m1 + (size_t)z * sdim, sdim, m2 + (size_t)z * sdim, sdim, sdim, 1) * c1;
            free(m1);
            free(m2);
          }
        }
      }
    }
  }
  blk_free(&sb);
  blk_free(&eb);
  *value = v;
  return 0;
}
/* sys_block_env_block_cor_ndia (measure.f90:5241-5480) */
int ora_sys_block_env_block_cor_ndia(const tj_block *a, const tj_block *b, const tj_basis *sbs, const tj_basis *ebs,
                                     const tj_wave *w, char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk sb, eb;
  blk_view(a, &sb);
  blk_view(b, &eb);
  int up_dif = sb.up_dif, d1 = sb.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up,
        edn = w->sub[i].env_num_down;
    for (int j = 0; j < sbs->num; j++) {
      if (sbs->sub[j].new_num_up != su || sbs->sub[j].new_num_down != sd) continue;
      for (int k = 0; k < ebs->num; k++) {
        if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
        for (int x = 0; x < sbs->sub[j].num; x++)
          for (int y = 0; y < ebs->sub[k].num; y++) {
            const tj_basis_sub *ms = BM(sbs, j, x), *me = BM(ebs, k, y);
            for (int dd = -d1; dd <= d1; dd += 2) {
              int nsb_up = ms->bl_num_up + up_dif, nsb_dn = ms->bl_num_down + dd;
              int ks = find_sub(&sb, ms->bl_num_up, ms->bl_num_down, dd, 1);
              for (int edd = -d1; edd <= d1; edd += 2) {
                int neb_up = me->bl_num_up - up_dif, neb_dn = me->bl_num_down - edd;
                int ke = find_sub(&eb, neb_up, neb_dn, edd, 1);
                for (int nsd = abs(sd - d1); nsd <= sd + d1; nsd += 2) {
                  int nsu = su + up_dif, neu = eu - up_dif, ned = nsd;
                  int nsp = -1, nsdim = 0, nep = -1, nedim = 0;
                  for (int mm = 0; mm < sbs->num && nsp < 0; mm++) {
                    if (sbs->sub[mm].new_num_up != nsu || sbs->sub[mm].new_num_down != nsd) continue;
                    for (int n = 0; n < sbs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(sbs, mm, n);
                      if (q->bl_num_up == nsb_up && q->bl_num_down == nsb_dn && q->st_num_up == ms->st_num_up &&
                          q->st_num_down == ms->st_num_down) {
                        nsp = q->spos;
                        nsdim = q->sdim;
                        break;
                      }
                    }
                  }
                  for (int mm = 0; mm < ebs->num && nep < 0; mm++) {
                    if (ebs->sub[mm].new_num_up != neu || ebs->sub[mm].new_num_down != ned) continue;
                    for (int n = 0; n < ebs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(ebs, mm, n);
                      if (q->bl_num_up == neb_up && q->bl_num_down == neb_dn && q->st_num_up == me->st_num_up &&
                          q->st_num_down == me->st_num_down) {
                        nep = q->spos;
                        nedim = q->sdim;
                        break;
                      }
                    }
                  }
                  int wid = find_out(w, nsu, nsd, neu, ned);
                  if (ks < 0 || ke < 0 || nsp < 0 || nep < 0 || wid < 0) continue;
                  double signs = sgn_flag(flag, sd + me->st_num_down);
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->bl_num_down, j5 = ms->st_num_down, j6 = nsb_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->bl_num_down, j55 = me->st_num_down, j66 = neb_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  c1 *= W6(j11, j22, j33, j44, j55, j66);
                  if (c1 == 0.0) continue;
                  c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                  if (((j6 + j5 + j3 + j2) / 2 + (j66 + j55 + j33 + j22) / 2) % 2 == 1) c1 = -c1;
                  double coef = signs * c1;
                  int sdim = ms->sdim, edim = me->sdim;
                  double *m1 = (double *)malloc(((size_t)nsdim * edim + 1) * sizeof(double));
                  double *m2 = (double *)malloc(((size_t)nsdim * edim + 1) * sizeof(double));
                  dg('N', 'N', nsdim, edim, sdim, 1.0, sb.sub[ks].mat, nsdim, WP(w, i, ms->spos, me->spos), LD(w, i),
                     0.0, m1, nsdim);
                  dg('N', 'T', nsdim, edim, nedim, coef, WP(w, wid, nsp, nep), LD(w, wid), eb.sub[ke].mat, edim, 0.0,
                     m2, nsdim);
                  v += dot_cols(m1, nsdim, m2, nsdim, nsdim, edim);
                  free(m1);
                  free(m2);
                }
              }
            }
          }
      }
    }
  }
  blk_free(&sb);
  blk_free(&eb);
  *value = v;
  return 0;
}
/* sys_block_site_cor_ndia (measure.f90:4939-5083) */
int ora_sys_block_site_cor_ndia(const tj_block *a, const tj_block *stb, const tj_basis *sbs, const tj_wave *w,
                                char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk bl, st;
  blk_view(a, &bl);
  blk_view(stb, &st);
  int up_dif = bl.up_dif, d1 = bl.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, ed = w->sub[i].env_dim;
    for (int j = 0; j < sbs->num; j++) {
      if (sbs->sub[j].new_num_up != su || sbs->sub[j].new_num_down != sd) continue;
      for (int k = 0; k < sbs->sub[j].num; k++) {
        const tj_basis_sub *m = BM(sbs, j, k);
        for (int dd = -d1; dd <= d1; dd += 2)
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            int nbl_up = m->bl_num_up + up_dif, nbl_dn = m->bl_num_down + dd;
            int nst_up = m->st_num_up - up_dif, nst_dn = m->st_num_down - sdd;
            int kb = find_sub(&bl, m->bl_num_up, m->bl_num_down, dd, 1);
            int ks = find_sub(&st, nst_up, nst_dn, sdd, 1);
            int np = -1, nd = 0;
            for (int x = 0; x < sbs->sub[j].num; x++) {
              const tj_basis_sub *q = BM(sbs, j, x);
              if (q->bl_num_up == nbl_up && q->bl_num_down == nbl_dn && q->st_num_up == nst_up &&
                  q->st_num_down == nst_dn) {
                np = q->spos;
                nd = q->sdim;
                break;
              }
            }
            if (kb < 0 || ks < 0 || np < 0) continue;
            double signs = sgn_flag(flag, m->bl_num_down);
            int j1 = nbl_dn, j2 = m->bl_num_down, j3 = d1, j4 = m->st_num_down, j5 = nst_dn, j6 = sd;
            double c1 = 1.0 / sqrt(1.0 + d1) * W6(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * ipow_m1((j2 + j5 + j3 + j6) / 2);
            double coef = signs * st.sub[ks].mat[0] * c1;
            double *mid = (double *)malloc(((size_t)nd * ed + 1) * sizeof(double));
            dg('N', 'N', nd, ed, m->sdim, coef, bl.sub[kb].mat, nd, WP(w, i, m->spos, 0), LD(w, i), 0.0, mid, nd);
            v += dot_cols(WP(w, i, np, 0), LD(w, i), mid, nd, nd, ed);
            free(mid);
          }
      }
    }
  }
  blk_free(&bl);
  blk_free(&st);
  *value = v;
  return 0;
}
/* env_block_site_cor_ndia (measure.f90:5085-5238) */
int ora_env_block_site_cor_ndia(const tj_block *b, const tj_block *stb, const tj_basis *ebs, const tj_wave *w,
                                char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk bl, st;
  blk_view(b, &bl);
  blk_view(stb, &st);
  int up_dif = bl.up_dif, d1 = bl.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up, edn = w->sub[i].env_num_down,
        sdm = w->sub[i].sys_dim;
    for (int j = 0; j < ebs->num; j++) {
      if (ebs->sub[j].new_num_up != eu || ebs->sub[j].new_num_down != edn) continue;
      for (int k = 0; k < ebs->sub[j].num; k++) {
        const tj_basis_sub *m = BM(ebs, j, k);
        for (int bdd = -d1; bdd <= d1; bdd += 2) {
          int nbl_up = m->bl_num_up - up_dif, nbl_dn = m->bl_num_down - bdd;
          int kb = find_sub(&bl, nbl_up, nbl_dn, bdd, 1);
          for (int sdd = -d1; sdd <= d1; sdd += 2) {
            int nst_up = m->st_num_up + up_dif, nst_dn = m->st_num_down + sdd;
            int ks = find_sub(&st, m->st_num_up, m->st_num_down, sdd, 1);
            int np = -1, nd = 0;
            for (int x = 0; x < ebs->sub[j].num; x++) {
              const tj_basis_sub *q = BM(ebs, j, x);
              if (q->bl_num_up == nbl_up && q->bl_num_down == nbl_dn && q->st_num_up == nst_up &&
                  q->st_num_down == nst_dn) {
                np = q->spos;
                nd = q->sdim;
                break;
              }
            }
            if (kb < 0 || ks < 0 || np < 0) continue;
            double signs = sgn_flag(flag, sd + m->st_num_down + sd);
            int j1 = nbl_dn, j2 = m->bl_num_down, j3 = d1, j4 = m->st_num_down, j5 = nst_dn, j6 = edn;
            double c1 = 1.0 / sqrt(1.0 + d1) * W6(j1, j2, j3, j4, j5, j6);
            c1 = c1 * ipow_m1((j2 + j5 + j3 + j6) / 2);
            if (c1 == 0.0) continue;
            double coef = signs * st.sub[ks].mat[0] * c1;
            double *mid = (double *)malloc(((size_t)sdm * nd + 1) * sizeof(double));
            dg('N', 'N', sdm, nd, m->sdim, coef, WP(w, i, 0, m->spos), LD(w, i), bl.sub[kb].mat, m->sdim, 0.0, mid,
               sdm);
            v += dot_cols(WP(w, i, 0, np), LD(w, i), mid, sdm, sdm, nd);
            free(mid);
          }
        }
      }
    }
  }
  blk_free(&bl);
  blk_free(&st);
  *value = v;
  return 0;
}
/* sys_block_env_site_cor_ndia (measure.f90:5482-5706) */
int ora_sys_block_env_site_cor_ndia(const tj_block *a, const tj_block *stb, const tj_basis *sbs, const tj_basis *ebs,
                                    const tj_wave *w, char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk bl, st;
  blk_view(a, &bl);
  blk_view(stb, &st);
  int up_dif = bl.up_dif, d1 = bl.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up,
        edn = w->sub[i].env_num_down;
    for (int j = 0; j < sbs->num; j++) {
      if (sbs->sub[j].new_num_up != su || sbs->sub[j].new_num_down != sd) continue;
      for (int k = 0; k < ebs->num; k++) {
        if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
        for (int x = 0; x < sbs->sub[j].num; x++)
          for (int y = 0; y < ebs->sub[k].num; y++) {
            const tj_basis_sub *ms = BM(sbs, j, x), *me = BM(ebs, k, y);
            for (int bdd = -bl.down_dif; bdd <= bl.down_dif; bdd += 2) {
              int nsb_up = ms->bl_num_up + up_dif, nsb_dn = ms->bl_num_down + bdd;
              int kb = find_sub(&bl, ms->bl_num_up, ms->bl_num_down, bdd, 1);
              for (int sdd = -st.down_dif; sdd <= st.down_dif; sdd += 2) {
                int nes_up = me->st_num_up - up_dif, nes_dn = me->st_num_down - sdd;
                int ks = find_sub(&st, nes_up, nes_dn, sdd, 1);
                if (kb < 0 || ks < 0) continue;
                for (int nsd = abs(sd - bl.down_dif); nsd <= sd + bl.down_dif; nsd += 2) {
                  int nsu = su + up_dif, neu = eu - up_dif, ned = nsd;
                  int nsp = -1, nsdim = 0, nep = -1;
                  for (int mm = 0; mm < sbs->num && nsp < 0; mm++) {
                    if (sbs->sub[mm].new_num_up != nsu || sbs->sub[mm].new_num_down != nsd) continue;
                    for (int n = 0; n < sbs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(sbs, mm, n);
                      if (q->bl_num_up == nsb_up && q->bl_num_down == nsb_dn && q->st_num_up == ms->st_num_up &&
                          q->st_num_down == ms->st_num_down) {
                        nsp = q->spos;
                        nsdim = q->sdim;
                        break;
                      }
                    }
                  }
                  for (int mm = 0; mm < ebs->num && nep < 0; mm++) {
                    if (ebs->sub[mm].new_num_up != neu || ebs->sub[mm].new_num_down != ned) continue;
                    for (int n = 0; n < ebs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(ebs, mm, n);
                      if (q->st_num_up == nes_up && q->st_num_down == nes_dn && q->bl_num_down == me->bl_num_down) {
                        nep = q->spos;
                        break;
                      }
                    }
                  }
                  int wid = find_out(w, nsu, nsd, neu, ned);
                  if (nsp < 0 || nep < 0 || wid < 0) continue;
                  double signs = sgn_flag(flag, sd);
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->bl_num_down, j5 = ms->st_num_down, j6 = nsb_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->st_num_down, j55 = me->bl_num_down, j66 = nes_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  c1 *= W6(j11, j22, j33, j44, j55, j66);
                  if (c1 == 0.0) continue;
                  c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                  if (((j6 + j5 + j3 + j2) / 2 + (j55 + j44 + j11 + j22) / 2) % 2 != 0) c1 = -c1;
                  double coef = signs * st.sub[ks].mat[0] * c1;
                  int ed = me->sdim;
                  double *mat = (double *)malloc(((size_t)nsdim * ed + 1) * sizeof(double));
                  dg('N', 'N', nsdim, ed, ms->sdim, coef, bl.sub[kb].mat, nsdim, WP(w, i, ms->spos, me->spos),
                     LD(w, i), 0.0, mat, nsdim);
                  v += dot_cols(WP(w, wid, nsp, nep), LD(w, wid), mat, nsdim, nsdim, ed);
                  free(mat);
                }
              }
            }
          }
      }
    }
  }
  blk_free(&bl);
  blk_free(&st);
  *value = v;
  return 0;
}
/* sys_site_env_block_cor_ndia (measure.f90:5926-6154) */
int ora_sys_site_env_block_cor_ndia(const tj_block *stb, const tj_block *b, const tj_basis *sbs, const tj_basis *ebs,
                                    const tj_wave *w, char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk st, bl;
  blk_view(stb, &st);
  blk_view(b, &bl);
  int up_dif = st.up_dif, d1 = st.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up,
        edn = w->sub[i].env_num_down;
    for (int j = 0; j < sbs->num; j++) {
      if (sbs->sub[j].new_num_up != su || sbs->sub[j].new_num_down != sd) continue;
      for (int k = 0; k < ebs->num; k++) {
        if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
        for (int x = 0; x < sbs->sub[j].num; x++)
          for (int y = 0; y < ebs->sub[k].num; y++) {
            const tj_basis_sub *ms = BM(sbs, j, x), *me = BM(ebs, k, y);
            for (int sdd = -st.down_dif; sdd <= st.down_dif; sdd += 2) {
              int nss_up = ms->st_num_up + up_dif, nss_dn = ms->st_num_down + sdd;
              int ks = find_sub(&st, ms->st_num_up, ms->st_num_down, sdd, 1);
              for (int bdd = -bl.down_dif; bdd <= bl.down_dif; bdd += 2) {
                int neb_up = me->bl_num_up - up_dif, neb_dn = me->bl_num_down - bdd;
                int kb = find_sub(&bl, neb_up, neb_dn, bdd, 1);
                if (ks < 0 || kb < 0) continue;
                for (int nsd = abs(sd - st.down_dif); nsd <= sd + st.down_dif; nsd += 2) {
                  int nsu = su + up_dif, neu = eu - up_dif, ned = nsd;
                  int nsp = -1, nep = -1, nedim = 0;
                  for (int mm = 0; mm < sbs->num && nsp < 0; mm++) {
                    if (sbs->sub[mm].new_num_up != nsu || sbs->sub[mm].new_num_down != nsd) continue;
                    for (int n = 0; n < sbs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(sbs, mm, n);
                      if (q->st_num_up == nss_up && q->st_num_down == nss_dn && q->bl_num_down == ms->bl_num_down) {
                        nsp = q->spos;
                        break;
                      }
                    }
                  }
                  for (int mm = 0; mm < ebs->num && nep < 0; mm++) {
                    if (ebs->sub[mm].new_num_up != neu || ebs->sub[mm].new_num_down != ned) continue;
                    for (int n = 0; n < ebs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(ebs, mm, n);
                      if (q->bl_num_up == neb_up && q->bl_num_down == neb_dn && q->st_num_down == me->st_num_down) {
                        nep = q->spos;
                        nedim = q->sdim;
                        break;
                      }
                    }
                  }
                  int wid = find_out(w, nsu, nsd, neu, ned);
                  if (nsp < 0 || nep < 0 || wid < 0) continue;
                  double signs = sgn_flag(flag, sd + me->st_num_down + ms->bl_num_down);
                  double coef = signs * st.sub[ks].mat[0];
                  if (coef == 0.0) continue;
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->st_num_down, j5 = ms->bl_num_down, j6 = nss_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->bl_num_down, j55 = me->st_num_down, j66 = neb_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  c1 *= W6(j11, j22, j33, j44, j55, j66);
                  if (c1 == 0.0) continue;
                  c1 *= sqrt((1.0 + j11) * (j33 + 1.0) / (1.0 + d1));
                  if (((j66 + j55 + j33 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                  coef = coef * c1;
                  int sdm = ms->sdim, ed = me->sdim;
                  double *mat = (double *)malloc(((size_t)sdm * ed + 1) * sizeof(double));
                  dg('N', 'T', sdm, ed, nedim, coef, WP(w, wid, nsp, nep), LD(w, wid), bl.sub[kb].mat, ed, 0.0, mat,
                     sdm);
                  v += dot_cols(mat, sdm, WP(w, i, ms->spos, me->spos), LD(w, i), sdm, ed);
                  free(mat);
                }
              }
            }
          }
      }
    }
  }
  blk_free(&st);
  blk_free(&bl);
  *value = v;
  return 0;
}
/* sys_site_env_site_cor_ndia (measure.f90:5709-5924) */
int ora_sys_site_env_site_cor_ndia(const tj_block *stb, const tj_block *st2b, const tj_basis *sbs,
                                   const tj_basis *ebs, const tj_wave *w, char flag, double *value) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk st, et;
  blk_view(stb, &st);
  blk_view(st2b, &et);
  int up_dif = st.up_dif, d1 = st.down_dif;
  double v = 0.0;
  for (int i = 0; i < w->num; i++) {
    int su = w->sub[i].sys_num_up, sd = w->sub[i].sys_num_down, eu = w->sub[i].env_num_up,
        edn = w->sub[i].env_num_down;
    for (int j = 0; j < sbs->num; j++) {
      if (sbs->sub[j].new_num_up != su || sbs->sub[j].new_num_down != sd) continue;
      for (int k = 0; k < ebs->num; k++) {
        if (ebs->sub[k].new_num_up != eu || ebs->sub[k].new_num_down != edn) continue;
        for (int x = 0; x < sbs->sub[j].num; x++)
          for (int y = 0; y < ebs->sub[k].num; y++) {
            const tj_basis_sub *ms = BM(sbs, j, x), *me = BM(ebs, k, y);
            for (int sdd1 = -st.down_dif; sdd1 <= st.down_dif; sdd1 += 2) {
              int nss_up = ms->st_num_up + up_dif, nss_dn = ms->st_num_down + sdd1;
              int ks = find_sub(&st, ms->st_num_up, ms->st_num_down, sdd1, 1);
              for (int sdd2 = -st.down_dif; sdd2 <= st.down_dif; sdd2 += 2) {
                int nes_up = me->st_num_up - up_dif, nes_dn = me->st_num_down - sdd2;
                int ke = find_sub(&et, nes_up, nes_dn, sdd2, 1);
                if (ks < 0 || ke < 0) continue;
                for (int nsd = abs(sd - st.down_dif); nsd <= sd + st.down_dif; nsd += 2) {
                  int nsu = su + up_dif, neu = eu - up_dif, ned = nsd;
                  int nsp = -1, nep = -1;
                  for (int mm = 0; mm < sbs->num && nsp < 0; mm++) {
                    if (sbs->sub[mm].new_num_up != nsu || sbs->sub[mm].new_num_down != nsd) continue;
                    for (int n = 0; n < sbs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(sbs, mm, n);
                      if (q->st_num_up == nss_up && q->st_num_down == nss_dn && q->bl_num_down == ms->bl_num_down) {
                        nsp = q->spos;
                        break;
                      }
                    }
                  }
                  for (int mm = 0; mm < ebs->num && nep < 0; mm++) {
                    if (ebs->sub[mm].new_num_up != neu || ebs->sub[mm].new_num_down != ned) continue;
                    for (int n = 0; n < ebs->sub[mm].num; n++) {
                      const tj_basis_sub *q = BM(ebs, mm, n);
                      if (q->st_num_up == nes_up && q->st_num_down == nes_dn && q->bl_num_down == me->bl_num_down) {
                        nep = q->spos;
                        break;
                      }
                    }
                  }
                  int wid = find_out(w, nsu, nsd, neu, ned);
                  if (nsp < 0 || nep < 0 || wid < 0) continue;
                  double signs = sgn_flag(flag, sd + ms->bl_num_down);
                  double coef = signs * st.sub[ks].mat[0] * et.sub[ke].mat[0];
                  if (coef == 0.0) continue;
                  int j1 = nsd, j2 = d1, j3 = sd, j4 = ms->st_num_down, j5 = ms->bl_num_down, j6 = nss_dn;
                  int j11 = ned, j22 = d1, j33 = edn, j44 = me->st_num_down, j55 = me->bl_num_down, j66 = nes_dn;
                  double c1 = W6(j1, j2, j3, j4, j5, j6);
                  if (c1 == 0.0) continue;
                  c1 *= W6(j11, j22, j33, j44, j55, j66);
                  if (c1 == 0.0) continue;
                  c1 *= sqrt((1.0 + j11) * (1.0 + j33) / (1.0 + d1));
                  if (((j55 + j44 + j11 + j22) / 2 + (j5 + j4 + j1 + j2) / 2) % 2 != 0) c1 = -c1;
                  coef = coef * c1;
                  double t = dot_cols(WP(w, wid, nsp, nep), LD(w, wid), WP(w, i, ms->spos, me->spos), LD(w, i),
                                      ms->sdim, me->sdim);
                  v += t * coef;
                }
              }
            }
          }
      }
    }
  }
  blk_free(&st);
  blk_free(&et);
  *value = v;
  return 0;
}

/* ============================================ operator renormalisation */
/* Get_Hamiltonian_Sys / Get_Hamiltonian_Env (get_sys.f90:4-480) with the
 * block-update routines they call (block.f90:382-1503).  Every routine builds
 * its new block as a dense sub-block per sector (pair), as the reference
 * does, and the truncation is the reference's pair of DGEMMs per sub-block. */

static OSub *osub_alloc(int n) { return (OSub *)calloc(n > 0 ? n : 1, sizeof(OSub)); }
static double *mat_zero(int r, int c) { return (double *)calloc((size_t)r * c + 1, sizeof(double)); }
static void blk_new(OBlk *o, int len, int num, int up_dif, int down_dif) {
  memset(o, 0, sizeof *o);
  o->len = len; o->num = num; o->up_dif = up_dif; o->down_dif = down_dif;
  o->sub = osub_alloc(num);
  o->owns = 1;
}
/* block_transfer (block.f90:1708-1735): a deep copy */
static void blk_copy(const OBlk *in, OBlk *out) {
  blk_new(out, in->len, in->num, in->up_dif, in->down_dif);
  out->dim = in->dim;
  for (int i = 0; i < in->num; i++) {
    out->sub[i] = in->sub[i];
    size_t n = (size_t)in->sub[i].row_dim * in->sub[i].sdim;
    out->sub[i].mat = (double *)malloc((n + 1) * sizeof(double));
    memcpy(out->sub[i].mat, in->sub[i].mat, n * sizeof(double));
  }
}
/* mat(r0.., c0..) += a * src(0.., 0..) over nr x nc (src leading dimension lds) */
static void mat_axpy(double *m, int ldm, int r0, int c0, double a, const double *src, int lds, int nr, int nc) {
  for (int c = 0; c < nc; c++)
    for (int r = 0; r < nr; r++) m[(size_t)(c0 + c) * ldm + r0 + r] += a * src[(size_t)c * lds + r];
}

/* update_block_dia (block.f90:382-433) */
static void upd_block_dia(const OBlk *blk, const tj_basis *bs, OBlk *nb) {
  blk_new(nb, bs->len, bs->num, 0, 0);
  nb->dim = bs->dim;
  for (int i = 0; i < bs->num; i++) {
    int d = bs->sub[i].dim;
    nb->sub[i] = (OSub){bs->sub[i].new_num_up, bs->sub[i].new_num_down, 0, d, d, mat_zero(d, d)};
  }
  for (int k = 0; k < nb->num; k++)
    for (int x = 0; x < bs->sub[k].num; x++) {
      const tj_basis_sub *m = BM(bs, k, x);
      for (int i = 0; i < blk->num; i++) {
        if (blk->sub[i].num_up != m->bl_num_up || blk->sub[i].num_down != m->bl_num_down) continue;
        double c1 = sqrt((1.0 + nb->sub[k].num_down) / (1.0 + blk->sub[i].num_down));
        mat_axpy(nb->sub[k].mat, nb->sub[k].row_dim, m->spos, m->spos, c1, blk->sub[i].mat, blk->sub[i].row_dim,
                 m->sdim, m->sdim);
        break;
      }
    }
}
/* update_site_dia (block.f90:439-494) */
static void upd_site_dia(const OBlk *site, const tj_basis *bs, OBlk *nb) {
  blk_new(nb, bs->len, bs->num, 0, 0);
  nb->dim = bs->dim;
  for (int i = 0; i < bs->num; i++) {
    int d = bs->sub[i].dim;
    nb->sub[i] = (OSub){bs->sub[i].new_num_up, bs->sub[i].new_num_down, 0, d, d, mat_zero(d, d)};
  }
  for (int k = 0; k < nb->num; k++)
    for (int x = 0; x < bs->sub[k].num; x++) {
      const tj_basis_sub *m = BM(bs, k, x);
      for (int i = 0; i < site->num; i++) {
        if (site->sub[i].num_up != m->st_num_up || site->sub[i].num_down != m->st_num_down) continue;
        double c1 = sqrt((1.0 + nb->sub[k].num_down) / (1.0 + site->sub[i].num_down));
        double v = site->sub[i].mat[0] * c1;
        for (int y = 0; y < m->sdim; y++) nb->sub[k].mat[(size_t)(m->spos + y) * nb->sub[k].row_dim + m->spos + y] += v;
        break;
      }
    }
}
/* The sub-block structure shared by update_block_ndia_sys/env and
 * update_site_ndia_sys/env (steps <1>-<2>): one sub-block per basis sector x
 * and spin transfer down_dif in -d..d (step su = 2) whose target sector
 * exists, in that loop order. */
static void ndia_structure(const tj_basis *bs, int len, int up_dif, int d1, OBlk *nb) {
  int num = 0;
  for (int x = 0; x < bs->num; x++)
    for (int dd = -d1; dd <= d1; dd += 2)
      if (find_bs(bs, bs->sub[x].new_num_up + up_dif, bs->sub[x].new_num_down + dd) >= 0) num++;
  blk_new(nb, len, num, up_dif, d1);
  int id = 0;
  for (int x = 0; x < bs->num; x++)
    for (int dd = -d1; dd <= d1; dd += 2) {
      int y = find_bs(bs, bs->sub[x].new_num_up + up_dif, bs->sub[x].new_num_down + dd);
      if (y < 0) continue;
      int ld = bs->sub[y].dim, rd = bs->sub[x].dim;
      nb->dim += rd;
      nb->sub[id++] = (OSub){bs->sub[x].new_num_up, bs->sub[x].new_num_down, dd, ld, rd, mat_zero(ld, rd)};
    }
}
/* update_block_ndia_sys (block.f90:497-690), env_side = 0, and
 * update_block_ndia_env (block.f90:695-881), env_side = 1 (fermion sign
 * from the parity of the site's 2S) */
static void upd_block_ndia(const OBlk *blk, const tj_basis *bs, OBlk *nb, int env_side, char flag) {
  const int up_dif = blk->up_dif, d1 = blk->down_dif;
  ndia_structure(bs, bs->len, up_dif, d1, nb);
  for (int i = 0; i < nb->num; i++) {
    int rnu = nb->sub[i].num_up, rnd = nb->sub[i].num_down, dd = nb->sub[i].down_dif;
    int rid = find_bs(bs, rnu, rnd), lid = find_bs(bs, rnu + up_dif, rnd + dd);
    if (rid < 0 || lid < 0) continue;
    int lnd = rnd + dd;
    for (int x = 0; x < bs->sub[rid].num; x++) {
      const tj_basis_sub *m = BM(bs, rid, x);
      for (int sdd = -d1; sdd <= d1; sdd += 2) {
        int bid = find_sub(blk, m->bl_num_up, m->bl_num_down, sdd, 1);
        if (bid < 0) continue;
        int lsnu = m->bl_num_up + up_dif, lsnd = m->bl_num_down + sdd;
        const tj_basis_sub *ml = NULL;
        for (int y = 0; y < bs->sub[lid].num; y++) {
          const tj_basis_sub *q = BM(bs, lid, y);
          if (q->bl_num_up == lsnu && q->bl_num_down == lsnd && q->st_num_down == m->st_num_down) {
            ml = q;
            break;
          }
        }
        if (!ml) continue;
        double signs = 1.0;
        if (env_side) signs = sgn_flag(flag, m->st_num_down);
        int j1 = lnd, j2 = d1, j3 = rnd, j4 = m->bl_num_down, j5 = m->st_num_down, j6 = lsnd;
        double coef = W6(j1, j2, j3, j4, j5, j6) * sqrt((1.0 + j1) * (1.0 + j3)) * ipow_m1((j6 + j5 + j3 + j2) / 2);
        if (coef == 0.0) continue;
        coef *= signs;
        mat_axpy(nb->sub[i].mat, nb->sub[i].row_dim, ml->spos, m->spos, coef, blk->sub[bid].mat, blk->sub[bid].row_dim,
                 ml->sdim, m->sdim);
      }
    }
  }
}
/* update_site_ndia_sys (block.f90:888-1105), env_side = 0 (fermion sign from
 * the parity of the block's 2S), and update_site_ndia_env (block.f90:1107-
 * 1306), env_side = 1 (no sign) */
static void upd_site_ndia(const OBlk *site, const tj_basis *bs, OBlk *nb, int env_side, char flag) {
  const int up_dif = site->up_dif, d1 = site->down_dif;
  ndia_structure(bs, bs->len, up_dif, d1, nb);
  for (int i = 0; i < nb->num; i++) {
    int rnu = nb->sub[i].num_up, rnd = nb->sub[i].num_down, dd = nb->sub[i].down_dif;
    int rid = find_bs(bs, rnu, rnd), lid = find_bs(bs, rnu + up_dif, rnd + dd);
    if (rid < 0 || lid < 0) continue;
    int lnd = rnd + dd;
    for (int x = 0; x < bs->sub[rid].num; x++) {
      const tj_basis_sub *m = BM(bs, rid, x);
      for (int sdd = -d1; sdd <= d1; sdd += 2) {
        int sid = find_sub(site, m->st_num_up, m->st_num_down, sdd, 1);
        if (sid < 0) continue;
        int lsnu = m->st_num_up + up_dif, lsnd = m->st_num_down + sdd;
        const tj_basis_sub *ml = NULL;
        for (int y = 0; y < bs->sub[lid].num; y++) {
          const tj_basis_sub *q = BM(bs, lid, y);
          if (q->st_num_up == lsnu && q->st_num_down == lsnd && q->bl_num_down == m->bl_num_down) {
            ml = q;
            break;
          }
        }
        if (!ml) continue;
        double signs = env_side ? 1.0 : sgn_flag(flag, m->bl_num_down);
        int j1 = lnd, j2 = d1, j3 = rnd, j4 = m->st_num_down, j5 = m->bl_num_down, j6 = lsnd;
        double coef = W6(j1, j2, j3, j4, j5, j6) * ipow_m1((j5 + j4 + j1 + j2) / 2) * sqrt((1.0 + j1) * (1.0 + j3));
        if (coef == 0.0) continue;
        coef *= signs;
        double v = coef * site->sub[sid].mat[0];
        for (int y = 0; y < m->sdim; y++)
          nb->sub[i].mat[(size_t)(m->spos + y) * nb->sub[i].row_dim + ml->spos + y] += v;
      }
    }
  }
}
/* Get_hamiltonian_ndia (get_sys.f90:578-759): coef * [block x site^T + h.c.]
 * added into the enlarged Hamiltonian; sys_side = 1 for Flags = 'S' */
static void ham_ndia(const OBlk *blk, const OBlk *site, const tj_basis *bs, double coef, OBlk *ham, char flagsign,
                     int sys_side) {
  const int up_dif = blk->up_dif, d1 = blk->down_dif;
  for (int i = 0; i < ham->num; i++) {
    int rnu = ham->sub[i].num_up, rnd = ham->sub[i].num_down;
    int rid = find_bs(bs, rnu, rnd), lid = find_bs(bs, rnu, rnd + ham->sub[i].down_dif);
    if (rid < 0 || lid < 0) continue;
    for (int x = 0; x < bs->sub[rid].num; x++) {
      const tj_basis_sub *m = BM(bs, rid, x);
      for (int sdd = -d1; sdd <= d1; sdd += 2) {
        int bid = find_sub(blk, m->bl_num_up, m->bl_num_down, sdd, 1);
        if (bid < 0) continue;
        int lsnu = m->bl_num_up + up_dif, lsnd = m->bl_num_down + sdd;
        for (int nsd = abs(m->st_num_down - site->down_dif); nsd <= m->st_num_down + site->down_dif; nsd += 2) {
          int st_dd = m->st_num_down - nsd, nsu = m->st_num_up - site->up_dif;
          int sid = find_sub(site, nsu, nsd, st_dd, 1);
          const tj_basis_sub *ml = NULL;
          for (int y = 0; y < bs->sub[lid].num; y++) {
            const tj_basis_sub *q = BM(bs, lid, y);
            if (q->bl_num_up == lsnu && q->bl_num_down == lsnd && q->st_num_down == nsd) {
              ml = q;
              break;
            }
          }
          if (!ml || sid < 0) continue;
          int j1 = lsnd, j2 = m->bl_num_down, j3 = d1, j4 = m->st_num_down, j5 = nsd, j6 = rnd;
          double c1 = W6(j1, j2, j3, j4, j5, j6);
          c1 = c1 * sqrt((1.0 + j6) / (1.0 + j3)) * ipow_m1((j2 + j5 + j3 + j6) / 2) * site->sub[sid].mat[0];
          double sign = 1.0;
          if (sys_side && flagsign == 'F') {
            if (m->bl_num_up % 2 == 1) sign = -1.0;
            if (m->bl_num_down % 2 == 1) sign = -1.0;
          }
          if (c1 == 0.0) continue;
          c1 = c1 * coef * sign;
          const OSub *b = &blk->sub[bid];
          mat_axpy(ham->sub[i].mat, ham->sub[i].row_dim, ml->spos, m->spos, c1, b->mat, b->row_dim, ml->sdim, m->sdim);
          if (site->down_dif == 1) {
            for (int c = 0; c < ml->sdim; c++)
              for (int r = 0; r < m->sdim; r++)
                ham->sub[i].mat[(size_t)(ml->spos + c) * ham->sub[i].row_dim + m->spos + r] +=
                    c1 * b->mat[(size_t)r * b->row_dim + c];
          }
        }
      }
    }
  }
}
/* Get_hamiltonian_dia (get_sys.f90:507-565) with Flag1 = Flag2 = 'N' and no
 * conjugate part, as Get_Hamiltonian_Sys/Env call it */
static void ham_dia(const OBlk *o1, const OBlk *o2, double coef, OBlk *ham) {
  for (int i = 0; i < ham->num; i++) {
    int nu = ham->sub[i].num_up, nd = ham->sub[i].num_down, sd = ham->sub[i].sdim;
    int a = find_sub(o1, nu, nd, 0, 0), b = find_sub(o2, nu, nd, 0, 0);
    if (a < 0 || b < 0) continue;
    double c1 = coef / sqrt(1.0 + nd);
    dg('N', 'N', sd, sd, sd, c1, o1->sub[a].mat, sd, o2->sub[b].mat, sd, 1.0, ham->sub[i].mat, sd);
  }
}
/* update_trun_dia (block.f90:1311-1362) */
static void upd_trun_dia(const OBlk *ori, const OBlk *trun, OBlk *eff) {
  blk_new(eff, ori->len, trun->num, ori->up_dif, ori->down_dif);
  eff->dim = trun->dim;
  for (int i = 0; i < trun->num; i++) {
    int k = trun->sub[i].sdim;
    eff->sub[i] = (OSub){trun->sub[i].num_up, trun->sub[i].num_down, 0, k, k, mat_zero(k, k)};
  }
  for (int i = 0; i < eff->num; i++) {
    int ed = eff->sub[i].sdim;
    int x = find_sub(ori, eff->sub[i].num_up, eff->sub[i].num_down, 0, 0);
    if (x < 0) continue;
    int od = ori->sub[x].row_dim;
    double *mid = mat_zero(od, ed);
    dg('N', 'N', od, ed, od, 1.0, ori->sub[x].mat, od, trun->sub[i].mat, od, 0.0, mid, od);
    dg('T', 'N', ed, ed, od, 1.0, trun->sub[i].mat, od, mid, od, 0.0, eff->sub[i].mat, ed);
    free(mid);
  }
}
/* update_trun_ndia (block.f90:1365-1503) */
static void upd_trun_ndia(const OBlk *ori, const OBlk *trun, OBlk *eff) {
  const int up_dif = ori->up_dif, d1 = ori->down_dif;
  int num = 0;
  for (int x = 0; x < trun->num; x++)
    for (int dd = -d1; dd <= d1; dd += 2)
      if (find_sub(trun, trun->sub[x].num_up + up_dif, trun->sub[x].num_down + dd, 0, 0) >= 0) num++;
  blk_new(eff, ori->len, num, up_dif, d1);
  int id = 0;
  for (int x = 0; x < trun->num; x++)
    for (int dd = -d1; dd <= d1; dd += 2) {
      int y = find_sub(trun, trun->sub[x].num_up + up_dif, trun->sub[x].num_down + dd, 0, 0);
      if (y < 0) continue;
      int ld = trun->sub[y].sdim, rd = trun->sub[x].sdim;
      eff->dim += rd;
      eff->sub[id++] = (OSub){trun->sub[x].num_up, trun->sub[x].num_down, dd, ld, rd, mat_zero(ld, rd)};
    }
  for (int i = 0; i < eff->num; i++) {
    int rnu = eff->sub[i].num_up, rnd = eff->sub[i].num_down, dd = eff->sub[i].down_dif;
    int rid = find_sub(trun, rnu, rnd, 0, 0), lid = find_sub(trun, rnu + up_dif, rnd + dd, 0, 0);
    int oid = find_sub(ori, rnu, rnd, dd, 1);
    if (rid < 0 || lid < 0 || oid < 0) continue;
    int orow = ori->sub[oid].row_dim, ocol = ori->sub[oid].sdim;
    int rd = trun->sub[rid].sdim, ld = trun->sub[lid].sdim;
    double *mid = mat_zero(orow, rd);
    dg('N', 'N', orow, rd, ocol, 1.0, ori->sub[oid].mat, orow, trun->sub[rid].mat, ocol, 0.0, mid, orow);
    dg('T', 'N', ld, rd, orow, 1.0, trun->sub[lid].mat, orow, mid, orow, 0.0, eff->sub[i].mat, ld);
    free(mid);
  }
}

/* Writes a model into the two-call result (layout of tj_model_result). */
static void put_block(const OBlk *b, tj_model_result *out, int *ns, int64_t *nd, tj_block *dst) {
  const int write = out->sets && out->subs && out->data;
  if (write) {
    *dst = (tj_block){b->len, b->num, b->dim, b->up_dif, b->down_dif, 0, out->subs + *ns, out->data};
  }
  for (int i = 0; i < b->num; i++) {
    const OSub *s = &b->sub[i];
    const int64_t n = (int64_t)s->row_dim * s->sdim;
    if (write) {
      out->subs[*ns + i] = (tj_block_sub){s->num_up, s->num_down, s->down_dif, s->row_dim, s->sdim, 0, *nd};
      memcpy(out->data + *nd, s->mat, (size_t)n * sizeof(double));
    }
    *nd += n;
  }
  *ns += b->num;
}

/* Get_Hamiltonian_Sys (get_sys.f90:4-239), side 0, and Get_Hamiltonian_Env
 * (get_sys.f90:245-480), side 1. */
int ora_get_hamiltonian(const tj_lattice *lat, int side, int mshift, const tj_model *prem, const tj_basis *basis,
                        const tj_block *trunb, tj_model_result *out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  if (!lat || !prem || !basis || !trunb || !out) return fail(TJ_ERR_ARG, "ora_get_hamiltonian: null argument");
  Geo g;
  memset(&g, 0, sizeof g);
  g.L = lat;
  g.ns1 = lat->num_site + 1;
  const int neibt = lat->neibt, len0 = prem->len, env = side != 0;
  SiteOps so;
  site_ops_build(lat->up_bias, &so);
  OModel pre;
  model_view(prem, &pre, 0);
  OBlk trun;
  blk_view(trunb, &trun);
  const int nl0 = NLEG11(&g, len0), nl1 = NLEG11(&g, len0 + 1);
  const int nslot = (nl0 > nl1 ? nl0 : nl1) + 1;
  OSet *next = (OSet *)calloc(nslot, sizeof(OSet));   /* next%sub(1:...) */
  OSet *res = (OSet *)calloc(nl1 > 0 ? nl1 : 1, sizeof(OSet));
  OBlk next_ham, tmp, tmp1, new_ham;
  memset(&tmp, 0, sizeof tmp);
  memset(&tmp1, 0, sizeof tmp1);
  int rc = 0;
  if (pre.nsub < nl0) {
    rc = fail(TJ_ERR_ARG, "ora_get_hamiltonian: pre has fewer operator sets than nleg11(len)");
    goto done;
  }
  upd_block_dia(&pre.ham, basis, &next_ham);
  /* the new site J, the block site II it bonds to, and the coupling row */
  for (int ij = 1; ij <= 5; ij += 2) {
    const int J = env ? len0 + 1 + mshift : len0 + 1;
    const int jl = env ? NPOSI_LAT(&g, J) : J;   /* lattice index of the new site */
    for (int k = 1; k <= neibt; k++) {
      int I = NEIB(&g, jl, k);
      int II = env ? NPOSI_DM(&g, I) - mshift : I;
      if (!(II <= len0 && II > 0)) continue;
      int i1 = INB1(&g, II, len0);
      if (!(i1 > 0 && i1 <= nl0)) continue;
      double coefx = JT(&g, k, jl), coefsd = JD(&g, k, jl);
      if (ij == 1 && coefx != 0.0)
        ham_ndia(&pre.sub[i1 - 1].op[EU], &so.eu, basis, coefx, &next_ham, 'F', !env);
      if (ij == 3 && coefsd != 0.0)
        ham_ndia(&pre.sub[i1 - 1].op[SD], &so.sd, basis, coefsd, &next_ham, 'B', !env);
    }
    for (int y = 1; y <= len0; y++) {
      int i1 = INB1(&g, y, len0);
      if (i1 > nl0 || i1 < 1) continue;
      OSet *p = &pre.sub[i1 - 1], *n = &next[i1];
      if (ij == 1) {
        blk_free(&n->op[EU]);
        blk_free(&n->op[ED]);
        upd_block_ndia(&p->op[EU], basis, &n->op[EU], env, 'F');
        upd_block_ndia(&p->op[ED], basis, &n->op[ED], env, 'F');
      } else if (ij == 3) {
        blk_free(&n->op[SD]);
        upd_block_ndia(&p->op[SD], basis, &n->op[SD], env, 'B');
      } else {
        blk_free(&n->op[SN]);
        upd_block_dia(&p->op[SN], basis, &n->op[SN]);
      }
    }
    blk_free(&tmp);
    blk_free(&tmp1);
    if (ij == 1) {
      upd_site_ndia(&so.eu, basis, &tmp, env, 'F');
      upd_site_ndia(&so.ed, basis, &tmp1, env, 'F');
    } else if (ij == 3) {
      upd_site_ndia(&so.sd, basis, &tmp, env, 'B');
    } else {
      upd_site_dia(&so.ne, basis, &tmp);
    }
    if (ij == 5) {
      for (int k = 1; k <= neibt; k++) {
        int I = NEIB(&g, jl, k);
        int II = env ? NPOSI_DM(&g, I) - mshift : I;
        if (!(II <= len0 && II > 0)) continue;
        int i1 = INB1(&g, II, len0);
        if (!(i1 > 0 && i1 <= nl0)) continue;
        ham_dia(&next[i1].op[SN], &tmp, JN(&g, k), &next_ham);
      }
      if (ESITE(&g, jl) != 0.0) blk_add_two(&tmp, ESITE(&g, jl), &next_ham);
    }
    /* reorder: operators of the sites that keep bonds, then the new site */
    const int kind[2] = {ij == 1 ? EU : ij == 3 ? SD : SN, ED};
    const int nk = ij == 1 ? 2 : 1;
    for (int I = 1; I <= len0; I++) {
      int i1 = INB1(&g, I, len0), j = INB1(&g, I, len0 + 1);
      if (j <= nl1 && j != i1)
        for (int q = 0; q < nk; q++) {
          blk_free(&next[j].op[kind[q]]);
          blk_copy(&next[i1].op[kind[q]], &next[j].op[kind[q]]);
        }
    }
    {
      int j = INB1(&g, len0 + 1, len0 + 1);
      if (j < 1 || j >= nslot) {
        rc = fail(TJ_ERR_ARG, "ora_get_hamiltonian: new site has no operator slot");
        goto done;
      }
      blk_free(&next[j].op[kind[0]]);
      blk_copy(&tmp, &next[j].op[kind[0]]);
      if (ij == 1) {
        blk_free(&next[j].op[ED]);
        blk_copy(&tmp1, &next[j].op[ED]);
      }
    }
    for (int ii = 1; ii <= nl1; ii++)
      for (int q = 0; q < nk; q++) {
        if (ij == 5)
          upd_trun_dia(&next[ii].op[SN], &trun, &res[ii - 1].op[SN]);
        else
          upd_trun_ndia(&next[ii].op[kind[q]], &trun, &res[ii - 1].op[kind[q]]);
      }
  }
  upd_trun_dia(&next_ham, &trun, &new_ham);
  {
    /* result: ham, then sets 1..nl1 (elec_up, elec_down, spin_sd, spin_sz (empty), num_sn) */
    int ns = 0;
    int64_t nd = 0;
    tj_block tb;
    put_block(&new_ham, out, &ns, &nd, &tb);
    if (out->sets && out->subs && out->data) out->model.ham = tb;
    for (int ii = 0; ii < nl1; ii++) {
      OBlk empty;
      blk_new(&empty, len0 + 1, 0, 0, 0);
      const OBlk *ops[5] = {&res[ii].op[EU], &res[ii].op[ED], &res[ii].op[SD], &empty, &res[ii].op[SN]};
      tj_block b5[5];
      for (int q = 0; q < 5; q++) put_block(ops[q], out, &ns, &nd, &b5[q]);
      if (out->sets && out->subs && out->data)
        out->sets[ii] = (tj_block_set){b5[0], b5[1], b5[2], b5[3], b5[4]};
      blk_free(&empty);
    }
    out->len = len0 + 1;
    out->nsub = nl1;
    out->n_subs = ns;
    out->data_len = nd;
    if (out->sets && out->subs && out->data) {
      out->model.len = len0 + 1;
      out->model.nsub = nl1;
      out->model.sub = out->sets;
    }
  }
  blk_free(&new_ham);
done:
  blk_free(&next_ham);
  blk_free(&tmp);
  blk_free(&tmp1);
  for (int i = 0; i < nslot; i++)
    for (int q = 0; q < 5; q++) blk_free(&next[i].op[q]);
  for (int i = 0; i < (nl1 > 0 ? nl1 : 1); i++)
    for (int q = 0; q < 5; q++) blk_free(&res[i].op[q]);
  free(next);
  free(res);
  blk_free(&trun);
  model_free(&pre);
  return rc;
}

/* ============================================ wavefunction prediction */
static void wave_norm_scale(tj_wave *w) {
  double s = wave_product(w, w->data, w->data);
  wave_scale(w->dim, w->data, sqrt(s));   /* divides by the norm */
}
/* wave_trans_LR (dmrg_sub.f90:1093-1238), direction 0, and wave_trans_RL
 * (dmrg_sub.f90:1242-1384), direction 1 */
int ora_wave_trans(int direction, const tj_basis *sys_bs, const tj_basis *env_bs, const tj_block *sys_trunb,
                   const tj_block *env_trunb, const tj_wave *old, tj_wave *nw) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  if (!sys_bs || !env_bs || !sys_trunb || !env_trunb || !old || !nw) return fail(TJ_ERR_ARG, "ora_wave_trans: null");
  OBlk st, et;
  blk_view(sys_trunb, &st);
  blk_view(env_trunb, &et);
  memset(nw->data, 0, (size_t)nw->dim * sizeof(double));
  for (int i = 0; i < old->num; i++) {
    const int snu = old->sub[i].sys_num_up, snd = old->sub[i].sys_num_down;
    const int enu = old->sub[i].env_num_up, end = old->sub[i].env_num_down;
    const int osd = old->sub[i].sys_dim, oed = old->sub[i].env_dim;
    if (direction == 0) {
      const int tid = find_sub(&st, snu, snd, 0, 0);
      if (tid < 0) continue;
      for (int k = 0; k < env_bs->num; k++) {
        if (env_bs->sub[k].new_num_up != enu || env_bs->sub[k].new_num_down != end) continue;
        for (int x = 0; x < env_bs->sub[k].num; x++) {
          const tj_basis_sub *m = BM(env_bs, k, x);
          const int stu = m->st_num_up, std_ = m->st_num_down, neu = m->bl_num_up, ned = m->bl_num_down;
          const int opos = m->spos, osub = m->sdim;
          const int eid = find_sub(&et, neu, ned, 0, 0);
          for (int nsd = abs(snd - std_); nsd <= snd + std_; nsd += 2) {
            const int nsu = snu + stu;
            int bid = -1, bsub = -1;
            for (int y = 0; y < sys_bs->num && bid < 0; y++) {
              if (sys_bs->sub[y].new_num_up != nsu || sys_bs->sub[y].new_num_down != nsd) continue;
              for (int z = 0; z < sys_bs->sub[y].num; z++) {
                const tj_basis_sub *q = BM(sys_bs, y, z);
                if (q->bl_num_up == snu && q->bl_num_down == snd && q->st_num_up == stu && q->st_num_down == std_) {
                  bid = y;
                  bsub = z;
                  break;
                }
              }
            }
            const int wid = find_out(nw, nsu, nsd, neu, ned);
            if (eid < 0 || bid < 0 || wid < 0) continue;
            const int nedim = nw->sub[wid].env_dim;
            const int npos = BM(sys_bs, bid, bsub)->spos, nsub = BM(sys_bs, bid, bsub)->sdim;
            const int j12 = snd, j3 = std_, j4 = ned, j123 = nsd, j34 = end;
            double c1 = ipow_m1((j12 + j3 + j123) / 2) / sqrt((1.0 + j12) * (1.0 + j123));
            c1 *= sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j12 + j3 + j4) / 2) % 2 != 0) c1 = -c1;
            if (((j3 + j4 - j34) / 2) % 2 != 0) c1 = -c1;
            double *sub = mat_zero(nsub, osub);
            dg('T', 'N', nsub, osub, osd, c1, st.sub[tid].mat, osd, WP(old, i, 0, opos), LD(old, i), 0.0, sub, nsub);
            dg('N', 'T', nsub, nedim, osub, 1.0, sub, nsub, et.sub[eid].mat, nedim, 1.0, WP(nw, wid, npos, 0),
               LD(nw, wid));
            free(sub);
          }
        }
      }
    } else {
      const int tid = find_sub(&et, enu, end, 0, 0);
      if (tid < 0) continue;
      for (int k = 0; k < sys_bs->num; k++) {
        if (sys_bs->sub[k].new_num_up != snu || sys_bs->sub[k].new_num_down != snd) continue;
        for (int x = 0; x < sys_bs->sub[k].num; x++) {
          const tj_basis_sub *m = BM(sys_bs, k, x);
          const int stu = m->st_num_up, std_ = m->st_num_down, nsu = m->bl_num_up, nsd = m->bl_num_down;
          for (int ned = abs(end - std_); ned <= end + std_; ned += 2) {
            const int neu = enu + stu;
            const int opos = m->spos, osub = m->sdim;
            const int sid = find_sub(&st, nsu, nsd, 0, 0);
            int bid = -1, bsub = -1;
            for (int y = 0; y < env_bs->num && bid < 0; y++) {
              if (env_bs->sub[y].new_num_up != neu || env_bs->sub[y].new_num_down != ned) continue;
              for (int z = 0; z < env_bs->sub[y].num; z++) {
                const tj_basis_sub *q = BM(env_bs, y, z);
                if (q->bl_num_up == enu && q->bl_num_down == end && q->st_num_up == stu && q->st_num_down == std_) {
                  bid = y;
                  bsub = z;
                  break;
                }
              }
            }
            const int wid = find_out(nw, nsu, nsd, neu, ned);
            if (sid < 0 || bid < 0 || wid < 0) continue;
            const int nsdim = nw->sub[wid].sys_dim;
            const int npos = BM(env_bs, bid, bsub)->spos, nsub = BM(env_bs, bid, bsub)->sdim;
            const int j12 = end, j3 = std_, j4 = nsd, j123 = ned, j34 = snd;
            double c1 = ipow_m1((j34 + j4 + j3) / 2) / sqrt((1.0 + j12) * (1.0 + j4));
            c1 *= sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j4 + j3 + j12) / 2) % 2 != 0) c1 = -c1;
            if (((j12 + j3 - j123) / 2) % 2 != 0) c1 = -c1;
            double *sub = mat_zero(nsdim, oed);
            dg('N', 'N', nsdim, oed, osub, c1, st.sub[sid].mat, nsdim, WP(old, i, opos, 0), LD(old, i), 0.0, sub,
               nsdim);
            dg('N', 'N', nsdim, nsub, oed, 1.0, sub, nsdim, et.sub[tid].mat, oed, 1.0, WP(nw, wid, 0, npos), LD(nw, wid));
            free(sub);
          }
        }
      }
    }
  }
  wave_norm_scale(nw);
  blk_free(&st);
  blk_free(&et);
  return 0;
}

/* ============================================ measurement operators */
static void put_block_result(const OBlk *b, tj_block_result *out) {
  out->num = b->num;
  int64_t n = 0;
  for (int i = 0; i < b->num; i++) n += (int64_t)b->sub[i].row_dim * b->sub[i].sdim;
  out->data_len = n;
  if (!out->subs || !out->data) return;
  int64_t off = 0;
  for (int i = 0; i < b->num; i++) {
    const OSub *s = &b->sub[i];
    const int64_t m = (int64_t)s->row_dim * s->sdim;
    out->subs[i] = (tj_block_sub){s->num_up, s->num_down, s->down_dif, s->row_dim, s->sdim, 0, off};
    memcpy(out->data + off, s->mat, (size_t)m * sizeof(double));
    off += m;
  }
  out->block = (tj_block){b->len, b->num, b->dim, b->up_dif, b->down_dif, 0, out->subs, out->data};
}
/* one enlargement of a block operator (update_block_dia / update_block_ndia_sys/env) */
static void enlarge_block(const OBlk *o, const tj_basis *bs, int side, int dia, char types, OBlk *out) {
  if (dia)
    upd_block_dia(o, bs, out);
  else
    upd_block_ndia(o, bs, out, side, types);
}
static void truncate_op(const OBlk *o, const OBlk *trun, int dia, OBlk *out) {
  if (dia)
    upd_trun_dia(o, trun, out);
  else
    upd_trun_ndia(o, trun, out);
}
static int chain_check(const tj_chain *ch, int idx) {
  if (!ch || idx < 1 || idx > ch->n || !ch->bsm || !ch->truns) return fail(TJ_ERR_ARG, "chain index out of range");
  return 0;
}
/* the loop shared by Get_*_oper_* and Change_*_oper_*: from a block operator
 * of length idx carried (enlarge, then truncate unless idx <= trun_idx) to
 * the enlarged basis of length idx_two, truncated there when truns */
static int carry(const tj_chain *ch, int side, int dia, char types, OBlk *op, int idx, int idx_two, int truns,
                 OBlk *res) {
  while (idx + 1 <= idx_two - 1) {
    if (chain_check(ch, idx + 1)) return TJ_ERR_ARG;
    OBlk mid;
    enlarge_block(op, &ch->bsm[idx], side, dia, types, &mid);
    blk_free(op);
    idx++;
    if (idx <= ch->trun_idx) {
      *op = mid;
    } else {
      OBlk t;
      blk_view(&ch->truns[idx - 1], &t);
      truncate_op(&mid, &t, dia, op);
      blk_free(&t);
      blk_free(&mid);
    }
  }
  if (chain_check(ch, idx + 1)) return TJ_ERR_ARG;
  enlarge_block(op, &ch->bsm[idx], side, dia, types, res);
  blk_free(op);
  if (truns) {
    OBlk t, r2;
    blk_view(&ch->truns[idx_two - 1], &t);
    truncate_op(res, &t, dia, &r2);
    blk_free(&t);
    blk_free(res);
    *res = r2;
  }
  return 0;
}
/* Get_sys_oper_dia / Get_env_oper_dia / Get_sys_oper_ndia / Get_env_oper_ndia
 * (get_sys.f90:764-891, 998-1130) */
int ora_get_oper(int side, int dia, const tj_chain *ch, const tj_block *st_oper, int old_idx, int new_idx,
                 int truns, char types, tj_block_result *out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  const int i1 = old_idx < new_idx ? old_idx : new_idx, i2 = old_idx < new_idx ? new_idx : old_idx;
  OBlk st, op, res;
  memset(&res, 0, sizeof res);
  blk_view(st_oper, &st);
  int rc = 0;
  if (i1 <= i2 - 1) {
    if (i1 <= 1) {
      blk_copy(&st, &op);
    } else {
      if ((rc = chain_check(ch, i1))) goto out;
      OBlk mid;
      if (dia) upd_site_dia(&st, &ch->bsm[i1 - 1], &mid);
      else upd_site_ndia(&st, &ch->bsm[i1 - 1], &mid, side, types);
      if (i1 <= ch->trun_idx) {
        op = mid;
      } else {
        OBlk t;
        blk_view(&ch->truns[i1 - 1], &t);
        truncate_op(&mid, &t, dia, &op);
        blk_free(&t);
        blk_free(&mid);
      }
    }
    rc = carry(ch, side, dia, types, &op, i1, i2, truns, &res);
    if (rc) goto out;
  } else {
    if (i1 <= 1) {
      blk_copy(&st, &res);
    } else {
      if ((rc = chain_check(ch, i2))) goto out;
      if (dia) upd_site_dia(&st, &ch->bsm[i2 - 1], &res);
      else upd_site_ndia(&st, &ch->bsm[i2 - 1], &res, side, types);
    }
    if (truns) {
      if ((rc = chain_check(ch, i2))) goto out;
      OBlk t, r2;
      blk_view(&ch->truns[i2 - 1], &t);
      truncate_op(&res, &t, dia, &r2);
      blk_free(&t);
      blk_free(&res);
      res = r2;
    }
  }
  put_block_result(&res, out);
out:
  blk_free(&res);
  blk_free(&st);
  return rc;
}
/* Change_sys_oper_dia / Change_env_oper_dia / Change_sys_oper_ndia /
 * Change_env_oper_ndia (get_sys.f90:893-996, 1134-1238) */
int ora_change_oper(int side, int dia, const tj_chain *ch, const tj_block *old_oper, int old_idx, int new_idx,
                    int truns, char types, tj_block_result *out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  const int i1 = old_idx < new_idx ? old_idx : new_idx, i2 = old_idx < new_idx ? new_idx : old_idx;
  OBlk in, op, res;
  memset(&res, 0, sizeof res);
  blk_view(old_oper, &in);
  int rc = 0;
  if (i1 <= i2 - 1) {
    blk_copy(&in, &op);
    rc = carry(ch, side, dia, types, &op, i1, i2, truns, &res);
    if (rc) goto out;
  } else {
    blk_copy(&in, &res);
  }
  put_block_result(&res, out);
out:
  blk_free(&res);
  blk_free(&in);
  return rc;
}
/* block_mul_block_ndia (block.f90:1956-2197) */
int ora_block_mul_block_ndia(const tj_block *o1b, char f1, const tj_block *o2b, char f2, double coef, int down_dif,
                             const tj_basis *bs, tj_block_result *out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk o1, o2;
  blk_view(o1b, &o1);
  blk_view(o2b, &o2);
  const int up1 = f1 == 'N' ? o1.up_dif : -o1.up_dif, up2 = f2 == 'N' ? o2.up_dif : -o2.up_dif;
  const int d2 = o2.down_dif;
  const int up_dif = up1 + up2;
  int num = 0;
  for (int i = 0; i < bs->num; i++) {
    int nu = bs->sub[i].new_num_up, nd = bs->sub[i].new_num_down;
    for (int nnd = abs(nd - down_dif); nnd <= nd + down_dif; nnd += 2)
      if (find_bs(bs, nu + up_dif, nnd) >= 0) num++;
  }
  OBlk nb;
  blk_new(&nb, bs->len, num, up_dif, down_dif);
  int id = 0;
  for (int i = 0; i < bs->num; i++) {
    const int nu = bs->sub[i].new_num_up, nd = bs->sub[i].new_num_down, nnu = nu + up_dif;
    for (int nnd = abs(nd - down_dif); nnd <= nd + down_dif; nnd += 2) {
      const int x = find_bs(bs, nnu, nnd);
      if (x < 0) continue;
      const int old_dim = bs->sub[i].dim, new_dim = bs->sub[x].dim;
      OSub *S = &nb.sub[id++];
      *S = (OSub){nu, nd, nnd - nd, new_dim, old_dim, mat_zero(new_dim, old_dim)};
      nb.dim += old_dim;
      for (int mnd = abs(nd - d2); mnd <= nd + d2; mnd += 2) {
        int m2u, m2d, dd22;
        if (f2 == 'N') {
          m2u = nu;
          m2d = nd;
          dd22 = mnd - nd;
        } else {
          m2u = nu + up2;
          m2d = mnd;
          dd22 = nd - mnd;
        }
        const int idx2 = find_sub(&o2, m2u, m2d, dd22, 1);
        int m1u, m1d, dd11;
        if (f1 == 'N') {
          m1u = nu + up2;
          m1d = mnd;
          dd11 = nnd - mnd;
        } else {
          m1u = nnu;
          m1d = nnd;
          dd11 = mnd - nnd;
        }
        const int idx1 = find_sub(&o1, m1u, m1d, dd11, 1);
        if (idx1 < 0 || idx2 < 0) continue;
        int mid_dim, lda, ldb;
        if (f1 == 'N') {
          mid_dim = o1.sub[idx1].sdim;
          lda = new_dim;
        } else {
          mid_dim = o1.sub[idx1].row_dim;
          lda = mid_dim;
        }
        ldb = f2 == 'N' ? mid_dim : old_dim;
        int j1 = nnd, j4 = -j1, j3 = nd, j6 = j3, j2 = nb.down_dif, j5 = -j4 - j6;   /* new_oper%down_dif */
        const int kq = j5;
        const double c11 = ora_w3js(j1, j2, j3, j4, j5, j6);
        if (c11 == 0.0) {
          blk_free(&nb);
          blk_free(&o1);
          blk_free(&o2);
          return fail(TJ_ERR_NUMERIC, "block_mul_block_ndia: vanishing 3j normalisation");
        }
        double c1 = 0.0;
        for (int jj6 = -mnd; jj6 <= mnd; jj6 += 2) {
          const int a1 = nnd, a4 = -a1, a2 = o1.down_dif, a3 = mnd, a5 = -a4 - jj6;
          double c12 = ora_w3js(a1, a2, a3, a4, a5, jj6);
          const int b1 = mnd, b4 = -jj6, b2 = o2.down_dif, b3 = nd, b6 = b3, b5 = -b4 - b6;
          c12 *= ora_w3js(b1, b2, b3, b4, b5, b6) * ipow_m1((b1 + b4) / 2);
          const int i1 = o1.down_dif, i2 = o2.down_dif, i3 = down_dif, i4 = a5, i5 = b5, i6 = -kq;
          c12 *= ora_w3js(i1, i2, i3, i4, i5, i6) * ipow_m1((-i1 + i2 + kq) / 2) * sqrt(i3 + 1.0);
          c1 += c12;
        }
        if (c1 == 0.0) continue;
        c1 = coef * c1 / c11;
        dg(f1, f2, new_dim, old_dim, mid_dim, c1, o1.sub[idx1].mat, lda, o2.sub[idx2].mat, ldb, 1.0, S->mat, new_dim);
      }
    }
  }
  put_block_result(&nb, out);
  blk_free(&nb);
  blk_free(&o1);
  blk_free(&o2);
  return 0;
}
/* update_trun_dia / update_trun_ndia (block.f90:1311-1503) on their own */
int ora_update_trun(int dia, const tj_block *ori, const tj_block *trunb, tj_block_result *out) {
  if (!p_dgemm) return fail(TJ_ERR_ARG, "oracle not initialised (ora_init)");
  OBlk o, t, r;
  blk_view(ori, &o);
  blk_view(trunb, &t);
  truncate_op(&o, &t, dia, &r);
  put_block_result(&r, out);
  blk_free(&r);
  blk_free(&o);
  blk_free(&t);
  return 0;
}
