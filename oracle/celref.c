/*
 * celref.c -- CPU oracle for the CEL solver hot path (TEST INFRASTRUCTURE).
 *
 * Restates, in C, the arithmetic of the Fortran reference
 * (hpcdkhab/cel_v3).  Only the test-suite, the smoke check and the CPU
 * baseline leg of the benchmark may load this library.  See celref.h for
 * the conventions; each function cites the reference lines it follows.
 * Build with -ffp-contract=off (oracle/Makefile does).
 */
#include "celref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* work split                                                                */
/* ------------------------------------------------------------------------ */

/* cel_omp_shared_work_distr, src/fbase/cel_omp_shared_work_module.f90:196-220.
 * The work is cut into blocks of AW_SMALLEST_OMP_TASK=4 elements
 * (src/fbase/cel_types_module.f90:84); every worker gets the same number of
 * whole blocks and the last worker also takes the remainder.  `worker` is
 * 1-based as in the reference; the result is the 0-based half-open range
 * [*start, *end). */
void celref_work_chunk(int len, int nworkers, int worker, int* start, int* end) {
  const int task = 4;
  int aligned = (len / task) * task;
  int delta_len = len - aligned;
  int nblocks = aligned / task;
  int bpt = nblocks / nworkers;
  int delta_blocks = nblocks - bpt * nworkers;
  int s1 = bpt * task * (worker - 1) + 1;           /* 1-based inclusive */
  int e1 = s1 + bpt * task - 1;
  e1 += (worker / nworkers) * (delta_len + delta_blocks * task);
  if (s1 < 0) s1 = 0;
  if (e1 < -1) e1 = -1;
  *start = s1 - 1;
  *end = e1;
  if (*end < *start) *end = *start;
}

/* ------------------------------------------------------------------------ */
/* block-tree reduction (the CUDA kernels' fixed order)                      */
/* ------------------------------------------------------------------------ */

/* 256 lane sums -> one value: a butterfly inside each 32-lane warp
 * (partner lane l^16, l^8, l^4, l^2, l^1), then the eight warp sums added
 * in warp order starting from warp 0. */
static double fold256(double* s) {
  for (int w = 0; w < 8; w++) {
    double* q = s + 32 * w;
    for (int off = 16; off >= 1; off >>= 1) {
      double t[32];
      for (int l = 0; l < 32; l++) t[l] = q[l] + q[l ^ off];
      memcpy(q, t, sizeof(t));
    }
  }
  double tot = s[0];
  for (int w = 1; w < 8; w++) tot = tot + s[32 * w];
  return tot;
}

/* lane j sums vals[j], vals[j+256], ... from 0.0, then fold256 */
double celref_reduce256(const double* vals, long cnt) {
  double s[CELREF_LANES];
  for (int j = 0; j < CELREF_LANES; j++) {
    double acc = 0.0;
    for (long k = j; k < cnt; k += CELREF_LANES) acc = acc + vals[k];
    s[j] = acc;
  }
  return fold256(s);
}

static double tile_dot(const double* a, const double* b, long base, long cnt) {
  double s[CELREF_LANES];
  for (int j = 0; j < CELREF_LANES; j++) {
    double acc = 0.0;
    for (long k = j; k < cnt; k += CELREF_LANES) acc = acc + a[base + k] * b[base + k];
    s[j] = acc;
  }
  return fold256(s);
}

static double tile_dot_f32(const float* a, const float* b, long base, long cnt) {
  double s[CELREF_LANES];
  for (int j = 0; j < CELREF_LANES; j++) {
    double acc = 0.0;
    for (long k = j; k < cnt; k += CELREF_LANES)
      acc = acc + (double)a[base + k] * (double)b[base + k];
    s[j] = acc;
  }
  return fold256(s);
}

static double tile_dot_perm(const double* a, const double* b, const int* perm, long base,
                            long cnt) {
  double s[CELREF_LANES];
  for (int j = 0; j < CELREF_LANES; j++) {
    double acc = 0.0;
    for (long k = j; k < cnt; k += CELREF_LANES) {
      int r = perm[base + k];
      acc = acc + a[r] * b[r];
    }
    s[j] = acc;
  }
  return fold256(s);
}

static long ntiles_of(long n) { return (n + CELREF_TILE - 1) / CELREF_TILE; }

static double dot_tree(int n, const double* a, const double* b) {
  long nt = ntiles_of(n);
  double* part = (double*)malloc(sizeof(double) * (nt > 0 ? nt : 1));
  for (long t = 0; t < nt; t++) {
    long base = t * CELREF_TILE;
    long cnt = n - base < CELREF_TILE ? n - base : CELREF_TILE;
    part[t] = tile_dot(a, b, base, cnt);
  }
  double r = celref_reduce256(part, nt);
  free(part);
  return r;
}

double celref_dot_tree_perm(int n, const double* a, const double* b, const int* perm) {
  long nt = ntiles_of(n);
  double* part = (double*)malloc(sizeof(double) * (nt > 0 ? nt : 1));
  for (long t = 0; t < nt; t++) {
    long base = t * CELREF_TILE;
    long cnt = n - base < CELREF_TILE ? n - base : CELREF_TILE;
    part[t] = tile_dot_perm(a, b, perm, base, cnt);
  }
  double r = celref_reduce256(part, nt);
  free(part);
  return r;
}

/* ------------------------------------------------------------------------ */
/* worker team: the reference's thread model                                 */
/* ------------------------------------------------------------------------ */

/* Thread 0 is the MPI "master" and does no vector work; workers 1..W take
 * chunks from celref_work_chunk (src/fbase/cel_omp_module.f90:71-84).
 * Without OpenMP (or W == 1 in sequential mode) one thread plays both. */
typedef struct {
  int par;
  int W;
  int tid;
  double* part;   /* shared partial sums: max(W, tiles) */
  double* slot;   /* shared reduction result */
} team_t;

static int t_worker(const team_t* t) { return !t->par || t->tid >= 1; }
static int t_wnum(const team_t* t) { return t->par ? t->tid : 1; }
static int t_master(const team_t* t) { return !t->par || t->tid == 0; }
static void t_bar(const team_t* t) {
  (void)t;
#ifdef _OPENMP
  if (t->par) {
#pragma omp barrier
  }
#endif
}
static void t_chunk(const team_t* t, int len, int* s, int* e) {
  celref_work_chunk(len, t->W, t_wnum(t), s, e);
}

/* dot with the chosen order; every thread returns the same value.
 * Reference partial/atomic/allreduce sequence:
 * src/fop/cel_fop_vec_distr_module.f90:752-766 (dot), :460-474 (norm). */
static double t_dot(team_t* t, int n, const double* a, const double* b, int red) {
  if (red == CELREF_RED_SEQ) {
    if (t_worker(t)) {
      int s, e;
      t_chunk(t, n, &s, &e);
      double acc = 0.0;
      for (int i = s; i < e; i++) acc = acc + a[i] * b[i];
      t->part[t_wnum(t) - 1] = acc;
    }
    t_bar(t);
    if (t_master(t)) {
      double tot = 0.0;
      for (int w = 0; w < t->W; w++) tot = tot + t->part[w];
      *t->slot = tot;
    }
  } else {
    long nt = ntiles_of(n);
    if (t_worker(t)) {
      int s, e;
      t_chunk(t, (int)nt, &s, &e);
      for (int tt = s; tt < e; tt++) {
        long base = (long)tt * CELREF_TILE;
        long cnt = n - base < CELREF_TILE ? n - base : CELREF_TILE;
        t->part[tt] = tile_dot(a, b, base, cnt);
      }
    }
    t_bar(t);
    if (t_master(t)) *t->slot = celref_reduce256(t->part, nt);
  }
  t_bar(t);
  return *t->slot;
}

static double t_dot_perm(team_t* t, int n, const double* a, const double* b, const int* perm) {
  long nt = ntiles_of(n);
  if (t_worker(t)) {
    int s, e;
    t_chunk(t, (int)nt, &s, &e);
    for (int tt = s; tt < e; tt++) {
      long base = (long)tt * CELREF_TILE;
      long cnt = n - base < CELREF_TILE ? n - base : CELREF_TILE;
      t->part[tt] = tile_dot_perm(a, b, perm, base, cnt);
    }
  }
  t_bar(t);
  if (t_master(t)) *t->slot = celref_reduce256(t->part, nt);
  t_bar(t);
  return *t->slot;
}

static size_t part_len(int n, int W) {
  long nt = ntiles_of(n);
  long m = nt > W ? nt : W;
  return (size_t)(m > 0 ? m : 1);
}

/* ------------------------------------------------------------------------ */
/* SpMV                                                                      */
/* ------------------------------------------------------------------------ */

/* One CSR row: src/fop/cel_fop_mv_module.f90:215-229.  The row sum starts
 * at 0.0 and accumulates value*x left to right; the result is added to y. */
static inline double csr_row(const int* rp, const int* ci, const double* v, const double* x,
                             int i) {
  double t = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; k++) t = t + v[k] * x[ci[k]];
  return t;
}

static void t_spmv_csr(team_t* t, int n, const int* rp, const int* ci, const double* v,
                       const double* x, double* y, int accumulate) {
  if (t_worker(t)) {
    int s, e;
    t_chunk(t, n, &s, &e);
    for (int i = s; i < e; i++) {
      double tt = csr_row(rp, ci, v, x, i);
      y[i] = (accumulate ? y[i] : 0.0) + tt;
    }
  }
  t_bar(t);
}

/* JAD SpMV, src/fop/cel_fop_mv_module.f90:267-326: tmp(i) accumulates the
 * jagged diagonals in order 1..mmax, then y(perm(i)) = tmp(i) (overwrite).
 * Phase 2 of the reference splits diagonals across workers and races on
 * tmp; this restatement keeps the one-worker order (diagonal order per
 * row) and parallelises over permuted rows instead. */
static inline double jad_row(int mmax, const int* jb, const int* jci, const double* jv,
                             const double* x, int i) {
  double t = 0.0;
  for (int k = 0; k < mmax; k++) {
    int len = jb[k + 1] - jb[k];
    if (i >= len) break;
    int q = jb[k] + i;
    t = t + jv[q] * x[jci[q]];
  }
  return t;
}

static void t_spmv_jad(team_t* t, int n, int mmax, const int* jb, const int* jci,
                       const double* jv, const int* perm, const double* x, double* y) {
  if (t_worker(t)) {
    int s, e;
    t_chunk(t, n, &s, &e);
    for (int i = s; i < e; i++) y[perm[i]] = jad_row(mmax, jb, jci, jv, x, i);
  }
  t_bar(t);
}

/* y = 0 + A x for the CSR path ("to_zero" then "y = y + A x"), overwrite
 * for JAD: both paths give 0.0 + row sum. */
static void t_spmv(team_t* t, const celref_mat* A, const double* x, double* y) {
  if (A->fmt == CELREF_FMT_JAD)
    t_spmv_jad(t, A->n, A->mmax, A->jbegin, A->jci, A->jv, A->perm, x, y);
  else
    t_spmv_csr(t, A->n, A->rp, A->ci, A->v, x, y, 0);
}

void celref_spmv_csr(int n, const int* rp, const int* ci, const double* v, const double* x,
                     double* y, int accumulate, int nworkers) {
  int W = nworkers < 1 ? 1 : nworkers;
  if (W == 1) {
    for (int i = 0; i < n; i++) y[i] = (accumulate ? y[i] : 0.0) + csr_row(rp, ci, v, x, i);
    return;
  }
#pragma omp parallel num_threads(W + 1)
  {
    team_t t = {1, W, 0, NULL, NULL};
#ifdef _OPENMP
    t.tid = omp_get_thread_num();
#endif
    t_spmv_csr(&t, n, rp, ci, v, x, y, accumulate);
  }
}

void celref_spmv_csr_f32(int n, const int* rp, const int* ci, const float* v, const float* x,
                         float* y, int accumulate) {
  for (int i = 0; i < n; i++) {
    float t = 0.0f;
    for (int k = rp[i]; k < rp[i + 1]; k++) t = t + v[k] * x[ci[k]];
    y[i] = (accumulate ? y[i] : 0.0f) + t;
  }
}

void celref_spmv_jad(int n, int mmax, const int* jb, const int* jci, const double* jv,
                     const int* perm, const double* x, double* y) {
  for (int i = 0; i < n; i++) y[perm[i]] = jad_row(mmax, jb, jci, jv, x, i);
}

void celref_spmv(const celref_mat* A, const double* x, double* y, int nworkers) {
  if (A->fmt == CELREF_FMT_JAD)
    celref_spmv_jad(A->n, A->mmax, A->jbegin, A->jci, A->jv, A->perm, x, y);
  else
    celref_spmv_csr(A->n, A->rp, A->ci, A->v, x, y, 0, nworkers);
}

/* ------------------------------------------------------------------------ */
/* JAD conversion                                                            */
/* ------------------------------------------------------------------------ */

/* Row lengths and the stable counting sort of cel_sp_mat_jad_dcsort
 * (src/fspmtconverter/cel_sp_mat_jad_converter_module.f90:57-88) as driven by
 * cel_sp_mat_jad_from_sp_mat_local (:118-135): ilo starts at nrow, idiag at
 * 0; counts over [ilo, idiag], suffix sums from idiag-1 down to ilo, then
 * rows scattered from the last to the first.  The result orders rows by
 * descending length, ties by ascending row index.  perm[k] = original row at
 * permuted position k (0-based). */
int celref_jad_perm(int n, const int* rp, int* perm, int* mmax) {
  int lo = n, hi = 0;
  for (int i = 0; i < n; i++) {
    int len = rp[i + 1] - rp[i];
    if (len < lo) lo = len;
    if (len > hi) hi = len;
  }
  *mmax = hi;
  if (n == 0) return 0;
  int span = hi - lo + 1;
  int* icnt = (int*)calloc((size_t)span, sizeof(int));
  if (!icnt) return CELREF_ERR_ARG;
  for (int i = 0; i < n; i++) icnt[(rp[i + 1] - rp[i]) - lo]++;
  for (int L = hi - 1; L >= lo; L--) icnt[L - lo] += icnt[L + 1 - lo];
  for (int j = n - 1; j >= 0; j--) {
    int L = rp[j + 1] - rp[j];
    perm[icnt[L - lo] - 1] = j;
    icnt[L - lo]--;
  }
  free(icnt);
  return 0;
}

/* The counts the reference leaves in jad_begin(1 .. idiag-ilo+1) after the
 * sort: icnt(L) = count(len > L), stored from ilo on
 * (src/fspmtconverter/cel_sp_mat_jad_converter_module.f90:134-149).  Used only
 * to document that the reference's per-diagonal counts are wrong. */
void celref_jad_begin_literal(int n, const int* rp, int* icnt_out, int* lo_out, int* hi_out) {
  int lo = n, hi = 0;
  for (int i = 0; i < n; i++) {
    int len = rp[i + 1] - rp[i];
    if (len < lo) lo = len;
    if (len > hi) hi = len;
  }
  *lo_out = lo;
  *hi_out = hi;
  for (int L = lo; L <= hi; L++) {
    int c = 0;
    for (int i = 0; i < n; i++)
      if (rp[i + 1] - rp[i] > L) c++;
    icnt_out[L - lo] = c;
  }
}

/* Full JAD: the reference's permutation, then jagged diagonal k (0-based)
 * holds the (k+1)-th entry of the first count(len > k) permuted rows (Saad's
 * definition, which the reference intends at :145-159 but computes with
 * wrong counts).  jbegin has mmax+1 entries. */
int celref_jad_build(int n, const int* rp, const int* ci, const double* v, int* perm,
                     int* jbegin, int* jci, double* jv, int* mmax) {
  int err = celref_jad_perm(n, rp, perm, mmax);
  if (err) return err;
  int q = 0;
  jbegin[0] = 0;
  for (int k = 0; k < *mmax; k++) {
    for (int i = 0; i < n; i++) {
      int r = perm[i];
      if (rp[r + 1] - rp[r] <= k) break; /* rows are sorted by length */
      jv[q] = v[rp[r] + k];
      jci[q] = ci[rp[r] + k];
      q++;
    }
    jbegin[k + 1] = q;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* set-up                                                                    */
/* ------------------------------------------------------------------------ */

/* Diagonal extraction, src/fspmtdistr/cel_sp_mat_distr_module.f90:197-207:
 * every stored entry with col == row is written to diagonal(row), so the
 * last one wins.  Rows without a stored diagonal keep 0.0. */
void celref_diag(int n, const int* rp, const int* ci, const double* v, double* d) {
  for (int i = 0; i < n; i++) {
    d[i] = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; k++)
      if (ci[k] == i) d[i] = v[k];
  }
}

/* cel_sp_mat_distr_set_jacobi, src/fspmtdistr/cel_sp_mat_distr_format_module.f90:181-189:
 * jacobi = 1/d, or scaled_diagonal/d when the matrix was row-scaled. */
void celref_jacobi(int n, const double* d, const double* s, double* J) {
  for (int i = 0; i < n; i++) J[i] = s ? s[i] / d[i] : 1.0 / d[i];
}

/* Block-Jacobi set-up: the intended form of cel_prec_build_diagonal and
 * cel_prec_build_diagonal_inv (src/fspmtdistr/cel_prec_module.f90:27-339;
 * dead code in the reference, whose block indexing is out of range for
 * every block after the first).  Rows are cut into blocks of bs from row 0,
 * the last one possibly shorter.
 *  - extraction (:96-130): a row's entries are scanned in stored order; an
 *    entry left of the block is skipped, one inside is written to the dense
 *    block (the last one wins), the first one right of it ends the row;
 *  - inverse (:256-339, cel_prec_inverse_matrix_serial1_nxn): Doolittle LU
 *    without pivoting, then for every unit vector e_k the forward solve
 *    L d = e_k and the back solve U x = d give column k of the inverse; a
 *    1x1 block is 1/a.
 * inv is n x bs, row-major: inv[i*bs + j] = (D_b^-1)(i - b0, j), zero-padded
 * for the last block.  Returns 0, or 1 when an entry of an inverse is not
 * finite (a zero pivot). */
int celref_block_jacobi_inv(int n, const int* rp, const int* ci, const double* v, int bs,
                            double* inv) {
  int bad = 0;
  double* a = (double*)calloc((size_t)bs * bs, sizeof(double));
  double* L = (double*)calloc((size_t)bs * bs, sizeof(double));
  double* c = (double*)calloc((size_t)bs * bs, sizeof(double));
  double* d = (double*)calloc((size_t)bs, sizeof(double));
  double* x = (double*)calloc((size_t)bs, sizeof(double));
  double* b = (double*)calloc((size_t)bs, sizeof(double));
  for (int b0 = 0; b0 < n; b0 += bs) {
    const int nb = (n - b0 < bs) ? n - b0 : bs;
    for (int q = 0; q < bs * bs; q++) a[q] = L[q] = c[q] = 0.0;
    for (int i = 0; i < nb; i++) {
      const int row = b0 + i;
      for (int k = rp[row]; k < rp[row + 1]; k++) {
        const int col = ci[k];
        if (col < b0) continue;
        if (col >= b0 + nb) break;
        a[i * bs + (col - b0)] = v[k];
      }
    }
    if (nb == 1) {
      c[0] = 1.0 / a[0];
    } else {
      for (int k = 0; k < nb - 1; k++)
        for (int i = k + 1; i < nb; i++) {
          const double coeff = a[i * bs + k] / a[k * bs + k];
          L[i * bs + k] = coeff;
          for (int j = k + 1; j < nb; j++) a[i * bs + j] = a[i * bs + j] - coeff * a[k * bs + j];
        }
      for (int k = 0; k < nb; k++) {
        for (int i = 0; i < nb; i++) b[i] = 0.0;
        b[k] = 1.0;
        d[0] = b[0];
        for (int i = 1; i < nb; i++) {
          d[i] = b[i];
          for (int j = 0; j < i; j++) d[i] = d[i] - L[i * bs + j] * d[j];
        }
        x[nb - 1] = d[nb - 1] / a[(nb - 1) * bs + (nb - 1)];
        for (int i = nb - 2; i >= 0; i--) {
          x[i] = d[i];
          for (int j = nb - 1; j > i; j--) x[i] = x[i] - a[i * bs + j] * x[j];
          x[i] = x[i] / a[i * bs + i];
        }
        for (int i = 0; i < nb; i++) c[i * bs + k] = x[i];
      }
    }
    for (int i = 0; i < nb; i++)
      for (int j = 0; j < bs; j++) {
        const double e = j < nb ? c[i * bs + j] : 0.0;
        if (!isfinite(e)) bad = 1;
        inv[(size_t)(b0 + i) * bs + j] = e;
      }
  }
  free(a); free(L); free(c); free(d); free(x); free(b);
  return bad;
}

/* z = blockdiag(D_b^-1) r (cel_fop_vec_mult_distr_jacobi_block,
 * src/fop/cel_fop_block_jacobi_module.f90:96-190, in its intended form: the
 * reference's n x n case multiplies by r(i) where r(j) is meant):
 * z_i = r_b0 inv_i0 + r_b0+1 inv_i1 + ... left to right over the block. */
void celref_block_jacobi_apply(int n, int bs, const double* inv, const double* r, double* z) {
  for (int i = 0; i < n; i++) {
    const int b0 = i - i % bs;
    const int nb = (n - b0 < bs) ? n - b0 : bs;
    const double* row = inv + (size_t)i * bs;
    double s = r[b0] * row[0];
    for (int j = 1; j < nb; j++) s = s + r[b0 + j] * row[j];
    z[i] = s;
  }
}

/* Diagonal row scaling, src/fspmtdistr/cel_sp_mat_distr_format_module.f90:120-121
 * (s = sqrt|d|) and :298-303 (row i divided by s_i).  d stays unscaled. */
void celref_row_scale(int n, const int* rp, double* v, const double* d, double* s) {
  for (int i = 0; i < n; i++) {
    s[i] = sqrt(fabs(d[i]));
    for (int k = rp[i]; k < rp[i + 1]; k++) v[k] = v[k] / s[i];
  }
}

double celref_dot(int n, const double* a, const double* b, int red, int nworkers) {
  int W = nworkers < 1 ? 1 : nworkers;
  if (red == CELREF_RED_TREE) return dot_tree(n, a, b);
  double tot = 0.0;
  for (int w = 1; w <= W; w++) {
    int s, e;
    celref_work_chunk(n, W, w, &s, &e);
    double acc = 0.0;
    for (int i = s; i < e; i++) acc = acc + a[i] * b[i];
    tot = tot + acc;
  }
  return tot;
}

double celref_dot_f32(int n, const float* a, const float* b, int red) {
  if (red == CELREF_RED_TREE) {
    long nt = ntiles_of(n);
    double* part = (double*)malloc(sizeof(double) * (nt > 0 ? nt : 1));
    for (long t = 0; t < nt; t++) {
      long base = t * CELREF_TILE;
      long cnt = n - base < CELREF_TILE ? n - base : CELREF_TILE;
      part[t] = tile_dot_f32(a, b, base, cnt);
    }
    double r = celref_reduce256(part, nt);
    free(part);
    return r;
  }
  double acc = 0.0;
  for (int i = 0; i < n; i++) acc = acc + (double)a[i] * (double)b[i];
  return acc;
}

/* ------------------------------------------------------------------------ */
/* Jacobi-PCG: cel_cgalg_jacobi, src/fcgalg/cel_cgalg_module.f90:178-305      */
/* ------------------------------------------------------------------------ */

typedef struct {
  const celref_mat* A;
  const double* J;
  const double* b;
  double* x;
  const celref_params* p;
  double* hist;
  double *r, *z, *pv, *v;
  double alpha, sigma, norm, bnorm, eps, rz, pvd;
  int ii, err, stop;
} pcg_ctx;

static void pcg_body(team_t* t, pcg_ctx* c) {
  const celref_mat* A = c->A;
  const celref_params* P = c->p;
  int n = A->n;
  int s = 0, e = 0;
  if (t_worker(t)) t_chunk(t, n, &s, &e);

  /* x0 (:209 sets x=1) */
  if (t_worker(t)) {
    if (P->x0_mode == CELREF_X0_ONES)
      for (int i = s; i < e; i++) c->x[i] = 1.0;
    else if (P->x0_mode == CELREF_X0_ZERO)
      for (int i = s; i < e; i++) c->x[i] = 0.0;
  }
  t_bar(t);
  double bb = t_dot(t, n, c->b, c->b, P->red);
  if (t_master(t)) {
    c->bnorm = sqrt(bb);
    c->eps = P->eps_abs;
    if (P->eps_rel > 0.0 && P->eps_rel * c->bnorm > c->eps) c->eps = P->eps_rel * c->bnorm;
  }
  /* r = 0; r = r + A x; r = b - r   (:207-218) */
  t_spmv(t, A, c->x, c->r);
  if (t_worker(t))
    for (int i = s; i < e; i++) c->r[i] = c->b[i] - c->r[i];
  t_bar(t);
  /* p = J r   (:220, src/fop/cel_fop_vec_distr_module.f90:364-366) */
  if (t_worker(t))
    for (int i = s; i < e; i++) c->pv[i] = c->r[i] * c->J[i];
  t_bar(t);
  /* alpha = r.p (:230); norm = ||r|| (:234) */
  double a0 = t_dot(t, n, c->r, c->pv, P->red);
  double rr = t_dot(t, n, c->r, c->r, P->red);
  if (t_master(t)) {
    c->alpha = a0;
    c->norm = sqrt(rr);
    if (c->hist) c->hist[0] = c->norm;
    c->ii = 0;
    c->err = 0;
  }
  t_bar(t);
  /* loop condition :247-249 */
  while (c->ii < P->iter_max && fabs(c->alpha) > CELREF_REAL_SMALL && c->norm > c->eps) {
    /* v = 0; v = v + A p (:251-256) */
    t_spmv(t, A, c->pv, c->v);
    double pvd;
    if (A->fmt == CELREF_FMT_JAD && P->red == CELREF_RED_TREE)
      pvd = t_dot_perm(t, n, c->v, c->pv, A->perm);
    else
      pvd = t_dot(t, n, c->v, c->pv, P->red);
    /* sigma = alpha/(v.p)  (:259, src/fop/cel_fop_vec_distr_module.f90:711) */
    if (t_master(t)) {
      c->ii++;
      c->pvd = pvd;
      c->sigma = c->alpha / pvd;
      c->stop = !isfinite(c->sigma);
      if (c->stop) c->err = CELREF_ERR_BREAKDOWN;
    }
    t_bar(t);
    if (c->stop) break;
    double sg = c->sigma;
    /* x = x + sigma p; r = r + (-sigma) v (:263-269, :862-864) */
    if (t_worker(t)) {
      double ms = -sg;
      for (int i = s; i < e; i++) {
        c->x[i] = c->x[i] + sg * c->pv[i];
        c->r[i] = c->r[i] + ms * c->v[i];
      }
    }
    t_bar(t);
    /* z = J r (:271) */
    if (t_worker(t))
      for (int i = s; i < e; i++) c->z[i] = c->r[i] * c->J[i];
    t_bar(t);
    /* sigma = (r.z)/alpha; alpha = r.z (:277, :821-822) */
    double rz = t_dot(t, n, c->r, c->z, P->red);
    if (t_master(t)) {
      c->rz = rz;
      c->sigma = rz / c->alpha;
      c->alpha = rz;
    }
    t_bar(t);
    /* p = sigma p + z (:282, :944-946) */
    double bt = c->sigma;
    if (t_worker(t))
      for (int i = s; i < e; i++) c->pv[i] = bt * c->pv[i] + c->z[i];
    t_bar(t);
    /* norm = ||r|| (:287) */
    double rr2 = t_dot(t, n, c->r, c->r, P->red);
    if (t_master(t)) {
      c->norm = sqrt(rr2);
      if (c->hist) c->hist[c->ii] = c->norm;
    }
    t_bar(t);
  }
}

static int run_team(int W, void (*body)(team_t*, void*), void* ctx, size_t plen) {
  double* part = (double*)malloc(sizeof(double) * plen);
  double slot = 0.0;
  if (!part) return CELREF_ERR_ARG;
  if (W <= 1) {
    team_t t = {0, 1, 1, part, &slot};
    body(&t, ctx);
  } else {
#pragma omp parallel num_threads(W + 1)
    {
      team_t t = {1, W, 0, part, &slot};
#ifdef _OPENMP
      t.tid = omp_get_thread_num();
#endif
      body(&t, ctx);
    }
  }
  free(part);
  return 0;
}

static void pcg_body_v(team_t* t, void* c) { pcg_body(t, (pcg_ctx*)c); }

int celref_pcg_jacobi(const celref_mat* A, const double* J, const double* b, double* x,
                      const celref_params* p, double* hist, celref_result* res) {
  int n = A->n;
  int W = p->nworkers < 1 ? 1 : p->nworkers;
  pcg_ctx c;
  memset(&c, 0, sizeof(c));
  c.A = A;
  c.J = J;
  c.b = b;
  c.x = x;
  c.p = p;
  c.hist = hist;
  size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
  c.r = (double*)malloc(nb);
  c.z = (double*)malloc(nb);
  c.pv = (double*)malloc(nb);
  c.v = (double*)malloc(nb);
  if (!c.r || !c.z || !c.pv || !c.v) return CELREF_ERR_ARG;
  run_team(W, pcg_body_v, &c, part_len(n, W));
  res->iter_done = c.ii;
  res->final_norm = c.norm;
  res->bnorm = c.bnorm;
  res->eps_used = c.eps;
  res->err = c.err;
  if (!res->err && c.norm > c.eps && c.ii >= p->iter_max) res->err = CELREF_ERR_NOCONV;
  res->arnoldi_steps = 0;
  free(c.r);
  free(c.z);
  free(c.pv);
  free(c.v);
  return res->err;
}

/* ------------------------------------------------------------------------ */
/* CG without preconditioner: cel_cgalg, src/fcgalg/cel_cgalg_module.f90:34-175 */
/* ------------------------------------------------------------------------ */

/* literal != 0 reproduces the reference exactly: the direction update uses
 * alpha (d = alpha d + r, :151) and the loop runs while
 * sigma_new > sigma_old*eps^2 (:106-108), sigma_old being the previous
 * iteration's sigma_new.  literal == 0 uses beta = sigma_new/sigma_old and
 * stops on ||r||_2 <= eps like the PCG. */
int celref_cg(const celref_mat* A, const double* b, double* x, const celref_params* p,
              double* hist, celref_result* res) {
  int n = A->n;
  double *r = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  double *d = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  double *q = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  double* part = (double*)malloc(sizeof(double) * part_len(n, 1));
  double slot;
  team_t t = {0, 1, 1, part, &slot};
  int red = p->red;
  if (p->x0_mode == CELREF_X0_ONES)
    for (int i = 0; i < n; i++) x[i] = 1.0;
  else if (p->x0_mode == CELREF_X0_ZERO)
    for (int i = 0; i < n; i++) x[i] = 0.0;
  double bnorm = sqrt(t_dot(&t, n, b, b, red));
  double eps = p->eps_abs;
  if (p->eps_rel > 0.0 && p->eps_rel * bnorm > eps) eps = p->eps_rel * bnorm;
  /* r = 0; r = r + A x (:62-69); norm2 = ||A x|| before r = b - r (:77) */
  t_spmv(&t, A, x, r);
  double norm = sqrt(t_dot(&t, n, r, r, red));
  /* r = b - r; d = r (:82, src/fop/cel_fop_vec_distr_module.f90:54-56) */
  for (int i = 0; i < n; i++) {
    r[i] = b[i] - r[i];
    d[i] = r[i];
  }
  /* sigma_new = sigma_old = r.r; alpha = 1 (:89, :590-596) */
  double sigma_new = t_dot(&t, n, r, r, red);
  double sigma_old = sigma_new, alpha = 1.0;
  if (!p->literal) norm = sqrt(sigma_new);
  if (hist) hist[0] = norm;
  int ii = 0, err = 0;
  for (;;) {
    int go;
    if (p->literal)
      go = ii < p->iter_max && sigma_new > sigma_old * p->eps_abs * p->eps_abs &&
           fabs(sigma_new) > CELREF_REAL_SMALL;
    else
      go = ii < p->iter_max && norm > eps && fabs(sigma_new) > CELREF_REAL_SMALL;
    if (!go) break;
    /* q = 0; q = q + A d (:111-116) */
    t_spmv(&t, A, d, q);
    ii++;
    /* alpha = sigma_new/(d.q) (:119, :697, :711) */
    double dq = t_dot(&t, n, d, q, red);
    alpha = sigma_new / dq;
    if (!isfinite(alpha)) {
      err = CELREF_ERR_BREAKDOWN;
      break;
    }
    /* x = x + alpha d; r = r + (-alpha) q (:123-131) */
    for (int i = 0; i < n; i++) {
      x[i] = x[i] + alpha * d[i];
      r[i] = r[i] + (-alpha) * q[i];
    }
    /* sigma_old = sigma_new; sigma_new = r.r (:146, :628-651) */
    sigma_old = sigma_new;
    sigma_new = t_dot(&t, n, r, r, red);
    /* d = beta d + r, beta = alpha in the reference (:151) */
    double beta = p->literal ? alpha : sigma_new / sigma_old;
    for (int i = 0; i < n; i++) d[i] = beta * d[i] + r[i];
    norm = sqrt(t_dot(&t, n, r, r, red));
    if (hist) hist[ii] = norm;
  }
  res->iter_done = ii;
  res->final_norm = norm;
  res->bnorm = bnorm;
  res->eps_used = eps;
  res->err = err;
  if (!p->literal && !err && norm > eps && ii >= p->iter_max) res->err = CELREF_ERR_NOCONV;
  res->arnoldi_steps = 0;
  free(r);
  free(d);
  free(q);
  free(part);
  return res->err;
}

/* ------------------------------------------------------------------------ */
/* GMRES(m) with right Jacobi: cel_gmresalg_2jacobi,                          */
/* src/fcgalg/cel_gmresalg_module.f90:570-851                                 */
/* ------------------------------------------------------------------------ */

/* Restated line by line with one correction: the reference's Givens update
 * of column j (:722-727) writes both results to hh(ii,jj) and never rotates
 * hh(ii+1,jj); here hh(ii+1,jj) receives -hh(ii,jj)*s + hh(ii+1,jj)*c with the
 * un-rotated hh(ii,jj).  When p->literal is set the reference's two lines are
 * kept as written.  Arrays are 0-based: V[0..m], Z[0..m-1], W[0..m-1]. */
int celref_gmres_jacobi(const celref_mat* A, const double* J, const double* b, double* x,
                        const celref_params* p, double* hist, celref_result* res) {
  int n = A->n;
  int m = p->restart;
  if (m <= 0) return CELREF_ERR_ARG;
  int red = p->red;
  size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
  double* r = (double*)malloc(nb);
  double** V = (double**)malloc(sizeof(double*) * (size_t)(m + 1));
  double** Z = (double**)malloc(sizeof(double*) * (size_t)m);
  double** Wv = (double**)malloc(sizeof(double*) * (size_t)m);
  for (int j = 0; j <= m; j++) V[j] = (double*)malloc(nb);
  for (int j = 0; j < m; j++) {
    Z[j] = (double*)malloc(nb);
    Wv[j] = (double*)malloc(nb);
  }
  /* hh(i,j), i=0..m, j=0..m-1 column-major (m+1) x m */
  double* hh = (double*)calloc((size_t)(m + 1) * (size_t)m, sizeof(double));
  double* cc = (double*)calloc((size_t)m + 1, sizeof(double));
  double* ss = (double*)calloc((size_t)m + 1, sizeof(double));
  double* gam = (double*)calloc((size_t)m + 2, sizeof(double));
  double* al = (double*)calloc((size_t)m + 1, sizeof(double));
  double* part = (double*)malloc(sizeof(double) * part_len(n, 1));
  double slot;
  team_t t = {0, 1, 1, part, &slot};
#define H(i, j) hh[(size_t)(j) * (size_t)(m + 1) + (size_t)(i)]

  double bnorm = sqrt(t_dot(&t, n, b, b, red));
  double eps = p->eps_abs;
  if (p->eps_rel > 0.0 && p->eps_rel * bnorm > eps) eps = p->eps_rel * bnorm;
  long hpos = 0;

  /* x = 1 (:638) */
  if (p->x0_mode == CELREF_X0_ONES)
    for (int i = 0; i < n; i++) x[i] = 1.0;
  else if (p->x0_mode == CELREF_X0_ZERO)
    for (int i = 0; i < n; i++) x[i] = 0.0;
  int converged = 0; /* GMRES_REASON_XN reached */
  int iter = 0, steps = 0;
  double resnorm = 0.0;
  while (iter <= p->iter_max && !converged) {
    iter++;
    /* r = 0; r = r + A x; r = b - r; ||r|| (:643-663) */
    t_spmv(&t, A, x, r);
    for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
    resnorm = sqrt(t_dot(&t, n, r, r, red));
    if (hist && hpos == 0) hist[hpos++] = resnorm;
    double local_res = resnorm;
    int restart = 0;
    while (restart <= m && !converged) {
      /* v1 = r * (1/||r||)  (:669, src/fop/cel_fop_vec_distr_module.f90:94-97) */
      double inv = 1.0 / local_res;
      for (int i = 0; i < n; i++) V[0][i] = r[i] * inv;
      gam[0] = resnorm;
      int jdone = m;
      for (int j = 0; j < m; j++) {
        /* w = 0; z_j = J v_j; w = w + A z_j (:680-697) */
        for (int i = 0; i < n; i++) Z[j][i] = V[j][i] * J[i];
        t_spmv(&t, A, Z[j], Wv[j]);
        steps++;
        /* modified Gram-Schmidt (:699-712) */
        for (int i = 0; i <= j; i++) {
          double h = t_dot(&t, n, V[i], Wv[j], red);
          H(i, j) = h;
          for (int k = 0; k < n; k++) Wv[j][k] = Wv[j][k] - h * V[i][k];
        }
        /* h(j+1,j) = ||w|| (:714-717) */
        H(j + 1, j) = sqrt(t_dot(&t, n, Wv[j], Wv[j], red));
        /* previous rotations on column j (:722-727) */
        for (int i = 0; i < j; i++) {
          if (p->literal) {
            H(i, j) = H(i, j) * cc[i] + H(i + 1, j) * ss[i];
            H(i, j) = -H(i, j) * ss[i] + H(i + 1, j) * cc[i];
          } else {
            double top = H(i, j) * cc[i] + H(i + 1, j) * ss[i];
            double bot = -H(i, j) * ss[i] + H(i + 1, j) * cc[i];
            H(i, j) = top;
            H(i + 1, j) = bot;
          }
        }
        /* new rotation (:728-733) */
        double beta = sqrt(H(j, j) * H(j, j) + H(j + 1, j) * H(j + 1, j));
        ss[j] = H(j + 1, j) / beta;
        cc[j] = H(j, j) / beta;
        H(j, j) = beta;
        gam[j + 1] = -ss[j] * gam[j];
        gam[j] = cc[j] * gam[j];
        if (hist) hist[hpos++] = fabs(gam[j + 1]);
        if (fabs(gam[j + 1]) <= eps) {
          jdone = j + 1;
          converged = 1;
          break;
        }
        /* v_{j+1} = w_j / h(j+1,j) (:774-777) */
        double hn = H(j + 1, j);
        for (int i = 0; i < n; i++) V[j + 1][i] = Wv[j][i] / hn;
      }
      /* back substitution (:739-747 and :784-792) and x = x + sum al_i z_i */
      for (int i = jdone - 1; i >= 0; i--) {
        double acc = 0.0;
        for (int k = i + 1; k < jdone; k++) acc = acc + H(i, k) * al[k];
        al[i] = (1.0 / H(i, i)) * (gam[i] - acc);
      }
      for (int i = 0; i < jdone; i++) {
        double a = al[i];
        for (int k = 0; k < n; k++) x[k] = x[k] + a * Z[i][k];
      }
      /* r = b - A x; ||r|| (:808-824) */
      t_spmv(&t, A, x, r);
      for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
      resnorm = sqrt(t_dot(&t, n, r, r, red));
      local_res = resnorm;
      restart++;
    }
  }
#undef H
  res->iter_done = iter;
  res->final_norm = resnorm;
  res->bnorm = bnorm;
  res->eps_used = eps;
  res->err = converged ? 0 : CELREF_ERR_NOCONV;
  res->arnoldi_steps = steps;
  free(r);
  for (int j = 0; j <= m; j++) free(V[j]);
  for (int j = 0; j < m; j++) {
    free(Z[j]);
    free(Wv[j]);
  }
  free(V);
  free(Z);
  free(Wv);
  free(hh);
  free(cc);
  free(ss);
  free(gam);
  free(al);
  free(part);
  return res->err;
}

/* ------------------------------------------------------------------------ */
/* FP32-storage Jacobi-PCG (inner solve of the iterative refinement)         */
/* ------------------------------------------------------------------------ */

/* Same recurrence as celref_pcg_jacobi with matrix, Jacobi and vectors held
 * in binary32: SpMV rows in float arithmetic, every vector update computed in
 * double from the float operands and rounded once to float, reductions in
 * double over exact float*float products, scalars in double. */
int celref_pcg_jacobi_f32(int n, const int* rp, const int* ci, const float* v, const float* J,
                          const float* b, float* x, const celref_params* p, double* hist,
                          celref_result* res) {
  size_t nb = sizeof(float) * (size_t)(n > 0 ? n : 1);
  float* r = (float*)malloc(nb);
  float* pv = (float*)malloc(nb);
  float* w = (float*)malloc(nb);
  int red = p->red;
  if (p->x0_mode == CELREF_X0_ONES)
    for (int i = 0; i < n; i++) x[i] = 1.0f;
  else if (p->x0_mode == CELREF_X0_ZERO)
    for (int i = 0; i < n; i++) x[i] = 0.0f;
  double bnorm = sqrt(celref_dot_f32(n, b, b, red));
  double eps = p->eps_abs;
  if (p->eps_rel > 0.0 && p->eps_rel * bnorm > eps) eps = p->eps_rel * bnorm;
  celref_spmv_csr_f32(n, rp, ci, v, x, r, 0);
  for (int i = 0; i < n; i++) r[i] = (float)((double)b[i] - (double)r[i]);
  /* z = J r is formed in double and never stored; p = (float) z */
  double* zd = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* rd = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    zd[i] = (double)r[i] * (double)J[i];
    rd[i] = (double)r[i];
    pv[i] = (float)zd[i];
  }
  double alpha = red == CELREF_RED_TREE ? dot_tree(n, rd, zd) : celref_dot(n, rd, zd, red, 1);
  double norm = sqrt(celref_dot_f32(n, r, r, red));
  if (hist) hist[0] = norm;
  int ii = 0, err = 0;
  while (ii < p->iter_max && fabs(alpha) > CELREF_REAL_SMALL && norm > eps) {
    celref_spmv_csr_f32(n, rp, ci, v, pv, w, 0);
    ii++;
    double pvd = celref_dot_f32(n, w, pv, red);
    double sigma = alpha / pvd;
    if (!isfinite(sigma)) {
      err = CELREF_ERR_BREAKDOWN;
      break;
    }
    double ms = -sigma;
    for (int i = 0; i < n; i++) {
      x[i] = (float)((double)x[i] + sigma * (double)pv[i]);
      r[i] = (float)((double)r[i] + ms * (double)w[i]);
      rd[i] = (double)r[i];
      zd[i] = (double)r[i] * (double)J[i];
    }
    double rz = red == CELREF_RED_TREE ? dot_tree(n, rd, zd) : celref_dot(n, rd, zd, red, 1);
    double beta = rz / alpha;
    alpha = rz;
    for (int i = 0; i < n; i++) pv[i] = (float)(beta * (double)pv[i] + zd[i]);
    norm = sqrt(celref_dot_f32(n, r, r, red));
    if (hist) hist[ii] = norm;
  }
  res->iter_done = ii;
  res->final_norm = norm;
  res->bnorm = bnorm;
  res->eps_used = eps;
  res->err = err;
  if (!err && norm > eps && ii >= p->iter_max) res->err = CELREF_ERR_NOCONV;
  res->arnoldi_steps = 0;
  free(r);
  free(pv);
  free(w);
  free(zd);
  free(rd);
  return res->err;
}
