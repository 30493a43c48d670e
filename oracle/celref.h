/*
 * celref.h -- CPU oracle for the CEL solver hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the Fortran hot path of the CRESTA
 * Exascale Library (hpcdkhab/cel_v3): CSR and JAD SpMV, the JAD
 * permutation, point-Jacobi set-up and application, the vector
 * reductions, Jacobi-PCG, CG and restarted GMRES(m) with right Jacobi
 * preconditioning.  It exists to check the CUDA library (libcelgpu.so)
 * and to serve as the timed CPU baseline; no product code path may call
 * it.  Every function names the reference lines it follows.
 *
 * Conventions
 *   - indices are 0-based int32 (the reference stores 1-based int32,
 *     src/fbase/cel_types_module.f90:14, and subtracts col_offset);
 *   - values are IEEE binary64 (rk=8, src/fbase/cel_types_module.f90:13)
 *     or binary32 for the *_f32 variants;
 *   - the library is compiled with -ffp-contract=off so that a*b+c is
 *     a rounded multiply followed by a rounded add, as written in the
 *     Fortran source.
 *
 * Reduction orders (the only place where the reference is not
 * deterministic, because it combines per-thread partials with
 * `!$omp atomic`, e.g. src/fop/cel_fop_vec_distr_module.f90:463-466):
 *   CELREF_RED_SEQ   worker chunks from cel_omp_shared_work_distr
 *                    (src/fbase/cel_omp_shared_work_module.f90:183-230),
 *                    each summed left to right from 0.0, chunk partials
 *                    added in worker order.  With one worker this is the
 *                    plain sequential sum of the reference.
 *   CELREF_RED_TREE  the fixed block-tree order the CUDA kernels use
 *                    (1024-element tiles, 256 lanes, butterfly over each
 *                    32-lane warp, warps added in order; tile partials
 *                    reduced the same way).  It lets the oracle reproduce
 *                    a GPU solve bit for bit.
 */
#ifndef CELREF_H
#define CELREF_H
#ifdef __cplusplus
extern "C" {
#endif

#define CELREF_RED_SEQ 0
#define CELREF_RED_TREE 1

#define CELREF_FMT_CSR 0
#define CELREF_FMT_JAD 1

#define CELREF_X0_ONES 0 /* reference: x=1, src/fcgalg/cel_cgalg_module.f90:209 */
#define CELREF_X0_ZERO 1
#define CELREF_X0_USER 2

#define CELREF_OK 0
#define CELREF_ERR_ARG 1
#define CELREF_ERR_BREAKDOWN 3
#define CELREF_ERR_NOCONV 4

/* 1.1*EPSILON(1.0_rk), src/fbase/cel_types_module.f90:33 */
#define CELREF_REAL_SMALL (1.1 * 2.220446049250313e-16)

/* reduction tile geometry shared with the CUDA kernels */
#define CELREF_TILE 1024
#define CELREF_LANES 256

typedef struct {
  int fmt;            /* CELREF_FMT_CSR or CELREF_FMT_JAD */
  int n;              /* rows (square) */
  int nnz;
  const int* rp;      /* CSR row pointer, n+1 */
  const int* ci;      /* CSR columns, nnz */
  const double* v;    /* CSR values, nnz */
  /* JAD arrays (fmt == CELREF_FMT_JAD) */
  int mmax;
  const int* jbegin;  /* mmax+1 */
  const int* jci;
  const double* jv;
  const int* perm;    /* n */
} celref_mat;

typedef struct {
  int x0_mode;      /* CELREF_X0_* */
  double eps_abs;   /* stop when ||r||_2 <= eps (reference: absolute) */
  double eps_rel;   /* if > 0: eps = max(eps_abs, eps_rel*||b||_2) */
  int iter_max;
  int red;          /* CELREF_RED_* */
  int nworkers;     /* reference worker threads (the master thread is extra) */
  int literal;      /* CG: reproduce the reference's alpha-as-beta update */
  int restart;      /* GMRES(m): m */
} celref_params;

typedef struct {
  int iter_done;
  double final_norm;  /* last ||r||_2 seen by the recurrence */
  double bnorm;
  double eps_used;
  int err;
  int arnoldi_steps;  /* GMRES only: total inner steps */
} celref_result;

/* --- work split: cel_omp_shared_work_distr ------------------------------ */
void celref_work_chunk(int len, int nworkers, int worker, int* start, int* end);

/* --- SpMV --------------------------------------------------------------- */
void celref_spmv_csr(int n, const int* rp, const int* ci, const double* v,
                     const double* x, double* y, int accumulate, int nworkers);
void celref_spmv_csr_f32(int n, const int* rp, const int* ci, const float* v,
                         const float* x, float* y, int accumulate);
int celref_jad_perm(int n, const int* rp, int* perm, int* mmax);
int celref_jad_build(int n, const int* rp, const int* ci, const double* v,
                     int* perm, int* jbegin, int* jci, double* jv, int* mmax);
void celref_jad_begin_literal(int n, const int* rp, int* icnt_out, int* lo_out, int* hi_out);
void celref_spmv_jad(int n, int mmax, const int* jbegin, const int* jci,
                     const double* jv, const int* perm, const double* x, double* y);
void celref_spmv(const celref_mat* A, const double* x, double* y, int nworkers);

/* --- set-up ------------------------------------------------------------- */
void celref_diag(int n, const int* rp, const int* ci, const double* v, double* d);
void celref_jacobi(int n, const double* d, const double* s, double* J);
void celref_row_scale(int n, const int* rp, double* v, const double* d, double* s);
int celref_block_jacobi_inv(int n, const int* rp, const int* ci, const double* v, int bs,
                            double* inv);
void celref_block_jacobi_apply(int n, int bs, const double* inv, const double* r, double* z);

/* --- reductions and sweeps ------------------------------------------------ */
double celref_dot(int n, const double* a, const double* b, int red, int nworkers);
double celref_dot_f32(int n, const float* a, const float* b, int red);
double celref_reduce256(const double* vals, long cnt);
double celref_dot_tree_perm(int n, const double* a, const double* b, const int* perm);

/* --- solvers ------------------------------------------------------------ */
int celref_pcg_jacobi(const celref_mat* A, const double* J, const double* b,
                      double* x, const celref_params* p, double* hist,
                      celref_result* res);
int celref_cg(const celref_mat* A, const double* b, double* x,
              const celref_params* p, double* hist, celref_result* res);
int celref_gmres_jacobi(const celref_mat* A, const double* J, const double* b,
                        double* x, const celref_params* p, double* hist,
                        celref_result* res);
int celref_pcg_jacobi_f32(int n, const int* rp, const int* ci, const float* v,
                          const float* J, const float* b, float* x,
                          const celref_params* p, double* hist, celref_result* res);

#ifdef __cplusplus
}
#endif
#endif
