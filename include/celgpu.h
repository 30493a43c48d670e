/*
 * celgpu.h -- C ABI of libcelgpu.so, the B200 (sm_100a) implementation of the
 * CEL solver hot path: CSR/JAD SpMV, point-Jacobi, the fused PCG / CG /
 * GMRES(m) iteration bodies, FP32-storage iterative refinement, batched
 * and multi-right-hand-side PCG, and the adjoint gradient of a PCG solve.
 *
 * Every entry point returns an int status (CELG_OK == 0) and never aborts.
 * Index arrays are int32 as in the reference (ik=4,
 * src/fbase/cel_types_module.f90:14); values are binary64 (rk=8, :13).
 * Pointers named *_d are device pointers on the handle's device; all other
 * pointers are host pointers owned by the caller.  A handle owns one CUDA
 * stream (or borrows the caller's) and its work buffers; a handle is not
 * thread-safe, distinct handles may be used from distinct threads.
 *
 * Reference interfaces each entry point replaces are cited as
 * file:line within hpcdkhab/cel_v3.
 */
#ifndef CELGPU_H
#define CELGPU_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference's integer err_code convention,
 *      src/fbase/cel_error_module.f90:17-32, without its STOP) ------------- */
#define CELG_OK 0
#define CELG_ERR_ARG 1        /* bad argument or malformed matrix          */
#define CELG_ERR_CUDA 2       /* a CUDA runtime call failed                */
#define CELG_ERR_BREAKDOWN 3  /* alpha/beta/sigma not finite (p.Ap == 0)   */
#define CELG_ERR_NOCONV 4     /* iteration limit reached before tolerance  */
#define CELG_ERR_TIMEOUT 5    /* a device-side bounded wait gave up        */
#define CELG_ERR_STATE 6      /* call out of order (e.g. DoIt before MatrixCompleted) */
#define CELG_ERR_COMM 7       /* an exchange between ranks (callback or NCCL) failed */

/* ---- formats and modes (mv_algorithm, src/fbase/cel_types_module.f90:58-81) */
#define CELG_FMT_CSR 0
#define CELG_FMT_JAD 1

#define CELG_X0_REF_ONES 0 /* x0 = 1 as in src/fcgalg/cel_cgalg_module.f90:209 */
#define CELG_X0_ZERO 1
#define CELG_X0_USER 2     /* x_d holds the start vector on entry */

#define CELG_PREC_FP64 0
#define CELG_PREC_FP32_IR 1 /* FP32 matrix/Krylov vectors inside FP64 refinement:
                             * each correction is a fresh inner PCG solve      */
#define CELG_PREC_FP32_RU 2 /* FP32 PCG with FP64 reliable updates: the outer
                             * residual, update and test in FP64, the search
                             * direction kept across corrections              */

#define CELG_PRECOND_JACOBI 0       /* point Jacobi, the reference's cel_cgalg_jacobi */
#define CELG_PRECOND_BLOCK_JACOBI 1 /* inverse diagonal blocks (celg_mat_block_jacobi) */

#define CELG_SOLVER_PCG 0   /* cel_cgalg_jacobi   (BENCHMARK_CG + Jacobi)     */
#define CELG_SOLVER_CG 1    /* cel_cgalg          (BENCHMARK_CG, no precond.) */
#define CELG_SOLVER_GMRES 2 /* cel_gmresalg_2jacobi (BENCHMARK_GMRES + Jacobi) */

typedef struct celg_handle celg_handle;
typedef struct celg_mat celg_mat;

/* Solver parameters: cel_cgalg_parameter_type / cel_gmresalg_parameter_type
 * (src/fcgalg/cel_alg_module.f90:26-54) plus the selections the reference
 * keeps in input_parameters (src/fbase/cel_input_parameters_module.f90:128-170). */
typedef struct {
  int x0_mode;          /* CELG_X0_*                                             */
  double eps_abs;       /* stop when ||r||_2 <= eps (reference: absolute, :247-249) */
  double eps_rel;       /* if > 0, eps = max(eps_abs, eps_rel * ||b||_2)          */
  int iter_max;         /* PCG/CG iterations; GMRES outer iterations            */
  int fmt;              /* CELG_FMT_CSR or CELG_FMT_JAD                          */
  int precision;        /* CELG_PREC_*                                           */
  int literal_ref_bugs; /* CG: alpha-as-beta (:151); GMRES: unrotated Givens (:722-727) */
  int restart;          /* GMRES(m): m (gmres_max_restart)                      */
  double inner_eps_rel; /* FP32-IR: tightest inner PCG relative tolerance
                         (default 1e-4; a single-system refinement step asks
                         for the looser tolerance that spreads the remaining
                         reduction evenly over the steps it needs);
                         FP32-RU: residual drop that triggers an FP64 update */
  int inner_iter_max;   /* FP32-IR: inner iteration cap                         */
  int outer_max;        /* FP32-IR: refinement steps cap                        */
  int precond;          /* CELG_PRECOND_*: PCG preconditioner (FP64 CSR solves)  */
} celg_params;

/* Solve report.  history (caller-owned host buffer of history_cap doubles,
 * nullable) receives ||r||_2 per iteration (PCG/CG), |gamma_{j+1}| per
 * Arnoldi step (GMRES) or the outer residual per refinement (FP32-IR). */
typedef struct {
  int iter_done;          /* niter of cel_elmSolverDoIt                   */
  double final_norm2;     /* ftol: last recurrence ||r||_2                */
  double bnorm;           /* ||b||_2                                      */
  double verified_relres; /* ||b - A x||_2 / ||b||_2 recomputed in FP64   */
  int err;                /* same as the return value                     */
  int arnoldi_steps;      /* GMRES inner steps; FP32-IR inner iterations  */
  double* history;
  int history_cap;
  int history_len;        /* entries written                              */
} celg_result;

void celg_params_default(celg_params* p);

/* ---- handle ---------------------------------------------------------------- */
/* stream: NULL -> the handle creates and owns a non-blocking stream; any
 * cudaStream_t otherwise, including cudaStreamLegacy ((cudaStream_t)0x1) for
 * the legacy default stream.  Solve graphs are captured on a private stream
 * and launched on this one. */
int celg_create(celg_handle** h, int device, void* stream);
int celg_destroy(celg_handle* h);
int celg_set_stream(celg_handle* h, void* stream);
const char* celg_status_string(int status);
int celg_sm_count(celg_handle* h, int* sms);

/* ---- matrix ---------------------------------------------------------------- */
/* CSR upload.  Replaces cel_sp_mat_to_csr (src/fspmt/cel_sp_mat_module.f90:430-456)
 * and the single-subdomain case of cel_sp_mat_distr_from_sp_mat_local
 * (src/fspmtdistr/cel_sp_mat_distr_module.f90:34-301).  index_base 0 or 1
 * (the reference is 1-based, xadj(1)=1).  Rows must be given in order;
 * columns may be in any order inside a row and are summed in the given order.
 * Host arrays are copied; the caller keeps ownership. */
int celg_mat_from_csr(celg_handle* h, int n, int nnz, const int* row_ptr, const int* cols,
                      const double* vals, int index_base, celg_mat** out);
/* One rank's row block of a matrix distributed by rows (the reference's
 * vtxdist blocks, src/fspmtdistr/cel_sp_mat_distr_module.f90:330-339): n local
 * rows whose columns 0..n-1 are the local rows and n..ncols-1 the halo values
 * received from other ranks.  Usable with celg_spmv (x of ncols entries),
 * celg_mat_jacobi and the celg_dist_* solver below; the single-system solvers
 * reject it (CELG_ERR_ARG). */
int celg_mat_from_csr_ext(celg_handle* h, int n, int ncols, int nnz, const int* row_ptr,
                          const int* cols, const double* vals, int index_base, celg_mat** out);
/* COO triplets (host arrays, any order, duplicates allowed and kept) -> CSR on
 * the device: a stable sort by (row, column), so equal keys keep their input
 * order, and the row pointer from the row counts.  Replaces
 * cel_sp_mat_format_sparse_31_sort (src/fspmt/cel_sp_mat_module.f90:518-585)
 * followed by cel_sp_mat_to_csr (:430-456).  ncols >= n (halo columns as in
 * celg_mat_from_csr_ext). */
int celg_mat_from_coo(celg_handle* h, int n, int ncols, int nnz, const int* rows, const int* cols,
                      const double* vals, int index_base, celg_mat** out);
/* MatrixMarket files, read as mmread does (src/fbase/cel_mmio_module.f90:17-341):
 * coordinate or array, real / integer / pattern (pattern values are 1.0),
 * general / symmetric / skew-symmetric; complex files are rejected.  Entries
 * come back 1-based in file order, exactly as stored; expand != 0 adds the
 * mirrored entry (negated for skew-symmetric) after each off-diagonal entry
 * of a symmetric file.  celg_mm_info gives the sizes and the entry count for
 * that choice of expand. */
#define CELG_MM_GENERAL 0
#define CELG_MM_SYMMETRIC 1
#define CELG_MM_SKEW 2
int celg_mm_info(const char* path, int expand, int* nrows, int* ncols, int* nnz, int* symmetry);
int celg_mm_read(const char* path, int expand, int nnz_cap, int* rows, int* cols, double* vals);
/* same with device arrays (0-based), copied device to device */
int celg_mat_from_csr_device(celg_handle* h, int n, int nnz, const int* row_ptr_d,
                             const int* cols_d, const double* vals_d, celg_mat** out);
int celg_mat_destroy(celg_mat* m);
int celg_mat_info(const celg_mat* m, int* n, int* nnz, int* jad_mmax);
/* The column data the solver sweeps (and the JAD SpMV) read for this matrix,
 * which sets their bytes per non-zero: CELG_COLS_INT32 (the int32 columns),
 * CELG_COLS_OFFSET8 (1-byte indices into a dictionary of at most 256 column
 * offsets col - row) or CELG_COLS_PATTERN (one byte per row indexing at most
 * 256 sequences of at most 8 offsets; no column data per entry).  The last
 * two are built on the first solve, FP32 copy or JAD conversion of a matrix
 * whose rows fit them; results are the same bits in every form.  celg_spmv
 * in CSR reads the int32 columns.  No counterpart in the reference. */
#define CELG_COLS_INT32 0
#define CELG_COLS_OFFSET8 1
#define CELG_COLS_PATTERN 2
int celg_mat_column_form(const celg_mat* m, int* form);
/* CSR -> JAD, cel_sp_mat_jad_from_sp_mat_local
 * (src/fspmtconverter/cel_sp_mat_jad_converter_module.f90:93-175): the reference's
 * permutation (stable sort by descending row length) and Saad's jagged
 * diagonals.  perm_out (host, n entries, nullable) receives the 0-based
 * permutation. */
int celg_mat_to_jad(celg_mat* m, int* perm_out);
/* JAD arrays back to the host (for checking): perm n, begin mmax+1, cols/vals nnz */
int celg_mat_get_jad(const celg_mat* m, int* perm, int* begin, int* cols, double* vals);
/* Point-Jacobi set-up, cel_sp_mat_distr_set_jacobi
 * (src/fspmtdistr/cel_sp_mat_distr_format_module.f90:149-203) with the diagonal
 * of src/fspmtdistr/cel_sp_mat_distr_module.f90:197-207 (last stored diagonal
 * entry wins; missing diagonal -> 1/0 = inf, as in the reference). */
int celg_mat_jacobi(celg_mat* m);
int celg_mat_get_jacobi(const celg_mat* m, double* jacobi_host);
/* Diagonal row scaling, cel_sp_mat_distr_scale
 * (src/fspmtdistr/cel_sp_mat_distr_format_module.f90:91-145): A_ij /= sqrt|d_i|,
 * jacobi = sqrt|d|/d.  celg_elm_doit divides b by sqrt|d| itself
 * (cel_sp_mat_distr_boundary_diag_scale); direct solver calls expect a
 * right-hand side that is already scaled. */
int celg_mat_scale_diagonal(celg_mat* m);
/* FP32 copy of the matrix values for the refinement inner solve */
int celg_mat_make_fp32(celg_mat* m);

/* ---- operators (device pointers, on the handle's stream) -------------------- */
/* y = (accumulate ? y : 0) + A x.  cel_fop_mv_axy_distr
 * (src/fop/cel_fop_mv_module.f90:28-87) -> worker_local_csr (:189-247) or
 * worker_local_jad (:250-352).  Each row is summed left to right from 0.0 in
 * stored order, multiply and add rounded separately. */
int celg_spmv(celg_handle* h, const celg_mat* m, int fmt, const double* x_d, double* y_d,
              int accumulate);
int celg_spmv_f32(celg_handle* h, const celg_mat* m, const float* x_d, float* y_d, int accumulate);
/* cel_fop_vec_distr_dot_allreduce (src/fop/cel_fop_vec_distr_module.f90:724-775) */
int celg_dot(celg_handle* h, int n, const double* a_d, const double* b_d, double* out);
/* cel_fop_vec_distr_norm2_allreduce (:433-483), returns the square root */
int celg_norm2(celg_handle* h, int n, const double* a_d, double* out);
/* y = y + alpha x: cel_fop_vec_distr_scale (:836-874) */
int celg_axpy(celg_handle* h, int n, double alpha, const double* x_d, double* y_d);
/* y = beta y + x: cel_fop_vec_distr_scale_1 (:918-956) */
int celg_xpby(celg_handle* h, int n, const double* x_d, double beta, double* y_d);
/* Block Jacobi: inverse diagonal blocks of block_size rows (1, 2, 4, 8, 16 or
 * 32; the last block may be shorter), built as the reference's dead
 * cel_prec_build_diagonal + cel_prec_build_diagonal_inv intend
 * (src/fspmtdistr/cel_prec_module.f90:27-339): a row's entries are scanned in
 * stored order up to the first column right of the block, Doolittle LU without
 * pivoting, inverse by forward and back substitution per unit vector.
 * CELG_ERR_BREAKDOWN when an inverse has a non-finite entry (zero pivot).
 * Used by celg_pcg_jacobi with params.precond = CELG_PRECOND_BLOCK_JACOBI. */
int celg_mat_block_jacobi(celg_mat* m, int block_size);
/* host copy of the n x block_size inverse rows (row-major, zero-padded) */
int celg_mat_get_block_jacobi(const celg_mat* m, double* inv_host);
/* z = blockdiag(D^-1) r (cel_fop_block_jacobi_vec_mult,
 * src/fop/cel_fop_block_jacobi_module.f90:29-190, with r(j) where the
 * reference's general case reads r(i)) */
int celg_block_jacobi_apply(celg_handle* h, const celg_mat* m, const double* r_d, double* z_d);
/* z = r * jacobi: cel_fop_vec_mult_distr_jacobi (:338-375) */
int celg_jacobi_apply(celg_handle* h, const celg_mat* m, const double* r_d, double* z_d);

/* ---- solvers (b_d, x_d device vectors of length n) ---------------------------- */
/* Jacobi-PCG, cel_cgalg_jacobi (src/fcgalg/cel_cgalg_module.f90:178-305).
 * The loop runs while iter < iter_max, ||r|| > eps and |r.z| > 1.1 eps_mach:
 * the last test is the reference's absolute guard (:248), so a solve whose
 * residual is already tiny in absolute terms (small ||b||, tight eps_rel) can
 * end with CELG_OK before ||r|| <= eps; final_norm2 and verified_relres say
 * where it ended.
 * precision CELG_PREC_FP32_IR runs FP32-storage PCG sweeps inside FP64
 * iterative refinement; the outer residual, update and test stay FP64. */
int celg_pcg_jacobi(celg_handle* h, celg_mat* m, const double* b_d, double* x_d,
                    const celg_params* p, celg_result* res);
/* Unpreconditioned CG, cel_cgalg (src/fcgalg/cel_cgalg_module.f90:34-175). */
int celg_cg(celg_handle* h, celg_mat* m, const double* b_d, double* x_d, const celg_params* p,
            celg_result* res);
/* Restarted GMRES(m) with right Jacobi, cel_gmresalg_2jacobi
 * (src/fcgalg/cel_gmresalg_module.f90:570-851), Givens update corrected unless
 * literal_ref_bugs. */
int celg_gmres_jacobi(celg_handle* h, celg_mat* m, const double* b_d, double* x_d,
                      const celg_params* p, celg_result* res);
/* Host-buffer convenience: copies b in and x out on the handle's stream. */
int celg_solve_host(celg_handle* h, celg_mat* m, int solver, const double* b_host,
                    double* x_host, const celg_params* p, celg_result* res);

/* ---- batched form -------------------------------------------------------------- */
/* Jacobi-PCG on `count` independent systems of uneven size in one device-driven
 * loop (one CUDA graph launch for the whole batch).  mats[k] must have Jacobi
 * set; b_d[k], x_d[k] are device vectors of mats[k]'s size.  p applies to every
 * system (eps_rel relative to each system's own ||b||).  res (count entries,
 * nullable) receives the per-system reports; history is not recorded.  Each
 * system's result is bit-identical to celg_pcg_jacobi on it alone.  The
 * concatenated copy of the matrices is cached on the handle until another
 * batch or a celg_mat_destroy.  precision CELG_PREC_FP64, CELG_PREC_FP32_IR
 * (FP32 inner solves inside FP64 refinement of every system: iter_done is
 * then the outer step count, arnoldi_steps the inner iterations, as for
 * celg_pcg_jacobi) or CELG_PREC_FP32_RU (FP32 PCG with FP64 reliable updates
 * of every system: arnoldi_steps = reliable updates, final_norm2 = the last
 * FP64 residual norm); each system's result equals celg_pcg_jacobi with the
 * same precision on it alone, bit for bit. */
int celg_pcg_batched(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                     double* const* x_d, const celg_params* p, celg_result* res);

/* ---- diagnostics --------------------------------------------------------------- */
/* Runs the library's bounded device wait on an mbarrier that nothing arrives
 * on, with a limit of limit_ms (1..10000) milliseconds, and stores the status
 * the kernel reported (CELG_ERR_TIMEOUT when the bound works).  The handle and
 * its context remain usable.  No counterpart in the reference, whose waits
 * (MPI_Test polling, src/felmsolver/cel_elmsolver_module.f90:637-644) have no
 * limit. */
int celg_check_bounded_wait(celg_handle* h, int limit_ms, int* status);

/* Jacobi-PCG on k (1..32) right-hand sides sharing one matrix: B_d and X_d
 * are n x k row-major (entry (i,c) at i*k + c).  Every column runs its own
 * recurrence (own scalars, own convergence); each iteration reads the matrix
 * once for all columns (block SpMM).  res (k entries, nullable) receives the
 * per-column reports.  Per-column SpMVs are bit-identical to celg_spmv; the
 * column dot products use a warp-ordered tile reduction (see multirhs.cu).
 * precision CELG_PREC_FP32_IR refines every column around FP32 inner solves
 * (iter_done = outer steps, arnoldi_steps = inner iterations);
 * CELG_PREC_FP32_RU runs every column as FP32 PCG with FP64 reliable updates
 * (threshold inner_eps_rel, default 1e-2; arnoldi_steps = reliable updates,
 * final_norm2 = the last FP64 residual norm), the column's arithmetic that of
 * celg_pcg_jacobi with CELG_PREC_FP32_RU. */
int celg_pcg_multirhs(celg_handle* h, celg_mat* m, int k, const double* B_d, double* X_d,
                      const celg_params* p, celg_result* res);

/* The launch configuration the autotuners picked on this handle, for the
 * last batched solve (what = CELG_TUNE_BATCH: out[0] = resident CTAs per SM
 * of the SpMV sweep, 0 meaning as many as fit; out[1] = CTAs per SM of the
 * vector sweeps) or multi-right-hand-side solve (what = CELG_TUNE_SPMM:
 * out[0] = the FP64 SpMM variant, 0..14; out[1] = the FP32 SpMM shape of
 * the FP32 forms, 0..4, or -1 before the first of them).  No counterpart in
 * the reference, which has no autotuner.  CELG_ERR_STATE before the first
 * such solve. */
#define CELG_TUNE_BATCH 0
#define CELG_TUNE_SPMM 1
int celg_tuned_config(celg_handle* h, int what, int out[2]);

/* ---- differentiation --------------------------------------------------------- */
/* Adjoint of a Jacobi-PCG solve x = A^{-1} b (A symmetric): given x_d and
 * g_d = dL/dx, solves A lambda = g with Jacobi-PCG under p (the precision
 * field is ignored: FP64), writes lambda_d = dL/db and, when grad_vals_d is
 * not NULL, dL/dA on the sparsity pattern: grad_vals_d[k] = -lambda_i x_j for
 * stored entry k = (i, j).  res reports the adjoint solve. */
int celg_pcg_adjoint(celg_handle* h, celg_mat* m, const double* x_d, const double* g_d,
                     double* lambda_d, double* grad_vals_d, const celg_params* p, celg_result* res);
/* Face-coefficient gradient of a 7-point diffusion operator on an nx x ny x nz
 * grid (A_ii = sum of the cell's six face coefficients, A_ij = -k_f):
 * dL/dk_f = -(lambda_i - lambda_j)(x_i - x_j) for the face between cells i, j
 * and -(lambda_i x_i) for a Dirichlet face of cell i.  Face arrays are x-fastest
 * with shapes (nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx). */
int celg_diffusion7_face_grad(celg_handle* h, int nx, int ny, int nz, const double* lambda_d,
                              const double* x_d, double* gkx_d, double* gky_d, double* gkz_d);

/* ---- distributed Jacobi-PCG (one row block per rank) ------------------------------ */
/* The multi-process form of cel_cgalg_jacobi (src/fcgalg/cel_cgalg_module.f90:
 * 178-305): per iteration a halo exchange of p before the SpMV
 * (src/fspmtdistr/cel_sp_mat_distr_vec_module.f90:265-724) and sum-allreduces
 * of the dot products (src/fop/cel_fop_vec_distr_module.f90:419-832).  The
 * library runs the local sweeps as stream-ordered kernels; the caller runs the
 * exchanges (NCCL, CUDA-aware MPI, ...) on the handle's stream between them.
 * Nothing synchronises the host except _poll and _result, so iterations can be
 * queued back to back or captured in a CUDA graph together with the caller's
 * collectives.
 *
 * Vectors: b_d, r_d, v_d have n entries; x_ext_d and p_ext_d have ncols
 * entries (local part first, halo after).  The exchange buffer holds
 * CELG_DIST_NEXCH doubles on the device; each phase marked [R] below
 * overwrites all of them with this rank's partial sums, and the caller then
 * sum-all-reduces the whole buffer before the next phase.  Sequence:
 *   begin [R]; halo(x); init [R]; start;
 *   repeat: halo(p); ap [R]; update [R]; direction;    (until poll says done)
 *   halo(x); verify [R]; result.
 * With the halo of p overlapped: start halo(p) on another stream, then
 * ap_interior; wait for the halo; ap_boundary [R] (in place of ap).
 * Iterations queued after convergence do no work (their exchanges still run,
 * identically on every rank).  Every rank reaches the same decisions because
 * they are taken from the reduced values only; a bounded-wait timeout on any
 * rank is reduced with the sums and stops all ranks.
 * state_d: CELG_DIST_STATE_BYTES of 16-byte aligned device memory owned by
 * the caller (exchange buffer at its start), or NULL to let the library
 * allocate it.  hist_d: device array of hist_cap doubles for ||r|| per
 * iteration, or NULL.  params: x0_mode, eps_abs, eps_rel, iter_max (FP64
 * CSR only). */
#define CELG_DIST_NEXCH 5
#define CELG_DIST_STATE_BYTES 256
typedef struct celg_dist celg_dist;
int celg_dist_create(celg_handle* h, celg_mat* m, const celg_params* p, void* state_d,
                     double* hist_d, int hist_cap, celg_dist** out);
int celg_dist_destroy(celg_dist* d);
int celg_dist_exchange_buffer(celg_dist* d, double** xch_d);
int celg_dist_pcg_begin(celg_dist* d, const double* b_d, double* x_ext_d);            /* [R] */
int celg_dist_pcg_init(celg_dist* d, const double* b_d, const double* x_ext_d, double* r_d,
                       double* p_ext_d);                                              /* [R] */
int celg_dist_pcg_start(celg_dist* d);
int celg_dist_pcg_ap(celg_dist* d, const double* p_ext_d, double* v_d);               /* [R] */
/* celg_dist_pcg_ap in two launches with the same results: the interior rows
 * (the longest run of 1024-row tiles that read no halo column) need only the
 * local part of p, so they may run while the halo of p is in flight; the
 * boundary launch (after the halo) does the other rows and the p.v partial
 * sums.  interior_rows gives that row range [row_lo, row_hi).  A block with
 * no halo reads does all of ap in the interior half. */
int celg_dist_pcg_ap_interior(celg_dist* d, const double* p_ext_d, double* v_d);
int celg_dist_pcg_ap_boundary(celg_dist* d, const double* p_ext_d, double* v_d);      /* [R] */
int celg_dist_interior_rows(celg_dist* d, int* row_lo, int* row_hi);
int celg_dist_pcg_update(celg_dist* d, double* r_d, const double* v_d);               /* [R] */
/* applies the preceding update's x += sigma p (old p), then p = beta p + J r */
int celg_dist_pcg_direction(celg_dist* d, double* x_ext_d, const double* r_d, double* p_ext_d);
/* synchronises the stream; active = 0 once the loop has ended */
int celg_dist_pcg_poll(celg_dist* d, int* active, int* iter);
int celg_dist_pcg_verify(celg_dist* d, const double* b_d, const double* x_ext_d);      /* [R] */
/* synchronises; returns the solve status, fills res (history from hist_d) */
int celg_dist_pcg_result(celg_dist* d, celg_result* res);

/* ---- distributed Jacobi-PCG in one call ------------------------------------------- */
/* The whole solve of one rank, with the exchanges inside the call as in the
 * reference: the halo of p before every SpMV (cel_fop_mv_axy_distr,
 * src/fop/cel_fop_mv_module.f90:48-81) and a sum all-reduce per reduction
 * phase (the MPI_ALLREDUCE in every cel_fop_vec_distr_* dot,
 * src/fop/cel_fop_vec_distr_module.f90:419-832; the communicator the ELM API
 * takes, src/felmsolver/cel_elmsolver_module.f90:103).  It runs the phase
 * sequence above on work vectors the celg_dist object keeps; the caller's
 * part is the start vector x_ext_d (ncols entries, local part used with
 * CELG_X0_USER) and b_d.  The host polls the stopping flag every poll_every
 * iterations (queued iterations after convergence do no work).  res as
 * celg_dist_pcg_result.  Every rank must make the same calls.
 *
 * Exchanges through the caller's communication layer: each callback
 * enqueues its work on `stream` (the handle's stream) or finishes it before
 * returning, and returns 0 on success (anything else ends the solve with
 * CELG_ERR_COMM).  allreduce_sum sums `count` doubles at buf_d (device)
 * over all ranks, in place; halo sends this rank's rows that other ranks
 * read and receives their values into entries n..ncols-1 of vec_ext_d. */
typedef struct {
  void* ctx;
  int (*allreduce_sum)(void* ctx, double* buf_d, int count, void* stream);
  int (*halo)(void* ctx, double* vec_ext_d, void* stream);
} celg_dist_comm;
int celg_dist_pcg_solve(celg_dist* d, const celg_dist_comm* comm, const double* b_d,
                        double* x_ext_d, int poll_every, celg_result* res);
/* The same with the library running the exchanges over NCCL (libnccl.so.2,
 * loaded on first use; CELG_ERR_STATE when it cannot be loaded).  The
 * exchange plan lists, per neighbour (nneigh of them): its rank, the
 * send_counts[q] local rows (0-based, concatenated over the neighbours in
 * send_rows) whose values it reads, and the recv_counts[q] halo entries it
 * provides, which land at vec_ext_d[n + recv_starts[q] ...].  A communicator
 * comes from celg_nccl_comm_create on every rank with the unique id that
 * one rank made with celg_nccl_unique_id (the caller broadcasts it).
 * overlap != 0 sends the halo of p on a side stream while the interior
 * rows' SpMV runs (celg_dist_pcg_ap_interior / _boundary). */
#define CELG_NCCL_ID_BYTES 128
int celg_dist_set_exchange(celg_dist* d, int nneigh, const int* peers, const int* send_counts,
                           const int* send_rows, const int* recv_starts, const int* recv_counts);
int celg_nccl_unique_id(unsigned char id[CELG_NCCL_ID_BYTES]);
int celg_nccl_comm_create(const unsigned char id[CELG_NCCL_ID_BYTES], int nranks, int rank,
                          int device, void** nccl_comm);
int celg_nccl_comm_destroy(void* nccl_comm);
int celg_dist_pcg_solve_nccl(celg_dist* d, void* nccl_comm, const double* b_d, double* x_ext_d,
                             int poll_every, int overlap, celg_result* res);

/* ---- allocation-free entry point ------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (their device memory belongs to their own pool or to another
 * framework's caching allocator): a dot product that needs no handle and
 * keeps its reduction scratch in a fixed file-scope device array of the
 * library.  out_d[0] = a.b in the same order as celg_dot.  n may not exceed
 * CELG_NOALLOC_MAX_ROWS (CELG_ERR_ARG otherwise).  Calls share the array:
 * calls whose kernels overlap on the GPU race.  A call outside a stream
 * capture looks the array's device address up again (so it stays valid
 * across a cudaDeviceReset); a call on a capturing stream uses the address
 * an earlier call found, so make one call on the device before capturing.
 * stream: a cudaStream_t of the current device, NULL for the default stream. */
#define CELG_NOALLOC_MAX_ROWS 67108864
int celg_dot_noalloc(int n, const double* a_d, const double* b_d, double* out_d, void* stream);

/* ---- ELM assembly API (src/felmsolver/cel_elmsolver_module.f90) -------------- */
/* cel_elmSolverInitialization (:103-153): n_total rows, n_local local rows
 * starting at 1-based row row_low, nnz_hint[2] nonzeros per row (diagonal and
 * off-diagonal block).  Defaults as the reference: GMRES(3) + Jacobi +
 * diagonal scaling, eps 1e-8, iter_max 5000 (:134-151). */
int celg_elm_init(celg_handle* h, int n_total, int n_local, int row_low, const int nnz_hint[2]);
int celg_elm_set_solver(celg_handle* h, int solver, const celg_params* p, int diag_scaling);
int celg_elm_row_start(celg_handle* h, int row);                     /* :155-159 */
int celg_elm_insert(celg_handle* h, int col, double value);          /* :161-172 */
int celg_elm_reinsert(celg_handle* h, int col, double value);        /* :174-187 */
int celg_elm_row_completed(celg_handle* h);                          /* :189-191 */
/* bulk form of row_start/insert for whole rows, 1-based like the above */
int celg_elm_insert_rows(celg_handle* h, int first_row, int nrows, const int* row_ptr,
                         const int* cols, const double* vals);
int celg_elm_matrix_completed(celg_handle* h);                       /* :193-439 */
/* cel_elmSolverDoIt (:441-651): b on the host; iierr/niter/ftol as the reference */
int celg_elm_doit(celg_handle* h, const double* b, int* iierr, int* niter, double* ftol);
int celg_elm_redoit(celg_handle* h, const double* b, int* iierr, int* niter, double* ftol);
/* cel_elmSolverCollectSolution (:790-815): x into a caller-owned buffer of n_local */
int celg_elm_collect_solution(celg_handle* h, double* x);
/* cel_elmSolverPerformance (:879-900): last solve's device time and counters */
int celg_elm_performance(celg_handle* h, double* solve_ms, int* iters, double* bytes_per_iter);
int celg_elm_destroy(celg_handle* h);                                /* :817-877 */

#ifdef __cplusplus
}
#endif
#endif
