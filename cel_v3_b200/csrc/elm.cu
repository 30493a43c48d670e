// elm.cu -- the ELM assembly interface of the reference
// (src/felmsolver/cel_elmsolver_module.f90) on one GPU: row-wise insertion of
// 1-based entries, MatrixCompleted (sort, CSR, Jacobi, optional diagonal
// scaling and JAD), DoIt/ReDoIt with a host right-hand side, CollectSolution
// into a caller-owned buffer.  Single sub-domain only: the MPI gather onto
// reduce-masters (:299-345) has nothing to do on one rank.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "celg_internal.h"

struct Elm {
  int n_total = 0, n_local = 0, row_low = 1;
  std::vector<int> rows, cols;
  std::vector<double> vals;
  std::vector<long long> diag_idx;
  int cur_row = -1;
  celg_mat* mat = nullptr;
  bool completed = false;
  int solver = CELG_SOLVER_GMRES;
  celg_params params;
  int diag_scaling = 1;
  double* b_d = nullptr;
  double* x_d = nullptr;
  bool solved = false;
};

using namespace celg;

extern "C" int celg_elm_destroy(celg_handle* h) {
  if (!h || !h->elm) return CELG_OK;
  Elm* e = h->elm;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  if (e->mat) celg_mat_destroy(e->mat);
  cudaFree(e->b_d);
  cudaFree(e->x_d);
  delete e;
  h->elm = nullptr;
  return CELG_OK;
}

// Defaults of cel_elmSolverInitialization (:134-151): GMRES with restart
// 4-1 = 3, Jacobi, diagonal scaling, eps 1e-8 (absolute), iter_max 5000,
// CSR, x0 = 1 as in the solvers.
extern "C" int celg_elm_init(celg_handle* h, int n_total, int n_local, int row_low,
                             const int nnz_hint[2]) {
  if (!h || n_total < 0 || n_local < 0) return CELG_ERR_ARG;
  if (n_local != n_total || row_low != 1) return CELG_ERR_ARG;  // one sub-domain
  celg_elm_destroy(h);
  Elm* e = new Elm();
  e->n_total = n_total;
  e->n_local = n_local;
  e->row_low = row_low;
  long long hint = nnz_hint ? (long long)(nnz_hint[0] + nnz_hint[1]) * n_local : 0;
  if (hint > 0 && hint < (1LL << 31)) {
    e->rows.reserve((size_t)hint);
    e->cols.reserve((size_t)hint);
    e->vals.reserve((size_t)hint);
  }
  e->diag_idx.assign((size_t)n_local, -1);
  celg_params_default(&e->params);
  e->params.x0_mode = CELG_X0_REF_ONES;
  e->params.eps_abs = 1e-8;
  e->params.eps_rel = 0.0;
  e->params.iter_max = 5000;
  e->params.restart = 3;
  e->solver = CELG_SOLVER_GMRES;
  e->diag_scaling = 1;
  h->elm = e;
  return CELG_OK;
}

extern "C" int celg_elm_set_solver(celg_handle* h, int solver, const celg_params* p,
                                   int diag_scaling) {
  if (!h || !h->elm || !p) return CELG_ERR_STATE;
  if (solver < CELG_SOLVER_PCG || solver > CELG_SOLVER_GMRES) return CELG_ERR_ARG;
  Elm* e = h->elm;
  if (e->completed && (diag_scaling != 0) != (e->diag_scaling != 0)) return CELG_ERR_STATE;
  e->solver = solver;
  e->params = *p;
  e->diag_scaling = diag_scaling != 0;
  return CELG_OK;
}

extern "C" int celg_elm_row_start(celg_handle* h, int row) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (e->completed) return CELG_ERR_STATE;
  if (row < e->row_low || row >= e->row_low + e->n_local) return CELG_ERR_ARG;
  e->cur_row = row;
  return CELG_OK;
}

extern "C" int celg_elm_insert(celg_handle* h, int col, double value) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (e->completed || e->cur_row < 0) return CELG_ERR_STATE;
  if (col < 1 || col > e->n_total) return CELG_ERR_ARG;
  e->rows.push_back(e->cur_row);
  e->cols.push_back(col);
  e->vals.push_back(value);
  if (col == e->cur_row) e->diag_idx[(size_t)(e->cur_row - e->row_low)] = (long long)e->vals.size() - 1;
  return CELG_OK;
}

// Only the diagonal can be re-inserted; the reference stops with an error
// for off-diagonal entries (:180-184).
extern "C" int celg_elm_reinsert(celg_handle* h, int col, double value) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (e->completed || e->cur_row < 0) return CELG_ERR_STATE;
  if (col != e->cur_row) return CELG_ERR_ARG;
  const long long k = e->diag_idx[(size_t)(e->cur_row - e->row_low)];
  if (k < 0) return CELG_ERR_ARG;
  e->vals[(size_t)k] = value;
  return CELG_OK;
}

extern "C" int celg_elm_row_completed(celg_handle* h) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  return CELG_OK;
}

extern "C" int celg_elm_insert_rows(celg_handle* h, int first_row, int nrows, const int* row_ptr,
                                    const int* cols, const double* vals) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (e->completed) return CELG_ERR_STATE;
  if (nrows < 0 || !row_ptr || first_row < e->row_low ||
      first_row + nrows > e->row_low + e->n_local)
    return CELG_ERR_ARG;
  const int base = row_ptr[0];
  const long long total = (long long)row_ptr[nrows] - base;
  if (total < 0) return CELG_ERR_ARG;
  e->rows.reserve(e->rows.size() + (size_t)total);
  e->cols.reserve(e->cols.size() + (size_t)total);
  e->vals.reserve(e->vals.size() + (size_t)total);
  for (int i = 0; i < nrows; ++i) {
    const int row = first_row + i;
    if (row_ptr[i + 1] < row_ptr[i]) return CELG_ERR_ARG;
    for (int k = row_ptr[i] - base; k < row_ptr[i + 1] - base; ++k) {
      const int c = cols[k];
      if (c < 1 || c > e->n_total) return CELG_ERR_ARG;
      e->rows.push_back(row);
      e->cols.push_back(c);
      e->vals.push_back(vals[k]);
      if (c == row) e->diag_idx[(size_t)(row - e->row_low)] = (long long)e->vals.size() - 1;
    }
  }
  e->cur_row = first_row + nrows - 1;
  return CELG_OK;
}

// cel_elmSolverMatrixCompleted (:193-439) for one rank: entries sorted by
// row, then column (cel_sp_mat_format_sparse_31_sort,
// src/fspmt/cel_sp_mat_module.f90:518-585; equal keys keep insertion order)
// and the CSR row pointer (cel_sp_mat_to_csr, :430-456), both on the device;
// then Jacobi, optional diagonal scaling (:375-388 of the ELM module), JAD
// when selected.
extern "C" int celg_elm_matrix_completed(celg_handle* h) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (e->completed) return CELG_ERR_STATE;
  const size_t nnz = e->vals.size();
  if (nnz >= (size_t)1 << 31) return CELG_ERR_ARG;
  // the triplets go to the device as inserted; the stable (row, column) sort
  // and the row pointer are built there (assemble.cu)
  const size_t nz = std::max<size_t>(nnz, 1);
  int *r_d = nullptr, *c_d = nullptr;
  double* v_d = nullptr;
  cudaError_t ce = cudaMalloc(&r_d, sizeof(int) * nz);
  if (ce == cudaSuccess) ce = cudaMalloc(&c_d, sizeof(int) * nz);
  if (ce == cudaSuccess) ce = cudaMalloc(&v_d, sizeof(double) * nz);
  if (ce == cudaSuccess && nnz)
    ce = cudaMemcpyAsync(r_d, e->rows.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (ce == cudaSuccess && nnz)
    ce = cudaMemcpyAsync(c_d, e->cols.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (ce == cudaSuccess && nnz)
    ce = cudaMemcpyAsync(v_d, e->vals.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, h->stream);
  celg_mat* m = nullptr;
  int st = ce == cudaSuccess ? coo_to_mat_device(h, e->n_local, e->n_local, (int)nnz, r_d, c_d, v_d,
                                                 e->row_low, 1, &m)
                             : cuda_status(ce, "ELM triplet upload");
  cudaStreamSynchronize(h->stream);
  cudaFree(r_d);
  cudaFree(c_d);
  cudaFree(v_d);
  if (st) return st;
  st = celg_mat_jacobi(m);
  if (!st && e->diag_scaling) st = celg_mat_scale_diagonal(m);
  if (!st && e->params.fmt == CELG_FMT_JAD) st = celg_mat_to_jad(m, nullptr);
  if (!st && e->params.precision == CELG_PREC_FP32_IR) st = celg_mat_make_fp32(m);
  if (st) {
    celg_mat_destroy(m);
    return st;
  }
  e->mat = m;
  const size_t n = (size_t)std::max(1, e->n_local);
  if (cudaMalloc(&e->b_d, sizeof(double) * n) != cudaSuccess ||
      cudaMalloc(&e->x_d, sizeof(double) * n) != cudaSuccess)
    return CELG_ERR_CUDA;
  e->completed = true;
  std::vector<int>().swap(e->rows);
  std::vector<int>().swap(e->cols);
  std::vector<double>().swap(e->vals);
  return CELG_OK;
}

// cel_elmSolverDoIt (:441-651): b copied from the host, divided by sqrt|d|
// when the matrix is scaled (cel_sp_mat_distr_boundary_diag_scale), solved;
// iierr is the status (0 = converged), niter the iteration count of the
// solver (outer iterations for GMRES) and ftol its final residual norm.
extern "C" int celg_elm_doit(celg_handle* h, const double* b, int* iierr, int* niter,
                             double* ftol) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (!e->completed) return CELG_ERR_STATE;
  if (!b && e->n_local > 0) return CELG_ERR_ARG;
  cudaSetDevice(h->device);
  const size_t n = (size_t)e->n_local;
  CELG_CUDA(cudaMemcpyAsync(e->b_d, b, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  int st = CELG_OK;
  if (e->diag_scaling) st = launch_scale_vec(h, (long)n, e->b_d, e->mat->scale, e->b_d, 1);
  if (st) return st;
  celg_result res;
  std::memset(&res, 0, sizeof(res));
  celg_params p = e->params;
  int ret;
  if (e->solver == CELG_SOLVER_PCG) ret = celg_pcg_jacobi(h, e->mat, e->b_d, e->x_d, &p, &res);
  else if (e->solver == CELG_SOLVER_CG) ret = cg_solve(h, e->mat, e->b_d, e->x_d, &p, &res);
  else ret = gmres_solve(h, e->mat, e->b_d, e->x_d, &p, &res);
  e->solved = ret == CELG_OK || ret == CELG_ERR_NOCONV;
  if (iierr) *iierr = ret;
  if (niter) *niter = res.iter_done;
  if (ftol) *ftol = res.final_norm2;
  return ret;
}

extern "C" int celg_elm_redoit(celg_handle* h, const double* b, int* iierr, int* niter,
                               double* ftol) {
  return celg_elm_doit(h, b, iierr, niter, ftol);
}

extern "C" int celg_elm_collect_solution(celg_handle* h, double* x) {
  if (!h || !h->elm) return CELG_ERR_STATE;
  Elm* e = h->elm;
  if (!e->solved) return CELG_ERR_STATE;
  if (!x && e->n_local > 0) return CELG_ERR_ARG;
  CELG_CUDA(cudaMemcpyAsync(x, e->x_d, sizeof(double) * (size_t)e->n_local, cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  return CELG_OK;
}

extern "C" int celg_elm_performance(celg_handle* h, double* solve_ms, int* iters,
                                    double* bytes_per_iter) {
  if (!h) return CELG_ERR_ARG;
  if (solve_ms) *solve_ms = h->last_ms;
  if (iters) *iters = h->last_iters;
  if (bytes_per_iter) *bytes_per_iter = h->last_bytes_per_iter;
  return CELG_OK;
}
