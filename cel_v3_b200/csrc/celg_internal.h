// celg_internal.h -- host-side objects of libcelgpu.so (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/celgpu.h"

namespace celg {

// Device copy of a CSR matrix, 0-based.  row_ptr has n+1+4 entries and
// cols/vals nnz+4 (tails filled with nnz / 0) so that the 16-byte rounded
// bulk copies of the SpMV pipeline never leave the allocation.
struct CsrDev {
  int n = 0;
  int nnz = 0;
  int ncols = 0;          // n, or more for a row block with halo columns

  int* rp = nullptr;
  int* ci = nullptr;
  double* v = nullptr;
  float* v32 = nullptr;   // FP32 copy (refinement inner solve), nnz+32
  int cap = 0;            // staged entries per 256-row sub-tile
  // column indices as 1-byte indices into a dictionary of column offsets
  // (col - row), when the matrix has at most 256 of them (FP32 copy and
  // the FP64 PCG sweeps)
  uint8_t* ci8 = nullptr; // nnz+32
  int* dict = nullptr;    // ndict offsets, ascending
  int ndict = 0;
  int cap_dict = 0;       // staging capacity with 16-entry alignment
  // row patterns (spmv_kernels.cuh, kPatLen/kPatMax): one pattern index per
  // row (n + 16 bytes) and the pattern table (npat x 8 column offsets), when
  // the dictionary's rows fit them
  uint8_t* pid = nullptr;
  int* pat = nullptr;
  int npat = 0;
};

struct JadDev {
  int mmax = -1;          // -1: not built
  int* begin = nullptr;   // mmax+1
  int* ci = nullptr;      // nnz
  double* v = nullptr;    // nnz
  int* perm = nullptr;    // n
  uint8_t* pid = nullptr; // pattern index of each permuted row (n + 16), with row patterns
};

struct PcgState;  // device scalar state of one solve (pcg_internal.cuh)

struct GraphEntry {
  std::string key;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

}  // namespace celg

struct celg_handle {
  int device = 0;
  cudaStream_t stream = nullptr;      // work stream (owned, or the caller's)
  bool own_stream = false;
  cudaStream_t cap_stream = nullptr;  // private stream used only to capture graphs
  int sms = 148;
  // reduction scratch: partials (2 rows of max tiles) and a completion ticket
  double* partials = nullptr;
  size_t partials_cap = 0;   // doubles
  unsigned* ticket = nullptr;
  int* err_d = nullptr;      // device error word (bounded waits)
  double* scal_d = nullptr;  // small device scalars for blas1 results
  double* scal_h = nullptr;  // pinned mirror
  // PCG work vectors
  double* wr = nullptr;
  double* wp = nullptr;
  double* wv = nullptr;
  double* wq = nullptr;  // second PCG direction (paired K3)
  size_t wcap = 0;           // elements
  double* wz = nullptr;      // z = M r of block-Jacobi solves (wzcap elements)
  size_t wzcap = 0;
  celg::PcgState* state_d = nullptr;
  celg::PcgState* state_h = nullptr;  // pinned
  void* ru_state_d = nullptr;         // reliable-update solver state
  void* ru_state_h = nullptr;         // pinned
  // cached solve graphs (keyed by matrix, vectors and parameters)
  std::vector<celg::GraphEntry> graphs;
  double* hist_d = nullptr;
  int hist_cap = 0;
  // host-buffer solve staging (stable pointers keep cached graphs valid)
  double* sb = nullptr;
  double* sx = nullptr;
  size_t scap = 0;
  // FP32 refinement work vectors
  float* f32 = nullptr;   // 6 vectors of f32cap floats
  size_t f32cap = 0;
  double* ir_d = nullptr; // FP64 correction / residual
  size_t ircap = 0;
  // ELM assembly state
  struct Elm* elm = nullptr;
  // concatenated systems of the last batched solve
  struct Batch* batch = nullptr;
  // work vectors and per-column state of multi-right-hand-side solves
  struct Multi* multi = nullptr;
  // GMRES(m) work space (V, Z, H) and device state, kept between solves
  double* gm_work = nullptr;
  size_t gm_cap = 0;          // doubles
  void* gm_state_d = nullptr;
  void* gm_state_h = nullptr; // pinned
  // last solve timing
  float last_ms = 0.f;
  int last_iters = 0;
  double last_bytes_per_iter = 0.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tile order of the next sweep (RedCtx::sweep bit 0)
  int sweep_rev = 0;
};

struct celg_mat {
  celg_handle* h = nullptr;
  celg::CsrDev csr;
  celg::JadDev jad;
  double* diag = nullptr;     // n
  double* jacobi = nullptr;   // n
  float* jacobi32 = nullptr;  // n
  double* scale = nullptr;    // sqrt|d| when row-scaled, else null
  double* bjinv = nullptr;    // n x bj_bs inverse diagonal blocks (block Jacobi)
  bool dict_tried = false;    // the offset dictionary was attempted (csr.ci8 set if it fits)
  int bj_bs = 0;
  bool scaled = false;
};

namespace celg {

int cuda_status(cudaError_t e, const char* what);
#define CELG_CUDA(call)                                       \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::celg::cuda_status(e_, #call); \
  } while (0)

int ensure_partials(celg_handle* h, long ntiles, int nred);
void graph_cache_clear(celg_handle* h);
void graph_cache_drop_matrix(celg_handle* h, const void* m);
int ensure_work(celg_handle* h, size_t n);
long ntiles_of(long n);
int grid_for_tiles(celg_handle* h, long ntiles, int blocks_per_sm);

// spmv.cu
int launch_spmv_csr(celg_handle* h, const CsrDev& A, const double* x, double* y, int accumulate);
int launch_spmv_csr_f32(celg_handle* h, const CsrDev& A, const float* x, float* y, int accumulate);
int launch_spmv_jad(celg_handle* h, const CsrDev& A, const JadDev& J, const double* x, double* y);
int csr_compute_cap(celg_handle* h, CsrDev& A);

// blas1.cu
int launch_dot(celg_handle* h, long n, const double* a, const double* b, double* out_d, int take_sqrt);
int launch_axpy(celg_handle* h, long n, double alpha, const double* x, double* y);
int launch_xpby(celg_handle* h, long n, const double* x, double beta, double* y);
int launch_mul(celg_handle* h, long n, const double* a, const double* b, double* z);
int launch_residual(celg_handle* h, celg_mat* m, int fmt, const double* b, const double* x,
                    double* r, double* norm_out_d);
int launch_jacobi_setup(celg_handle* h, celg_mat* m);
int launch_row_scale(celg_handle* h, celg_mat* m);
int launch_to_f32(celg_handle* h, long n, const double* a, float* b);
int launch_scale_vec(celg_handle* h, long n, const double* a, const double* s, double* out, int divide);

// pcg.cu / gmres.cu / ir.cu
int pcg_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
              celg_result* res);
int cg_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res);
int gmres_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
                celg_result* res);
int ir_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res);
int ru_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res);
int ensure_f32(celg_handle* h, size_t n);
// api.cu: matrix storage (alloc_csr leaves row_ptr/cols/vals for the caller
// to fill; finish_csr shifts to 0-based, validates and sets the staging cap)
// Build the 1-byte column offsets of the matrix once (no-op when built,
// attempted before, or the matrix has more than 256 column offsets).
int ensure_offset_dict(celg_handle* h, celg_mat* m);
// the same for any CSR array set (left unset beyond 256 distinct offsets)
int build_offset_dict_csr(celg_handle* h, CsrDev& A);
int alloc_csr(celg_mat* m, int n, int nnz, int ncols);
int finish_csr(celg_handle* h, celg_mat* m, int base);
void free_mat_arrays(celg_mat* m);
// assemble.cu: COO (device arrays, row and column bases) -> CSR matrix
int coo_to_mat_device(celg_handle* h, int n, int ncols, int nnz, const int* rows_d,
                      const int* cols_d, const double* vals_d, int row_base, int col_base,
                      celg_mat** out);
// dist.cu / dist_solve.cu: the one-call distributed solve's data on a celg_dist
int dist_internals(celg_dist* d, celg_handle** h, int* n, int* ncols, void*** solve_slot);
void dist_solve_free(void* solve);
void batch_free(::Batch* b);
void multi_free(::Multi* m);
void multi_forget_matrix(::Multi* m, const void* mat);
int multi_tuned_cfg(::Multi* m);  // the SpMM variant the tuner picked, -1 if none
int multi_tuned_cfg32(::Multi* m);  // the FP32 SpMM shape the tuner picked, -1 if none

}  // namespace celg
