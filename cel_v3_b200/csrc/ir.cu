// ir.cu -- FP64 iterative refinement around an FP32-storage Jacobi-PCG.
//
//   x = x0;  for k = 0, 1, ...:
//     r = b - A x,  ||r||            (FP64 matrix, FP64 vectors, on the GPU)
//     stop when ||r|| <= max(eps_abs, eps_rel ||b||)
//     d = PCG_fp32(A32, r/||r||)      (inner tolerance tau_k, below)
//     x = x + ||r|| d                 (FP64)
// The outer residual, update and stopping test stay in binary64, so the
// reported accuracy is the FP64-verified ||b - A x|| / ||b||.  The inner
// solve reads 8 bytes per non-zero (float value + int32 column) and float
// vectors instead of 12 bytes and doubles.
//
// Each refinement step asks its inner solve for ir_step_tolerance(||r||, eps,
// inner_eps_rel) (celg_device.cuh): never tighter than inner_eps_rel, looser
// when one or two more steps at inner_eps_rel would more than finish.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pcg_internal.cuh"

namespace celg {

// The inner system is solved for the normalised residual r / ||r|| (so that
// its scale does not meet the absolute |alpha| guard of the PCG loop or the
// FP32 range) and the correction is scaled back:
//   r32 = (float)(r * (1/||r||)),   x = x + ||r|| * (double) d32
struct OpAddF32 {
  static constexpr int NRED = 0;
  struct Regs { double x; float d; };
  double* x;
  const float* d;
  double scale;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.x = x[i]; g.d = __ldg(d + i); }
  __device__ void compute(long i, Regs& g, double*) const {
    x[i] = dadd(g.x, dmul(scale, (double)g.d));
  }
  __device__ void finish(double*) const {}
};

struct OpToF32 {
  static constexpr int NRED = 0;
  struct Regs { double r; };
  const double* r;
  float* r32;
  double inv;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.r = __ldg(r + i); }
  __device__ void compute(long i, Regs& g, double*) const { r32[i] = (float)dmul(g.r, inv); }
  __device__ void finish(double*) const {}
};

struct OpX0 {
  static constexpr int NRED = 0;
  struct Regs { int unused; };
  double* x;
  double val;
  __device__ bool prepare() { return true; }
  __device__ void load(long, Regs&) const {}
  __device__ void compute(long i, Regs&, double*) const { x[i] = val; }
  __device__ void finish(double*) const {}
};

int ensure_f32(celg_handle* h, size_t n) {
  if (n <= h->f32cap && h->f32 && h->ir_d) return CELG_OK;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  graph_cache_clear(h);
  cudaFree(h->f32);
  cudaFree(h->ir_d);
  h->f32 = nullptr;
  h->ir_d = nullptr;
  const size_t cap = std::max<size_t>(n, 1024);
  CELG_CUDA(cudaMalloc(&h->f32, sizeof(float) * cap * 6));  // 6 float vectors
  CELG_CUDA(cudaMalloc(&h->ir_d, sizeof(double) * cap));
  h->f32cap = cap;
  h->ircap = cap;
  return CELG_OK;
}

int ir_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res) {
  const long n = m->csr.n;
  if (!m->jacobi) return CELG_ERR_STATE;
  if (!m->csr.v32 || !m->jacobi32) {
    int st = celg_mat_make_fp32(m);
    if (st) return st;
  }
  int st = ensure_f32(h, (size_t)n);
  if (!st) st = ensure_partials(h, ntiles_of(n), 2);
  if (st) return st;
  if (res) res->history_len = 0;
  const size_t cap = h->f32cap;
  float* b32 = h->f32;
  float* d32 = b32 + cap;
  float* r32 = d32 + cap;
  float* p32 = r32 + cap;
  float* v32 = p32 + cap;
  float* q32 = v32 + cap;  // second direction of the paired K3
  double* r = h->ir_d;
  double* sd = h->scal_d;

  celg_params ip;
  std::memcpy(&ip, p, sizeof(ip));
  ip.x0_mode = CELG_X0_ZERO;
  ip.eps_abs = 0.0;
  const double tau = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-4;
  ip.iter_max = p->inner_iter_max > 0 ? p->inner_iter_max : 1000;

  PcgBind<float> B;
  B.A = &m->csr;
  B.vals = m->csr.v32;
  B.verify_vals = nullptr;
  B.b = b32;
  B.x = d32;
  B.r = r32;
  B.p = p32;
  B.q = q32;
  B.v = v32;
  B.J = m->jacobi32;

  cudaEvent_t e0, e1;
  CELG_CUDA(cudaEventCreate(&e0));
  CELG_CUDA(cudaEventCreate(&e1));
  cudaEventRecord(e0, h->stream);
  if (p->x0_mode != CELG_X0_USER && n > 0)
    st = launch_tile(h, n, OpX0{x, p->x0_mode == CELG_X0_REF_ONES ? 1.0 : 0.0});
  double bnorm = 0.0, rn = 0.0;
  if (!st) st = launch_dot(h, n, b, b, sd, 1);
  if (!st) {
    CELG_CUDA(cudaMemcpyAsync(h->scal_h, sd, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    bnorm = h->scal_h[0];
  }
  double tol = p->eps_abs;
  if (p->eps_rel > 0.0 && p->eps_rel * bnorm > tol) tol = p->eps_rel * bnorm;
  const int outer_max = p->outer_max > 0 ? p->outer_max : 20;
  int outer = 0, inner_total = 0, ret = CELG_ERR_NOCONV;
  while (!st) {
    st = launch_residual(h, m, CELG_FMT_CSR, b, x, r, sd);
    if (st) break;
    CELG_CUDA(cudaMemcpyAsync(h->scal_h, sd, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    rn = h->scal_h[0];
    if (res && res->history && outer < res->history_cap) {
      res->history[outer] = rn;
      res->history_len = outer + 1;
    }
    if (rn <= tol) {
      ret = CELG_OK;
      break;
    }
    if (!std::isfinite(rn)) {
      ret = CELG_ERR_BREAKDOWN;
      break;
    }
    if (outer >= outer_max) break;
    st = launch_tile(h, n, OpToF32{r, b32, 1.0 / rn});
    if (st) break;
    ip.eps_rel = ir_step_tolerance(rn, tol, tau);
    PcgState s;
    const int ist = pcg_run<float>(h, B, &ip, m, &s);
    inner_total += s.iter;
    if (ist && ist != CELG_ERR_NOCONV) {
      st = ist;
      break;
    }
    st = launch_tile(h, n, OpAddF32{x, d32, rn});
    ++outer;
  }
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&h->last_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  h->last_iters = inner_total;
  h->last_bytes_per_iter = 8.0 * m->csr.nnz + 4.0 * (n + 1) + 50.0 * n;
  if (res) {
    res->iter_done = outer;
    res->final_norm2 = rn;
    res->bnorm = bnorm;
    res->verified_relres = bnorm > 0 ? rn / bnorm : rn;
    res->err = ret;
    res->arnoldi_steps = inner_total;
  }
  return ret;
}

}  // namespace celg
