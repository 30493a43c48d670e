// blas1.cu -- vector operators of the ABI (dot, norm, axpy, xpby, Jacobi
// multiply), matrix set-up kernels (diagonal, Jacobi, row scaling, FP32
// copy) and the handle's scratch management.
#include <algorithm>
#include <cmath>

#include "tile_kernels.cuh"

namespace celg {

long ntiles_of(long n) { return (n + kTile - 1) / kTile; }

int grid_for_tiles(celg_handle* h, long ntiles, int blocks_per_sm) {
  return (int)std::max(1L, std::min(ntiles, (long)h->sms * blocks_per_sm));
}

int ensure_partials(celg_handle* h, long ntiles, int nred) {
  const size_t need = (size_t)std::max(1L, ntiles) * (size_t)std::max(1, nred);
  if (need <= h->partials_cap) return CELG_OK;
  if (h->partials) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);  // cached graphs hold the old buffer
    CELG_CUDA(cudaFree(h->partials));
    h->partials = nullptr;
  }
  const size_t cap = std::max(need, (size_t)4096);
  CELG_CUDA(cudaMalloc(&h->partials, cap * sizeof(double)));
  h->partials_cap = cap;
  return CELG_OK;
}

// ---- elementwise kernels (grid-stride) --------------------------------------

__global__ void axpy_kernel(long n, double alpha, const double* __restrict__ x, double* y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = dadd(y[i], dmul(alpha, __ldg(x + i)));
}

__global__ void xpby_kernel(long n, const double* __restrict__ x, double beta, double* y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = dadd(dmul(beta, y[i]), __ldg(x + i));
}

__global__ void mul_kernel(long n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ z) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = dmul(__ldg(a + i), __ldg(b + i));
}

__global__ void to_f32_kernel(long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// out = a / s (divide) or a * s
__global__ void scale_vec_kernel(long n, const double* __restrict__ a, const double* __restrict__ s,
                                 double* __restrict__ out, int divide) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = divide ? __ddiv_rn(a[i], s[i]) : dmul(a[i], s[i]);
}

// diagonal (last stored diagonal entry of each row wins, 0.0 if none) and
// jacobi = 1/d.  For a row-scaled matrix the stored (unscaled) diagonal is
// used instead and jacobi = sqrt|d|/d.
__global__ void jacobi_setup_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const double* __restrict__ v, const double* __restrict__ scale,
                                    double* __restrict__ diag, double* __restrict__ J) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (scale) {
      J[i] = __ddiv_rn(scale[i], diag[i]);
      continue;
    }
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == (int)i) d = v[k];
    diag[i] = d;
    J[i] = __ddiv_rn(1.0, d);
  }
}

// s = sqrt|d|; the entries of row i are divided by s_i
__global__ void row_scale_kernel(int n, const int* __restrict__ rp, double* __restrict__ v,
                                 const double* __restrict__ diag, double* __restrict__ s) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double si = sqrt(fabs(diag[i]));
    s[i] = si;
    for (int k = rp[i]; k < rp[i + 1]; ++k) v[k] = __ddiv_rn(v[k], si);
  }
}

static int ew_grid(celg_handle* h, long n) {
  return (int)std::max(1L, std::min((n + 255) / 256, (long)h->sms * 16));
}

int launch_dot(celg_handle* h, long n, const double* a, const double* b, double* out_d,
               int take_sqrt) {
  return launch_tile(h, n, OpDot{a, b, out_d, take_sqrt});
}

int launch_axpy(celg_handle* h, long n, double alpha, const double* x, double* y) {
  if (n <= 0) return CELG_OK;
  axpy_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, alpha, x, y);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_xpby(celg_handle* h, long n, const double* x, double beta, double* y) {
  if (n <= 0) return CELG_OK;
  xpby_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, x, beta, y);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_mul(celg_handle* h, long n, const double* a, const double* b, double* z) {
  if (n <= 0) return CELG_OK;
  mul_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, a, b, z);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_to_f32(celg_handle* h, long n, const double* a, float* b) {
  if (n <= 0) return CELG_OK;
  to_f32_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, a, b);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_scale_vec(celg_handle* h, long n, const double* a, const double* s, double* out,
                     int divide) {
  if (n <= 0) return CELG_OK;
  scale_vec_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, a, s, out, divide);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_jacobi_setup(celg_handle* h, celg_mat* m) {
  const int n = m->csr.n;
  if (!m->diag) CELG_CUDA(cudaMalloc(&m->diag, sizeof(double) * std::max(1, n)));
  if (!m->jacobi) CELG_CUDA(cudaMalloc(&m->jacobi, sizeof(double) * std::max(1, n)));
  if (n <= 0) return CELG_OK;
  jacobi_setup_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v,
                                                             m->scaled ? m->scale : nullptr,
                                                             m->diag, m->jacobi);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int launch_row_scale(celg_handle* h, celg_mat* m) {
  const int n = m->csr.n;
  if (!m->scale) CELG_CUDA(cudaMalloc(&m->scale, sizeof(double) * std::max(1, n)));
  if (n <= 0) return CELG_OK;
  row_scale_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, m->csr.rp, m->csr.v, m->diag, m->scale);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

}  // namespace celg
