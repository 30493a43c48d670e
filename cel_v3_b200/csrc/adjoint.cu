// adjoint.cu -- gradients of a Jacobi-PCG solve.
//
// For x = A^{-1} b with A symmetric and a loss L(x) with g = dL/dx:
//   A lambda = g                       (a second Jacobi-PCG: A^T = A)
//   dL/db    = lambda
//   dL/dA_ij = -lambda_i x_j           on every stored entry (i, j)
// For the 7-point diffusion operator with one coefficient k_f per face
// (A_ii = sum of the cell's faces, A_ij = -k_f), contracting dL/dA with
// dA/dk_f gives
//   interior face between cells i and j:  dL/dk_f = -(lambda_i - lambda_j)(x_i - x_j)
//   Dirichlet boundary face of cell i:    dL/dk_f = -(lambda_i x_i)
// computed directly from lambda and x by celg_diffusion7_face_grad.  Face
// arrays are x-fastest with shapes (nz, ny, nx+1), (nz, ny+1, nx),
// (nz+1, ny, nx) as in cel_v3_b200/synth.py.
#include <algorithm>

#include "pcg_internal.cuh"

namespace celg {

__global__ void pattern_grad_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const double* __restrict__ lambda, const double* __restrict__ x,
                                    double* __restrict__ g) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double li = lambda[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) g[k] = -dmul(li, __ldg(x + ci[k]));
  }
}

// Faces along one axis, laid out as [outer][a = 0..na][inner]: face a lies
// between cells a-1 and a of that axis (a = 0 and a = na are the Dirichlet
// faces of cells 0 and na-1); the cell at position a is
// outer*na*inner + a*inner + inner_index.
__global__ void face_grad_kernel(long nfaces, int na, long inner,
                                 const double* __restrict__ lambda, const double* __restrict__ x,
                                 double* __restrict__ gk) {
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < nfaces; f += (long)gridDim.x * blockDim.x) {
    const long in = f % inner;
    const long a = (f / inner) % (na + 1);
    const long outer = f / (inner * (na + 1));
    const long base = outer * (long)na * inner + in;
    double gval;
    if (a == 0) {
      const long c = base;
      gval = -dmul(lambda[c], x[c]);
    } else if (a == na) {
      const long c = base + (na - 1) * inner;
      gval = -dmul(lambda[c], x[c]);
    } else {
      const long ci_ = base + (a - 1) * inner, cj = base + a * inner;
      gval = -dmul(__dsub_rn(lambda[ci_], lambda[cj]), __dsub_rn(x[ci_], x[cj]));
    }
    gk[f] = gval;
  }
}

}  // namespace celg

using namespace celg;

extern "C" int celg_pcg_adjoint(celg_handle* h, celg_mat* m, const double* x_d, const double* g_d,
                                double* lambda_d, double* grad_vals_d, const celg_params* p,
                                celg_result* res) {
  if (!h || !m || !p || m->h != h || m->csr.ncols != m->csr.n) return CELG_ERR_ARG;
  if (m->csr.n > 0 && (!x_d || !g_d || !lambda_d)) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  CELG_CUDA(cudaSetDevice(h->device));
  celg_params q = *p;
  q.precision = CELG_PREC_FP64;
  const int ret = pcg_solve(h, m, g_d, lambda_d, &q, res);
  if (ret != CELG_OK && ret != CELG_ERR_NOCONV) return ret;
  if (grad_vals_d && m->csr.n > 0) {
    const int grid = (int)std::max(1L, std::min(((long)m->csr.n + 255) / 256, (long)h->sms * 16));
    pattern_grad_kernel<<<grid, 256, 0, h->stream>>>(m->csr.n, m->csr.rp, m->csr.ci, lambda_d, x_d,
                                                     grad_vals_d);
    CELG_CUDA(cudaGetLastError());
    CELG_CUDA(cudaStreamSynchronize(h->stream));
  }
  return ret;
}

extern "C" int celg_diffusion7_face_grad(celg_handle* h, int nx, int ny, int nz,
                                         const double* lambda_d, const double* x_d, double* gkx_d,
                                         double* gky_d, double* gkz_d) {
  if (!h || nx <= 0 || ny <= 0 || nz <= 0 || !lambda_d || !x_d || !gkx_d || !gky_d || !gkz_d)
    return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(h->device));
  const long NX = nx, NY = ny, NZ = nz;
  struct Axis { long nfaces; int na; long inner; double* g; };
  // x-faces: (nz, ny, nx+1): inner = 1 (a is fastest), outer = z*ny + y
  // y-faces: (nz, ny+1, nx): inner = nx, outer = z
  // z-faces: (nz+1, ny, nx): inner = nx*ny, outer = 0
  const Axis axes[3] = {{NZ * NY * (NX + 1), nx, 1, gkx_d},
                        {NZ * (NY + 1) * NX, ny, NX, gky_d},
                        {(NZ + 1) * NY * NX, nz, NX * NY, gkz_d}};
  for (const Axis& a : axes) {
    const int grid = (int)std::max(1L, std::min((a.nfaces + 255) / 256, (long)h->sms * 16));
    face_grad_kernel<<<grid, 256, 0, h->stream>>>(a.nfaces, a.na, a.inner, lambda_d, x_d, a.g);
    CELG_CUDA(cudaGetLastError());
  }
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  return CELG_OK;
}
