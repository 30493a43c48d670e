// spmv.cu -- standalone SpMV entry points, the staging-capacity set-up of a
// CSR matrix, and the fused residual r = b - A x with ||r||.
#include <algorithm>

#include "tile_kernels.cuh"

namespace celg {

int csr_smem_bytes(int cap, int vt_size, int ct_size, int pat_ints) {
  if (pat_ints >= 0) {
    StageLayout L(cap, vt_size, 1, true);
    return kCsrHeader + ((pat_ints * 4 + 127) & ~127) + kStages * L.bytes;
  }
  StageLayout L(cap, vt_size, ct_size);
  return kCsrHeader + (ct_size == 1 ? kDictMax * 4 : 0) + kStages * L.bytes;
}

// Largest 16-byte-rounded entry span of any 256-row sub-tile.
__global__ void subtile_span_kernel(const int* __restrict__ rp, int n, int* out) {
  const long nsub = ((long)n + kSub - 1) / kSub;
  int best = 0;
  for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < nsub;
       s += (long)gridDim.x * blockDim.x) {
    const long r0 = s * kSub;
    const long r1 = r0 + kSub < (long)n ? r0 + kSub : (long)n;
    const int a0 = rp[r0] & ~3;
    const int a1 = (rp[r1] + 3) & ~3;
    best = max(best, a1 - a0);
  }
  for (int off = 16; off >= 1; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

// Staging capacity: the largest sub-tile span if four stages of it fit two
// CTAs per SM (113 KB each), otherwise as much as four stages in one CTA
// allow; sub-tiles above the capacity are read from global memory instead.
int csr_compute_cap(celg_handle* h, CsrDev& A) {
  int* d = h->err_d + 1;  // scratch int next to the error word
  CELG_CUDA(cudaMemsetAsync(d, 0, sizeof(int), h->stream));
  if (A.n > 0) {
    const long nsub = ((long)A.n + kSub - 1) / kSub;
    const int grid = (int)std::max(1L, std::min((long)h->sms * 4, (nsub + 255) / 256));
    subtile_span_kernel<<<grid, 256, 0, h->stream>>>(A.rp, A.n, d);
    CELG_CUDA(cudaGetLastError());
  }
  int span = 0;
  CELG_CUDA(cudaMemcpyAsync(&span, d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  int cap = std::max(16, (span + 3) & ~3);
  const int two_cta = 113 * 1024, one_cta = 227 * 1024;
  if (csr_smem_bytes(cap, 8) > two_cta) {
    int lim = cap;
    while (lim > 16 && csr_smem_bytes(lim, 8) > one_cta) lim -= 64;
    cap = std::max(16, lim & ~3);
  }
  A.cap = cap;
  return CELG_OK;
}

int launch_spmv_csr(celg_handle* h, const CsrDev& A, const double* x, double* y, int accumulate) {
  EpiStore<double> epi{y, accumulate};
  return launch_csr<double>(h, A, A.v, x, epi);
}

int launch_spmv_csr_f32(celg_handle* h, const CsrDev& A, const float* x, float* y, int accumulate) {
  if (!A.v32) return CELG_ERR_STATE;
  EpiStore<float> epi{y, accumulate};
  return launch_csr<float>(h, A, A.v32, x, epi);
}

int launch_spmv_jad(celg_handle* h, const CsrDev& A, const JadDev& J, const double* x, double* y) {
  if (J.mmax < 0) return CELG_ERR_STATE;
  EpiStore<double> epi{y, 0};
  return launch_jad(h, A, J, x, epi);
}

// r = b - A x and ||r||_2 into *norm_out_d (device).  The JAD path sums rows in
// permuted order, so its norm is taken afterwards in natural row order.
int launch_residual(celg_handle* h, celg_mat* m, int fmt, const double* b, const double* x,
                    double* r, double* norm_out_d) {
  if (fmt == CELG_FMT_JAD) {
    int st = launch_spmv_jad(h, m->csr, m->jad, x, r);
    if (st) return st;
    return launch_tile(h, m->csr.n, OpResidNat{b, r, norm_out_d});
  }
  EpiResidual epi{b, r, norm_out_d};
  return launch_csr<double>(h, m->csr, m->csr.v, x, epi);
}

}  // namespace celg
