// blockjacobi.cu -- block-Jacobi preconditioner: set-up, standalone apply and
// the PCG sweeps that use it.
//
// Set-up (cel_prec_build_diagonal + cel_prec_build_diagonal_inv,
// src/fspmtdistr/cel_prec_module.f90:27-339, in their intended form -- the
// reference's routines are never called and index every block after the
// first out of range): rows are cut into blocks of bs from row 0 (the last
// one may be shorter); one thread per block extracts the dense block from its
// rows (entries scanned in stored order, stopping at the first column right
// of the block; the last write to a position wins), factors it by Doolittle LU
// without pivoting and forms the inverse column by column with a forward and
// a back substitution, in the reference's operation order.  The inverse is
// stored as n x bs rows (row i holds row i - b0 of its block's inverse).
//
// Apply (cel_fop_block_jacobi_vec_mult, src/fop/cel_fop_block_jacobi_module.f90:
// 29-190, with r(j) where the reference's general case reads r(i)):
// z_i = r_b0 inv_i0 + r_b0+1 inv_i1 + ..., left to right.  Inside the PCG
// sweeps bs divides 32, so the rows of a block are consecutive lanes of one
// warp and the r values of the block are exchanged with warp shuffles.
#include <algorithm>

#include "pcg_internal.cuh"

namespace celg {

template <int BS>
__global__ void bj_setup_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const double* __restrict__ v, double* __restrict__ inv, int* bad) {
  const long nblk = ((long)n + BS - 1) / BS;
  for (long blk = blockIdx.x * (long)blockDim.x + threadIdx.x; blk < nblk;
       blk += (long)gridDim.x * blockDim.x) {
    const long b0 = blk * BS;
    const int nb = (int)min((long)BS, (long)n - b0);
    double a[BS][BS], L[BS][BS], c[BS][BS], d[BS], x[BS];
    for (int i = 0; i < BS; ++i)
      for (int j = 0; j < BS; ++j) a[i][j] = L[i][j] = c[i][j] = 0.0;
    for (int i = 0; i < nb; ++i) {
      const long row = b0 + i;
      for (int k = rp[row]; k < rp[row + 1]; ++k) {
        const long col = ci[k];
        if (col < b0) continue;
        if (col >= b0 + nb) break;
        a[i][col - b0] = v[k];
      }
    }
    if (nb == 1) {
      c[0][0] = 1.0 / a[0][0];
    } else {
      for (int k = 0; k < nb - 1; ++k)
        for (int i = k + 1; i < nb; ++i) {
          const double coeff = a[i][k] / a[k][k];
          L[i][k] = coeff;
          for (int j = k + 1; j < nb; ++j) a[i][j] = __dsub_rn(a[i][j], dmul(coeff, a[k][j]));
        }
      for (int k = 0; k < nb; ++k) {
        d[0] = k == 0 ? 1.0 : 0.0;
        for (int i = 1; i < nb; ++i) {
          d[i] = i == k ? 1.0 : 0.0;
          for (int j = 0; j < i; ++j) d[i] = __dsub_rn(d[i], dmul(L[i][j], d[j]));
        }
        x[nb - 1] = d[nb - 1] / a[nb - 1][nb - 1];
        for (int i = nb - 2; i >= 0; --i) {
          x[i] = d[i];
          for (int j = nb - 1; j > i; --j) x[i] = __dsub_rn(x[i], dmul(a[i][j], x[j]));
          x[i] = x[i] / a[i][i];
        }
        for (int i = 0; i < nb; ++i) c[i][k] = x[i];
      }
    }
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < BS; ++j) {
        const double e = j < nb ? c[i][j] : 0.0;
        if (!isfinite(e)) atomicExch(bad, 1);
        inv[(b0 + i) * BS + j] = e;
      }
  }
}

// z_i of row i from the block's r values fetched from global memory
__global__ void bj_apply_kernel(long n, int bs, const double* __restrict__ inv,
                                const double* __restrict__ r, double* __restrict__ z) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long b0 = i - i % bs;
    const int nb = (int)min((long)bs, n - b0);
    const double* row = inv + i * bs;
    double s = dmul(r[b0], row[0]);
    for (int j = 1; j < nb; ++j) s = dadd(s, dmul(r[b0 + j], row[j]));
    z[i] = s;
  }
}

// z_i for row i (lane `lane`, value ri) with the block's r values taken from
// the neighbouring lanes; every lane of the warp must call it.
template <int BS>
__device__ __forceinline__ double bj_row(long i, long n, double ri, const double* __restrict__ inv) {
  const int lane = threadIdx.x & 31;
  const int l0 = lane & ~(BS - 1);
  const long b0 = i - (i & (BS - 1));
  const int nb = (int)min((long)BS, n - b0);
  const bool valid = i < n;
  double w[BS];
#pragma unroll
  for (int j = 0; j < BS; ++j) w[j] = (valid && j < nb) ? __ldg(inv + i * BS + j) : 0.0;
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < BS; ++j) {
    const double rj = __shfl_sync(0xffffffffu, ri, l0 + j);
    if (j < nb) s = j == 0 ? dmul(rj, w[0]) : dadd(s, dmul(rj, w[j]));
  }
  return s;
}

// set-up tail: z = M r, p = z, alpha = r.z, ||r|| (r already holds b - A x0)
template <int BS>
struct OpInitBJ {
  static constexpr int NRED = 2;
  static constexpr bool kAllLanes = true;
  struct Regs { double r; };
  const double* r;
  double* p;
  const double* inv;
  long n;
  PcgArgs a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.r = i < n ? r[i] : 0.0; }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const double z = bj_row<BS>(i, n, g.r, inv);
    if (i < n) {
      p[i] = z;
      acc[0] = dadd(acc[0], dmul(g.r, z));
      acc[1] = dadd(acc[1], dmul(g.r, g.r));
    }
  }
  __device__ void finish(double* tot) const { init_finish(a, tot[0], tot[1]); }
};

// K2: x += sigma p; r += (-sigma) v; z = M r (stored); r.z, r.r; scalars and test
template <int BS>
struct OpUpdateBJ {
  static constexpr int NRED = 2;
  static constexpr bool kAllLanes = true;
  struct Regs { double x, r, p, v; };
  double* x;
  double* r;
  double* z;
  const double* p;
  const double* v;
  const double* inv;
  long n;
  PcgArgs a;
  double sg;
  __device__ bool prepare() {
    if (*(volatile int*)&a.st->active == 0) {
      if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(a.cond, 0);
      return false;
    }
    sg = a.st->sigma;
    return true;
  }
  __device__ void load(long i, Regs& g) const {
    if (i < n) {
      g.x = x[i];
      g.r = r[i];
      g.p = __ldg(p + i);
      g.v = __ldg(v + i);
    } else {
      g.x = g.r = g.p = g.v = 0.0;
    }
  }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const double ri = dadd(g.r, dmul(-sg, g.v));
    const double zi = bj_row<BS>(i, n, ri, inv);
    if (i < n) {
      x[i] = dadd(g.x, dmul(sg, g.p));
      r[i] = ri;
      z[i] = zi;
      acc[0] = dadd(acc[0], dmul(ri, zi));
      acc[1] = dadd(acc[1], dmul(ri, ri));
    }
  }
  __device__ void finish(double* tot) const {
    PcgState* st = a.st;
    st->rz = tot[0];
    st->beta = tot[0] / st->alpha;
    st->alpha = tot[0];
    st->norm = sqrt(tot[1]);
    st->iter += 1;
    if (a.hist && st->iter < a.hist_cap) a.hist[st->iter] = st->norm;
    st->hist_len = st->iter + 1;
    st->active = pcg_go(st, a.iter_max, a.errw);
    set_cond(a.cond, st->active);
  }
};

// K3: p = beta p + z
struct OpDirectionZ {
  static constexpr int NRED = 0;
  struct Regs { double p, z; };
  double* p;
  const double* z;
  PcgArgs a;
  double bt;
  __device__ bool prepare() {
    if (*(volatile int*)&a.st->active == 0) return false;
    bt = a.st->beta;
    return true;
  }
  __device__ void load(long i, Regs& g) const { g.p = p[i]; g.z = __ldg(z + i); }
  __device__ void compute(long i, Regs& g, double*) const { p[i] = dadd(dmul(bt, g.p), g.z); }
  __device__ void finish(double*) const {}
};

// r = b - (0 + A x), no reduction (the block-Jacobi set-up's first sweep)
struct EpiResidStore {
  static constexpr int NRED = 0;
  const double* b;
  double* r;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double*) const { r[i] = __dsub_rn(b[i], dadd(0.0, s)); }
  __device__ void finish(double*) const {}
};

template <template <int> class Op, class... Args>
static int launch_bs(celg_handle* h, long n, int bs, Args&&... args) {
  switch (bs) {
    case 1: return launch_tile(h, n, Op<1>{args...});
    case 2: return launch_tile(h, n, Op<2>{args...});
    case 4: return launch_tile(h, n, Op<4>{args...});
    case 8: return launch_tile(h, n, Op<8>{args...});
    case 16: return launch_tile(h, n, Op<16>{args...});
    case 32: return launch_tile(h, n, Op<32>{args...});
    default: return CELG_ERR_ARG;
  }
}

int bj_pcg_setup_tail(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a) {
  const long n = B.A->n;
  int st = launch_csr<double>(h, *B.A, B.vals, B.x, EpiResidStore{B.b, B.r});
  if (!st) st = launch_bs<OpInitBJ>(h, n, B.bs, (const double*)B.r, B.p, B.bj, n, a);
  return st;
}

int bj_pcg_update(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a) {
  const long n = B.A->n;
  return launch_bs<OpUpdateBJ>(h, n, B.bs, B.x, B.r, B.z, (const double*)B.p, (const double*)B.v,
                               B.bj, n, a, 0.0);
}

int bj_pcg_direction(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a) {
  return launch_tile(h, B.A->n, OpDirectionZ{B.p, B.z, a, 0.0});
}

static bool bs_ok(int bs) { return bs == 1 || bs == 2 || bs == 4 || bs == 8 || bs == 16 || bs == 32; }

}  // namespace celg

using namespace celg;

extern "C" int celg_mat_block_jacobi(celg_mat* m, int block_size) {
  if (!m || !bs_ok(block_size) || m->csr.ncols != m->csr.n) return CELG_ERR_ARG;
  celg_handle* h = m->h;
  CELG_CUDA(cudaSetDevice(h->device));
  const int n = m->csr.n;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  graph_cache_drop_matrix(h, m);
  cudaFree(m->bjinv);
  m->bjinv = nullptr;
  m->bj_bs = 0;
  CELG_CUDA(cudaMalloc(&m->bjinv, sizeof(double) * (size_t)std::max(1, n) * block_size));
  int* bad = h->err_d + 2;
  CELG_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
  const long nblk = ((long)n + block_size - 1) / block_size;
  const int grid = (int)std::max(1L, std::min((nblk + 127) / 128, (long)h->sms * 16));
  if (n > 0) {
    switch (block_size) {
      case 1: bj_setup_kernel<1><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
      case 2: bj_setup_kernel<2><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
      case 4: bj_setup_kernel<4><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
      case 8: bj_setup_kernel<8><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
      case 16: bj_setup_kernel<16><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
      default: bj_setup_kernel<32><<<grid, 128, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, m->bjinv, bad); break;
    }
    CELG_CUDA(cudaGetLastError());
  }
  int hb = 0;
  CELG_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  m->bj_bs = block_size;
  return hb ? CELG_ERR_BREAKDOWN : CELG_OK;
}

extern "C" int celg_mat_get_block_jacobi(const celg_mat* m, double* inv_host) {
  if (!m || !inv_host) return CELG_ERR_ARG;
  if (!m->bjinv) return CELG_ERR_STATE;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  if (m->csr.n)
    CELG_CUDA(cudaMemcpy(inv_host, m->bjinv, sizeof(double) * (size_t)m->csr.n * m->bj_bs,
                         cudaMemcpyDeviceToHost));
  return CELG_OK;
}

extern "C" int celg_block_jacobi_apply(celg_handle* h, const celg_mat* m, const double* r_d,
                                       double* z_d) {
  if (!h || !m || (m->csr.n > 0 && (!r_d || !z_d))) return CELG_ERR_ARG;
  if (!m->bjinv) return CELG_ERR_STATE;
  CELG_CUDA(cudaSetDevice(h->device));
  const long n = m->csr.n;
  if (n == 0) return CELG_OK;
  const int grid = (int)std::max(1L, std::min((n + 255) / 256, (long)h->sms * 16));
  bj_apply_kernel<<<grid, 256, 0, h->stream>>>(n, m->bj_bs, m->bjinv, r_d, z_d);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}
