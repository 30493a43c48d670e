// dist.cu -- the local sweeps of a Jacobi-PCG solve whose rows are split into
// blocks over ranks (one GPU each), with the caller running the exchange
// steps between them.
//
// The multi-process path of cel_cgalg_jacobi (src/fcgalg/cel_cgalg_module.f90:
// 178-305) does, per iteration, a halo exchange of p before the SpMV
// (src/fspmtdistr/cel_sp_mat_distr_vec_module.f90:265-724) and one
// MPI_Allreduce per global scalar (src/fop/cel_fop_vec_distr_module.f90:
// 419-832).  Here each rank holds its rows with halo columns appended after
// the local ones (celg_mat_from_csr_ext), and the phases below are stream-
// ordered kernels that read the all-reduced scalars from a small device
// buffer: no host synchronisation inside the loop, so a caller can queue the
// collectives (NCCL, or MPI on device memory) on the same stream and capture
// whole iterations in a CUDA graph.
//
// Exchange buffer: CELG_DIST_NEXCH doubles at the start of the state.  Every
// phase that produces partial sums overwrites all of them (its own sums, 0
// elsewhere; the last one is this rank's error flag), so the caller's rule is
// uniform: after begin, init, ap (or ap_boundary), update and verify,
// sum-all-reduce the whole buffer.  ap_interior runs the rows that read no
// halo value ahead of the halo's arrival and writes no exchange value, except
// for a block that reads no halo value at all: its ap_interior is the whole
// one-launch ap phase (exchange values included) and ap_boundary does
// nothing, so the caller's rule stays the same (all-reduce after
// ap_boundary).  The scalars of the recurrence are computed from the reduced
// values identically on every rank, so every rank takes the same number of
// steps.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pcg_internal.cuh"

namespace celg {

struct DistState {
  double xch[CELG_DIST_NEXCH];  // [b.b | r.z | r.r | p.v | error flag]
  double alpha, sigma, beta, norm, bnorm, eps;
  int iter, active, err, hist_len;
};
static_assert(sizeof(DistState) <= CELG_DIST_STATE_BYTES, "state buffer too small");

enum { X_BB = 0, X_RZ = 1, X_RR = 2, X_PV = 3, X_ERR = 4 };

struct DistArgs {
  DistState* st;
  double* hist;
  int hist_cap;
  int iter_max;
  const int* errw;  // this rank's device error word (bounded waits)
};

__device__ __forceinline__ void xch_store(DistState* st, const DistArgs& a, double s0, double s1,
                                          double s2, double s3) {
  st->xch[X_BB] = s0;
  st->xch[X_RZ] = s1;
  st->xch[X_RR] = s2;
  st->xch[X_PV] = s3;
  st->xch[X_ERR] = (st->err != 0 || *(volatile const int*)a.errw != 0) ? 1.0 : 0.0;
}

__device__ __forceinline__ int dist_go(const DistState* st, int iter_max) {
  return (st->err == 0 && st->iter < iter_max && fabs(st->alpha) > kRealSmall &&
          st->norm > st->eps)
             ? 1
             : 0;
}

// begin: x0 on the local rows, local b.b
struct DOpPre {
  static constexpr int NRED = 1;
  struct Regs { double b; };
  const double* b;
  double* x;
  int x0_mode;
  DistArgs a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); }
  __device__ void compute(long i, Regs& g, double* acc) const {
    if (x0_mode == CELG_X0_REF_ONES) x[i] = 1.0;
    else if (x0_mode == CELG_X0_ZERO) x[i] = 0.0;
    acc[0] = dadd(acc[0], dmul(g.b, g.b));
  }
  __device__ void finish(double* tot) const {
    DistState* st = a.st;
    st->err = 0;
    st->iter = 0;
    st->active = 1;
    st->alpha = st->sigma = st->beta = st->norm = 0.0;
    xch_store(st, a, tot[0], 0.0, 0.0, 0.0);
  }
};

// init (after the b.b reduction and the halo of x): r = b - A x, p = J r,
// local r.p and r.r; ||b|| and eps from the reduced b.b
struct DEpiInit {
  static constexpr int NRED = 2;
  const double* b;
  double* r;
  double* p;
  const double* J;
  double eps_abs, eps_rel;
  DistArgs a;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    r[i] = ri;
    const double z = dmul(ri, J[i]);
    p[i] = z;
    acc[0] = dadd(acc[0], dmul(ri, z));
    acc[1] = dadd(acc[1], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const {
    DistState* st = a.st;
    st->bnorm = sqrt(st->xch[X_BB]);
    double e = eps_abs;
    if (eps_rel > 0.0 && eps_rel * st->bnorm > e) e = eps_rel * st->bnorm;
    st->eps = e;
    if (st->xch[X_ERR] != 0.0) st->err = kErrTimeout;
    xch_store(st, a, 0.0, tot[0], tot[1], 0.0);
  }
};

// start (after the r.p / r.r reduction): alpha, ||r||, the first test
__global__ void dist_start_kernel(DistArgs a) {
  DistState* st = a.st;
  st->alpha = st->xch[X_RZ];
  st->norm = sqrt(st->xch[X_RR]);
  if (st->xch[X_ERR] != 0.0 && st->err == 0) st->err = kErrTimeout;
  st->iter = 0;
  if (a.hist && a.hist_cap > 0) a.hist[0] = st->norm;
  st->hist_len = 1;
  st->active = dist_go(st, a.iter_max);
}

// ap (after the halo of p): v = 0 + A p, local p.v
struct DEpiAp {
  static constexpr int NRED = 1;
  double* v;
  const double* p;
  DistArgs a;
  __device__ bool active() const { return *(volatile int*)&a.st->active != 0; }
  __device__ void row(long i, double s, double* acc) const {
    const double vi = dadd(0.0, s);
    v[i] = vi;
    acc[0] = dadd(acc[0], dmul(vi, __ldg(p + i)));
  }
  __device__ void finish(double* tot) const { xch_store(a.st, a, 0.0, 0.0, 0.0, tot[0]); }
};

// update (after the p.v reduction): sigma = alpha / p.v;
// r += (-sigma) v; local r.z and r.r with z = J r.  x += sigma p is left to
// the direction phase, which reads p anyway: an update that ran (active, sigma
// finite) always leaves the loop active, so a direction phase follows it.
struct DOpUpdate {
  static constexpr int NRED = 2;
  struct Regs { double r, v, J; };
  double* r;
  const double* v;
  const double* J;
  DistArgs a;
  double sg;
  bool ok;
  __device__ bool prepare() {
    const DistState* st = a.st;
    if (*(volatile const int*)&st->active == 0) return false;
    sg = st->alpha / st->xch[X_PV];
    ok = isfinite(sg) && st->xch[X_ERR] == 0.0;
    return true;
  }
  // v is not read again before the next update: streamed (evict-first)
  __device__ void load(long i, Regs& g) const {
    g.r = r[i];
    g.v = __ldcs(v + i);
    g.J = __ldg(J + i);
  }
  __device__ void compute(long i, Regs& g, double* acc) const {
    if (!ok) return;
    const double ri = dadd(g.r, dmul(-sg, g.v));
    r[i] = ri;
    const double z = dmul(ri, g.J);
    acc[0] = dadd(acc[0], dmul(ri, z));
    acc[1] = dadd(acc[1], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const {
    DistState* st = a.st;
    if (!ok) {
      if (st->err == 0) st->err = st->xch[X_ERR] != 0.0 ? kErrTimeout : kErrBreakdown;
      st->active = 0;
    }
    st->sigma = sg;
    xch_store(st, a, 0.0, tot[0], tot[1], 0.0);
  }
};

// direction (after the r.z / r.r reduction): x += sigma p with the old p
// (the update phase's step); beta = r.z / alpha; p = beta p + J r; then
// alpha = r.z, ||r||, iteration count and the test (by the last CTA, after
// every CTA has read the old alpha)
struct DOpDirection {
  static constexpr int NRED = 0;
  static constexpr bool kFinishAlways = true;
  struct Regs { double p, r, J, x; };
  double* p;
  const double* r;
  const double* J;
  double* x;
  DistArgs a;
  double bt, sg;
  __device__ bool prepare() {
    const DistState* st = a.st;
    if (*(volatile const int*)&st->active == 0) return false;
    bt = st->xch[X_RZ] / st->alpha;
    sg = st->sigma;
    return true;
  }
  // r, J and x are streamed (evict-first), so that L2 keeps the new p for
  // the next SpMV
  __device__ void load(long i, Regs& g) const {
    g.p = p[i];
    g.r = __ldcs(r + i);
    g.J = __ldcs(J + i);
    g.x = __ldcs(x + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    __stcs(x + i, dadd(g.x, dmul(sg, g.p)));
    p[i] = dadd(dmul(bt, g.p), dmul(g.r, g.J));
  }
  __device__ void finish(double*) const {
    DistState* st = a.st;
    if (st->xch[X_ERR] != 0.0 && st->err == 0) st->err = kErrTimeout;
    st->beta = bt;
    st->alpha = st->xch[X_RZ];
    st->norm = sqrt(st->xch[X_RR]);
    st->iter += 1;
    if (a.hist && st->iter < a.hist_cap) a.hist[st->iter] = st->norm;
    st->hist_len = st->iter + 1;
    st->active = dist_go(st, a.iter_max);
  }
};

// Tiles whose rows read a halo column (a column index >= n): flags[t] = 1.
__global__ void halo_tile_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                 int* __restrict__ flags) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    bool halo = false;
    for (int k = rp[i], e = rp[i + 1]; k < e; ++k) halo = halo || ci[k] >= n;
    if (halo) flags[i / kTile] = 1;
  }
}

// verify (after the halo of x): local ||b - A x||^2
struct DEpiVerify {
  static constexpr int NRED = 1;
  const double* b;
  DistArgs a;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const { xch_store(a.st, a, tot[0], 0.0, 0.0, 0.0); }
};

}  // namespace celg

using namespace celg;

struct celg_dist {
  celg_handle* h = nullptr;
  celg_mat* m = nullptr;
  DistState* st = nullptr;
  bool own_state = false;
  double* hist = nullptr;
  int hist_cap = 0;
  celg_params p{};
  DistState* host = nullptr;  // pinned mirror for poll/result
  // interior tiles [win_lo, win_hi): the longest run of tiles that read no
  // halo value; part: the tile partials of the split SpMV phase
  long win_lo = 0, win_hi = 0;
  double* part = nullptr;
  // work vectors and exchange plan of celg_dist_pcg_solve (dist_solve.cu)
  void* solve = nullptr;
  DistArgs args() const { return DistArgs{st, hist, hist_cap, p.iter_max, h->err_d}; }
};

namespace celg {
int dist_internals(celg_dist* d, celg_handle** h, int* n, int* ncols, void*** solve_slot) {
  if (!d || !d->h || !d->m) return CELG_ERR_ARG;
  *h = d->h;
  *n = d->m->csr.n;
  *ncols = d->m->csr.ncols;
  *solve_slot = &d->solve;
  return CELG_OK;
}
}  // namespace celg

static int dist_check(const celg_dist* d) {
  if (!d || !d->h || !d->m) return CELG_ERR_ARG;
  return CELG_OK;
}

// SpMV phase of the block: row patterns or 1-byte column offsets when the
// block has them (same values in the same order, so the same sums), else
// int32 columns.
template <class Epi>
static int dist_csr(celg_dist* d, const double* x, const Epi& epi, const TileWindow* win = nullptr) {
  const CsrDev& A = d->m->csr;
  bool done = false;
  const int st = launch_csr_compact<double>(d->h, A, A.v, x, epi, win, 0, &done);
  if (done) return st;
  return launch_csr_ct<double, int>(d->h, A, A.v, A.ci, A.cap, x, epi, win);
}

// The interior window of the block and the partials of the split SpMV.
static int dist_find_interior(celg_dist* d) {
  celg_handle* h = d->h;
  const CsrDev& A = d->m->csr;
  const long nt = ntiles_of(A.n);
  if (nt == 0) return CELG_OK;
  CELG_CUDA(cudaMalloc(&d->part, sizeof(double) * (size_t)nt));
  int* flags = nullptr;
  CELG_CUDA(cudaMalloc(&flags, sizeof(int) * (size_t)nt));
  std::vector<int> f((size_t)nt);
  cudaError_t e = cudaMemsetAsync(flags, 0, sizeof(int) * (size_t)nt, h->stream);
  if (e == cudaSuccess) {
    const int grid = (int)std::max(1L, std::min(((long)A.n + 255) / 256, (long)h->sms * 16));
    halo_tile_kernel<<<grid, 256, 0, h->stream>>>(A.n, A.rp, A.ci, flags);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(f.data(), flags, sizeof(int) * (size_t)nt, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(flags);
  if (e != cudaSuccess) return cuda_status(e, "celg_dist_create");
  for (long t = 0; t < nt;) {
    if (f[t]) { ++t; continue; }
    long u = t;
    while (u < nt && !f[u]) ++u;
    if (u - t > d->win_hi - d->win_lo) {
      d->win_lo = t;
      d->win_hi = u;
    }
    t = u;
  }
  return CELG_OK;
}

extern "C" int celg_dist_create(celg_handle* h, celg_mat* m, const celg_params* p, void* state_d,
                                double* hist_d, int hist_cap, celg_dist** out) {
  if (!h || !m || !p || !out || m->h != h || hist_cap < 0 || (hist_cap > 0 && !hist_d))
    return CELG_ERR_ARG;
  if (p->x0_mode < CELG_X0_REF_ONES || p->x0_mode > CELG_X0_USER || p->iter_max < 0)
    return CELG_ERR_ARG;
  if (p->fmt != CELG_FMT_CSR || p->precision != CELG_PREC_FP64 || p->precond != CELG_PRECOND_JACOBI)
    return CELG_ERR_ARG;
  if (m->csr.n <= 0) return CELG_ERR_ARG;  // every rank holds at least one row
  if (!m->jacobi) return CELG_ERR_STATE;
  if (state_d && (reinterpret_cast<uintptr_t>(state_d) & 15)) return CELG_ERR_ARG;
  *out = nullptr;
  CELG_CUDA(cudaSetDevice(h->device));
  // 1-byte column offsets for the block's SpMV phases when its columns (halo
  // included) use at most 256 distinct offsets col - row
  if (const int st = ensure_offset_dict(h, m)) return st;
  celg_dist* d = new celg_dist();
  d->h = h;
  d->m = m;
  d->p = *p;
  d->hist = hist_cap > 0 ? hist_d : nullptr;
  d->hist_cap = hist_cap;
  cudaError_t e = cudaSuccess;
  if (state_d) {
    d->st = static_cast<DistState*>(state_d);
  } else {
    e = cudaMalloc(&d->st, CELG_DIST_STATE_BYTES);
    d->own_state = e == cudaSuccess;
  }
  if (e == cudaSuccess) e = cudaMallocHost(&d->host, sizeof(DistState));
  if (e == cudaSuccess) e = cudaMemsetAsync(d->st, 0, sizeof(DistState), h->stream);
  if (e != cudaSuccess) {
    if (d->own_state) cudaFree(d->st);
    if (d->host) cudaFreeHost(d->host);
    delete d;
    return cuda_status(e, "celg_dist_create");
  }
  if (const int st = dist_find_interior(d)) {
    celg_dist_destroy(d);
    return st;
  }
  *out = d;
  return CELG_OK;
}

extern "C" int celg_dist_destroy(celg_dist* d) {
  if (!d) return CELG_OK;
  cudaSetDevice(d->h->device);
  cudaStreamSynchronize(d->h->stream);
  if (d->own_state) cudaFree(d->st);
  cudaFreeHost(d->host);
  cudaFree(d->part);
  dist_solve_free(d->solve);
  delete d;
  return CELG_OK;
}

extern "C" int celg_dist_exchange_buffer(celg_dist* d, double** xch_d) {
  if (dist_check(d) || !xch_d) return CELG_ERR_ARG;
  *xch_d = d->st->xch;
  return CELG_OK;
}

extern "C" int celg_dist_pcg_begin(celg_dist* d, const double* b_d, double* x_ext_d) {
  if (dist_check(d) || !b_d || !x_ext_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  return launch_tile(d->h, d->m->csr.n, DOpPre{b_d, x_ext_d, d->p.x0_mode, d->args()});
}

extern "C" int celg_dist_pcg_init(celg_dist* d, const double* b_d, const double* x_ext_d,
                                  double* r_d, double* p_ext_d) {
  if (dist_check(d) || !b_d || !x_ext_d || !r_d || !p_ext_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  DEpiInit epi{b_d, r_d, p_ext_d, d->m->jacobi, d->p.eps_abs, d->p.eps_rel, d->args()};
  return dist_csr(d, x_ext_d, epi);
}

extern "C" int celg_dist_pcg_start(celg_dist* d) {
  if (dist_check(d)) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  dist_start_kernel<<<1, 1, 0, d->h->stream>>>(d->args());
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

extern "C" int celg_dist_pcg_ap(celg_dist* d, const double* p_ext_d, double* v_d) {
  if (dist_check(d) || !p_ext_d || !v_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  return dist_csr(d, p_ext_d, DEpiAp{v_d, p_ext_d, d->args()});
}

// A block that reads no halo value (every tile interior) runs the whole
// one-launch phase as its interior half and nothing as its boundary half.
static bool dist_all_interior(const celg_dist* d) {
  return d->win_lo == 0 && d->win_hi == ntiles_of(d->m->csr.n);
}

extern "C" int celg_dist_pcg_ap_interior(celg_dist* d, const double* p_ext_d, double* v_d) {
  if (dist_check(d) || !p_ext_d || !v_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  if (dist_all_interior(d)) return dist_csr(d, p_ext_d, DEpiAp{v_d, p_ext_d, d->args()});
  const TileWindow w{d->win_lo, d->win_hi, true, d->part, ntiles_of(d->m->csr.n)};
  return dist_csr(d, p_ext_d, DEpiAp{v_d, p_ext_d, d->args()}, &w);
}

extern "C" int celg_dist_pcg_ap_boundary(celg_dist* d, const double* p_ext_d, double* v_d) {
  if (dist_check(d) || !p_ext_d || !v_d) return CELG_ERR_ARG;
  if (dist_all_interior(d)) return CELG_OK;
  CELG_CUDA(cudaSetDevice(d->h->device));
  const TileWindow w{d->win_lo, d->win_hi, false, d->part, ntiles_of(d->m->csr.n)};
  return dist_csr(d, p_ext_d, DEpiAp{v_d, p_ext_d, d->args()}, &w);
}

extern "C" int celg_dist_interior_rows(celg_dist* d, int* row_lo, int* row_hi) {
  if (dist_check(d) || !row_lo || !row_hi) return CELG_ERR_ARG;
  const long n = d->m->csr.n;
  *row_lo = (int)std::min(n, d->win_lo * kTile);
  *row_hi = (int)std::min(n, d->win_hi * kTile);
  return CELG_OK;
}

extern "C" int celg_dist_pcg_update(celg_dist* d, double* r_d, const double* v_d) {
  if (dist_check(d) || !r_d || !v_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  DOpUpdate op{r_d, v_d, d->m->jacobi, d->args(), 0.0, true};
  return launch_tile(d->h, d->m->csr.n, op);
}

extern "C" int celg_dist_pcg_direction(celg_dist* d, double* x_ext_d, const double* r_d,
                                       double* p_ext_d) {
  if (dist_check(d) || !x_ext_d || !r_d || !p_ext_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  DOpDirection op{p_ext_d, r_d, d->m->jacobi, x_ext_d, d->args(), 0.0, 0.0};
  return launch_tile(d->h, d->m->csr.n, op);
}

extern "C" int celg_dist_pcg_verify(celg_dist* d, const double* b_d, const double* x_ext_d) {
  if (dist_check(d) || !b_d || !x_ext_d) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(d->h->device));
  return dist_csr(d, x_ext_d, DEpiVerify{b_d, d->args()});
}

static int dist_fetch(celg_dist* d) {
  CELG_CUDA(cudaSetDevice(d->h->device));
  CELG_CUDA(cudaMemcpyAsync(d->host, d->st, sizeof(DistState), cudaMemcpyDeviceToHost, d->h->stream));
  CELG_CUDA(cudaStreamSynchronize(d->h->stream));
  return CELG_OK;
}

extern "C" int celg_dist_pcg_poll(celg_dist* d, int* active, int* iter) {
  if (dist_check(d)) return CELG_ERR_ARG;
  int st = dist_fetch(d);
  if (st) return st;
  if (active) *active = d->host->active;
  if (iter) *iter = d->host->iter;
  return CELG_OK;
}

extern "C" int celg_dist_pcg_result(celg_dist* d, celg_result* res) {
  if (dist_check(d)) return CELG_ERR_ARG;
  int st = dist_fetch(d);
  if (st) return st;
  const DistState& s = *d->host;
  int ret = CELG_OK;
  if (s.err) ret = s.err;
  else if (s.xch[X_ERR] != 0.0) ret = CELG_ERR_TIMEOUT;
  else if (!(s.norm <= s.eps) && s.iter >= d->p.iter_max && std::fabs(s.alpha) > kRealSmall)
    ret = CELG_ERR_NOCONV;
  if (res) {
    res->iter_done = s.iter;
    res->final_norm2 = s.norm;
    res->bnorm = s.bnorm;
    res->verified_relres = s.bnorm > 0.0 ? std::sqrt(s.xch[X_BB]) / s.bnorm : std::sqrt(s.xch[X_BB]);
    res->err = ret;
    res->arnoldi_steps = 0;
    res->history_len = 0;
    if (res->history && res->history_cap > 0 && d->hist) {
      const int len = std::min(std::min(s.hist_len, d->hist_cap), res->history_cap);
      CELG_CUDA(cudaMemcpy(res->history, d->hist, sizeof(double) * (size_t)len, cudaMemcpyDeviceToHost));
      res->history_len = len;
    }
  }
  return ret;
}
