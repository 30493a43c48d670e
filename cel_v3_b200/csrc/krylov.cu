// krylov.cu -- unpreconditioned CG (cel_cgalg) and restarted GMRES(m) with
// right Jacobi preconditioning (cel_gmresalg_2jacobi).  The vector sweeps
// run on the device with the fixed-order reductions.  CG's scalar recurrence
// runs on the host; GMRES runs entirely on the device: the Hessenberg column,
// the Givens rotations, the convergence test, the back substitution and the
// restart decisions are one-thread kernels between the sweeps, in the
// reference's operation order, so that a whole solve is one CUDA graph (a
// WHILE node over restart cycles) with no host synchronisation inside.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "graph.cuh"
#include "pcg_internal.cuh"

namespace celg {

// ---- device sweeps ------------------------------------------------------------

// r = b - (0 + r); d = r   (cel_fop_vec_distr_calc_r_and_d, :54-56)
struct OpCalcRD {
  static constexpr int NRED = 0;
  struct Regs { double b, r; };
  const double* b;
  double* r;
  double* d;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); g.r = r[i]; }
  __device__ void compute(long i, Regs& g, double*) const {
    const double ri = __dsub_rn(g.b, dadd(0.0, g.r));
    r[i] = ri;
    d[i] = ri;
  }
  __device__ void finish(double*) const {}
};

// x = x + a d ; r = r + (-a) q     (cel_fop_vec_distr_scale, :862-864)
struct OpXR {
  static constexpr int NRED = 0;
  struct Regs { double x, d, r, q; };
  double* x;
  const double* d;
  double* r;
  const double* q;
  double a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const {
    g.x = x[i]; g.d = __ldg(d + i); g.r = r[i]; g.q = __ldg(q + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    x[i] = dadd(g.x, dmul(a, g.d));
    r[i] = dadd(g.r, dmul(-a, g.q));
  }
  __device__ void finish(double*) const {}
};

// v = r * inv ; z = v * J     (scale_inv :94-97 and vec_mult_distr_jacobi :364-366)
struct OpV1 {
  static constexpr int NRED = 0;
  struct Regs { double r, J; };
  const double* r;
  double* v;
  double* z;
  const double* J;
  const double* rn;   // ||r|| (device): v = r * (1 / ||r||)
  double inv = 0.0;
  __device__ bool prepare() {
    inv = 1.0 / *(volatile const double*)rn;
    return true;
  }
  __device__ void load(long i, Regs& g) const { g.r = __ldg(r + i); g.J = __ldg(J + i); }
  __device__ void compute(long i, Regs& g, double*) const {
    const double vi = dmul(g.r, inv);
    v[i] = vi;
    z[i] = dmul(vi, g.J);
  }
  __device__ void finish(double*) const {}
};

// v_{j+1} = w / h ; z_{j+1} = v_{j+1} * J   (:774-777, :683)
struct OpVNext {
  static constexpr int NRED = 0;
  struct Regs { double w, J; };
  const double* w;
  double* v;
  double* z;
  const double* J;
  const double* hd;   // h(j+1, j) before the rotations (device)
  const int* act;     // the cycle's Arnoldi steps go on (device)
  double hdiv = 0.0;
  __device__ bool prepare() {
    if (!*(volatile const int*)act) return false;
    hdiv = *hd;
    return true;
  }
  __device__ void load(long i, Regs& g) const { g.w = __ldg(w + i); g.J = __ldg(J + i); }
  __device__ void compute(long i, Regs& g, double*) const {
    const double vi = __ddiv_rn(g.w, hdiv);
    v[i] = vi;
    z[i] = dmul(vi, g.J);
  }
  __device__ void finish(double*) const {}
};

// modified Gram-Schmidt step i: w = w - h_ij v_i (h_ij read from device
// memory), then the next coefficient v_{i+1}.w or, after the last step,
// ||w|| (:699-717)
struct OpMgs {
  static constexpr int NRED = 1;
  struct Regs { double w, v, vn; };
  double* w;
  const double* vi;
  const double* vnext;  // null: norm of w
  const double* hij;
  double* out;
  const int* act;     // the cycle's Arnoldi steps go on (device)
  double h = 0.0;
  __device__ bool prepare() {
    if (!*(volatile const int*)act) return false;
    h = *hij;
    return true;
  }
  __device__ void load(long i, Regs& g) const {
    g.w = w[i];
    g.v = __ldg(vi + i);
    g.vn = vnext ? __ldg(vnext + i) : 0.0;
  }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const double wn = __dsub_rn(g.w, dmul(h, g.v));
    w[i] = wn;
    acc[0] = dadd(acc[0], vnext ? dmul(g.vn, wn) : dmul(wn, wn));
  }
  __device__ void finish(double* tot) const { *out = vnext ? tot[0] : sqrt(tot[0]); }
};

// v_0 . w -> h(0, j), skipped when the cycle has ended
struct OpDotIf {
  static constexpr int NRED = 1;
  struct Regs { double a, b; };
  const double* a;
  const double* b;
  double* out;
  const int* act;
  __device__ bool prepare() { return *(volatile const int*)act != 0; }
  __device__ void load(long i, Regs& r) const { r.a = __ldg(a + i); r.b = __ldg(b + i); }
  __device__ void compute(long, Regs& r, double* acc) const { acc[0] = dadd(acc[0], dmul(r.a, r.b)); }
  __device__ void finish(double* tot) const { *out = tot[0]; }
};

// w = 0 + A z_j, skipped when the cycle has ended
struct EpiStoreIf {
  static constexpr int NRED = 0;
  double* y;
  const int* act;
  __device__ bool active() const { return *(volatile const int*)act != 0; }
  __device__ void row(long r, double s, double*) const { y[r] = dadd(0.0, s); }
  __device__ void finish(double*) const {}
};

// ---- GMRES device state and its one-thread kernels -----------------------------

constexpr int kMaxRestart = 128;

struct GmState {
  double eps, bnorm, resnorm, local;
  int iter, steps, restart, hpos, jdone, conv, act, go;
  double hn[kMaxRestart];   // h(j+1, j) before the rotations: v_{j+1} = w / hn[j]
  double cc[kMaxRestart], ss[kMaxRestart], gam[kMaxRestart + 1], al[kMaxRestart];
};

struct GmArgs {
  GmState* st;
  double* H;     // (M+1) x M Hessenberg, column-major: H(i, j) = H[j (M+1) + i]
  int M;
  double* hist;  // |gamma| history (device, hist_cap entries) or null
  int hist_cap;
  int iter_max;
  int literal;   // the reference's unrotated Givens update (:722-727)
  cudaGraphConditionalHandle cond;
  const int* errw;
  __device__ double& h(int i, int j) const { return H[(size_t)j * (M + 1) + i]; }
  __device__ void push_hist(double v) const {
    if (hist && st->hpos < hist_cap) hist[st->hpos] = v;
    st->hpos += 1;
  }
};

// after ||b||: the tolerance and the counters of the first outer iteration
__global__ void gm_setup_kernel(GmArgs a, double eps_abs, double eps_rel) {
  GmState* s = a.st;
  double e = eps_abs;
  if (eps_rel > 0.0 && eps_rel * s->bnorm > e) e = eps_rel * s->bnorm;
  s->eps = e;
  s->iter = 1;  // the outer loop's first ++iter (:643)
  s->steps = 0;
  s->restart = 0;
  s->hpos = 0;
  s->conv = 0;
  s->act = 0;
  s->go = 1;
}

// after the first residual: its norm opens the history
__global__ void gm_begin_kernel(GmArgs a) {
  GmState* s = a.st;
  a.push_hist(s->resnorm);
  s->local = s->resnorm;
}

// a restart cycle begins: gamma_0 = ||r|| (:669-672)
__global__ void gm_cycle_start_kernel(GmArgs a) {
  GmState* s = a.st;
  s->gam[0] = s->resnorm;
  s->jdone = a.M;
  s->act = 1;
}

// Arnoldi step j after the Gram-Schmidt sweeps left the raw column
// h(0..j+1, j): the previous rotations, the new rotation, gamma and the
// convergence test (:722-737), in the host restatement's operation order.
__global__ void gm_givens_kernel(GmArgs a, int j) {
  GmState* s = a.st;
  if (!s->act) return;
  s->steps += 1;
  for (int i = 0; i < j; ++i) {
    if (a.literal) {
      const double t = dadd(dmul(a.h(i, j), s->cc[i]), dmul(a.h(i + 1, j), s->ss[i]));
      a.h(i, j) = dadd(dmul(-t, s->ss[i]), dmul(a.h(i + 1, j), s->cc[i]));
    } else {
      const double top = dadd(dmul(a.h(i, j), s->cc[i]), dmul(a.h(i + 1, j), s->ss[i]));
      const double bot = dadd(dmul(-a.h(i, j), s->ss[i]), dmul(a.h(i + 1, j), s->cc[i]));
      a.h(i, j) = top;
      a.h(i + 1, j) = bot;
    }
  }
  const double hjj = a.h(j, j), hn = a.h(j + 1, j);
  s->hn[j] = hn;
  const double beta = sqrt(dadd(dmul(hjj, hjj), dmul(hn, hn)));
  s->ss[j] = hn / beta;
  s->cc[j] = hjj / beta;
  a.h(j, j) = beta;
  s->gam[j + 1] = dmul(-s->ss[j], s->gam[j]);
  s->gam[j] = dmul(s->cc[j], s->gam[j]);
  const double g = fabs(s->gam[j + 1]);
  a.push_hist(g);
  if (g <= s->eps) {
    s->jdone = j + 1;
    s->conv = 1;
    s->act = 0;
  }
}

// al = H^-1 gamma over the cycle's jdone steps (:739-747, :784-792)
__global__ void gm_backsub_kernel(GmArgs a) {
  GmState* s = a.st;
  const int k = s->jdone;
  for (int i = k - 1; i >= 0; --i) {
    double acc = 0.0;
    for (int t = i + 1; t < k; ++t) acc = dadd(acc, dmul(a.h(i, t), s->al[t]));
    s->al[i] = dmul(1.0 / a.h(i, i), __dsub_rn(s->gam[i], acc));
  }
  s->act = 0;
}

// after the cycle's residual: the restart and outer-loop decisions
// (:643, :664-668, :824-830); sets the WHILE node's condition
__global__ void gm_cycle_end_kernel(GmArgs a) {
  GmState* s = a.st;
  s->local = s->resnorm;
  s->restart += 1;
  int go = 1;
  if (s->conv || *(volatile const int*)a.errw) {
    go = 0;
  } else if (s->restart > a.M) {
    // the inner while ends; the outer one goes on while iter <= iter_max
    // (its residual is the one just computed, x being unchanged)
    if (s->iter <= a.iter_max) {
      s->iter += 1;
      s->restart = 0;
    } else {
      go = 0;
    }
  }
  s->go = go;
  if (a.cond) cudaGraphSetConditional(a.cond, (unsigned)go);
}

// x = x + sum_i al_i z_i over the cycle's steps, terms added in order
// i = 0..k-1 (:755-760, :799-803)
__global__ void x_update_kernel(long n, double* __restrict__ x, const double* __restrict__ Z,
                                size_t nn, const GmState* __restrict__ st) {
  const int k = st->jdone;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double xi = x[i];
    for (int t = 0; t < k; ++t) xi = dadd(xi, dmul(st->al[t], __ldg(Z + nn * (size_t)t + i)));
    x[i] = xi;
  }
}

// ---- helpers --------------------------------------------------------------------

static int read_scalar(celg_handle* h, const double* d, double* out) {
  CELG_CUDA(cudaMemcpyAsync(h->scal_h, d, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  *out = h->scal_h[0];
  return CELG_OK;
}

static int spmv_fmt(celg_handle* h, celg_mat* m, int fmt, const double* x, double* y) {
  if (fmt == CELG_FMT_JAD) return launch_spmv_jad(h, m->csr, m->jad, x, y);
  return launch_spmv_csr(h, m->csr, x, y, 0);
}

struct OpFillOne {
  static constexpr int NRED = 0;
  struct Regs { int unused; };
  double* x;
  __device__ bool prepare() { return true; }
  __device__ void load(long, Regs&) const {}
  __device__ void compute(long i, Regs&, double*) const { x[i] = 1.0; }
  __device__ void finish(double*) const {}
};

static int set_x0(celg_handle* h, long n, int mode, double* x) {
  if (mode == CELG_X0_USER || n == 0) return CELG_OK;
  if (mode == CELG_X0_ZERO) {
    CELG_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n, h->stream));
    return CELG_OK;
  }
  return launch_tile(h, n, OpFillOne{x});
}

static void store_hist(celg_result* res, int idx, double v) {
  if (res && res->history && idx < res->history_cap) {
    res->history[idx] = v;
    res->history_len = std::max(res->history_len, idx + 1);
  }
}

// ---- CG: cel_cgalg, src/fcgalg/cel_cgalg_module.f90:34-175 --------------------------

int cg_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res) {
  const long n = m->csr.n;
  const int fmt = p->fmt;
  if (fmt == CELG_FMT_JAD && m->jad.mmax < 0) return CELG_ERR_STATE;
  int st = ensure_work(h, (size_t)n);
  if (st) return st;
  if (res) res->history_len = 0;
  double* r = h->wr;
  double* d = h->wp;
  double* q = h->wv;
  double* sd = h->scal_d;
  cudaEventRecord(h->ev0, h->stream);
  if ((st = set_x0(h, n, p->x0_mode, x))) return st;
  double bnorm, norm, sigma_new, sigma_old, alpha = 1.0, dq;
  if ((st = launch_dot(h, n, b, b, sd, 1)) || (st = read_scalar(h, sd, &bnorm))) return st;
  double eps = p->eps_abs;
  if (p->eps_rel > 0.0 && p->eps_rel * bnorm > eps) eps = p->eps_rel * bnorm;
  // r = 0 + A x; ||A x|| (:67-77)
  if ((st = spmv_fmt(h, m, fmt, x, r))) return st;
  if ((st = launch_dot(h, n, r, r, sd, 1)) || (st = read_scalar(h, sd, &norm))) return st;
  if ((st = launch_tile(h, n, OpCalcRD{b, r, d}))) return st;
  if ((st = launch_dot(h, n, r, r, sd, 0)) || (st = read_scalar(h, sd, &sigma_new))) return st;
  sigma_old = sigma_new;
  if (!p->literal_ref_bugs) norm = std::sqrt(sigma_new);
  store_hist(res, 0, norm);
  int ii = 0, err = CELG_OK;
  for (;;) {
    bool go;
    if (p->literal_ref_bugs)
      go = ii < p->iter_max && sigma_new > sigma_old * p->eps_abs * p->eps_abs &&
           std::fabs(sigma_new) > kRealSmall;
    else
      go = ii < p->iter_max && norm > eps && std::fabs(sigma_new) > kRealSmall;
    if (!go) break;
    if ((st = spmv_fmt(h, m, fmt, d, q))) return st;
    ++ii;
    if ((st = launch_dot(h, n, d, q, sd, 0)) || (st = read_scalar(h, sd, &dq))) return st;
    alpha = sigma_new / dq;
    if (!std::isfinite(alpha)) {
      err = CELG_ERR_BREAKDOWN;
      break;
    }
    if ((st = launch_tile(h, n, OpXR{x, d, r, q, alpha}))) return st;
    sigma_old = sigma_new;
    if ((st = launch_dot(h, n, r, r, sd, 0)) || (st = read_scalar(h, sd, &sigma_new))) return st;
    const double beta = p->literal_ref_bugs ? alpha : sigma_new / sigma_old;  // :151
    if ((st = launch_xpby(h, n, r, beta, d))) return st;
    norm = std::sqrt(sigma_new);
    store_hist(res, ii, norm);
  }
  // verification
  double vres = 0.0;
  if ((st = launch_residual(h, m, fmt, b, x, q, sd)) || (st = read_scalar(h, sd, &vres))) return st;
  cudaEventRecord(h->ev1, h->stream);
  cudaEventSynchronize(h->ev1);
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  h->last_iters = ii;
  int ret = err;
  if (!ret && !p->literal_ref_bugs && norm > eps && ii >= p->iter_max) ret = CELG_ERR_NOCONV;
  if (res) {
    res->iter_done = ii;
    res->final_norm2 = norm;
    res->bnorm = bnorm;
    res->verified_relres = bnorm > 0 ? vres / bnorm : vres;
    res->err = ret;
    res->arnoldi_steps = 0;
  }
  return ret;
}

// ---- GMRES(m): cel_gmresalg_2jacobi, src/fcgalg/cel_gmresalg_module.f90:570-851 -------

// The work space of a GMRES(M) solve on n rows, kept by the handle:
// V[0..M], Z[0..M-1] and H ((M+1) x M), plus the device state.
static int ensure_gmres_work(celg_handle* h, size_t nn, int M) {
  const size_t need = nn * (size_t)(2 * M + 1) + (size_t)(M + 1) * M + 8;
  if (!h->gm_state_d) CELG_CUDA(cudaMalloc(&h->gm_state_d, sizeof(GmState)));
  if (!h->gm_state_h) CELG_CUDA(cudaMallocHost(&h->gm_state_h, sizeof(GmState)));
  if (need <= h->gm_cap && h->gm_work) return CELG_OK;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  graph_cache_clear(h);
  cudaFree(h->gm_work);
  h->gm_work = nullptr;
  h->gm_cap = 0;
  CELG_CUDA(cudaMalloc(&h->gm_work, sizeof(double) * need));
  h->gm_cap = need;
  return CELG_OK;
}

struct GmPlan {
  celg_mat* m;
  int fmt;
  long n;
  size_t nn;
  const double* b;
  double* x;
  const celg_params* p;
  double* V;
  double* Z;
  double* r;
  double* w;
  GmArgs a;
  double* Vp(int i) const { return V + nn * (size_t)i; }
  double* Zp(int i) const { return Z + nn * (size_t)i; }
  double* Hp(int i, int j) const { return a.H + (size_t)j * (a.M + 1) + i; }
};

// w = A z on the row patterns or 1-byte offsets when the matrix has them
// (same columns in the same order: the same sums)
static int gm_spmv(celg_handle* h, const GmPlan& g, const double* x, double* y) {
  const EpiStoreIf epi{y, &g.a.st->act};
  if (g.fmt == CELG_FMT_JAD) return launch_jad(h, g.m->csr, g.m->jad, x, epi);
  bool done = false;
  const int st = launch_csr_compact<double>(h, g.m->csr, g.m->csr.v, x, epi, nullptr, 0, &done);
  if (done) return st;
  return launch_csr<double>(h, g.m->csr, g.m->csr.v, x, epi);
}

// x0, ||b||, the tolerance and the first residual
static int gm_record_setup(celg_handle* h, const GmPlan& g) {
  int st = set_x0(h, g.n, g.p->x0_mode, g.x);
  if (!st) st = launch_dot(h, g.n, g.b, g.b, &g.a.st->bnorm, 1);
  if (st) return st;
  gm_setup_kernel<<<1, 1, 0, h->stream>>>(g.a, g.p->eps_abs, g.p->eps_rel);
  CELG_CUDA(cudaGetLastError());
  st = launch_residual(h, g.m, g.fmt, g.b, g.x, g.r, &g.a.st->resnorm);
  if (st) return st;
  gm_begin_kernel<<<1, 1, 0, h->stream>>>(g.a);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// One restart cycle: M Arnoldi steps (the kernels of the steps after
// convergence return at once), back substitution, x update, the new
// residual and the loop decision.
static int gm_record_cycle(celg_handle* h, const GmPlan& g) {
  const int M = g.a.M;
  const int* act = &g.a.st->act;
  const double* J = g.m->jacobi;
  gm_cycle_start_kernel<<<1, 1, 0, h->stream>>>(g.a);
  CELG_CUDA(cudaGetLastError());
  // v_0 = r * (1/||r||); z_0 = J v_0 (:669, :683)
  int st = launch_tile(h, g.n, OpV1{g.r, g.Vp(0), g.Zp(0), J, &g.a.st->local});
  for (int j = 0; !st && j < M; ++j) {
    // w = 0 + A z_j (:680-697)
    st = gm_spmv(h, g, g.Zp(j), g.w);
    // h_0j = v_0 . w, then modified Gram-Schmidt with the next coefficient fused
    if (!st) st = launch_tile(h, g.n, OpDotIf{g.Vp(0), g.w, g.Hp(0, j), act});
    for (int i = 0; !st && i <= j; ++i) {
      const bool last = i == j;
      st = launch_tile(h, g.n, OpMgs{g.w, g.Vp(i), last ? nullptr : g.Vp(i + 1), g.Hp(i, j),
                                     last ? g.Hp(j + 1, j) : g.Hp(i + 1, j), act});
    }
    if (st) break;
    gm_givens_kernel<<<1, 1, 0, h->stream>>>(g.a, j);
    CELG_CUDA(cudaGetLastError());
    // v_{j+1} = w / h(j+1,j); z_{j+1} = J v_{j+1}
    if (j + 1 < M)
      st = launch_tile(h, g.n, OpVNext{g.w, g.Vp(j + 1), g.Zp(j + 1), J, &g.a.st->hn[j], act});
  }
  if (st) return st;
  gm_backsub_kernel<<<1, 1, 0, h->stream>>>(g.a);
  CELG_CUDA(cudaGetLastError());
  if (g.n > 0) {
    const int grid = (int)std::max(1L, std::min((g.n + 255) / 256, (long)h->sms * 16));
    x_update_kernel<<<grid, 256, 0, h->stream>>>(g.n, g.x, g.Z, g.nn, g.a.st);
    CELG_CUDA(cudaGetLastError());
  }
  // r = b - A x ; ||r|| (:808-824)
  st = launch_residual(h, g.m, g.fmt, g.b, g.x, g.r, &g.a.st->resnorm);
  if (st) return st;
  gm_cycle_end_kernel<<<1, 1, 0, h->stream>>>(g.a);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

int gmres_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
                celg_result* res) {
  const long n = m->csr.n;
  const int fmt = p->fmt;
  const int M = p->restart;
  if (M <= 0 || M > kMaxRestart) return CELG_ERR_ARG;
  if (p->iter_max < 0) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  if (fmt == CELG_FMT_JAD && m->jad.mmax < 0) return CELG_ERR_STATE;
  const size_t nn = (size_t)std::max(1L, n);
  int st = ensure_work(h, (size_t)n);
  if (!st) st = ensure_offset_dict(h, m);
  if (!st) st = ensure_gmres_work(h, nn, M);
  if (!st) st = ensure_partials(h, ntiles_of(n), 2);
  const int hist_cap = (res && res->history && res->history_cap > 0) ? res->history_cap : 0;
  if (!st && hist_cap) st = ensure_state(h, hist_cap);
  if (st) return st;
  if (res) res->history_len = 0;
  GmPlan g;
  g.m = m;
  g.fmt = fmt;
  g.n = n;
  g.nn = nn;
  g.b = b;
  g.x = x;
  g.p = p;
  g.V = h->gm_work;
  g.Z = g.V + nn * (size_t)(M + 1);
  g.r = h->wr;
  g.w = h->wv;
  GmState* sd = static_cast<GmState*>(h->gm_state_d);
  g.a = GmArgs{sd, g.Z + nn * (size_t)M, M, hist_cap ? h->hist_d : nullptr, hist_cap, p->iter_max,
               p->literal_ref_bugs, 0, h->err_d};
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  if (!graphs_enabled()) {
    // host-driven (profiling): one poll of the loop flag per restart cycle
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = gm_record_setup(h, g);
    GmState* sh = static_cast<GmState*>(h->gm_state_h);
    while (!st) {
      st = gm_record_cycle(h, g);
      if (st) break;
      CELG_CUDA(cudaMemcpyAsync(&sh->go, &sd->go, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      CELG_CUDA(cudaStreamSynchronize(h->stream));
      if (!sh->go) break;
    }
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    char kb[512];
    std::snprintf(kb, sizeof(kb), "gmres|%p|%d|%d|%p|%p|%d|%d|%d|%.17g|%.17g|%d|%d", (const void*)m,
                  m->csr.n, fmt, (const void*)b, (const void*)x, M, p->x0_mode, p->literal_ref_bugs,
                  p->eps_abs, p->eps_rel, p->iter_max, hist_cap);
    const std::string key(kb);
    GraphEntry* ge = graph_cache_find(h, key);
    if (!ge) {
      st = graph_build(h, key, [&](cudaGraphConditionalHandle cond) -> int {
        GmPlan gc = g;
        gc.a.cond = cond;
        int s2 = gm_record_setup(h, gc);
        if (!s2) s2 = capture_while(h, cond, [&]() -> int { return gm_record_cycle(h, gc); });
        return s2;
      }, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  GmState* sh = static_cast<GmState*>(h->gm_state_h);
  CELG_CUDA(cudaMemcpyAsync(sh, sd, sizeof(GmState), cudaMemcpyDeviceToHost, h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(h->scal_h + 8, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  std::memcpy(&err_word, h->scal_h + 8, sizeof(int));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  h->last_iters = sh->steps;
  int ret = sh->conv ? CELG_OK : CELG_ERR_NOCONV;
  if (err_word) ret = err_word;
  if (res) {
    res->iter_done = sh->iter;
    res->final_norm2 = sh->resnorm;
    res->bnorm = sh->bnorm;
    res->verified_relres = sh->bnorm > 0 ? sh->resnorm / sh->bnorm : sh->resnorm;
    res->err = ret;
    res->arnoldi_steps = sh->steps;
    if (hist_cap) {
      st = copy_history(h, std::min(sh->hpos, hist_cap), res);
      if (st) return st;
    }
  }
  return ret;
}

}  // namespace celg
