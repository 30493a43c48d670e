// krylov.cu -- unpreconditioned CG (cel_cgalg) and restarted GMRES(m) with
// right Jacobi preconditioning (cel_gmresalg_2jacobi).  The vector sweeps
// run on the device with the fixed-order reductions; the scalar recurrences
// (CG step lengths, GMRES Hessenberg column, Givens rotations and back
// substitution) run on the host in IEEE binary64, in the reference's order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

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
  double inv;
  __device__ bool prepare() { return true; }
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
  double hdiv;
  __device__ bool prepare() { return true; }
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
  double h;
  __device__ bool prepare() { h = *hij; return true; }
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

// x = x + sum_i al_i z_i, terms added in order i = 0..k-1 (:755-760, :799-803)
constexpr int kMaxRestart = 128;
struct ZList {
  const double* z[kMaxRestart];
  double al[kMaxRestart];
};
__global__ void x_update_kernel(long n, double* __restrict__ x, ZList zl, int k) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double xi = x[i];
    for (int t = 0; t < k; ++t) xi = dadd(xi, dmul(zl.al[t], __ldg(zl.z[t] + i)));
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

int gmres_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
                celg_result* res) {
  const long n = m->csr.n;
  const int fmt = p->fmt;
  const int M = p->restart;
  if (M <= 0 || M > kMaxRestart) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  if (fmt == CELG_FMT_JAD && m->jad.mmax < 0) return CELG_ERR_STATE;
  int st = ensure_work(h, (size_t)n);
  if (st) return st;
  if (res) res->history_len = 0;
  // V[0..M], Z[0..M-1], w, r ; H raw coefficients (M+1) x M on the device
  const size_t nn = (size_t)std::max(1L, n);
  double* base = nullptr;
  CELG_CUDA(cudaMalloc(&base, sizeof(double) * (nn * (size_t)(2 * M + 1) + (size_t)(M + 1) * M + 8)));
  double* V = base;
  double* Z = V + nn * (size_t)(M + 1);
  double* Hd = Z + nn * (size_t)M;
  double* w = h->wv;
  double* r = h->wr;
  double* sd = h->scal_d;
  const double* J = m->jacobi;
  auto Vp = [&](int i) { return V + nn * (size_t)i; };
  auto Zp = [&](int i) { return Z + nn * (size_t)i; };
  std::vector<double> H((size_t)(M + 1) * M, 0.0), cc(M + 1), ss(M + 1), gam(M + 2), al(M + 1);
  auto Hh = [&](int i, int j) -> double& { return H[(size_t)j * (M + 1) + i]; };
  auto Hdev = [&](int i, int j) { return Hd + (size_t)j * (M + 1) + i; };

  cudaEventRecord(h->ev0, h->stream);
  double bnorm = 0.0, resnorm = 0.0;
  int iter = 0, steps = 0, hpos = 0;
  bool converged = false;
  do {
    if ((st = launch_dot(h, n, b, b, sd, 1)) || (st = read_scalar(h, sd, &bnorm))) break;
    double eps = p->eps_abs;
    if (p->eps_rel > 0.0 && p->eps_rel * bnorm > eps) eps = p->eps_rel * bnorm;
    if ((st = set_x0(h, n, p->x0_mode, x))) break;
    while (iter <= p->iter_max && !converged && !st) {
      ++iter;
      // r = b - A x ; ||r|| (:643-663)
      if ((st = launch_residual(h, m, fmt, b, x, r, sd)) || (st = read_scalar(h, sd, &resnorm))) break;
      if (hpos == 0) store_hist(res, hpos++, resnorm);
      double local_res = resnorm;
      int restart = 0;
      while (restart <= M && !converged && !st) {
        // v1 = r * (1/||r||); z1 = J v1 (:669, :683)
        if ((st = launch_tile(h, n, OpV1{r, Vp(0), Zp(0), J, 1.0 / local_res}))) break;
        gam[0] = resnorm;
        int jdone = M;
        for (int j = 0; j < M; ++j) {
          // w = 0 + A z_j (:680-697)
          if ((st = spmv_fmt(h, m, fmt, Zp(j), w))) break;
          ++steps;
          // h_0j = v_0 . w, then MGS with the next coefficient fused
          if ((st = launch_dot(h, n, Vp(0), w, Hdev(0, j), 0))) break;
          for (int i = 0; i <= j; ++i) {
            const bool last = i == j;
            st = launch_tile(h, n, OpMgs{w, Vp(i), last ? nullptr : Vp(i + 1), Hdev(i, j),
                                         last ? Hdev(j + 1, j) : Hdev(i + 1, j), 0.0});
            if (st) break;
          }
          if (st) break;
          CELG_CUDA(cudaMemcpyAsync(&Hh(0, j), Hdev(0, j), sizeof(double) * (size_t)(j + 2),
                                    cudaMemcpyDeviceToHost, h->stream));
          CELG_CUDA(cudaStreamSynchronize(h->stream));
          // previous rotations on column j (:722-727; corrected unless literal)
          for (int i = 0; i < j; ++i) {
            if (p->literal_ref_bugs) {
              Hh(i, j) = Hh(i, j) * cc[i] + Hh(i + 1, j) * ss[i];
              Hh(i, j) = -Hh(i, j) * ss[i] + Hh(i + 1, j) * cc[i];
            } else {
              const double top = Hh(i, j) * cc[i] + Hh(i + 1, j) * ss[i];
              const double bot = -Hh(i, j) * ss[i] + Hh(i + 1, j) * cc[i];
              Hh(i, j) = top;
              Hh(i + 1, j) = bot;
            }
          }
          // new rotation (:728-733)
          const double hn = Hh(j + 1, j);
          const double beta = std::sqrt(Hh(j, j) * Hh(j, j) + Hh(j + 1, j) * Hh(j + 1, j));
          ss[j] = Hh(j + 1, j) / beta;
          cc[j] = Hh(j, j) / beta;
          Hh(j, j) = beta;
          gam[j + 1] = -ss[j] * gam[j];
          gam[j] = cc[j] * gam[j];
          store_hist(res, hpos++, std::fabs(gam[j + 1]));
          if (std::fabs(gam[j + 1]) <= eps) {
            jdone = j + 1;
            converged = true;
            break;
          }
          // v_{j+1} = w / h(j+1,j); z_{j+1} = J v_{j+1}
          if (j + 1 < M) {
            if ((st = launch_tile(h, n, OpVNext{w, Vp(j + 1), Zp(j + 1), J, hn}))) break;
          }
        }
        if (st) break;
        // back substitution (:739-747, :784-792)
        for (int i = jdone - 1; i >= 0; --i) {
          double acc = 0.0;
          for (int k = i + 1; k < jdone; ++k) acc = acc + Hh(i, k) * al[k];
          al[i] = (1.0 / Hh(i, i)) * (gam[i] - acc);
        }
        ZList zl;
        for (int i = 0; i < jdone; ++i) {
          zl.z[i] = Zp(i);
          zl.al[i] = al[i];
        }
        if (n > 0) {
          const int grid = (int)std::max(1L, std::min((n + 255) / 256, (long)h->sms * 16));
          x_update_kernel<<<grid, 256, 0, h->stream>>>(n, x, zl, jdone);
          if (cudaGetLastError() != cudaSuccess) { st = CELG_ERR_CUDA; break; }
        }
        // r = b - A x ; ||r|| (:808-824)
        if ((st = launch_residual(h, m, fmt, b, x, r, sd)) || (st = read_scalar(h, sd, &resnorm))) break;
        local_res = resnorm;
        ++restart;
      }
    }
  } while (0);
  cudaEventRecord(h->ev1, h->stream);
  cudaEventSynchronize(h->ev1);
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  cudaFree(base);
  if (st) return st;
  h->last_iters = steps;
  const int ret = converged ? CELG_OK : CELG_ERR_NOCONV;
  if (res) {
    res->iter_done = iter;
    res->final_norm2 = resnorm;
    res->bnorm = bnorm;
    res->verified_relres = bnorm > 0 ? resnorm / bnorm : resnorm;
    res->err = ret;
    res->arnoldi_steps = steps;
  }
  return ret;
}

}  // namespace celg
