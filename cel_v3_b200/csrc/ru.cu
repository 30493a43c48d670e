// ru.cu -- FP32-storage Jacobi-PCG with FP64 reliable updates.
//
// A refinement scheme that keeps the Krylov direction across corrections
// (the "reliable update" mixed-precision CG of Clark, Babich, Barros,
// Brower and Rebbi, Comput. Phys. Commun. 181 (2010) 1517, with point-Jacobi
// preconditioning):
//
//   x64 = x0;  r64 = b - A x64;  r = (float) r64;  d = 0;  p = J r;  rz = r.J r
//   loop (FP32 matrix and vectors, FP64 scalars and reductions):
//     v = A32 p;  sigma = rz / (p.v)
//     d += sigma p;  r -= sigma v;  rz' = r.J r;  ||r||
//     if ||r|| < delta * ||r64|| or ||r|| <= eps:          reliable update
//         x64 += d;  d = 0;                                 (FP64)
//         r64 = b - A x64 with the FP64 matrix;  r = (float) r64
//         stop when ||r64|| <= eps                          (FP64 test)
//         rz' = r.J r
//     beta = rz'/rz;  rz = rz';  p = J r + beta p
//
// Compared with restarting an inner solve at every correction (ir.cu), the
// search direction survives the residual replacement, so the iteration count
// stays close to the FP64 solver's while every sweep moves FP32 data.  The
// update threshold delta is celg_params.inner_eps_rel.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "graph.cuh"
#include "pcg_internal.cuh"

namespace celg {

struct RuState {
  PcgState s;      // alpha = rz, sigma, beta, norm = ||r|| (FP32 recurrence), bnorm, eps
  double maxr;     // ||r64|| at the last reliable update
  double rz_prev;  // rz before the current iteration's update
  double norm64;   // last FP64 residual norm
  double delta;
  int update;      // 1: the FP32 recurrence asks for a reliable update
  int updates;
};

struct RuArgs {
  RuState* st;
  double* hist;
  int hist_cap;
  int iter_max;
  cudaGraphConditionalHandle cond;
  const int* errw;
  cudaGraphConditionalHandle cond_update;  // IF node guarding the reliable update (0: none)
  PcgArgs pcg() const {
    return PcgArgs{&st->s, hist, hist_cap, iter_max, cond, errw};
  }
};

__device__ __forceinline__ int ru_go(const RuState* r, int iter_max, const int* errw) {
  const PcgState* s = &r->s;
  return (s->err == 0 && *(volatile const int*)errw == 0 && s->iter < iter_max &&
          r->norm64 > s->eps)
             ? 1
             : 0;
}

// RU0: x0 and ||b||, eps
struct OpRuPre {
  static constexpr int NRED = 1;
  struct Regs { double b; };
  const double* b;
  double* x;
  int x0_mode;
  double eps_abs, eps_rel, delta;
  RuArgs a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); }
  __device__ void compute(long i, Regs& g, double* acc) const {
    if (x0_mode == CELG_X0_REF_ONES) x[i] = 1.0;
    else if (x0_mode == CELG_X0_ZERO) x[i] = 0.0;
    acc[0] = dadd(acc[0], dmul(g.b, g.b));
  }
  __device__ void finish(double* tot) const {
    RuState* r = a.st;
    r->s.bnorm = sqrt(tot[0]);
    double e = eps_abs;
    if (eps_rel > 0.0 && eps_rel * r->s.bnorm > e) e = eps_rel * r->s.bnorm;
    r->s.eps = e;
    r->s.err = 0;
    r->s.iter = 0;
    r->s.active = 1;
    r->s.vres = 0.0;
    r->delta = delta;
    r->update = 1;  // the set-up residual is a reliable update
    r->updates = 0;
    r->s.xpend = 0;
    r->s.xprev = 0;
    r->s.sigprev = 0.0;
  }
};

// FP64 residual with the FP64 matrix, and its FP32 copy:
//   r64 = b - (0 + A x);  r = (float) r64;  z = (double) r * J;  rz = r.z;  ||r64||^2
// init: also p = (float) z.  Active only when a reliable update is pending.
struct EpiRuResidual {
  static constexpr int NRED = 2;
  const double* b;
  float* r;
  float* p;        // non-null only at set-up
  const float* J;
  RuArgs a;
  int init;
  __device__ bool active() const { return *(volatile int*)&a.st->update != 0; }
  __device__ void row(long i, double s, double* acc) const {
    const double r64 = __dsub_rn(b[i], dadd(0.0, s));
    const float rf = (float)r64;
    r[i] = rf;
    const double z = dmul((double)rf, (double)J[i]);
    if (init) p[i] = (float)z;
    acc[0] = dadd(acc[0], dmul((double)rf, z));
    acc[1] = dadd(acc[1], dmul(r64, r64));
  }
  __device__ void finish(double* tot) const {
    RuState* st = a.st;
    st->norm64 = sqrt(tot[1]);
    st->maxr = st->norm64;
    st->update = 0;
    st->updates += 1;
    if (init) {
      st->s.alpha = tot[0];
      st->s.norm = st->norm64;
      if (a.hist && a.hist_cap > 0) a.hist[0] = st->norm64;
      st->s.hist_len = 1;
    } else {
      st->s.beta = tot[0] / st->rz_prev;
      st->s.alpha = tot[0];
      if (a.hist && st->s.iter < a.hist_cap) a.hist[st->s.iter] = st->norm64;
    }
    st->s.active = ru_go(st, a.iter_max, a.errw);
    set_cond(a.cond, st->s.active);
  }
};

// r -= sigma v ; rz' = r.J r ; ||r||^2 ; update decision.  The iteration's
// d += sigma p is left pending (s.xpend) for the flush or the direction
// sweep, which read p anyway, so this sweep reads neither d nor p.  The
// FP32 residual is updated in FP32 arithmetic (r + (float)(-sigma) v, each
// operation rounded once); its dot products stay FP64 on exact products.
// Done in FP64 and rounded back, the update took three more conversions per
// element, and the sweep was bound by the conversion rate, not by memory.
struct OpRuStep {
  static constexpr int NRED = 2;
  static constexpr int kTilesPerPass = 2;
  struct Regs { float r, v, J; };
  float* r;
  const float* v;
  const float* J;
  RuArgs a;
  float nsg;
  __device__ bool prepare() {
    if (*(volatile int*)&a.st->s.active == 0) {
      if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(a.cond, 0);
      return false;
    }
    nsg = (float)(-a.st->s.sigma);
    return true;
  }
  __device__ void load(long i, Regs& g) const {
    g.r = r[i];
    g.v = __ldcs(v + i);
    g.J = __ldg(J + i);
  }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const float ri = fadd(g.r, fmul(nsg, g.v));
    r[i] = ri;
    const double z = dmul((double)ri, (double)g.J);
    acc[0] = dadd(acc[0], dmul((double)ri, z));
    acc[1] = dacc_prod(acc[1], ri, ri);
  }
  __device__ void finish(double* tot) const {
    RuState* st = a.st;
    st->rz_prev = st->s.alpha;
    st->s.beta = tot[0] / st->s.alpha;
    st->s.alpha = tot[0];
    st->s.norm = sqrt(tot[1]);
    st->s.iter += 1;
    if (a.hist && st->s.iter < a.hist_cap) a.hist[st->s.iter] = st->s.norm;
    st->s.hist_len = min(st->s.iter + 1, a.hist_cap);
    st->s.xpend = 1;
    const int upd = (st->s.norm < st->delta * st->maxr) || (st->s.norm <= st->s.eps) ||
                    (st->s.iter >= a.iter_max);
    st->update = upd;
    set_cond(a.cond_update, upd);
    if (!upd) {
      // FP32 recurrence continues; stop only on the iteration cap or an error
      const int go = (st->s.err == 0 && *(volatile const int*)a.errw == 0 &&
                      st->s.iter < a.iter_max && fabs(st->s.alpha) > 0.0)
                         ? 1
                         : 0;
      st->s.active = go;
      set_cond(a.cond, go);
    }
  }
};

// x64 += (double) d ; d = 0   (pending update, or unconditionally at the end).
// The d += sigma p updates still pending are applied first, in order and
// with the step's rounding: the even iteration's (s.xprev, direction pp)
// when the flush follows the odd step of a pair, then the step's own
// (s.xpend, direction p).  The last CTA clears both marks.
struct OpRuFlush {
  static constexpr int NRED = 0;
  static constexpr bool kFinishAlways = true;
  struct Regs { double x; float d, p, pp; };
  double* x;
  float* d;
  const float* p;
  const float* pp;
  RuArgs a;
  int always;
  int dp = 0, dq = 0;
  double sg = 0.0, sp = 0.0;
  __device__ bool prepare() {
    if (!(always || *(volatile int*)&a.st->update != 0)) return false;
    dp = p != nullptr && *(volatile int*)&a.st->s.xpend;
    dq = pp != nullptr && *(volatile int*)&a.st->s.xprev;
    sg = a.st->s.sigma;
    sp = a.st->s.sigprev;
    return true;
  }
  __device__ void load(long i, Regs& g) const {
    g.x = x[i];
    g.d = d[i];
    if (dp) g.p = __ldg(p + i);
    if (dq) g.pp = __ldg(pp + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    float di = g.d;
    if (dq) di = (float)dadd((double)di, dmul(sp, (double)g.pp));
    if (dp) di = (float)dadd((double)di, dmul(sg, (double)g.p));
    x[i] = dadd(g.x, (double)di);
    d[i] = 0.0f;
  }
  __device__ void finish(double*) const {
    a.st->s.xpend = 0;
    a.st->s.xprev = 0;
  }
};

// final check ||b - A x|| / ||b|| in FP64
struct EpiRuVerify {
  static constexpr int NRED = 1;
  const double* b;
  RuState* st;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const {
    st->s.vres = st->s.bnorm > 0.0 ? sqrt(tot[0]) / st->s.bnorm : sqrt(tot[0]);
  }
};

struct OpZeroF {
  static constexpr int NRED = 0;
  struct Regs { int unused; };
  float* d;
  __device__ bool prepare() { return true; }
  __device__ void load(long, Regs&) const {}
  __device__ void compute(long i, Regs&, double*) const { d[i] = 0.0f; }
  __device__ void finish(double*) const {}
};

static int ru_setup(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
                    RuArgs a, float* r, float* pv, float* d) {
  const long n = m->csr.n;
  const double delta = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-2;
  int st = launch_tile(h, n, OpRuPre{b, x, p->x0_mode, p->eps_abs, p->eps_rel, delta, a});
  if (!st) st = launch_tile(h, n, OpZeroF{d});
  if (!st)
    st = launch_csr<double>(h, m->csr, m->csr.v, x, EpiRuResidual{b, r, pv, m->jacobi32, a, 1});
  return st;
}

// One iteration: K1, K2, then (only when K2 asked for it) the reliable
// update -- inside an IF conditional node when recorded into a graph, as
// self-skipping kernels otherwise -- then K3.  Iterations run in pairs
// whose directions are pv and pq in turn (odd = false, then true); K3 is
// the paired direction sweep of the PCG (OpDirectionDefer, OpDirectionPair)
// with the correction d in place of x, so d is read and stored once per
// pair.
static int ru_body(celg_handle* h, celg_mat* m, const double* b, double* x, RuArgs a, float* r,
                   float* pv, float* pq, float* v, float* d, bool odd, bool in_graph) {
  const long n = m->csr.n;
  if (in_graph) {
    int st = capture_new_handle(h, 0, &a.cond_update);
    if (st) return st;
  }
  PcgArgs pa = a.pcg();
  float* pc = odd ? pq : pv;
  int st = launch_csr<float>(h, m->csr, m->csr.v32, pc, EpiAp<float>{v, pc, pa});
  if (!st) st = launch_tile(h, n, OpRuStep{r, v, m->jacobi32, a, 0.0f});
  auto update = [&]() -> int {
    int s2 = launch_tile(h, n, OpRuFlush{x, d, pc, odd ? pv : nullptr, a, 0});
    if (!s2)
      s2 = launch_csr<double>(h, m->csr, m->csr.v, x,
                              EpiRuResidual{b, r, nullptr, m->jacobi32, a, 0});
    return s2;
  };
  if (!st) st = in_graph ? capture_if(h, a.cond_update, update) : update();
  if (st) return st;
  const float* J = m->jacobi32;
  if (odd) return launch_tile(h, n, OpDirectionPair<float>{pv, pq, r, J, d, pa});
  return launch_tile(h, n, OpDirectionDefer<float>{pv, pq, r, J, d, pa});
}

static int ru_tail(celg_handle* h, celg_mat* m, const double* b, double* x, RuArgs a, float* d) {
  int st = launch_tile(h, m->csr.n, OpRuFlush{x, d, nullptr, nullptr, a, 1});
  if (!st) st = launch_csr<double>(h, m->csr, m->csr.v, x, EpiRuVerify{b, a.st});
  return st;
}

int ru_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
             celg_result* res) {
  const long n = m->csr.n;
  if (!m->jacobi) return CELG_ERR_STATE;
  if (!m->csr.v32 || !m->jacobi32) {
    int st = celg_mat_make_fp32(m);
    if (st) return st;
  }
  if (p->iter_max < 0) return CELG_ERR_ARG;
  int st = ensure_f32(h, (size_t)n);
  if (!st) st = ensure_partials(h, ntiles_of(n), 2);
  const int hist_cap = p->iter_max + 1;
  if (!st) st = ensure_state(h, hist_cap);
  if (st) return st;
  if (!h->ru_state_d) CELG_CUDA(cudaMalloc(&h->ru_state_d, sizeof(RuState)));
  if (!h->ru_state_h) CELG_CUDA(cudaMallocHost(&h->ru_state_h, sizeof(RuState)));
  RuState* sd = static_cast<RuState*>(h->ru_state_d);
  RuState* sh = static_cast<RuState*>(h->ru_state_h);
  const size_t cap = h->f32cap;
  float* r = h->f32;
  float* pv = r + cap;
  float* v = pv + cap;
  float* d = v + cap;
  float* pq = d + cap;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));

  char kb[512];
  std::snprintf(kb, sizeof(kb), "ru|%p|%d|%p|%p|%p|%d|%.17g|%.17g|%.17g|%d", (const void*)m,
                m->csr.n, (const void*)b, (const void*)x, (const void*)r, p->x0_mode, p->eps_abs,
                p->eps_rel, p->inner_eps_rel, p->iter_max);
  const std::string key(kb);
  RuArgs a0{sd, h->hist_d, hist_cap, p->iter_max, 0, h->err_d, 0};
  if (!graphs_enabled()) {
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = ru_setup(h, m, b, x, p, a0, r, pv, d);
    for (int it = 0; !st && it < p->iter_max; it += 8) {
      for (int k = 0; k < 8 && !st; ++k)
        st = ru_body(h, m, b, x, a0, r, pv, pq, v, d, (k & 1) != 0, false);
      if (st) break;
      CELG_CUDA(cudaMemcpyAsync(sh, sd, sizeof(RuState), cudaMemcpyDeviceToHost, h->stream));
      CELG_CUDA(cudaStreamSynchronize(h->stream));
      if (!sh->s.active) break;
    }
    if (!st) st = ru_tail(h, m, b, x, a0, d);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    GraphEntry* ge = graph_cache_find(h, key);
    if (!ge) {
      st = graph_build(h, key, [&](cudaGraphConditionalHandle cond) -> int {
        RuArgs a{sd, h->hist_d, hist_cap, p->iter_max, cond, h->err_d, 0};
        int s2 = ru_setup(h, m, b, x, p, a, r, pv, d);
        if (!s2)
          s2 = capture_while(h, cond, [&]() -> int {
            int s3 = ru_body(h, m, b, x, a, r, pv, pq, v, d, false, true);
            if (!s3) s3 = ru_body(h, m, b, x, a, r, pv, pq, v, d, true, true);
            return s3;
          });
        if (!s2) s2 = ru_tail(h, m, b, x, a, d);
        return s2;
      }, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  CELG_CUDA(cudaMemcpyAsync(sh, sd, sizeof(RuState), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaMemcpyAsync(h->scal_h + 8, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  int err_word = 0;
  std::memcpy(&err_word, h->scal_h + 8, sizeof(int));
  const RuState s = *sh;
  int ret = CELG_OK;
  if (err_word) ret = err_word;
  else if (s.s.err) ret = s.s.err;
  else if (!(s.norm64 <= s.s.eps)) ret = CELG_ERR_NOCONV;
  h->last_iters = s.s.iter;
  // K1 (matrix, p gathered, v stored: 8 n), K2 (r, v, J read, r stored:
  // 16 n), K3 (p, r, J read, p stored, d read and stored once per pair of
  // iterations: 20 n on average); 5 bytes per non-zero with the 1-byte
  // column offsets, else 8
  h->last_bytes_per_iter = (m->csr.ci8 ? 5.0 : 8.0) * m->csr.nnz + 4.0 * (n + 1) + 44.0 * n;
  if (res) {
    res->iter_done = s.s.iter;
    res->final_norm2 = s.norm64;
    res->bnorm = s.s.bnorm;
    res->verified_relres = s.s.vres;
    res->err = ret;
    res->arnoldi_steps = s.updates;
    st = copy_history(h, std::min(s.s.hist_len, hist_cap), res);
    if (st) return st;
  }
  return ret;
}

}  // namespace celg
