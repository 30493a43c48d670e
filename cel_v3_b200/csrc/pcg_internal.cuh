// pcg_internal.cuh -- device state, argument packs and the fused sweeps of
// the Jacobi-PCG iteration (see pcg.cu), shared with the refinement and
// batched solvers.
#pragma once
#include <type_traits>

#include "tile_kernels.cuh"

namespace celg {

constexpr double kRealSmall = 1.1 * 2.220446049250313e-16;  // cel_real_small

struct PcgState {
  double alpha, sigma, beta, norm, bnorm, eps, pvd, rz, vres;
  int iter, active, err, hist_len;
  int xpend;  // K2 ran: K3 owes x += sigma p
  int xprev;  // paired form: the odd K3 owes x += sigprev p_prev first
  double sigprev;
};

struct PcgArgs {
  PcgState* st;
  double* hist;
  int hist_cap;
  int iter_max;
  cudaGraphConditionalHandle cond;
  const int* errw;  // device error word of the handle (bounded-wait timeouts)
};

// Vectors and matrix one PCG solve runs on.
template <typename VT>
struct PcgBind {
  const CsrDev* A = nullptr;
  const JadDev* jad = nullptr;  // FP64 JAD path when set
  const VT* vals = nullptr;     // CSR values used by the iteration
  const double* verify_vals = nullptr;  // FP64 values for the final check (null: skip)
  const VT* b = nullptr;
  VT* x = nullptr;
  VT* r = nullptr;
  VT* p = nullptr;
  VT* q = nullptr;  // second direction buffer: the paired K3 (CSR, Jacobi only)
  VT* v = nullptr;
  const VT* J = nullptr;
  // block Jacobi (FP64 CSR only): inverse rows, block size, z = M r
  const double* bj = nullptr;
  int bs = 0;
  double* z = nullptr;
  // FP64 CSR sweeps read the 1-byte column offsets (A->ci8) instead of the
  // int32 columns: 9 instead of 12 bytes per non-zero
  bool dict = false;
};

// blockjacobi.cu: the block-Jacobi forms of the set-up and of K2/K3
int bj_pcg_setup_tail(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a);
int bj_pcg_update(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a);
int bj_pcg_direction(celg_handle* h, const PcgBind<double>& B, const PcgArgs& a);

int ensure_state(celg_handle* h, int hist_cap);
template <typename VT>
int pcg_run(celg_handle* h, const PcgBind<VT>& B, const celg_params* p, const void* mat,
            PcgState* out_state);
int copy_history(celg_handle* h, int len, celg_result* res);

template <typename VT>
__device__ __forceinline__ double D(VT v) { return (double)v; }
template <typename VT>
__device__ __forceinline__ VT R(double v) { return (VT)v; }

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle c, int v) {
  if (c) cudaGraphSetConditional(c, (unsigned)v);
}

__device__ __forceinline__ int pcg_go(const PcgState* st, int iter_max, const int* errw) {
  return (st->err == 0 && *(volatile const int*)errw == 0 && st->iter < iter_max &&
          fabs(st->alpha) > kRealSmall && st->norm > st->eps)
             ? 1
             : 0;
}

__device__ __forceinline__ void init_finish(const PcgArgs& a, double rp, double rr) {
  PcgState* st = a.st;
  st->alpha = rp;
  st->norm = sqrt(rr);
  st->iter = 0;
  if (a.hist && a.hist_cap > 0) a.hist[0] = st->norm;
  st->hist_len = 1;
  st->active = pcg_go(st, a.iter_max, a.errw);
  set_cond(a.cond, st->active);
}

// Kpre: x0 and ||b||, eps = max(eps_abs, eps_rel ||b||)
template <typename VT>
struct OpPre {
  static constexpr int NRED = 1;
  struct Regs { VT b; };
  const VT* b;
  VT* x;
  int x0_mode;
  double eps_abs, eps_rel;
  PcgArgs a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); }
  __device__ void compute(long i, Regs& g, double* acc) const {
    if (x0_mode == CELG_X0_REF_ONES) x[i] = VT(1);
    else if (x0_mode == CELG_X0_ZERO) x[i] = VT(0);
    acc[0] = dadd(acc[0], dmul(D(g.b), D(g.b)));
  }
  __device__ void finish(double* tot) const {
    PcgState* st = a.st;
    st->bnorm = sqrt(tot[0]);
    double e = eps_abs;
    if (eps_rel > 0.0 && eps_rel * st->bnorm > e) e = eps_rel * st->bnorm;
    st->eps = e;
    st->err = 0;
    st->iter = 0;
    st->active = 1;
    st->alpha = st->sigma = st->beta = st->pvd = st->rz = 0.0;
    st->vres = 0.0;
    st->xpend = 0;
    st->xprev = 0;
    st->sigprev = 0.0;
  }
};

// Kinit on CSR: r = b - (0 + A x); p = J r; alpha = r.p; rr = r.r
template <typename VT>
struct EpiInit {
  static constexpr int NRED = 2;
  const VT* b;
  VT* r;
  VT* p;
  const VT* J;
  PcgArgs a;
  __device__ bool active() const { return true; }
  __device__ void row(long i, VT s, double* acc) const {
    const VT ri = R<VT>(__dsub_rn(D(b[i]), D(vadd(VT(0), s))));
    r[i] = ri;
    const double z = dmul(D(ri), D(J[i]));
    p[i] = R<VT>(z);
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
  }
  __device__ void finish(double* tot) const { init_finish(a, tot[0], tot[1]); }
};

// Kinit tail on JAD (after r = A x by the JAD kernel), natural row order
template <typename VT>
struct OpInitNat {
  static constexpr int NRED = 2;
  struct Regs { VT b, r, J; };
  const VT* b;
  VT* r;
  VT* p;
  const VT* J;
  PcgArgs a;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); g.r = r[i]; g.J = __ldg(J + i); }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const VT ri = R<VT>(__dsub_rn(D(g.b), D(vadd(VT(0), g.r))));
    r[i] = ri;
    const double z = dmul(D(ri), D(g.J));
    p[i] = R<VT>(z);
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
  }
  __device__ void finish(double* tot) const { init_finish(a, tot[0], tot[1]); }
};

// K1: v = 0 + A p; pv = v.p; sigma = alpha / pv
template <typename VT>
struct EpiAp {
  static constexpr int NRED = 1;
  VT* v;
  const VT* p;
  PcgArgs a;
  __device__ bool active() const { return *(volatile int*)&a.st->active != 0; }
  // p(i) is loaded after the row's gathers: issued before them it cost 23 us
  // per 256^3 sweep (290 -> 267 us)
  __device__ void row(long i, VT s, double* acc) const {
    const VT vi = vadd(VT(0), s);
    v[i] = vi;
    acc[0] = dacc_prod(acc[0], vi, __ldg(p + i));
  }
  __device__ void finish(double* tot) const {
    PcgState* st = a.st;
    st->pvd = tot[0];
    const double sg = st->alpha / tot[0];
    st->sigma = sg;
    if (!isfinite(sg)) {
      st->err = kErrBreakdown;
      st->active = 0;
    }
  }
};

// K2: r += (-sigma) v; z = J r; rz, rr; scalars and stopping test.  The
// iteration's x += sigma p (:263-265) is left to K3, which reads the old p
// anyway, so this sweep reads neither x nor p; K2 marks it pending.  Each x
// element gets the same operation in the same iteration as before.
template <typename VT>
struct OpUpdate {
  static constexpr int NRED = 2;
  static constexpr int kTilesPerPass = sizeof(VT) == 4 ? 2 : 1;
  struct Regs { VT r, v, J; };
  VT* r;
  const VT* v;
  const VT* J;
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
  // v is not read again before the next update sweep: streamed (evict-first),
  // so that L2 keeps r and J for the direction sweep
  __device__ void load(long i, Regs& g) const {
    g.r = r[i];
    g.v = __ldcs(v + i);
    g.J = __ldg(J + i);
  }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const VT ri = R<VT>(dadd(D(g.r), dmul(-sg, D(g.v))));
    r[i] = ri;
    const double z = dmul(D(ri), D(g.J));
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
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
    st->xpend = 1;
    st->active = pcg_go(st, a.iter_max, a.errw);
    set_cond(a.cond, st->active);
  }
};

// K3 of the PCG: x += sigma p when K2 left it pending (also after K2 ended
// the solve), then p = beta p + J r (:282) while the solve goes on.  The
// last CTA clears the pending mark.
template <typename VT>
struct OpDirectionX {
  static constexpr int NRED = 0;
  static constexpr int kTilesPerPass = sizeof(VT) == 4 ? 2 : 1;
  static constexpr bool kFinishAlways = true;
  struct Regs { VT p, r, J, x; };
  VT* p;
  const VT* r;
  const VT* J;
  VT* x;
  PcgArgs a;
  double bt = 0.0, sg = 0.0;
  int xp = 0, act = 0;
  __device__ bool prepare() {
    xp = *(volatile int*)&a.st->xpend;
    act = *(volatile int*)&a.st->active;
    if (!xp && !act) return false;
    bt = a.st->beta;
    sg = a.st->sigma;
    return true;
  }
  // r, J and x are streamed (evict-first), so that L2 keeps the new p for
  // the next SpMV
  __device__ void load(long i, Regs& g) const {
    g.p = p[i];
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldcs(J + i);
    }
    if (xp) g.x = __ldcs(x + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    if (xp) __stcs(x + i, R<VT>(dadd(D(g.x), dmul(sg, D(g.p)))));
    if (act) p[i] = R<VT>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
  }
  __device__ void finish(double*) const { a.st->xpend = 0; }
};

// The paired form of K3 for two iterations, k (even sweep) and k+1 (odd
// sweep), whose directions live in two buffers: p_k in p, p_k+1 in q.  The
// even sweep writes p_k+1 = beta p_k + J r into q and leaves x += sigma_k p_k
// pending (xprev, sigprev); the odd sweep applies both updates to x in
// order, x = (x + sigma_k p_k) + sigma_k+1 p_k+1, and writes p_k+2 over p_k.
// x is read and stored once per two iterations instead of every iteration,
// and each element gets the same operations in the same order as with
// OpDirectionX.  When K2 ended the solve in the even iteration, the even
// sweep applies its own update at once.
template <typename VT>
struct OpDirectionDefer {
  static constexpr int NRED = 0;
  static constexpr int kTilesPerPass = sizeof(VT) == 4 ? 2 : 1;
  static constexpr bool kFinishAlways = true;
  struct Regs { VT p, r, J, x; };
  const VT* p;
  VT* q;
  const VT* r;
  const VT* J;
  VT* x;
  PcgArgs a;
  double bt = 0.0, sg = 0.0;
  int xp = 0, act = 0;
  __device__ bool prepare() {
    xp = *(volatile int*)&a.st->xpend;
    act = *(volatile int*)&a.st->active;
    if (!xp && !act) return false;
    bt = a.st->beta;
    sg = a.st->sigma;
    return true;
  }
  // p_k is read again by the odd sweep, after the SpMV and K2 of the next
  // iteration: streamed, so that L2 keeps the new direction for that SpMV
  __device__ void load(long i, Regs& g) const {
    g.p = __ldcs(p + i);
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldcs(J + i);
    } else if (xp) {
      g.x = __ldcs(x + i);
    }
  }
  __device__ void compute(long i, Regs& g, double*) const {
    if (act) q[i] = R<VT>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
    else if (xp) __stcs(x + i, R<VT>(dadd(D(g.x), dmul(sg, D(g.p)))));
  }
  __device__ void finish(double*) const {
    if (xp && act) {
      a.st->sigprev = sg;
      a.st->xprev = 1;
    }
    a.st->xpend = 0;
  }
};

template <typename VT>
struct OpDirectionPair {
  static constexpr int NRED = 0;
  static constexpr int kTilesPerPass = sizeof(VT) == 4 ? 2 : 1;
  static constexpr bool kFinishAlways = true;
  struct Regs { VT p, q, r, J, x; };
  VT* p;
  const VT* q;
  const VT* r;
  const VT* J;
  VT* x;
  PcgArgs a;
  double bt = 0.0, sg = 0.0, sp = 0.0;
  int xq = 0, xp = 0, act = 0;
  __device__ bool prepare() {
    xq = *(volatile int*)&a.st->xprev;
    xp = *(volatile int*)&a.st->xpend;
    act = *(volatile int*)&a.st->active;
    if (!xq && !xp && !act) return false;
    bt = a.st->beta;
    sg = a.st->sigma;
    sp = a.st->sigprev;
    return true;
  }
  __device__ void load(long i, Regs& g) const {
    if (xq) g.p = __ldcs(p + i);
    if (xp || act) g.q = q[i];
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldcs(J + i);
    }
    if (xq || xp) g.x = __ldcs(x + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    if (xq || xp) {
      VT xv = g.x;
      if (xq) xv = R<VT>(dadd(D(xv), dmul(sp, D(g.p))));
      if (xp) xv = R<VT>(dadd(D(xv), dmul(sg, D(g.q))));
      __stcs(x + i, xv);
    }
    if (act) p[i] = R<VT>(dadd(dmul(bt, D(g.q)), dmul(D(g.r), D(g.J))));
  }
  __device__ void finish(double*) const {
    a.st->xprev = 0;
    a.st->xpend = 0;
  }
};

// verification: ||b - A x|| / ||b|| (residual not stored)
struct EpiVerify {
  static constexpr int NRED = 1;
  const double* b;
  PcgState* st;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const {
    st->vres = st->bnorm > 0.0 ? sqrt(tot[0]) / st->bnorm : sqrt(tot[0]);
  }
};

struct OpVerifyNat {
  static constexpr int NRED = 1;
  struct Regs { double b, r; };
  const double* b;
  const double* r;
  PcgState* st;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); g.r = __ldg(r + i); }
  __device__ void compute(long, Regs& g, double* acc) const {
    const double ri = __dsub_rn(g.b, dadd(0.0, g.r));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const {
    st->vres = st->bnorm > 0.0 ? sqrt(tot[0]) / st->bnorm : sqrt(tot[0]);
  }
};

}  // namespace celg
