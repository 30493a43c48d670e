// batched.cu -- Jacobi-PCG on many independent systems of uneven size in one
// device-driven loop.
//
// The systems are concatenated into one block-diagonal CSR matrix, each
// system's rows padded to whole 1024-row tiles (padding rows are empty, with
// b = x = 0 and Jacobi 0), so that every tile belongs to one system.  Every
// system keeps its own scalars (alpha, sigma, beta, ||r||, iteration count,
// active flag) in device memory.  One CUDA graph runs
//   set-up sweeps, WHILE(any system active){K1, K2, K3}, verification
// over all tiles at once; the tiles of systems that converged are skipped,
// and each system's reductions are finished by the CTA that completes its
// last tile, in the same order as a single solve.  A system's result is
// therefore bit-identical to solving it alone with celg_pcg_jacobi, while the
// small systems no longer leave most of the GPU idle and the per-iteration
// launch cost is paid once for the whole batch.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "graph.cuh"
#include "pcg_internal.cuh"

namespace celg {

struct BatchArgs {
  double *alpha, *sigma, *beta, *norm, *bnorm, *eps, *vres;
  int *iter, *active, *err, *n_active;
  int* xpend;  // per system: the update sweep ran, the direction sweep owes x += sigma p
  // paired direction sweeps (FP64 solve only; null otherwise): the odd
  // sweep owes x += sigprev p_k from the even one
  int* xprev;
  double* sigprev;
  BatchRed br;
  int nsys;
  int nlive;  // systems with rows (empty systems are never active)
  int iter_max;
  cudaGraphConditionalHandle cond;
  const int* errw;
  __device__ int go(int s) const {
    return (err[s] == 0 && *(volatile const int*)errw == 0 && iter[s] < iter_max &&
            fabs(alpha[s]) > kRealSmall && norm[s] > eps[s])
               ? 1
               : 0;
  }
  __device__ void settle(int s) const {
    const int g = go(s);
    active[s] = g;
    if (!g) atomicSub(n_active, 1);
  }
  __device__ int sys_of(long t) const { return br.tile_sys[t]; }
};

// x0, ||b|| and eps per system.  With `part` set (the refinement's inner
// solves) only the systems with part[s] != 0 take part; n_active is then
// *part_count.
template <typename VT>
struct BOpPre {
  static constexpr int NRED = 1;
  static constexpr bool kBatched = true;
  struct Regs { VT b; };
  const VT* b;
  VT* x;
  int x0_mode;
  double eps_abs, eps_rel;
  BatchArgs a;
  const int* part = nullptr;
  const int* part_count = nullptr;
  const double* eps_rel_sys = nullptr;  // per-system eps_rel (refinement inner solves)
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long) const { return TileInfo{1, 0.0}; }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int) const { return true; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); }
  __device__ void compute(long i, Regs& g, double* acc) const {
    if (x0_mode == CELG_X0_REF_ONES) x[i] = VT(1);
    else if (x0_mode == CELG_X0_ZERO) x[i] = VT(0);
    acc[0] = dadd(acc[0], dmul(D(g.b), D(g.b)));
  }
  __device__ void finish_sys(int s, double* tot) const {
    a.xpend[s] = 0;
    if (a.xprev) a.xprev[s] = 0;
    a.bnorm[s] = sqrt(tot[0]);
    double e = eps_abs;
    const double er = eps_rel_sys ? eps_rel_sys[s] : eps_rel;
    if (er > 0.0 && er * a.bnorm[s] > e) e = er * a.bnorm[s];
    a.eps[s] = e;
    a.err[s] = 0;
    a.iter[s] = 0;
    a.active[s] = part ? (part[s] ? 1 : 0) : 1;
    a.vres[s] = 0.0;
  }
  __device__ void finish_global() const { *a.n_active = part_count ? *part_count : a.nlive; }
};

// r = b - (0 + A x); p = J r; alpha = r.p; ||r||  (systems set active by BOpPre)
template <typename VT>
struct BEpiInit {
  static constexpr int NRED = 2;
  static constexpr bool kBatched = true;
  const VT* b;
  VT* r;
  VT* p;
  const VT* J;
  BatchArgs a;
  __device__ bool active() const { return true; }
  __device__ TileInfo tile_info(long t) const {
    return TileInfo{*(volatile int*)&a.active[a.sys_of(t)], 0.0};
  }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int s) const { return *(volatile int*)&a.active[s] != 0; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void row(long i, VT s, double* acc) const {
    const VT ri = R<VT>(__dsub_rn(D(b[i]), D(vadd(VT(0), s))));
    r[i] = ri;
    const double z = dmul(D(ri), D(J[i]));
    p[i] = R<VT>(z);
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
  }
  __device__ void finish_sys(int s, double* tot) const {
    a.alpha[s] = tot[0];
    a.norm[s] = sqrt(tot[1]);
    a.iter[s] = 0;
    a.settle(s);
  }
  __device__ void finish_global() const { set_cond(a.cond, *(volatile int*)a.n_active > 0); }
};

// K1: v = 0 + A p; pv = v.p; sigma = alpha / pv
template <typename VT>
struct BEpiAp {
  static constexpr int NRED = 1;
  static constexpr bool kBatched = true;
  VT* v;
  const VT* p;
  BatchArgs a;
  __device__ bool active() const { return *(volatile int*)a.n_active > 0; }
  __device__ TileInfo tile_info(long t) const {
    return TileInfo{*(volatile int*)&a.active[a.sys_of(t)], 0.0};
  }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int s) const { return *(volatile int*)&a.active[s] != 0; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void row(long i, VT s, double* acc) const {
    const VT vi = vadd(VT(0), s);
    v[i] = vi;
    acc[0] = dadd(acc[0], dmul(D(vi), D(__ldg(p + i))));
  }
  __device__ void finish_sys(int s, double* tot) const {
    const double sg = a.alpha[s] / tot[0];
    a.sigma[s] = sg;
    if (!isfinite(sg)) {
      a.err[s] = kErrBreakdown;
      a.active[s] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {}
};

// K2: r += (-sigma) v; rz, rr; scalars and per-system test.  The system's
// x += sigma p is left to the direction sweep, which reads the old p anyway
// (xpend[s]), so this sweep reads neither x nor p.
template <typename VT>
struct BOpUpdate {
  static constexpr int NRED = 2;
  static constexpr bool kBatched = true;
  struct Regs { VT r, v, J; };
  VT* r;
  const VT* v;
  const VT* J;
  BatchArgs a;
  double sg;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    return TileInfo{*(volatile int*)&a.active[s], a.sigma[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) { sg = ti.s; }
  __device__ bool sys_active(int s) const { return *(volatile int*)&a.active[s] != 0; }
  __device__ const BatchRed& bred() const { return a.br; }
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
  __device__ void finish_sys(int s, double* tot) const {
    a.beta[s] = tot[0] / a.alpha[s];
    a.alpha[s] = tot[0];
    a.norm[s] = sqrt(tot[1]);
    a.iter[s] += 1;
    a.xpend[s] = 1;
    a.settle(s);
  }
  __device__ void finish_global() const { set_cond(a.cond, *(volatile int*)a.n_active > 0); }
};

// K3: the direction sweeps for a pair of iterations whose directions live
// in two vectors, p_k in p and p_k+1 in q (FP64 solve, FP32 inner solves).
// The even sweep writes p_k+1 = beta p_k + J r into q; a system that goes
// on keeps its x += sigma_k p_k pending (defer_marks_kernel moves the mark
// to xprev with sigma_k), and a system that the update sweep just stopped
// gets its update at once.  The odd sweep applies x = (x + sigma_k p_k) +
// sigma_k+1 p_k+1 and writes p_k+2 over p_k.  x is read and stored once per
// two iterations, and each element gets the same roundings in the same
// order as two consecutive x += sigma p.
// TileInfo.act of the odd sweep: bit 0 active, bit 1 x pending, bit 2 the
// even iteration's update pending; s = beta, s2 = sigma, s3 = sigma_k.
template <typename VT>
struct BOpDirectionDefer {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { VT p, r, J, x; };
  const VT* p;
  VT* q;
  const VT* r;
  const VT* J;
  VT* x;
  BatchArgs a;
  double bt = 0.0, sg = 0.0;
  int act = 0, xp = 0;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    const int f = (*(volatile int*)&a.active[s] != 0 ? 1 : 0) |
                  (*(volatile int*)&a.xpend[s] != 0 ? 2 : 0);
    return TileInfo{f, a.beta[s], a.sigma[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) {
    act = ti.act & 1;
    xp = ti.act & 2;
    bt = ti.s;
    sg = ti.s2;
  }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  // p_k is read again by the odd sweep, after the next SpMV: streamed
  __device__ void load(long i, Regs& g) const {
    g.p = __ldcs(p + i);
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldg(J + i);
    } else if (xp) {
      g.x = __ldcs(x + i);
    }
  }
  __device__ void compute(long i, Regs& g, double*) const {
    if (act) q[i] = R<VT>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
    else if (xp) __stcs(x + i, R<VT>(dadd(D(g.x), dmul(sg, D(g.p)))));
  }
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

template <typename VT>
struct BOpDirectionPair {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { VT p, q, r, J, x; };
  VT* p;
  const VT* q;
  const VT* r;
  const VT* J;
  VT* x;
  BatchArgs a;
  double bt = 0.0, sg = 0.0, sp = 0.0;
  int act = 0, xp = 0, xq = 0;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    const int f = (*(volatile int*)&a.active[s] != 0 ? 1 : 0) |
                  (*(volatile int*)&a.xpend[s] != 0 ? 2 : 0) |
                  (*(volatile int*)&a.xprev[s] != 0 ? 4 : 0);
    return TileInfo{f, a.beta[s], a.sigma[s], a.sigprev[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) {
    act = ti.act & 1;
    xp = ti.act & 2;
    xq = ti.act & 4;
    bt = ti.s;
    sg = ti.s2;
    sp = ti.s3;
  }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const {
    if (xq) g.p = __ldcs(p + i);
    if (xp || act) g.q = __ldcs(q + i);
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldg(J + i);
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
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

// After the even sweep: a system whose update is still pending and that goes
// on owes it to the odd sweep (xprev, sigprev); every xpend mark is cleared.
__global__ void defer_marks_kernel(int count, int* xpend, int* xprev, const int* active,
                                   const double* sigma, double* sigprev) {
  for (int s = threadIdx.x; s < count; s += blockDim.x) {
    const int d = xpend[s] != 0 && active[s] != 0;
    if (d) sigprev[s] = sigma[s];
    xprev[s] = d;
    xpend[s] = 0;
  }
}

__global__ void clear_marks_kernel(int* marks, int count) {
  for (int s = threadIdx.x; s < count; s += blockDim.x) marks[s] = 0;
}

// ||b - A x|| / ||b|| per system
struct BEpiVerify {
  static constexpr int NRED = 1;
  static constexpr bool kBatched = true;
  const double* b;
  BatchArgs a;
  __device__ bool active() const { return true; }
  __device__ TileInfo tile_info(long) const { return TileInfo{1, 0.0}; }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int) const { return true; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish_sys(int s, double* tot) const {
    a.vres[s] = a.bnorm[s] > 0.0 ? sqrt(tot[0]) / a.bnorm[s] : sqrt(tot[0]);
  }
  __device__ void finish_global() const {}
};

// ---- FP32 refinement of every system (celg_pcg_batched, CELG_PREC_FP32_IR) -------
//
// The outer loop of ir_solve (ir.cu) run for all systems at once: each
// system keeps its own residual norm, outer count and status, and the outer
// steps of the systems that are still refining advance together.

struct IrState {
  int* part;         // system needs an inner solve in this outer step
  int* done;         // system finished (status set)
  int* status;       // CELG_OK / CELG_ERR_* per system
  int* outer;        // completed outer steps
  int* inner_total;  // inner iterations over all outer steps
  int* part_count;
  int outer_max;
  double* tau_sys;   // inner tolerance of the system's next inner solve
  double tau;        // inner_eps_rel
};

// r = b - (0 + A x) in FP64, ||r|| per system; the system's outer decision
struct BEpiIrResidual {
  static constexpr int NRED = 1;
  static constexpr bool kBatched = true;
  const double* b;
  double* r;
  BatchArgs a;  // outer state: norm[s] = ||r||, eps[s] = tolerance
  IrState ir;
  __device__ bool active() const { return true; }
  __device__ TileInfo tile_info(long t) const {
    return TileInfo{*(volatile int*)&ir.done[a.sys_of(t)] == 0 ? 1 : 0, 0.0};
  }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int s) const { return *(volatile int*)&ir.done[s] == 0; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = __dsub_rn(b[i], dadd(0.0, s));
    r[i] = ri;
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish_sys(int s, double* tot) const {
    const double rn = sqrt(tot[0]);
    a.norm[s] = rn;
    int st = -1;
    if (rn <= a.eps[s]) st = CELG_OK;
    else if (!isfinite(rn)) st = kErrBreakdown;
    else if (ir.outer[s] >= ir.outer_max) st = CELG_ERR_NOCONV;
    if (st >= 0) {
      ir.done[s] = 1;
      ir.status[s] = st;
    } else {
      ir.part[s] = 1;
      ir.tau_sys[s] = ir_step_tolerance(rn, a.eps[s], ir.tau);
      atomicAdd(ir.part_count, 1);
    }
  }
  __device__ void finish_global() const {}
};

// r32 = (float)(r * (1/||r||)) for the systems that refine
struct BOpIrToF32 {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { double r; };
  const double* r;
  float* r32;
  BatchArgs a;
  IrState ir;
  double inv;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    return TileInfo{*(volatile int*)&ir.part[s], 1.0 / a.norm[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) { inv = ti.s; }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const { g.r = __ldg(r + i); }
  __device__ void compute(long i, Regs& g, double*) const { r32[i] = (float)dmul(g.r, inv); }
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

// x = x + ||r|| * (double) d32 for the systems that refined
struct BOpIrAdd {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { double x; float d; };
  double* x;
  const float* d;
  BatchArgs a;
  IrState ir;
  double scale;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    return TileInfo{*(volatile int*)&ir.part[s], a.norm[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) { scale = ti.s; }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const { g.x = x[i]; g.d = __ldg(d + i); }
  __device__ void compute(long i, Regs& g, double*) const { x[i] = dadd(g.x, dmul(scale, (double)g.d)); }
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

// after an inner solve (before the update): count the inner iterations; an
// inner failure other than the iteration cap ends the system with that
// status and without the update, otherwise the outer step counts
__global__ void ir_count_kernel(int nsys, IrState ir, const int* inner_iter, const int* inner_err) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x) {
    if (!ir.part[s]) continue;
    ir.inner_total[s] += inner_iter[s];
    if (inner_err[s] != 0) {
      ir.done[s] = 1;
      ir.status[s] = inner_err[s];
      ir.part[s] = 0;
    } else {
      ir.outer[s] += 1;
    }
  }
}

// ---- completion of a batched sweep ------------------------------------------------

// ---- FP32 PCG with FP64 reliable updates of every system (CELG_PREC_FP32_RU) ---
// The recurrence of ru_solve (ru.cu) for all systems at once: one FP32 SpMV
// and vector sweep pair per iteration over the concatenated systems, and the
// FP64 correction of the systems that are due, under one IF node.  Each
// system's reductions are the single solve's (per-system finishers), so each
// system's result equals ru_solve on it alone, bit for bit.

struct BatchRu {
  double* maxr;     // ||r64|| at the system's last reliable update
  double* rz_prev;  // rz before the system's current step
  double* norm64;   // the system's last FP64 residual norm
  int* updates;     // reliable updates so far (the set-up residual included)
  int* upd;         // the system's reliable update is due
  int* n_upd;       // some system's update is due
  double delta;
  cudaGraphConditionalHandle cond_update;  // IF node of the update (0: none)
};

__device__ __forceinline__ int bru_go(const BatchArgs& a, const BatchRu& u, int s) {
  return (a.err[s] == 0 && *(volatile const int*)a.errw == 0 && a.iter[s] < a.iter_max &&
          u.norm64[s] > a.eps[s])
             ? 1
             : 0;
}

// set-up: every system with rows starts with a reliable update
__global__ void bru_init_kernel(int nsys, const int* sys_ntiles, BatchRu u) {
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    u.updates[s] = 0;
    u.upd[s] = sys_ntiles[s] > 0 ? 1 : 0;
  }
  if (threadIdx.x == 0) *u.n_upd = 1;
}

// the flushed systems owe no d += sigma p any more
__global__ void bru_clear_kernel(int nsys, int* xpend, const int* upd) {
  for (int s = threadIdx.x; s < nsys; s += blockDim.x)
    if (upd[s]) xpend[s] = 0;
}

// FP64 residual of the systems due for an update, and its FP32 copy:
//   r64 = b - (0 + A x);  r = (float) r64;  z = (double) r * J;  rz = r.z;  ||r64||^2
// init: also p = (float) z.
struct BEpiRuResidual {
  static constexpr int NRED = 2;
  static constexpr bool kBatched = true;
  const double* b;
  float* r;
  float* p;  // set-up only
  const float* J;
  BatchArgs a;
  BatchRu u;
  int init;
  __device__ bool active() const { return *(volatile int*)u.n_upd != 0; }
  __device__ TileInfo tile_info(long t) const {
    return TileInfo{*(volatile int*)&u.upd[a.sys_of(t)], 0.0};
  }
  __device__ void begin_tile(const TileInfo&) {}
  __device__ bool sys_active(int s) const { return *(volatile int*)&u.upd[s] != 0; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void row(long i, double s, double* acc) const {
    const double r64 = __dsub_rn(b[i], dadd(0.0, s));
    const float rf = (float)r64;
    r[i] = rf;
    const double z = dmul((double)rf, (double)J[i]);
    if (init) p[i] = (float)z;
    acc[0] = dadd(acc[0], dmul((double)rf, z));
    acc[1] = dadd(acc[1], dmul(r64, r64));
  }
  __device__ void finish_sys(int s, double* tot) const {
    u.norm64[s] = sqrt(tot[1]);
    u.maxr[s] = u.norm64[s];
    u.upd[s] = 0;
    u.updates[s] += 1;
    if (init) {
      a.alpha[s] = tot[0];
      a.norm[s] = u.norm64[s];
    } else {
      a.beta[s] = tot[0] / u.rz_prev[s];
      a.alpha[s] = tot[0];
    }
    if (!bru_go(a, u, s) && a.active[s]) {
      a.active[s] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {
    *u.n_upd = 0;
    set_cond(a.cond, *(volatile int*)a.n_active > 0);
  }
};

// r -= sigma v in FP32 arithmetic; rz' = r.J r, ||r||^2; the system's update
// decision.  d += sigma p is left pending (xpend) for the flush or the
// direction sweep.
struct BOpRuStep {
  static constexpr int NRED = 2;
  static constexpr bool kBatched = true;
  struct Regs { float r, v, J; };
  float* r;
  const float* v;
  const float* J;
  BatchArgs a;
  BatchRu u;
  float nsg = 0.0f;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    return TileInfo{*(volatile int*)&a.active[s], a.sigma[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) { nsg = (float)(-ti.s); }
  __device__ bool sys_active(int s) const { return *(volatile int*)&a.active[s] != 0; }
  __device__ const BatchRed& bred() const { return a.br; }
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
  __device__ void finish_sys(int s, double* tot) const {
    u.rz_prev[s] = a.alpha[s];
    a.beta[s] = tot[0] / a.alpha[s];
    a.alpha[s] = tot[0];
    a.norm[s] = sqrt(tot[1]);
    a.iter[s] += 1;
    a.xpend[s] = 1;
    const int upd = (a.norm[s] < u.delta * u.maxr[s]) || (a.norm[s] <= a.eps[s]) ||
                    (a.iter[s] >= a.iter_max);
    if (upd) {
      u.upd[s] = 1;
      atomicAdd(u.n_upd, 1);
    } else if (!(a.err[s] == 0 && *(volatile const int*)a.errw == 0 && a.iter[s] < a.iter_max &&
                 fabs(a.alpha[s]) > 0.0)) {
      a.active[s] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {
    set_cond(u.cond_update, *(volatile int*)u.n_upd > 0);
    set_cond(a.cond, *(volatile int*)a.n_active > 0);
  }
};

// x64 += (double) d ; d = 0 for the systems due for an update (every system
// with `always`).  A pending d += sigma p is applied first, with the step's
// rounding.  TileInfo.act: bit 0 flush, bit 1 d += sigma p pending.
struct BOpRuFlush {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { double x; float d, p; };
  double* x;
  float* d;
  const float* p;  // null: nothing pending (the final flush)
  BatchArgs a;
  BatchRu u;
  int always;
  int dp = 0;
  double sg = 0.0;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    const int f = (always || *(volatile int*)&u.upd[s] != 0 ? 1 : 0) |
                  (p != nullptr && *(volatile int*)&a.xpend[s] != 0 ? 2 : 0);
    return TileInfo{f & 1 ? f : 0, a.sigma[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) {
    dp = ti.act & 2;
    sg = ti.s;
  }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const {
    g.x = x[i];
    g.d = d[i];
    if (dp) g.p = __ldg(p + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    const float di = dp ? (float)dadd((double)g.d, dmul(sg, (double)g.p)) : g.d;
    x[i] = dadd(g.x, (double)di);
    d[i] = 0.0f;
  }
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

// d += sigma p where the step left it pending, then p = beta p + J r while
// the system goes on (TileInfo.act: bit 0 active, bit 1 pending; s = beta,
// s2 = sigma).  The marks are cleared by clear_marks_kernel after the sweep.
struct BOpRuDirection {
  static constexpr int NRED = 0;
  static constexpr bool kBatched = true;
  struct Regs { float p, r, J, d; };
  float* p;
  const float* r;
  const float* J;
  float* d;
  BatchArgs a;
  double bt = 0.0, sg = 0.0;
  int act = 0, dp = 0;
  __device__ bool prepare() { return true; }
  __device__ TileInfo tile_info(long t) const {
    const int s = a.sys_of(t);
    const int f = (*(volatile int*)&a.active[s] != 0 ? 1 : 0) |
                  (*(volatile int*)&a.xpend[s] != 0 ? 2 : 0);
    return TileInfo{f, a.beta[s], a.sigma[s]};
  }
  __device__ void begin_tile(const TileInfo& ti) {
    act = ti.act & 1;
    dp = ti.act & 2;
    bt = ti.s;
    sg = ti.s2;
  }
  __device__ bool sys_active(int) const { return false; }
  __device__ const BatchRed& bred() const { return a.br; }
  __device__ void load(long i, Regs& g) const {
    g.p = p[i];
    if (act) {
      g.r = __ldcs(r + i);
      g.J = __ldg(J + i);
    }
    if (dp) g.d = __ldcs(d + i);
  }
  __device__ void compute(long i, Regs& g, double*) const {
    if (dp) __stcs(d + i, (float)dadd((double)g.d, dmul(sg, (double)g.p)));
    if (act) p[i] = R<float>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
  }
  __device__ void finish_sys(int, double*) const {}
  __device__ void finish_global() const {}
};

// One CTA per system: if the system took part, its tile partials are reduced
// in the single-solve order (lane j sums partials j, j+256, ... from 0.0;
// butterfly; warps in order) and finish_sys runs; the last CTA to arrive
// runs finish_global.
template <int NRED, class Op>
__global__ void __launch_bounds__(kLanes) batch_finish_kernel(Op op, RedCtx red) {
  __shared__ double scratch[8];
  __shared__ int s_flag;
  const int s = blockIdx.x;
  const int tid = threadIdx.x;
  const BatchRed& br = op.bred();
  const long nt = br.sys_ntiles[s];
  if (nt > 0 && op.sys_active(s)) {
    double tot[NRED];
    const long t0 = br.sys_tile0[s];
#pragma unroll
    for (int r = 0; r < NRED; ++r) {
      double acc = 0.0;
      const double* p = red.partials + (long)r * red.ntiles + t0;
      for (long k = tid; k < nt; k += kLanes) acc = dadd(acc, __ldcg(p + k));
      tot[r] = group_fold256(acc, scratch, tid, 1);
    }
    if (tid == 0) op.finish_sys(s, tot);
  }
  if (tid == 0) {
    __threadfence();
    const unsigned tk = atomicAdd(red.ticket, 1u);
    s_flag = (tk == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (s_flag && tid == 0) {
    __threadfence();
    op.finish_global();
    *red.ticket = 0u;
  }
}

// ---- concatenation ------------------------------------------------------------

__global__ void batch_rows_kernel(int n, int pad, const int* __restrict__ rp_s, const double* __restrict__ J_s,
                                  int nnz_off, int nnz_s, int* __restrict__ rp_d, double* __restrict__ J_d) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < pad; i += (long)gridDim.x * blockDim.x) {
    rp_d[i] = i <= n ? rp_s[i] + nnz_off : nnz_off + nnz_s;
    J_d[i] = i < n ? J_s[i] : 0.0;
  }
}

__global__ void batch_cols_kernel(long nnz, const int* __restrict__ ci_s, int row_off,
                                  int* __restrict__ ci_d) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x)
    ci_d[k] = ci_s[k] + row_off;
}

__global__ void fill_int_kernel(long n, int v, int* __restrict__ a) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = v;
}

}  // namespace celg

struct Batch {
  std::string key;
  int nsys = 0;
  long N = 0, NT = 0;
  celg::CsrDev A;
  double* J = nullptr;
  double *B = nullptr, *X = nullptr, *R = nullptr, *P = nullptr, *V = nullptr;
  int* tile_arrays = nullptr;  // tile_sys[NT], sys_tile0[nsys], sys_ntiles[nsys]
  unsigned* sys_ticket = nullptr;
  double* dstate = nullptr;    // 8 x nsys doubles
  int* istate = nullptr;       // 3 x nsys ints + n_active + 2 x nsys pending marks
  double* Q = nullptr;         // second direction of the paired FP64 sweeps
  int nlive = 0;               // systems with at least one row
  // launch shape picked by batch_tune (index into kBatchShapes, -1: not tuned)
  int shape = -1;
  std::vector<long> row_off;
  std::vector<int> n;
  // FP32 refinement (allocated on first use): A.v32 holds the FP32 values
  float* J32 = nullptr;
  float* F = nullptr;          // 5 x N floats: B32 D32 R32 P32 V32
  int* irs = nullptr;          // part, done, status, outer, inner_total (nsys each), part_count
  double* irtau = nullptr;     // inner tolerance per system
  double* dstate2 = nullptr;   // inner-solve scalars, 7 x nsys
  int* istate2 = nullptr;      // inner-solve counters, 4 x nsys + 1
  // FP32 with reliable updates: maxr, rz_prev, norm64 (nsys each); updates,
  // upd (nsys each), n_upd
  double* rud = nullptr;
  int* rui = nullptr;
};

namespace celg {

void batch_free(Batch* b) {
  if (!b) return;
  cudaFree(b->A.rp);
  cudaFree(b->A.ci);
  cudaFree(b->A.v);
  cudaFree(b->A.ci8);
  cudaFree(b->A.pid);
  cudaFree(b->A.pat);
  cudaFree(b->A.dict);
  cudaFree(b->J);
  cudaFree(b->B);
  cudaFree(b->tile_arrays);
  cudaFree(b->sys_ticket);
  cudaFree(b->dstate);
  cudaFree(b->istate);
  cudaFree(b->A.v32);
  cudaFree(b->J32);
  cudaFree(b->F);
  cudaFree(b->irs);
  cudaFree(b->irtau);
  cudaFree(b->dstate2);
  cudaFree(b->istate2);
  cudaFree(b->rud);
  cudaFree(b->rui);
  delete b;
}

static int ew(celg_handle* h, long n) {
  return (int)std::max(1L, std::min((n + 255) / 256, (long)h->sms * 16));
}

static int batch_build(celg_handle* h, int count, celg_mat* const* mats, const std::string& key,
                       Batch** out) {
  Batch* bt = new Batch();
  bt->key = key;
  bt->nsys = count;
  bt->row_off.resize(count);
  bt->n.resize(count);
  long N = 0, NNZ = 0;
  std::vector<long> nnz_off(count);
  for (int s = 0; s < count; ++s) {
    bt->row_off[s] = N;
    nnz_off[s] = NNZ;
    bt->n[s] = mats[s]->csr.n;
    N += ((long)mats[s]->csr.n + kTile - 1) / kTile * kTile;
    NNZ += mats[s]->csr.nnz;
    if (mats[s]->csr.n > 0) bt->nlive++;
  }
  if (N >= (1L << 31) || NNZ >= (1L << 31)) {
    delete bt;
    return CELG_ERR_ARG;
  }
  bt->N = N;
  bt->NT = N / kTile;
  CsrDev& A = bt->A;
  A.n = (int)N;
  A.ncols = (int)N;
  A.nnz = (int)NNZ;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; return e == cudaSuccess; };
  ok(cudaMalloc(&A.rp, sizeof(int) * ((size_t)N + 1 + 8)));
  ok(cudaMalloc(&A.ci, sizeof(int) * ((size_t)NNZ + 8)));
  ok(cudaMalloc(&A.v, sizeof(double) * ((size_t)NNZ + 8)));
  ok(cudaMalloc(&bt->J, sizeof(double) * std::max<size_t>(N, 1)));
  ok(cudaMalloc(&bt->B, sizeof(double) * std::max<size_t>(N, 1) * 6));
  ok(cudaMalloc(&bt->tile_arrays, sizeof(int) * ((size_t)bt->NT + 2 * (size_t)count + 1)));
  ok(cudaMalloc(&bt->sys_ticket, sizeof(unsigned) * (size_t)count));
  ok(cudaMalloc(&bt->dstate, sizeof(double) * 8 * (size_t)count));
  ok(cudaMalloc(&bt->istate, sizeof(int) * (5 * (size_t)count + 1)));
  if (e != cudaSuccess) {
    batch_free(bt);
    return cuda_status(e, "batch allocation");
  }
  bt->X = bt->B + N;
  bt->R = bt->X + N;
  bt->P = bt->R + N;
  bt->V = bt->P + N;
  bt->Q = bt->V + N;
  ok(cudaMemsetAsync(bt->B, 0, sizeof(double) * (size_t)N * 6, h->stream));
  ok(cudaMemsetAsync(A.ci + NNZ, 0, sizeof(int) * 8, h->stream));
  ok(cudaMemsetAsync(A.v + NNZ, 0, sizeof(double) * 8, h->stream));
  ok(cudaMemsetAsync(bt->sys_ticket, 0, sizeof(unsigned) * (size_t)count, h->stream));
  for (int s = 0; s < count && e == cudaSuccess; ++s) {
    const celg_mat* m = mats[s];
    const long pad = ((long)m->csr.n + kTile - 1) / kTile * kTile;
    if (pad > 0)
      batch_rows_kernel<<<ew(h, pad), 256, 0, h->stream>>>(m->csr.n, (int)pad, m->csr.rp, m->jacobi,
                                                           (int)nnz_off[s], m->csr.nnz,
                                                           A.rp + bt->row_off[s], bt->J + bt->row_off[s]);
    if (m->csr.nnz > 0) {
      batch_cols_kernel<<<ew(h, m->csr.nnz), 256, 0, h->stream>>>(m->csr.nnz, m->csr.ci,
                                                                 (int)bt->row_off[s], A.ci + nnz_off[s]);
      ok(cudaMemcpyAsync(A.v + nnz_off[s], m->csr.v, sizeof(double) * (size_t)m->csr.nnz,
                         cudaMemcpyDeviceToDevice, h->stream));
    }
    ok(cudaGetLastError());
  }
  fill_int_kernel<<<1, 32, 0, h->stream>>>(9, (int)NNZ, A.rp + N);  // rp[N] and the padded tail
  std::vector<int> tiles((size_t)bt->NT + 2 * (size_t)count);
  long t = 0;
  for (int s = 0; s < count; ++s) {
    const long nt = ((long)mats[s]->csr.n + kTile - 1) / kTile;
    tiles[(size_t)bt->NT + s] = (int)t;
    tiles[(size_t)bt->NT + count + s] = (int)nt;
    for (long k = 0; k < nt; ++k) tiles[(size_t)(t + k)] = s;
    t += nt;
  }
  ok(cudaMemcpyAsync(bt->tile_arrays, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice,
                     h->stream));
  ok(cudaStreamSynchronize(h->stream));
  if (e != cudaSuccess) {
    batch_free(bt);
    return cuda_status(e, "batch assembly");
  }
  int st = csr_compute_cap(h, A);
  // 1-byte column offsets when the systems together use at most 256
  // distinct offsets col - row (7-point systems: -1, 0, 1 and +-side,
  // +-side^2 per distinct side): 9 instead of 12 bytes per non-zero
  if (!st) st = build_offset_dict_csr(h, A);
  if (st) {
    batch_free(bt);
    return st;
  }
  *out = bt;
  return CELG_OK;
}

// Launch shapes the batch tuner chooses from: resident CTAs per SM of the
// CSR sweep (0: as many as fit) and of the vector sweeps.  None changes a
// result: every tile is reduced on its own, whichever CTA takes it.
struct BatchShape {
  int csr_per_sm, tile_per_sm;
};
constexpr BatchShape kBatchShapes[] = {{0, 8}, {0, 6}, {0, 4}, {2, 8}, {2, 4}, {1, 8}};
constexpr int kNumBatchShapes = (int)(sizeof(kBatchShapes) / sizeof(kBatchShapes[0]));

static BatchShape batch_shape(const Batch* bt) {
  return kBatchShapes[bt->shape >= 0 && bt->shape < kNumBatchShapes ? bt->shape : 0];
}

// A CSR sweep over the concatenated systems, with the 1-byte column offsets
// when the batch has them (same values in the same order, same sums).
template <typename VT, class Epi>
static int batch_csr(celg_handle* h, const Batch* bt, const VT* vals, const VT* x, const Epi& epi) {
  const int cap = batch_shape(bt).csr_per_sm;
  bool done = false;
  const int st = launch_csr_compact<VT>(h, bt->A, vals, x, epi, nullptr, cap, &done);
  if (done) return st;
  return launch_csr_ct<VT, int>(h, bt->A, vals, bt->A.ci, bt->A.cap, x, epi, nullptr, cap);
}

// A vector sweep over the concatenated systems.
template <class Op>
static int batch_tile(celg_handle* h, const Batch* bt, const Op& op) {
  return launch_tile(h, bt->N, op, batch_shape(bt).tile_per_sm);
}

static BatchArgs batch_args(Batch* bt, int iter_max, cudaGraphConditionalHandle cond, const int* errw,
                            bool inner = false) {
  BatchArgs a;
  const int c = bt->nsys;
  a.alpha = inner ? bt->dstate2 : bt->dstate;
  a.sigma = a.alpha + c;
  a.beta = a.sigma + c;
  a.norm = a.beta + c;
  a.bnorm = a.norm + c;
  a.eps = a.bnorm + c;
  a.vres = a.eps + c;
  a.iter = inner ? bt->istate2 : bt->istate;
  a.active = a.iter + c;
  a.err = a.active + c;
  a.n_active = a.err + c;
  a.xpend = a.n_active + 1;
  a.xprev = a.xpend + c;
  a.sigprev = a.vres + c;
  a.br.tile_sys = bt->tile_arrays;
  a.br.sys_tile0 = bt->tile_arrays + bt->NT;
  a.br.sys_ntiles = bt->tile_arrays + bt->NT + c;
  a.br.sys_ticket = bt->sys_ticket;
  a.nsys = c;
  a.nlive = bt->nlive;
  a.iter_max = iter_max;
  a.cond = cond;
  a.errw = errw;
  return a;
}

// The solve as recorded into the graph; with a.cond == 0 (profiling mode,
// CELG_GRAPH=0) the loop body is instead launched from the host in chunks of
// 8 iterations between reads of the live-system count.
template <class Op>
static int batch_finish(celg_handle* h, const Batch* bt, const Op& op) {
  RedCtx red{h->partials, h->ticket, bt->NT};
  batch_finish_kernel<Op::NRED, Op><<<bt->nsys, kLanes, 0, h->stream>>>(op, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

static int clear_marks(celg_handle* h, const BatchArgs& a) {
  clear_marks_kernel<<<1, kLanes, 0, h->stream>>>(a.xpend, a.nsys);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// The direction sweep of the even (odd = false) or odd iteration of a pair,
// with the marks moved or cleared after it (xpend and xprev are adjacent).
template <typename VT>
static int batch_direction_pair(celg_handle* h, const Batch* bt, const BatchArgs& a, bool odd, VT* P,
                                VT* Q, const VT* R, const VT* J, VT* X) {
  if (!odd) {
    const int st = batch_tile(h, bt, BOpDirectionDefer<VT>{P, Q, R, J, X, a});
    if (st) return st;
    defer_marks_kernel<<<1, kLanes, 0, h->stream>>>(a.nsys, a.xpend, a.xprev, a.active, a.sigma,
                                                    a.sigprev);
  } else {
    const int st = batch_tile(h, bt, BOpDirectionPair<VT>{P, Q, R, J, X, a});
    if (st) return st;
    clear_marks_kernel<<<1, kLanes, 0, h->stream>>>(a.xpend, 2 * a.nsys);
  }
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// x0, ||b||, eps, then r = b - A x, p = J r and the first scalars per system
static int batch_setup(celg_handle* h, Batch* bt, int x0_mode, double eps_abs, double eps_rel,
                       const BatchArgs& a) {
  const BOpPre<double> pre{bt->B, bt->X, x0_mode, eps_abs, eps_rel, a};
  int st = launch_tile(h, bt->N, pre);
  if (!st) st = batch_finish(h, bt, pre);
  if (!st) st = batch_csr<double>(h, bt, bt->A.v, bt->X, BEpiInit<double>{bt->B, bt->R, bt->P, bt->J, a});
  if (!st) st = batch_finish(h, bt, BEpiInit<double>{bt->B, bt->R, bt->P, bt->J, a});
  return st;
}

// One iteration of every running system: K1, sigma, K2, beta and the test,
// then K3 with the marks moved or cleared after it: the even (odd = false)
// or the odd iteration of a pair, directions in P and then in Q.
static int batch_iteration(celg_handle* h, Batch* bt, const BatchArgs& a, bool odd) {
  double* pc = odd ? bt->Q : bt->P;
  const BEpiAp<double> ap{bt->V, pc, a};
  const BOpUpdate<double> upd{bt->R, bt->V, bt->J, a, 0.0};
  int s2 = batch_csr<double>(h, bt, bt->A.v, pc, ap);
  if (!s2) s2 = batch_finish(h, bt, ap);
  if (!s2) s2 = batch_tile(h, bt, upd);
  if (!s2) s2 = batch_finish(h, bt, upd);
  if (s2) return s2;
  return batch_direction_pair<double>(h, bt, a, odd, bt->P, bt->Q, bt->R, bt->J, bt->X);
}

// A pair of iterations (the loop body of the FP64 solve).
static int batch_pair(celg_handle* h, Batch* bt, const BatchArgs& a) {
  int st = batch_iteration(h, bt, a, false);
  if (!st) st = batch_iteration(h, bt, a, true);
  return st;
}

// The batch tuner: times a few iterations of the batch's own systems with
// each launch shape of kBatchShapes and keeps the fastest for the batch
// (CELG_BATCH_SHAPE=0..5 forces one).  It starts from x0 = 0 in the batch's
// work vectors, so the caller's vectors are neither read beyond b nor
// written; the solve that follows sets everything up again.
static int batch_tune(celg_handle* h, Batch* bt, const double* const* b_d) {
  if (bt->shape >= 0) return CELG_OK;
  if (const char* e = std::getenv("CELG_BATCH_SHAPE")) {
    const int v = std::atoi(e);
    bt->shape = (v >= 0 && v < kNumBatchShapes) ? v : 0;
    return CELG_OK;
  }
  for (int s = 0; s < bt->nsys; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(bt->B + bt->row_off[s], b_d[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
  }
  // no iteration cap, so that every system keeps running through the timing
  const BatchArgs a = batch_args(bt, 1 << 30, 0, h->err_d);
  cudaEvent_t e0, e1;
  CELG_CUDA(cudaEventCreate(&e0));
  CELG_CUDA(cudaEventCreate(&e1));
  float best = 0.f;
  int best_shape = 0, st = CELG_OK;
  for (int c = 0; c < kNumBatchShapes && !st; ++c) {
    bt->shape = c;
    st = batch_setup(h, bt, CELG_X0_ZERO, 0.0, 0.0, a);
    if (!st) st = batch_pair(h, bt, a);  // warm-up
    if (st) break;
    cudaEventRecord(e0, h->stream);
    for (int k = 0; k < 2 && !st; ++k) st = batch_pair(h, bt, a);
    cudaEventRecord(e1, h->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = CELG_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (!st && (c == 0 || ms < best)) {
      best = ms;
      best_shape = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  bt->shape = best_shape;
  return st;
}

static int record_batched(celg_handle* h, Batch* bt, const double* const* b_d, double* const* x_d,
                          const celg_params* p, BatchArgs a) {
  for (int s = 0; s < bt->nsys; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(bt->B + bt->row_off[s], b_d[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
    if (p->x0_mode == CELG_X0_USER)
      CELG_CUDA(cudaMemcpyAsync(bt->X + bt->row_off[s], x_d[s], sizeof(double) * (size_t)bt->n[s],
                                cudaMemcpyDeviceToDevice, h->stream));
  }
  int st = batch_setup(h, bt, p->x0_mode, p->eps_abs, p->eps_rel, a);
  auto body = [&]() -> int { return batch_pair(h, bt, a); };
  if (!st && a.cond) st = capture_while(h, a.cond, body);
  for (int it = 0; !st && !a.cond && it < p->iter_max; it += 8) {
    for (int q = 0; q < 4 && !st; ++q) st = body();
    int live = 0;
    if (!st) {
      CELG_CUDA(cudaMemcpyAsync(&live, a.n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      CELG_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (!live) break;
  }
  const BEpiVerify ver{bt->B, a};
  if (!st) st = batch_csr<double>(h, bt, bt->A.v, bt->X, ver);
  if (!st) st = batch_finish(h, bt, ver);
  if (st) return st;
  for (int s = 0; s < bt->nsys; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(x_d[s], bt->X + bt->row_off[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
  }
  return CELG_OK;
}

// The handle's concatenated batch for these matrices (built on first use).
static int batch_for(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                     double* const* x_d, Batch** out) {
  std::string mkey = "batch";
  char buf[64];
  for (int s = 0; s < count; ++s) {
    if (!mats[s] || !mats[s]->jacobi || mats[s]->h != h) return CELG_ERR_ARG;
    if (mats[s]->csr.n > 0 && (!b_d[s] || !x_d[s])) return CELG_ERR_ARG;
    std::snprintf(buf, sizeof(buf), "|%p", (const void*)mats[s]);
    mkey += buf;
  }
  Batch* bt = h->batch;
  if (!bt || bt->key != mkey) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    batch_free(h->batch);
    h->batch = nullptr;
    int st = batch_build(h, count, mats, mkey, &bt);
    if (st) return st;
    h->batch = bt;
  }
  *out = bt;
  return CELG_OK;
}

static int pcg_batched_ir(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                          double* const* x_d, const celg_params* p, celg_result* res);
static int pcg_batched_ru(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                          double* const* x_d, const celg_params* p, celg_result* res);

int pcg_batched(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                double* const* x_d, const celg_params* p, celg_result* res) {
  if (p->precision == CELG_PREC_FP32_IR) return pcg_batched_ir(h, count, mats, b_d, x_d, p, res);
  if (p->precision == CELG_PREC_FP32_RU) return pcg_batched_ru(h, count, mats, b_d, x_d, p, res);
  if (p->precision != CELG_PREC_FP64) return CELG_ERR_ARG;
  Batch* bt = nullptr;
  int st = batch_for(h, count, mats, b_d, x_d, &bt);
  if (st) return st;
  char buf[64];
  const std::string& mkey = bt->key;
  st = ensure_partials(h, bt->NT, 2);
  if (!st) st = batch_tune(h, bt, b_d);
  if (st) return st;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  std::string gkey = mkey;
  for (int s = 0; s < count; ++s) {
    std::snprintf(buf, sizeof(buf), "|%p|%p", (const void*)b_d[s], (const void*)x_d[s]);
    gkey += buf;
  }
  std::snprintf(buf, sizeof(buf), "|%d|%.17g|%.17g|%d", p->x0_mode, p->eps_abs, p->eps_rel, p->iter_max);
  gkey += buf;
  if (!graphs_enabled()) {
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = record_batched(h, bt, b_d, x_d, p, batch_args(bt, p->iter_max, 0, h->err_d));
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    GraphEntry* ge = graph_cache_find(h, gkey);
    if (!ge) {
      st = graph_build(h, gkey, [&](cudaGraphConditionalHandle cond) -> int {
        return record_batched(h, bt, b_d, x_d, p, batch_args(bt, p->iter_max, cond, h->err_d));
      }, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  std::vector<double> ds(7 * (size_t)count);
  std::vector<int> is(3 * (size_t)count + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), bt->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), bt->istate, sizeof(int) * is.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, iters = 0;
  for (int s = 0; s < count; ++s) {
    const double alpha = ds[(size_t)s], norm = ds[3 * (size_t)count + s];
    const double eps = ds[5 * (size_t)count + s];
    const int it = is[(size_t)s], err = is[2 * (size_t)count + s];
    int rs = CELG_OK;
    if (bt->n[s] == 0) {
      if (res) {
        std::memset(&res[s], 0, offsetof(celg_result, history));
        res[s].history_len = 0;
      }
      continue;
    }
    if (err) rs = err;
    else if (!(norm <= eps) && it >= p->iter_max && std::fabs(alpha) > kRealSmall) rs = CELG_ERR_NOCONV;
    if (rs && !ret) ret = rs;
    iters = std::max(iters, it);
    if (res) {
      res[s].iter_done = it;
      res[s].final_norm2 = norm;
      res[s].bnorm = ds[4 * (size_t)count + s];
      res[s].verified_relres = ds[6 * (size_t)count + s];
      res[s].err = rs;
      res[s].arnoldi_steps = 0;
      res[s].history_len = 0;
    }
  }
  h->last_iters = iters;
  return ret;
}

// FP32 refinement of every system: the outer loop of ir_solve (ir.cu) for
// all systems at once, each system's inner FP32 Jacobi-PCG in one batched
// inner solve (a graph with a WHILE node, captured once).  Each system's
// result equals ir_solve on that system alone, bit for bit.
static int batch_ensure_f32(celg_handle* h, Batch* bt) {
  if (bt->F) return CELG_OK;
  const size_t N = (size_t)std::max(1L, bt->N), NNZ = (size_t)bt->A.nnz, c = (size_t)bt->nsys;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; return e == cudaSuccess; };
  ok(cudaMalloc(&bt->A.v32, sizeof(float) * (NNZ + 32)));
  ok(cudaMalloc(&bt->J32, sizeof(float) * N));
  ok(cudaMalloc(&bt->F, sizeof(float) * N * 6));
  ok(cudaMalloc(&bt->irs, sizeof(int) * (5 * c + 1)));
  ok(cudaMalloc(&bt->irtau, sizeof(double) * c));
  ok(cudaMalloc(&bt->dstate2, sizeof(double) * 8 * c));
  ok(cudaMalloc(&bt->istate2, sizeof(int) * (5 * c + 1)));
  ok(cudaMemsetAsync(bt->F, 0, sizeof(float) * N * 6, h->stream));
  ok(cudaMemsetAsync(bt->A.v32 + NNZ, 0, sizeof(float) * 32, h->stream));
  if (e != cudaSuccess) return cuda_status(e, "batch FP32 allocation");
  int st = launch_to_f32(h, (long)NNZ, bt->A.v, bt->A.v32);
  if (!st && bt->N > 0) st = launch_to_f32(h, bt->N, bt->J, bt->J32);
  return st;
}

// `pair` records two iterations
template <class Body>
static int run_while(celg_handle* h, cudaGraphConditionalHandle cond, const int* n_active, int iter_max,
                     Body&& pair) {
  if (cond) return capture_while(h, cond, pair);
  for (int it = 0; it < iter_max; it += 8) {
    int st = CELG_OK;
    for (int q = 0; q < 4 && !st; ++q) st = pair();
    if (st) return st;
    int live = 0;
    CELG_CUDA(cudaMemcpyAsync(&live, n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    if (!live) break;
  }
  return CELG_OK;
}

static int record_batched_inner(celg_handle* h, Batch* bt, const IrState& ir, BatchArgs ai) {
  const long N = bt->N;
  float* B32 = bt->F;
  float* D32 = B32 + N;
  float* R32 = D32 + N;
  float* P32 = R32 + N;
  float* V32 = P32 + N;
  float* Q32 = V32 + N;  // second direction of the paired sweeps
  const BOpPre<float> pre{B32, D32, CELG_X0_ZERO, 0.0, ir.tau, ai, ir.part, ir.part_count,
                          ir.tau_sys};
  const BEpiInit<float> init{B32, R32, P32, bt->J32, ai};
  const BOpUpdate<float> upd{R32, V32, bt->J32, ai, 0.0};
  int st = launch_tile(h, N, pre);
  if (!st) st = batch_finish(h, bt, pre);
  if (!st) st = batch_csr<float>(h, bt, bt->A.v32, D32, init);
  if (!st) st = batch_finish(h, bt, init);
  if (!st)
    st = run_while(h, ai.cond, ai.n_active, ai.iter_max, [&]() -> int {
      int s2 = CELG_OK;
      for (int odd = 0; odd < 2 && !s2; ++odd) {
        float* pc = odd ? Q32 : P32;
        const BEpiAp<float> ap{V32, pc, ai};
        s2 = batch_csr<float>(h, bt, bt->A.v32, pc, ap);
        if (!s2) s2 = batch_finish(h, bt, ap);
        if (!s2) s2 = batch_tile(h, bt, upd);
        if (!s2) s2 = batch_finish(h, bt, upd);
        if (!s2) s2 = batch_direction_pair<float>(h, bt, ai, odd != 0, P32, Q32, R32, bt->J32, D32);
      }
      return s2;
    });
  return st;
}

static int pcg_batched_ir(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                          double* const* x_d, const celg_params* p, celg_result* res) {
  Batch* bt = nullptr;
  int st = batch_for(h, count, mats, b_d, x_d, &bt);
  if (!st) st = ensure_partials(h, bt->NT, 2);
  if (!st) st = batch_tune(h, bt, b_d);
  if (!st) st = batch_ensure_f32(h, bt);
  if (st) return st;
  const long N = bt->N;
  const int c = bt->nsys;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  const int inner_max = p->inner_iter_max > 0 ? p->inner_iter_max : 1000;
  const double inner_eps = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-4;
  IrState ir;
  ir.part = bt->irs;
  ir.done = ir.part + c;
  ir.status = ir.done + c;
  ir.outer = ir.status + c;
  ir.inner_total = ir.outer + c;
  ir.part_count = ir.inner_total + c;
  ir.outer_max = p->outer_max > 0 ? p->outer_max : 20;
  ir.tau_sys = bt->irtau;
  ir.tau = inner_eps;
  const BatchArgs a = batch_args(bt, p->iter_max, 0, h->err_d);
  CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
  for (int s = 0; s < c; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(bt->B + bt->row_off[s], b_d[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
    if (p->x0_mode == CELG_X0_USER)
      CELG_CUDA(cudaMemcpyAsync(bt->X + bt->row_off[s], x_d[s], sizeof(double) * (size_t)bt->n[s],
                                cudaMemcpyDeviceToDevice, h->stream));
  }
  // x0, ||b|| and the tolerance per system
  const BOpPre<double> pre{bt->B, bt->X, p->x0_mode, p->eps_abs, p->eps_rel, a};
  st = launch_tile(h, N, pre);
  if (!st) st = batch_finish(h, bt, pre);
  CELG_CUDA(cudaMemsetAsync(ir.part, 0, sizeof(int) * (5 * (size_t)c + 1), h->stream));
  // systems with no rows take no part at all
  std::vector<int> done0((size_t)c, 0);
  for (int s = 0; s < c; ++s) done0[(size_t)s] = bt->n[s] == 0 ? 1 : 0;
  CELG_CUDA(cudaMemcpyAsync(ir.done, done0.data(), sizeof(int) * (size_t)c, cudaMemcpyHostToDevice,
                            h->stream));
  const BatchArgs ai_host = batch_args(bt, inner_max, 0, h->err_d, true);
  char kb[96];
  std::snprintf(kb, sizeof(kb), "|ir|%d|%.17g", inner_max, inner_eps);
  const std::string gkey = bt->key + kb;
  for (int k = 0; !st && k <= ir.outer_max; ++k) {
    CELG_CUDA(cudaMemsetAsync(ir.part, 0, sizeof(int) * (size_t)c, h->stream));
    CELG_CUDA(cudaMemsetAsync(ir.part_count, 0, sizeof(int), h->stream));
    const BEpiIrResidual res_op{bt->B, bt->R, a, ir};
    st = batch_csr<double>(h, bt, bt->A.v, bt->X, res_op);
    if (!st) st = batch_finish(h, bt, res_op);
    if (st) break;
    int parts = 0;
    CELG_CUDA(cudaMemcpyAsync(&parts, ir.part_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    if (parts == 0) break;
    st = launch_tile(h, N, BOpIrToF32{bt->R, bt->F, a, ir, 0.0});
    if (st) break;
    if (graphs_enabled()) {
      GraphEntry* ge = graph_cache_find(h, gkey);
      if (!ge) {
        st = graph_build(h, gkey, [&](cudaGraphConditionalHandle cond) -> int {
          return record_batched_inner(h, bt, ir, batch_args(bt, inner_max, cond, h->err_d, true));
        }, &ge);
        if (st) break;
      }
      CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    } else {
      st = record_batched_inner(h, bt, ir, ai_host);
      if (st) break;
    }
    ir_count_kernel<<<(c + 127) / 128, 128, 0, h->stream>>>(c, ir, ai_host.iter, ai_host.err);
    CELG_CUDA(cudaGetLastError());
    st = launch_tile(h, N, BOpIrAdd{bt->X, bt->F + N, a, ir, 0.0});
  }
  if (st) return st;
  for (int s = 0; s < c; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(x_d[s], bt->X + bt->row_off[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
  }
  CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  std::vector<double> ds(7 * (size_t)c);
  std::vector<int> is(5 * (size_t)c + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), bt->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), ir.part, sizeof(int) * is.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, inner_max_total = 0;
  for (int s = 0; s < c; ++s) {
    const int done = is[(size_t)c + s], status = is[2 * (size_t)c + s];
    const int outer = is[3 * (size_t)c + s], inner = is[4 * (size_t)c + s];
    const double rn = ds[3 * (size_t)c + s], bn = ds[4 * (size_t)c + s];
    int rs = done ? status : CELG_ERR_NOCONV;
    if (bt->n[s] == 0) rs = CELG_OK;
    if (rs && !ret) ret = rs;
    inner_max_total = std::max(inner_max_total, inner);
    if (res) {
      std::memset(&res[s], 0, offsetof(celg_result, history));
      res[s].iter_done = outer;
      res[s].final_norm2 = rn;
      res[s].bnorm = bn;
      res[s].verified_relres = bn > 0 ? rn / bn : rn;
      res[s].err = rs;
      res[s].arnoldi_steps = inner;
      res[s].history_len = 0;
    }
  }
  h->last_iters = inner_max_total;
  return ret;
}

// FP32 PCG with FP64 reliable updates of every system: one graph launch with
// a WHILE node over { FP32 SpMV, step, IF(some system due) { flush, FP64
// residual }, direction }; self-skipping sweeps from a host loop when graphs
// are off.
static int record_batched_ru(celg_handle* h, Batch* bt, const double* const* b_d, double* const* x_d,
                             const celg_params* p, BatchArgs a, BatchRu u) {
  const long N = bt->N;
  float* D32 = bt->F + N;
  float* R32 = D32 + N;
  float* P32 = R32 + N;
  float* V32 = P32 + N;
  const float* J32 = bt->J32;
  for (int s = 0; s < bt->nsys; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(bt->B + bt->row_off[s], b_d[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
    if (p->x0_mode == CELG_X0_USER)
      CELG_CUDA(cudaMemcpyAsync(bt->X + bt->row_off[s], x_d[s], sizeof(double) * (size_t)bt->n[s],
                                cudaMemcpyDeviceToDevice, h->stream));
  }
  // x0, ||b||, eps; every system starts with a reliable update (its residual)
  const BOpPre<double> pre{bt->B, bt->X, p->x0_mode, p->eps_abs, p->eps_rel, a};
  int st = launch_tile(h, N, pre);
  if (!st) st = batch_finish(h, bt, pre);
  if (!st) {
    bru_init_kernel<<<1, kLanes, 0, h->stream>>>(bt->nsys, a.br.sys_ntiles, u);
    CELG_CUDA(cudaGetLastError());
    CELG_CUDA(cudaMemsetAsync(D32, 0, sizeof(float) * (size_t)std::max(1L, N), h->stream));
    const BEpiRuResidual r0{bt->B, R32, P32, J32, a, u, 1};
    st = batch_csr<double>(h, bt, bt->A.v, bt->X, r0);
    if (!st) st = batch_finish(h, bt, r0);
  }
  auto body = [&](bool in_graph) -> int {
    BatchRu uc = u;
    if (in_graph) {
      int s2 = capture_new_handle(h, 0, &uc.cond_update);
      if (s2) return s2;
    }
    const BEpiAp<float> ap{V32, P32, a};
    const BOpRuStep step{R32, V32, J32, a, uc, 0.0f};
    int s3 = batch_csr<float>(h, bt, bt->A.v32, P32, ap);
    if (!s3) s3 = batch_finish(h, bt, ap);
    if (!s3) s3 = batch_tile(h, bt, step);
    if (!s3) s3 = batch_finish(h, bt, step);
    auto update = [&]() -> int {
      int s4 = batch_tile(h, bt, BOpRuFlush{bt->X, D32, P32, a, uc, 0});
      if (!s4) {
        bru_clear_kernel<<<1, kLanes, 0, h->stream>>>(bt->nsys, a.xpend, uc.upd);
        CELG_CUDA(cudaGetLastError());
      }
      const BEpiRuResidual rr{bt->B, R32, nullptr, J32, a, uc, 0};
      if (!s4) s4 = batch_csr<double>(h, bt, bt->A.v, bt->X, rr);
      if (!s4) s4 = batch_finish(h, bt, rr);
      return s4;
    };
    if (!s3) s3 = in_graph ? capture_if(h, uc.cond_update, update) : update();
    if (!s3) s3 = batch_tile(h, bt, BOpRuDirection{P32, R32, J32, D32, a});
    if (!s3) s3 = clear_marks(h, a);
    return s3;
  };
  if (!st && a.cond) st = capture_while2(h, a.cond, [&]() -> int { return body(true); });
  for (int it = 0; !st && !a.cond && it < p->iter_max; it += 8) {
    for (int q = 0; q < 8 && !st; ++q) st = body(false);
    int live = 0;
    if (!st) {
      CELG_CUDA(cudaMemcpyAsync(&live, a.n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      CELG_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (!live) break;
  }
  // x64 += d for every system, then the FP64 check
  if (!st) st = batch_tile(h, bt, BOpRuFlush{bt->X, D32, nullptr, a, u, 1});
  const BEpiVerify ver{bt->B, a};
  if (!st) st = batch_csr<double>(h, bt, bt->A.v, bt->X, ver);
  if (!st) st = batch_finish(h, bt, ver);
  if (st) return st;
  for (int s = 0; s < bt->nsys; ++s) {
    if (bt->n[s] == 0) continue;
    CELG_CUDA(cudaMemcpyAsync(x_d[s], bt->X + bt->row_off[s], sizeof(double) * (size_t)bt->n[s],
                              cudaMemcpyDeviceToDevice, h->stream));
  }
  return CELG_OK;
}

static int pcg_batched_ru(celg_handle* h, int count, celg_mat* const* mats, const double* const* b_d,
                          double* const* x_d, const celg_params* p, celg_result* res) {
  Batch* bt = nullptr;
  int st = batch_for(h, count, mats, b_d, x_d, &bt);
  if (!st) st = ensure_partials(h, bt->NT, 2);
  if (!st) st = batch_tune(h, bt, b_d);
  if (!st) st = batch_ensure_f32(h, bt);
  if (st) return st;
  const int c = bt->nsys;
  if (!bt->rud) CELG_CUDA(cudaMalloc(&bt->rud, sizeof(double) * 3 * (size_t)c));
  if (!bt->rui) CELG_CUDA(cudaMalloc(&bt->rui, sizeof(int) * (2 * (size_t)c + 1)));
  BatchRu u;
  u.maxr = bt->rud;
  u.rz_prev = u.maxr + c;
  u.norm64 = u.rz_prev + c;
  u.updates = bt->rui;
  u.upd = u.updates + c;
  u.n_upd = u.upd + c;
  u.delta = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-2;
  u.cond_update = 0;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  std::string gkey = bt->key;
  char buf[96];
  for (int s = 0; s < count; ++s) {
    std::snprintf(buf, sizeof(buf), "|%p|%p", (const void*)b_d[s], (const void*)x_d[s]);
    gkey += buf;
  }
  std::snprintf(buf, sizeof(buf), "|ru|%d|%.17g|%.17g|%.17g|%d", p->x0_mode, p->eps_abs, p->eps_rel,
                u.delta, p->iter_max);
  gkey += buf;
  if (!graphs_enabled()) {
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = record_batched_ru(h, bt, b_d, x_d, p, batch_args(bt, p->iter_max, 0, h->err_d), u);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    GraphEntry* ge = graph_cache_find(h, gkey);
    if (!ge) {
      st = graph_build(h, gkey, [&](cudaGraphConditionalHandle cond) -> int {
        return record_batched_ru(h, bt, b_d, x_d, p, batch_args(bt, p->iter_max, cond, h->err_d), u);
      }, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  std::vector<double> ds(7 * (size_t)c), rd(3 * (size_t)c);
  std::vector<int> is(3 * (size_t)c + 1), ri(2 * (size_t)c + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), bt->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), bt->istate, sizeof(int) * is.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(rd.data(), bt->rud, sizeof(double) * rd.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(ri.data(), bt->rui, sizeof(int) * ri.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, iters = 0;
  for (int s = 0; s < c; ++s) {
    if (bt->n[s] == 0) {
      if (res) {
        std::memset(&res[s], 0, offsetof(celg_result, history));
        res[s].history_len = 0;
      }
      continue;
    }
    const double norm64 = rd[2 * (size_t)c + s], eps = ds[5 * (size_t)c + s];
    const int it = is[(size_t)s], err = is[2 * (size_t)c + s];
    int rs = CELG_OK;
    if (err) rs = err;
    else if (!(norm64 <= eps)) rs = CELG_ERR_NOCONV;
    if (rs && !ret) ret = rs;
    iters = std::max(iters, it);
    if (res) {
      res[s].iter_done = it;
      res[s].final_norm2 = norm64;
      res[s].bnorm = ds[4 * (size_t)c + s];
      res[s].verified_relres = ds[6 * (size_t)c + s];
      res[s].err = rs;
      res[s].arnoldi_steps = ri[(size_t)s];
      res[s].history_len = 0;
    }
  }
  h->last_iters = iters;
  return ret;
}

}  // namespace celg

extern "C" int celg_pcg_batched(celg_handle* h, int count, celg_mat* const* mats,
                                const double* const* b_d, double* const* x_d, const celg_params* p,
                                celg_result* res) {
  if (!h || count <= 0 || !mats || !b_d || !x_d || !p) return CELG_ERR_ARG;
  if (p->x0_mode < CELG_X0_REF_ONES || p->x0_mode > CELG_X0_USER || p->iter_max < 0) return CELG_ERR_ARG;
  if (p->precond != CELG_PRECOND_JACOBI) return CELG_ERR_ARG;
  for (int s = 0; s < count; ++s)
    if (mats[s] && mats[s]->csr.ncols != mats[s]->csr.n) return CELG_ERR_ARG;  // square systems only
  CELG_CUDA(cudaSetDevice(h->device));
  return celg::pcg_batched(h, count, mats, b_d, x_d, p, res);
}

extern "C" int celg_tuned_config(celg_handle* h, int what, int out[2]) {
  if (!h || !out) return CELG_ERR_ARG;
  out[0] = out[1] = -1;
  if (what == CELG_TUNE_BATCH) {
    if (!h->batch || h->batch->shape < 0) return CELG_ERR_STATE;
    const celg::BatchShape sh = celg::kBatchShapes[h->batch->shape];
    out[0] = sh.csr_per_sm;
    out[1] = sh.tile_per_sm;
    return CELG_OK;
  }
  if (what == CELG_TUNE_SPMM) {
    const int cfg = celg::multi_tuned_cfg(h->multi);
    if (cfg < 0) return CELG_ERR_STATE;
    out[0] = cfg;
    out[1] = celg::multi_tuned_cfg32(h->multi);
    return CELG_OK;
  }
  return CELG_ERR_ARG;
}
