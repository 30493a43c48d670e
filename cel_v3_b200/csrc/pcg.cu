// pcg.cu -- Jacobi-PCG (cel_cgalg_jacobi, src/fcgalg/cel_cgalg_module.f90:178-305)
// as three fused sweeps per iteration, run to convergence inside one CUDA
// graph whose WHILE conditional node is driven from the device.  The loop
// body holds two iterations; consecutive sweeps walk the tiles in opposite
// orders (RedCtx::sweep), so six sweeps make the order repeat.
//
// Per iteration (reference lines in brackets):
//   K1  v = 0 + A p, pv = v.p, sigma = alpha/pv          [:251-261]
//   K2  r += (-sigma) v, z = J r (not stored),
//       rz = r.z, rr = r.r, beta = rz/alpha, alpha = rz,
//       ||r|| = sqrt(rr), convergence test               [:265-277, :287, :247-249]
//   K3  x += sigma p (the iteration's x update, :263-264, moved here
//       because K3 reads the old p anyway), then p = beta p + J r  [:282]
// Set-up: x0, ||b|| and eps (Kpre); r = b - A x, p = J r, alpha = r.p,
// ||r|| (Kinit) [:207-236].  After the loop one more sweep recomputes
// ||b - A x|| in FP64 (verification; not part of the reference).
//
// The same kernels serve the FP32-storage inner solve of the iterative
// refinement (VT = float): matrix values and vectors are float, every
// vector update is computed in double from the float operands and rounded
// once, reductions and scalars are double.  For VT = double the arithmetic
// is exactly the reference's.
// Algorithmic bytes per FP64 CSR iteration: 12 nnz + 4 (n+1) + 96 n (K1
// 12 nnz + 4 (n+1) + 16 n, p gathered and v stored, the p of p.v coming
// from L1/L2; K2 32 n; K3 48 n).  When the matrix has at most 256 column
// offsets the CSR sweeps read 1-byte column codes instead of int32 columns:
// 9 nnz instead of 12 nnz.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "graph.cuh"
#include "pcg_internal.cuh"

namespace celg {

int ensure_work(celg_handle* h, size_t n) {
  if (n <= h->wcap && h->wr) return CELG_OK;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  graph_cache_clear(h);
  cudaFree(h->wr);
  cudaFree(h->wp);
  cudaFree(h->wv);
  cudaFree(h->wq);
  h->wr = h->wp = h->wv = h->wq = nullptr;
  h->wcap = 0;  // a failed allocation below leaves no stale capacity behind
  const size_t cap = std::max<size_t>(n, 1024);
  CELG_CUDA(cudaMalloc(&h->wr, cap * sizeof(double)));
  CELG_CUDA(cudaMalloc(&h->wp, cap * sizeof(double)));
  CELG_CUDA(cudaMalloc(&h->wv, cap * sizeof(double)));
  CELG_CUDA(cudaMalloc(&h->wq, cap * sizeof(double)));
  h->wcap = cap;
  return CELG_OK;
}

int ensure_state(celg_handle* h, int hist_cap) {
  if (!h->state_d) CELG_CUDA(cudaMalloc(&h->state_d, sizeof(PcgState)));
  if (!h->state_h) CELG_CUDA(cudaMallocHost(&h->state_h, sizeof(PcgState)));
  if (hist_cap > h->hist_cap) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(h->hist_d);
    h->hist_d = nullptr;
    h->hist_cap = 0;
    CELG_CUDA(cudaMalloc(&h->hist_d, sizeof(double) * (size_t)hist_cap));
    h->hist_cap = hist_cap;
  }
  return CELG_OK;
}

void graph_cache_clear(celg_handle* h) {
  for (auto& e : h->graphs) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
  }
  h->graphs.clear();
}

void graph_cache_drop_matrix(celg_handle* h, const void* m) {
  char tag[64];
  std::snprintf(tag, sizeof(tag), "|%p|", m);
  for (size_t i = 0; i < h->graphs.size();) {
    if (h->graphs[i].key.find(tag) != std::string::npos) {
      if (h->graphs[i].exec) cudaGraphExecDestroy(h->graphs[i].exec);
      if (h->graphs[i].graph) cudaGraphDestroy(h->graphs[i].graph);
      h->graphs.erase(h->graphs.begin() + (long)i);
    } else {
      ++i;
    }
  }
}

// A CSR sweep of the solve: FP64 with the 1-byte column offsets when the
// matrix has them (same values in the same order, so the same sums), else
// with the int32 columns.
template <typename VT, class Epi>
static int csr_sweep(celg_handle* h, const PcgBind<VT>& B, const VT* vals, const VT* x, const Epi& epi) {
  if constexpr (std::is_same<VT, double>::value) {
    if (B.dict) {
      bool done = false;
      const int st = launch_csr_compact<double>(h, *B.A, vals, x, epi, nullptr, 0, &done);
      if (done) return st;
    }
  }
  return launch_csr<VT>(h, *B.A, vals, x, epi);
}

template <typename VT>
static int pcg_setup(celg_handle* h, const PcgBind<VT>& B, const celg_params* p, PcgArgs a) {
  const long n = B.A->n;
  constexpr bool kF64 = std::is_same<VT, double>::value;
  int st = launch_tile(h, n, OpPre<VT>{B.b, B.x, p->x0_mode, p->eps_abs, p->eps_rel, a});
  if (st) return st;
  if constexpr (kF64) {
    if (B.jad) {
      st = launch_jad(h, *B.A, *B.jad, B.x, EpiStore<double>{B.r, 0});
      if (!st) st = launch_tile(h, n, OpInitNat<double>{B.b, B.r, B.p, B.J, a});
      return st;
    }
    if (B.bj) return bj_pcg_setup_tail(h, B, a);
  }
  return csr_sweep<VT>(h, B, B.vals, B.x, EpiInit<VT>{B.b, B.r, B.p, B.J, a});
}

// phase 0: one iteration, K3 = OpDirectionX.  Phases 1 and 2: the even and
// the odd iteration of a pair (B.q set: CSR sweeps, point Jacobi), whose
// directions are B.p and B.q in turn.
template <typename VT>
static int pcg_body(celg_handle* h, const PcgBind<VT>& B, PcgArgs a, int phase = 0) {
  const long n = B.A->n;
  VT* pc = phase == 2 ? B.q : B.p;
  int s2 = CELG_OK;
  if constexpr (std::is_same<VT, double>::value) {
    if (B.jad)
      s2 = launch_jad(h, *B.A, *B.jad, B.p, EpiAp<double>{B.v, B.p, a});
    else
      s2 = csr_sweep<VT>(h, B, B.vals, pc, EpiAp<VT>{B.v, pc, a});
  } else {
    s2 = csr_sweep<VT>(h, B, B.vals, pc, EpiAp<VT>{B.v, pc, a});
  }
  if constexpr (std::is_same<VT, double>::value) {
    if (B.bj) {
      if (!s2) s2 = bj_pcg_update(h, B, a);
      if (!s2) s2 = bj_pcg_direction(h, B, a);
      return s2;
    }
  }
  if (!s2) s2 = launch_tile(h, n, OpUpdate<VT>{B.r, B.v, B.J, a, 0.0});
  if (s2) return s2;
  if (phase == 1) return launch_tile(h, n, OpDirectionDefer<VT>{B.p, B.q, B.r, B.J, B.x, a});
  if (phase == 2) return launch_tile(h, n, OpDirectionPair<VT>{B.p, B.q, B.r, B.J, B.x, a});
  return launch_tile(h, n, OpDirectionX<VT>{B.p, B.r, B.J, B.x, a});
}

// Two iterations: a pair when B.q is set, else the one-iteration body twice.
template <typename VT>
static int pcg_body2(celg_handle* h, const PcgBind<VT>& B, PcgArgs a) {
  int st = pcg_body(h, B, a, B.q ? 1 : 0);
  if (!st) st = pcg_body(h, B, a, B.q ? 2 : 0);
  return st;
}

template <typename VT>
static int pcg_tail(celg_handle* h, const PcgBind<VT>& B, PcgArgs a) {
  const long n = B.A->n;
  if constexpr (std::is_same<VT, double>::value) {
    if (!B.verify_vals) return CELG_OK;
    // verification sweep in FP64
    if (B.jad) {
      int st = launch_jad(h, *B.A, *B.jad, B.x, EpiStore<double>{B.v, 0});
      if (!st) st = launch_tile(h, n, OpVerifyNat{B.b, B.v, a.st});
      return st;
    }
    return csr_sweep<double>(h, B, B.verify_vals, B.x, EpiVerify{B.b, a.st});
  }
  return CELG_OK;
}

template <typename VT>
static int record_pcg(celg_handle* h, const PcgBind<VT>& B, const celg_params* p, PcgArgs a) {
  int st = pcg_setup(h, B, p, a);
  if (st) return st;
  st = capture_while(h, a.cond, [&]() -> int { return pcg_body2(h, B, a); });
  if (st) return st;
  return pcg_tail(h, B, a);
}

// Profiling mode (CELG_GRAPH=0): the same kernels launched one by one from a
// host loop, so that kernel profilers can attribute time to each of them
// (they cannot see into graphs with conditional nodes).  Chunks of 8
// iterations are queued between reads of the device's continue flag; the
// kernels of an inactive solve return at once.
template <typename VT>
static int run_host_loop(celg_handle* h, const PcgBind<VT>& B, const celg_params* p, PcgArgs a) {
  a.cond = 0;
  int st = pcg_setup(h, B, p, a);
  for (int it = 0; !st && it < p->iter_max; it += 8) {
    for (int k = 0; k < 4 && !st; ++k) st = pcg_body2(h, B, a);
    if (st) break;
    CELG_CUDA(cudaMemcpyAsync(h->state_h, h->state_d, sizeof(PcgState), cudaMemcpyDeviceToHost,
                              h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    if (!h->state_h->active) break;
  }
  if (!st) st = pcg_tail(h, B, a);
  return st;
}

template <typename VT>
static std::string pcg_key(const PcgBind<VT>& B, const celg_params* p, int hist_cap,
                           const void* mat) {
  char buf[640];
  std::snprintf(buf, sizeof(buf), "pcg%d|%p|%d|%d|%p|%p|%p|%p|%p|%p|%p|%d|%.17g|%.17g|%d|%d|%p|%p|%p|%d|%p|%d",
                (int)sizeof(VT), mat, B.A->n, B.jad ? 1 : 0, (const void*)B.b, (const void*)B.x,
                (const void*)B.r, (const void*)B.p, (const void*)B.q, (const void*)B.v, (const void*)B.J,
                p->x0_mode, p->eps_abs, p->eps_rel, p->iter_max, hist_cap,
                (const void*)B.vals, (const void*)B.verify_vals, (const void*)B.bj, B.bs,
                (const void*)B.z, B.dict ? 1 : 0);
  return std::string(buf);
}

template <typename VT>
int pcg_run(celg_handle* h, const PcgBind<VT>& B, const celg_params* p, const void* mat,
            PcgState* out_state) {
  const long n = B.A->n;
  if (p->iter_max < 0) return CELG_ERR_ARG;
  int st = ensure_partials(h, ntiles_of(n), 2);
  const int hist_cap = p->iter_max + 1;
  if (!st) st = ensure_state(h, hist_cap);
  if (st) return st;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));

  if (!graphs_enabled()) {
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = run_host_loop(h, B, p, PcgArgs{h->state_d, h->hist_d, hist_cap, p->iter_max, 0, h->err_d});
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    const std::string key = pcg_key(B, p, hist_cap, mat);
    GraphEntry* ge = graph_cache_find(h, key);
    if (!ge) {
      st = graph_build(h, key, [&](cudaGraphConditionalHandle cond) -> int {
        return record_pcg<VT>(h, B, p, PcgArgs{h->state_d, h->hist_d, hist_cap, p->iter_max, cond, h->err_d});
      }, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  CELG_CUDA(cudaMemcpyAsync(h->state_h, h->state_d, sizeof(PcgState), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(h->scal_h + 8, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  *out_state = *h->state_h;
  int err_word = 0;
  std::memcpy(&err_word, h->scal_h + 8, sizeof(int));
  if (err_word) return err_word;
  const PcgState& s = *out_state;
  if (s.err) return s.err;
  if (!(s.norm <= s.eps) && s.iter >= p->iter_max && std::fabs(s.alpha) > kRealSmall)
    return CELG_ERR_NOCONV;
  return CELG_OK;
}

template int pcg_run<double>(celg_handle*, const PcgBind<double>&, const celg_params*, const void*,
                             PcgState*);
template int pcg_run<float>(celg_handle*, const PcgBind<float>&, const celg_params*, const void*,
                            PcgState*);

int copy_history(celg_handle* h, int len, celg_result* res) {
  res->history_len = 0;
  if (res->history && res->history_cap > 0 && len > 0) {
    const int l = std::min(len, res->history_cap);
    CELG_CUDA(cudaMemcpy(res->history, h->hist_d, sizeof(double) * (size_t)l, cudaMemcpyDeviceToHost));
    res->history_len = l;
  }
  return CELG_OK;
}

int pcg_solve(celg_handle* h, celg_mat* m, const double* b, double* x, const celg_params* p,
              celg_result* res) {
  const long n = m->csr.n;
  if (!m->jacobi) return CELG_ERR_STATE;
  const bool jad = p->fmt == CELG_FMT_JAD;
  if (jad && m->jad.mmax < 0) return CELG_ERR_STATE;
  int st = ensure_work(h, (size_t)n);
  if (st) return st;
  PcgBind<double> B;
  B.A = &m->csr;
  B.jad = jad ? &m->jad : nullptr;
  B.vals = m->csr.v;
  B.verify_vals = m->csr.v;
  B.b = b;
  B.x = x;
  B.r = h->wr;
  B.p = h->wp;
  B.v = h->wv;
  B.J = m->jacobi;
  if (!jad) {
    st = ensure_offset_dict(h, m);
    if (st) return st;
    B.dict = m->csr.ci8 != nullptr;
  }
  if (p->precond == CELG_PRECOND_BLOCK_JACOBI) {
    if (jad) return CELG_ERR_ARG;
    if (!m->bjinv) return CELG_ERR_STATE;
    if ((size_t)n > h->wzcap || !h->wz) {
      CELG_CUDA(cudaStreamSynchronize(h->stream));
      graph_cache_clear(h);
      cudaFree(h->wz);
      h->wz = nullptr;
      h->wzcap = std::max<size_t>((size_t)n, 1024);
      CELG_CUDA(cudaMalloc(&h->wz, h->wzcap * sizeof(double)));
    }
    B.bj = m->bjinv;
    B.bs = m->bj_bs;
    B.z = h->wz;
  } else if (p->precond != CELG_PRECOND_JACOBI) {
    return CELG_ERR_ARG;
  } else if (!jad) {
    B.q = h->wq;
  }
  PcgState s;
  std::memset(&s, 0, sizeof(s));
  const int ret = pcg_run<double>(h, B, p, m, &s);
  h->last_iters = s.iter;
  // K1 reads 8 bytes per non-zero and one per row with the row patterns, 9 per
  // non-zero with the 1-byte offsets, else 12; the paired K3 reads and stores
  // x once per two iterations (92 instead of 96 bytes per row)
  h->last_bytes_per_iter =
      (B.dict && m->csr.pid ? 8.0 * m->csr.nnz + 1.0 * n : (B.dict ? 9.0 : 12.0) * m->csr.nnz) +
      4.0 * (n + 1) + (B.q ? 92.0 : 96.0) * n;
  if (res) {
    res->iter_done = s.iter;
    res->final_norm2 = s.norm;
    res->bnorm = s.bnorm;
    res->verified_relres = s.vres;
    res->err = ret;
    res->arnoldi_steps = 0;
    st = copy_history(h, std::min(s.hist_len, p->iter_max + 1), res);
    if (st) return st;
  }
  return ret;
}

}  // namespace celg
