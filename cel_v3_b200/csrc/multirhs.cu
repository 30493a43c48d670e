// multirhs.cu -- Jacobi-PCG on k <= 32 right-hand sides that share one matrix
// (block SpMM-driven PCG): B and X are n x k row-major, every column runs its
// own PCG recurrence (own alpha, sigma, beta, ||r||, iteration count), and
// each iteration reads the matrix once for all k columns.
//
// Thread mapping: a 256-thread CTA works on 1024-row tiles; warp w handles
// rows t*1024 + q*256 + w*32 + r (q = 0..3, r = 0..31) and lane c handles
// column c, so a warp reads the k values of a row of X (k*8 contiguous bytes)
// per non-zero.  Row sums run over the stored entries in order with separate
// multiply/add roundings (each column's SpMV equals the single-vector SpMV).
//
// Reduction order (per column c; mirrored by the test-suite's oracle
// composition): warp w sums its 128 rows of the tile in (q, r) order from
// 0.0; the tile partial is warp 0 + warp 1 + ... + warp 7; the tile partials
// are reduced with the single-vector order (lane j sums j, j+256, ...,
// butterfly, warps in order).
//
// Algorithmic bytes per iteration: 12 nnz + 4 (n+1) + 80 n k + 16 n (SpMM
// 16 n k: P gathered, V stored; update sweep 24 n k + 8 n: R, V, J read, R
// stored; direction sweep 40 n k + 8 n: P, R, X, J read, P, X stored).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "graph.cuh"
#include "pcg_internal.cuh"

namespace celg {

constexpr int kMaxRhs = 32;

struct MultiArgs {
  double *alpha, *sigma, *beta, *norm, *bnorm, *eps, *vres;
  int *iter, *active, *err, *n_active;
  // columns whose update sweep ran and whose x += sigma p the direction
  // sweep still owes (bit c = column c)
  unsigned* xmask;
  // paired direction sweeps (FP64): columns whose x += sigma p_k the odd
  // sweep owes from the even one (bit c), with that sigma
  unsigned* pmask;
  double* sigprev;
  int k;
  int iter_max;
  cudaGraphConditionalHandle cond;
  const int* errw;
  __device__ int go(int c) const {
    return (err[c] == 0 && *(volatile const int*)errw == 0 && iter[c] < iter_max &&
            fabs(alpha[c]) > kRealSmall && norm[c] > eps[c])
               ? 1
               : 0;
  }
  __device__ void settle(int c) const {
    const int g = go(c);
    active[c] = g;
    if (!g) atomicSub(n_active, 1);
  }
};

// Per-column tile partials: after the warps accumulated their 128 rows,
// combine warps in order and store partials[(r*k + c)*ntiles + t].
template <int NRED>
__device__ __forceinline__ void multi_tile_store(double (&acc)[NRED], double* s_w, int k, long t,
                                                 long ntiles, double* partials, int warp, int lane) {
  // s_w: [NRED][8][32]
#pragma unroll
  for (int r = 0; r < NRED; ++r) s_w[(r * 8 + warp) * 32 + lane] = acc[r];
  named_bar_sync(1, kLanes);
  if (threadIdx.x < NRED * 32) {
    const int r = threadIdx.x / 32, c = threadIdx.x % 32;
    if (c < k) {
      double tot = s_w[(r * 8 + 0) * 32 + c];
#pragma unroll
      for (int w = 1; w < 8; ++w) tot = dadd(tot, s_w[(r * 8 + w) * 32 + c]);
      partials[((long)r * k + c) * ntiles + t] = tot;
    }
  }
  named_bar_sync(1, kLanes);
}

// Last CTA: per (reduction, column) the single-vector tile reduction; then
// op.finish_col(c, tot[]) for every column and op.finish_global().
template <int NRED, class Op>
__device__ __forceinline__ void multi_grid_finish(const RedCtx& red, const Op& op, int k,
                                                  double* scratch, int* s_flag, double* s_tot) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    __threadfence();
    const unsigned tk = atomicAdd(red.ticket, 1u);
    *s_flag = (tk == gridDim.x - 1) ? 1 : 0;
  }
  named_bar_sync(1, kLanes);
  if (!*s_flag) return;
  __threadfence();
  // (reduction, column) pairs spread over the 8 warps, each in the 256-lane order
  for (int rc = tid >> 5; rc < NRED * k; rc += 8) {
    const double v = warp_reduce256(red.partials + (long)rc * red.ntiles, red.ntiles, tid & 31);
    if ((tid & 31) == 0) s_tot[rc] = v;
  }
  named_bar_sync(1, kLanes);
  if (tid < k) {
    double tot[NRED];
#pragma unroll
    for (int r = 0; r < NRED; ++r) tot[r] = s_tot[r * k + tid];
    op.finish_col(tid, tot);
  }
  named_bar_sync(1, kLanes);
  if (tid == 0) {
    op.finish_global();
    *red.ticket = 0u;
  }
}


// ---- SpMM with a fused per-row epilogue ---------------------------------------
// Warp w takes rows in order; lane c owns column c, so each stored entry is
// one k-wide (k*8-byte contiguous) gather of X.  Rows are software-pipelined
// two deep: the gathers of row r+1's first 8 entries (and its epilogue
// operands, Epi::Pre) are issued before row r is added up, so two rows'
// gathers are in flight per warp.  A row's adds run over its entries in
// stored order from 0.0 (entries past the first 8 are gathered in further
// chunks of 8 when the row is added).  The row ends of the warp's 32 rows are
// held one per lane and shuffled out.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
constexpr int kAsyncU = 8;                    // gathers per row slot
// doubles per slot: U gathered entries and 2 epilogue operands per lane, then
// the row's U matrix values (padded to 16 bytes)
constexpr int kAsyncSlot = (kAsyncU + 2) * 32 + ((kAsyncU + 1) & ~1);

template <int U, typename VT>
__device__ __forceinline__ void spmm_gather(const int* __restrict__ ci, const VT* __restrict__ X,
                                            int b, int e, int k, int lane, bool on, VT (&x)[U]) {
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (b + u < e) {
      const int c = __ldg(ci + b + u);
      x[u] = on ? __ldg(X + (long)c * k + lane) : VT(0);
    }
  }
}

template <class Epi, int MINB, int U>
__global__ void __launch_bounds__(kLanes, MINB) spmm_kernel(const int* __restrict__ rp,
                                                            const int* __restrict__ ci,
                                                            const typename Epi::VT* __restrict__ v,
                                                            int n, int k,
                                                            const typename Epi::VT* __restrict__ X,
                                                            Epi epi, RedCtx red) {
  using VT = typename Epi::VT;
  constexpr int NR = Epi::NRED;
  constexpr unsigned kFull = 0xffffffffu;
  __shared__ double s_w[(NR > 0 ? NR : 1) * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[(NR > 0 ? NR : 1) * kMaxRhs];
  __shared__ int s_flag;
  if (!epi.active()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool on = lane < k && epi.col_active(lane);
  const long ntiles = ((long)n + kTile - 1) / kTile;
  for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      if (row0 >= n) break;
      const int nrows = (int)min(32L, (long)n - row0);
      const int re = lane < nrows ? __ldg(rp + row0 + lane + 1) : 0;  // end of row lane
      int bA = __ldg(rp + row0);
      int eA = __shfl_sync(kFull, re, 0);
      VT xA[U];
      spmm_gather<U>(ci, X, bA, eA, k, lane, on, xA);
      typename Epi::Pre preA;
      if (on) preA = epi.pre(row0, lane);
      for (int r = 0; r < nrows; ++r) {
        const bool more = r + 1 < nrows;
        const int bB = eA;
        const int eB = __shfl_sync(kFull, re, more ? r + 1 : r);
        VT xB[U];
        typename Epi::Pre preB;
        if (more) {
          spmm_gather<U>(ci, X, bB, eB, k, lane, on, xB);
          if (on) preB = epi.pre(row0 + r + 1, lane);
        }
        VT sum = VT(0);
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (bA + u < eA) sum = vadd(sum, vmul(__ldg(v + bA + u), xA[u]));
        for (int kk = bA + U; kk < eA; kk += U) {  // rows longer than U entries
          VT xv[U];
          spmm_gather<U>(ci, X, kk, eA, k, lane, on, xv);
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (kk + u < eA) sum = vadd(sum, vmul(__ldg(v + kk + u), xv[u]));
        }
        if (on) epi.row(row0 + r, lane, sum, preA, acc);
        bA = bB;
        eA = eB;
#pragma unroll
        for (int u = 0; u < U; ++u) xA[u] = xB[u];
        preA = preB;
      }
    }
    if (NR > 0) multi_tile_store<(NR > 0 ? NR : 1)>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<(NR > 0 ? NR : 1)>(red, epi, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, epi, 0, scratch, &s_flag, s_tot);
}

// The same SpMM with the gathers issued as asynchronous copies into a ring of
// S row slots per warp in shared memory (cp.async, 8 bytes per lane and
// entry), so the data in flight does not occupy registers: rows r+1..r+S-1
// are in flight while row r is added up.  A slot also receives the row's
// matrix values (lanes 0..U-1) and the epilogue's operands (Epi::stage_pre),
// and the column indices of the next row to issue are loaded one row ahead,
// so no global load is waited for on the issue path.  Each lane copies and
// reads only its own column of a slot (the values area is read by all lanes
// after the wait and the warp barrier).
template <class Epi, int S, int MINB>
__global__ void __launch_bounds__(kLanes, MINB) spmm_async_kernel(const int* __restrict__ rp,
                                                           const int* __restrict__ ci,
                                                           const double* __restrict__ v, int n,
                                                           int k, const double* __restrict__ X,
                                                           Epi epi, RedCtx red) {
  constexpr int NR = Epi::NRED;
  constexpr int U = kAsyncU;
  constexpr int SLOT = kAsyncSlot;
  constexpr int VOFF = (U + 2) * 32;  // matrix values of the row
  constexpr unsigned kFull = 0xffffffffu;
  __shared__ double s_w[(NR > 0 ? NR : 1) * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[(NR > 0 ? NR : 1) * kMaxRhs];
  __shared__ int s_flag;
  extern __shared__ __align__(16) double s_ring[];
  if (!epi.active()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool on = lane < k && epi.col_active(lane);
  double* ring = s_ring + (long)warp * S * SLOT;
  const long ntiles = ((long)n + kTile - 1) / kTile;
  for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      if (row0 >= n) break;
      const int nrows = (int)min(32L, (long)n - row0);
      const int re = lane < nrows ? __ldg(rp + row0 + lane + 1) : 0;  // end of row lane
      const int b0 = __ldg(rp + row0);
      // next row to issue (rI), its entry range and its first U column indices
      int rI = 0, bI = b0, eI = __shfl_sync(kFull, re, 0);
      int cn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) cn[u] = bI + u < eI ? __ldg(ci + bI + u) : 0;
      auto issue_next = [&]() {
        if (rI < nrows) {
          double* slot = ring + (rI % S) * SLOT;
          if (on) {
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (bI + u < eI) cp_async8(slot + u * 32 + lane, X + (long)cn[u] * k + lane);
            epi.stage_pre(row0 + rI, lane, slot + U * 32);
          }
          if (lane < U && bI + lane < eI) cp_async8(slot + VOFF + lane, v + bI + lane);
        }
        cp_async_commit();
        ++rI;
        if (rI < nrows) {
          bI = eI;
          eI = __shfl_sync(kFull, re, rI);
#pragma unroll
          for (int u = 0; u < U; ++u) cn[u] = bI + u < eI ? __ldg(ci + bI + u) : 0;
        }
      };
      for (int r = 0; r < S - 1; ++r) issue_next();
      int b = b0;
      for (int r = 0; r < nrows; ++r) {
        issue_next();  // row r + S - 1
        cp_async_wait<S - 1>();
        __syncwarp();  // the values area of the slot was filled by lanes 0..U-1
        const int e = __shfl_sync(kFull, re, r);
        const double* slot = ring + (r % S) * SLOT;
        double sum = 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (b + u < e) sum = dadd(sum, dmul(slot[VOFF + u], slot[u * 32 + lane]));
        for (int kk = b + U; kk < e; kk += U) {  // rows longer than U entries
          double xv[U];
          spmm_gather<U>(ci, X, kk, e, k, lane, on, xv);
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (kk + u < e) sum = dadd(sum, dmul(__ldg(v + kk + u), xv[u]));
        }
        if (on) epi.row(row0 + r, lane, sum, epi.staged(slot + U * 32, lane), acc);
        __syncwarp();  // every lane has read the values area before it is refilled
        b = e;
      }
      cp_async_wait<0>();
    }
    if (NR > 0) multi_tile_store<(NR > 0 ? NR : 1)>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<(NR > 0 ? NR : 1)>(red, epi, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, epi, 0, scratch, &s_flag, s_tot);
}

// Two rows per warp step (k even): half-warp h takes row 2j+h and lane l of a
// half owns columns 2l and 2l+1, so each gather is one 16-byte asynchronous
// copy and every instruction serves two rows.  A ring of S slots per warp
// holds a row pair's gathered entries, the two rows' matrix values and their
// epilogue operands.  Per column the rows still enter the reductions in
// order: each row's epilogue works on a zeroed term that is then added to the
// column's sum, the first row's before the second's.
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
constexpr int kPairU = 8;
// doubles per slot: X[U][32 lanes][2], epilogue operands [2 halves][2][32],
// matrix values [2 halves][U]
constexpr int kPairSlot = kPairU * 64 + 128 + 2 * kPairU;

template <class Epi, int S, int MINB>
__global__ void __launch_bounds__(kLanes, MINB) spmm_pair_kernel(const int* __restrict__ rp,
                                                                const int* __restrict__ ci,
                                                                const double* __restrict__ v, int n,
                                                                int k, const double* __restrict__ X,
                                                                Epi epi, RedCtx red) {
  constexpr int NR = Epi::NRED;
  constexpr int NR1 = NR > 0 ? NR : 1;
  constexpr int U = kPairU;
  constexpr int SLOT = kPairSlot;
  constexpr int PRE = U * 64;        // epilogue operands of half h at PRE + 64 h
  constexpr int VOFF = U * 64 + 128; // matrix values of half h at VOFF + U h
  constexpr unsigned kFull = 0xffffffffu;
  __shared__ double s_w[NR1 * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[NR1 * kMaxRhs];
  __shared__ int s_flag;
  extern __shared__ __align__(16) double s_ring[];
  if (!epi.active()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int hh = lane >> 4, hl = lane & 15;
  const int c0 = 2 * hl, c1 = c0 + 1;
  const bool in = c0 < k;
  const bool on0 = in && epi.col_active(c0), on1 = in && epi.col_active(c1);
  const bool on = on0 || on1;
  double* ring = s_ring + (long)warp * S * SLOT;
  const long ntiles = ((long)n + kTile - 1) / kTile;
  for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    double acc0[NR1], acc1[NR1];  // columns c0, c1 (kept in the first half)
#pragma unroll
    for (int r = 0; r < NR1; ++r) acc0[r] = acc1[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      if (row0 >= n) break;
      const int nrows = (int)min(32L, (long)n - row0);
      const int npairs = (nrows + 1) / 2;
      const int re = lane < nrows ? __ldg(rp + row0 + lane + 1) : 0;  // end of row lane
      const int b0 = __ldg(rp + row0);
      // next pair to issue and this half's row of it: entry range, first U columns
      int pI = 0;
      int rI = hh;
      bool vI = rI < nrows;
      const int prev0 = __shfl_sync(kFull, re, max(rI - 1, 0));
      int bI = rI == 0 ? b0 : prev0;
      int eI = __shfl_sync(kFull, re, min(rI, 31));
      if (!vI) bI = eI = 0;
      int cn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) cn[u] = bI + u < eI ? __ldg(ci + bI + u) : 0;
      auto issue_next = [&]() {
        if (pI < npairs) {
          double* slot = ring + (pI % S) * SLOT;
          if (vI) {
            if (on) {
#pragma unroll
              for (int u = 0; u < U; ++u)
                if (bI + u < eI) cp_async16(slot + u * 64 + lane * 2, X + (long)cn[u] * k + c0);
              if (on0) epi.stage_pre(row0 + rI, c0, slot + PRE + 64 * hh);
              if (on1) epi.stage_pre(row0 + rI, c1, slot + PRE + 64 * hh);
            }
            if (hl < U && bI + hl < eI) cp_async8(slot + VOFF + U * hh + hl, v + bI + hl);
          }
        }
        cp_async_commit();
        ++pI;
        if (pI < npairs) {
          rI = 2 * pI + hh;
          vI = rI < nrows;
          bI = __shfl_sync(kFull, re, max(rI - 1, 0));
          eI = __shfl_sync(kFull, re, min(rI, 31));
          if (!vI) bI = eI = 0;
#pragma unroll
          for (int u = 0; u < U; ++u) cn[u] = bI + u < eI ? __ldg(ci + bI + u) : 0;
        }
      };
      for (int r = 0; r < S - 1; ++r) issue_next();
      for (int pp = 0; pp < npairs; ++pp) {
        issue_next();  // pair pp + S - 1
        cp_async_wait<S - 1>();
        __syncwarp();
        const int row = 2 * pp + hh;
        const bool valid = row < nrows;
        const int prev = __shfl_sync(kFull, re, max(row - 1, 0));
        const int b = row == 0 ? b0 : prev;
        const int e = __shfl_sync(kFull, re, min(row, 31));
        const double* slot = ring + (pp % S) * SLOT;
        double t0[NR1], t1[NR1];
#pragma unroll
        for (int r = 0; r < NR1; ++r) t0[r] = t1[r] = 0.0;
        if (valid) {
          double s0 = 0.0, s1 = 0.0;
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (b + u < e) {
              const double vv = slot[VOFF + U * hh + u];
              s0 = dadd(s0, dmul(vv, slot[u * 64 + lane * 2]));
              s1 = dadd(s1, dmul(vv, slot[u * 64 + lane * 2 + 1]));
            }
          for (int kk = b + U; kk < e; ++kk) {  // rows longer than U entries
            const double vv = __ldg(v + kk);
            const long xo = (long)__ldg(ci + kk) * k + c0;
            s0 = dadd(s0, dmul(vv, on ? __ldg(X + xo) : 0.0));
            s1 = dadd(s1, dmul(vv, on ? __ldg(X + xo + 1) : 0.0));
          }
          const double* pre = slot + PRE + 64 * hh;
          if (on0) epi.row(row0 + row, c0, s0, epi.staged(pre, c0), t0);
          if (on1) epi.row(row0 + row, c1, s1, epi.staged(pre, c1), t1);
        }
        // the two rows' terms enter each column's sum in row order
#pragma unroll
        for (int r = 0; r < NR1; ++r) {
          const double u0 = __shfl_down_sync(kFull, t0[r], 16);
          const double u1 = __shfl_down_sync(kFull, t1[r], 16);
          acc0[r] = dadd(dadd(acc0[r], t0[r]), u0);
          acc1[r] = dadd(dadd(acc1[r], t1[r]), u1);
        }
        __syncwarp();  // every lane has read the slot before it is refilled
      }
      cp_async_wait<0>();
    }
    // lane c takes column c's sum from lane c/2 of the first half
    double acc[NR1];
#pragma unroll
    for (int r = 0; r < NR1; ++r) {
      const double ev = __shfl_sync(kFull, acc0[r], lane >> 1);
      const double od = __shfl_sync(kFull, acc1[r], lane >> 1);
      acc[r] = (lane & 1) ? od : ev;
    }
    if (NR > 0) multi_tile_store<NR1>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<NR1>(red, epi, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, epi, 0, scratch, &s_flag, s_tot);
}

// 16-byte vectors of the storage type and the row-sum step on them (each
// component: s = s + v x with separate roundings, as every SpMM here).
template <typename VT> struct Vec16;
template <> struct Vec16<double> { using T = double2; };
template <> struct Vec16<float> { using T = float4; };
__device__ __forceinline__ void vacc(double2& s, double v, const double2& x) {
  s.x = dadd(s.x, dmul(v, x.x));
  s.y = dadd(s.y, dmul(v, x.y));
}
__device__ __forceinline__ void vacc(float4& s, float v, const float4& x) {
  s.x = vadd(s.x, vmul(v, x.x));
  s.y = vadd(s.y, vmul(v, x.y));
  s.z = vadd(s.z, vmul(v, x.z));
  s.w = vadd(s.w, vmul(v, x.w));
}

// The same SpMM with 16-byte gathers and rows spread over lanes: a warp
// works on RS = 4 RP rows per step, lanes 8g..8g+7 on rows g, g+4, ... of
// the step (RP rows each, whose gathers are all in flight together).  Lane l
// of a row owns the W = 16 / sizeof(VT) columns W l + 8 W m (m < NV; FP64:
// columns 2l, 2l+1, 2l+16, 2l+17; FP32: 4l..4l+3), so one gather
// instruction reads 128 contiguous bytes of X for each of four rows (k a
// multiple of W, X 16-byte aligned).  Each lane sums its rows' entries in
// stored order for its columns; the row sums are then transposed through
// shared memory to lane = column, where the epilogue runs row by row in
// order, so the per-column reductions keep the (q, r) order of the other
// variants.  The FP64 epilogue's operands are staged into shared memory by
// cp.async at the start of the step (FP32: loaded into registers).  Per row
// and entry a warp issues half a gather (FP32: a quarter) instead of one,
// and the epilogue's loads and stores stay coalesced.  RP > 1 gives a warp
// more gathers in flight at fewer resident CTAs, which keeps the rows of X in
// use by all CTAs together within L2.
// PAT: the matrix's row patterns (pid, pat; spmv_kernels.cuh) give each
// entry's column as row + offset, so the X gathers need no column load.
template <class Epi, int MINB, int U, int RP, bool PAT>
__global__ void __launch_bounds__(kLanes, MINB) spmm_vec_kernel(const int* __restrict__ rp,
                                                               const int* __restrict__ ci,
                                                               const typename Epi::VT* __restrict__ v,
                                                               int n, int k,
                                                               const typename Epi::VT* __restrict__ X,
                                                               Epi epi, RedCtx red,
                                                               const uint8_t* __restrict__ pid,
                                                               const int* __restrict__ pat,
                                                               int pat_ints) {
  using VT = typename Epi::VT;
  using V16 = typename Vec16<VT>::T;
  constexpr int NR = Epi::NRED;
  constexpr int NR1 = NR > 0 ? NR : 1;
  constexpr int L = 8;                     // lanes per row
  constexpr int RS = 4 * RP;               // rows per step
  constexpr int W = 16 / (int)sizeof(VT);  // columns per 16-byte load
  constexpr int NV = 32 / (W * L);         // 16-byte loads per lane and entry
  constexpr bool kStaged = sizeof(VT) == 8;
  __shared__ double s_w[NR1 * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[NR1 * kMaxRhs];
  __shared__ int s_flag;
  // per warp: row sums [RS][32] (VT), then (FP64) the staged operands [RS][64]
  extern __shared__ __align__(16) double s_dyn[];
  if (!epi.active()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / L, l = lane % L;
  const bool on = lane < k && epi.col_active(lane);
  int cm[NV];
  bool gon[NV];
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    cm[m] = W * l + W * L * m;
    bool any = false;
#pragma unroll
    for (int w = 0; w < W; ++w) any = any || (cm[m] + w < k && epi.col_active(cm[m] + w));
    gon[m] = cm[m] < k && any;
  }
  constexpr int kWarpDoubles = RS * 32 * (int)sizeof(VT) / 8 + (kStaged ? RS * 64 : 0);
  VT* sw = reinterpret_cast<VT*>(s_dyn + (long)warp * kWarpDoubles);
  double* sp = s_dyn + (long)warp * kWarpDoubles + RS * 32 * (int)sizeof(VT) / 8;
  [[maybe_unused]] int* s_pat = reinterpret_cast<int*>(s_dyn + 8L * kWarpDoubles);
  if constexpr (PAT) {
    for (int q = threadIdx.x; q < pat_ints; q += blockDim.x) s_pat[q] = pat[q];
    __syncthreads();
  }
  const long ntiles = ((long)n + kTile - 1) / kTile;
  for (long kt = blockIdx.x; kt < ntiles; kt += gridDim.x) {
    const long t = tile_at(kt, ntiles, red.sweep);
    double acc[NR1];
#pragma unroll
    for (int r = 0; r < NR1; ++r) acc[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      if (row0 >= n) break;
      const int nrows = (int)min(32L, (long)n - row0);
      for (int s0 = 0; s0 < nrows; s0 += RS) {
        typename Epi::Pre pre[kStaged ? 1 : RS];
        if constexpr (kStaged) {
#pragma unroll
          for (int rr = 0; rr < RS; ++rr)
            if (on && s0 + rr < nrows) epi.stage_pre(row0 + s0 + rr, lane, sp + rr * 64);
          cp_async_commit();
        } else {
#pragma unroll
          for (int rr = 0; rr < RS; ++rr)
            if (on && s0 + rr < nrows) pre[rr] = epi.pre(row0 + s0 + rr, lane);
        }
        int b[RP], e[RP];
        [[maybe_unused]] const int* po[RP];
        int lmax = 0;
#pragma unroll
        for (int j = 0; j < RP; ++j) {
          const int r = s0 + g + 4 * j;
          b[j] = r < nrows ? __ldg(rp + row0 + r) : 0;
          e[j] = r < nrows ? __ldg(rp + row0 + r + 1) : 0;
          if constexpr (PAT) po[j] = s_pat + (r < nrows ? (int)__ldg(pid + row0 + r) : 0) * kPatLen;
          lmax = max(lmax, e[j] - b[j]);
        }
        V16 sum[RP][NV];
#pragma unroll
        for (int j = 0; j < RP; ++j)
#pragma unroll
          for (int m = 0; m < NV; ++m) sum[j][m] = V16{};
        for (int c0 = 0; c0 < lmax; c0 += U) {
          int cc[RP][U];
          VT vv[RP][U];
#pragma unroll
          for (int j = 0; j < RP; ++j)
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int kk = b[j] + c0 + u;
              if constexpr (PAT)
                cc[j][u] = kk < e[j] ? (int)(row0 + s0 + g + 4 * j) + po[j][c0 + u] : 0;
              else
                cc[j][u] = kk < e[j] ? __ldg(ci + kk) : 0;
              vv[j][u] = kk < e[j] ? __ldg(v + kk) : VT(0);
            }
          V16 xg[RP][U][NV];
#pragma unroll
          for (int j = 0; j < RP; ++j)
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const bool ok = b[j] + c0 + u < e[j];
              const VT* xr = X + (long)cc[j][u] * k;
#pragma unroll
              for (int m = 0; m < NV; ++m)
                xg[j][u][m] = (ok && gon[m]) ? __ldg(reinterpret_cast<const V16*>(xr + cm[m])) : V16{};
            }
#pragma unroll
          for (int j = 0; j < RP; ++j)
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (b[j] + c0 + u < e[j]) {
#pragma unroll
                for (int m = 0; m < NV; ++m) vacc(sum[j][m], vv[j][u], xg[j][u][m]);
              }
        }
#pragma unroll
        for (int j = 0; j < RP; ++j)
          if (s0 + g + 4 * j < nrows) {
            VT* srow = sw + (g + 4 * j) * 32;
#pragma unroll
            for (int m = 0; m < NV; ++m)
              if (cm[m] < k) *reinterpret_cast<V16*>(srow + cm[m]) = sum[j][m];
          }
        if constexpr (kStaged) cp_async_wait<0>();
        __syncwarp();
#pragma unroll
        for (int rr = 0; rr < RS; ++rr)
          if (on && s0 + rr < nrows) {
            if constexpr (kStaged)
              epi.row(row0 + s0 + rr, lane, sw[rr * 32 + lane], epi.staged(sp + rr * 64, lane), acc);
            else
              epi.row(row0 + s0 + rr, lane, sw[rr * 32 + lane], pre[rr], acc);
          }
        __syncwarp();  // the sums are read before the next step overwrites them
      }
    }
    if (NR > 0) multi_tile_store<NR1>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<NR1>(red, epi, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, epi, 0, scratch, &s_flag, s_tot);
}

// ---- n x k vector sweeps with per-column scalars ------------------------------
template <class Op>
__global__ void __launch_bounds__(kLanes) mtile_kernel(long n, int k, Op op_in, RedCtx red) {
  constexpr int NR = Op::NRED;
  __shared__ double s_w[(NR > 0 ? NR : 1) * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[(NR > 0 ? NR : 1) * kMaxRhs];
  __shared__ int s_flag;
  Op op = op_in;
  if (!op.prepare()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool on = lane < k && op.col_active(lane);
  op.begin_col(lane < k ? lane : 0);
  const long ntiles = (n + kTile - 1) / kTile;
  for (long kt = blockIdx.x; kt < ntiles; kt += gridDim.x) {
    const long t = tile_at(kt, ntiles, red.sweep);
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      for (int r4 = 0; r4 < 32; r4 += 4) {
        typename Op::Regs g[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (on && row0 + r4 + u < n) op.load((row0 + r4 + u) * k + lane, row0 + r4 + u, g[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (on && row0 + r4 + u < n) op.compute((row0 + r4 + u) * k + lane, row0 + r4 + u, g[u], acc);
      }
    }
    if (NR > 0) multi_tile_store<(NR > 0 ? NR : 1)>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<(NR > 0 ? NR : 1)>(red, op, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, op, 0, scratch, &s_flag, s_tot);
}

// The same sweeps with 16-byte accesses (k a multiple of W = 16 / element
// size, the arrays 16-byte aligned): in a step of W rows, lane l works on row
// l / (32 / W) of the step and the W columns W (l % (32 / W)) .. + W - 1, so
// every load and store moves 16 bytes per lane (FP32: 4 columns, FP64: 2).
// An op with W-column methods (loadv, begin_colv, computev, storev; kVecW)
// returns each element's reduction terms; they are transposed through
// shared memory to lane = column and added in row order there, so the
// per-column sums keep the order (and the bits) of mtile_kernel.
template <class T, class = void>
struct has_vecw : std::false_type {};
template <class T>
struct has_vecw<T, std::void_t<decltype(&T::storev)>> : std::true_type {};

template <class Op>
__global__ void __launch_bounds__(kLanes) mtile4_kernel(long n, int k, Op op_in, RedCtx red) {
  constexpr int W = Op::kVecW;
  static_assert(W == 2 || W == 4, "16-byte vectors of FP64 or FP32");
  // W-row steps whose loads are in flight together (FP32, 128^3 x 32
  // reliable-update step: 233 / 204 / 193 / 183 us for 1 / 2 / 4 / 8;
  // direction sweep 226 / 215 / 216 / 226 us)
  constexpr int RV = 4;
  static_assert(32 % (W * RV) == 0, "steps tile the warp's 32 rows");
  constexpr int NR = Op::NRED;
  constexpr int NR1 = NR > 0 ? NR : 1;
  __shared__ double s_w[NR1 * 8 * 32];
  __shared__ double scratch[8];
  __shared__ double s_tot[NR1 * kMaxRhs];
  __shared__ int s_flag;
  __shared__ __align__(16) double s_c[NR > 0 ? 8 : 1][NR1][W][32];
  Op op = op_in;
  if (!op.prepare()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gr = lane / (32 / W), c0 = W * (lane % (32 / W));
  const bool von = c0 < k;
  op.begin_colv(von ? c0 : 0);
  const long ntiles = (n + kTile - 1) / kTile;
  for (long kt = blockIdx.x; kt < ntiles; kt += gridDim.x) {
    const long t = tile_at(kt, ntiles, red.sweep);
    double acc[NR1];
#pragma unroll
    for (int r = 0; r < NR1; ++r) acc[r] = 0.0;
    for (int q = 0; q < 4; ++q) {
      const long row0 = t * kTile + q * kSub + warp * 32;
      if (row0 >= n) break;
      for (int r16 = 0; r16 < 32; r16 += W * RV) {
        // the loads of RV steps are issued before the first is used
        typename Op::RegsV g[RV];
#pragma unroll
        for (int v = 0; v < RV; ++v) {
          const long i = row0 + r16 + W * v + gr;
          if (von && i < n) op.loadv(i * k + c0, i, g[v]);
        }
#pragma unroll
        for (int v = 0; v < RV; ++v) {
        const int r4 = r16 + W * v;
        const long i = row0 + r4 + gr;
        const bool ok = von && i < n;
        double ct[NR1][W];
#pragma unroll
        for (int r = 0; r < NR1; ++r)
#pragma unroll
          for (int j = 0; j < W; ++j) ct[r][j] = 0.0;
        if (ok) {
          op.template computev<NR1>(g[v], ct);
          op.storev(i * k + c0, g[v]);
        }
        if constexpr (NR > 0) {
          if (von) {
#pragma unroll
            for (int r = 0; r < NR1; ++r)
#pragma unroll
              for (int j = 0; j < W; j += 2)
                *reinterpret_cast<double2*>(&s_c[warp][r][gr][c0 + j]) = make_double2(ct[r][j], ct[r][j + 1]);
          }
          __syncwarp();
          if (lane < k) {
#pragma unroll
            for (int gg = 0; gg < W; ++gg)
              if (row0 + r4 + gg < n) {
#pragma unroll
                for (int r = 0; r < NR1; ++r) acc[r] = dadd(acc[r], s_c[warp][r][gg][lane]);
              }
          }
          __syncwarp();  // the terms are read before the next step overwrites them
        }
        }
      }
    }
    if (NR > 0) multi_tile_store<NR1>(acc, s_w, k, t, red.ntiles, red.partials, warp, lane);
  }
  if (NR > 0) multi_grid_finish<NR1>(red, op, k, scratch, &s_flag, s_tot);
  else multi_grid_finish<1>(red, op, 0, scratch, &s_flag, s_tot);
}

__device__ __forceinline__ float f4c(const float4& v, int j) {
  return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}
__device__ __forceinline__ void f4s(float4& v, int j, float x) {
  if (j == 0) v.x = x;
  else if (j == 1) v.y = x;
  else if (j == 2) v.z = x;
  else v.w = x;
}

// ---- the sweeps of the multi-column PCG ------------------------------------------

// x0 and ||b|| per column.  With `part` set (the refinement's inner solves)
// only the columns with part[c] != 0 take part; n_active is then
// *part_count.
template <typename VT>
struct MOpPre {
  static constexpr int NRED = 1;
  struct Regs { VT b; };
  const VT* B;
  VT* X;
  int x0_mode;
  double eps_abs, eps_rel;
  MultiArgs a;
  const int* part = nullptr;
  const int* part_count = nullptr;
  const double* eps_rel_col = nullptr;  // per-column eps_rel (refinement inner solves)
  __device__ bool prepare() { return true; }
  __device__ bool col_active(int) const { return true; }
  __device__ void begin_col(int) {}
  __device__ void load(long e, long, Regs& g) const { g.b = __ldg(B + e); }
  __device__ void compute(long e, long, Regs& g, double* acc) const {
    if (x0_mode == CELG_X0_REF_ONES) X[e] = VT(1);
    else if (x0_mode == CELG_X0_ZERO) X[e] = VT(0);
    acc[0] = dadd(acc[0], dmul(D(g.b), D(g.b)));
  }
  __device__ void finish_col(int c, double* tot) const {
    a.bnorm[c] = sqrt(tot[0]);
    double e = eps_abs;
    const double er = eps_rel_col ? eps_rel_col[c] : eps_rel;
    if (er > 0.0 && er * a.bnorm[c] > e) e = er * a.bnorm[c];
    a.eps[c] = e;
    a.err[c] = 0;
    a.iter[c] = 0;
    a.active[c] = part ? (part[c] ? 1 : 0) : 1;
    a.vres[c] = 0.0;
  }
  __device__ void finish_global() const {
    *a.n_active = part_count ? *part_count : a.k;
    *a.xmask = 0u;
    *a.pmask = 0u;
  }
};

// r = b - (0 + A x); p = J r; alpha = r.p; ||r||  (columns set active by MOpPre)
template <typename VT_>
struct MEpiInit {
  using VT = VT_;
  static constexpr int NRED = 2;
  const VT* B;
  VT* R;
  VT* P;
  const VT* J;
  int k;
  MultiArgs a;
  struct Pre { VT b, J; };
  __device__ bool active() const { return true; }
  __device__ bool col_active(int c) const { return *(volatile int*)&a.active[c] != 0; }
  __device__ Pre pre(long i, int c) const { return Pre{__ldg(B + i * k + c), __ldg(J + i)}; }
  __device__ void stage_pre(long i, int c, double* st) const {
    cp_async8(st + c, B + i * k + c);
    cp_async8(st + 32 + c, J + i);
  }
  __device__ Pre staged(const double* st, int c) const { return Pre{st[c], st[32 + c]}; }
  __device__ void row(long i, int c, VT s, const Pre& g, double* acc) const {
    const long e = i * k + c;
    const VT ri = celg::R<VT>(__dsub_rn(D(g.b), D(vadd(VT(0), s))));
    R[e] = ri;
    const double z = dmul(D(ri), D(g.J));
    P[e] = celg::R<VT>(z);
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
  }
  __device__ void finish_col(int c, double* tot) const {
    if (!a.active[c]) return;
    a.alpha[c] = tot[0];
    a.norm[c] = sqrt(tot[1]);
    a.iter[c] = 0;
    a.settle(c);
  }
  __device__ void finish_global() const { set_cond(a.cond, *(volatile int*)a.n_active > 0); }
};

// K1: v = 0 + A p; pv per column; sigma = alpha / pv
template <typename VT_>
struct MEpiAp {
  using VT = VT_;
  static constexpr int NRED = 1;
  VT* V;
  const VT* P;
  int k;
  MultiArgs a;
  __device__ bool active() const { return *(volatile int*)a.n_active > 0; }
  struct Pre { VT p; };
  __device__ bool col_active(int c) const { return *(volatile int*)&a.active[c] != 0; }
  __device__ Pre pre(long i, int c) const { return Pre{__ldg(P + i * k + c)}; }
  __device__ void stage_pre(long i, int c, double* st) const { cp_async8(st + c, P + i * k + c); }
  __device__ Pre staged(const double* st, int c) const { return Pre{st[c]}; }
  __device__ void row(long i, int c, VT s, const Pre& g, double* acc) const {
    const VT vi = vadd(VT(0), s);
    V[i * k + c] = vi;
    acc[0] = dadd(acc[0], dmul(D(vi), D(g.p)));
  }
  __device__ void finish_col(int c, double* tot) const {
    if (!a.active[c]) return;
    const double sg = a.alpha[c] / tot[0];
    a.sigma[c] = sg;
    if (!isfinite(sg)) {
      a.err[c] = kErrBreakdown;
      a.active[c] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {}
};

// K2: r += (-sigma) v; rz, rr; per-column scalars and test.  The column's
// x += sigma p is left to the direction sweep, which reads the old p anyway
// (bit c of xmask), so this sweep reads neither X nor P.
template <typename VT>
struct MOpUpdate {
  static constexpr int NRED = 2;
  struct Regs { VT r, v, J; };
  VT* R;
  const VT* V;
  const VT* J;
  MultiArgs a;
  double sg;
  __device__ bool prepare() { return true; }
  __device__ bool col_active(int c) const { return *(volatile int*)&a.active[c] != 0; }
  __device__ void begin_col(int c) { sg = a.sigma[c]; }
  // v is not read again before the next update sweep: streamed
  // (evict-first), so that L2 keeps r for the direction sweep
  __device__ void load(long e, long i, Regs& g) const {
    g.r = R[e];
    g.v = __ldcs(V + e);
    g.J = __ldg(J + i);
  }
  __device__ void compute(long e, long, Regs& g, double* acc) const {
    const VT ri = celg::R<VT>(dadd(D(g.r), dmul(-sg, D(g.v))));
    R[e] = ri;
    const double z = dmul(D(ri), D(g.J));
    acc[0] = dadd(acc[0], dmul(D(ri), z));
    acc[1] = dadd(acc[1], dmul(D(ri), D(ri)));
  }
  __device__ void finish_col(int c, double* tot) const {
    if (!a.active[c]) return;
    a.beta[c] = tot[0] / a.alpha[c];
    a.alpha[c] = tot[0];
    a.norm[c] = sqrt(tot[1]);
    a.iter[c] += 1;
    atomicOr(a.xmask, 1u << c);
    a.settle(c);
  }
  __device__ void finish_global() const { set_cond(a.cond, *(volatile int*)a.n_active > 0); }
};

// K3: per column, x += sigma p when the update sweep left it pending (also
// after that sweep stopped the column), then p = beta p + J r while the
// column goes on.  The last CTA clears the pending mask.
template <typename VT>
struct MOpDirection {
  static constexpr int NRED = 0;
  struct Regs { VT p, r, J, x; };
  VT* P;
  const VT* R;
  const VT* J;
  VT* X;
  MultiArgs a;
  double bt = 0.0, sg = 0.0;
  bool xp = false, act = false;
  __device__ bool prepare() {
    return *(volatile int*)a.n_active > 0 || *(volatile unsigned*)a.xmask != 0u;
  }
  __device__ bool col_active(int c) const {
    return *(volatile int*)&a.active[c] != 0 || ((*(volatile unsigned*)a.xmask >> c) & 1u);
  }
  __device__ void begin_col(int c) {
    bt = a.beta[c];
    sg = a.sigma[c];
    act = *(volatile int*)&a.active[c] != 0;
    xp = ((*(volatile unsigned*)a.xmask >> c) & 1u) != 0;
  }
  // r and x are streamed (evict-first), so that L2 keeps the new p for the
  // SpMM
  __device__ void load(long e, long i, Regs& g) const {
    g.p = P[e];
    if (act) {
      g.r = __ldcs(R + e);
      g.J = __ldg(J + i);
    }
    if (xp) g.x = __ldcs(X + e);
  }
  __device__ void compute(long e, long, Regs& g, double*) const {
    if (xp) __stcs(X + e, celg::R<VT>(dadd(D(g.x), dmul(sg, D(g.p)))));
    if (act) P[e] = celg::R<VT>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const { *a.xmask = 0u; }
};

// The FP64 direction sweeps for a pair of iterations whose directions live
// in two blocks, p_k in P and p_k+1 in Q.  The even sweep writes p_k+1 =
// beta p_k + J r into Q and leaves x += sigma_k p_k pending for the columns
// that go on (bit c of pmask, sigma_k in sigprev[c]); a column that K2 just
// stopped gets its update at once.  The odd sweep applies x = (x + sigma_k
// p_k) + sigma_k+1 p_k+1 and writes p_k+2 over P.  X is read and stored once
// per two iterations, and every element gets the same roundings in the
// same order as with MOpDirection.
template <typename VT>
struct MOpDirectionDefer {
  static constexpr int NRED = 0;
  struct Regs { VT p, r, J, x; };
  const VT* P;
  VT* Q;
  const VT* R;
  const VT* J;
  VT* X;
  MultiArgs a;
  double bt = 0.0, sg = 0.0;
  bool xp = false, act = false;
  __device__ bool prepare() {
    return *(volatile int*)a.n_active > 0 || *(volatile unsigned*)a.xmask != 0u;
  }
  __device__ bool col_active(int c) const {
    return *(volatile int*)&a.active[c] != 0 || ((*(volatile unsigned*)a.xmask >> c) & 1u);
  }
  __device__ void begin_col(int c) {
    bt = a.beta[c];
    sg = a.sigma[c];
    act = *(volatile int*)&a.active[c] != 0;
    xp = ((*(volatile unsigned*)a.xmask >> c) & 1u) != 0;
  }
  // p_k is read again by the odd sweep, after the next SpMM: streamed
  __device__ void load(long e, long i, Regs& g) const {
    g.p = __ldcs(P + e);
    if (act) {
      g.r = __ldcs(R + e);
      g.J = __ldg(J + i);
    } else if (xp) {
      g.x = __ldcs(X + e);
    }
  }
  __device__ void compute(long e, long, Regs& g, double*) const {
    if (act) Q[e] = celg::R<VT>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
    else if (xp) __stcs(X + e, celg::R<VT>(dadd(D(g.x), dmul(sg, D(g.p)))));
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const {
    const unsigned xm = *(volatile unsigned*)a.xmask;
    unsigned pm = 0u;
    for (int c = 0; c < a.k; ++c)
      if (((xm >> c) & 1u) && *(volatile int*)&a.active[c] != 0) {
        a.sigprev[c] = a.sigma[c];
        pm |= 1u << c;
      }
    *a.pmask = pm;
    *a.xmask = 0u;
  }
};

template <typename VT>
struct MOpDirectionPair {
  static constexpr int NRED = 0;
  struct Regs { VT p, q, r, J, x; };
  VT* P;
  const VT* Q;
  const VT* R;
  const VT* J;
  VT* X;
  MultiArgs a;
  double bt = 0.0, sg = 0.0, sp = 0.0;
  bool xq = false, xp = false, act = false;
  __device__ bool prepare() {
    return *(volatile int*)a.n_active > 0 || *(volatile unsigned*)a.xmask != 0u ||
           *(volatile unsigned*)a.pmask != 0u;
  }
  __device__ bool col_active(int c) const {
    return *(volatile int*)&a.active[c] != 0 ||
           (((*(volatile unsigned*)a.xmask | *(volatile unsigned*)a.pmask) >> c) & 1u);
  }
  __device__ void begin_col(int c) {
    bt = a.beta[c];
    sg = a.sigma[c];
    sp = a.sigprev[c];
    act = *(volatile int*)&a.active[c] != 0;
    xp = ((*(volatile unsigned*)a.xmask >> c) & 1u) != 0;
    xq = ((*(volatile unsigned*)a.pmask >> c) & 1u) != 0;
  }
  __device__ void load(long e, long i, Regs& g) const {
    if (xq) g.p = __ldcs(P + e);
    if (xp || act) g.q = __ldcs(Q + e);
    if (act) {
      g.r = __ldcs(R + e);
      g.J = __ldg(J + i);
    }
    if (xq || xp) g.x = __ldcs(X + e);
  }
  __device__ void compute(long e, long, Regs& g, double*) const {
    if (xq || xp) {
      VT xv = g.x;
      if (xq) xv = celg::R<VT>(dadd(D(xv), dmul(sp, D(g.p))));
      if (xp) xv = celg::R<VT>(dadd(D(xv), dmul(sg, D(g.q))));
      __stcs(X + e, xv);
    }
    if (act) P[e] = celg::R<VT>(dadd(dmul(bt, D(g.q)), dmul(D(g.r), D(g.J))));
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const {
    *a.xmask = 0u;
    *a.pmask = 0u;
  }
};

// The FP32 update and direction sweeps of the refinement's inner solves
// with 4-column methods for mtile4_kernel (same arithmetic per element).
struct MOpUpdate32 : MOpUpdate<float> {
  static constexpr int kVecW = 4;
  struct RegsV { float4 r, v; float J; };
  double sg4[4];
  bool act4[4];
  __device__ void begin_colv(int c0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j < a.k ? c0 + j : 0;
      sg4[j] = a.sigma[c];
      act4[j] = c0 + j < a.k && *(volatile int*)&a.active[c] != 0;
    }
  }
  __device__ void loadv(long e, long i, RegsV& g) const {
    g.r = *reinterpret_cast<const float4*>(R + e);
    g.v = __ldcs(reinterpret_cast<const float4*>(V + e));
    g.J = __ldg(J + i);
  }
  template <int NR1>
  __device__ void computev(RegsV& g, double (&ct)[NR1][kVecW]) const {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (act4[j]) {
        const float ri = celg::R<float>(dadd(D(f4c(g.r, j)), dmul(-sg4[j], D(f4c(g.v, j)))));
        f4s(g.r, j, ri);
        const double z = dmul(D(ri), D(g.J));
        ct[0][j] = dmul(D(ri), z);
        ct[1][j] = dmul(D(ri), D(ri));
      }
  }
  __device__ void storev(long e, const RegsV& g) const { *reinterpret_cast<float4*>(R + e) = g.r; }
};

struct MOpDirection32 : MOpDirection<float> {
  static constexpr int kVecW = 4;
  struct RegsV { float4 p, r, x; float J; };
  double bt4[4], sg4[4];
  bool xp4[4], act4[4];
  bool anyx = false, anya = false;
  __device__ void begin_colv(int c0) {
    const unsigned xm = *(volatile unsigned*)a.xmask;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j < a.k ? c0 + j : 0;
      bt4[j] = a.beta[c];
      sg4[j] = a.sigma[c];
      act4[j] = c0 + j < a.k && *(volatile int*)&a.active[c] != 0;
      xp4[j] = c0 + j < a.k && ((xm >> c) & 1u) != 0;
    }
    anyx = xp4[0] || xp4[1] || xp4[2] || xp4[3];
    anya = act4[0] || act4[1] || act4[2] || act4[3];
  }
  __device__ void loadv(long e, long i, RegsV& g) const {
    g.p = *reinterpret_cast<const float4*>(P + e);
    if (anya) {
      g.r = __ldcs(reinterpret_cast<const float4*>(R + e));
      g.J = __ldg(J + i);
    }
    if (anyx) g.x = __ldcs(reinterpret_cast<const float4*>(X + e));
  }
  template <int NR1>
  __device__ void computev(RegsV& g, double (&)[NR1][kVecW]) const {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float pj = f4c(g.p, j);
      if (xp4[j]) f4s(g.x, j, celg::R<float>(dadd(D(f4c(g.x, j)), dmul(sg4[j], D(pj)))));
      if (act4[j])
        f4s(g.p, j, celg::R<float>(dadd(dmul(bt4[j], D(pj)), dmul(D(f4c(g.r, j)), D(g.J)))));
    }
  }
  __device__ void storev(long e, const RegsV& g) const {
    if (anyx) __stcs(reinterpret_cast<float4*>(X + e), g.x);
    if (anya) *reinterpret_cast<float4*>(P + e) = g.p;
  }
};

// The FP64 update sweep with 2-column methods for mtile4_kernel (16-byte
// accesses; same arithmetic per element): 302 -> 283 us at 128^3 x 32.  The
// direction sweep keeps one column per lane: at 2 columns per lane it needed
// 128 registers and took 437 us against 421.
__device__ __forceinline__ double d2c(const double2& v, int j) { return j == 0 ? v.x : v.y; }
__device__ __forceinline__ void d2s(double2& v, int j, double x) {
  if (j == 0) v.x = x;
  else v.y = x;
}

struct MOpUpdate64 : MOpUpdate<double> {
  static constexpr int kVecW = 2;
  struct RegsV { double2 r, v; double J; };
  double sg2[2];
  bool act2[2];
  __device__ void begin_colv(int c0) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = c0 + j < a.k ? c0 + j : 0;
      sg2[j] = a.sigma[c];
      act2[j] = c0 + j < a.k && *(volatile int*)&a.active[c] != 0;
    }
  }
  __device__ void loadv(long e, long i, RegsV& g) const {
    g.r = *reinterpret_cast<const double2*>(R + e);
    g.v = __ldcs(reinterpret_cast<const double2*>(V + e));
    g.J = __ldg(J + i);
  }
  template <int NR1>
  __device__ void computev(RegsV& g, double (&ct)[NR1][kVecW]) const {
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (act2[j]) {
        const double ri = dadd(d2c(g.r, j), dmul(-sg2[j], d2c(g.v, j)));
        d2s(g.r, j, ri);
        const double z = dmul(ri, g.J);
        ct[0][j] = dmul(ri, z);
        ct[1][j] = dmul(ri, ri);
      }
  }
  __device__ void storev(long e, const RegsV& g) const { *reinterpret_cast<double2*>(R + e) = g.r; }
};

// ||b - A x|| / ||b|| per column
struct MEpiVerify {
  using VT = double;
  static constexpr int NRED = 1;
  const double* B;
  int k;
  MultiArgs a;
  struct Pre { double b; };
  __device__ bool active() const { return true; }
  __device__ bool col_active(int) const { return true; }
  __device__ Pre pre(long i, int c) const { return Pre{__ldg(B + i * k + c)}; }
  __device__ void stage_pre(long i, int c, double* st) const { cp_async8(st + c, B + i * k + c); }
  __device__ Pre staged(const double* st, int c) const { return Pre{st[c]}; }
  __device__ void row(long, int, double s, const Pre& g, double* acc) const {
    const double ri = __dsub_rn(g.b, dadd(0.0, s));
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish_col(int c, double* tot) const {
    a.vres[c] = a.bnorm[c] > 0.0 ? sqrt(tot[0]) / a.bnorm[c] : sqrt(tot[0]);
  }
  __device__ void finish_global() const {}
};

// ---- FP32 PCG with FP64 reliable updates for every column (CELG_PREC_FP32_RU) ----
// The recurrence of ru_solve (ru.cu) for all columns at once: FP32 matrix and
// vectors, one FP32 SpMM per iteration, and per column the FP64 correction
// (x64 += d, r = b - A x64 with the FP64 matrix) whenever the column's FP32
// residual has fallen by delta since its last one.  A column's arithmetic is
// the single solve's; its reductions follow the multi-column order.

struct MultiRu {
  double* maxr;      // ||r64|| at the column's last reliable update
  double* rz_prev;   // rz before the column's current step
  double* norm64;    // the column's last FP64 residual norm
  int* updates;      // reliable updates so far (the set-up residual included)
  unsigned* umask;   // columns whose reliable update is due (bit c)
  double delta;
  cudaGraphConditionalHandle cond_update;  // IF node of the update (0: none)
};

__device__ __forceinline__ int mru_go(const MultiArgs& a, const MultiRu& u, int c) {
  return (a.err[c] == 0 && *(volatile const int*)a.errw == 0 && a.iter[c] < a.iter_max &&
          u.norm64[c] > a.eps[c])
             ? 1
             : 0;
}

// set-up: every column starts with a reliable update (the initial residual)
__global__ void mru_init_kernel(int k, MultiRu u) {
  const int c = threadIdx.x;
  if (c < k) u.updates[c] = 0;
  if (c == 0) *u.umask = k >= 32 ? 0xffffffffu : ((1u << k) - 1u);
}

// FP64 residual of the columns due for an update, and its FP32 copy:
//   r64 = b - (0 + A x);  r = (float) r64;  z = (double) r * J;  rz = r.z;  ||r64||^2
// init: also p = (float) z.
struct MEpiRuResidual {
  using VT = double;
  static constexpr int NRED = 2;
  const double* B;
  float* R32;
  float* P32;  // set-up only
  const float* J32;
  int k;
  MultiArgs a;
  MultiRu u;
  int init;
  struct Pre { double b; float J; };
  __device__ bool active() const { return *(volatile unsigned*)u.umask != 0u; }
  __device__ bool col_active(int c) const { return ((*(volatile unsigned*)u.umask >> c) & 1u) != 0; }
  __device__ Pre pre(long i, int c) const { return Pre{__ldg(B + i * k + c), __ldg(J32 + i)}; }
  __device__ void stage_pre(long i, int c, double* st) const {
    cp_async8(st + c, B + i * k + c);
    cp_async4(reinterpret_cast<float*>(st + 32) + c, J32 + i);
  }
  __device__ Pre staged(const double* st, int c) const {
    return Pre{st[c], reinterpret_cast<const float*>(st + 32)[c]};
  }
  __device__ void row(long i, int c, double s, const Pre& g, double* acc) const {
    const long e = i * k + c;
    const double r64 = __dsub_rn(g.b, dadd(0.0, s));
    const float rf = (float)r64;
    R32[e] = rf;
    const double z = dmul((double)rf, (double)g.J);
    if (init) P32[e] = (float)z;
    acc[0] = dadd(acc[0], dmul((double)rf, z));
    acc[1] = dadd(acc[1], dmul(r64, r64));
  }
  __device__ void finish_col(int c, double* tot) const {
    if (!((*u.umask >> c) & 1u)) return;
    u.norm64[c] = sqrt(tot[1]);
    u.maxr[c] = u.norm64[c];
    u.updates[c] += 1;
    if (init) {
      a.alpha[c] = tot[0];
      a.norm[c] = u.norm64[c];
    } else {
      a.beta[c] = tot[0] / u.rz_prev[c];
      a.alpha[c] = tot[0];
    }
    if (!mru_go(a, u, c) && a.active[c]) {
      a.active[c] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {
    *u.umask = 0u;
    set_cond(a.cond, *(volatile int*)a.n_active > 0);
  }
};

// r -= sigma v in FP32 arithmetic (r + (float)(-sigma) v); rz' = r.J r and
// ||r||^2 on exact products; the column's update decision.  d += sigma p is
// left pending (bit c of xmask) for the flush or the direction sweep.
struct MOpRuStep {
  static constexpr int NRED = 2;
  struct Regs { float r, v, J; };
  float* R32;
  const float* V32;
  const float* J32;
  MultiArgs a;
  MultiRu u;
  float nsg = 0.0f;
  __device__ bool prepare() {
    if (*(volatile int*)a.n_active > 0) return true;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      set_cond(u.cond_update, 0);
      set_cond(a.cond, 0);
    }
    return false;
  }
  __device__ bool col_active(int c) const { return *(volatile int*)&a.active[c] != 0; }
  __device__ void begin_col(int c) { nsg = (float)(-a.sigma[c]); }
  __device__ void load(long e, long i, Regs& g) const {
    g.r = R32[e];
    g.v = __ldcs(V32 + e);
    g.J = __ldg(J32 + i);
  }
  __device__ void compute(long e, long, Regs& g, double* acc) const {
    const float ri = fadd(g.r, fmul(nsg, g.v));
    R32[e] = ri;
    const double z = dmul((double)ri, (double)g.J);
    acc[0] = dadd(acc[0], dmul((double)ri, z));
    acc[1] = dadd(acc[1], dmul((double)ri, (double)ri));
  }
  // 4 columns c0..c0+3 per lane (mtile4_kernel, W = 4)
  static constexpr int kVecW = 4;
  struct RegsV { float4 r, v; float J; };
  float nsg4[4];
  bool act4[4];
  __device__ void begin_colv(int c0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j < a.k ? c0 + j : 0;
      nsg4[j] = (float)(-a.sigma[c]);
      act4[j] = c0 + j < a.k && *(volatile int*)&a.active[c] != 0;
    }
  }
  __device__ void loadv(long e, long i, RegsV& g) const {
    g.r = *reinterpret_cast<const float4*>(R32 + e);
    g.v = __ldcs(reinterpret_cast<const float4*>(V32 + e));
    g.J = __ldg(J32 + i);
  }
  template <int NR1>
  __device__ void computev(RegsV& g, double (&ct)[NR1][kVecW]) const {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (act4[j]) {
        const float ri = fadd(f4c(g.r, j), fmul(nsg4[j], f4c(g.v, j)));
        f4s(g.r, j, ri);
        const double z = dmul((double)ri, (double)g.J);
        ct[0][j] = dmul((double)ri, z);
        ct[1][j] = dmul((double)ri, (double)ri);
      }
  }
  __device__ void storev(long e, const RegsV& g) const {
    *reinterpret_cast<float4*>(R32 + e) = g.r;
  }
  __device__ void finish_col(int c, double* tot) const {
    if (!a.active[c]) return;
    u.rz_prev[c] = a.alpha[c];
    a.beta[c] = tot[0] / a.alpha[c];
    a.alpha[c] = tot[0];
    a.norm[c] = sqrt(tot[1]);
    a.iter[c] += 1;
    atomicOr(a.xmask, 1u << c);
    const int upd = (a.norm[c] < u.delta * u.maxr[c]) || (a.norm[c] <= a.eps[c]) ||
                    (a.iter[c] >= a.iter_max);
    if (upd) {
      atomicOr(u.umask, 1u << c);
    } else if (!(a.err[c] == 0 && *(volatile const int*)a.errw == 0 && a.iter[c] < a.iter_max &&
                 fabs(a.alpha[c]) > 0.0)) {
      a.active[c] = 0;
      atomicSub(a.n_active, 1);
    }
  }
  __device__ void finish_global() const {
    set_cond(u.cond_update, *(volatile unsigned*)u.umask != 0u);
    set_cond(a.cond, *(volatile int*)a.n_active > 0);
  }
};

// x64 += (double) d ; d = 0 for the columns due for an update (all columns
// with `always`).  A d += sigma p still pending from the step is applied
// first, with the step's rounding, and the column's mark is cleared.
struct MOpRuFlush {
  static constexpr int NRED = 0;
  struct Regs { double x; float d, p; };
  double* X;
  float* D32;
  const float* P32;  // null: nothing pending (the final flush)
  MultiArgs a;
  MultiRu u;
  int always;
  bool dp = false;
  double sg = 0.0;
  __device__ bool prepare() { return always || *(volatile unsigned*)u.umask != 0u; }
  __device__ bool col_active(int c) const {
    return always || ((*(volatile unsigned*)u.umask >> c) & 1u) != 0;
  }
  __device__ void begin_col(int c) {
    dp = P32 != nullptr && ((*(volatile unsigned*)a.xmask >> c) & 1u) != 0;
    sg = a.sigma[c];
  }
  __device__ void load(long e, long, Regs& g) const {
    g.x = X[e];
    g.d = D32[e];
    if (dp) g.p = __ldg(P32 + e);
  }
  __device__ void compute(long e, long, Regs& g, double*) const {
    const float di = dp ? (float)dadd((double)g.d, dmul(sg, (double)g.p)) : g.d;
    X[e] = dadd(g.x, (double)di);
    D32[e] = 0.0f;
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const {
    if (!always) *a.xmask &= ~*u.umask;
  }
};

// d += sigma p where the step left it pending, then p = beta p + J r while
// the column goes on.  The last CTA clears the pending marks.
struct MOpRuDirection {
  static constexpr int NRED = 0;
  struct Regs { float p, r, J, d; };
  float* P32;
  const float* R32;
  const float* J32;
  float* D32;
  MultiArgs a;
  double bt = 0.0, sg = 0.0;
  bool dp = false, act = false;
  __device__ bool prepare() {
    return *(volatile int*)a.n_active > 0 || *(volatile unsigned*)a.xmask != 0u;
  }
  __device__ bool col_active(int c) const {
    return *(volatile int*)&a.active[c] != 0 || ((*(volatile unsigned*)a.xmask >> c) & 1u);
  }
  __device__ void begin_col(int c) {
    bt = a.beta[c];
    sg = a.sigma[c];
    act = *(volatile int*)&a.active[c] != 0;
    dp = ((*(volatile unsigned*)a.xmask >> c) & 1u) != 0;
  }
  // r and d are streamed (evict-first), so that L2 keeps the new p
  __device__ void load(long e, long i, Regs& g) const {
    g.p = P32[e];
    if (act) {
      g.r = __ldcs(R32 + e);
      g.J = __ldg(J32 + i);
    }
    if (dp) g.d = __ldcs(D32 + e);
  }
  __device__ void compute(long e, long, Regs& g, double*) const {
    if (dp) __stcs(D32 + e, (float)dadd((double)g.d, dmul(sg, (double)g.p)));
    if (act) P32[e] = celg::R<float>(dadd(dmul(bt, D(g.p)), dmul(D(g.r), D(g.J))));
  }
  // 4 columns c0..c0+3 per lane (mtile4_kernel, W = 4)
  static constexpr int kVecW = 4;
  struct RegsV { float4 p, r, d; float J; };
  double bt4[4], sg4[4];
  bool dp4[4], act4[4];
  bool anyd = false, anya = false;
  __device__ void begin_colv(int c0) {
    const unsigned xm = *(volatile unsigned*)a.xmask;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j < a.k ? c0 + j : 0;
      bt4[j] = a.beta[c];
      sg4[j] = a.sigma[c];
      act4[j] = c0 + j < a.k && *(volatile int*)&a.active[c] != 0;
      dp4[j] = c0 + j < a.k && ((xm >> c) & 1u) != 0;
    }
    anyd = dp4[0] || dp4[1] || dp4[2] || dp4[3];
    anya = act4[0] || act4[1] || act4[2] || act4[3];
  }
  __device__ void loadv(long e, long i, RegsV& g) const {
    g.p = *reinterpret_cast<const float4*>(P32 + e);
    if (anya) {
      g.r = __ldcs(reinterpret_cast<const float4*>(R32 + e));
      g.J = __ldg(J32 + i);
    }
    if (anyd) g.d = __ldcs(reinterpret_cast<const float4*>(D32 + e));
  }
  template <int NR1>
  __device__ void computev(RegsV& g, double (&)[NR1][kVecW]) const {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float pj = f4c(g.p, j);
      if (dp4[j]) f4s(g.d, j, (float)dadd((double)f4c(g.d, j), dmul(sg4[j], (double)pj)));
      if (act4[j])
        f4s(g.p, j, celg::R<float>(dadd(dmul(bt4[j], D(pj)), dmul(D(f4c(g.r, j)), D(g.J)))));
    }
  }
  __device__ void storev(long e, const RegsV& g) const {
    if (anyd) __stcs(reinterpret_cast<float4*>(D32 + e), g.d);
    if (anya) *reinterpret_cast<float4*>(P32 + e) = g.p;
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const { *a.xmask = 0u; }
};

// ---- FP32 refinement of every column (celg_pcg_multirhs, CELG_PREC_FP32_IR) -----
// The outer loop of ir_solve (ir.cu) for all columns at once; each column
// keeps its own residual norm, outer count and status.

struct MultiIr {
  int* part;         // column needs an inner solve in this outer step
  int* done;
  int* status;
  int* outer;
  int* inner_total;
  int* part_count;
  int outer_max;
  double* tau_col;   // inner tolerance of the column's next inner solve
  double tau;        // inner_eps_rel
};

// r = b - (0 + A x) in FP64, ||r|| per column and the column's outer decision
struct MEpiIrResidual {
  using VT = double;
  static constexpr int NRED = 1;
  const double* B;
  double* Rr;
  int k;
  MultiArgs a;  // outer state: norm[c] = ||r||, eps[c] = tolerance
  MultiIr ir;
  struct Pre { double b; };
  __device__ bool active() const { return true; }
  __device__ bool col_active(int c) const { return *(volatile int*)&ir.done[c] == 0; }
  __device__ Pre pre(long i, int c) const { return Pre{__ldg(B + i * k + c)}; }
  __device__ void stage_pre(long i, int c, double* st) const { cp_async8(st + c, B + i * k + c); }
  __device__ Pre staged(const double* st, int c) const { return Pre{st[c]}; }
  __device__ void row(long i, int c, double s, const Pre& g, double* acc) const {
    const double ri = __dsub_rn(g.b, dadd(0.0, s));
    Rr[i * k + c] = ri;
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish_col(int c, double* tot) const {
    if (ir.done[c]) return;
    const double rn = sqrt(tot[0]);
    a.norm[c] = rn;
    int st = -1;
    if (rn <= a.eps[c]) st = CELG_OK;
    else if (!isfinite(rn)) st = kErrBreakdown;
    else if (ir.outer[c] >= ir.outer_max) st = CELG_ERR_NOCONV;
    if (st >= 0) {
      ir.done[c] = 1;
      ir.status[c] = st;
    } else {
      ir.part[c] = 1;
      ir.tau_col[c] = ir_step_tolerance(rn, a.eps[c], ir.tau);
      atomicAdd(ir.part_count, 1);
    }
  }
  __device__ void finish_global() const {}
};

// r32 = (float)(r * (1/||r||)) for the columns that refine
struct MOpIrToF32 {
  static constexpr int NRED = 0;
  struct Regs { double r; };
  const double* Rr;
  float* R32;
  MultiArgs a;
  MultiIr ir;
  double inv;
  __device__ bool prepare() { return true; }
  __device__ bool col_active(int c) const { return *(volatile int*)&ir.part[c] != 0; }
  __device__ void begin_col(int c) { inv = 1.0 / a.norm[c]; }
  __device__ void load(long e, long, Regs& g) const { g.r = __ldg(Rr + e); }
  __device__ void compute(long e, long, Regs& g, double*) const { R32[e] = (float)dmul(g.r, inv); }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const {}
};

// x = x + ||r|| * (double) d32 for the columns that refined
struct MOpIrAdd {
  static constexpr int NRED = 0;
  struct Regs { double x; float d; };
  double* X;
  const float* D32;
  MultiArgs a;
  MultiIr ir;
  double scale;
  __device__ bool prepare() { return true; }
  __device__ bool col_active(int c) const { return *(volatile int*)&ir.part[c] != 0; }
  __device__ void begin_col(int c) { scale = a.norm[c]; }
  __device__ void load(long e, long, Regs& g) const { g.x = X[e]; g.d = __ldg(D32 + e); }
  __device__ void compute(long e, long, Regs& g, double*) const {
    X[e] = dadd(g.x, dmul(scale, (double)g.d));
  }
  __device__ void finish_col(int, double*) const {}
  __device__ void finish_global() const {}
};

// after an inner solve (before the update): as ir_count_kernel of batched.cu
__global__ void mir_count_kernel(int k, MultiIr ir, const int* inner_iter, const int* inner_err) {
  const int c = threadIdx.x;
  if (c >= k || !ir.part[c]) return;
  ir.inner_total[c] += inner_iter[c];
  if (inner_err[c] != 0) {
    ir.done[c] = 1;
    ir.status[c] = inner_err[c];
    ir.part[c] = 0;
  } else {
    ir.outer[c] += 1;
  }
}

// SpMM launch variants: the register pipeline with the resident CTAs per SM
// its registers are budgeted for and its gather chunk width (2/8, 3/8, 3/4,
// 4/4), and the cp.async ring with row slots per warp / CTAs per SM of 2/4,
// 2/3, 3/3 and 4/2, and the two-rows-per-step ring (k even) with 2 slots at
// 2 CTAs per SM or 3 slots at 1.  The
// fastest for a matrix and k is picked by timing them (spmm_tune) before the
// first solve.
// 0-3 register pipeline, 4-7 cp.async ring, 8-9 row pairs, 10-14 16-byte
// gathers
constexpr int kSpmmNumCfgs = 15;

template <class Epi, int MINB, int U>
static int launch_spmm_cfg(celg_handle* h, const CsrDev& A, const typename Epi::VT* vals, int k,
                           const typename Epi::VT* X, const Epi& epi) {
  const long nt = ntiles_of(A.n);
  RedCtx red{h->partials, h->ticket, nt};
  if (A.n == 0) return CELG_OK;
  auto kern = spmm_kernel<Epi, MINB, U>;
  int per_sm = 0;
  CELG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLanes, 0));
  const int grid = grid_for_tiles(h, nt, std::max(1, per_sm));
  kern<<<grid, kLanes, 0, h->stream>>>(A.rp, A.ci, vals, A.n, k, X, epi, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

template <class Epi, int MINB, int U, int RP, bool PAT>
static int launch_spmm_vec_p(celg_handle* h, const CsrDev& A, const typename Epi::VT* vals, int k,
                             const typename Epi::VT* X, const Epi& epi) {
  using VT = typename Epi::VT;
  const long nt = ntiles_of(A.n);
  RedCtx red{h->partials, h->ticket, nt};
  if (A.n == 0) return CELG_OK;
  red.sweep = next_sweep(h, false);
  auto kern = spmm_vec_kernel<Epi, MINB, U, RP, PAT>;
  const int rs = 4 * RP;
  const int pat_ints = PAT ? A.npat * kPatLen : 0;
  const int smem =
      8 * (rs * 32 * (int)sizeof(VT) + (sizeof(VT) == 8 ? rs * 64 * 8 : 0)) + pat_ints * 4;
  if (const int st = allow_dynamic_smem<spmm_vec_kernel<Epi, MINB, U, RP, PAT>>(smem)) return st;
  int per_sm = 0;
  CELG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLanes, smem));
  const int grid = grid_for_tiles(h, nt, std::max(1, per_sm));
  kern<<<grid, kLanes, smem, h->stream>>>(A.rp, A.ci, vals, A.n, k, X, epi, red, A.pid, A.pat,
                                          pat_ints);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// The 16-byte-gather SpMM, on the row patterns when the matrix has them
// (same columns in the same order: the same sums).
template <class Epi, int MINB, int U, int RP>
static int launch_spmm_vec(celg_handle* h, const CsrDev& A, const typename Epi::VT* vals, int k,
                           const typename Epi::VT* X, const Epi& epi) {
  if (A.pid) return launch_spmm_vec_p<Epi, MINB, U, RP, true>(h, A, vals, k, X, epi);
  return launch_spmm_vec_p<Epi, MINB, U, RP, false>(h, A, vals, k, X, epi);
}

// SpMM of the FP32 solves: the 16-byte-gather kernel when k is a multiple
// of 4 and X is 16-byte aligned, in one of kSpmm32NumCfgs launch shapes
// (resident CTAs per SM / entries per gather round / rows per lane group:
// 4/4/1, 3/4/1, 3/2/2, 2/4/2, 2/8/1; picked by spmm_tune32), else the
// register pipeline.
constexpr int kSpmm32NumCfgs = 5;
template <class Epi>
static int launch_spmm_f32(celg_handle* h, const CsrDev& A, int k, const float* X, const Epi& epi,
                           int cfg32 = 0) {
  if ((k & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0) {
    switch (cfg32) {
      case 1: return launch_spmm_vec<Epi, 3, 4, 1>(h, A, A.v32, k, X, epi);
      case 2: return launch_spmm_vec<Epi, 3, 2, 2>(h, A, A.v32, k, X, epi);
      case 3: return launch_spmm_vec<Epi, 2, 4, 2>(h, A, A.v32, k, X, epi);
      case 4: return launch_spmm_vec<Epi, 2, 8, 1>(h, A, A.v32, k, X, epi);
      default: return launch_spmm_vec<Epi, 4, 4, 1>(h, A, A.v32, k, X, epi);
    }
  }
  return launch_spmm_cfg<Epi, 4, 4>(h, A, A.v32, k, X, epi);
}

template <class Epi, int S, int MINB>
static int launch_spmm_async(celg_handle* h, const CsrDev& A, int k, const double* X, const Epi& epi) {
  const long nt = ntiles_of(A.n);
  RedCtx red{h->partials, h->ticket, nt};
  if (A.n == 0) return CELG_OK;
  auto kern = spmm_async_kernel<Epi, S, MINB>;
  const int smem = 8 * S * kAsyncSlot * (int)sizeof(double);
  if (const int st = allow_dynamic_smem<spmm_async_kernel<Epi, S, MINB>>(smem)) return st;
  int per_sm = 0;
  CELG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLanes, smem));
  const int grid = grid_for_tiles(h, nt, std::max(1, per_sm));
  kern<<<grid, kLanes, smem, h->stream>>>(A.rp, A.ci, A.v, A.n, k, X, epi, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

template <class Epi, int S, int MINB>
static int launch_spmm_pair(celg_handle* h, const CsrDev& A, int k, const double* X, const Epi& epi) {
  const long nt = ntiles_of(A.n);
  RedCtx red{h->partials, h->ticket, nt};
  if (A.n == 0) return CELG_OK;
  auto kern = spmm_pair_kernel<Epi, S, MINB>;
  const int smem = 8 * S * kPairSlot * (int)sizeof(double);
  if (const int st = allow_dynamic_smem<spmm_pair_kernel<Epi, S, MINB>>(smem)) return st;
  int per_sm = 0;
  CELG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLanes, smem));
  const int grid = grid_for_tiles(h, nt, std::max(1, per_sm));
  kern<<<grid, kLanes, smem, h->stream>>>(A.rp, A.ci, A.v, A.n, k, X, epi, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

template <class Epi>
static int launch_spmm(celg_handle* h, const CsrDev& A, int k, const double* X, const Epi& epi,
                       int cfg) {
  // the two-rows-per-step and 16-byte-gather kernels need k even and 16-byte
  // aligned rows of X
  if (cfg >= 8 && ((k & 1) || (reinterpret_cast<uintptr_t>(X) & 15))) cfg = 5;
  switch (cfg) {
    case 10: return launch_spmm_vec<Epi, 2, 8, 1>(h, A, A.v, k, X, epi);
    case 11: return launch_spmm_vec<Epi, 3, 4, 1>(h, A, A.v, k, X, epi);
    case 12: return launch_spmm_vec<Epi, 4, 4, 1>(h, A, A.v, k, X, epi);
    case 13: return launch_spmm_vec<Epi, 2, 4, 2>(h, A, A.v, k, X, epi);
    case 14: return launch_spmm_vec<Epi, 3, 2, 2>(h, A, A.v, k, X, epi);
    case 8: return launch_spmm_pair<Epi, 2, 2>(h, A, k, X, epi);
    case 9: return launch_spmm_pair<Epi, 3, 1>(h, A, k, X, epi);
    case 0: return launch_spmm_cfg<Epi, 2, 8>(h, A, A.v, k, X, epi);
    case 1: return launch_spmm_cfg<Epi, 3, 8>(h, A, A.v, k, X, epi);
    case 2: return launch_spmm_cfg<Epi, 3, 4>(h, A, A.v, k, X, epi);
    case 3: return launch_spmm_cfg<Epi, 4, 4>(h, A, A.v, k, X, epi);
    case 4: return launch_spmm_async<Epi, 2, 4>(h, A, k, X, epi);
    case 5: return launch_spmm_async<Epi, 2, 3>(h, A, k, X, epi);
    case 6: return launch_spmm_async<Epi, 3, 3>(h, A, k, X, epi);
    default: return launch_spmm_async<Epi, 4, 2>(h, A, k, X, epi);
  }
}

// vec4: the op's FP32 arrays are 16-byte aligned (checked by the caller);
// the 16-byte sweep then runs when k is a multiple of 4
template <class Op>
static int launch_mtile(celg_handle* h, long n, int k, const Op& op, bool vec4 = false) {
  const long nt = ntiles_of(n);
  RedCtx red{h->partials, h->ticket, nt};
  red.sweep = next_sweep(h, false);
  if constexpr (has_vecw<Op>::value) {
    if (vec4 && k % Op::kVecW == 0) {
      const int grid =
          grid_for_tiles(h, nt, std::min(8, resident_per_sm<mtile4_kernel<Op>>(kLanes, 0)));
      mtile4_kernel<Op><<<grid, kLanes, 0, h->stream>>>(n, k, op, red);
      CELG_CUDA(cudaGetLastError());
      return CELG_OK;
    }
  }
  const int grid = grid_for_tiles(h, nt, std::min(8, resident_per_sm<mtile_kernel<Op>>(kLanes, 0)));
  mtile_kernel<Op><<<grid, kLanes, 0, h->stream>>>(n, k, op, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

}  // namespace celg

struct Multi {
  // SpMM variant picked for the last (matrix, n, k) tuned
  const void* tuned_mat = nullptr;
  int tuned_n = -1, tuned_k = -1, cfg = 0;
  size_t cap = 0;        // n*k of the work vectors
  double* work = nullptr;  // R, P, V
  size_t qcap = 0;
  double* work_q = nullptr;  // Q: the second direction block of the FP64 pairs
  double* dstate = nullptr;
  int* istate = nullptr;
  // FP32 refinement (allocated on first use)
  size_t f32cap = 0;
  float* f32 = nullptr;      // 5 x n*k floats: B32 D32 R32 P32 V32
  int* irs = nullptr;        // part, done, status, outer, inner_total (kMaxRhs each), part_count
  double* irtau = nullptr;   // inner tolerance per column
  double* dstate2 = nullptr; // inner-solve scalars
  int* istate2 = nullptr;
  // FP32 with reliable updates: maxr, rz_prev, norm64 (kMaxRhs each);
  // updates (kMaxRhs), umask
  double* rud = nullptr;
  int* rui = nullptr;
  // FP32 SpMM shape picked for the last (matrix, n, k) tuned
  const void* tuned32_mat = nullptr;
  int tuned32_n = -1, tuned32_k = -1, cfg32 = 0;
};

namespace celg {

// a destroyed matrix's address may be reused: drop its tuning record
int multi_tuned_cfg(Multi* m) { return (m && m->tuned_mat) ? m->cfg : -1; }
int multi_tuned_cfg32(Multi* m) { return (m && m->tuned32_mat) ? m->cfg32 : -1; }

void multi_forget_matrix(Multi* m, const void* mat) {
  if (m && m->tuned_mat == mat) m->tuned_mat = nullptr;
  if (m && m->tuned32_mat == mat) m->tuned32_mat = nullptr;
}

void multi_free(Multi* m) {
  if (!m) return;
  cudaFree(m->work);
  cudaFree(m->work_q);
  cudaFree(m->dstate);
  cudaFree(m->istate);
  cudaFree(m->f32);
  cudaFree(m->irs);
  cudaFree(m->irtau);
  cudaFree(m->dstate2);
  cudaFree(m->istate2);
  cudaFree(m->rud);
  cudaFree(m->rui);
  delete m;
}

// Times every SpMM variant (3 launches each after one warm-up) on this
// matrix and k with the iteration's own epilogue (v = A p with the per-column
// p.v), applied to B with the output in a work vector; the per-column state
// is set up first by MOpPre in the user-start mode, which leaves X alone, and
// the solve's own set-up overwrites everything the timing wrote.  Returns the
// fastest variant; CELG_SPMM_CFG=0..14 forces one (profiling).
static int spmm_tune(celg_handle* h, const CsrDev& A, int k, const double* B, double* X,
                     double* work, const MultiArgs& a, int* best) {
  if (const char* e = std::getenv("CELG_SPMM_CFG")) {
    *best = std::min(std::max(std::atoi(e), 0), kSpmmNumCfgs - 1);
    return CELG_OK;
  }
  int st = launch_mtile(h, A.n, k, MOpPre<double>{B, X, CELG_X0_USER, 0.0, 0.0, a});
  if (st) return st;
  // alpha = 0 keeps sigma = 0 / p.v finite, so no column drops out
  CELG_CUDA(cudaMemsetAsync(a.alpha, 0, sizeof(double) * kMaxRhs, h->stream));
  const MEpiAp<double> ep{work, B, k, a};
  float best_ms = 0.f;
  *best = 0;
  for (int c = 0; c < kSpmmNumCfgs; ++c) {
    st = launch_spmm(h, A, k, B, ep, c);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    for (int r = 0; r < 3 && !st; ++r) st = launch_spmm(h, A, k, B, ep, c);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
    CELG_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CELG_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (c == 0 || ms < best_ms) {
      best_ms = ms;
      *best = c;
    }
  }
  return CELG_OK;
}

// The FP32 SpMM shapes timed the same way on the FP32 copy of the matrix,
// with the iteration's epilogue applied to P32 (set to a finite constant) and
// the output in V32; the solve's own set-up overwrites both and the state.
// CELG_SPMM32_CFG=0..4 forces one (profiling).
static int spmm_tune32(celg_handle* h, const CsrDev& A, int k, const double* B, double* X,
                       float* P32, float* V32, size_t nk, const MultiArgs& a, int* best) {
  if (const char* e = std::getenv("CELG_SPMM32_CFG")) {
    *best = std::min(std::max(std::atoi(e), 0), kSpmm32NumCfgs - 1);
    return CELG_OK;
  }
  *best = 0;
  if ((k & 3) != 0 || (reinterpret_cast<uintptr_t>(P32) & 15) != 0) return CELG_OK;
  int st = launch_mtile(h, A.n, k, MOpPre<double>{B, X, CELG_X0_USER, 0.0, 0.0, a});
  if (st) return st;
  CELG_CUDA(cudaMemsetAsync(a.alpha, 0, sizeof(double) * kMaxRhs, h->stream));
  CELG_CUDA(cudaMemsetAsync(P32, 0x3f, sizeof(float) * nk, h->stream));  // 0.747f everywhere
  const MEpiAp<float> ep{V32, P32, k, a};
  float best_ms = 0.f;
  for (int c = 0; c < kSpmm32NumCfgs; ++c) {
    st = launch_spmm_f32(h, A, k, P32, ep, c);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    for (int r = 0; r < 3 && !st; ++r) st = launch_spmm_f32(h, A, k, P32, ep, c);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
    CELG_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CELG_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (c == 0 || ms < best_ms) {
      best_ms = ms;
      *best = c;
    }
  }
  return CELG_OK;
}

static int ensure_tuned32(celg_handle* h, Multi* mu, celg_mat* m, int k, const double* B, double* X,
                          float* P32, float* V32, size_t nk, const MultiArgs& a) {
  if (mu->tuned32_mat == (const void*)m && mu->tuned32_n == m->csr.n && mu->tuned32_k == k)
    return CELG_OK;
  const int st = spmm_tune32(h, m->csr, k, B, X, P32, V32, nk, a, &mu->cfg32);
  if (st) return st;
  mu->tuned32_mat = m;
  mu->tuned32_n = m->csr.n;
  mu->tuned32_k = k;
  return CELG_OK;
}

static MultiArgs multi_args(double* ds, int* is, int k, int iter_max, cudaGraphConditionalHandle cond,
                            const int* errw) {
  MultiArgs a;
  a.alpha = ds;
  a.sigma = a.alpha + kMaxRhs;
  a.beta = a.sigma + kMaxRhs;
  a.norm = a.beta + kMaxRhs;
  a.bnorm = a.norm + kMaxRhs;
  a.eps = a.bnorm + kMaxRhs;
  a.vres = a.eps + kMaxRhs;
  a.iter = is;
  a.active = a.iter + kMaxRhs;
  a.err = a.active + kMaxRhs;
  a.n_active = a.err + kMaxRhs;
  a.xmask = reinterpret_cast<unsigned*>(a.n_active + 1);
  a.pmask = a.xmask + 1;
  a.sigprev = a.vres + kMaxRhs;
  a.k = k;
  a.iter_max = iter_max;
  a.errw = errw;
  a.cond = cond;
  return a;
}

static int multirhs_ir(celg_handle* h, celg_mat* m, int k, const double* B, double* X,
                       const celg_params* p, celg_result* res);
static int multirhs_ru(celg_handle* h, celg_mat* m, int k, const double* B, double* X,
                       const celg_params* p, celg_result* res);

int pcg_multirhs(celg_handle* h, celg_mat* m, int k, const double* B, double* X,
                 const celg_params* p, celg_result* res) {
  // row patterns (or 1-byte offsets) of the matrix, before the SpMM variants
  // are timed: the 16-byte-gather SpMM reads them instead of the columns
  if (const int st = ensure_offset_dict(h, m)) return st;
  if (p->precision == CELG_PREC_FP32_IR) return multirhs_ir(h, m, k, B, X, p, res);
  if (p->precision == CELG_PREC_FP32_RU) return multirhs_ru(h, m, k, B, X, p, res);
  if (p->precision != CELG_PREC_FP64) return CELG_ERR_ARG;
  const long n = m->csr.n;
  const size_t nk = (size_t)n * (size_t)k;
  if (!h->multi) h->multi = new Multi();
  Multi* mu = h->multi;
  if (nk > mu->cap || !mu->work) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->work);
    mu->work = nullptr;
    CELG_CUDA(cudaMalloc(&mu->work, sizeof(double) * std::max<size_t>(nk, 1) * 3));
    mu->cap = nk;
  }
  if (!mu->dstate) CELG_CUDA(cudaMalloc(&mu->dstate, sizeof(double) * 8 * kMaxRhs));
  if (!mu->istate) CELG_CUDA(cudaMalloc(&mu->istate, sizeof(int) * (3 * kMaxRhs + 3)));
  if (nk > mu->qcap || !mu->work_q) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->work_q);
    mu->work_q = nullptr;
    CELG_CUDA(cudaMalloc(&mu->work_q, sizeof(double) * std::max<size_t>(nk, 1)));
    mu->qcap = nk;
  }
  int st = ensure_partials(h, ntiles_of(n), 2 * k);
  if (st) return st;
  double* R = mu->work;
  double* P = R + nk;
  double* V = P + nk;
  double* Q = mu->work_q;
  MultiArgs a;
  a.alpha = mu->dstate;
  a.sigma = a.alpha + kMaxRhs;
  a.beta = a.sigma + kMaxRhs;
  a.norm = a.beta + kMaxRhs;
  a.bnorm = a.norm + kMaxRhs;
  a.eps = a.bnorm + kMaxRhs;
  a.vres = a.eps + kMaxRhs;
  a.iter = mu->istate;
  a.active = a.iter + kMaxRhs;
  a.err = a.active + kMaxRhs;
  a.n_active = a.err + kMaxRhs;
  a.xmask = reinterpret_cast<unsigned*>(a.n_active + 1);
  a.pmask = a.xmask + 1;
  a.sigprev = a.vres + kMaxRhs;
  a.k = k;
  a.iter_max = p->iter_max;
  a.errw = h->err_d;
  a.cond = 0;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  if (mu->tuned_mat != (const void*)m || mu->tuned_n != (int)n || mu->tuned_k != k) {
    st = spmm_tune(h, m->csr, k, B, X, V, a, &mu->cfg);
    if (st) return st;
    mu->tuned_mat = m;
    mu->tuned_n = (int)n;
    mu->tuned_k = k;
  }
  const int cfg = mu->cfg;
  auto setup = [&](const MultiArgs& ac) -> int {
    int s2 = launch_mtile(h, n, k, MOpPre<double>{B, X, p->x0_mode, p->eps_abs, p->eps_rel, ac});
    if (!s2) s2 = launch_spmm(h, m->csr, k, X, MEpiInit<double>{B, R, P, m->jacobi, k, ac}, cfg);
    return s2;
  };
  // the 16-byte update sweep: R and V start at multiples of n k doubles from
  // a cudaMalloc base
  const bool vw_r = (k & 1) == 0;
  // one iteration of a pair: directions in P, then in Q
  auto body = [&](const MultiArgs& ac, bool odd) -> int {
    double* Pc = odd ? Q : P;
    int s3 = launch_spmm(h, m->csr, k, Pc, MEpiAp<double>{V, Pc, k, ac}, cfg);
    if (!s3) s3 = launch_mtile(h, n, k, MOpUpdate64{{R, V, m->jacobi, ac, 0.0}}, vw_r);
    if (s3) return s3;
    if (odd) return launch_mtile(h, n, k, MOpDirectionPair<double>{P, Q, R, m->jacobi, X, ac});
    return launch_mtile(h, n, k, MOpDirectionDefer<double>{P, Q, R, m->jacobi, X, ac});
  };
  auto tail = [&](const MultiArgs& ac) -> int {
    return launch_spmm(h, m->csr, k, X, MEpiVerify{B, k, ac}, cfg);
  };
  if (!graphs_enabled()) {
    // profiling mode: the same kernels from a host loop (see graph.cuh)
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    a.cond = 0;
    st = setup(a);
    for (int it = 0; !st && it < p->iter_max; it += 8) {
      for (int q = 0; q < 8 && !st; ++q) st = body(a, (q & 1) != 0);
      int act = 0;
      if (!st) {
        CELG_CUDA(cudaMemcpyAsync(&act, a.n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CELG_CUDA(cudaStreamSynchronize(h->stream));
      }
      if (!act) break;
    }
    if (!st) st = tail(a);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    auto record = [&](cudaGraphConditionalHandle cond) -> int {
      MultiArgs ac = a;
      ac.cond = cond;
      int s2 = setup(ac);
      if (!s2) s2 = capture_while(h, cond, [&]() -> int {
        int s3 = body(ac, false);
        if (!s3) s3 = body(ac, true);
        return s3;
      });
      if (!s2) s2 = tail(ac);
      return s2;
    };
    char kb[256];
    std::snprintf(kb, sizeof(kb), "mrhs|%p|%d|%d|%p|%p|%p|%d|%.17g|%.17g|%d|%d", (const void*)m, m->csr.n,
                  k, (const void*)B, (const void*)X, (const void*)R, p->x0_mode, p->eps_abs, p->eps_rel,
                  p->iter_max, cfg);
    const std::string key(kb);
    GraphEntry* ge = graph_cache_find(h, key);
    if (!ge) {
      st = graph_build(h, key, record, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  std::vector<double> ds(7 * kMaxRhs);
  std::vector<int> is(3 * kMaxRhs + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), mu->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), mu->istate, sizeof(int) * is.size(), cudaMemcpyDeviceToHost, h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, iters = 0;
  for (int c = 0; c < k; ++c) {
    const double alpha = ds[c], norm = ds[3 * kMaxRhs + c], eps = ds[5 * kMaxRhs + c];
    const int it = is[c], err = is[2 * kMaxRhs + c];
    int rs = CELG_OK;
    if (err) rs = err;
    else if (!(norm <= eps) && it >= p->iter_max && std::fabs(alpha) > kRealSmall) rs = CELG_ERR_NOCONV;
    if (rs && !ret) ret = rs;
    iters = std::max(iters, it);
    if (res) {
      res[c].iter_done = it;
      res[c].final_norm2 = norm;
      res[c].bnorm = ds[4 * kMaxRhs + c];
      res[c].verified_relres = ds[6 * kMaxRhs + c];
      res[c].err = rs;
      res[c].arnoldi_steps = 0;
      res[c].history_len = 0;
    }
  }
  h->last_iters = iters;
  h->last_bytes_per_iter = 12.0 * m->csr.nnz + 4.0 * (n + 1) + 76.0 * (double)nk + 16.0 * n;
  return ret;
}

// FP32 refinement of every column: the outer loop of ir_solve for all
// columns at once around one FP32 multi-column inner PCG per outer step (the
// same sweeps instantiated for float storage; register-pipeline SpMM).
template <class Body>
static int multi_run_while(celg_handle* h, cudaGraphConditionalHandle cond, const int* n_active,
                           int iter_max, Body&& body) {
  if (cond) return capture_while2(h, cond, body);
  for (int it = 0; it < iter_max; it += 8) {
    int st = CELG_OK;
    for (int q = 0; q < 8 && !st; ++q) st = body();
    if (st) return st;
    int live = 0;
    CELG_CUDA(cudaMemcpyAsync(&live, n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    if (!live) break;
  }
  return CELG_OK;
}

static int record_multi_inner(celg_handle* h, celg_mat* m, int k, float* F, size_t nk,
                              const MultiIr& ir, MultiArgs ai, double inner_eps, int cfg32) {
  const long n = m->csr.n;
  float* B32 = F;
  float* D32 = B32 + nk;
  float* R32 = D32 + nk;
  float* P32 = R32 + nk;
  float* V32 = P32 + nk;
  const float* J32 = m->jacobi32;
  // the arrays start at multiples of n k floats from a cudaMalloc base
  const bool vec4 = (k & 3) == 0 && (reinterpret_cast<uintptr_t>(F) & 15) == 0;
  const MOpPre<float> pre{B32, D32, CELG_X0_ZERO, 0.0, inner_eps, ai, ir.part, ir.part_count,
                          ir.tau_col};
  int st = launch_mtile(h, n, k, pre);
  if (!st)
    st = launch_spmm_f32(h, m->csr, k, D32, MEpiInit<float>{B32, R32, P32, J32, k, ai}, cfg32);
  if (!st)
    st = multi_run_while(h, ai.cond, ai.n_active, ai.iter_max, [&]() -> int {
      int s2 = launch_spmm_f32(h, m->csr, k, P32, MEpiAp<float>{V32, P32, k, ai}, cfg32);
      if (!s2) s2 = launch_mtile(h, n, k, MOpUpdate32{{R32, V32, J32, ai, 0.0}}, vec4);
      if (!s2) s2 = launch_mtile(h, n, k, MOpDirection32{{P32, R32, J32, D32, ai}}, vec4);
      return s2;
    });
  return st;
}

static int multirhs_ir(celg_handle* h, celg_mat* m, int k, const double* B, double* X,
                       const celg_params* p, celg_result* res) {
  const long n = m->csr.n;
  const size_t nk = (size_t)n * (size_t)k;
  if (!m->csr.v32 || !m->jacobi32) {
    int st = celg_mat_make_fp32(m);
    if (st) return st;
  }
  if (!h->multi) h->multi = new Multi();
  Multi* mu = h->multi;
  if (nk > mu->cap || !mu->work) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->work);
    mu->work = nullptr;
    CELG_CUDA(cudaMalloc(&mu->work, sizeof(double) * std::max<size_t>(nk, 1) * 3));
    mu->cap = nk;
  }
  if (!mu->dstate) CELG_CUDA(cudaMalloc(&mu->dstate, sizeof(double) * 8 * kMaxRhs));
  if (!mu->istate) CELG_CUDA(cudaMalloc(&mu->istate, sizeof(int) * (3 * kMaxRhs + 3)));
  if (nk > mu->f32cap || !mu->f32) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->f32);
    mu->f32 = nullptr;
    CELG_CUDA(cudaMalloc(&mu->f32, sizeof(float) * std::max<size_t>(nk, 1) * 5));
    mu->f32cap = nk;
  }
  if (!mu->irs) CELG_CUDA(cudaMalloc(&mu->irs, sizeof(int) * (5 * kMaxRhs + 1)));
  if (!mu->irtau) CELG_CUDA(cudaMalloc(&mu->irtau, sizeof(double) * kMaxRhs));
  if (!mu->dstate2) CELG_CUDA(cudaMalloc(&mu->dstate2, sizeof(double) * 8 * kMaxRhs));
  if (!mu->istate2) CELG_CUDA(cudaMalloc(&mu->istate2, sizeof(int) * (3 * kMaxRhs + 3)));
  int st = ensure_partials(h, ntiles_of(n), 2 * k);
  if (st) return st;
  double* Rr = mu->work;
  const int inner_max = p->inner_iter_max > 0 ? p->inner_iter_max : 1000;
  const double inner_eps = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-4;
  MultiIr ir;
  ir.part = mu->irs;
  ir.done = ir.part + kMaxRhs;
  ir.status = ir.done + kMaxRhs;
  ir.outer = ir.status + kMaxRhs;
  ir.inner_total = ir.outer + kMaxRhs;
  ir.part_count = ir.inner_total + kMaxRhs;
  ir.outer_max = p->outer_max > 0 ? p->outer_max : 20;
  ir.tau_col = mu->irtau;
  ir.tau = inner_eps;
  const MultiArgs a = multi_args(mu->dstate, mu->istate, k, p->iter_max, 0, h->err_d);
  const MultiArgs ai_host = multi_args(mu->dstate2, mu->istate2, k, inner_max, 0, h->err_d);
  if (mu->tuned_mat != (const void*)m || mu->tuned_n != (int)n || mu->tuned_k != k) {
    st = spmm_tune(h, m->csr, k, B, X, mu->work + 2 * nk, a, &mu->cfg);
    if (st) return st;
    mu->tuned_mat = m;
    mu->tuned_n = (int)n;
    mu->tuned_k = k;
  }
  const int cfg = mu->cfg;
  st = ensure_tuned32(h, mu, m, k, B, X, mu->f32 + 3 * nk, mu->f32 + 4 * nk, nk, a);
  if (st) return st;
  const int cfg32 = mu->cfg32;
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
  st = launch_mtile(h, n, k, MOpPre<double>{B, X, p->x0_mode, p->eps_abs, p->eps_rel, a});
  CELG_CUDA(cudaMemsetAsync(ir.part, 0, sizeof(int) * (5 * kMaxRhs + 1), h->stream));
  char kb[160];
  std::snprintf(kb, sizeof(kb), "mrhs-ir|%p|%d|%d|%p|%d|%.17g|%d", (const void*)m, m->csr.n, k,
                (const void*)mu->f32, inner_max, inner_eps, cfg32);
  const std::string gkey(kb);
  for (int it = 0; !st && it <= ir.outer_max; ++it) {
    CELG_CUDA(cudaMemsetAsync(ir.part, 0, sizeof(int) * kMaxRhs, h->stream));
    CELG_CUDA(cudaMemsetAsync(ir.part_count, 0, sizeof(int), h->stream));
    st = launch_spmm(h, m->csr, k, X, MEpiIrResidual{B, Rr, k, a, ir}, cfg);
    if (st) break;
    int parts = 0;
    CELG_CUDA(cudaMemcpyAsync(&parts, ir.part_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    if (parts == 0) break;
    st = launch_mtile(h, n, k, MOpIrToF32{Rr, mu->f32, a, ir, 0.0});
    if (st) break;
    if (graphs_enabled()) {
      GraphEntry* ge = graph_cache_find(h, gkey);
      if (!ge) {
        st = graph_build(h, gkey, [&](cudaGraphConditionalHandle cond) -> int {
          return record_multi_inner(h, m, k, mu->f32, nk, ir,
                                    multi_args(mu->dstate2, mu->istate2, k, inner_max, cond, h->err_d),
                                    inner_eps, cfg32);
        }, &ge);
        if (st) break;
      }
      CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    } else {
      st = record_multi_inner(h, m, k, mu->f32, nk, ir, ai_host, inner_eps, cfg32);
      if (st) break;
    }
    mir_count_kernel<<<1, kMaxRhs, 0, h->stream>>>(k, ir, ai_host.iter, ai_host.err);
    CELG_CUDA(cudaGetLastError());
    st = launch_mtile(h, n, k, MOpIrAdd{X, mu->f32 + nk, a, ir, 0.0});
  }
  if (st) return st;
  CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  std::vector<double> ds(7 * kMaxRhs);
  std::vector<int> is(5 * kMaxRhs + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), mu->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), ir.part, sizeof(int) * is.size(), cudaMemcpyDeviceToHost,
                            h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, inner_most = 0;
  for (int c = 0; c < k; ++c) {
    const int done = is[kMaxRhs + c], status = is[2 * kMaxRhs + c];
    const int outer = is[3 * kMaxRhs + c], inner = is[4 * kMaxRhs + c];
    const double rn = ds[3 * kMaxRhs + c], bn = ds[4 * kMaxRhs + c];
    const int rs = done ? status : CELG_ERR_NOCONV;
    if (rs && !ret) ret = rs;
    inner_most = std::max(inner_most, inner);
    if (res) {
      res[c].iter_done = outer;
      res[c].final_norm2 = rn;
      res[c].bnorm = bn;
      res[c].verified_relres = bn > 0 ? rn / bn : rn;
      res[c].err = rs;
      res[c].arnoldi_steps = inner;
      res[c].history_len = 0;
    }
  }
  h->last_iters = inner_most;
  return ret;
}

// FP32 PCG with FP64 reliable updates for every column: one graph launch
// with a WHILE node over { FP32 SpMM, step, IF(any column due) { flush, FP64
// residual SpMM }, direction }; self-skipping kernels from a host loop when
// graphs are off.
static int multirhs_ru(celg_handle* h, celg_mat* m, int k, const double* B, double* X,
                       const celg_params* p, celg_result* res) {
  const long n = m->csr.n;
  const size_t nk = (size_t)n * (size_t)k;
  if (!m->csr.v32 || !m->jacobi32) {
    int st = celg_mat_make_fp32(m);
    if (st) return st;
  }
  if (!h->multi) h->multi = new Multi();
  Multi* mu = h->multi;
  if (nk > mu->cap || !mu->work) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->work);
    mu->work = nullptr;
    CELG_CUDA(cudaMalloc(&mu->work, sizeof(double) * std::max<size_t>(nk, 1) * 3));
    mu->cap = nk;
  }
  if (!mu->dstate) CELG_CUDA(cudaMalloc(&mu->dstate, sizeof(double) * 8 * kMaxRhs));
  if (!mu->istate) CELG_CUDA(cudaMalloc(&mu->istate, sizeof(int) * (3 * kMaxRhs + 3)));
  if (nk > mu->f32cap || !mu->f32) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(mu->f32);
    mu->f32 = nullptr;
    CELG_CUDA(cudaMalloc(&mu->f32, sizeof(float) * std::max<size_t>(nk, 1) * 5));
    mu->f32cap = nk;
  }
  if (!mu->rud) CELG_CUDA(cudaMalloc(&mu->rud, sizeof(double) * 3 * kMaxRhs));
  if (!mu->rui) CELG_CUDA(cudaMalloc(&mu->rui, sizeof(int) * (kMaxRhs + 1)));
  int st = ensure_partials(h, ntiles_of(n), 2 * k);
  if (st) return st;
  float* D32 = mu->f32;
  float* R32 = D32 + nk;
  float* P32 = R32 + nk;
  float* V32 = P32 + nk;
  const float* J32 = m->jacobi32;
  MultiArgs a = multi_args(mu->dstate, mu->istate, k, p->iter_max, 0, h->err_d);
  MultiRu u;
  u.maxr = mu->rud;
  u.rz_prev = u.maxr + kMaxRhs;
  u.norm64 = u.rz_prev + kMaxRhs;
  u.updates = mu->rui;
  u.umask = reinterpret_cast<unsigned*>(u.updates + kMaxRhs);
  u.delta = p->inner_eps_rel > 0 ? p->inner_eps_rel : 1e-2;
  u.cond_update = 0;
  if (mu->tuned_mat != (const void*)m || mu->tuned_n != (int)n || mu->tuned_k != k) {
    st = spmm_tune(h, m->csr, k, B, X, mu->work + 2 * nk, a, &mu->cfg);
    if (st) return st;
    mu->tuned_mat = m;
    mu->tuned_n = (int)n;
    mu->tuned_k = k;
  }
  const int cfg = mu->cfg;
  st = ensure_tuned32(h, mu, m, k, B, X, P32, V32, nk, a);
  if (st) return st;
  const int cfg32 = mu->cfg32;
  // the FP32 work arrays start at multiples of n k floats from a cudaMalloc
  // base: 16-byte aligned when k is a multiple of 4
  const bool vec4 = (k & 3) == 0 && (reinterpret_cast<uintptr_t>(D32) & 15) == 0;
  auto setup = [&](const MultiArgs& ac) -> int {
    int s2 = launch_mtile(h, n, k, MOpPre<double>{B, X, p->x0_mode, p->eps_abs, p->eps_rel, ac});
    if (!s2) {
      mru_init_kernel<<<1, kMaxRhs, 0, h->stream>>>(k, u);
      CELG_CUDA(cudaGetLastError());
      CELG_CUDA(cudaMemsetAsync(D32, 0, sizeof(float) * nk, h->stream));
      s2 = launch_spmm(h, m->csr, k, X, MEpiRuResidual{B, R32, P32, J32, k, ac, u, 1}, cfg);
    }
    return s2;
  };
  auto body = [&](const MultiArgs& ac, bool in_graph) -> int {
    MultiRu uc = u;
    if (in_graph) {
      int s2 = capture_new_handle(h, 0, &uc.cond_update);
      if (s2) return s2;
    }
    int s3 = launch_spmm_f32(h, m->csr, k, P32, MEpiAp<float>{V32, P32, k, ac}, cfg32);
    if (!s3) s3 = launch_mtile(h, n, k, MOpRuStep{R32, V32, J32, ac, uc}, vec4);
    auto update = [&]() -> int {
      int s4 = launch_mtile(h, n, k, MOpRuFlush{X, D32, P32, ac, uc, 0});
      if (!s4) s4 = launch_spmm(h, m->csr, k, X, MEpiRuResidual{B, R32, nullptr, J32, k, ac, uc, 0}, cfg);
      return s4;
    };
    if (!s3) s3 = in_graph ? capture_if(h, uc.cond_update, update) : update();
    if (!s3) s3 = launch_mtile(h, n, k, MOpRuDirection{P32, R32, J32, D32, ac}, vec4);
    return s3;
  };
  auto tail = [&](const MultiArgs& ac) -> int {
    int s2 = launch_mtile(h, n, k, MOpRuFlush{X, D32, nullptr, ac, u, 1});
    if (!s2) s2 = launch_spmm(h, m->csr, k, X, MEpiVerify{B, k, ac}, cfg);
    return s2;
  };
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  if (!graphs_enabled()) {
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    st = setup(a);
    for (int it = 0; !st && it < p->iter_max; it += 8) {
      for (int q = 0; q < 8 && !st; ++q) st = body(a, false);
      int act = 0;
      if (!st) {
        CELG_CUDA(cudaMemcpyAsync(&act, a.n_active, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CELG_CUDA(cudaStreamSynchronize(h->stream));
      }
      if (!act) break;
    }
    if (!st) st = tail(a);
    if (st) return st;
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  } else {
    auto record = [&](cudaGraphConditionalHandle cond) -> int {
      MultiArgs ac = a;
      ac.cond = cond;
      int s2 = setup(ac);
      if (!s2) s2 = capture_while2(h, cond, [&]() -> int { return body(ac, true); });
      if (!s2) s2 = tail(ac);
      return s2;
    };
    char kb[256];
    std::snprintf(kb, sizeof(kb), "mrhs-ru|%p|%d|%d|%p|%p|%p|%d|%.17g|%.17g|%.17g|%d|%d|%d",
                  (const void*)m, m->csr.n, k, (const void*)B, (const void*)X, (const void*)D32,
                  p->x0_mode, p->eps_abs, p->eps_rel, u.delta, p->iter_max, cfg, cfg32);
    const std::string key(kb);
    GraphEntry* ge = graph_cache_find(h, key);
    if (!ge) {
      st = graph_build(h, key, record, &ge);
      if (st) return st;
    }
    CELG_CUDA(cudaEventRecord(h->ev0, h->stream));
    CELG_CUDA(cudaGraphLaunch(ge->exec, h->stream));
    CELG_CUDA(cudaEventRecord(h->ev1, h->stream));
  }
  std::vector<double> ds(7 * kMaxRhs), rd(3 * kMaxRhs);
  std::vector<int> is(3 * kMaxRhs + 1), ri(kMaxRhs + 1);
  CELG_CUDA(cudaMemcpyAsync(ds.data(), mu->dstate, sizeof(double) * ds.size(), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaMemcpyAsync(is.data(), mu->istate, sizeof(int) * is.size(), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaMemcpyAsync(rd.data(), mu->rud, sizeof(double) * rd.size(), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaMemcpyAsync(ri.data(), mu->rui, sizeof(int) * ri.size(), cudaMemcpyDeviceToHost, h->stream));
  int err_word = 0;
  CELG_CUDA(cudaMemcpyAsync(&err_word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  if (err_word) return err_word;
  int ret = CELG_OK, iters = 0;
  for (int c = 0; c < k; ++c) {
    const double norm64 = rd[2 * kMaxRhs + c], eps = ds[5 * kMaxRhs + c];
    const int it = is[c], err = is[2 * kMaxRhs + c];
    int rs = CELG_OK;
    if (err) rs = err;
    else if (!(norm64 <= eps)) rs = CELG_ERR_NOCONV;
    if (rs && !ret) ret = rs;
    iters = std::max(iters, it);
    if (res) {
      res[c].iter_done = it;
      res[c].final_norm2 = norm64;
      res[c].bnorm = ds[4 * kMaxRhs + c];
      res[c].verified_relres = ds[6 * kMaxRhs + c];
      res[c].err = rs;
      res[c].arnoldi_steps = ri[c];
      res[c].history_len = 0;
    }
  }
  h->last_iters = iters;
  // FP32 SpMM (matrix; P gathered, V stored: 8 n k), step (R, V read, R
  // stored: 12 n k; J 4 n), direction (P, R, D read, P, D stored: 20 n k;
  // J 4 n); 4 bytes per non-zero and one per row on row patterns, else 5
  // per non-zero with the 1-byte offsets, 8 with int32 columns
  const double mat = m->csr.pid ? 4.0 * m->csr.nnz + n : (m->csr.ci8 ? 5.0 : 8.0) * m->csr.nnz;
  h->last_bytes_per_iter = mat + 4.0 * (n + 1) + 40.0 * (double)nk + 8.0 * n;
  return ret;
}

}  // namespace celg

extern "C" int celg_pcg_multirhs(celg_handle* h, celg_mat* m, int k, const double* B_d, double* X_d,
                                 const celg_params* p, celg_result* res) {
  if (!h || !m || !p || k <= 0 || k > celg::kMaxRhs || m->h != h) return CELG_ERR_ARG;
  if (m->csr.ncols != m->csr.n || p->precond != CELG_PRECOND_JACOBI) return CELG_ERR_ARG;
  if (m->csr.n > 0 && (!B_d || !X_d)) return CELG_ERR_ARG;
  if (p->x0_mode < CELG_X0_REF_ONES || p->x0_mode > CELG_X0_USER || p->iter_max < 0) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  CELG_CUDA(cudaSetDevice(h->device));
  return celg::pcg_multirhs(h, m, k, B_d, X_d, p, res);
}
