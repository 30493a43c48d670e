// tile_kernels.cuh -- streaming vector kernels over 1024-row tiles with the
// fixed-order reductions of celg_device.cuh, plus the host launch helpers
// for them and for the SpMV kernel templates.
//
// An Op supplies
//   NRED                                  number of fused reductions
//   bool prepare()                        read device scalars; false = skip
//   void load(long i, Regs& r)            all global loads of row i
//   void compute(long i, Regs& r, acc)    arithmetic, stores, reductions
//   void finish(double* tot)              lane 0 of the last CTA
// Each lane handles rows t*1024 + j + 256k (k = 0..3): loads of the four rows
// are issued before any arithmetic so that 4 x (loads per row) requests are
// in flight per thread, and the reduction order is the oracle's.
#pragma once
#include <algorithm>
#include <mutex>

#include "celg_internal.h"
#include "spmv_kernels.cuh"

namespace celg {

// An op with `static constexpr bool kAllLanes = true` has load/compute called
// for every lane of every tile, including rows past n.
template <class T, class = void>
struct all_lanes : std::false_type {};
template <class T>
struct all_lanes<T, std::void_t<decltype(T::kAllLanes)>> : std::integral_constant<bool, T::kAllLanes> {};

// An op with `static constexpr int kTilesPerPass = 2` has each CTA take two
// of its tiles (k and k + grid) per pass: the loads of both are issued before
// any arithmetic, and their reductions share the barriers of one fold.  Every
// tile is still reduced on its own, in the same order.
template <class T, class = void>
struct tiles_per_pass : std::integral_constant<int, 1> {};
template <class T>
struct tiles_per_pass<T, std::void_t<decltype(T::kTilesPerPass)>>
    : std::integral_constant<int, T::kTilesPerPass> {};

// Tile partials without a barrier per tile: each warp folds its lanes of a
// tile with the butterfly and parks the warp sum in shared memory; every
// kHeldTiles tiles (and at the end) the CTA meets once and adds the parked
// warp sums of each tile in warp order.  That is group_fold256's order, so
// the tile partials are the same bits, but the warps no longer wait for one
// another after every tile.  (Measured on the 256^3 FP32 update sweep: the
// per-tile barrier pair was about a quarter of its time.)

template <class Op>
__global__ void __launch_bounds__(kLanes) tile_kernel(long n, Op op_in, RedCtx red) {
  constexpr int NR = Op::NRED;
  constexpr bool kB = is_batched<Op>::value;
  constexpr int TP = kB ? 1 : tiles_per_pass<Op>::value;
  constexpr int NF = (NR > 0 ? NR : 1) * TP;
  constexpr int NR1 = NR > 0 ? NR : 1;
  constexpr bool kHold = !kB && NR > 0;
  __shared__ double scratch[8 * NF];
  __shared__ double held[kHold ? kHeldTiles : 1][NR1][8];
  __shared__ long held_tile[kHold ? kHeldTiles : 1];
  __shared__ int s_flag;
  [[maybe_unused]] int nheld = 0;
  // the parked warp sums of the held tiles -> their tile partials
  auto flush = [&]() {
    __syncthreads();
    for (int q = threadIdx.x; q < nheld * NR1; q += kLanes) {
      const int sl = q / NR1, r = q % NR1;
      double tot = held[sl][r][0];
#pragma unroll
      for (int w = 1; w < 8; ++w) tot = dadd(tot, held[sl][r][w]);
      red.partials[(long)r * red.ntiles + held_tile[sl]] = tot;
    }
    __threadfence();  // every writer's partials visible before the grid's ticket
    __syncthreads();
    nheld = 0;
  };
  Op op = op_in;
  if (!op.prepare()) return;
  const int j = threadIdx.x;
  const long ntiles = (n + kTile - 1) / kTile;
  const int sweep = red.sweep;
  TileInfo nxt{0, 0.0};
  if constexpr (kB) {
    if (blockIdx.x < ntiles) nxt = op.tile_info(tile_at(blockIdx.x, ntiles, sweep));
  }
  for (long k = blockIdx.x; k < ntiles; k += (long)TP * gridDim.x) {
    long t[TP];
    bool on[TP];
#pragma unroll
    for (int p = 0; p < TP; ++p) {
      const long kp = k + (long)p * gridDim.x;
      on[p] = kp < ntiles;
      t[p] = on[p] ? tile_at(kp, ntiles, sweep) : 0;
    }
    if constexpr (kB) {
      const TileInfo cur = nxt;
      if (k + gridDim.x < ntiles) nxt = op.tile_info(tile_at(k + gridDim.x, ntiles, sweep));
      if (!cur.act) continue;
      op.begin_tile(cur);
    }
    double acc[TP][NR > 0 ? NR : 1];
#pragma unroll
    for (int p = 0; p < TP; ++p)
#pragma unroll
      for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[p][r] = 0.0;
    typename Op::Regs regs[TP][4];
    if constexpr (all_lanes<Op>::value) {
      // every lane takes part (rows past n included: the op guards them), so
      // ops may exchange values between lanes with warp shuffles
#pragma unroll
      for (int p = 0; p < TP; ++p)
        if (on[p])
#pragma unroll
          for (int q = 0; q < 4; ++q) op.load(t[p] * kTile + j + (long)q * kLanes, regs[p][q]);
#pragma unroll
      for (int p = 0; p < TP; ++p)
        if (on[p])
#pragma unroll
          for (int q = 0; q < 4; ++q)
            op.compute(t[p] * kTile + j + (long)q * kLanes, regs[p][q], acc[p]);
    } else {
#pragma unroll
      for (int p = 0; p < TP; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long i = t[p] * kTile + j + (long)q * kLanes;
          if (on[p] && i < n) op.load(i, regs[p][q]);
        }
#pragma unroll
      for (int p = 0; p < TP; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const long i = t[p] * kTile + j + (long)q * kLanes;
          if (on[p] && i < n) op.compute(i, regs[p][q], acc[p]);
        }
    }
    if constexpr (kHold) {
      if (nheld + TP > kHeldTiles) flush();
#pragma unroll
      for (int p = 0; p < TP; ++p) {
        if (!on[p]) continue;
#pragma unroll
        for (int r = 0; r < NR1; ++r) {
          const double w = warp_fold(acc[p][r]);
          if ((j & 31) == 0) held[nheld][r][j >> 5] = w;
        }
        if (j == 0) held_tile[nheld] = t[p];
        ++nheld;
      }
    } else if (NR > 0) {
      double f[NF];
#pragma unroll
      for (int p = 0; p < TP; ++p)
#pragma unroll
        for (int r = 0; r < (NR > 0 ? NR : 1); ++r) f[p * (NR > 0 ? NR : 1) + r] = acc[p][r];
      group_fold256_n<NF>(f, scratch, j, 1);
      if (j == 0) {
#pragma unroll
        for (int p = 0; p < TP; ++p)
          if (on[p])
#pragma unroll
            for (int r = 0; r < (NR > 0 ? NR : 1); ++r)
              red.partials[(long)r * red.ntiles + t[p]] = f[p * (NR > 0 ? NR : 1) + r];
      }
      // batched: the systems are completed by batch_finish_kernel
    }
  }
  if constexpr (kHold) flush();
  if constexpr (kB) {
    // completed by batch_finish_kernel
  } else if constexpr (NR > 0) {
    double tot[NR > 0 ? NR : 1];
    if (grid_finish<(NR > 0 ? NR : 1)>(red, tot, scratch, &s_flag, j, 1)) op.finish(tot);
  } else if constexpr (finishes_always<Op>::value) {
    if (grid_last(red.ticket, &s_flag, j, 1)) op.finish(nullptr);
  }
}

// Allow `bytes` of dynamic shared memory for a kernel on the current device.
// The attribute belongs to the function, shared by every handle and thread
// of the process, so it is only ever raised (under a lock): a launch of
// another handle that needs less is never left above the attribute.
template <auto Kern>
int allow_dynamic_smem(int bytes) {
  static std::mutex mu;
  static int allowed[64] = {};
  int dev = 0;
  CELG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const int slot = dev >= 0 && dev < 64 ? dev : 0;
  if (bytes > allowed[slot] || dev >= 64) {
    CELG_CUDA(cudaFuncSetAttribute(Kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    allowed[slot] = bytes;
  }
  return CELG_OK;
}

// Resident CTAs per SM of a kernel at a fixed block size and dynamic shared
// memory (queried once per kernel).
template <auto Kern>
int resident_per_sm(int threads, int smem) {
  static int cached = 0;
  if (!cached) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, Kern, threads, smem) != cudaSuccess)
      per_sm = 1;
    cached = std::max(1, per_sm);
  }
  return cached;
}

// Sweep options of the next launch: consecutive sweeps walk the tiles in
// opposite orders, so each one starts on the rows whose vectors the previous
// one touched last (still in L2); CSR sweeps stream the matrix, read once
// per sweep, with the evict-first policy so that it does not push those
// vectors out.
// (Measured on the 256^3 Poisson PCG: DRAM traffic per iteration 3217 ->
// 3083 MB, time 538 -> 526 us, together with the streaming loads and stores
// of the update and direction sweeps.)
inline int next_sweep(celg_handle* h, bool csr) {
  const int s = h->sweep_rev;
  h->sweep_rev ^= 1;
  return csr ? (s | 2) : s;
}

// The grid holds as many CTAs as are resident at once (no second wave: each
// CTA walks its share of the tiles), at most blocks_per_sm per SM.
template <class Op>
int launch_tile(celg_handle* h, long n, const Op& op, int blocks_per_sm = 8) {
  const long nt = ntiles_of(n);
  RedCtx red{h->partials, h->ticket, nt};
  red.sweep = next_sweep(h, false);
  if (Op::NRED > 0) {
    int st = ensure_partials(h, nt, Op::NRED);
    if (st) return st;
    red.partials = h->partials;
  }
  const int grid =
      grid_for_tiles(h, nt, std::min(blocks_per_sm, resident_per_sm<tile_kernel<Op>>(kLanes, 0)));
  tile_kernel<Op><<<grid, kLanes, 0, h->stream>>>(n, op, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// One half of a CSR sweep split in two launches: the tiles [lo, hi)
// (inside = true; their partials are left for the other half) or all tiles
// but those (inside = false; its last CTA combines every tile's partials).
// partials: NRED x ntiles doubles shared by the two halves; partials_cap is
// the buffer's length in doubles (a launch whose epilogue needs more is
// rejected with CELG_ERR_ARG).
struct TileWindow {
  long lo = 0, hi = 0;
  bool inside = true;
  double* partials = nullptr;
  long partials_cap = 0;
};

// max_per_sm > 0 caps the resident CTAs per SM (the batched solves' tuner).
template <typename VT, typename CT, class Epi>
int launch_csr_ct(celg_handle* h, const CsrDev& A, const VT* vals, const CT* cols, int cap,
                  const VT* x, const Epi& epi, const TileWindow* win = nullptr, int max_per_sm = 0) {
  const long nt = ntiles_of(A.n);
  RedCtx red{nullptr, h->ticket, nt};
  long nvis = nt;
  if (win) {
    const long len = win->hi - win->lo;
    if (win->lo < 0 || len < 0 || win->hi > nt) return CELG_ERR_ARG;
    if (Epi::NRED > 0 && (!win->partials || win->partials_cap < (long)Epi::NRED * nt))
      return CELG_ERR_ARG;
    if (win->inside) {
      red.win_a = 0;
      red.win_shift = win->lo;
      nvis = len;
      red.finish = false;
    } else {
      red.win_a = win->lo;
      red.win_shift = len;
      nvis = nt - len;
    }
    red.nvisit = nvis;
    red.partials = win->partials;
    if (win->inside && nvis == 0) return CELG_OK;
  } else if (Epi::NRED > 0) {
    int st = ensure_partials(h, nt, Epi::NRED);
    if (st) return st;
    red.partials = h->partials;
  }
  if (A.n == 0) return CELG_OK;
  red.sweep = next_sweep(h, true);
  constexpr bool kPat = std::is_same<CT, PatIdx>::value;
  const int* tab = kPat ? A.pat : (std::is_same<CT, uint8_t>::value ? A.dict : nullptr);
  const int ntab = kPat ? A.npat * kPatLen : (std::is_same<CT, uint8_t>::value ? A.ndict : 0);
  const int smem = csr_smem_bytes(cap, (int)sizeof(VT), (int)sizeof(CT), kPat ? ntab : -1);
  auto kern = csr_tma_kernel<VT, Epi, CT>;
  if (const int st = allow_dynamic_smem<csr_tma_kernel<VT, Epi, CT>>(smem)) return st;
  int per_sm = 0;
  CELG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCsrThreads, smem));
  per_sm = std::max(1, per_sm);
  if (max_per_sm > 0) per_sm = std::min(per_sm, max_per_sm);
  const int grid = (int)std::max(1L, std::min(nvis, (long)h->sms * per_sm));
  kern<<<grid, kCsrThreads, smem, h->stream>>>(A.rp, cols, vals, A.n, cap, x, epi, red, h->err_d,
                                               tab, ntab);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// CSR sweep over the row patterns when the matrix has them (same values,
// same columns, same order: the same sums), else over the 1-byte column
// offsets, else (fallback false) nothing is launched and 1 is returned.
template <typename VT, class Epi>
int launch_csr_compact(celg_handle* h, const CsrDev& A, const VT* vals, const VT* x, const Epi& epi,
                       const TileWindow* win, int max_per_sm, bool* done) {
  *done = true;
  if (A.pid)
    return launch_csr_ct<VT, PatIdx>(h, A, vals, reinterpret_cast<const PatIdx*>(A.pid), A.cap, x,
                                     epi, win, max_per_sm);
  if (A.ci8) return launch_csr_ct<VT, uint8_t>(h, A, vals, A.ci8, A.cap_dict, x, epi, win, max_per_sm);
  *done = false;
  return CELG_OK;
}

// CSR sweep with the matrix's own column indices; the FP32 copy uses the
// row patterns or the 1-byte offset dictionary when the matrix has them.
template <typename VT, class Epi>
int launch_csr(celg_handle* h, const CsrDev& A, const VT* vals, const VT* x, const Epi& epi) {
  if constexpr (sizeof(VT) == 4) {
    bool done = false;
    const int st = launch_csr_compact<VT>(h, A, vals, x, epi, nullptr, 0, &done);
    if (done) return st;
  }
  return launch_csr_ct<VT, int>(h, A, vals, A.ci, A.cap, x, epi);
}

template <class Epi>
int launch_jad(celg_handle* h, const CsrDev& A, const JadDev& J, const double* x, const Epi& epi) {
  const long nt = ntiles_of(A.n);
  RedCtx red{nullptr, h->ticket, nt};
  if (Epi::NRED > 0) {
    int st = ensure_partials(h, nt, Epi::NRED);
    if (st) return st;
    red.partials = h->partials;
  }
  if (A.n == 0) return CELG_OK;
  red.sweep = next_sweep(h, false);
  if (J.pid && A.pat && J.mmax <= kPatLen) {
    // the columns from the row patterns (same columns in the same order)
    const int grid =
        grid_for_tiles(h, nt, std::min(8, resident_per_sm<jad_kernel<Epi, true>>(kLanes, 0)));
    jad_kernel<Epi, true><<<grid, kLanes, 0, h->stream>>>(J.begin, J.ci, J.v, J.perm, A.n, J.mmax,
                                                          x, epi, red, J.pid, A.pat,
                                                          A.npat * kPatLen);
    CELG_CUDA(cudaGetLastError());
    return CELG_OK;
  }
  const int grid = grid_for_tiles(h, nt, std::min(8, resident_per_sm<jad_kernel<Epi>>(kLanes, 0)));
  jad_kernel<Epi><<<grid, kLanes, 0, h->stream>>>(J.begin, J.ci, J.v, J.perm, A.n, J.mmax, x, epi,
                                                    red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}

// ---- simple ops ----------------------------------------------------------

// acc += a*b ; finish: *out = tot (or sqrt(tot))
struct OpDot {
  static constexpr int NRED = 1;
  struct Regs { double a, b; };
  const double* a;
  const double* b;
  double* out;
  int take_sqrt;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& r) const { r.a = __ldg(a + i); r.b = __ldg(b + i); }
  __device__ void compute(long, Regs& r, double* acc) const { acc[0] = dadd(acc[0], dmul(r.a, r.b)); }
  __device__ void finish(double* tot) const { *out = take_sqrt ? sqrt(tot[0]) : tot[0]; }
};

// r = b - (0 + r) in place, acc += r*r; finish *out = sqrt(tot)
struct OpResidNat {
  static constexpr int NRED = 1;
  struct Regs { double b, r; };
  const double* b;
  double* r;
  double* out;
  __device__ bool prepare() { return true; }
  __device__ void load(long i, Regs& g) const { g.b = __ldg(b + i); g.r = r[i]; }
  __device__ void compute(long i, Regs& g, double* acc) const {
    const double ri = __dsub_rn(g.b, dadd(0.0, g.r));
    r[i] = ri;
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ void finish(double* tot) const { *out = sqrt(tot[0]); }
};

}  // namespace celg
