// celg_device.cuh -- device-side building blocks shared by the libcelgpu
// kernels: bulk-copy/mbarrier wrappers (sm_90+ PTX, used here on sm_100a),
// bounded waits, and the fixed-order block-tree reduction.
//
// Reduction order (kept identical in the CPU oracle so that a GPU solve can
// be reproduced bit for bit):
//   * a vector of length n is cut into tiles of kTile = 1024 consecutive
//     elements; lane j (0..255) of the tile sums elements j, j+256, j+512,
//     j+768 from 0.0 in that order;
//   * each 32-lane warp folds its lanes with a butterfly (xor 16, 8, 4, 2, 1);
//   * the eight warp sums are added in warp order, giving the tile partial;
//   * the tile partials are reduced the same way (lane j sums partials j,
//     j+256, ... then butterfly and warp order) by the last CTA to finish.
#pragma once
#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

namespace celg {

constexpr int kTile = 1024;     // rows per reduction tile
constexpr int kLanes = 256;     // lanes per tile
constexpr int kSub = 256;       // rows per pipeline sub-tile of the CSR kernel
constexpr int kSubPerTile = kTile / kSub;
constexpr int kStages = 4;      // bulk-copy pipeline depth of the CSR kernel
constexpr int kConsumerWarps = 8;
constexpr int kHeldTiles = 16;  // tiles whose warp sums wait in shared memory before their fold
constexpr int kCsrThreads = (kConsumerWarps + 1) * 32;  // + one producer warp
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // bounded wait on an mbarrier: 2 s

constexpr int kErrTimeout = 5;   // CELG_ERR_TIMEOUT
constexpr int kErrBreakdown = 3; // CELG_ERR_BREAKDOWN

// Cross-block reduction context: per-tile partials (nred rows of ntiles) and
// a completion ticket reset by the last block.
struct RedCtx {
  double* partials;
  unsigned* ticket;
  long ntiles;
  // bit 0: walk the tiles from the last to the first; bit 1: stream the
  // matrix with the L2 evict-first policy.  Neither changes a result: every
  // tile is reduced on its own and the tile partials are combined in index
  // order.
  int sweep = 0;
  // Tile window of a CSR sweep split in two launches (the rows that read no
  // halo value, then the others): the launch visits nvisit tiles (-1: all),
  // its k-th visited tile being k, plus win_shift once k reaches win_a.
  // finish = false leaves the tile partials to the second launch, whose last
  // CTA combines all ntiles of them in index order.
  long nvisit = -1;
  long win_a = 0x3fffffffffffffffL;
  long win_shift = 0;
  bool finish = true;
};

// Tile index of the k-th tile a sweep visits.
__device__ __forceinline__ long tile_at(long k, long ntiles, int sweep) {
  return (sweep & 1) ? ntiles - 1 - k : k;
}

// Tile index of the k-th tile a windowed sweep visits (nvis tiles in all).
__device__ __forceinline__ long tile_of(const RedCtx& red, long k, long nvis) {
  const long t = tile_at(k, nvis, red.sweep);
  return t >= red.win_a ? t + red.win_shift : t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the given phase parity; give up after about kWaitLimitNs, record
// CELG_ERR_TIMEOUT in *err and return false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0 && global_ns() - t0 > limit_ns) break;
  }
  atomicExch(err, kErrTimeout);
  return false;
}

// Untiled bulk copy global -> shared, completion signalled on `bar`.
// dst, src 16-byte aligned and bytes a multiple of 16 (checked by callers).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// The same copy with an L2 cache policy (from createpolicy).
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
      "%2, [%3], %4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// L2 policy that evicts the lines it covers first (for data read once).
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// exact IEEE binary64 operations with no contraction into FMA
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

template <typename VT>
__device__ __forceinline__ VT vadd(VT a, VT b);
template <>
__device__ __forceinline__ double vadd<double>(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float vadd<float>(float a, float b) { return __fadd_rn(a, b); }
template <typename VT>
__device__ __forceinline__ VT vmul(VT a, VT b);
template <>
__device__ __forceinline__ double vmul<double>(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float vmul<float>(float a, float b) { return __fmul_rn(a, b); }

// acc + a b accumulated as dadd(acc, dmul(a, b)).  With float operands the
// product is exact in double (24 + 24 significant bits), so one fused
// multiply-add gives the same bits with one rounding instruction less.
__device__ __forceinline__ double dacc_prod(double acc, float a, float b) {
  return __fma_rn((double)a, (double)b, acc);
}
__device__ __forceinline__ double dacc_prod(double acc, double a, double b) {
  return dadd(acc, dmul(a, b));
}

__device__ __forceinline__ double warp_fold(double v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// Fold one value per lane of a 256-thread group (lane = tid 0..255) into
// thread 0.  `scratch` holds 8 doubles of shared memory.  All 256 threads of
// the group must call it; `bar_id`/named barrier restricts the sync to them.
__device__ __forceinline__ double group_fold256(double v, double* scratch, int tid, int bar_id) {
  v = warp_fold(v);
  if ((tid & 31) == 0) scratch[tid >> 5] = v;
  named_bar_sync(bar_id, kLanes);
  double tot = 0.0;
  if (tid == 0) {
    tot = scratch[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) tot = dadd(tot, scratch[w]);
  }
  named_bar_sync(bar_id, kLanes);
  return tot;
}

// group_fold256 of M values at once (each in the same order as alone), with
// two barriers in all; `scratch` holds 8 M doubles.  The results are in
// v[] of thread 0.
template <int M>
__device__ __forceinline__ void group_fold256_n(double (&v)[M], double* scratch, int tid,
                                                int bar_id) {
#pragma unroll
  for (int i = 0; i < M; ++i) v[i] = warp_fold(v[i]);
  if ((tid & 31) == 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) scratch[(tid >> 5) * M + i] = v[i];
  }
  named_bar_sync(bar_id, kLanes);
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      double tot = scratch[i];
#pragma unroll
      for (int w = 1; w < 8; ++w) tot = dadd(tot, scratch[w * M + i]);
      v[i] = tot;
    }
  }
  named_bar_sync(bar_id, kLanes);
}

// The 256-lane order computed by one warp: lane l plays the virtual lanes
// l + 32 g (g = 0..7) -- virtual lane j sums p[j], p[j+256], ... from 0.0;
// each group of 32 virtual lanes folds with the butterfly; the 8 group sums
// are added in order.  Bit-identical to group_fold256 over 256 threads, and
// lets independent reductions run in parallel warps.  Result in all lanes.
__device__ __forceinline__ double warp_reduce256(const double* p, long cnt, int lane) {
  double s[8];
#pragma unroll
  for (int g = 0; g < 8; ++g) s[g] = 0.0;
  // rounds of 4 x 256 elements: the 32 loads of a lane are issued before
  // its adds, which stay in element order within each virtual lane
  for (long base = 0; base < cnt; base += 4 * kLanes) {
    double v[4][8];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        const long k = base + (long)u * kLanes + 32 * g + lane;
        v[u][g] = k < cnt ? __ldcg(p + k) : 0.0;
      }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int g = 0; g < 8; ++g)
        if (base + (long)u * kLanes + 32 * g + lane < cnt) s[g] = dadd(s[g], v[u][g]);
  }
  double tot = 0.0;
#pragma unroll
  for (int g = 0; g < 8; ++g) {
    const double f = warp_fold(s[g]);
    tot = g == 0 ? f : dadd(tot, f);
  }
  return tot;
}

// Last-block-done completion for NRED reductions whose tile partials are in
// red.partials[r * ntiles + t].  Called by the 256 lanes of each CTA after
// all of its partials were written (by lane 0).  Returns true in lane 0 of
// the last CTA, with the totals in tot[].
template <int NRED>
__device__ __forceinline__ bool grid_finish(const RedCtx& red, double (&tot)[NRED],
                                            double* scratch, int* s_flag, int tid, int bar_id) {
  if (tid == 0) {
    __threadfence();
    unsigned tk = atomicAdd(red.ticket, 1u);
    *s_flag = (tk == gridDim.x - 1) ? 1 : 0;
  }
  named_bar_sync(bar_id, kLanes);
  if (*s_flag == 0) return false;
  __threadfence();
#pragma unroll
  for (int r = 0; r < NRED; ++r) {
    double s = 0.0;
    const double* p = red.partials + (long)r * red.ntiles;
    for (long k = tid; k < red.ntiles; k += kLanes) s = dadd(s, __ldcg(p + k));
    tot[r] = group_fold256(s, scratch, tid, bar_id);
  }
  if (tid == 0) *red.ticket = 0u;
  return tid == 0;
}

// Last-block-done completion without partials (an op with no reduction that
// still needs one thread to run after every CTA has read its inputs).
// Returns true in lane 0 of the CTA that finished last.
__device__ __forceinline__ bool grid_last(unsigned* ticket, int* s_flag, int tid, int bar_id) {
  if (tid == 0) {
    __threadfence();
    unsigned tk = atomicAdd(ticket, 1u);
    *s_flag = (tk == gridDim.x - 1) ? 1 : 0;
  }
  named_bar_sync(bar_id, kLanes);
  if (*s_flag == 0) return false;
  __threadfence();
  if (tid == 0) *ticket = 0u;
  return tid == 0;
}

// An op with NRED == 0 and `static constexpr bool kFinishAlways = true`
// gets finish(nullptr) from the last CTA.
template <class T, class = void>
struct finishes_always : std::false_type {};
template <class T>
struct finishes_always<T, std::void_t<decltype(T::kFinishAlways)>>
    : std::integral_constant<bool, T::kFinishAlways> {};

// ---- FP32 refinement: inner tolerance of an outer step ----------------------
//
// tau (inner_eps_rel) is the tightest relative tolerance an inner FP32 solve
// is asked for.  At an outer step with residual norm rn and outer tolerance
// tol, the goal g = tol / (2 rn) is the reduction still needed (with a margin
// of 2).  If one inner solve at tau reaches it (tau <= g), the step asks for
// g itself; if two do (tau^2 <= g), for sqrt(g), so that the remaining two
// steps share the reduction; otherwise for tau.  A step then never does more
// than the remaining steps need, and the last one does not end just short of
// tol, which would cost a further restart of the Krylov space.  Only a
// division and a square root are used, correctly rounded on the host and on
// the GPU alike, so every form of the refinement takes the same decisions.
__host__ __device__ inline double ir_step_tolerance(double rn, double tol, double tau) {
  if (!(tol > 0.0) || !(rn > tol) || !(tau > 0.0 && tau < 1.0) || !(rn < 1.0e308)) return tau;
  const double g = tol / (2.0 * rn);
  if (tau <= g) return g;
  if (tau * tau <= g) {
    const double r = sqrt(g);
    return r > tau ? r : tau;
  }
  return tau;
}

// ---- batched solves --------------------------------------------------------
//
// An epilogue/op with `static constexpr bool kBatched = true` runs over the
// concatenated rows of many systems (each padded to whole tiles).  It provides
//   TileInfo tile_info(long t)    the tile's system state (active flag and the
//                                 scalar the op needs), loaded by the kernels
//                                 one tile ahead so that the dependent loads
//                                 (tile -> system -> scalars) overlap the
//                                 current tile's work
//   void begin_tile(const TileInfo&)  take the tile's system scalars
//   bool sys_active(int s)        whether system s took part in the sweep
//   void finish_sys(int s, tot)   per-system scalars
//   void finish_global()          after every system's finish_sys
//   const BatchRed& bred()
// The sweep kernels only store the tile partials; batch_finish_kernel (one
// CTA per system, batched.cu) reduces each system's partials in the same
// order as a single solve and runs finish_sys, then finish_global.
struct BatchRed {
  const int* tile_sys;    // system of each tile
  const int* sys_tile0;  // first tile of each system
  const int* sys_ntiles;  // tiles of each system
  unsigned* sys_ticket;   // spare per-system counters
};

// per-tile system state of a batched op (act != 0: the tile's system runs)
struct TileInfo {
  int act;
  double s;
  double s2 = 0.0;
  double s3 = 0.0;
};

template <class T, class = void>
struct is_batched : std::false_type {};
template <class T>
struct is_batched<T, std::void_t<decltype(T::kBatched)>> : std::integral_constant<bool, T::kBatched> {};

}  // namespace celg
