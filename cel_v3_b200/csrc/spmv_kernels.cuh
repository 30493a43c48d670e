// spmv_kernels.cuh -- the SpMV kernels of libcelgpu, templated on an
// epilogue so that each solver step fuses its vector update and dot
// products into the matrix sweep.
//
// CSR (reference: src/fop/cel_fop_mv_module.f90:189-247).  Persistent CTAs
// walk 1024-row reduction tiles (tile b, b+grid, ...), each as four 256-row
// sub-tiles.  A producer warp stages every sub-tile's row pointers, column
// indices and values into shared memory with bulk copies
// (cp.async.bulk + mbarrier, kStages deep); eight consumer warps compute one
// row per thread from shared memory, gathering x through the read-only
// path.  Row sums start at 0.0 and add value*x in stored order with separate
// multiply and add roundings, exactly like the Fortran loop at :216-228.
// A sub-tile whose entries exceed the staging capacity (very long rows) is
// read straight from global memory with the same arithmetic.
//
// JAD (reference: src/fop/cel_fop_mv_module.f90:250-352).  One thread per
// permuted row, four rows per thread per 1024-row tile, jagged diagonals
// read column-major (coalesced) and accumulated in a register in diagonal
// order; the result is written through perm (y(perm(i)) = tmp(i), :325).
#pragma once
#include "celg_device.cuh"

namespace celg {

// Shared-memory layout of one pipeline stage for `cap` staged entries with
// column indices of ct_size bytes (4: int32 columns; 1: offset-dictionary
// indices) and values of vt_size bytes.
// With per_row, the column data is one pattern index per row (kSub + 16
// bytes) instead of one index per entry.
struct StageLayout {
  int ci_off, v_off, bytes;
  __host__ __device__ StageLayout(int cap, int vt_size, int ct_size = 4, bool per_row = false) {
    ci_off = (kSub + 4) * 4;                                          // 1040, 16B multiple
    v_off = ci_off + (per_row ? kSub + 16 : (((cap + 32) * ct_size + 15) & ~15));
    int end = v_off + (cap + 32) * vt_size;
    bytes = (end + 127) & ~127;
  }
};
constexpr int kDictMax = 256;  // offset-dictionary entries (uint8 indices)

// Row patterns.  When every row has at most kPatLen entries and the rows use
// at most kPatMax distinct sequences of column offsets col - row (a
// structured-grid stencil has a few dozen: interior rows, faces, edges,
// corners), each row stores one byte -- the index of its sequence in a
// pattern table of kPatLen offsets per pattern -- and the entries store no
// column data at all: 8 (FP64) or 4 (FP32) bytes per non-zero plus one per
// row, against 9 or 5 with the 1-byte offset dictionary.
constexpr int kPatLen = 8;
constexpr int kPatMax = 256;
struct PatIdx {
  uint8_t v;
};

// column of stored entry k of row `row`: int32 columns are absolute, uint8
// indices select an offset col - row from the matrix's dictionary
__device__ __forceinline__ int entry_col(int c, long, const int*) { return c; }
__device__ __forceinline__ int entry_col(uint8_t c, long row, const int* dict) {
  return (int)row + dict[c];
}
constexpr int kCsrHeader = 256;  // mbarriers, stage meta, fold scratch

// An epilogue's own vector loads belong in row(), after the row's gathers.
// Issued before the gathers (tried for the p of p.v), they cost 23 us per
// 256^3 sweep.

// Sum of a row of L entries, 0 + v0 x0 + v1 x1 + ... in stored order, with
// separate multiply and add roundings; G: values read from global memory.
template <int L, bool G, typename VT>
__device__ __forceinline__ VT pat_dot(const VT* vs, const VT (&xv)[kPatLen]) {
  VT s = VT(0);
#pragma unroll
  for (int u = 0; u < L; ++u) s = vadd(s, vmul(G ? __ldg(vs + u) : vs[u], xv[u]));
  return s;
}

// The same for a row of len entries: one branch on the length instead of a
// predicate per entry.
template <bool G, typename VT>
__device__ __forceinline__ VT pat_dot_len(int len, const VT* vs, const VT (&xv)[kPatLen]) {
  static_assert(kPatLen == 8, "lengths 1..8");
  switch (len) {
    case 7: return pat_dot<7, G>(vs, xv);
    case 6: return pat_dot<6, G>(vs, xv);
    case 5: return pat_dot<5, G>(vs, xv);
    case 4: return pat_dot<4, G>(vs, xv);
    case 8: return pat_dot<8, G>(vs, xv);
    case 3: return pat_dot<3, G>(vs, xv);
    case 2: return pat_dot<2, G>(vs, xv);
    case 1: return pat_dot<1, G>(vs, xv);
    default: return VT(0);
  }
}

// x[base + off] through the read-only path, the address formed by one
// 32 x 32 -> 64-bit multiply-add (at 256^3 this took the FP32 pattern sweep
// from 109 to 101 M warp instructions, 141 -> 139 us)
template <typename VT>
__device__ __forceinline__ VT ldg_at(const VT* base, int off) {
  if constexpr (sizeof(VT) == 8) {
    double v;
    asm("{\n\t.reg .u64 a;\n\tmad.wide.s32 a, %1, 8, %2;\n\tld.global.nc.f64 %0, [a];\n\t}"
        : "=d"(v) : "r"(off), "l"(base));
    return v;
  } else {
    float v;
    asm("{\n\t.reg .u64 a;\n\tmad.wide.s32 a, %1, 4, %2;\n\tld.global.nc.f32 %0, [a];\n\t}"
        : "=f"(v) : "r"(off), "l"(base));
    return v;
  }
}

template <int N>
struct Acc {
  double a[N > 0 ? N : 1];
};

template <typename VT, class Epi, typename CT = int>
__global__ void __launch_bounds__(kCsrThreads, sizeof(VT) == 4 ? 4 : (sizeof(CT) == 1 ? 3 : 2))
    csr_tma_kernel(const int* __restrict__ rp, const CT* __restrict__ ci,
                   const VT* __restrict__ v, int n, int cap, const VT* __restrict__ x, Epi epi,
                   RedCtx red, int* err, const int* __restrict__ dict, int ndict) {
  constexpr int NR = Epi::NRED;
  constexpr bool kB = is_batched<Epi>::value;
  constexpr bool kPat = std::is_same<CT, PatIdx>::value;
  constexpr bool kDict = std::is_same<CT, uint8_t>::value;
  // sub-tiles per consumer pass on row patterns (at 256^3: FP32 sweep 155 ->
  // 148 us, FP64 205 -> 197 us against one per pass)
  constexpr int kPR = kPat ? 2 : 1;
  // entries per 16 bytes of the narrowest per-entry array
  constexpr int kAlign = kPat ? 16 / (int)sizeof(VT) : (kDict ? 16 : 4);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  int* meta = reinterpret_cast<int*>(empty + kStages);        // a0, fallback per stage
  double* scratch = reinterpret_cast<double*>(smem + 128);    // 8 doubles
  int* s_flag = reinterpret_cast<int*>(smem + 192);
  // offset dictionary (kDict: ndict entries) or pattern table (kPat: ndict =
  // patterns x kPatLen offsets)
  int* s_dict = reinterpret_cast<int*>(smem + kCsrHeader);
  const int tab_bytes = kPat ? ((ndict * 4 + 127) & ~127) : (kDict ? kDictMax * 4 : 0);
  unsigned char* stages = smem + kCsrHeader + tab_bytes;
  const StageLayout L(cap, (int)sizeof(VT), (int)sizeof(CT), kPat);

  if (!epi.active()) return;
  const long nsub = ((long)n + kSub - 1) / kSub;
  const long nvis = red.nvisit >= 0 ? red.nvisit : ((long)n + kTile - 1) / kTile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_mbar_init();
  }
  if constexpr (kDict || kPat) {
    for (int q = threadIdx.x; q < ndict; q += blockDim.x) s_dict[q] = dict[q];
  }
  __syncthreads();

  const int sweep = red.sweep;
  if (warp == kConsumerWarps) {
    // ---------------- producer warp ----------------
    [[maybe_unused]] const uint64_t pol = (sweep & 2) ? l2_evict_first_policy() : 0;
    long k = blockIdx.x;
    int it = 0;
    int bnd = 0;  // lane q (0..4) holds rp at sub-tile boundary q of tile t
    if (k < nvis && lane <= kSubPerTile)
      bnd = __ldg(rp + min(tile_of(red, k, nvis) * kTile + (long)lane * kSub, (long)n));
    TileInfo nxt{0, 0.0};
    if constexpr (kB) {
      if (k < nvis) nxt = epi.tile_info(tile_of(red, k, nvis));
    }
    for (; k < nvis; k += gridDim.x) {
      const long t = tile_of(red, k, nvis);
      const int cur = bnd;
      const long kn = k + gridDim.x;
      if (kn < nvis && lane <= kSubPerTile)
        bnd = __ldg(rp + min(tile_of(red, kn, nvis) * kTile + (long)lane * kSub, (long)n));
      if constexpr (kB) {
        const TileInfo ti = nxt;
        if (kn < nvis) nxt = epi.tile_info(tile_of(red, kn, nvis));
        if (!ti.act) continue;
      }
      for (int q = 0; q < kSubPerTile; ++q) {
        const long s = t * kSubPerTile + q;
        if (s >= nsub) break;
        const int e0 = __shfl_sync(0xffffffffu, cur, q);
        const int e1 = __shfl_sync(0xffffffffu, cur, q + 1);
        int abort_ = 0;
        if (lane == 0) {
          const int st = it % kStages;
          if (it >= kStages &&
              !mbar_wait_bounded(&empty[st], (uint32_t)(((it / kStages) - 1) & 1), err)) {
            abort_ = 1;
          } else {
            const long row0 = s * kSub;
            const int rows = (int)min((long)kSub, (long)n - row0);
            const int a0 = e0 & ~(kAlign - 1);
            const int a1 = (e1 + kAlign - 1) & ~(kAlign - 1);
            const int cnt = a1 - a0;
            const int fb = cnt > cap ? 1 : 0;
            meta[2 * st] = a0;
            meta[2 * st + 1] = fb;
            const uint32_t rpb = (uint32_t)(((rows + 1 + 3) & ~3) * 4);
            // column data: per entry (int32 or 1-byte offsets) from a0, or
            // (row patterns) one byte per row from row0
            const CT* csrc = kPat ? ci + row0 : ci + a0;
            const uint32_t cb =
                kPat ? (uint32_t)((rows + 15) & ~15) : (uint32_t)cnt * (uint32_t)sizeof(CT);
            const bool copy = !fb && (cnt > 0 || kPat);
            const uint32_t mb = copy ? cb + (uint32_t)cnt * (uint32_t)sizeof(VT) : 0u;
            unsigned char* sb = stages + (size_t)st * L.bytes;
            mbar_arrive_expect_tx(&full[st], rpb + mb);
            if (sweep & 2) {
              bulk_g2s_hint(sb, rp + row0, rpb, &full[st], pol);
              if (copy) {
                bulk_g2s_hint(sb + L.ci_off, csrc, cb, &full[st], pol);
                if (cnt > 0)
                  bulk_g2s_hint(sb + L.v_off, v + a0, (uint32_t)cnt * (uint32_t)sizeof(VT),
                                &full[st], pol);
              }
            } else {
              bulk_g2s(sb, rp + row0, rpb, &full[st]);
              if (copy) {
                bulk_g2s(sb + L.ci_off, csrc, cb, &full[st]);
                if (cnt > 0)
                  bulk_g2s(sb + L.v_off, v + a0, (uint32_t)cnt * (uint32_t)sizeof(VT), &full[st]);
              }
            }
          }
        }
        abort_ = __shfl_sync(0xffffffffu, abort_, 0);
        if (abort_) return;
        ++it;
      }
    }
    return;
  }

  // ---------------- consumer warps (256 threads, lane j = row in sub-tile) ----
  const int j = threadIdx.x;
  int it = 0;
  Epi ep = epi;
  TileInfo nxt{0, 0.0};
  if constexpr (kB) {
    if (blockIdx.x < nvis) nxt = ep.tile_info(tile_of(red, blockIdx.x, nvis));
  }
  for (long k = blockIdx.x; k < nvis; k += gridDim.x) {
    const long t = tile_of(red, k, nvis);
    if constexpr (kB) {
      const TileInfo ti = nxt;
      if (k + gridDim.x < nvis) nxt = ep.tile_info(tile_of(red, k + gridDim.x, nvis));
      if (!ti.act) continue;
      ep.begin_tile(ti);
    }
    Acc<NR> acc;
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc.a[r] = 0.0;
    if constexpr (kPat) {
      // Row patterns: kPR sub-tiles per pass, one row of each per thread.
      // All gathers of the pass are issued before the first sum, and the
      // per-stage bookkeeping (waits, stage pointers, release) is shared by
      // kPR rows.  Rows j, j + 256, ... still reach the epilogue in order,
      // so the tile sums keep their order.
      static_assert(kSubPerTile % kPR == 0, "passes tile the tile");
      static_assert(kPatLen == 8, "two int4 per pattern");
      for (int q = 0; q < kSubPerTile; q += kPR) {
        const long s0 = t * kSubPerTile + q;
        if (s0 >= nsub) break;
        const int nr = (int)min((long)kPR, nsub - s0);
        int stg[kPR];
#pragma unroll
        for (int r = 0; r < kPR; ++r) {
          stg[r] = (it + r) % kStages;
          if (r < nr && !mbar_wait_bounded(&full[stg[r]], (uint32_t)(((it + r) / kStages) & 1), err))
            return;
        }
        VT xv[kPR][kPatLen];
        int len[kPR], vb[kPR], fbr[kPR];
        // row indices as unsigned: s0 * kSub + j < n + kPR * kSub < 2^32
        const unsigned row0 = (unsigned)s0 * (unsigned)kSub + (unsigned)j;
        // a full pass -- kPR whole sub-tiles, all staged -- runs without
        // per-row bound and fallback tests (the same sums)
        bool full_pass = nr == kPR && (s0 + kPR) * kSub <= (long)n;
#pragma unroll
        for (int r = 0; r < kPR; ++r) full_pass = full_pass && meta[2 * stg[r] + 1] == 0;
        if (full_pass) {
          const VT* vsr[kPR];
#pragma unroll
          for (int r = 0; r < kPR; ++r) {
            const unsigned char* sb = stages + (size_t)stg[r] * L.bytes;
            const int* rps = reinterpret_cast<const int*>(sb);
            const int b = rps[j];
            len[r] = rps[j + 1] - b;
            vsr[r] = reinterpret_cast<const VT*>(sb + L.v_off) + (b - meta[2 * stg[r]]);
            const int4* pq =
                reinterpret_cast<const int4*>(s_dict + (int)(sb + L.ci_off)[j] * kPatLen);
            const int4 q0 = pq[0], q1 = pq[1];
            const int po[kPatLen] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            const VT* xr = x + (row0 + (unsigned)(r * kSub));
#pragma unroll
            for (int u = 0; u < kPatLen; ++u) xv[r][u] = ldg_at(xr, po[u]);
          }
#pragma unroll
          for (int r = 0; r < kPR; ++r)
            ep.row((long)(row0 + (unsigned)(r * kSub)), pat_dot_len<false>(len[r], vsr[r], xv[r]),
                   acc.a);
        } else {
#pragma unroll
        for (int r = 0; r < kPR; ++r) {
          len[r] = 0;
          const unsigned row = row0 + (unsigned)(r * kSub);
          if (r < nr && row < (unsigned)n) {
            const unsigned char* sb = stages + (size_t)stg[r] * L.bytes;
            const int* rps = reinterpret_cast<const int*>(sb);
            const int b = rps[j];
            len[r] = rps[j + 1] - b;
            fbr[r] = meta[2 * stg[r] + 1];
            vb[r] = fbr[r] ? b : b - meta[2 * stg[r]];
            // the row's offsets from its pattern (two 16-byte shared loads;
            // the table is 16-byte aligned, kPatLen ints per pattern, and a
            // shorter pattern is padded with offset 0, so all kPatLen gathers
            // are issued unpredicated: the padding reads x(row))
            const int pv = fbr[r] ? (int)ci[row].v : (int)(sb + L.ci_off)[j];
            const int4* pq = reinterpret_cast<const int4*>(s_dict + pv * kPatLen);
            const int4 q0 = pq[0], q1 = pq[1];
            const int po[kPatLen] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            const VT* xr = x + row;
#pragma unroll
            for (int u = 0; u < kPatLen; ++u) xv[r][u] = ldg_at(xr, po[u]);
          }
        }
#pragma unroll
        for (int r = 0; r < kPR; ++r) {
          const unsigned row = row0 + (unsigned)(r * kSub);
          if (r < nr && row < (unsigned)n) {
            const VT sum =
                fbr[r] ? pat_dot_len<true>(len[r], v + vb[r], xv[r])
                       : pat_dot_len<false>(
                             len[r],
                             reinterpret_cast<const VT*>(stages + (size_t)stg[r] * L.bytes + L.v_off) + vb[r],
                             xv[r]);
            ep.row((long)row, sum, acc.a);
          }
        }
        }
        __syncwarp();
        if (lane == 0) {
#pragma unroll
          for (int r = 0; r < kPR; ++r)
            if (r < nr) mbar_arrive(&empty[stg[r]]);
        }
        it += nr;
      }
    }
    for (int q = 0; q < (kPat ? 0 : kSubPerTile); ++q) {
      const long s = t * kSubPerTile + q;
      if (s >= nsub) break;
      const int st = it % kStages;
      if (!mbar_wait_bounded(&full[st], (uint32_t)((it / kStages) & 1), err)) return;
      const unsigned char* sb = stages + (size_t)st * L.bytes;
      const int* rps = reinterpret_cast<const int*>(sb);
      const CT* cis = reinterpret_cast<const CT*>(sb + L.ci_off);
      const VT* vs = reinterpret_cast<const VT*>(sb + L.v_off);
      const int a0 = meta[2 * st];
      const int fb = meta[2 * st + 1];
      const long row = s * kSub + j;
      if (row < n) {
        const int b = rps[j], e = rps[j + 1];
        VT sum = VT(0);
        if constexpr (kPat) {
          // handled by the pass loop above
        } else if (kDict && sizeof(VT) == 4 && !fb) {
          // FP32 with 1-byte column offsets: the gathers address x from the
          // row's base (one dictionary lookup and one add per entry), and the
          // values are read from the stage when they are added (store-only
          // sweep at 256^3: 151 -> 140 us; the FP64 sweep is slower this way,
          // 251 -> 278 us, and keeps the loop below)
          const VT* xr = x + row;
          for (int k = b - a0, ke = e - a0; k < ke; k += 8) {
            VT xv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (k + u < ke) xv[u] = __ldg(xr + s_dict[cis[k + u]]);
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (k + u < ke) sum = vadd(sum, vmul(vs[k + u], xv[u]));
          }
        } else if (!fb) {
          // chunks of 8 entries: all gathers of a chunk are issued before the
          // first add, so a row of up to 8 entries costs one memory round trip;
          // the adds stay in stored order
          for (int k = b - a0, ke = e - a0; k < ke; k += 8) {
            VT xv[8], vv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              if (k + u < ke) {
                vv[u] = vs[k + u];
                xv[u] = __ldg(x + entry_col(cis[k + u], row, s_dict));
              }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (k + u < ke) sum = vadd(sum, vmul(vv[u], xv[u]));
          }
        } else {
          for (int k = b; k < e; ++k)
            sum = vadd(sum, vmul(__ldg(v + k), __ldg(x + entry_col(__ldg(ci + k), row, s_dict))));
        }
        ep.row(row, sum, acc.a);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      ++it;
    }
    if (NR > 0) {
#pragma unroll
      for (int r = 0; r < (NR > 0 ? NR : 1); ++r) {
        const double tot = group_fold256(acc.a[r], scratch, j, 1);
        if (j == 0) red.partials[(long)r * red.ntiles + t] = tot;
      }
      // batched: the systems are completed by batch_finish_kernel
    }
  }
  // (Tile partials parked per warp with one barrier per 16 tiles, as in
  // tile_kernel, made the 256^3 FP64 sweep slower here: 197 -> 206 us.)
  if constexpr (!kB && NR > 0) {
    double tot[NR > 0 ? NR : 1];
    if (red.finish && grid_finish<(NR > 0 ? NR : 1)>(red, tot, scratch, s_flag, j, 1)) ep.finish(tot);
  }
}

// PAT: the matrix has row patterns and ppid holds the pattern index of each
// permuted row (ppid[i] = pid[perm[i]]): the column of diagonal d of permuted
// row i is perm[i] + pat[ppid[i] * kPatLen + d], so the x gathers of a group
// wait for no column load (one memory round trip per group instead of two).
template <class Epi, bool PAT = false>
__global__ void __launch_bounds__(kLanes, 3)
    jad_kernel(const int* __restrict__ jb, const int* __restrict__ jci,
               const double* __restrict__ jv, const int* __restrict__ perm, int n, int mmax,
               const double* __restrict__ x, Epi epi, RedCtx red,
               const uint8_t* __restrict__ ppid = nullptr, const int* __restrict__ pat = nullptr,
               int pat_ints = 0) {
  constexpr int NR = Epi::NRED;
  __shared__ double scratch[8];
  __shared__ int s_flag;
  __shared__ int s_pat[PAT ? kPatMax * kPatLen : 1];
  if (!epi.active()) return;
  if constexpr (PAT) {
    for (int q = threadIdx.x; q < pat_ints; q += blockDim.x) s_pat[q] = pat[q];
    __syncthreads();
  }
  const int j = threadIdx.x;
  const long ntiles = ((long)n + kTile - 1) / kTile;
  for (long kt = blockIdx.x; kt < ntiles; kt += gridDim.x) {
    const long t = tile_at(kt, ntiles, red.sweep);
    Acc<NR> acc;
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc.a[r] = 0.0;
    long i[4];
    double sum[4];
    [[maybe_unused]] int prow[4];
    [[maybe_unused]] const int* po[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      i[k] = t * kTile + (long)k * kLanes + j;
      sum[k] = 0.0;
      if constexpr (PAT) {
        const bool ok = i[k] < n;
        prow[k] = ok ? __ldg(perm + i[k]) : 0;
        po[k] = s_pat + (ok ? (int)__ldg(ppid + i[k]) : 0) * kPatLen;
      }
    }
    // diagonals in groups of kJadDiag: every load of the group (values,
    // columns, then the x gathers) is issued before the group's adds, which
    // keep the diagonal order of each row
    constexpr int kJadDiag = 2;
    for (int d = 0; d < mmax; d += kJadDiag) {
      int beg[kJadDiag], len[kJadDiag];
#pragma unroll
      for (int g = 0; g < kJadDiag; ++g) {
        const bool ok = d + g < mmax;
        beg[g] = ok ? __ldg(jb + d + g) : 0;
        len[g] = ok ? __ldg(jb + d + g + 1) - beg[g] : 0;
      }
      if (i[0] >= len[0]) break;  // permuted rows are sorted by decreasing length
      int col[kJadDiag][4];
      double vv[kJadDiag][4], xv[kJadDiag][4];
#pragma unroll
      for (int g = 0; g < kJadDiag; ++g)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (i[k] < len[g]) {
            if constexpr (PAT)
              col[g][k] = prow[k] + po[k][d + g];
            else
              col[g][k] = __ldg(jci + beg[g] + i[k]);
            vv[g][k] = __ldg(jv + beg[g] + i[k]);
          }
#pragma unroll
      for (int g = 0; g < kJadDiag; ++g)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (i[k] < len[g]) xv[g][k] = __ldg(x + col[g][k]);
#pragma unroll
      for (int g = 0; g < kJadDiag; ++g)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (i[k] < len[g]) sum[k] = dadd(sum[k], dmul(vv[g][k], xv[g][k]));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (i[k] < n) {
        const long row = (long)__ldg(perm + i[k]);
        epi.row(row, sum[k], acc.a);
      }
    }
    if (NR > 0) {
#pragma unroll
      for (int r = 0; r < (NR > 0 ? NR : 1); ++r) {
        const double tot = group_fold256(acc.a[r], scratch, j, 1);
        if (j == 0) red.partials[(long)r * red.ntiles + t] = tot;
      }
    }
  }
  if (NR > 0) {
    double tot[NR > 0 ? NR : 1];
    if (grid_finish<(NR > 0 ? NR : 1)>(red, tot, scratch, &s_flag, j, 1)) epi.finish(tot);
  }
}

// ---- plain epilogues -------------------------------------------------------

// y = (accumulate ? y : 0) + row sum
template <typename VT>
struct EpiStore {
  static constexpr int NRED = 0;
  VT* y;
  int accumulate;
  __device__ bool active() const { return true; }
  __device__ void row(long r, VT s, double*) const {
    y[r] = vadd(accumulate ? y[r] : VT(0), s);
  }
  __device__ void finish(double*) const {}
};

// r = b - (0 + A x), and ||r||^2 into *out (sqrt taken in finish)
struct EpiResidual {
  static constexpr int NRED = 1;
  const double* b;
  double* r;
  double* out;
  __device__ bool active() const { return true; }
  __device__ void row(long i, double s, double* acc) const {
    const double ri = dsub_exact(b[i], s);
    r[i] = ri;
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  __device__ static double dsub_exact(double a, double s) { return __dsub_rn(a, dadd(0.0, s)); }
  __device__ void finish(double* tot) const { *out = sqrt(tot[0]); }
};

// Host helpers (spmv.cu): dynamic shared memory of csr_tma_kernel;
// pat_ints >= 0 selects the row-pattern layout with that many table entries
int csr_smem_bytes(int cap, int vt_size, int ct_size = 4, int pat_ints = -1);

}  // namespace celg
