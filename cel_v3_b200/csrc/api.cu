// api.cu -- the extern "C" entry points of libcelgpu.so declared in
// include/celgpu.h: handle, matrix upload and set-up, operators, solvers and
// the ELM assembly API.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "tile_kernels.cuh"

namespace celg {

int cuda_status(cudaError_t e, const char* what) {
  if (std::getenv("CELG_VERBOSE"))
    std::fprintf(stderr, "libcelgpu: %s failed: %s\n", what, cudaGetErrorString(e));
  (void)cudaGetLastError();  // clear sticky-free errors
  return CELG_ERR_CUDA;
}

// ---- matrix set-up kernels ---------------------------------------------------

// 0-based conversion, padding of the row-pointer tail and validation.
// bad[0] is set when row_ptr is not monotone or its ends are wrong, bad[1]
// when a column index is out of range.
__global__ void csr_prepare_kernel(int n, int ncols, int nnz, int base, int* rp, int* ci,
                                   int pad_rp, int* bad) {
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long i = tid; i <= n; i += stride) {
    const int v = rp[i] - base;
    rp[i] = v;
    if (v < 0 || v > nnz) atomicExch(&bad[0], 1);
  }
  for (long k = tid; k < nnz; k += stride) {
    const int c = ci[k] - base;
    ci[k] = c;
    if (c < 0 || c >= ncols) atomicExch(&bad[1], 1);
  }
  for (long i = tid; i < pad_rp; i += stride) rp[n + 1 + i] = nnz;
}

__global__ void csr_check_rows_kernel(int n, int nnz, const int* rp, int* bad) {
  const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long stride = (long)gridDim.x * blockDim.x;
  if (tid == 0 && (rp[0] != 0 || rp[n] != nnz)) atomicExch(&bad[0], 1);
  for (long i = tid; i < n; i += stride)
    if (rp[i + 1] < rp[i]) atomicExch(&bad[0], 1);
}

__global__ void row_len_kernel(int n, const int* __restrict__ rp, int* __restrict__ len_key,
                               int* __restrict__ idx, int* __restrict__ maxlen) {
  int best = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int L = rp[i + 1] - rp[i];
    len_key[i] = L;
    idx[i] = (int)i;
    best = max(best, L);
  }
  for (int off = 16; off >= 1; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(maxlen, best);
}

// key = mmax - len, so an ascending stable sort gives descending lengths with
// ties in ascending row order (the reference's dcsort order)
__global__ void jad_key_kernel(int n, int mmax, int* key, int* hist) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int L = key[i];
    atomicAdd(&hist[L], 1);
    key[i] = mmax - L;
  }
}

// pattern index of each permuted row
__global__ void jad_pid_kernel(int n, const int* __restrict__ perm, const uint8_t* __restrict__ pid,
                               uint8_t* __restrict__ ppid) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    ppid[i] = pid[perm[i]];
}

__global__ void jad_fill_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                const double* __restrict__ v, const int* __restrict__ perm,
                                const int* __restrict__ jb, int* __restrict__ jci,
                                double* __restrict__ jv) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int r = perm[i];
    const int b = rp[r], L = rp[r + 1] - b;
    for (int k = 0; k < L; ++k) {
      const long q = (long)jb[k] + i;
      jci[q] = ci[b + k];
      jv[q] = v[b + k];
    }
  }
}

static int ew_grid(celg_handle* h, long n) {
  return (int)std::max(1L, std::min((n + 255) / 256, (long)h->sms * 16));
}

// ---- column-offset dictionary of the FP32 copy --------------------------------

constexpr int kOffSlots = 1024;
constexpr int kOffEmpty = INT_MIN;

// distinct column offsets (col - row) into an open-addressed set; gives up
// (overflow) beyond kDictMax distinct offsets
__global__ void offset_set_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                  int* table, int* count, int* overflow) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      if (*(volatile int*)overflow) return;
      const int off = ci[k] - (int)i;
      unsigned hsh = ((unsigned)off * 2654435761u) & (kOffSlots - 1);
      for (int probe = 0; probe < kOffSlots; ++probe) {
        const int cur = *(volatile int*)&table[hsh];
        if (cur == off) break;
        if (cur == kOffEmpty) {
          const int prev = atomicCAS(&table[hsh], kOffEmpty, off);
          if (prev == kOffEmpty) {
            if (atomicAdd(count, 1) >= kDictMax) atomicExch(overflow, 1);
            break;
          }
          if (prev == off) break;
        }
        hsh = (hsh + 1) & (kOffSlots - 1);
      }
    }
  }
}

__global__ void offset_index_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const int* __restrict__ dict, int ndict, uint8_t* __restrict__ ci8) {
  __shared__ int s_dict[kDictMax];
  for (int q = threadIdx.x; q < ndict; q += blockDim.x) s_dict[q] = dict[q];
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int off = ci[k] - (int)i;
      int lo = 0, hi = ndict - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_dict[mid] < off) lo = mid + 1; else hi = mid;
      }
      ci8[k] = (uint8_t)lo;
    }
  }
}

// ---- row patterns (csr_tma_kernel with PatIdx) -----------------------------------

constexpr int kPatSlots = 4096;
constexpr unsigned long long kPatEmpty = 0xFFFFFFFFFFFFFFFEull;  // no key has a low byte 0xFE

// The row's 1-byte offset codes as one key: code k in byte k, 0xFF past the
// row's end (the dictionary has at most 254 entries, so no code is 0xFE or
// 0xFF).  Rows longer than kPatLen set *too_long.
__device__ __forceinline__ unsigned long long pat_row_key(const int* __restrict__ rp,
                                                          const uint8_t* __restrict__ ci8, long i,
                                                          int* too_long) {
  const int b = rp[i], len = rp[i + 1] - b;
  if (len > kPatLen) {
    *too_long = 1;
    return kPatEmpty;
  }
  unsigned long long key = ~0ull;
  for (int k = 0; k < len; ++k)
    key = (key & ~(0xFFull << (8 * k))) | ((unsigned long long)ci8[b + k] << (8 * k));
  return key;
}

// distinct row keys into an open-addressed set; gives up (flags[1]) beyond
// kPatMax keys or for a row longer than kPatLen
__global__ void pat_set_kernel(int n, const int* __restrict__ rp, const uint8_t* __restrict__ ci8,
                               unsigned long long* table, int* flags) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (*(volatile int*)&flags[1]) return;
    int too_long = 0;
    const unsigned long long key = pat_row_key(rp, ci8, i, &too_long);
    if (too_long) {
      atomicExch(&flags[1], 1);
      return;
    }
    unsigned slot = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 52) & (kPatSlots - 1);
    for (int probe = 0; probe < kPatSlots; ++probe) {
      const unsigned long long cur = *(volatile unsigned long long*)&table[slot];
      if (cur == key) break;
      if (cur == kPatEmpty) {
        const unsigned long long prev = atomicCAS(&table[slot], kPatEmpty, key);
        if (prev == kPatEmpty) {
          if (atomicAdd(&flags[0], 1) >= kPatMax) atomicExch(&flags[1], 1);
          break;
        }
        if (prev == key) break;
      }
      slot = (slot + 1) & (kPatSlots - 1);
    }
  }
}

// each row's pattern index: the position of its key among the sorted keys
__global__ void pat_index_kernel(int n, const int* __restrict__ rp, const uint8_t* __restrict__ ci8,
                                 const unsigned long long* __restrict__ keys, int nkeys,
                                 uint8_t* __restrict__ pid) {
  __shared__ unsigned long long s_keys[kPatMax];
  for (int q = threadIdx.x; q < nkeys; q += blockDim.x) s_keys[q] = keys[q];
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    int too_long = 0;
    const unsigned long long key = pat_row_key(rp, ci8, i, &too_long);
    int lo = 0, hi = nkeys - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (s_keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    pid[i] = (uint8_t)lo;
  }
}

// Row patterns from the 1-byte offsets (left unset when a row is longer than
// kPatLen, the dictionary has more than 254 entries or the rows use more
// than kPatMax distinct offset sequences).
static int build_row_patterns(celg_handle* h, CsrDev& A) {
  cudaFree(A.pid);
  cudaFree(A.pat);
  A.pid = nullptr;
  A.pat = nullptr;
  A.npat = 0;
  if (!A.ci8 || A.ndict > 254 || A.n == 0) return CELG_OK;
  unsigned long long* table = nullptr;
  CELG_CUDA(cudaMalloc(&table, sizeof(unsigned long long) * kPatSlots + 2 * sizeof(int)));
  int* flags = reinterpret_cast<int*>(table + kPatSlots);
  std::vector<unsigned long long> init(kPatSlots, kPatEmpty);
  cudaError_t e = cudaMemcpyAsync(table, init.data(), sizeof(unsigned long long) * kPatSlots,
                                  cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 2 * sizeof(int), h->stream);
  if (e == cudaSuccess) {
    pat_set_kernel<<<ew_grid(h, A.n), 256, 0, h->stream>>>(A.n, A.rp, A.ci8, table, flags);
    e = cudaGetLastError();
  }
  std::vector<unsigned long long> out(kPatSlots);
  int fl[2] = {0, 0};
  std::vector<int> dict(A.ndict);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out.data(), table, sizeof(unsigned long long) * kPatSlots,
                        cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(fl, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dict.data(), A.dict, sizeof(int) * A.ndict, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess || fl[1] || fl[0] > kPatMax) {
    cudaFree(table);
    return e != cudaSuccess ? cuda_status(e, "row patterns") : CELG_OK;
  }
  std::vector<unsigned long long> keys;
  for (unsigned long long k : out)
    if (k != kPatEmpty) keys.push_back(k);
  std::sort(keys.begin(), keys.end());
  std::vector<int> tab(keys.size() * kPatLen, 0);
  for (size_t p = 0; p < keys.size(); ++p)
    for (int k = 0; k < kPatLen; ++k) {
      const int code = (int)((keys[p] >> (8 * k)) & 0xFF);
      tab[p * kPatLen + k] = code == 0xFF ? 0 : dict[code];
    }
  // the sorted keys travel in the table buffer
  e = cudaMemcpyAsync(table, keys.data(), sizeof(unsigned long long) * keys.size(),
                      cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMalloc(&A.pid, (size_t)A.n + 16);
  if (e == cudaSuccess) e = cudaMemsetAsync(A.pid + A.n, 0, 16, h->stream);
  if (e == cudaSuccess) e = cudaMalloc(&A.pat, sizeof(int) * tab.size());
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(A.pat, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice,
                        h->stream);
  if (e == cudaSuccess) {
    pat_index_kernel<<<ew_grid(h, A.n), 256, 0, h->stream>>>(A.n, A.rp, A.ci8, table,
                                                             (int)keys.size(), A.pid);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(table);
  if (e != cudaSuccess) {
    cudaFree(A.pid);
    cudaFree(A.pat);
    A.pid = nullptr;
    A.pat = nullptr;
    return cuda_status(e, "row patterns");
  }
  A.npat = (int)keys.size();
  return CELG_OK;
}

// Build ci8/dict (1-byte column offsets col - row); leaves them unset when the matrix has
// more than kDictMax distinct offsets.
int build_offset_dict_csr(celg_handle* h, CsrDev& A) {
  cudaFree(A.pid);
  cudaFree(A.pat);
  A.pid = nullptr;
  A.pat = nullptr;
  A.npat = 0;
  cudaFree(A.ci8);
  cudaFree(A.dict);
  A.ci8 = nullptr;
  A.dict = nullptr;
  A.ndict = 0;
  if (A.n == 0 || A.nnz == 0) return CELG_OK;
  int* table = nullptr;
  CELG_CUDA(cudaMalloc(&table, sizeof(int) * (kOffSlots + 2)));
  std::vector<int> init(kOffSlots + 2, kOffEmpty);
  init[kOffSlots] = 0;
  init[kOffSlots + 1] = 0;
  CELG_CUDA(cudaMemcpyAsync(table, init.data(), sizeof(int) * init.size(), cudaMemcpyHostToDevice, h->stream));
  offset_set_kernel<<<ew_grid(h, A.n), 256, 0, h->stream>>>(A.n, A.rp, A.ci, table, table + kOffSlots,
                                                           table + kOffSlots + 1);
  std::vector<int> out(kOffSlots + 2);
  cudaError_t e = cudaMemcpyAsync(out.data(), table, sizeof(int) * out.size(), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(table);
  if (e != cudaSuccess) return cuda_status(e, "offset dictionary");
  if (out[kOffSlots + 1] || out[kOffSlots] > kDictMax) return CELG_OK;  // too many offsets
  std::vector<int> dict;
  for (int q = 0; q < kOffSlots; ++q)
    if (out[q] != kOffEmpty) dict.push_back(out[q]);
  std::sort(dict.begin(), dict.end());
  // on any failure the matrix keeps its int32 columns only
  e = cudaMalloc(&A.dict, sizeof(int) * dict.size());
  if (e == cudaSuccess) e = cudaMalloc(&A.ci8, (size_t)A.nnz + 32);
  if (e == cudaSuccess) e = cudaMemsetAsync(A.ci8 + A.nnz, 0, 32, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(A.dict, dict.data(), sizeof(int) * dict.size(), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    offset_index_kernel<<<ew_grid(h, A.n), 256, 0, h->stream>>>(A.n, A.rp, A.ci, A.dict,
                                                               (int)dict.size(), A.ci8);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaFree(A.ci8);
    cudaFree(A.dict);
    A.ci8 = nullptr;
    A.dict = nullptr;
    return cuda_status(e, "offset dictionary");
  }
  A.ndict = (int)dict.size();
  A.cap_dict = (A.cap + 24 + 15) & ~15;  // 16-entry aligned spans are at most 24 entries wider
  return build_row_patterns(h, A);
}

int ensure_offset_dict(celg_handle* h, celg_mat* m) {
  if (m->csr.ci8 || m->dict_tried) return CELG_OK;
  m->dict_tried = true;
  return build_offset_dict_csr(h, m->csr);
}

void free_mat_arrays(celg_mat* m) {
  cudaFree(m->csr.rp);
  cudaFree(m->csr.ci);
  cudaFree(m->csr.v);
  cudaFree(m->csr.v32);
  cudaFree(m->csr.ci8);
  cudaFree(m->csr.dict);
  cudaFree(m->csr.pid);
  cudaFree(m->csr.pat);
  cudaFree(m->jad.begin);
  cudaFree(m->jad.ci);
  cudaFree(m->jad.v);
  cudaFree(m->jad.perm);
  cudaFree(m->jad.pid);
  cudaFree(m->diag);
  cudaFree(m->jacobi);
  cudaFree(m->jacobi32);
  cudaFree(m->scale);
  cudaFree(m->bjinv);
}

// Allocate the padded CSR arrays; the caller fills rp[0..n], ci, v.  The
// SpMV's bulk copies round a sub-tile's entry range out to 16-byte units of
// the narrowest column array: up to 3 entries past nnz with int32 columns,
// up to 15 with the 1-byte offsets, so ci and v carry 32 zeroed entries.
constexpr int kCsrPad = 32;
int alloc_csr(celg_mat* m, int n, int nnz, int ncols) {
  m->csr.n = n;
  m->csr.nnz = nnz;
  m->csr.ncols = ncols;
  CELG_CUDA(cudaMalloc(&m->csr.rp, sizeof(int) * ((size_t)n + 1 + 8)));
  CELG_CUDA(cudaMalloc(&m->csr.ci, sizeof(int) * ((size_t)nnz + kCsrPad)));
  CELG_CUDA(cudaMalloc(&m->csr.v, sizeof(double) * ((size_t)nnz + kCsrPad)));
  CELG_CUDA(cudaMemsetAsync(m->csr.ci + nnz, 0, sizeof(int) * kCsrPad, m->h->stream));
  CELG_CUDA(cudaMemsetAsync(m->csr.v + nnz, 0, sizeof(double) * kCsrPad, m->h->stream));
  return CELG_OK;
}

int finish_csr(celg_handle* h, celg_mat* m, int base) {
  const int n = m->csr.n, nnz = m->csr.nnz;
  int* bad = h->err_d + 2;
  CELG_CUDA(cudaMemsetAsync(bad, 0, 2 * sizeof(int), h->stream));
  csr_prepare_kernel<<<ew_grid(h, std::max(n + 1, nnz)), 256, 0, h->stream>>>(
      n, m->csr.ncols, nnz, base, m->csr.rp, m->csr.ci, 8, bad);
  CELG_CUDA(cudaGetLastError());
  csr_check_rows_kernel<<<ew_grid(h, n + 1), 256, 0, h->stream>>>(n, nnz, m->csr.rp, bad);
  CELG_CUDA(cudaGetLastError());
  int hb[2] = {0, 0};
  CELG_CUDA(cudaMemcpyAsync(hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  if (hb[0] || hb[1]) return CELG_ERR_ARG;
  return csr_compute_cap(h, m->csr);
}

static int build_jad(celg_mat* m) {
  celg_handle* h = m->h;
  const int n = m->csr.n, nnz = m->csr.nnz;
  JadDev& J = m->jad;
  cudaFree(J.begin);
  cudaFree(J.ci);
  cudaFree(J.v);
  cudaFree(J.perm);
  cudaFree(J.pid);
  J = JadDev();
  int *key = nullptr, *key2 = nullptr, *idx = nullptr, *hist = nullptr;
  void* tmp = nullptr;
  int st = CELG_OK;
  auto fail = [&](cudaError_t e, const char* w) {
    st = cuda_status(e, w);
  };
  int* maxlen_d = h->err_d + 4;
  int mmax = 0;
  cudaError_t e;
  do {
    if ((e = cudaMalloc(&key, sizeof(int) * std::max(1, n))) != cudaSuccess) { fail(e, "jad"); break; }
    if ((e = cudaMalloc(&key2, sizeof(int) * std::max(1, n))) != cudaSuccess) { fail(e, "jad"); break; }
    if ((e = cudaMalloc(&idx, sizeof(int) * std::max(1, n))) != cudaSuccess) { fail(e, "jad"); break; }
    if ((e = cudaMalloc(&J.perm, sizeof(int) * std::max(1, n))) != cudaSuccess) { fail(e, "jad"); break; }
    cudaMemsetAsync(maxlen_d, 0, sizeof(int), h->stream);
    if (n > 0) row_len_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, m->csr.rp, key, idx, maxlen_d);
    cudaMemcpyAsync(&mmax, maxlen_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) { fail(e, "jad lengths"); break; }
    if ((e = cudaMalloc(&hist, sizeof(int) * (size_t)(mmax + 1))) != cudaSuccess) { fail(e, "jad"); break; }
    cudaMemsetAsync(hist, 0, sizeof(int) * (size_t)(mmax + 1), h->stream);
    if (n > 0) jad_key_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, mmax, key, hist);
    int bits = 1;
    while ((1 << bits) <= mmax) ++bits;
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, idx, J.perm, n, 0, bits,
                                    h->stream);
    if ((e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16))) != cudaSuccess) { fail(e, "jad"); break; }
    if (n > 0 && (e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, idx, J.perm, n, 0,
                                                      bits, h->stream)) != cudaSuccess) {
      fail(e, "radix sort");
      break;
    }
    std::vector<int> hh((size_t)mmax + 1), jb((size_t)mmax + 1);
    cudaMemcpyAsync(hh.data(), hist, sizeof(int) * (size_t)(mmax + 1), cudaMemcpyDeviceToHost,
                    h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) { fail(e, "jad hist"); break; }
    // rows with length > k, k = 0..mmax-1
    int above = n;
    jb[0] = 0;
    for (int k = 0; k < mmax; ++k) {
      above -= hh[(size_t)k];  // remove rows of length k
      jb[(size_t)k + 1] = jb[(size_t)k] + above;
    }
    if ((e = cudaMalloc(&J.begin, sizeof(int) * (size_t)(mmax + 1))) != cudaSuccess) { fail(e, "jad"); break; }
    if ((e = cudaMalloc(&J.ci, sizeof(int) * ((size_t)nnz + 8))) != cudaSuccess) { fail(e, "jad"); break; }
    if ((e = cudaMalloc(&J.v, sizeof(double) * ((size_t)nnz + 8))) != cudaSuccess) { fail(e, "jad"); break; }
    cudaMemcpyAsync(J.begin, jb.data(), sizeof(int) * (size_t)(mmax + 1), cudaMemcpyHostToDevice,
                    h->stream);
    if (n > 0)
      jad_fill_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, m->csr.rp, m->csr.ci, m->csr.v, J.perm,
                                                          J.begin, J.ci, J.v);
    // the pattern index of each permuted row, when the matrix has row patterns
    if (m->csr.pid && n > 0) {
      if ((e = cudaMalloc(&J.pid, (size_t)n + 16)) != cudaSuccess) { fail(e, "jad"); break; }
      jad_pid_kernel<<<ew_grid(h, n), 256, 0, h->stream>>>(n, J.perm, m->csr.pid, J.pid);
    }
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) { fail(e, "jad fill"); break; }
    J.mmax = mmax;
  } while (0);
  cudaFree(key);
  cudaFree(key2);
  cudaFree(idx);
  cudaFree(hist);
  cudaFree(tmp);
  return st;
}

}  // namespace celg

using namespace celg;

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------

extern "C" void celg_params_default(celg_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->x0_mode = CELG_X0_ZERO;
  p->eps_abs = 0.0;
  p->eps_rel = 1e-8;
  p->iter_max = 1000;
  p->fmt = CELG_FMT_CSR;
  p->precision = CELG_PREC_FP64;
  p->literal_ref_bugs = 0;
  p->restart = 30;
  p->inner_eps_rel = 1e-4;
  p->inner_iter_max = 1000;
  p->outer_max = 20;
  p->precond = CELG_PRECOND_JACOBI;
}

extern "C" const char* celg_status_string(int s) {
  switch (s) {
    case CELG_OK: return "ok";
    case CELG_ERR_ARG: return "invalid argument";
    case CELG_ERR_CUDA: return "CUDA error";
    case CELG_ERR_BREAKDOWN: return "breakdown (non-finite step length)";
    case CELG_ERR_NOCONV: return "iteration limit reached";
    case CELG_ERR_TIMEOUT: return "device wait timed out";
    case CELG_ERR_STATE: return "call out of order";
    case CELG_ERR_COMM: return "an exchange between ranks failed";
    default: return "unknown status";
  }
}

extern "C" int celg_create(celg_handle** out, int device, void* stream) {
  if (!out) return CELG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  CELG_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(device));
  celg_handle* h = new celg_handle();
  h->device = device;
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete h;
      return CELG_ERR_CUDA;
    }
    h->own_stream = true;
  }
  if (cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    celg_destroy(h);
    return CELG_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc(&h->ticket, 64) != cudaSuccess || cudaMalloc(&h->err_d, 64) != cudaSuccess ||
      cudaMalloc(&h->scal_d, 64 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->scal_h, 64 * sizeof(double)) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    celg_destroy(h);
    return CELG_ERR_CUDA;
  }
  cudaMemset(h->ticket, 0, 64);
  cudaMemset(h->err_d, 0, 64);
  cudaDeviceSynchronize();
  *out = h;
  return CELG_OK;
}

extern "C" int celg_elm_destroy(celg_handle* h);

extern "C" int celg_destroy(celg_handle* h) {
  if (!h) return CELG_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->elm) celg_elm_destroy(h);
  batch_free(h->batch);
  h->batch = nullptr;
  multi_free(h->multi);
  h->multi = nullptr;
  graph_cache_clear(h);
  cudaFree(h->partials);
  cudaFree(h->sb);
  cudaFree(h->sx);
  cudaFree(h->f32);
  cudaFree(h->ir_d);
  cudaFree(h->ticket);
  cudaFree(h->err_d);
  cudaFree(h->scal_d);
  cudaFreeHost(h->scal_h);
  cudaFree(h->wr);
  cudaFree(h->wp);
  cudaFree(h->wv);
  cudaFree(h->wq);
  cudaFree(h->wz);
  cudaFree(h->state_d);
  cudaFreeHost(h->state_h);
  cudaFree(h->ru_state_d);
  cudaFreeHost(h->ru_state_h);
  cudaFree(h->hist_d);
  cudaFree(h->gm_work);
  cudaFree(h->gm_state_d);
  cudaFreeHost(h->gm_state_h);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
  delete h;
  return CELG_OK;
}

extern "C" int celg_set_stream(celg_handle* h, void* stream) {
  if (!h) return CELG_ERR_ARG;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->own_stream = false;
  h->stream = (cudaStream_t)stream;
  if (!stream) {
    CELG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return CELG_OK;
}

extern "C" int celg_sm_count(celg_handle* h, int* sms) {
  if (!h || !sms) return CELG_ERR_ARG;
  *sms = h->sms;
  return CELG_OK;
}

// ---------------------------------------------------------------------------
// matrix
// ---------------------------------------------------------------------------

static int mat_upload(celg_handle* h, int n, int ncols, int nnz, const int* row_ptr,
                      const int* cols, const double* vals, int index_base, celg_mat** out) {
  if (!h || !out || n < 0 || ncols < n || nnz < 0 || !row_ptr || (nnz > 0 && (!cols || !vals)) ||
      (index_base != 0 && index_base != 1))
    return CELG_ERR_ARG;
  *out = nullptr;
  CELG_CUDA(cudaSetDevice(h->device));
  celg_mat* m = new celg_mat();
  m->h = h;
  int st = alloc_csr(m, n, nnz, ncols);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(m->csr.rp, row_ptr, sizeof(int) * ((size_t)n + 1),
                                    cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->csr.ci, cols, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->csr.v, vals, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) st = cuda_status(e, "matrix upload");
  }
  if (!st) st = finish_csr(h, m, index_base);
  if (st) {
    cudaStreamSynchronize(h->stream);
    free_mat_arrays(m);
    delete m;
    return st;
  }
  *out = m;
  return CELG_OK;
}

extern "C" int celg_mat_from_csr(celg_handle* h, int n, int nnz, const int* row_ptr,
                                 const int* cols, const double* vals, int index_base,
                                 celg_mat** out) {
  return mat_upload(h, n, n, nnz, row_ptr, cols, vals, index_base, out);
}

extern "C" int celg_mat_from_csr_ext(celg_handle* h, int n, int ncols, int nnz, const int* row_ptr,
                                     const int* cols, const double* vals, int index_base,
                                     celg_mat** out) {
  return mat_upload(h, n, ncols, nnz, row_ptr, cols, vals, index_base, out);
}

extern "C" int celg_mat_from_csr_device(celg_handle* h, int n, int nnz, const int* row_ptr_d,
                                        const int* cols_d, const double* vals_d, celg_mat** out) {
  if (!h || !out || n < 0 || nnz < 0 || !row_ptr_d || (nnz > 0 && (!cols_d || !vals_d)))
    return CELG_ERR_ARG;
  *out = nullptr;
  CELG_CUDA(cudaSetDevice(h->device));
  celg_mat* m = new celg_mat();
  m->h = h;
  int st = alloc_csr(m, n, nnz, n);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(m->csr.rp, row_ptr_d, sizeof(int) * ((size_t)n + 1),
                                    cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->csr.ci, cols_d, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToDevice,
                          h->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->csr.v, vals_d, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToDevice,
                          h->stream);
    if (e != cudaSuccess) st = cuda_status(e, "matrix copy");
  }
  if (!st) st = finish_csr(h, m, 0);
  if (st) {
    cudaStreamSynchronize(h->stream);
    free_mat_arrays(m);
    delete m;
    return st;
  }
  *out = m;
  return CELG_OK;
}

extern "C" int celg_mat_destroy(celg_mat* m) {
  if (!m) return CELG_OK;
  celg_handle* h = m->h;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  // cached solve graphs (and a cached batch) may reference this matrix
  graph_cache_drop_matrix(h, m);
  multi_forget_matrix(h->multi, m);
  if (h->batch) {
    graph_cache_clear(h);
    batch_free(h->batch);
    h->batch = nullptr;
  }
  free_mat_arrays(m);
  delete m;
  return CELG_OK;
}

extern "C" int celg_mat_info(const celg_mat* m, int* n, int* nnz, int* jad_mmax) {
  if (!m) return CELG_ERR_ARG;
  if (n) *n = m->csr.n;
  if (nnz) *nnz = m->csr.nnz;
  if (jad_mmax) *jad_mmax = m->jad.mmax;
  return CELG_OK;
}

extern "C" int celg_mat_column_form(const celg_mat* m, int* form) {
  if (!m || !form) return CELG_ERR_ARG;
  *form = m->csr.pid ? CELG_COLS_PATTERN : (m->csr.ci8 ? CELG_COLS_OFFSET8 : CELG_COLS_INT32);
  return CELG_OK;
}

extern "C" int celg_mat_to_jad(celg_mat* m, int* perm_out) {
  if (!m || m->csr.ncols != m->csr.n) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(m->h->device));
  // the row patterns first, so that the JAD sweep can take its columns from them
  int st = ensure_offset_dict(m->h, m);
  if (!st) st = build_jad(m);
  if (st) return st;
  if (perm_out && m->csr.n > 0)
    CELG_CUDA(cudaMemcpy(perm_out, m->jad.perm, sizeof(int) * (size_t)m->csr.n, cudaMemcpyDeviceToHost));
  return CELG_OK;
}

extern "C" int celg_mat_get_jad(const celg_mat* m, int* perm, int* begin, int* cols, double* vals) {
  if (!m || m->jad.mmax < 0) return CELG_ERR_STATE;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  const size_t n = (size_t)m->csr.n, nnz = (size_t)m->csr.nnz;
  if (perm && n) CELG_CUDA(cudaMemcpy(perm, m->jad.perm, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (begin) CELG_CUDA(cudaMemcpy(begin, m->jad.begin, sizeof(int) * ((size_t)m->jad.mmax + 1), cudaMemcpyDeviceToHost));
  if (cols && nnz) CELG_CUDA(cudaMemcpy(cols, m->jad.ci, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
  if (vals && nnz) CELG_CUDA(cudaMemcpy(vals, m->jad.v, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
  return CELG_OK;
}

extern "C" int celg_mat_jacobi(celg_mat* m) {
  if (!m) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(m->h->device));
  int st = launch_jacobi_setup(m->h, m);
  if (st) return st;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  return CELG_OK;
}

extern "C" int celg_mat_get_jacobi(const celg_mat* m, double* jacobi_host) {
  if (!m || !jacobi_host) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  if (m->csr.n)
    CELG_CUDA(cudaMemcpy(jacobi_host, m->jacobi, sizeof(double) * (size_t)m->csr.n, cudaMemcpyDeviceToHost));
  return CELG_OK;
}

extern "C" int celg_mat_scale_diagonal(celg_mat* m) {
  if (!m || m->csr.ncols != m->csr.n) return CELG_ERR_ARG;
  if (m->scaled) return CELG_OK;
  CELG_CUDA(cudaSetDevice(m->h->device));
  m->scaled = false;
  int st = launch_jacobi_setup(m->h, m);  // unscaled diagonal
  if (!st) st = launch_row_scale(m->h, m);
  if (st) return st;
  m->scaled = true;
  st = launch_jacobi_setup(m->h, m);  // jacobi = sqrt|d| / d
  if (st) return st;
  if (m->jad.mmax >= 0) st = build_jad(m);
  if (!st && m->csr.v32) st = launch_to_f32(m->h, m->csr.nnz, m->csr.v, m->csr.v32);
  if (st) return st;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  return CELG_OK;
}

extern "C" int celg_mat_make_fp32(celg_mat* m) {
  if (!m || m->csr.ncols != m->csr.n) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(m->h->device));
  if (!m->csr.v32) {
    CELG_CUDA(cudaMalloc(&m->csr.v32, sizeof(float) * ((size_t)m->csr.nnz + 32)));
    CELG_CUDA(cudaMemsetAsync(m->csr.v32 + m->csr.nnz, 0, sizeof(float) * 32, m->h->stream));
  }
  int st = launch_to_f32(m->h, m->csr.nnz, m->csr.v, m->csr.v32);
  if (!st) st = ensure_offset_dict(m->h, m);
  if (!st && m->jacobi) {
    if (!m->jacobi32) CELG_CUDA(cudaMalloc(&m->jacobi32, sizeof(float) * std::max(1, m->csr.n)));
    st = launch_to_f32(m->h, m->csr.n, m->jacobi, m->jacobi32);
  }
  if (st) return st;
  CELG_CUDA(cudaStreamSynchronize(m->h->stream));
  return CELG_OK;
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------

extern "C" int celg_spmv(celg_handle* h, const celg_mat* m, int fmt, const double* x_d, double* y_d,
                         int accumulate) {
  if (!h || !m || (m->csr.n > 0 && (!x_d || !y_d))) return CELG_ERR_ARG;
  if (fmt == CELG_FMT_JAD) {
    if (accumulate) return CELG_ERR_ARG;  // the reference's JAD kernel overwrites y
    return launch_spmv_jad(h, m->csr, m->jad, x_d, y_d);
  }
  if (fmt != CELG_FMT_CSR) return CELG_ERR_ARG;
  return launch_spmv_csr(h, m->csr, x_d, y_d, accumulate);
}

extern "C" int celg_spmv_f32(celg_handle* h, const celg_mat* m, const float* x_d, float* y_d,
                             int accumulate) {
  if (!h || !m || (m->csr.n > 0 && (!x_d || !y_d))) return CELG_ERR_ARG;
  return launch_spmv_csr_f32(h, m->csr, x_d, y_d, accumulate);
}

static int blas_scalar(celg_handle* h, long n, const double* a, const double* b, double* out,
                       int take_sqrt) {
  if (!h || !out || n < 0 || (n > 0 && (!a || !b))) return CELG_ERR_ARG;
  int st = launch_dot(h, n, a, b, h->scal_d, take_sqrt);
  if (st) return st;
  if (n == 0) CELG_CUDA(cudaMemsetAsync(h->scal_d, 0, sizeof(double), h->stream));
  CELG_CUDA(cudaMemcpyAsync(h->scal_h, h->scal_d, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  *out = h->scal_h[0];
  return CELG_OK;
}

extern "C" int celg_dot(celg_handle* h, int n, const double* a_d, const double* b_d, double* out) {
  return blas_scalar(h, n, a_d, b_d, out, 0);
}

extern "C" int celg_norm2(celg_handle* h, int n, const double* a_d, double* out) {
  return blas_scalar(h, n, a_d, a_d, out, 1);
}

extern "C" int celg_axpy(celg_handle* h, int n, double alpha, const double* x_d, double* y_d) {
  if (!h || n < 0) return CELG_ERR_ARG;
  return launch_axpy(h, n, alpha, x_d, y_d);
}

extern "C" int celg_xpby(celg_handle* h, int n, const double* x_d, double beta, double* y_d) {
  if (!h || n < 0) return CELG_ERR_ARG;
  return launch_xpby(h, n, x_d, beta, y_d);
}

extern "C" int celg_jacobi_apply(celg_handle* h, const celg_mat* m, const double* r_d, double* z_d) {
  if (!h || !m) return CELG_ERR_ARG;
  if (!m->jacobi) return CELG_ERR_STATE;
  return launch_mul(h, m->csr.n, r_d, m->jacobi, z_d);
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------

static int check_solve_args(celg_handle* h, celg_mat* m, const double* b, double* x,
                            const celg_params* p) {
  if (!h || !m || !p || (m->csr.n > 0 && (!b || !x))) return CELG_ERR_ARG;
  if (p->fmt != CELG_FMT_CSR && p->fmt != CELG_FMT_JAD) return CELG_ERR_ARG;
  if (p->x0_mode < CELG_X0_REF_ONES || p->x0_mode > CELG_X0_USER) return CELG_ERR_ARG;
  if (p->precond != CELG_PRECOND_JACOBI && p->precond != CELG_PRECOND_BLOCK_JACOBI) return CELG_ERR_ARG;
  if (m->h != h) return CELG_ERR_ARG;
  if (m->csr.ncols != m->csr.n) return CELG_ERR_ARG;  // row blocks: celg_dist_* only
  return CELG_OK;
}

extern "C" int celg_pcg_jacobi(celg_handle* h, celg_mat* m, const double* b_d, double* x_d,
                               const celg_params* p, celg_result* res) {
  int st = check_solve_args(h, m, b_d, x_d, p);
  if (st) return st;
  CELG_CUDA(cudaSetDevice(h->device));
  if (p->precision != CELG_PREC_FP64 && p->precond != CELG_PRECOND_JACOBI) return CELG_ERR_ARG;
  if (p->precision == CELG_PREC_FP32_IR) return ir_solve(h, m, b_d, x_d, p, res);
  if (p->precision == CELG_PREC_FP32_RU) return ru_solve(h, m, b_d, x_d, p, res);
  return pcg_solve(h, m, b_d, x_d, p, res);
}

extern "C" int celg_cg(celg_handle* h, celg_mat* m, const double* b_d, double* x_d,
                       const celg_params* p, celg_result* res) {
  int st = check_solve_args(h, m, b_d, x_d, p);
  if (st) return st;
  if (p->precond != CELG_PRECOND_JACOBI) return CELG_ERR_ARG;  // no preconditioner in CG
  CELG_CUDA(cudaSetDevice(h->device));
  return cg_solve(h, m, b_d, x_d, p, res);
}

extern "C" int celg_gmres_jacobi(celg_handle* h, celg_mat* m, const double* b_d, double* x_d,
                                 const celg_params* p, celg_result* res) {
  int st = check_solve_args(h, m, b_d, x_d, p);
  if (st) return st;
  if (p->precond != CELG_PRECOND_JACOBI) return CELG_ERR_ARG;  // point Jacobi only
  CELG_CUDA(cudaSetDevice(h->device));
  return gmres_solve(h, m, b_d, x_d, p, res);
}

extern "C" int celg_solve_host(celg_handle* h, celg_mat* m, int solver, const double* b_host,
                               double* x_host, const celg_params* p, celg_result* res) {
  int st = check_solve_args(h, m, b_host, x_host, p);
  if (st) return st;
  CELG_CUDA(cudaSetDevice(h->device));
  const size_t n = (size_t)m->csr.n;
  if (n > h->scap || !h->sb) {
    CELG_CUDA(cudaStreamSynchronize(h->stream));
    graph_cache_clear(h);
    cudaFree(h->sb);
    cudaFree(h->sx);
    h->sb = h->sx = nullptr;
    h->scap = 0;  // a failed allocation below leaves no stale capacity behind
    const size_t cap = std::max<size_t>(n, 1024);
    CELG_CUDA(cudaMalloc(&h->sb, sizeof(double) * cap));
    CELG_CUDA(cudaMalloc(&h->sx, sizeof(double) * cap));
    h->scap = cap;
  }
  // host -> device copies of this solve's inputs, on the handle's stream
  CELG_CUDA(cudaMemcpyAsync(h->sb, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  if (p->x0_mode == CELG_X0_USER)
    CELG_CUDA(cudaMemcpyAsync(h->sx, x_host, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  int ret;
  if (solver == CELG_SOLVER_PCG) ret = celg_pcg_jacobi(h, m, h->sb, h->sx, p, res);
  else if (solver == CELG_SOLVER_CG) ret = cg_solve(h, m, h->sb, h->sx, p, res);
  else if (solver == CELG_SOLVER_GMRES) ret = gmres_solve(h, m, h->sb, h->sx, p, res);
  else ret = CELG_ERR_ARG;
  if (ret == CELG_OK || ret == CELG_ERR_NOCONV) {
    // device -> host copy of the solution
    CELG_CUDA(cudaMemcpyAsync(x_host, h->sx, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CELG_CUDA(cudaStreamSynchronize(h->stream));
  }
  return ret;
}
