// assemble.cu -- COO -> CSR on the device, and the MatrixMarket reader.
//
// The reference assembles a matrix as COO triplets, sorts them by row and
// then column (cel_sp_mat_format_sparse_31_sort,
// src/fspmt/cel_sp_mat_module.f90:518-585; entries with equal (row, column)
// keep their insertion order, and explicit zeros are kept) and builds the
// row pointer from the row counts (cel_sp_mat_to_csr, :430-456).  Here the
// sort is one stable radix sort of 64-bit (row, column) keys carrying the
// entry's position, the values are gathered through that permutation, and
// the row pointer is an exclusive scan of the row counts.
//
// MatrixMarket files are read as the reference's mmread does
// (src/fbase/cel_mmio_module.f90:17-341, called from
// cel_sp_mat_read_matrix_market_file, src/fspmt/cel_sp_mat_generate_module.f90:
// 219-273): coordinate or array representation, real / integer / pattern
// field, entries returned exactly as stored (1-based), so a symmetric file
// yields only its stored triangle unless the caller asks for the mirrored
// entries as well.
#include <cub/cub.cuh>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "celg_internal.h"

namespace celg {

__global__ void coo_key_kernel(int nnz, int n, int ncols, const int* __restrict__ rows,
                               const int* __restrict__ cols, int row_base, int col_base,
                               unsigned long long* __restrict__ key, int* __restrict__ idx,
                               int* __restrict__ counts, int* bad) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x) {
    const int r = rows[k] - row_base, c = cols[k] - col_base;
    if (r < 0 || r >= n || c < 0 || c >= ncols) {
      atomicExch(bad, 1);
      key[k] = 0ull;
    } else {
      key[k] = ((unsigned long long)(unsigned)r << 32) | (unsigned)c;
      atomicAdd(counts + r, 1);
    }
    idx[k] = (int)k;
  }
}

__global__ void coo_gather_kernel(int nnz, const unsigned long long* __restrict__ key,
                                  const int* __restrict__ perm, const double* __restrict__ vals,
                                  int* __restrict__ ci, double* __restrict__ v) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x) {
    ci[k] = (int)(unsigned)(key[k] & 0xffffffffull);
    v[k] = vals[perm[k]];
  }
}

static int bits_for(long v) {
  int b = 1;
  while (b < 31 && (1L << b) <= v) ++b;
  return b;
}

int coo_to_mat_device(celg_handle* h, int n, int ncols, int nnz, const int* rows_d,
                      const int* cols_d, const double* vals_d, int row_base, int col_base,
                      celg_mat** out) {
  *out = nullptr;
  celg_mat* m = new celg_mat();
  m->h = h;
  unsigned long long *key = nullptr, *key2 = nullptr;
  int *idx = nullptr, *perm = nullptr, *counts = nullptr;
  void* tmp = nullptr;
  int st = alloc_csr(m, n, nnz, ncols);
  cudaError_t e = cudaSuccess;
  const size_t nz = (size_t)std::max(1, nnz);
  auto chk = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
    return e == cudaSuccess;
  };
  const int grid = (int)std::max(1L, std::min(((long)nnz + 255) / 256, (long)h->sms * 16));
  int* bad = h->err_d + 2;
  if (!st) {
    chk(cudaMalloc(&key, sizeof(*key) * nz)) && chk(cudaMalloc(&key2, sizeof(*key2) * nz)) &&
        chk(cudaMalloc(&idx, sizeof(int) * nz)) && chk(cudaMalloc(&perm, sizeof(int) * nz)) &&
        chk(cudaMalloc(&counts, sizeof(int) * ((size_t)n + 1)));
    chk(cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)n + 1), h->stream));
    chk(cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
    if (e == cudaSuccess && nnz > 0) {
      coo_key_kernel<<<grid, 256, 0, h->stream>>>(nnz, n, ncols, rows_d, cols_d, row_base, col_base,
                                                  key, idx, counts, bad);
      chk(cudaGetLastError());
    }
    // stable sort of (row, column) keys: equal keys keep their input order
    const int end_bit = 32 + bits_for(n);
    size_t tb = 0;
    if (e == cudaSuccess)
      chk(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, idx, perm, nnz, 0, end_bit,
                                          h->stream));
    size_t sb = 0;
    if (e == cudaSuccess)
      chk(cub::DeviceScan::ExclusiveSum(nullptr, sb, counts, m->csr.rp, n + 1, h->stream));
    if (e == cudaSuccess) chk(cudaMalloc(&tmp, std::max<size_t>(std::max(tb, sb), 16)));
    if (e == cudaSuccess && nnz > 0)
      chk(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, idx, perm, nnz, 0, end_bit, h->stream));
    // row pointer: exclusive scan of the counts over n+1 entries (the last
    // count is 0, so rp[n] = nnz of the valid entries)
    if (e == cudaSuccess) chk(cub::DeviceScan::ExclusiveSum(tmp, sb, counts, m->csr.rp, n + 1, h->stream));
    if (e == cudaSuccess && nnz > 0) {
      coo_gather_kernel<<<grid, 256, 0, h->stream>>>(nnz, key2, perm, vals_d, m->csr.ci, m->csr.v);
      chk(cudaGetLastError());
    }
    int hb = 0;
    if (e == cudaSuccess) chk(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (e == cudaSuccess) chk(cudaStreamSynchronize(h->stream));
    if (e != cudaSuccess) st = cuda_status(e, "COO to CSR");
    else if (hb) st = CELG_ERR_ARG;
  }
  cudaFree(key);
  cudaFree(key2);
  cudaFree(idx);
  cudaFree(perm);
  cudaFree(counts);
  cudaFree(tmp);
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

// ---- MatrixMarket -------------------------------------------------------------

namespace {

struct MmHeader {
  bool coordinate = true;
  int field = 0;  // 0 real, 1 integer, 2 pattern
  int symm = CELG_MM_GENERAL;
  long nrows = 0, ncols = 0, nstored = 0;
};

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// Parses the banner and the size line; leaves f at the first entry.
int mm_header(FILE* f, MmHeader* hd) {
  char line[4096];
  if (!std::fgets(line, sizeof(line), f)) return CELG_ERR_ARG;
  char b[64] = {0}, obj[64] = {0}, rep[64] = {0}, fld[64] = {0}, sym[64] = {0};
  if (std::sscanf(line, "%63s %63s %63s %63s %63s", b, obj, rep, fld, sym) != 5) return CELG_ERR_ARG;
  if (lower(b) != "%%matrixmarket" || lower(obj) != "matrix") return CELG_ERR_ARG;
  const std::string r = lower(rep), fl = lower(fld), sy = lower(sym);
  if (r == "coordinate") hd->coordinate = true;
  else if (r == "array") hd->coordinate = false;
  else return CELG_ERR_ARG;
  if (fl == "real" || fl == "double") hd->field = 0;
  else if (fl == "integer") hd->field = 1;
  else if (fl == "pattern" && hd->coordinate) hd->field = 2;
  else return CELG_ERR_ARG;  // complex data has no place in a real solver
  if (sy == "general") hd->symm = CELG_MM_GENERAL;
  else if (sy == "symmetric") hd->symm = CELG_MM_SYMMETRIC;
  else if (sy == "skew-symmetric") hd->symm = CELG_MM_SKEW;
  else return CELG_ERR_ARG;
  do {
    if (!std::fgets(line, sizeof(line), f)) return CELG_ERR_ARG;
  } while (line[0] == '%' || std::strspn(line, " \t\r\n") == std::strlen(line));
  if (hd->coordinate) {
    if (std::sscanf(line, "%ld %ld %ld", &hd->nrows, &hd->ncols, &hd->nstored) != 3) return CELG_ERR_ARG;
  } else {
    if (std::sscanf(line, "%ld %ld", &hd->nrows, &hd->ncols) != 2) return CELG_ERR_ARG;
    const long N = hd->nrows, M = hd->ncols;
    if (hd->symm == CELG_MM_GENERAL) hd->nstored = N * M;
    else if (hd->symm == CELG_MM_SYMMETRIC) hd->nstored = N * (N + 1) / 2;
    else hd->nstored = N * (N - 1) / 2;
  }
  if (hd->nrows < 0 || hd->ncols < 0 || hd->nstored < 0 || hd->nrows > INT32_MAX ||
      hd->ncols > INT32_MAX)
    return CELG_ERR_ARG;
  return CELG_OK;
}

// Calls emit(row, col, value) (1-based) for every stored entry, in file order.
template <class F>
int mm_entries(FILE* f, const MmHeader& hd, F&& emit) {
  if (hd.coordinate) {
    for (long k = 0; k < hd.nstored; ++k) {
      long r = 0, c = 0;
      double v = 1.0;
      if (hd.field == 2) {
        if (std::fscanf(f, "%ld %ld", &r, &c) != 2) return CELG_ERR_ARG;
      } else if (std::fscanf(f, "%ld %ld %lf", &r, &c, &v) != 3) {
        return CELG_ERR_ARG;
      }
      if (r < 1 || r > hd.nrows || c < 1 || c > hd.ncols) return CELG_ERR_ARG;
      emit((int)r, (int)c, v);
    }
  } else {
    // dense, column-major; symmetric: lower triangle incl. the diagonal;
    // skew-symmetric: strictly lower triangle
    for (long j = 1; j <= hd.ncols; ++j) {
      const long i0 = hd.symm == CELG_MM_GENERAL ? 1 : (hd.symm == CELG_MM_SYMMETRIC ? j : j + 1);
      for (long i = i0; i <= hd.nrows; ++i) {
        double v = 0.0;
        if (std::fscanf(f, "%lf", &v) != 1) return CELG_ERR_ARG;
        emit((int)i, (int)j, v);
      }
    }
  }
  return CELG_OK;
}

}  // namespace

}  // namespace celg

using namespace celg;

extern "C" int celg_mat_from_coo(celg_handle* h, int n, int ncols, int nnz, const int* rows,
                                 const int* cols, const double* vals, int index_base,
                                 celg_mat** out) {
  if (!h || !out || n < 0 || ncols < n || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)) ||
      (index_base != 0 && index_base != 1))
    return CELG_ERR_ARG;
  *out = nullptr;
  CELG_CUDA(cudaSetDevice(h->device));
  const size_t nz = (size_t)std::max(1, nnz);
  int *r_d = nullptr, *c_d = nullptr;
  double* v_d = nullptr;
  cudaError_t e = cudaMalloc(&r_d, sizeof(int) * nz);
  if (e == cudaSuccess) e = cudaMalloc(&c_d, sizeof(int) * nz);
  if (e == cudaSuccess) e = cudaMalloc(&v_d, sizeof(double) * nz);
  if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(r_d, rows, sizeof(int) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(c_d, cols, sizeof(int) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && nnz > 0)
    e = cudaMemcpyAsync(v_d, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, h->stream);
  int st = e == cudaSuccess ? coo_to_mat_device(h, n, ncols, nnz, r_d, c_d, v_d, index_base,
                                                index_base, out)
                            : cuda_status(e, "COO upload");
  cudaStreamSynchronize(h->stream);
  cudaFree(r_d);
  cudaFree(c_d);
  cudaFree(v_d);
  return st;
}

extern "C" int celg_mm_info(const char* path, int expand, int* nrows, int* ncols, int* nnz,
                            int* symmetry) {
  if (!path) return CELG_ERR_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return CELG_ERR_ARG;
  MmHeader hd;
  int st = mm_header(f, &hd);
  long count = hd.nstored;
  if (!st && expand && hd.symm != CELG_MM_GENERAL) {
    count = 0;
    st = mm_entries(f, hd, [&](int r, int c, double) { count += (r == c) ? 1 : 2; });
  }
  std::fclose(f);
  if (st) return st;
  if (count > INT32_MAX) return CELG_ERR_ARG;
  if (nrows) *nrows = (int)hd.nrows;
  if (ncols) *ncols = (int)hd.ncols;
  if (nnz) *nnz = (int)count;
  if (symmetry) *symmetry = hd.symm;
  return CELG_OK;
}

extern "C" int celg_mm_read(const char* path, int expand, int nnz_cap, int* rows, int* cols,
                            double* vals) {
  if (!path || nnz_cap < 0 || (nnz_cap > 0 && (!rows || !cols || !vals))) return CELG_ERR_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return CELG_ERR_ARG;
  MmHeader hd;
  int st = mm_header(f, &hd);
  long k = 0;
  bool overflow = false;
  auto put = [&](int r, int c, double v) {
    if (k >= nnz_cap) {
      overflow = true;
      return;
    }
    rows[k] = r;
    cols[k] = c;
    vals[k] = v;
    ++k;
  };
  if (!st)
    st = mm_entries(f, hd, [&](int r, int c, double v) {
      put(r, c, v);
      if (expand && hd.symm != CELG_MM_GENERAL && r != c)
        put(c, r, hd.symm == CELG_MM_SKEW ? -v : v);
    });
  std::fclose(f);
  if (st) return st;
  return overflow ? CELG_ERR_ARG : CELG_OK;
}
