// noalloc.cu -- an allocation-free dot product for callers that cannot
// allocate device memory.
//
// Some callers of this library do not own the device memory of their
// process: a Fortran application that hands every device allocation to its
// own pool, or a framework whose caching allocator has already committed the
// GPU, cannot let a library call cudaMalloc from inside its solver step.  The
// handle-based entry points allocate their scratch (tile partials, the
// completion ticket, result slots) when a handle is created or grows.  This
// entry point needs no handle: it keeps that scratch in a fixed file-scope
// device array instead, and writes the result to a device pointer the caller
// passes, so it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits and sharing:
//   * at most CELG_NOALLOC_MAX_ROWS (2^26 = 67,108,864) elements; longer
//     vectors are rejected with CELG_ERR_ARG before anything is launched;
//   * the array (512 KiB of tile partials plus a 256-byte header with the
//     ticket) exists on every GPU that loads the library, until the process
//     exits;
//   * every call shares it: two calls whose kernels overlap on the GPU (on
//     different streams, or from different threads) race on it and their
//     results are undefined.  Calls ordered on one stream are safe; the
//     ticket is cleared by each call before its kernel starts.
//   * each call outside a stream capture looks up the array's device
//     address on the current device (cudaGetSymbolAddress, with that device
//     current) and caches it; a call on a capturing stream uses the cached
//     address, so make one call on the device before any stream capture.
//     Looking the address up again on every uncaptured call keeps it valid
//     across a cudaDeviceReset, which recreates the device's context and
//     with it the array.
#include <mutex>

#include "tile_kernels.cuh"

namespace {

constexpr long kMaxRows = CELG_NOALLOC_MAX_ROWS;
constexpr long kMaxTiles = kMaxRows / celg::kTile;  // 65,536 tile partials
constexpr size_t kHeader = 256;                     // completion ticket lives here

// file-scope scratch: [0, 256) ticket, [256, ...) tile partials (f64)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kHeader + kMaxTiles * sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// Device address of the scratch array on `dev`, with that device current:
// looked up again unless the stream is capturing (then the address cached by
// an earlier call is used).
int scratch_for_device(int dev, cudaStream_t stream, void** addr, int* sms) {
  if (dev < 0 || dev >= kMaxDevices) return CELG_ERR_ARG;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CELG_CUDA(cudaStreamIsCapturing(stream, &cap));
  std::lock_guard<std::mutex> lock(g_mutex);
  if (cap == cudaStreamCaptureStatusNone || !g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return celg::cuda_status(e, "cudaGetSymbolAddress(noalloc scratch)");
    int s = 0;
    e = cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return celg::cuda_status(e, "cudaDeviceGetAttribute");
    g_sms[dev] = s;
    g_addr[dev] = p;
  }
  *addr = g_addr[dev];
  *sms = g_sms[dev];
  return CELG_OK;
}

}  // namespace

// out_d[0] = sum_i a_d[i] * b_d[i] in the library's fixed reduction order
// (bit-identical to celg_dot), computed on `stream` (NULL: the default
// stream) of the calling thread's current device.
extern "C" int celg_dot_noalloc(int n, const double* a_d, const double* b_d, double* out_d,
                                void* stream) {
  if (n < 0 || !out_d || (n > 0 && (!a_d || !b_d))) return CELG_ERR_ARG;
  if ((long)n > kMaxRows) return CELG_ERR_ARG;  // beyond the fixed scratch
  int dev = 0;
  CELG_CUDA(cudaGetDevice(&dev));
  void* base = nullptr;
  int sms = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = scratch_for_device(dev, s, &base, &sms);
  if (st) return st;
  unsigned* ticket = static_cast<unsigned*>(base);
  double* partials = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kHeader);
  CELG_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  const long ntiles = celg::ntiles_of(n);
  const int grid = (int)std::max(1L, std::min(ntiles, (long)sms * 8));
  celg::RedCtx red{partials, ticket, ntiles};
  celg::tile_kernel<celg::OpDot><<<grid, celg::kLanes, 0, s>>>(
      (long)n, celg::OpDot{a_d, b_d, out_d, 0}, red);
  CELG_CUDA(cudaGetLastError());
  return CELG_OK;
}
