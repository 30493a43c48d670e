// selftest.cu -- check of the bounded device waits.
//
// Every spin-wait of the library's kernels (the mbarrier waits of the SpMV
// bulk-copy pipeline) gives up after a time limit, records CELG_ERR_TIMEOUT
// in the handle's error word and returns, so that a wait which can never end
// turns into an error status instead of a hung GPU.  celg_check_bounded_wait
// runs that same wait on an mbarrier that nothing ever arrives on, with a
// short limit, and reports the status the host reads back; the context stays
// usable afterwards.
#include "tile_kernels.cuh"

namespace celg {

__global__ void bounded_wait_probe_kernel(int* err, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // expects one arrival; none will come
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) (void)mbar_wait_bounded(&bar, 0u, err, limit_ns);
}

}  // namespace celg

extern "C" int celg_check_bounded_wait(celg_handle* h, int limit_ms, int* status) {
  if (!h || !status || limit_ms <= 0 || limit_ms > 10000) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(h->device));
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  celg::bounded_wait_probe_kernel<<<1, 32, 0, h->stream>>>(h->err_d,
                                                          (unsigned long long)limit_ms * 1000000ull);
  CELG_CUDA(cudaGetLastError());
  int word = 0;
  CELG_CUDA(cudaMemcpyAsync(&word, h->err_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  CELG_CUDA(cudaMemsetAsync(h->err_d, 0, sizeof(int), h->stream));
  *status = word;
  return CELG_OK;
}
