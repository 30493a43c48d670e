// dist_solve.cu -- the whole distributed Jacobi-PCG of one rank in one call.
//
// In the reference the exchanges live inside the solver: the master thread
// posts the halo of p inside the SpMV (cel_fop_mv_axy_distr,
// src/fop/cel_fop_mv_module.f90:48-81) and every dot product ends in an
// MPI_ALLREDUCE (src/fop/cel_fop_vec_distr_module.f90:419, 471, 530, ...).
// celg_dist_pcg_solve does the same for the phases of dist.cu: it runs the
// whole sequence
//   begin [R]; halo(x); init [R]; start;
//   repeat (poll every `poll_every` iterations): halo(p); ap [R]; update [R];
//                                                direction;
//   halo(x); verify [R]; result
// ([R]: sum-all-reduce of the exchange buffer) with the exchanges done by
//   * callbacks of the caller's communication layer (MPI, NCCL, a thread
//     barrier ...), or
//   * NCCL, which the library drives itself (celg_dist_pcg_solve_nccl) from
//     an exchange plan (celg_dist_set_exchange): the rows each neighbour
//     reads are gathered into a send buffer, the received values land in the
//     halo part of the vector, all enqueued on the handle's stream; with
//     `overlap` the halo of p travels on a side stream while the interior
//     rows' SpMV runs (celg_dist_pcg_ap_interior / _boundary).
// NCCL is loaded at run time (dlopen of libnccl.so.2, the copy already in
// the process when there is one), so the library itself needs NCCL only
// when these entry points are used.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "tile_kernels.cuh"

namespace celg {

// ---- NCCL, loaded on first use -------------------------------------------------

struct NcclApi {
  bool ok = false;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
};

static const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
    if (!lib) return;
    auto sym = [&](auto& f, const char* name) {
      f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(lib, name));
      return f != nullptr;
    };
    api.ok = sym(api.GetUniqueId, "ncclGetUniqueId") && sym(api.CommInitRank, "ncclCommInitRank") &&
             sym(api.CommDestroy, "ncclCommDestroy") && sym(api.AllReduce, "ncclAllReduce") &&
             sym(api.Send, "ncclSend") && sym(api.Recv, "ncclRecv") &&
             sym(api.GroupStart, "ncclGroupStart") && sym(api.GroupEnd, "ncclGroupEnd");
  });
  return api;
}

#define CELG_NCCL(call)                                                      \
  do {                                                                       \
    if ((call) != ncclSuccess) return CELG_ERR_COMM;                         \
  } while (0)

// out[k] = vec[rows[k]]: the values a neighbour reads, packed for sending
__global__ void dist_pack_kernel(int count, const int* __restrict__ rows,
                                 const double* __restrict__ vec, double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
    out[k] = vec[rows[k]];
}

}  // namespace celg

using namespace celg;

// Work vectors and exchange plan of the one-call solve, kept by the celg_dist
// object (dist.cu frees them through dist_solve_free).
struct DistSolveData {
  double* r = nullptr;
  double* v = nullptr;
  double* p = nullptr;
  int n = 0, ncols = 0;
  // exchange plan: per neighbour its rank, the slice [send_off, send_off +
  // send_cnt) of send_rows (this rank's local rows it reads), and where its
  // values land in the halo: entries n + recv_start .. + recv_cnt - 1
  std::vector<int> peer, send_off, send_cnt, recv_start, recv_cnt;
  int nsend = 0;
  int* send_rows_d = nullptr;
  double* send_buf_d = nullptr;
  bool plan = false;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_go = nullptr, ev_done = nullptr;
};

namespace celg {
void dist_solve_free(void* p) {
  DistSolveData* s = static_cast<DistSolveData*>(p);
  if (!s) return;
  cudaFree(s->r);
  cudaFree(s->v);
  cudaFree(s->p);
  cudaFree(s->send_rows_d);
  cudaFree(s->send_buf_d);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->ev_go) cudaEventDestroy(s->ev_go);
  if (s->ev_done) cudaEventDestroy(s->ev_done);
  delete s;
}
}  // namespace celg

static int solve_data(celg_dist* d, DistSolveData** out) {
  celg_handle* h = nullptr;
  int n = 0, ncols = 0;
  void** slot = nullptr;
  int st = dist_internals(d, &h, &n, &ncols, &slot);
  if (st) return st;
  DistSolveData* s = static_cast<DistSolveData*>(*slot);
  if (!s) {
    s = new DistSolveData();
    s->n = n;
    s->ncols = ncols;
    *slot = s;
    CELG_CUDA(cudaMalloc(&s->r, sizeof(double) * (size_t)n));
    CELG_CUDA(cudaMalloc(&s->v, sizeof(double) * (size_t)n));
    CELG_CUDA(cudaMalloc(&s->p, sizeof(double) * (size_t)ncols));
    CELG_CUDA(cudaMemsetAsync(s->p, 0, sizeof(double) * (size_t)ncols, h->stream));
  }
  *out = s;
  return CELG_OK;
}

extern "C" int celg_dist_set_exchange(celg_dist* d, int nneigh, const int* peers,
                                      const int* send_counts, const int* send_rows,
                                      const int* recv_starts, const int* recv_counts) {
  if (!d || nneigh < 0 || (nneigh > 0 && (!peers || !send_counts || !recv_starts || !recv_counts)))
    return CELG_ERR_ARG;
  celg_handle* h = nullptr;
  int n = 0, ncols = 0;
  void** slot = nullptr;
  int st = dist_internals(d, &h, &n, &ncols, &slot);
  if (st) return st;
  long nsend = 0, nrecv = 0;
  for (int q = 0; q < nneigh; ++q) {
    if (peers[q] < 0 || send_counts[q] < 0 || recv_counts[q] < 0 || recv_starts[q] < 0 ||
        n + (long)recv_starts[q] + recv_counts[q] > ncols)
      return CELG_ERR_ARG;
    nsend += send_counts[q];
    nrecv += recv_counts[q];
  }
  if (nsend > 0 && !send_rows) return CELG_ERR_ARG;
  for (long k = 0; k < nsend; ++k)
    if (send_rows[k] < 0 || send_rows[k] >= n) return CELG_ERR_ARG;
  if (nsend > INT_MAX || nrecv > INT_MAX) return CELG_ERR_ARG;
  CELG_CUDA(cudaSetDevice(h->device));
  DistSolveData* s = nullptr;
  if ((st = solve_data(d, &s))) return st;
  CELG_CUDA(cudaStreamSynchronize(h->stream));
  cudaFree(s->send_rows_d);
  cudaFree(s->send_buf_d);
  s->send_rows_d = nullptr;
  s->send_buf_d = nullptr;
  s->peer.assign(peers, peers + nneigh);
  s->send_cnt.assign(send_counts, send_counts + nneigh);
  s->recv_start.assign(recv_starts, recv_starts + nneigh);
  s->recv_cnt.assign(recv_counts, recv_counts + nneigh);
  s->send_off.assign(nneigh, 0);
  for (int q = 1; q < nneigh; ++q) s->send_off[q] = s->send_off[q - 1] + send_counts[q - 1];
  s->nsend = (int)nsend;
  if (nsend > 0) {
    CELG_CUDA(cudaMalloc(&s->send_rows_d, sizeof(int) * (size_t)nsend));
    CELG_CUDA(cudaMalloc(&s->send_buf_d, sizeof(double) * (size_t)nsend));
    CELG_CUDA(cudaMemcpy(s->send_rows_d, send_rows, sizeof(int) * (size_t)nsend,
                         cudaMemcpyHostToDevice));
  }
  s->plan = true;
  return CELG_OK;
}

namespace {

// The exchanges of one solve: callbacks of the caller, or NCCL with the plan.
struct Exchanger {
  const celg_dist_comm* cb = nullptr;
  ncclComm_t comm = nullptr;
  DistSolveData* s = nullptr;
  celg_handle* h = nullptr;
  double* xch = nullptr;

  int allreduce(cudaStream_t stream) {
    if (cb) return cb->allreduce_sum(cb->ctx, xch, CELG_DIST_NEXCH, stream) ? CELG_ERR_COMM : CELG_OK;
    CELG_NCCL(nccl().AllReduce(xch, xch, CELG_DIST_NEXCH, ncclDouble, ncclSum, comm, stream));
    return CELG_OK;
  }
  int halo(double* vec, cudaStream_t stream) {
    if (cb) return cb->halo(cb->ctx, vec, stream) ? CELG_ERR_COMM : CELG_OK;
    if (s->peer.empty()) return CELG_OK;
    if (s->nsend > 0) {
      const int grid = std::max(1, std::min((s->nsend + 255) / 256, h->sms * 4));
      dist_pack_kernel<<<grid, 256, 0, stream>>>(s->nsend, s->send_rows_d, vec, s->send_buf_d);
      CELG_CUDA(cudaGetLastError());
    }
    const NcclApi& api = nccl();
    CELG_NCCL(api.GroupStart());
    for (size_t q = 0; q < s->peer.size(); ++q) {
      if (s->send_cnt[q] > 0)
        CELG_NCCL(api.Send(s->send_buf_d + s->send_off[q], (size_t)s->send_cnt[q], ncclDouble,
                           s->peer[q], comm, stream));
      if (s->recv_cnt[q] > 0)
        CELG_NCCL(api.Recv(vec + s->n + s->recv_start[q], (size_t)s->recv_cnt[q], ncclDouble,
                           s->peer[q], comm, stream));
    }
    CELG_NCCL(api.GroupEnd());
    return CELG_OK;
  }
};

int run_solve(celg_dist* d, Exchanger& ex, const double* b_d, double* x_ext_d, int poll_every,
              bool overlap, celg_result* res) {
  DistSolveData* s = ex.s;
  celg_handle* h = ex.h;
  cudaStream_t stream = h->stream;
  int st = celg_dist_exchange_buffer(d, &ex.xch);
#define STEP(call)         \
  do {                     \
    if ((st = (call))) return st; \
  } while (0)
  if (st) return st;
  STEP(celg_dist_pcg_begin(d, b_d, x_ext_d));
  STEP(ex.allreduce(stream));
  STEP(ex.halo(x_ext_d, stream));
  STEP(celg_dist_pcg_init(d, b_d, x_ext_d, s->r, s->p));
  STEP(ex.allreduce(stream));
  STEP(celg_dist_pcg_start(d));
  if (overlap && !s->side) {
    CELG_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    CELG_CUDA(cudaEventCreateWithFlags(&s->ev_go, cudaEventDisableTiming));
    CELG_CUDA(cudaEventCreateWithFlags(&s->ev_done, cudaEventDisableTiming));
  }
  for (;;) {
    int active = 0;
    STEP(celg_dist_pcg_poll(d, &active, nullptr));
    if (!active) break;
    for (int k = 0; k < poll_every; ++k) {
      if (overlap) {
        // the halo of p on the side stream, after the work queued so far
        CELG_CUDA(cudaEventRecord(s->ev_go, stream));
        CELG_CUDA(cudaStreamWaitEvent(s->side, s->ev_go, 0));
        STEP(ex.halo(s->p, s->side));
        CELG_CUDA(cudaEventRecord(s->ev_done, s->side));
        STEP(celg_dist_pcg_ap_interior(d, s->p, s->v));
        CELG_CUDA(cudaStreamWaitEvent(stream, s->ev_done, 0));
        STEP(celg_dist_pcg_ap_boundary(d, s->p, s->v));
      } else {
        STEP(ex.halo(s->p, stream));
        STEP(celg_dist_pcg_ap(d, s->p, s->v));
      }
      STEP(ex.allreduce(stream));
      STEP(celg_dist_pcg_update(d, s->r, s->v));
      STEP(ex.allreduce(stream));
      STEP(celg_dist_pcg_direction(d, x_ext_d, s->r, s->p));
    }
  }
  STEP(ex.halo(x_ext_d, stream));
  STEP(celg_dist_pcg_verify(d, b_d, x_ext_d));
  STEP(ex.allreduce(stream));
#undef STEP
  return celg_dist_pcg_result(d, res);
}

}  // namespace

extern "C" int celg_dist_pcg_solve(celg_dist* d, const celg_dist_comm* comm, const double* b_d,
                                   double* x_ext_d, int poll_every, celg_result* res) {
  if (!d || !comm || !comm->allreduce_sum || !comm->halo || !b_d || !x_ext_d || poll_every < 1)
    return CELG_ERR_ARG;
  Exchanger ex;
  ex.cb = comm;
  int st = solve_data(d, &ex.s);
  if (st) return st;
  int n = 0, ncols = 0;
  void** slot = nullptr;
  if ((st = dist_internals(d, &ex.h, &n, &ncols, &slot))) return st;
  CELG_CUDA(cudaSetDevice(ex.h->device));
  return run_solve(d, ex, b_d, x_ext_d, poll_every, false, res);
}

extern "C" int celg_nccl_unique_id(unsigned char id[CELG_NCCL_ID_BYTES]) {
  if (!id) return CELG_ERR_ARG;
  if (!nccl().ok) return CELG_ERR_STATE;
  static_assert(sizeof(ncclUniqueId) == CELG_NCCL_ID_BYTES, "NCCL unique id size");
  ncclUniqueId u;
  CELG_NCCL(nccl().GetUniqueId(&u));
  std::memcpy(id, &u, sizeof(u));
  return CELG_OK;
}

extern "C" int celg_nccl_comm_create(const unsigned char id[CELG_NCCL_ID_BYTES], int nranks, int rank,
                                     int device, void** comm) {
  if (!id || !comm || nranks < 1 || rank < 0 || rank >= nranks) return CELG_ERR_ARG;
  if (!nccl().ok) return CELG_ERR_STATE;
  CELG_CUDA(cudaSetDevice(device));
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof(u));
  ncclComm_t c = nullptr;
  CELG_NCCL(nccl().CommInitRank(&c, nranks, u, rank));
  *comm = c;
  return CELG_OK;
}

extern "C" int celg_nccl_comm_destroy(void* comm) {
  if (!comm) return CELG_OK;
  if (!nccl().ok) return CELG_ERR_STATE;
  CELG_NCCL(nccl().CommDestroy(static_cast<ncclComm_t>(comm)));
  return CELG_OK;
}

extern "C" int celg_dist_pcg_solve_nccl(celg_dist* d, void* comm, const double* b_d,
                                        double* x_ext_d, int poll_every, int overlap,
                                        celg_result* res) {
  if (!d || !comm || !b_d || !x_ext_d || poll_every < 1) return CELG_ERR_ARG;
  if (!nccl().ok) return CELG_ERR_STATE;
  Exchanger ex;
  ex.comm = static_cast<ncclComm_t>(comm);
  int st = solve_data(d, &ex.s);
  if (st) return st;
  if (!ex.s->plan) return CELG_ERR_STATE;  // celg_dist_set_exchange first
  int n = 0, ncols = 0;
  void** slot = nullptr;
  if ((st = dist_internals(d, &ex.h, &n, &ncols, &slot))) return st;
  CELG_CUDA(cudaSetDevice(ex.h->device));
  return run_solve(d, ex, b_d, x_ext_d, poll_every, overlap != 0, res);
}
