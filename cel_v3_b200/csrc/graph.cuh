// graph.cuh -- CUDA-graph helpers shared by the device-driven solvers: a
// small per-handle cache of instantiated solve graphs, capture of a WHILE
// conditional node whose body is recorded by a callback, and the switch to
// the host-driven profiling mode (CELG_GRAPH=0).
#pragma once
#include <cstdlib>
#include <cstring>
#include <string>

#include "celg_internal.h"

namespace celg {

inline bool graphs_enabled() {
  const char* e = std::getenv("CELG_GRAPH");
  return !(e && e[0] == '0');
}

inline GraphEntry* graph_cache_find(celg_handle* h, const std::string& key) {
  for (auto& e : h->graphs)
    if (e.key == key) return &e;
  return nullptr;
}

// Append a WHILE conditional node after the work captured so far on
// h->stream and capture the loop body (recorded by `body`) into it.
template <class Body>
int capture_while(celg_handle* h, cudaGraphConditionalHandle cond, Body body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cap_graph;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  CELG_CUDA(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cap_graph, &deps, &ndeps));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  CELG_CUDA(cudaGraphAddNode(&cnode, cap_graph, deps, ndeps, &cp));
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  CELG_CUDA(cudaStreamUpdateCaptureDependencies(h->stream, &cnode, 1,
                                                cudaStreamSetCaptureDependencies));
  cudaStream_t side;
  CELG_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCaptureToGraph(side, bodyg, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed);
  int st = CELG_OK;
  if (e == cudaSuccess) {
    cudaStream_t main_stream = h->stream;
    h->stream = side;
    st = body();
    h->stream = main_stream;
    cudaGraph_t out;
    e = cudaStreamEndCapture(side, &out);
  }
  cudaStreamDestroy(side);
  if (st) return st;
  CELG_CUDA(e);
  return CELG_OK;
}

// The same with the loop body recorded twice.  Consecutive sweeps walk the
// tiles in opposite orders (RedCtx::sweep), so a body of an odd number of
// sweeps would repeat the same orders in every iteration; with two
// iterations per body the orders alternate across iterations too.  The
// body's kernels must return at once when the solve has ended, since the
// second iteration runs after the first one stopped the loop.
template <class Body>
int capture_while2(celg_handle* h, cudaGraphConditionalHandle cond, Body body) {
  return capture_while(h, cond, [&]() -> int {
    int st = body();
    if (!st) st = body();
    return st;
  });
}

// Create a conditional handle on the graph being captured on h->stream
// (used for an IF node inside a loop body).
inline int capture_new_handle(celg_handle* h, unsigned default_value, cudaGraphConditionalHandle* out) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g;
  CELG_CUDA(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &g, nullptr, nullptr));
  CELG_CUDA(cudaGraphConditionalHandleCreate(out, g, default_value, cudaGraphCondAssignDefault));
  return CELG_OK;
}

// Append an IF conditional node after the work captured so far on h->stream;
// `body` records the work it guards.
template <class Body>
int capture_if(celg_handle* h, cudaGraphConditionalHandle cond, Body body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cap_graph;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  CELG_CUDA(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cap_graph, &deps, &ndeps));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  CELG_CUDA(cudaGraphAddNode(&cnode, cap_graph, deps, ndeps, &cp));
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  CELG_CUDA(cudaStreamUpdateCaptureDependencies(h->stream, &cnode, 1,
                                                cudaStreamSetCaptureDependencies));
  cudaStream_t side;
  CELG_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCaptureToGraph(side, bodyg, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed);
  int st = CELG_OK;
  if (e == cudaSuccess) {
    cudaStream_t main_stream = h->stream;
    h->stream = side;
    st = body();
    h->stream = main_stream;
    cudaGraph_t out;
    e = cudaStreamEndCapture(side, &out);
  }
  cudaStreamDestroy(side);
  if (st) return st;
  CELG_CUDA(e);
  return CELG_OK;
}

// Capture `record(cond)` on the handle's private capture stream (the caller's
// stream may be the legacy default stream, which cannot be captured),
// instantiate it and add it to the cache under `key`.
template <class Record>
int graph_build(celg_handle* h, const std::string& key, Record record, GraphEntry** out) {
  if (h->graphs.size() >= 16) {
    cudaStreamSynchronize(h->stream);
    graph_cache_clear(h);
  }
  cudaStream_t work_stream = h->stream;
  h->stream = h->cap_stream;
  cudaError_t e = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeRelaxed);
  cudaStreamCaptureStatus cs;
  cudaGraph_t cap_graph;
  if (e == cudaSuccess)
    e = cudaStreamGetCaptureInfo(h->cap_stream, &cs, nullptr, &cap_graph, nullptr, nullptr);
  cudaGraphConditionalHandle cond = 0;
  if (e == cudaSuccess)
    e = cudaGraphConditionalHandleCreate(&cond, cap_graph, 1, cudaGraphCondAssignDefault);
  int rst = e == cudaSuccess ? record(cond) : CELG_ERR_CUDA;
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(h->cap_stream, &g);
  h->stream = work_stream;
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_status(e, "graph capture set-up");
  }
  if (rst || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rst ? rst : cuda_status(e2, "cudaStreamEndCapture");
  }
  cudaGraphExec_t gx;
  cudaError_t e3 = cudaGraphInstantiate(&gx, g, 0);
  if (e3 != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(e3, "cudaGraphInstantiate");
  }
  h->graphs.push_back(GraphEntry{key, g, gx});
  *out = &h->graphs.back();
  return CELG_OK;
}

}  // namespace celg
