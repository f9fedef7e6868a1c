// CUDA graphs for the passes the time step repeats.
//
// A pass (the kernels, memsets and copies of one culling pass, or one block of Krylov
// iterations) is captured once on the simulator's private capture stream and replayed on
// the working stream with one launch.  Every argument a captured kernel reads by value
// (pointers, capacities, parameters) is part of the pass's key; a different key recaptures.
// Values that change between replays (the line-search step, the iteration counter, the
// number of preconditioner clusters) live in device memory or are copied from pinned host
// memory by a node of the graph itself.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "abd_common.cuh"

namespace abd {

// FNV-1a over the bytes of a key description
struct KeyHash {
  uint64_t h = 1469598103934665603ULL;
  template <class T>
  KeyHash& add(const T& v) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
    for (size_t i = 0; i < sizeof(T); ++i) {
      h ^= b[i];
      h *= 1099511628211ULL;
    }
    return *this;
  }
};

// Replays slot g (capturing it first when the key differs).  issue() enqueues the pass on
// s.stream (redirected to the capture stream while capturing) and returns an ABD status.
template <class F>
int run_graph(Sim& s, GraphSlot& g, uint64_t key, F&& issue) {
  if (!g.exec || g.key != key) {
    if (g.exec) {
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
    const cudaStream_t work = s.stream;
    const long long l0 = s.launches;
    s.stream = s.cap_stream;
    cudaError_t e = ABD_NOTE(cudaStreamBeginCapture(s.cap_stream, cudaStreamCaptureModeThreadLocal));
    int r = e == cudaSuccess ? issue() : ABD_ERR_CUDA;
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = e == cudaSuccess ? ABD_NOTE(cudaStreamEndCapture(s.cap_stream, &graph)) : e;
    s.stream = work;
    if (r == ABD_OK && e2 != cudaSuccess) r = ABD_ERR_CUDA;
    if (r == ABD_OK && ABD_NOTE(cudaGraphInstantiate(&g.exec, graph, 0)) != cudaSuccess) r = ABD_ERR_CUDA;
    if (graph) cudaGraphDestroy(graph);
    g.nlaunch = s.launches - l0;
    s.launches = l0;
    if (r != ABD_OK) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
      return r;
    }
    g.key = key;
  }
  if (ABD_NOTE(cudaGraphLaunch(g.exec, s.stream)) != cudaSuccess) return ABD_ERR_CUDA;
  s.launches += g.nlaunch;
  return ABD_OK;
}

// Conditional nodes built during stream capture: a handle of the graph being captured, a
// WHILE or IF node after the work captured so far, and the capture of its body graph on a
// stream of its own.
#define GCK(x)                                         \
  do {                                                 \
    if (ABD_NOTE(x) != cudaSuccess) return ABD_ERR_CUDA; \
  } while (0)

// A conditional handle of the graph being captured on st (its value is set by kernels)
inline int make_handle(cudaStream_t st, cudaGraphConditionalHandle* hc) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t graph = nullptr;
  GCK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, nullptr, nullptr));
  if (cs != cudaStreamCaptureStatusActive) return ABD_ERR_CUDA;
  GCK(cudaGraphConditionalHandleCreate(hc, graph, 0, 0));
  return ABD_OK;
}

// Adds a conditional node (hc, type) after the work captured on st so far; what st captures
// next follows the node.  *body: the node's body graph.
inline int add_conditional(cudaStream_t st, cudaGraphConditionalHandle hc, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  GCK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps));
  if (cs != cudaStreamCaptureStatusActive) return ABD_ERR_CUDA;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = hc;
  np.conditional.type = type;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  GCK(cudaGraphAddNode(&node, graph, deps, ndeps, &np));
  *body = np.conditional.phGraph_out[0];
  GCK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  return ABD_OK;
}

// Captures issue() into the body graph of a conditional node, on stream bs (the simulator's
// stream points there meanwhile)
template <class F>
inline int capture_body(Sim& s, cudaGraph_t body, cudaStream_t bs, F&& issue) {
  GCK(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const cudaStream_t saved = s.stream;
  s.stream = bs;
  const int r = issue();
  s.stream = saved;
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(bs, &out);
  if (r) return r;
  return e == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
}

#undef GCK

}  // namespace abd
