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

}  // namespace abd
