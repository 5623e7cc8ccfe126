// A batch's launch set captured once as a CUDA graph and replayed.
//
// The dense pipeline for a fixed batch layout (pair sizes, disparity ranges, input,
// output and workspace buffers) is a status-word reset and the four kernels of each
// launch set, whose descriptors travel as kernel parameters (a batch of several pairs
// runs as two launch sets on streams forked from the capturing stream and joined back
// to it, which the graph keeps as two branches).  Capturing them turns a repeated
// batch (a camera rig's frames, a fixed-size benchmark batch) into one graph launch,
// so the host pays one launch per batch instead of one per kernel.  Replays read
// whatever the captured input buffers hold at replay time.

#include <cuda_runtime.h>

#include "de_internal.h"

struct de_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

extern "C" {

int de_graph_create(const de_cfg* cfg, const de_pair* pairs, int n, void* workspace,
                    size_t bytes, de_graph** out) {
  if (!out) return de::set_error(DE_ERR_ARG, "out is NULL");
  size_t need = 0;
  if (int rc = de_dense_workspace_bytes(cfg, pairs, n, &need)) return rc;
  if (!workspace || bytes < need)
    return de::set_error(DE_ERR_ARG, "workspace %zu bytes < %zu", bytes, need);
  de_graph* g = new de_graph;
  cudaGetDevice(&g->device);
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    if (s) cudaStreamDestroy(s);
    delete g;
    return de::set_error(DE_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
  }
  const int rc = de_dense_dev(cfg, pairs, n, workspace, bytes, s);
  e = cudaStreamEndCapture(s, &g->graph);
  cudaStreamDestroy(s);
  if (rc || e != cudaSuccess) {
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc ? rc : de::set_error(DE_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g->graph);
    delete g;
    return de::set_error(DE_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
  }
  *out = g;
  return DE_OK;
}

int de_graph_launch(de_graph* g, void* stream) {
  if (!g) return de::set_error(DE_ERR_ARG, "graph is NULL");
  const cudaError_t e = cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
  return DE_OK;
}

int de_graph_destroy(de_graph* g) {
  if (!g) return DE_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return DE_OK;
}

}  // extern "C"
