// Host-side plumbing kept out of Python's way: CUDA graph capture of a stream (begin /
// end+instantiate / launch / free), so the solver records its set-up, CG head and CG tail once
// and replays each with one launch; capturable asynchronous copies and fills.
#include "lp_common.cuh"

#define LP_ST ((cudaStream_t)stream)

extern "C" {

int lpb_capture_begin(void* stream) {
  return cudaStreamBeginCapture(LP_ST, cudaStreamCaptureModeThreadLocal) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

// ends the capture and instantiates it; *exec receives a cudaGraphExec_t
int lpb_capture_end(void* stream, void** exec) {
  if (!exec) return LP_ERR_ARG;
  cudaGraph_t graph = nullptr;
  if (cudaStreamEndCapture(LP_ST, &graph) != cudaSuccess || !graph) return LP_ERR_LAUNCH;
  cudaGraphExec_t ge = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ge, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return LP_ERR_LAUNCH;
  *exec = (void*)ge;
  return LP_OK;
}

int lpb_graph_launch(void* exec, void* stream) {
  if (!exec) return LP_ERR_ARG;
  return cudaGraphLaunch((cudaGraphExec_t)exec, LP_ST) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

// cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, stream): capturable scalar moves
int lpb_memcpy_async(void* dst, const void* src, long long bytes, void* stream) {
  if (!dst || !src || bytes < 0) return LP_ERR_ARG;
  return cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDefault, LP_ST) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

// cudaMemsetAsync(dst, value, bytes, stream): capturable zero fills
int lpb_memset_async(void* dst, int value, long long bytes, void* stream) {
  if (!dst || bytes < 0) return LP_ERR_ARG;
  return cudaMemsetAsync(dst, value, (size_t)bytes, LP_ST) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

int lpb_graph_free(void* exec) {
  if (!exec) return LP_OK;
  return cudaGraphExecDestroy((cudaGraphExec_t)exec) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

}  // extern "C"
