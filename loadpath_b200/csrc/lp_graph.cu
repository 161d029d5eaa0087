// Host-side plumbing kept out of Python's way: CUDA graph capture of a stream (begin /
// end+instantiate / launch / free), so the solver records its set-up, CG head and CG tail once
// and replays each with one launch; capturable asynchronous copies and fills.
#include <cstring>
#include <mutex>

#include "lp_common.cuh"

#define LP_ST ((cudaStream_t)stream)

namespace {

// The PCG's stopping test on the device (loadpath/mg.py:872-926, as the host loop makes it):
// sc[0] = |b|^2, sc[3] = p.Ap, sc[4] = |r|^2 after this iteration's head; state[0] counts
// iterations, state[1] is left 1 converged, 2 zero right-hand side, 3 p.Ap not positive, 0
// otherwise. The loop continues while the test fails and fewer than maxiter iterations ran.
__global__ void k_cg_continue(cudaGraphConditionalHandle handle, const double* __restrict__ sc,
                              long long* __restrict__ state, double rtol, long long maxiter) {
  const long long it = state[0] + 1;
  state[0] = it;
  const double bb = sc[0], pap = sc[3], rr = sc[4];
  long long status = 0;
  if (bb == 0.0) status = 2;
  else if (!(pap > 0.0)) status = 3;
  else if (sqrt(rr) <= rtol * sqrt(bb)) status = 1;
  state[1] = status;
  cudaGraphSetConditional(handle, (status == 0 && it < maxiter) ? 1u : 0u);
}

// The same test for the k columns of a block solve: sc (k, 8) their scalars; state (k + 1, 2):
// row j the iteration at which column j stopped and its status (0 while it runs), row k the
// iteration count. The loop continues while a column runs and fewer than maxiter iterations ran.
__global__ void k_cg_continue_cols(cudaGraphConditionalHandle handle, const double* __restrict__ sc,
                                   long long* __restrict__ state, int k, double rtol, long long maxiter) {
  const long long it = state[2 * k] + 1;
  state[2 * k] = it;
  bool running = false;
  for (int j = 0; j < k; ++j) {
    if (state[2 * j + 1] != 0) continue;
    const double* s = sc + 8 * j;
    const double bb = s[0], pap = s[3], rr = s[4];
    long long status = 0;
    if (bb == 0.0) status = 2;
    else if (!(pap > 0.0)) status = 3;
    else if (sqrt(rr) <= rtol * sqrt(bb)) status = 1;
    if (status) {
      state[2 * j] = it;
      state[2 * j + 1] = status;
    } else {
      running = true;
    }
  }
  cudaGraphSetConditional(handle, (running && it < maxiter) ? 1u : 0u);
}

// out = m x (the solved bits) when column col converged at this iteration (state as above)
__global__ void k_snapshot_converged(double* __restrict__ out, const double* __restrict__ x,
                                     const uint8_t* __restrict__ m, const long long* __restrict__ state, int col,
                                     int k, LpGrid g) {
  if (state[2 * col + 1] != 1 || state[2 * col] != state[2 * k]) return;
  const long long nn = g.nodes_padded();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * nn; t += (long long)gridDim.x * blockDim.x) {
    const int c = t >= nn ? (t >= 2 * nn ? 2 : 1) : 0;
    out[t] = ((m[t - c * nn] >> c) & 1) ? x[t] : 0.0;
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)

namespace {
struct TuneEntry {
  int knob, nx, ny, nz, value;
};
std::mutex g_tune_mu;
TuneEntry g_tune[256];
int g_ntune = 0;
}  // namespace

int lp_tune_lookup(int knob, int nx, int ny, int nz) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (int i = 0; i < g_ntune; ++i)
    if (g_tune[i].knob == knob && g_tune[i].nx == nx && g_tune[i].ny == ny && g_tune[i].nz == nz)
      return g_tune[i].value;
  return 0;
}

extern "C" {

// Sets (value > 0) or clears (value 0) the tuned launch geometry of a knob for one grid; the
// launchers read it on their next call. -3 when the table is full.
int lpb_tune_set(int knob, int nx, int ny, int nz, int value) {
  if (knob < 1 || knob > LP_KNOB_MAX || nx < 1 || ny < 1 || nz < 1 || value < 0) return LP_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (int i = 0; i < g_ntune; ++i)
    if (g_tune[i].knob == knob && g_tune[i].nx == nx && g_tune[i].ny == ny && g_tune[i].nz == nz) {
      g_tune[i].value = value;
      return LP_OK;
    }
  if (value == 0) return LP_OK;
  if (g_ntune >= 256) return LP_ERR_SIZE;
  g_tune[g_ntune++] = TuneEntry{knob, nx, ny, nz, value};
  return LP_OK;
}

// the tuned value of a knob for a grid, 0 when none is set
int lpb_tune_get(int knob, int nx, int ny, int nz) {
  if (knob < 1 || knob > LP_KNOB_MAX) return LP_ERR_ARG;
  return lp_tune_lookup(knob, nx, ny, nz);
}

// Starts recording the body of a device-side while loop: a graph with one conditional WHILE node
// (its condition 1 at each launch of the graph), the stream capturing into the node's body.
// *handle: the condition's handle (for lpb_cg_continue); *graph: the outer graph, for
// lpb_while_end.
int lpb_while_begin(void* stream, long long* handle, void** graph) {
  if (!handle || !graph) return LP_ERR_ARG;
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return LP_ERR_LAUNCH;
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGraphDestroy(g);
    return LP_ERR_LAUNCH;
  }
  // a zeroed parameter block (the struct's union makes its default constructor deleted)
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& p = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, nullptr, 0, &p) != cudaSuccess ||
      cudaStreamBeginCaptureToGraph(LP_ST, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGraphDestroy(g);
    return LP_ERR_LAUNCH;
  }
  *handle = (long long)h;
  *graph = (void*)g;
  return LP_OK;
}

// Ends the body's capture and instantiates the outer graph; *exec receives a cudaGraphExec_t
int lpb_while_end(void* stream, void* graph, void** exec) {
  if (!graph || !exec) return LP_ERR_ARG;
  cudaGraph_t g = (cudaGraph_t)graph;
  cudaGraph_t body = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(LP_ST, &body);
  cudaGraphExec_t ge = nullptr;
  const cudaError_t ei = ec == cudaSuccess ? cudaGraphInstantiate(&ge, g, 0) : ec;
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return LP_ERR_LAUNCH;
  *exec = (void*)ge;
  return LP_OK;
}

// The loop's stopping test (k_cg_continue) as one launch in the body: sc the solve's scalars,
// state two device long longs (iterations, status), zeroed before the loop's launch
int lpb_cg_continue(long long handle, const double* sc, long long* state, double rtol, long long maxiter,
                    void* stream) {
  if (!sc || !state || maxiter < 1) return LP_ERR_ARG;
  k_cg_continue<<<1, 1, 0, LP_ST>>>((cudaGraphConditionalHandle)handle, sc, state, rtol, maxiter);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

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

// the block solve's test: k columns, sc (k, 8), state (k + 1, 2) zeroed before the loop
int lpb_cg_continue_cols(long long handle, const double* sc, long long* state, int k, double rtol, long long maxiter,
                         void* stream) {
  if (!sc || !state || k < 1 || maxiter < 1) return LP_ERR_ARG;
  k_cg_continue_cols<<<1, 1, 0, LP_ST>>>((cudaGraphConditionalHandle)handle, sc, state, k, rtol, maxiter);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out = m x if column col of a block solve converged at the current iteration (else nothing)
int lpb_snapshot_converged(double* out, const double* x, const uint8_t* mask, const long long* state, int col, int k,
                           LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !x || !mask || !state || col < 0 || col >= k || out == x) return LP_ERR_ARG;
  k_snapshot_converged<<<lp_blocks(3 * g.nodes_padded(), 256), 256, 0, LP_ST>>>(out, x, mask, state, col, k, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
