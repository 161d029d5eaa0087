// Host-side plumbing kept out of Python's way:
//  - CUDA graph capture of a stream (begin / end+instantiate / launch / free), so the solver can
//    record a CG iteration once per solve and replay it with one launch;
//  - the coarsest level's dense inverse: Cholesky (cusolverDnDpotrf) and inverse from the
//    factor (cusolverDnDpotri) on the device, then the triangle copied across. Once per
//    hierarchy; the V-cycle then applies the inverse with lpb_coarse_solve_*.
#include <cusolverDn.h>

#include <mutex>

#include "lp_common.cuh"

namespace {

// copy the upper triangle (row-major view) onto the lower: a[j][i] = a[i][j] for j > i
__global__ void k_symmetrize_from_upper(double* __restrict__ a, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * n; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / n, j = t % n;
    if (j < i) a[t] = a[j * n + i];
  }
}

cusolverDnHandle_t solver_handle() {
  static std::mutex mu;
  static cusolverDnHandle_t h[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!h[dev] && cusolverDnCreate(&h[dev]) != CUSOLVER_STATUS_SUCCESS) h[dev] = nullptr;
  return h[dev];
}

}  // namespace

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

int lpb_graph_free(void* exec) {
  if (!exec) return LP_OK;
  return cudaGraphExecDestroy((cudaGraphExec_t)exec) == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

// workspace (doubles) lpb_coarse_inverse needs for an n x n matrix; < 0 on failure
long long lpb_coarse_inverse_work(int n) {
  cusolverDnHandle_t h = solver_handle();
  if (!h || n <= 0) return LP_ERR_ARG;
  int l1 = 0, l2 = 0;
  if (cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, nullptr, n, &l1) != CUSOLVER_STATUS_SUCCESS)
    return LP_ERR_LAUNCH;
  if (cusolverDnDpotri_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, nullptr, n, &l2) != CUSOLVER_STATUS_SUCCESS)
    return LP_ERR_LAUNCH;
  return l1 > l2 ? l1 : l2;
}

// a (n x n symmetric positive definite, row-major, float64) -> its inverse, in place, on the
// device; info (two device ints): the factorization's and the inversion's status, 0 when fine
// (info[0] > 0: the leading minor of that order is not positive definite)
int lpb_coarse_inverse(double* a, int n, double* work, long long lwork, int* info, void* stream) {
  cusolverDnHandle_t h = solver_handle();
  if (!h || !a || !work || !info || n <= 0 || lwork <= 0 || lwork > 2147483647LL) return LP_ERR_ARG;
  if (cusolverDnSetStream(h, LP_ST) != CUSOLVER_STATUS_SUCCESS) return LP_ERR_LAUNCH;
  // the row-major symmetric matrix read column-major is itself; the factor and inverse land in
  // the column-major lower triangle, the row-major upper one
  if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, n, a, n, work, (int)lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return LP_ERR_LAUNCH;
  if (cusolverDnDpotri(h, CUBLAS_FILL_MODE_LOWER, n, a, n, work, (int)lwork, info + 1) != CUSOLVER_STATUS_SUCCESS)
    return LP_ERR_LAUNCH;
  const long long nn = (long long)n * n;
  k_symmetrize_from_upper<<<lp_blocks(nn, 256), 256, 0, LP_ST>>>(a, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
