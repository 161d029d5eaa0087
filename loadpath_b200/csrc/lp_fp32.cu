// The float32-only solve's pieces (loadpath/gpu.py:119-149 `_two_sum` / `_rigid_free`,
// :233-258 `apply_rf`, :429-481 `solve_fp32`): the fine-level operator on a float32 pair
// u = hi + lo, each cell's matrix applied to its rigid-motion-free deformation formed in pair
// arithmetic (K annihilates rigid motion, so K d = K u in exact arithmetic, and nothing large
// is rounded on a slender part), and the pair updates of the iterative refinement.
//
// Error-free sums use __fadd_rn / __fsub_rn so the compiler can neither contract nor reorder them.
#include "lp_common.cuh"

namespace {

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// ft (24, cells): E_c Ke d_c with d_c the cell's corner displacements of (h + l) (both masked by
// the level mask's solved bits) less its corner-0 translation and its mean rotation
__global__ void __launch_bounds__(128) k_rf_cells(float* __restrict__ ft, const float* __restrict__ h,
                                                  const float* __restrict__ l, const uint8_t* __restrict__ mask,
                                                  const float* __restrict__ e, const float* __restrict__ ke, LpGrid g) {
  __shared__ float sk[576];
  for (int i = threadIdx.x; i < 576; i += blockDim.x) sk[i] = ke[i];
  __syncthreads();
  const long long ncp = g.cells_padded(), cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncp; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    const float ec = e[t];
    float s[24], er[24];
    float h0[3], l0[3];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const long long n = g.node(x + cx_(k), y + cy_(k), z + cz_(k));
      const uint8_t mb = mask[n];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const bool on = (mb >> c) & 1;
        const float hv = on ? h[c * cs + n] : 0.0f;
        const float lv = (on && l) ? l[c * cs + n] : 0.0f;
        if (k == 0) {
          h0[c] = hv;
          l0[c] = lv;
        }
        two_sum(hv, -h0[c], s[3 * k + c], er[3 * k + c]);
        er[3 * k + c] = __fadd_rn(er[3 * k + c], __fsub_rn(lv, l0[c]));
      }
    }
    // mean displacement gradient over the cell (cell units), its skew part w
    float gr[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float d = __fadd_rn(s[3 * k + i], er[3 * k + i]);
          const float ca = (((k >> a) & 1) ? 0.5f : -0.5f);
          acc = __fadd_rn(acc, __fmul_rn(ca, d));
        }
        gr[i][a] = 0.5f * acc;
      }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if ((k >> a) & 1)
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const float wia = 0.5f * __fsub_rn(gr[i][a], gr[a][i]);
            float s2, e2;
            two_sum(s[3 * k + i], -wia, s2, e2);
            s[3 * k + i] = s2;
            er[3 * k + i] = __fadd_rn(er[3 * k + i], e2);
          }
    float d[24];
#pragma unroll
    for (int j = 0; j < 24; ++j) d[j] = __fadd_rn(s[j], er[j]);
#pragma unroll 4
    for (int r = 0; r < 24; ++r) {
      float acc = 0.0f;
#pragma unroll
      for (int j = 0; j < 24; ++j) acc += sk[r * 24 + j] * d[j];
      ft[(long long)r * ncp + t] = ec * acc;
    }
  }
}

// out = m * (sum of the node's cells' rows) + (1 - m) * h
__global__ void k_rf_gather(float* __restrict__ out, const float* __restrict__ ft, const float* __restrict__ h,
                            const uint8_t* __restrict__ mask, LpGrid g) {
  const long long total = g.nodes_padded();
  const long long ncp = g.cells_padded(), cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    float a[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int cx = x - cx_(k), cy = y - cy_(k), cz = z - cz_(k);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      const long long c = g.cell(cx, cy, cz);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) a[cc] += ft[(long long)(3 * k + cc) * ncp + c];
    }
    const uint8_t mb = mask[t];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) out[cc * cs + t] = ((mb >> cc) & 1) ? a[cc] : h[cc * cs + t];
  }
}

// r = (bh - ax) + bl
__global__ void k_pair_residual(float* __restrict__ r, const float* __restrict__ bh, const float* __restrict__ ax,
                                const float* __restrict__ bl, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    r[i] = __fadd_rn(__fsub_rn(bh[i], ax[i]), bl[i]);
}

// (xh, xl) += d in pair arithmetic: xh, e = two_sum(xh, d); xl += e; xh, xl = two_sum(xh, xl)
__global__ void k_pair_add(float* __restrict__ xh, float* __restrict__ xl, const float* __restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float s, e;
    two_sum(xh[i], d[i], s, e);
    const float lo = __fadd_rn(xl[i], e);
    float s2, e2;
    two_sum(s, lo, s2, e2);
    xh[i] = s2;
    xl[i] = e2;
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)

extern "C" {

// out = m K (h + l) + (1 - m) h on the fine level with each cell's rigid motion removed in pair
// arithmetic (l may be NULL); e: float32 cell moduli; ke: 24 x 24 float32 (device); ft: caller
// scratch of 24 * cells floats
int lpb_apply_rf_f32(float* out, const float* h, const float* l, const uint8_t* mask, const float* e,
                     const float* ke, float* ft, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !h || !mask || !e || !ke || !ft || out == h || out == l) return LP_ERR_ARG;
  k_rf_cells<<<lp_blocks(g.cells_padded(), 128), 128, 0, LP_ST>>>(ft, h, l, mask, e, ke, g);
  k_rf_gather<<<lp_blocks(g.nodes_padded(), 256), 256, 0, LP_ST>>>(out, ft, h, mask, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_pair_residual_f32(float* r, const float* bh, const float* ax, const float* bl, long long n, void* stream) {
  if (!r || !bh || !ax || !bl || n < 0) return LP_ERR_ARG;
  k_pair_residual<<<lp_blocks(n, 256), 256, 0, LP_ST>>>(r, bh, ax, bl, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_pair_add_f32(float* xh, float* xl, const float* d, long long n, void* stream) {
  if (!xh || !xl || !d || n < 0) return LP_ERR_ARG;
  k_pair_add<<<lp_blocks(n, 256), 256, 0, LP_ST>>>(xh, xl, d, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
