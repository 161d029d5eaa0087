// Cell stresses of the minimum-mass loop under a stress limit (loadpath/constrained.py:597-652,
// STRESS_POINTS = "corners"): for every cell that moved (a corner node with a nonzero
// displacement) and is counted (touches no support and no load), the stress C B_k u_e at its 8
// corners from the unit-modulus displacement u, the von Mises value vm = sqrt(s . VM s) and the
// relaxed ratio r = xe * vm / limit (q = 1). Three passes over the cells, each forming the
// corner stresses again from u:
//   mode 0: the largest r (partial maxima per block);
//   mode 1: partial sums of (r / sc)^8, sc the largest r (the P-mean's scaled sum, P = 8);
//   mode 2: per cell the explicit gradient g = sum_k w_k vm_k / limit and the 24-vector
//           sum_k w_k xe / (vm_k limit) B_k^T C VM s_k the adjoint right-hand side gathers, with
//           w_k = kappa (r_k / pm)^7 / nc (zero on cells that are not active).
// lpb_cell_vectors_to_nodes then sums each node's share of its cells' 24-vectors (the
// transpose of the corner gather). Float64 throughout.
#include "lp_common.cuh"

namespace {

constexpr int ST_THREADS = 128;
constexpr int ST_BLOCKS = 1184;   // 148 SMs x 8

__device__ __forceinline__ void st_corner(const double* __restrict__ cb, const double (&ue)[24], double (&sig)[6],
                                          double (&sv)[6], double& vm) {
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 24; ++j) s += cb[i * 24 + j] * ue[j];
    sig[i] = s;
  }
  // VM (loadpath/constrained.py:107-114) applied to sig
  sv[0] = sig[0] - 0.5 * sig[1] - 0.5 * sig[2];
  sv[1] = -0.5 * sig[0] + sig[1] - 0.5 * sig[2];
  sv[2] = -0.5 * sig[0] - 0.5 * sig[1] + sig[2];
  sv[3] = 3.0 * sig[3];
  sv[4] = 3.0 * sig[4];
  sv[5] = 3.0 * sig[5];
  double q = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) q += sv[i] * sig[i];
  vm = sqrt(fmax(q, 1e-30));
}

template <int MODE>
__global__ void __launch_bounds__(ST_THREADS) k_stress_pass(const double* __restrict__ u,
                                                            const double* __restrict__ xe,
                                                            const uint8_t* __restrict__ counted,
                                                            const double* __restrict__ cb_g, double lim, double sc,
                                                            double pm, double kappa, double nc, LpGrid g,
                                                            double* __restrict__ part, double* __restrict__ gxe,
                                                            double* __restrict__ fe) {
  __shared__ double cb[8 * 6 * 24];
  __shared__ double sh[32];
  __shared__ double sfv[MODE == 2 ? ST_THREADS * 25 : 1];
  for (int i = threadIdx.x; i < 8 * 6 * 24; i += blockDim.x) cb[i] = cb_g[i];
  __syncthreads();
  const long long total = g.cells_padded();
  const long long cs = g.comp_stride();
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    double ue[24];
    bool moved = false;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long nd = g.node(x + (q & 1), y + ((q >> 1) & 1), z + ((q >> 2) & 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ue[3 * q + c] = u[c * cs + nd];
        moved |= ue[3 * q + c] != 0.0;
      }
    }
    const bool act = moved && counted[t] != 0;
    if constexpr (MODE == 2) {
      // the cell's 24-vector accumulates in this thread's row of shared memory
      double* fv = sfv + threadIdx.x * 25;
      double gx = 0.0;
      for (int j = 0; j < 24; ++j) fv[j] = 0.0;
      if (act) {
        const double xa = xe[t];
#pragma unroll 1
        for (int k = 0; k < 8; ++k) {
          double sig[6], sv[6], vm;
          st_corner(cb + k * 144, ue, sig, sv, vm);
          const double r = xa * vm / lim;
          const double tt = r / fmax(pm, 1e-30);
          const double t2 = tt * tt, t4 = t2 * t2;
          const double w = kappa * (t4 * t2 * tt) / nc;
          gx += w * (vm / lim);
          const double coef = w * (xa / (vm * lim));
#pragma unroll 1
          for (int j = 0; j < 24; ++j) {
            double d = 0.0;
#pragma unroll
            for (int i = 0; i < 6; ++i) d += sv[i] * cb[k * 144 + i * 24 + j];
            fv[j] += coef * d;
          }
        }
      }
      gxe[t] = gx;
      for (int j = 0; j < 24; ++j) fe[t * 24 + j] = fv[j];
      continue;
    } else {
    if (!act) continue;
    const double xa = xe[t];
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      double sig[6], sv[6], vm;
      st_corner(cb + k * 144, ue, sig, sv, vm);
      const double r = xa * vm / lim;
      if constexpr (MODE == 0) {
        acc = fmax(acc, r);
      } else {
        const double rr = r / sc, r2 = rr * rr, r4 = r2 * r2;
        acc += r4 * r4;
      }
    }
    }
  }
  if constexpr (MODE == 2) return;
  if constexpr (MODE == 0) {
    for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
      acc = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) acc = fmax(acc, __shfl_down_sync(0xffffffffu, acc, o));
      if (threadIdx.x == 0) part[blockIdx.x] = acc;
    }
  } else {
    acc = lp_block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
  }
}

// the max (mode 0) or the sum (mode 1) of the block partials
__global__ void k_stress_final(int mode, const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a = mode == 0 ? fmax(a, part[i]) : a + part[i];
  if (mode == 0) {
    for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x < 32) {
      a = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
      if (threadIdx.x == 0) *out = a;
    }
  } else {
    a = lp_block_sum(a, sh);
    if (threadIdx.x == 0) *out = a;
  }
}

// out (node field, all three components) = each node's share of its cells' 24-vectors fe
// (cells_padded x 24, dof 3 q + component at corner q = (q & 1, q >> 1 & 1, q >> 2 & 1))
__global__ void k_cell_vectors_to_nodes(double* __restrict__ out, const double* __restrict__ fe, LpGrid g) {
  const long long total = g.nodes_padded();
  const long long cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int cx = x - (q & 1), cy = y - ((q >> 1) & 1), cz = z - ((q >> 2) & 1);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      const double* f = fe + g.cell(cx, cy, cz) * 24 + 3 * q;
      s0 += f[0];
      s1 += f[1];
      s2 += f[2];
    }
    out[t] = s0;
    out[cs + t] = s1;
    out[2 * cs + t] = s2;
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)

extern "C" {

// one stress pass (see above); u: float64 node field; xe: float64 cell field; counted: uint8
// cell field (nonzero: counted); cb: 8 x 6 x 24 float64 (device), corners x outermost;
// mode 0 / 1: *out = the largest ratio / the scaled sum (part: ST_BLOCKS doubles);
// mode 2: gxe (cell field) and fe (cells_padded x 24 doubles)
int lpb_stress_pass(int mode, const double* u, const double* xe, const uint8_t* counted, const double* cb,
                    double lim, double sc, double pm, double kappa, double nc, double* part, double* out,
                    double* gxe, double* fe, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !u || !xe || !counted || !cb || !(lim > 0.0) || mode < 0 || mode > 2) return LP_ERR_ARG;
  if (mode < 2 && (!part || !out)) return LP_ERR_ARG;
  if (mode == 1 && !(sc > 0.0)) return LP_ERR_ARG;
  if (mode == 2 && (!gxe || !fe || !(nc > 0.0))) return LP_ERR_ARG;
  if (mode == 0)
    k_stress_pass<0><<<ST_BLOCKS, ST_THREADS, 0, LP_ST>>>(u, xe, counted, cb, lim, sc, pm, kappa, nc, g, part, gxe, fe);
  else if (mode == 1)
    k_stress_pass<1><<<ST_BLOCKS, ST_THREADS, 0, LP_ST>>>(u, xe, counted, cb, lim, sc, pm, kappa, nc, g, part, gxe, fe);
  else
    k_stress_pass<2><<<ST_BLOCKS, ST_THREADS, 0, LP_ST>>>(u, xe, counted, cb, lim, sc, pm, kappa, nc, g, part, gxe, fe);
  if (mode < 2) k_stress_final<<<1, 1024, 0, LP_ST>>>(mode, part, ST_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out (float64 node field) = the nodes' sums of the cells' 24-vectors fe; padding left as it was
int lpb_cell_vectors_to_nodes(double* out, const double* fe, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !fe) return LP_ERR_ARG;
  k_cell_vectors_to_nodes<<<lp_blocks(g.nodes_padded(), 256), 256, 0, LP_ST>>>(out, fe, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
