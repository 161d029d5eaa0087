// Live-cell reduction on the device (loadpath/simp.py:263-289 `_connected`, :725 the alive set,
// :795-826 `_solve_mg`): the cells the solve keeps are the alive cells (projected density above
// ALIVE, or an anchor: touching a support or a load, or preserved) 26-connected to an alive cell
// that touches a support; the others get modulus 0 on the fixed grid. The reference labels every
// 26-connected component on the host (scipy.ndimage.label) and keeps the labels found on support
// cells; only that union matters, so here it is a flood fill from those cells.
//
// Cell state bytes: 0 not alive, 1 alive and not (yet) reached, 2 reached. A pass loads an
// 8 x 8 x 8 tile with a one-cell halo into shared memory and spreads 2 over its 1 cells until the
// tile settles (at most 512 sweeps: every sweep that goes on reaches a new cell); passes repeat
// until none changes a cell. States only go from 1 to 2, so a tile that reads a neighbour tile's
// state mid-pass only spreads later, never wrongly.
#include "lp_common.cuh"

namespace {

constexpr int LT = 8;            // tile edge (cells)
constexpr int LH = LT + 2;       // with the halo

// state from the projected density and the cell flags (bit 0: touches a support, bit 1: anchor);
// partial counts of alive cells
__global__ void k_live_seed(uint8_t* __restrict__ state, const double* __restrict__ xp,
                            const uint8_t* __restrict__ flags, double thr, LpGrid g, double* __restrict__ part) {
  __shared__ double sh[32];
  const long long total = g.cells_padded();
  double cnt = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    uint8_t s = 0;
    if (g.cell_at(t, x, y, z)) {
      const uint8_t fl = flags ? flags[t] : 0;
      const bool alive = xp[t] > thr || (fl & 2);
      if (alive) {
        s = (fl & 1) ? 2 : 1;
        cnt += 1.0;
      }
    }
    state[t] = s;
  }
  cnt = lp_block_sum(cnt, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = cnt;
}

// partial counts of the cells alive in state (seeded: nonzero) but not kept in keep (a flooded state: 2)
__global__ void k_live_outside(const uint8_t* __restrict__ state, const uint8_t* __restrict__ keep, LpGrid g,
                               double* __restrict__ part) {
  __shared__ double sh[32];
  const long long total = g.cells_padded();
  double cnt = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x)
    if (state[t] != 0 && keep[t] != 2) cnt += 1.0;
  cnt = lp_block_sum(cnt, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = cnt;
}

__global__ void k_live_count_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

__global__ void __launch_bounds__(LT * LT * LT) k_live_flood(uint8_t* __restrict__ state, LpGrid g,
                                                            int* __restrict__ changed) {
  __shared__ uint8_t s[LH][LH][LH];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * LT - 1, y0 = blockIdx.y * LT - 1, z0 = blockIdx.z * LT - 1;
  for (int e = tid; e < LH * LH * LH; e += blockDim.x) {
    const int ix = e % LH, iy = (e / LH) % LH, iz = e / (LH * LH);
    const int x = x0 + ix, y = y0 + iy, z = z0 + iz;
    const bool in = x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz;
    s[iz][iy][ix] = in ? state[g.cell(x, y, z)] : (uint8_t)0;
  }
  __syncthreads();
  const int lx = 1 + tid % LT, ly = 1 + (tid / LT) % LT, lz = 1 + tid / (LT * LT);
  const bool mine = x0 + lx < g.nx && y0 + ly < g.ny && z0 + lz < g.nz;
  bool any = false;
  for (int sweep = 0; sweep < LT * LT * LT; ++sweep) {
    bool ch = false;
    if (mine && s[lz][ly][lx] == 1) {
      bool hit = false;
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) hit = hit || s[lz + dz][ly + dy][lx + dx] == 2;
      if (hit) {
        s[lz][ly][lx] = 2;
        ch = true;
      }
    }
    any = any || ch;
    if (!__syncthreads_or(ch)) break;
  }
  if (mine && any) state[g.cell(x0 + lx, y0 + ly, z0 + lz)] = 2;
  if (__syncthreads_or(any) && tid == 0) atomicExch(changed, 1);
}

// e_out = e on reached cells, 0 elsewhere
__global__ void k_live_moduli(double* __restrict__ e_out, const double* __restrict__ e,
                              const uint8_t* __restrict__ state, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    e_out[t] = state[t] == 2 ? e[t] : 0.0;
}

// dofs that carry a load but no stiffness (the level-0 mask's alive bits clear)
__global__ void k_dead_loads(const double* __restrict__ f, const uint8_t* __restrict__ mask, LpGrid g,
                             double* __restrict__ part) {
  __shared__ double sh[32];
  const long long nn = g.nodes_padded();
  double cnt = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
    const uint8_t mb = mask[t];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (f[c * nn + t] != 0.0 && !((mb >> (3 + c)) & 1)) cnt += 1.0;
  }
  cnt = lp_block_sum(cnt, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = cnt;
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)
#define LP_LIVE_BLOCKS 592

extern "C" {

// state (uint8 cell field) of every cell; *n_alive = the alive cells; part: 592 doubles
int lpb_live_seed(uint8_t* state, const double* xp, const uint8_t* flags, double alive_thr, double* part,
                  double* n_alive, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !state || !xp || !part || !n_alive) return LP_ERR_ARG;
  k_live_seed<<<LP_LIVE_BLOCKS, 256, 0, LP_ST>>>(state, xp, flags, alive_thr, g, part);
  k_live_count_final<<<1, 1024, 0, LP_ST>>>(part, LP_LIVE_BLOCKS, n_alive);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// one flood pass over all tiles; *changed (device int, caller zeroes it) set when a cell changed
int lpb_live_flood(uint8_t* state, int* changed, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !state || !changed) return LP_ERR_ARG;
  const dim3 grid((g.nx + LT - 1) / LT, (g.ny + LT - 1) / LT, (g.nz + LT - 1) / LT);
  k_live_flood<<<grid, LT * LT * LT, 0, LP_ST>>>(state, g, changed);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_live_moduli(double* e_out, const double* e, const uint8_t* state, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !e_out || !e || !state) return LP_ERR_ARG;
  const long long n = g.cells_padded();
  k_live_moduli<<<lp_blocks(n, 256), 256, 0, LP_ST>>>(e_out, e, state, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// *count = cells alive in a seeded state but outside the kept cells of an earlier flooded state
// (the reference's test for reusing a reduced system, loadpath/simp.py:295); padding cells are 0
// in both
int lpb_live_outside(const uint8_t* state, const uint8_t* keep, double* part, double* count, LP_GRID_ARGS,
                     void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !state || !keep || !part || !count) return LP_ERR_ARG;
  k_live_outside<<<LP_LIVE_BLOCKS, 256, 0, LP_ST>>>(state, keep, g, part);
  k_live_count_final<<<1, 1024, 0, LP_ST>>>(part, LP_LIVE_BLOCKS, count);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// *count = loaded dofs (f float64 node field) without stiffness (mask: the level-0 node mask)
int lpb_dead_loads(const double* f, const uint8_t* mask, double* part, double* count, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !f || !mask || !part || !count) return LP_ERR_ARG;
  k_dead_loads<<<LP_LIVE_BLOCKS, 256, 0, LP_ST>>>(f, mask, g, part);
  k_live_count_final<<<1, 1024, 0, LP_ST>>>(part, LP_LIVE_BLOCKS, count);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
