// Shared definitions for the loadpath_b200 CUDA kernels (sm_100a).
//
// Layouts (all C order). A level's z extent is cut into chunks of four planes, and the chunk
// index is the slowest axis, so one chunk's four planes of a row of x are contiguous:
//   node field  (3, PZ/4, NY, NX, 4)   NX = nx + 1, NY = ny + 1, PZ >= nz + 1, PZ % 4 == 0
//   cell field  (CPZ/4, ny, nx, 4)     CPZ >= nz, CPZ % 4 == 0
//   node mask   (PZ/4, NY, NX, 4) uint8: bits 0..2 = dof is solved for (alive and not held) per
//               component; bits 3..5 = dof carries stiffness (alive) per component.
// Node (x, y, z) sits at ((z / 4 * NY + y) * NX + x) * 4 + z % 4 of its component; a tile of
// node columns moves as rows of 16 * (x extent) bytes, and the z padding (z > nz for nodes,
// z >= nz for cells) holds zeros.
// Corner k of a cell sits at (k & 1, k >> 1 & 1, k >> 2 & 1); a cell's 24 dofs are ordered
// 3 * corner + component (loadpath/fem.py:30, loadpath/fem.py:127-145).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LP_OK 0
#define LP_ERR_ARG -1
#define LP_ERR_LAUNCH -2
#define LP_ERR_SIZE -3

struct LpGrid {
  int nx, ny, nz;   // cells
  int pz;           // node z pitch
  int cpz;          // cell z pitch
  __host__ __device__ int NX() const { return nx + 1; }
  __host__ __device__ int NY() const { return ny + 1; }
  __host__ __device__ int NZ() const { return nz + 1; }
  __host__ __device__ long long comp_stride() const { return (long long)(nx + 1) * (ny + 1) * pz; }
  __host__ __device__ long long node(int x, int y, int z) const {
    return (((long long)(z >> 2) * (ny + 1) + y) * (nx + 1) + x) * 4 + (z & 3);
  }
  __host__ __device__ long long cell(int x, int y, int z) const {
    return (((long long)(z >> 2) * ny + y) * nx + x) * 4 + (z & 3);
  }
  // index step from one z chunk of a column to the next
  __host__ __device__ long long node_zc_stride() const { return 4LL * (nx + 1) * (ny + 1); }
  __host__ __device__ long long cell_zc_stride() const { return 4LL * nx * ny; }
  __host__ __device__ long long nodes_padded() const { return (long long)(nx + 1) * (ny + 1) * pz; }
  __host__ __device__ long long cells_padded() const { return (long long)nx * ny * cpz; }
  // the node / cell at index t of a field (memory order); false on the z padding. The column
  // index t / 4 is taken in 32-bit unsigned arithmetic (a field of one component holds fewer
  // than 2^34 entries), which divides several times faster than 64-bit.
  __host__ __device__ bool node_at(long long t, int& x, int& y, int& z) const {
    const unsigned r = (unsigned)(t >> 2), NXu = (unsigned)(nx + 1), NYu = (unsigned)(ny + 1);
    const unsigned q = r / NXu, w = q / NYu;
    x = (int)(r - q * NXu);
    y = (int)(q - w * NYu);
    z = 4 * (int)w + (int)(t & 3);
    return z <= nz;
  }
  __host__ __device__ bool cell_at(long long t, int& x, int& y, int& z) const {
    const unsigned r = (unsigned)(t >> 2), nxu = (unsigned)nx, nyu = (unsigned)ny;
    const unsigned q = r / nxu, w = q / nyu;
    x = (int)(r - q * nxu);
    y = (int)(q - w * nyu);
    z = 4 * (int)w + (int)(t & 3);
    return z < nz;
  }
};

static inline LpGrid lp_grid(int nx, int ny, int nz, int pz, int cpz) {
  LpGrid g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.pz = pz; g.cpz = cpz;
  return g;
}

static inline bool lp_grid_ok(const LpGrid& g) {
  return g.nx >= 1 && g.ny >= 1 && g.nz >= 1 && g.pz >= g.nz + 1 && g.cpz >= g.nz && g.pz % 4 == 0 &&
         g.cpz % 4 == 0;
}

// Launch-geometry tuning table (lp_graph.cu): a value set for (knob, grid) by lpb_tune_set, or 0
// when none is (the launcher's own cost model then decides). Knobs: the z-segment length in
// chunks of the fine float32 / float64 apply and of the level-1 float32 / float64 apply.
enum { LP_KNOB_FINE_F32 = 1, LP_KNOB_FINE_F64 = 2, LP_KNOB_L1_F32 = 3, LP_KNOB_L1_F64 = 4, LP_KNOB_MAX = 4 };
int lp_tune_lookup(int knob, int nx, int ny, int nz);

// The degree-2 Chebyshev updates, one definition for the standalone vector kernels and the
// explicit levels' gather that applies them as it forms A u (the same expression, so the same bits)
template <typename T>
__device__ __forceinline__ T lp_cheb2_zero_v(T di, T bi, T adi, T dinvi, T c1, T c2) {
  const T ri = bi - adi;
  return di + (c1 * di + c2 * dinvi * ri);
}
template <typename T>
__device__ __forceinline__ T lp_cheb2_v(T xi, T di, T rin, T adi, T dinvi, T c1, T c2) {
  const T ri = rin - adi;
  return (xi + di) + (c1 * di + c2 * dinvi * ri);
}
template <typename T>
__device__ __forceinline__ void lp_residual_scaled_v(T bi, T axi, T dinvi, T s, T& r, T& d) {
  const T ri = bi - axi;
  r = ri;
  d = s * dinvi * ri;
}

static inline int lp_blocks(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 2147483647LL) b = 2147483647LL;
  return (int)b;
}

// The coarsest level as a band: dofs numbered 3 * node + component, nodes ordered with the
// longest axis slowest (perm[0]) and the shortest fastest (perm[2]); half-bandwidth
// bw = 3 (N1 N2 + N2 + 1) + 2; 32-row tiles, D off-diagonal tiles per tile row.
struct LpBand {
  int perm[3];
  int N1, N2;      // extents of axes perm[1], perm[2]
  long long n;     // 3 * nodes
  int nt, D;       // n padded to 32 * nt
  __host__ __device__ void coords(long long node, int& x, int& y, int& z) const {
    const int p2 = (int)(node % N2);
    const long long q = node / N2;
    const int p1 = (int)(q % N1), p0 = (int)(q / N1);
    int c[3];
    c[perm[0]] = p0;
    c[perm[1]] = p1;
    c[perm[2]] = p2;
    x = c[0];
    y = c[1];
    z = c[2];
  }
};

static inline LpBand lp_band(int NX, int NY, int NZ) {
  const int ext[3] = {NX, NY, NZ};
  LpBand b;
  b.perm[0] = 0; b.perm[1] = 1; b.perm[2] = 2;
  for (int i = 0; i < 3; ++i)          // stable sort of the axes by extent, longest first
    for (int j = 0; j + 1 < 3 - i; ++j)
      if (ext[b.perm[j]] < ext[b.perm[j + 1]]) { int t = b.perm[j]; b.perm[j] = b.perm[j + 1]; b.perm[j + 1] = t; }
  b.N1 = ext[b.perm[1]];
  b.N2 = ext[b.perm[2]];
  b.n = 3LL * NX * NY * NZ;
  b.nt = (int)((b.n + 31) / 32);
  const long long bw = 3LL * ((long long)b.N1 * b.N2 + b.N2 + 1) + 2;
  b.D = (int)((bw + 31) / 32);
  return b;
}

// The work of a launch: units (tile, chunk), tile-major (tile = x tile + gx * y tile), block b
// taking units [b U / B, (b + 1) U / B), so every block has the same number of chunks. A run of
// consecutive chunks [cb, ce) of one tile is a segment; it loads one halo chunk below cb (its top
// cell starts the z carry) and the chunk above ce - 1 (the upper plane of the last cell).
struct LpSeg {
  int tile, cb, ce;
  int cstart, nload, nproc;   // loads from chunk cstart, nload of them; chunks processed
};

__device__ __forceinline__ LpSeg lp_seg(long long u, long long u1, int nchunks) {
  LpSeg s;
  s.tile = (int)(u / nchunks);
  s.cb = (int)(u - (long long)s.tile * nchunks);
  const long long left = u1 - u;
  s.ce = left < (long long)(nchunks - s.cb) ? s.cb + (int)left : nchunks;
  s.cstart = s.cb > 0 ? s.cb - 1 : 0;
  s.nload = min(s.ce + 1, nchunks) - s.cstart;
  s.nproc = s.ce - s.cstart;
  return s;
}

#define LP_LAUNCH_CHECK()                                   \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) return LP_ERR_LAUNCH;            \
  } while (0)

// corner offsets
__host__ __device__ __forceinline__ int cx_(int k) { return k & 1; }
__host__ __device__ __forceinline__ int cy_(int k) { return (k >> 1) & 1; }
__host__ __device__ __forceinline__ int cz_(int k) { return (k >> 2) & 1; }

template <typename T>
__device__ __forceinline__ T lp_ldg(const T* p) { return __ldg(p); }

// Block-wide sum of a double; every thread gets the result. blockDim.x <= 1024.
__device__ __forceinline__ double lp_block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) sh[0] = v;
  __syncthreads();
  double r = sh[0];
  __syncthreads();
  return r;
}
