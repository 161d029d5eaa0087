// Level operators of the matrix-free multigrid, node-centric (one output node per thread,
// its eight cells' rows gathered, no scatter and no atomics):
//   out = m * K (m * u) + (1 - m) * u          (loadpath/mg.py:317-346)
// for the three level kinds of the reference hierarchy (loadpath/mg.py:174-199):
//   scaled    K_c = e[c] * ke                   (fine level)
//   weights   K_c = sum_q w[q, c] M_q, or an explicit patch matrix for cells listed in patch_id
//   explicit  K_c stored per cell (24 x 24)
// plus the diagonal of K (loadpath/mg.py:348-371) and the masks / inverse diagonal built from
// it (loadpath/mg.py:537-550, :575-576).
//
// This file holds the general kernels (every level kind, any mask); lp_apply_fine.cu holds the
// tiled fine-level kernel the solver uses on its hot path.
#include "lp_common.cuh"

namespace {

constexpr int KIND_SCALED = 0;
constexpr int KIND_WEIGHTS = 1;
constexpr int KIND_EXPLICIT = 2;

template <typename T>
struct LevelArgs {
  const T* e;          // scaled: cell moduli (cells)
  const T* ke;         // scaled: 24 x 24
  const T* w;          // weights: (8, cells)
  const T* mcat;       // weights: (8, 24, 24)
  const int* patch_id; // weights: per cell, row of patch_k or -1
  const T* patch_k;    // weights: (npatch, 24, 24)
  const T* k;          // explicit: (cells, 24, 24)
};

// gather the 24 (optionally masked) corner dofs of cell (x, y, z)
template <typename T>
__device__ __forceinline__ void gather24(const T* __restrict__ u, const uint8_t* __restrict__ mask, bool mask_in,
                                         const LpGrid& g, int x, int y, int z, T* ue) {
  const long long cs = g.comp_stride();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    long long n = g.node(x + cx_(q), y + cy_(q), z + cz_(q));
    uint8_t mb = mask_in ? mask[n] : (uint8_t)7;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T v = u[c * cs + n];
      ue[3 * q + c] = ((mb >> c) & 1) ? v : T(0);
    }
  }
}

template <typename T, int KIND>
__global__ void k_apply_level(T* __restrict__ out, const T* __restrict__ u, const uint8_t* __restrict__ mask,
                              LpGrid g, LevelArgs<T> a, int mask_in, int finish) {
  extern __shared__ unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  // stage the level's fixed matrices in shared memory
  if (KIND == KIND_SCALED) {
    for (int i = threadIdx.x; i < 576; i += blockDim.x) sm[i] = a.ke[i];
  } else if (KIND == KIND_WEIGHTS) {
    for (int i = threadIdx.x; i < 8 * 576; i += blockDim.x) sm[i] = a.mcat[i];
  }
  __syncthreads();
  const long long total = g.nodes_padded();
  const long long cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    T acc[3] = {T(0), T(0), T(0)};
#pragma unroll 1
    for (int kk = 0; kk < 8; ++kk) {
      // the cell that has this node as its corner kk
      int cx = x - cx_(kk), cy = y - cy_(kk), cz = z - cz_(kk);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      long long c = g.cell(cx, cy, cz);
      T ue[24];
      gather24<T>(u, mask, mask_in != 0, g, cx, cy, cz, ue);
      if (KIND == KIND_SCALED) {
        T ec = a.e[c];
        if (ec == T(0)) continue;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T* row = sm + (3 * kk + i) * 24;
          T s = T(0);
#pragma unroll
          for (int j = 0; j < 24; ++j) s += row[j] * ue[j];
          acc[i] += ec * s;
        }
      } else if (KIND == KIND_WEIGHTS) {
        int p = a.patch_id ? a.patch_id[c] : -1;
        if (p >= 0) {
          const T* kp = a.patch_k + (long long)p * 576;
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const T* row = kp + (3 * kk + i) * 24;
            T s = T(0);
#pragma unroll
            for (int j = 0; j < 24; ++j) s += row[j] * ue[j];
            acc[i] += s;
          }
        }
        const long long cstride = g.cells_padded();
#pragma unroll 1
        for (int q = 0; q < 8; ++q) {
          T wq = a.w[q * cstride + c];
          if (wq == T(0)) continue;
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const T* row = sm + q * 576 + (3 * kk + i) * 24;
            T s = T(0);
#pragma unroll
            for (int j = 0; j < 24; ++j) s += row[j] * ue[j];
            acc[i] += wq * s;
          }
        }
      } else {
        const T* kc = a.k + c * 576;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T* row = kc + (3 * kk + i) * 24;
          T s = T(0);
#pragma unroll
          for (int j = 0; j < 24; ++j) s += row[j] * ue[j];
          acc[i] += s;
        }
      }
    }
    long long n = g.node(x, y, z);
    uint8_t mb = mask ? mask[n] : (uint8_t)7;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T v = acc[i];
      if (finish) {
        T m = ((mb >> i) & 1) ? T(1) : T(0);
        v = v * m + (T(1) - m) * u[i * cs + n];
      }
      out[i * cs + n] = v;
    }
  }
}

template <typename T, int KIND>
int launch_apply(T* out, const T* u, const uint8_t* mask, LpGrid g, LevelArgs<T> a, int mask_in, int finish,
                 cudaStream_t st) {
  if (!lp_grid_ok(g) || !out || !u) return LP_ERR_ARG;
  size_t smem = KIND == KIND_SCALED ? 576 * sizeof(T) : KIND == KIND_WEIGHTS ? 8 * 576 * sizeof(T) : 0;
  if (smem > 48 * 1024) {
    cudaFuncSetAttribute(k_apply_level<T, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  long long total = g.nodes_padded();
  int threads = 256;
  int blocks = lp_blocks(total, threads);
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_apply_level<T, KIND><<<blocks, threads, smem, st>>>(out, u, mask, g, a, mask_in, finish);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// diagonal of the unmasked K, float64 (3, nodes)
template <typename T, int KIND>
__global__ void k_diag_level(double* __restrict__ d, LpGrid g, LevelArgs<T> a) {
  const long long total = g.nodes_padded();
  const long long cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int kk = 0; kk < 8; ++kk) {
      int cx = x - cx_(kk), cy = y - cy_(kk), cz = z - cz_(kk);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      long long c = g.cell(cx, cy, cz);
      for (int i = 0; i < 3; ++i) {
        int dd = (3 * kk + i) * 25;
        double v;
        if (KIND == KIND_SCALED) {
          v = (double)a.ke[dd] * (double)a.e[c];
        } else if (KIND == KIND_WEIGHTS) {
          v = 0.0;
          for (int q = 0; q < 8; ++q) v += (double)a.mcat[q * 576 + dd] * (double)a.w[q * g.cells_padded() + c];
          int p = a.patch_id ? a.patch_id[c] : -1;
          if (p >= 0) v += (double)a.patch_k[(long long)p * 576 + dd];
        } else {
          v = (double)a.k[c * 576 + dd];
        }
        acc[i] += v;
      }
    }
    long long n = g.node(x, y, z);
    for (int i = 0; i < 3; ++i) d[i * cs + n] = acc[i];
  }
}

template <typename T, int KIND>
int launch_diag(double* d, LpGrid g, LevelArgs<T> a, cudaStream_t st) {
  if (!lp_grid_ok(g) || !d) return LP_ERR_ARG;
  long long total = g.nodes_padded();
  k_diag_level<T, KIND><<<lp_blocks(total, 256), 256, 0, st>>>(d, g, a);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// masks and inverse diagonal from the diagonal:
//   alive = d > alive_thr;  live = d > live_thr
//   solved = live & ~held (held from held_bits) ; strict: also & kept >= 1
//   dinv = solved ? 1 / d : 1
// With thr_scale given (a device scalar, the level's largest diagonal), both thresholds are
// relative: thr * max(*thr_scale, 1e-300) (loadpath/mg.py:565-567), so no host read is needed.
__global__ void k_masks(uint8_t* __restrict__ mask, double* __restrict__ dinv64, float* __restrict__ dinv32,
                        const double* __restrict__ d, const uint8_t* __restrict__ held_bits,
                        const float* __restrict__ kept, LpGrid g, double alive_thr, double live_thr,
                        const double* __restrict__ thr_scale) {
  if (thr_scale) {
    const double sc = fmax(*thr_scale, 1e-300);
    alive_thr *= sc;
    live_thr *= sc;
  }
  const long long total = g.nodes_padded();
  const long long cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    long long n = g.node(x, y, z);
    uint8_t hb = held_bits ? held_bits[n] : 0;
    uint8_t mb = 0;
    for (int i = 0; i < 3; ++i) {
      double di = d[i * cs + n];
      bool alive = di > alive_thr;
      bool live = di > live_thr;
      bool solved = live && !((hb >> i) & 1);
      if (kept) solved = solved && kept[i * cs + n] >= 1.0f;
      if (alive) mb |= (uint8_t)(8u << i);
      if (solved) mb |= (uint8_t)(1u << i);
      double inv = solved ? 1.0 / (live ? di : 1.0) : 1.0;
      if (dinv64) dinv64[i * cs + n] = inv;
      if (dinv32) dinv32[i * cs + n] = (float)inv;
    }
    mask[n] = mb;
  }
}

// max of a float64 array (one block per slice; partials then a final pass on the host side
// of the caller, which reads back one value per block)
__global__ void k_max_abs_diff_partial(const double* __restrict__ a, const double* __restrict__ b, long long n,
                                       double* __restrict__ part) {
  __shared__ double sh[32];
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(a[i] - b[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) part[blockIdx.x] = m;
  }
}

__global__ void k_max_partial(const double* __restrict__ a, long long n, double* __restrict__ part) {
  __shared__ double sh[32];
  double m = -1e308;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, a[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : -1e308;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) part[blockIdx.x] = m;
  }
}

__global__ void k_max_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double m = -1e308;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, part[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : -1e308;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) *out = m;
  }
}


// ---- active-cell and mismatch counts (loadpath/mg.py:559, :593-599), into device scalars --
// Each block writes a partial count, one block adds them in order: exact integer sums in
// float64, the same bits every run, and no host read between the kernels that need them.
#define LP_COUNT_BLOCKS 592

__device__ __forceinline__ void lp_count_store(double c, double* part) {
  __shared__ double sh[32];
  c = lp_block_sum(c, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = c;
}

// cells with modulus > 0 (all padded cells; the padding holds zeros)
__global__ void k_count_pos(const double* __restrict__ e, long long n, double* __restrict__ part) {
  double c = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += e[i] > 0.0 ? 1.0 : 0.0;
  lp_count_store(c, part);
}

// level-1 cells with a non-zero child weight or a patch matrix
template <typename T>
__global__ void k_count_weights(const T* __restrict__ w, const int* __restrict__ patch_id, LpGrid g,
                                double* __restrict__ part) {
  const long long ncp = g.cells_padded();
  double c = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncp;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    const long long cell = t;
    bool act = patch_id && patch_id[cell] >= 0;
    for (int k = 0; k < 8 && !act; ++k) act = w[k * ncp + cell] != T(0);
    c += act ? 1.0 : 0.0;
  }
  lp_count_store(c, part);
}

// explicit-level cells whose 24 x 24 matrix has a non-zero entry; one warp per cell
template <typename T>
__global__ void k_count_explicit(const T* __restrict__ k, LpGrid g, double* __restrict__ part) {
  const long long total = g.cells_padded();
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  double c = 0.0;
  for (long long t = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); t < total; t += warps) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    const T* kc = k + t * 576;
    bool nz = false;
    for (int i = lane; i < 576; i += 32) nz = nz || kc[i] != T(0);
    if (__any_sync(0xffffffffu, nz) && lane == 0) c += 1.0;
  }
  lp_count_store(c, part);
}

// positions where two byte arrays differ
__global__ void k_count_ne_u8(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, long long n,
                              double* __restrict__ part) {
  double c = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += a[i] != b[i] ? 1.0 : 0.0;
  lp_count_store(c, part);
}

__global__ void k_count_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)

extern "C" {

int lpb_apply_scaled_f32(float* out, const float* u, const float* e, const uint8_t* mask, const float* ke,
                         LP_GRID_ARGS, int mask_in, int finish, void* stream) {
  LevelArgs<float> a{};
  a.e = e; a.ke = ke;
  if (!e || !ke) return LP_ERR_ARG;
  return launch_apply<float, KIND_SCALED>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_apply_scaled_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* ke,
                         LP_GRID_ARGS, int mask_in, int finish, void* stream) {
  LevelArgs<double> a{};
  a.e = e; a.ke = ke;
  if (!e || !ke) return LP_ERR_ARG;
  return launch_apply<double, KIND_SCALED>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_apply_weights_f32(float* out, const float* u, const float* w, const float* mcat, const int* patch_id,
                          const float* patch_k, const uint8_t* mask, LP_GRID_ARGS, int mask_in, int finish,
                          void* stream) {
  LevelArgs<float> a{};
  a.w = w; a.mcat = mcat; a.patch_id = patch_id; a.patch_k = patch_k;
  if (!w || !mcat) return LP_ERR_ARG;
  return launch_apply<float, KIND_WEIGHTS>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_apply_weights_f64(double* out, const double* u, const double* w, const double* mcat, const int* patch_id,
                          const double* patch_k, const uint8_t* mask, LP_GRID_ARGS, int mask_in, int finish,
                          void* stream) {
  LevelArgs<double> a{};
  a.w = w; a.mcat = mcat; a.patch_id = patch_id; a.patch_k = patch_k;
  if (!w || !mcat) return LP_ERR_ARG;
  return launch_apply<double, KIND_WEIGHTS>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_apply_explicit_f32(float* out, const float* u, const float* k, const uint8_t* mask, LP_GRID_ARGS,
                           int mask_in, int finish, void* stream) {
  LevelArgs<float> a{};
  a.k = k;
  if (!k) return LP_ERR_ARG;
  return launch_apply<float, KIND_EXPLICIT>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_apply_explicit_f64(double* out, const double* u, const double* k, const uint8_t* mask, LP_GRID_ARGS,
                           int mask_in, int finish, void* stream) {
  LevelArgs<double> a{};
  a.k = k;
  if (!k) return LP_ERR_ARG;
  return launch_apply<double, KIND_EXPLICIT>(out, u, mask, LP_GRID, a, mask_in, finish, (cudaStream_t)stream);
}

int lpb_diag_scaled_f64(double* d, const double* e, const double* ke, LP_GRID_ARGS, void* stream) {
  LevelArgs<double> a{};
  a.e = e; a.ke = ke;
  return launch_diag<double, KIND_SCALED>(d, LP_GRID, a, (cudaStream_t)stream);
}

int lpb_diag_weights_f32(double* d, const float* w, const float* mcat, const int* patch_id, const float* patch_k,
                         LP_GRID_ARGS, void* stream) {
  LevelArgs<float> a{};
  a.w = w; a.mcat = mcat; a.patch_id = patch_id; a.patch_k = patch_k;
  return launch_diag<float, KIND_WEIGHTS>(d, LP_GRID, a, (cudaStream_t)stream);
}

int lpb_diag_weights_f64(double* d, const double* w, const double* mcat, const int* patch_id, const double* patch_k,
                         LP_GRID_ARGS, void* stream) {
  LevelArgs<double> a{};
  a.w = w; a.mcat = mcat; a.patch_id = patch_id; a.patch_k = patch_k;
  return launch_diag<double, KIND_WEIGHTS>(d, LP_GRID, a, (cudaStream_t)stream);
}

int lpb_diag_explicit_f64(double* d, const double* k, LP_GRID_ARGS, void* stream) {
  LevelArgs<double> a{};
  a.k = k;
  return launch_diag<double, KIND_EXPLICIT>(d, LP_GRID, a, (cudaStream_t)stream);
}

int lpb_diag_explicit_f32(double* d, const float* k, LP_GRID_ARGS, void* stream) {
  LevelArgs<float> a{};
  a.k = k;
  return launch_diag<float, KIND_EXPLICIT>(d, LP_GRID, a, (cudaStream_t)stream);
}

int lpb_masks(uint8_t* mask, double* dinv64, float* dinv32, const double* d, const uint8_t* held_bits,
              const float* kept, LP_GRID_ARGS, double alive_thr, double live_thr, const double* thr_scale,
              void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !mask || !d) return LP_ERR_ARG;
  long long total = g.nodes_padded();
  k_masks<<<lp_blocks(total, 256), 256, 0, (cudaStream_t)stream>>>(mask, dinv64, dinv32, d, held_bits, kept, g,
                                                                   alive_thr, live_thr, thr_scale);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// max over n doubles into *out (device); part: scratch of at least 1024 doubles
int lpb_max_f64(const double* a, long long n, double* part, double* out, void* stream) {
  if (!a || !part || !out || n < 0) return LP_ERR_ARG;
  int blocks = lp_blocks(n, 256);
  if (blocks > 1024) blocks = 1024;
  k_max_partial<<<blocks, 256, 0, (cudaStream_t)stream>>>(a, n, part);
  k_max_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, blocks, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// max |a - b| over n doubles into *out (device; 0 for n = 0); part: scratch of at least 1024 doubles
int lpb_max_abs_diff_f64(const double* a, const double* b, long long n, double* part, double* out, void* stream) {
  if (!a || !b || !part || !out || n < 0) return LP_ERR_ARG;
  int blocks = lp_blocks(n, 256);
  if (blocks > 1024) blocks = 1024;
  k_max_abs_diff_partial<<<blocks, 256, 0, (cudaStream_t)stream>>>(a, b, n, part);
  k_max_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, blocks, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// ---- counts into a device scalar; part: scratch of at least 592 doubles ----------------
int lpb_count_positive_f64(const double* e, long long n, double* part, double* out, void* stream) {
  if (!e || !part || !out || n < 0) return LP_ERR_ARG;
  k_count_pos<<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(e, n, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_count_active_weights_f32(const float* w, const int* patch_id, LP_GRID_ARGS, double* part, double* out,
                                 void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !w || !part || !out) return LP_ERR_ARG;
  k_count_weights<float><<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(w, patch_id, g, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_count_active_weights_f64(const double* w, const int* patch_id, LP_GRID_ARGS, double* part, double* out,
                                 void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !w || !part || !out) return LP_ERR_ARG;
  k_count_weights<double><<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(w, patch_id, g, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_count_active_explicit_f32(const float* k, LP_GRID_ARGS, double* part, double* out, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !k || !part || !out) return LP_ERR_ARG;
  k_count_explicit<float><<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(k, g, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_count_active_explicit_f64(const double* k, LP_GRID_ARGS, double* part, double* out, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !k || !part || !out) return LP_ERR_ARG;
  k_count_explicit<double><<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(k, g, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_count_ne_u8(const uint8_t* a, const uint8_t* b, long long n, double* part, double* out, void* stream) {
  if (!a || !b || !part || !out || n < 0) return LP_ERR_ARG;
  k_count_ne_u8<<<LP_COUNT_BLOCKS, 256, 0, (cudaStream_t)stream>>>(a, b, n, part);
  k_count_final<<<1, 1024, 0, (cudaStream_t)stream>>>(part, LP_COUNT_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
