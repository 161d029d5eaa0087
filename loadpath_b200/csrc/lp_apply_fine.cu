// Fine-level operator on the hot path: out = m * K(E) u + (1 - m) * u for u that is zero on
// masked dofs (every vector the solver makes), K = sum_cells E_c Ke
// (loadpath/mg.py:317-346 -> loadpath/mgops.py:86-103 + :181-217 with finish).
//
// Corner-parity basis. A cell's eight corner values of one component, rewritten in the modes
// {1, sx, sy, sxsy, sz, sxsz, sysz, sxsysz} (s = +-1 per axis), turn the 24 x 24 element matrix
// into one with 45 non-zeros (for the plain and the incompatible-mode brick alike, any
// isotropic nu): three decoupled blocks (linear, bilinear and trilinear modes). The transforms
// are sums and differences, so a cell costs about 190 flops instead of the dense 1152, which
// brings the operator under the HBM roofline on CUDA cores.
//
// Work layout. A block owns a 15 x 15 patch of node columns and runs 16 x 16 threads, one per
// cell column of the patch plus a one-cell halo on the low x and y sides. Each thread marches
// its column along z four cells at a time: it loads four z-planes of its four node columns
// with 16-byte loads (and the fifth plane with a scalar load), forms per plane the x-y modes
// (4 per component), combines consecutive
// planes into the cell's z modes, applies E_c K^ in the modal basis and transforms back to
// the cell's two faces. A node plane's modal force is the upper face of the cell below plus
// the lower face of the cell above, both in this thread, so z needs no exchange; the four cell
// columns around a node column exchange their corner forces through shared memory.
// No atomics, no scatter: every output is written once by its owner.
//
// Requirements (checked by the host entry): pz % 4 == 0 and cpz == pz; u, e and the mask
// hold zeros in the z padding; u is zero on dofs whose mask bit is 0, so the identity rows
// (1 - m) u of the masked operator vanish and the kernel writes m * K u.
#include "lp_common.cuh"

namespace {

constexpr int TXC = 16;   // cell columns per block in x (15 owned node columns)
constexpr int TYC = 16;   // in y

template <typename T>
struct KModal {
  T c[45];
};

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  static __device__ __forceinline__ void load(const float* p, float (&v)[4]) {
    float4 a = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  static __device__ __forceinline__ void store(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct Vec4<double> {
  static __device__ __forceinline__ void load(const double* p, double (&v)[4]) {
    double2 a = __ldg(reinterpret_cast<const double2*>(p));
    double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  static __device__ __forceinline__ void store(double* p, const double (&v)[4]) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
  }
};

// f = K^ v on the 21 non-constant modes (index 3 * mode + component, mode = mx + 2 my + 4 mz);
// the pattern is fixed, the 45 values come from lpb_modal_ke
template <typename T>
__device__ __forceinline__ void modal_product(const KModal<T>& km, const T (&v)[24], T (&f)[24]) {
  f[0] = f[1] = f[2] = T(0);
  f[3] = km.c[0] * v[3] + km.c[1] * v[7] + km.c[2] * v[14];
  f[4] = km.c[3] * v[4] + km.c[4] * v[6];
  f[5] = km.c[5] * v[5] + km.c[6] * v[12];
  f[6] = km.c[7] * v[4] + km.c[8] * v[6];
  f[7] = km.c[9] * v[3] + km.c[10] * v[7] + km.c[11] * v[14];
  f[8] = km.c[12] * v[8] + km.c[13] * v[13];
  f[9] = km.c[14] * v[9] + km.c[15] * v[20];
  f[10] = km.c[16] * v[10] + km.c[17] * v[17];
  f[11] = km.c[18] * v[11] + km.c[19] * v[16] + km.c[20] * v[18];
  f[12] = km.c[21] * v[5] + km.c[22] * v[12];
  f[13] = km.c[23] * v[8] + km.c[24] * v[13];
  f[14] = km.c[25] * v[3] + km.c[26] * v[7] + km.c[27] * v[14];
  f[15] = km.c[28] * v[15] + km.c[29] * v[19];
  f[16] = km.c[30] * v[11] + km.c[31] * v[16] + km.c[32] * v[18];
  f[17] = km.c[33] * v[10] + km.c[34] * v[17];
  f[18] = km.c[35] * v[11] + km.c[36] * v[16] + km.c[37] * v[18];
  f[19] = km.c[38] * v[15] + km.c[39] * v[19];
  f[20] = km.c[40] * v[9] + km.c[41] * v[20];
  f[21] = km.c[42] * v[21];
  f[22] = km.c[43] * v[22];
  f[23] = km.c[44] * v[23];
}

template <typename T>
__global__ void __launch_bounds__(TXC * TYC, 1)
k_apply_fine(T* __restrict__ out, const T* __restrict__ u, const T* __restrict__ e,
             const uint8_t* __restrict__ mask, const KModal<T> km, LpGrid g) {
  // corner forces for the neighbours: [corner 10/01/11][component][plane][thread]
  extern __shared__ unsigned char smem_raw[];
  T(*red)[3][4][TXC * TYC] = reinterpret_cast<T(*)[3][4][TXC * TYC]>(smem_raw);
  const int tid = threadIdx.x;
  const int i = tid % TXC, j = tid / TXC;
  const int x0 = blockIdx.x * (TXC - 1), y0 = blockIdx.y * (TYC - 1);
  const int cx = x0 - 1 + i, cy = y0 - 1 + j;  // this thread's cell column = its owned node column
  const int NX = g.NX(), NY = g.NY();
  const long long cs = g.comp_stride();
  const bool cell_ok = cx >= 0 && cx < g.nx && cy >= 0 && cy < g.ny;
  const bool own = i >= 1 && j >= 1 && cx < NX && cy < NY;
  bool col_ok[4];
  long long col_base[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int nx_ = cx + (q & 1), ny_ = cy + (q >> 1);
    col_ok[q] = nx_ >= 0 && nx_ < NX && ny_ >= 0 && ny_ < NY;
    col_base[q] = col_ok[q] ? g.node(nx_, ny_, 0) : 0;
  }
  const long long ebase = cell_ok ? g.cell(cx, cy, 0) : 0;
  const long long obase = own ? g.node(cx, cy, 0) : 0;

  T up_carry[4][3];    // upper-face modal force of the cell below this chunk
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) up_carry[q][c] = T(0);

  for (int z = 0; z < g.pz; z += 4) {
    // ---- planes z..z+3 of the four node columns (16-byte loads) and plane z+4 (scalar)
    T un[4][3][5];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T v4[4];
        if (col_ok[q]) {
          Vec4<T>::load(u + c * cs + col_base[q] + z, v4);
        } else {
          v4[0] = v4[1] = v4[2] = v4[3] = T(0);
        }
        un[q][c][0] = v4[0]; un[q][c][1] = v4[1]; un[q][c][2] = v4[2]; un[q][c][3] = v4[3];
        un[q][c][4] = (col_ok[q] && z + 4 < g.pz) ? __ldg(u + c * cs + col_base[q] + z + 4) : T(0);
      }
    T ev[4];
    if (cell_ok) {
      Vec4<T>::load(e + ebase + z, ev);
    } else {
      ev[0] = ev[1] = ev[2] = ev[3] = T(0);
    }
    // x-y modes of plane z
    T a_lo[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T u00 = un[0][c][0], u10 = un[1][c][0], u01 = un[2][c][0], u11 = un[3][c][0];
      T sx0 = u00 + u10, dx0 = u10 - u00, sx1 = u01 + u11, dx1 = u11 - u01;
      a_lo[0][c] = sx0 + sx1;
      a_lo[1][c] = dx0 + dx1;
      a_lo[2][c] = sx1 - sx0;
      a_lo[3][c] = dx1 - dx0;
    }
    // ---- cells z .. z+3: lower plane z+t, upper plane z+t+1
    T own_f[4][3];  // corner-00 force of this thread's cell column on node planes z..z+3
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      T a_hi[4][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T u00 = un[0][c][t + 1], u10 = un[1][c][t + 1], u01 = un[2][c][t + 1], u11 = un[3][c][t + 1];
        T sx0 = u00 + u10, dx0 = u10 - u00, sx1 = u01 + u11, dx1 = u11 - u01;
        a_hi[0][c] = sx0 + sx1;
        a_hi[1][c] = dx0 + dx1;
        a_hi[2][c] = sx1 - sx0;
        a_hi[3][c] = dx1 - dx0;
      }
      const T ec = ev[t];
      T v[24], f[24];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T lo = a_lo[q][c], hi = a_hi[q][c];
          v[3 * q + c] = (lo + hi) * ec;
          v[3 * (q + 4) + c] = (hi - lo) * ec;
        }
      modal_product<T>(km, v, f);
      // node plane z+t: upper face of the cell below + lower face of this cell
      T fp[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T f0 = f[3 * q + c], f1 = f[3 * (q + 4) + c];
          fp[q][c] = up_carry[q][c] + (f0 - f1);
          up_carry[q][c] = f0 + f1;
          a_lo[q][c] = a_hi[q][c];
        }
      // back to the four corner columns
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T t0 = fp[0][c] - fp[2][c], t1 = fp[1][c] - fp[3][c];
        T t2 = fp[0][c] + fp[2][c], t3 = fp[1][c] + fp[3][c];
        own_f[t][c] = t0 - t1;                 // corner 00
        red[0][c][t][tid] = t0 + t1;           // corner 10 -> node (cx + 1, cy)
        red[1][c][t][tid] = t2 - t3;           // corner 01 -> node (cx, cy + 1)
        red[2][c][t][tid] = t2 + t3;           // corner 11 -> node (cx + 1, cy + 1)
      }
    }
    __syncthreads();
    // ---- own node columns: add the three neighbours' corner forces, store planes z..z+3
    if (own) {
      const int t10 = tid - 1, t01 = tid - TXC, t11 = tid - TXC - 1;
      const uchar4 mb = *reinterpret_cast<const uchar4*>(mask + obase + z);
      const uint8_t mbs[4] = {mb.x, mb.y, mb.z, mb.w};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T o[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          T s = own_f[t][c] + red[0][c][t][t10] + red[1][c][t][t01] + red[2][c][t][t11];
          o[t] = ((mbs[t] >> c) & 1) ? s : T(0);
        }
        Vec4<T>::store(out + c * cs + obase + z, o);
      }
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" {

// Ke (24 x 24, row-major, float64) -> the 45 coefficients of T Ke T^T / 64 in the fixed
// pattern the kernel uses; -1 if Ke has weight outside the pattern (not an isotropic brick).
int lpb_modal_ke(const double* ke, double* kmodal_out) {
  static const int rows[45] = {3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12,
                               13, 13, 14, 14, 14, 15, 15, 16, 16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21, 22, 23};
  static const int cols[45] = {3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12,
                               8, 13, 3, 7, 14, 15, 19, 11, 16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22, 23};
  if (!ke || !kmodal_out) return LP_ERR_ARG;
  // H[m][k] = prod over axes a with bit a of m set of (2 * bit a of k - 1)
  double h[8][8];
  for (int m = 0; m < 8; ++m)
    for (int k = 0; k < 8; ++k) {
      double v = 1.0;
      for (int a = 0; a < 3; ++a)
        if ((m >> a) & 1) v *= ((k >> a) & 1) ? 1.0 : -1.0;
      h[m][k] = v;
    }
  // K^ = T ke T^T / 64 with T = kron(H, I3)
  double kh[24][24];
  double amax = 0.0;
  for (int r = 0; r < 24; ++r)
    for (int c = 0; c < 24; ++c) {
      int mr = r / 3, cr = r % 3, mc = c / 3, cc = c % 3;
      double s = 0.0;
      for (int k1 = 0; k1 < 8; ++k1)
        for (int k2 = 0; k2 < 8; ++k2) s += h[mr][k1] * ke[(3 * k1 + cr) * 24 + 3 * k2 + cc] * h[mc][k2];
      kh[r][c] = s / 64.0;
      if (fabs(kh[r][c]) > amax) amax = fabs(kh[r][c]);
    }
  bool in_pattern[24][24] = {};
  for (int i = 0; i < 45; ++i) in_pattern[rows[i]][cols[i]] = true;
  for (int r = 0; r < 24; ++r)
    for (int c = 0; c < 24; ++c)
      if (!in_pattern[r][c] && fabs(kh[r][c]) > 1e-12 * amax) return -1;
  for (int i = 0; i < 45; ++i) kmodal_out[i] = kh[rows[i]][cols[i]];
  return 45;
}

static bool fine_args_ok(const LpGrid& g) { return lp_grid_ok(g) && g.pz % 4 == 0 && g.cpz == g.pz; }

// kmodal: host memory (copied into the launch parameters)

int lpb_apply_fine_f32(float* out, const float* u, const float* e, const uint8_t* mask, const float* kmodal, int nx,
                       int ny, int nz, int pz, int cpz, void* stream) {
  LpGrid g = lp_grid(nx, ny, nz, pz, cpz);
  if (!fine_args_ok(g) || !out || !u || !e || !mask || !kmodal || out == u) return LP_ERR_ARG;
  KModal<float> km;
  for (int i = 0; i < 45; ++i) km.c[i] = kmodal[i];
  dim3 grid((g.NX() + TXC - 2) / (TXC - 1), (g.NY() + TYC - 2) / (TYC - 1));
  const int smem = 3 * 3 * 4 * TXC * TYC * sizeof(float);
  k_apply_fine<float><<<grid, TXC * TYC, smem, (cudaStream_t)stream>>>(out, u, e, mask, km, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_apply_fine_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* kmodal,
                       int nx, int ny, int nz, int pz, int cpz, void* stream) {
  LpGrid g = lp_grid(nx, ny, nz, pz, cpz);
  if (!fine_args_ok(g) || !out || !u || !e || !mask || !kmodal || out == u) return LP_ERR_ARG;
  KModal<double> km;
  for (int i = 0; i < 45; ++i) km.c[i] = kmodal[i];
  dim3 grid((g.NX() + TXC - 2) / (TXC - 1), (g.NY() + TYC - 2) / (TYC - 1));
  const int smem = 3 * 3 * 4 * TXC * TYC * sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_apply_fine<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  k_apply_fine<double><<<grid, TXC * TYC, smem, (cudaStream_t)stream>>>(out, u, e, mask, km, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
