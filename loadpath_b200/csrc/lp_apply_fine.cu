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
// cell column of the patch plus a one-cell halo on the low x and y sides, lanes along x. It
// marches along z one chunk of four planes at a time: TMA brings the chunk's 17 x 17 node
// columns (and cell moduli) into a ring of shared-memory stages; in the z-chunked field layout
// each box row is 17 columns x 4 planes, one contiguous run. A thread reads its four node
// columns' four planes (and the next chunk's first), forms per plane the x-y modes
// (4 per component), combines consecutive planes into the cell's z modes, applies E_c K^ in
// the modal basis and transforms back to the cell's two faces. A node plane's modal force is the upper face of the cell below plus
// the lower face of the cell above, both in this thread, so z needs no exchange; the four cell
// columns around a node column exchange their corner forces through shared memory.
// No atomics, no scatter: every output is written once by its owner.
//
// Requirements (checked by the host entry): pz % 4 == 0 and cpz == pz; u, e and the mask
// hold zeros in the z padding; u is zero on dofs whose mask bit is 0, so the identity rows
// (1 - m) u of the masked operator vanish and the kernel writes m * K u.
#include <cstring>
#include <mutex>

#include "lp_common.cuh"
#include "lp_modal.cuh"
#include "lp_tma.cuh"

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
  static __device__ __forceinline__ void lds(const float* p, float (&v)[4]) {
    float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  static __device__ __forceinline__ void sts(float* p, const float (&v)[4]) {
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
  static __device__ __forceinline__ void lds(const double* p, double (&v)[4]) {
    double2 a = *reinterpret_cast<const double2*>(p);
    double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  static __device__ __forceinline__ void sts(double* p, const double (&v)[4]) {
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

constexpr int NSTAGE = 3;           // TMA ring depth (chunks of four z-planes)
constexpr int BOX = TXC + 1;         // 17 node columns per side in a loaded box

// every TMA destination / source starts on a 128-byte boundary
template <typename T, int N>
struct alignas(128) Slot {
  T v[(N * sizeof(T) + 127) / 128 * 128 / sizeof(T)];
};

template <typename T>
struct FineSmem {
  Slot<T, 3 * BOX * BOX * 4> u[NSTAGE];              // node values: [comp][y][x][z]
  Slot<T, BOX * BOX * 4> e[NSTAGE];                  // cell moduli: [y][x][z] (16 used per side)
  Slot<T, 3 * (TXC - 1) * (TYC - 1) * 4> o[2];       // outputs staged for the TMA store [comp][y][x][z]
  T red[3][4][TXC * TYC];                            // y-neighbour exchange
  alignas(8) uint64_t full[NSTAGE];
};

template <typename T>
__device__ __forceinline__ T* u_at(FineSmem<T>& sm, int s, int c, int x, int y) {
  return &sm.u[s].v[((c * BOX + y) * BOX + x) * 4];
}

// The fields as TMA tensors: a chunk's row of x columns (4 z values each) is the inner
// dimension, so every box row is 16 * (x extent) contiguous bytes.
template <typename T>
struct TileMaps {
  CUtensorMap u;    // (4 NX, NY, pz / 4, 3), box (4 * 17, 17, 1, 3)
  CUtensorMap e;    // (4 nx, ny, cpz / 4),    box (4 * 17, 17, 1)
  CUtensorMap out;  // (4 NX, NY, pz / 4, 3), box (4 * 15, 15, 1, 3)
};

template <typename T>
__device__ __forceinline__ void xy_modes(const T (&v)[4], T (&a)[4]) {
  // v: node columns 00, 10, 01, 11 -> modes 1, sx, sy, sxsy
  T sx0 = v[0] + v[1], dx0 = v[1] - v[0], sx1 = v[2] + v[3], dx1 = v[3] - v[2];
  a[0] = sx0 + sx1;
  a[1] = dx0 + dx1;
  a[2] = sx1 - sx0;
  a[3] = dx1 - dx0;
}

template <typename T>
__global__ void __launch_bounds__(TXC * TYC, (sizeof(T) == 4 ? 2 : 1))
k_apply_fine(const __grid_constant__ TileMaps<T> maps, const uint8_t* __restrict__ mask, const KModal<T> km,
             LpGrid g, int zch, int nchunks, int* __restrict__ err, double* __restrict__ dotp) {
  extern __shared__ unsigned char smem_raw[];
  // 128-byte alignment in the shared window (what TMA addresses), not in the generic space
  const uint32_t raw_off = lp_smem_addr(smem_raw);
  FineSmem<T>& sm = *reinterpret_cast<FineSmem<T>*>(smem_raw + ((128u - (raw_off & 127u)) & 127u));
  const int tid = threadIdx.x;
  const int i = tid % TXC, j = tid / TXC;
  const int x0 = blockIdx.x * (TXC - 1), y0 = blockIdx.y * (TYC - 1);
  const int c_begin = blockIdx.z * zch;
  const int c_end = min(c_begin + zch, nchunks);
  const long long bid = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
  if (c_begin >= c_end) {
    if (dotp && tid == 0) dotp[bid] = 0.0;
    return;
  }
  const int cstart = c_begin > 0 ? c_begin - 1 : 0;     // one halo chunk below the segment
  const int nload = min(c_end + 1, nchunks) - cstart;   // + the plane above the last chunk
  const int nproc = c_end - cstart;
  const bool own = i >= 1 && j >= 1;
  constexpr uint32_t UBYTES = 3 * BOX * BOX * 4 * sizeof(T);
  constexpr uint32_t EBYTES = BOX * BOX * 4 * sizeof(T);

  // alignment contract of every TMA operand and vector access, checked once per block: a
  // violation is recorded in *err (codes 10..16) and the block returns without touching memory
  __shared__ int bad;
  if (tid == 0) {
    int code = 0;
    uint32_t so = 0;
    for (int s = 0; s < NSTAGE; ++s) so |= lp_smem_addr(sm.u[s].v) | lp_smem_addr(sm.e[s].v);
    so |= lp_smem_addr(sm.o[0].v) | lp_smem_addr(sm.o[1].v);
    if (so & 127) code = 10;
    else if (reinterpret_cast<uintptr_t>(&maps.u) & 63) code = 11;
    else if (reinterpret_cast<uintptr_t>(&maps.e) & 63) code = 12;
    else if (reinterpret_cast<uintptr_t>(&maps.out) & 63) code = 13;
    else if (lp_smem_addr(&sm.full[0]) & 7) code = 15;
    else if (reinterpret_cast<uintptr_t>(mask) & 3) code = 16;
    bad = code;
    if (code) atomicExch(err, code);
  }
  __syncthreads();
  if (bad) {
    if (dotp && tid == 0) dotp[bid] = 0.0;
    return;
  }
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) lp_mbar_init(&sm.full[s], 1);
    lp_fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int k) {
    const int s = k % NSTAGE;
    lp_mbar_expect_tx(&sm.full[s], UBYTES + EBYTES);
    lp_tma_load_4d(sm.u[s].v, &maps.u, 4 * (x0 - 1), y0 - 1, cstart + k, 0, &sm.full[s]);
    lp_tma_load_3d(sm.e[s].v, &maps.e, 4 * (x0 - 1), y0 - 1, cstart + k, &sm.full[s]);
  };
  if (tid == 0) {
    issue(0);
    if (nload > 1) issue(1);
  }

  T up_carry[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) up_carry[q][c] = T(0);
  double pacc = 0.0;   // u . (K u) over this thread's own nodes (when dotp is given)

  for (int k = 0; k < nproc; ++k) {
    const int c = cstart + k;
    const bool halo = c < c_begin;
    const int s = k % NSTAGE;
    if (tid == 0) {
      if (k + 2 < nload) issue(k + 2);
      lp_bulk_wait_read<1>();   // the store from two chunks ago has read its staging buffer
    }
    bool ok = lp_mbar_wait(&sm.full[s], (k / NSTAGE) & 1);
    const bool has_next = k + 1 < nload;
    if (has_next) ok = ok && lp_mbar_wait(&sm.full[(k + 1) % NSTAGE], ((k + 1) / NSTAGE) & 1);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        // let the loads already issued land before the block exits (bounded as well)
        for (int kk = k; kk < min(k + 3, nload); ++kk) lp_mbar_wait(&sm.full[kk % NSTAGE], (kk / NSTAGE) & 1);
      }
      break;
    }
    // ---- this thread's four node columns: planes z..z+3 and plane z+4
    T un[4][3][5];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const T* col = u_at(sm, s, cc, i + (q & 1), j + (q >> 1));
        T v4[4];
        Vec4<T>::lds(col, v4);
        un[q][cc][0] = v4[0]; un[q][cc][1] = v4[1]; un[q][cc][2] = v4[2]; un[q][cc][3] = v4[3];
        un[q][cc][4] = has_next ? *u_at(sm, (k + 1) % NSTAGE, cc, i + (q & 1), j + (q >> 1)) : T(0);
      }
    T ev[4];
    Vec4<T>::lds(&sm.e[s].v[(j * BOX + i) * 4], ev);

    T a_lo[4][3];
    {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        T v[4], a[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = halo ? un[q][cc][3] : un[q][cc][0];
        xy_modes(v, a);
#pragma unroll
        for (int q = 0; q < 4; ++q) a_lo[q][cc] = a[q];
      }
    }
    T s0v[4][3];   // this node column's force from its own and its -x neighbour's cells
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (halo && t < 3) continue;
      T a_hi[4][3];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        T v[4] = {un[0][cc][t + 1], un[1][cc][t + 1], un[2][cc][t + 1], un[3][cc][t + 1]}, a[4];
        xy_modes(v, a);
#pragma unroll
        for (int q = 0; q < 4; ++q) a_hi[q][cc] = a[q];
      }
      const T ec = ev[t];
      T v[24], f[24];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          T lo = a_lo[q][cc], hi = a_hi[q][cc];
          v[3 * q + cc] = (lo + hi) * ec;
          v[3 * (q + 4) + cc] = (hi - lo) * ec;
        }
      modal_product<T>(km, v, f);
      T fp[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          T f0 = f[3 * q + cc], f1 = f[3 * (q + 4) + cc];
          fp[q][cc] = up_carry[q][cc] + (f0 - f1);
          up_carry[q][cc] = f0 + f1;
          a_lo[q][cc] = a_hi[q][cc];
        }
      if (!halo) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          T t0 = fp[0][cc] - fp[2][cc], t1 = fp[1][cc] - fp[3][cc];
          T t2 = fp[0][cc] + fp[2][cc], t3 = fp[1][cc] + fp[3][cc];
          // corners 00, 10 (-> x+1), 01 (-> y+1), 11 (-> x+1, y+1); x through shuffles
          T c10 = __shfl_up_sync(0xffffffffu, t0 + t1, 1, TXC);
          T c11 = __shfl_up_sync(0xffffffffu, t2 + t3, 1, TXC);
          s0v[t][cc] = (t0 - t1) + c10;
          sm.red[cc][t][tid] = (t2 - t3) + c11;
        }
      }
    }
    if (halo) {           // uniform across the block: the halo chunk only sets up_carry
      __syncthreads();    // its stage is refilled next iteration: every thread is done reading
      continue;
    }
    __syncthreads();
    if (own) {
      const bool inside = x0 - 1 + i < g.NX() && y0 - 1 + j < g.NY();
      uint8_t mbs[4] = {0, 0, 0, 0};
      if (inside) {
        const uchar4 mb = *reinterpret_cast<const uchar4*>(mask + g.node(x0 - 1 + i, y0 - 1 + j, 4 * c));
        mbs[0] = mb.x; mbs[1] = mb.y; mbs[2] = mb.z; mbs[3] = mb.w;
      }
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        T o[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          T v = s0v[t][cc] + sm.red[cc][t][tid - TXC];
          o[t] = ((mbs[t] >> cc) & 1) ? v : T(0);
          pacc += (double)o[t] * (double)un[0][cc][t];   // this node's u: column q = 0
        }
        Vec4<T>::sts(&sm.o[k & 1].v[((cc * (TYC - 1) + (j - 1)) * (TXC - 1) + (i - 1)) * 4], o);
      }
    }
    lp_fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      lp_tma_store_4d(&maps.out, 4 * x0, y0, c, 0, sm.o[k & 1].v);
      lp_bulk_commit();
    }
  }
  if (tid == 0) lp_bulk_wait_all();
  if (dotp) {
    __shared__ double sh[32];
    pacc = lp_block_sum(pacc, sh);
    if (tid == 0) dotp[bid] = pacc;
  }
}

// ordered sum of the per-block partials (the same bits every run)
__global__ void k_fine_dot_final(const double* __restrict__ part, long long n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

// ---- float32: pairs of cells in packed float32x2 arithmetic ------------------------------------
// The float32 kernel forms cells (z, z+1) and (z+2, z+3) of a chunk as pairs: a 128-bit load of
// a node column's four planes is two register pairs, the x-y modes and the modal product run on
// pairs (add / sub / mul / fma .f32x2), and the two steps that shift by one plane (lower plane +
// upper plane of a cell, face forces into node planes) are scalar operations writing pair
// halves. Same arithmetic as the scalar kernel, half the floating-point instructions.
typedef unsigned long long f2_t;

__device__ __forceinline__ f2_t pk2(float lo, float hi) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float lo2(f2_t v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return a;
}
__device__ __forceinline__ float hi2(f2_t v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return b;
}
__device__ __forceinline__ f2_t add2(f2_t a, f2_t b) {
  f2_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t sub2(f2_t a, f2_t b) {
  f2_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t mul2(f2_t a, f2_t b) {
  f2_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2_t fma2(f2_t a, f2_t b, f2_t c) {
  f2_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

struct KModal2 {
  f2_t c[45];   // each coefficient in both lanes
};

// the modal product of lpb_modal_ke's pattern on a pair of cells (rows 0..2 are zero)
__device__ __forceinline__ void modal_product2(const KModal2& km, const f2_t (&v)[24], f2_t (&f)[24]) {
  f[3] = fma2(km.c[2], v[14], fma2(km.c[1], v[7], mul2(km.c[0], v[3])));
  f[4] = fma2(km.c[4], v[6], mul2(km.c[3], v[4]));
  f[5] = fma2(km.c[6], v[12], mul2(km.c[5], v[5]));
  f[6] = fma2(km.c[8], v[6], mul2(km.c[7], v[4]));
  f[7] = fma2(km.c[11], v[14], fma2(km.c[10], v[7], mul2(km.c[9], v[3])));
  f[8] = fma2(km.c[13], v[13], mul2(km.c[12], v[8]));
  f[9] = fma2(km.c[15], v[20], mul2(km.c[14], v[9]));
  f[10] = fma2(km.c[17], v[17], mul2(km.c[16], v[10]));
  f[11] = fma2(km.c[20], v[18], fma2(km.c[19], v[16], mul2(km.c[18], v[11])));
  f[12] = fma2(km.c[22], v[12], mul2(km.c[21], v[5]));
  f[13] = fma2(km.c[24], v[13], mul2(km.c[23], v[8]));
  f[14] = fma2(km.c[27], v[14], fma2(km.c[26], v[7], mul2(km.c[25], v[3])));
  f[15] = fma2(km.c[29], v[19], mul2(km.c[28], v[15]));
  f[16] = fma2(km.c[32], v[18], fma2(km.c[31], v[16], mul2(km.c[30], v[11])));
  f[17] = fma2(km.c[34], v[17], mul2(km.c[33], v[10]));
  f[18] = fma2(km.c[37], v[18], fma2(km.c[36], v[16], mul2(km.c[35], v[11])));
  f[19] = fma2(km.c[39], v[19], mul2(km.c[38], v[15]));
  f[20] = fma2(km.c[41], v[20], mul2(km.c[40], v[9]));
  f[21] = mul2(km.c[42], v[21]);
  f[22] = mul2(km.c[43], v[22]);
  f[23] = mul2(km.c[44], v[23]);
}

__device__ __forceinline__ void xy_modes2(const f2_t (&v)[4], f2_t (&a)[4]) {
  const f2_t sx0 = add2(v[0], v[1]), dx0 = sub2(v[1], v[0]), sx1 = add2(v[2], v[3]), dx1 = sub2(v[3], v[2]);
  a[0] = add2(sx0, sx1);
  a[1] = add2(dx0, dx1);
  a[2] = sub2(sx1, sx0);
  a[3] = sub2(dx1, dx0);
}

// One pair of cells (lower cell planes lo.., upper ..): forms the pair's modal vectors from the
// x-y modes of three consecutive planes (m0, m1 as a pair and m2), applies E and K^, and returns
// the two node-plane forces as a pair (carry + lower face of the first cell, upper face of the
// first + lower face of the second) and the second cell's upper face as the next carry.
__device__ __forceinline__ void cell_pair(const KModal2& km, const f2_t (&m01)[4][3], const float (&m2)[4][3], f2_t e,
                                          float (&carry)[4][3], f2_t (&fp)[4][3]) {
  f2_t v[24], f[24];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const float a0 = lo2(m01[q][cc]), a1 = hi2(m01[q][cc]), a2 = m2[q][cc];
      v[3 * q + cc] = mul2(pk2(a0 + a1, a1 + a2), e);
      v[3 * (q + 4) + cc] = mul2(pk2(a1 - a0, a2 - a1), e);
    }
  modal_product2(km, v, f);
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const f2_t f1 = f[3 * (q + 4) + cc];
      f2_t lw, up;
      if (q == 0) {
        lw = sub2(0ull, f1);   // rows 0..2 (the constant mode) are zero
        up = f1;
      } else {
        const f2_t f0 = f[3 * q + cc];
        lw = sub2(f0, f1);
        up = add2(f0, f1);
      }
      fp[q][cc] = pk2(carry[q][cc] + lo2(lw), lo2(up) + hi2(lw));
      carry[q][cc] = hi2(up);
    }
}

// corner forces of one pair of node planes: own corner pair (00 + the -x neighbour's 10) kept,
// the y + 1 corners (01 + 11 of the -x neighbour) to shared memory
__device__ __forceinline__ void plane_corners2(const f2_t (&fp)[4][3], f2_t (&s0v)[3], float2* red, int tid) {
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    const f2_t t0 = sub2(fp[0][cc], fp[2][cc]), t1 = sub2(fp[1][cc], fp[3][cc]);
    const f2_t t2 = add2(fp[0][cc], fp[2][cc]), t3 = add2(fp[1][cc], fp[3][cc]);
    const f2_t a = add2(t0, t1), b = add2(t2, t3);
    const f2_t ca = pk2(__shfl_up_sync(0xffffffffu, lo2(a), 1, TXC), __shfl_up_sync(0xffffffffu, hi2(a), 1, TXC));
    const f2_t cb = pk2(__shfl_up_sync(0xffffffffu, lo2(b), 1, TXC), __shfl_up_sync(0xffffffffu, hi2(b), 1, TXC));
    s0v[cc] = add2(sub2(t0, t1), ca);
    const f2_t r = add2(sub2(t2, t3), cb);
    red[cc * TXC * TYC + tid] = make_float2(lo2(r), hi2(r));
  }
}

constexpr int NST2 = 3;   // TMA ring depth of the float32 kernel (loads run NST2 - 1 chunks ahead)

struct FineSmem2 {
  Slot<float, 3 * BOX * BOX * 4> u[NST2];
  Slot<float, BOX * BOX * 4> e[NST2];
  float2 red[2][2][3][TXC * TYC];                 // [chunk parity][plane pair][component][thread]
  alignas(8) uint64_t full[NST2];
};

__device__ __forceinline__ const float* u_at2(const FineSmem2& sm, int s, int c, int x, int y) {
  return &sm.u[s].v[((c * BOX + y) * BOX + x) * 4];
}

// The degree-2 Chebyshev update formed where A u is stored (the vector kernels' expressions, so
// the same bits): mode 1 (u = d) x = d + (c1 d + c2 dinv (b - A d)); mode 2 (u = x) r = b - A x,
// d = s dinv r; mode 3 (u = d) x = (x + d) + (c1 d + c2 dinv (r - A d)).
struct FineCheb {
  float* x;
  float* r;
  float* d;
  const float* b;
  const float* dinv;
  const double* coef;
};

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

template <int MODE>
__device__ __forceinline__ void cheb_store(const FineCheb& ch, long long i, const float4 ad4, float s, float c1,
                                           float c2) {
  const float4 dv4 = ldg4(ch.dinv + i);
  const float* ad = &ad4.x;
  const float* dv = &dv4.x;
  if constexpr (MODE == 1) {
    const float4 d4 = ldg4(ch.d + i), b4 = ldg4(ch.b + i);
    const float *d = &d4.x, *b = &b4.x;
    float4 x4;
    float* x = &x4.x;
#pragma unroll
    for (int t = 0; t < 4; ++t) x[t] = lp_cheb2_zero_v(d[t], b[t], ad[t], dv[t], c1, c2);
    *reinterpret_cast<float4*>(ch.x + i) = x4;
  } else if constexpr (MODE == 2) {
    const float4 b4 = ldg4(ch.b + i);
    const float* b = &b4.x;
    float4 r4, d4;
    float *r = &r4.x, *d = &d4.x;
#pragma unroll
    for (int t = 0; t < 4; ++t) lp_residual_scaled_v(b[t], ad[t], dv[t], s, r[t], d[t]);
    *reinterpret_cast<float4*>(ch.r + i) = r4;
    *reinterpret_cast<float4*>(ch.d + i) = d4;
  } else {
    const float4 x4 = *reinterpret_cast<const float4*>(ch.x + i);   // read, then written, by this thread
    const float4 d4 = ldg4(ch.d + i), r4 = ldg4(ch.r + i);
    const float *x = &x4.x, *d = &d4.x, *r = &r4.x;
    float4 o4;
    float* o = &o4.x;
#pragma unroll
    for (int t = 0; t < 4; ++t) o[t] = lp_cheb2_v(x[t], d[t], r[t], ad[t], dv[t], c1, c2);
    *reinterpret_cast<float4*>(ch.x + i) = o4;
  }
}

// One barrier per chunk: each thread waits for its stage, computes, publishes its y-corner
// forces into the exchange buffer of the chunk's parity, and the block meets once (which also
// settles a wait that gave up); the owners then add their -y neighbour's corners and store
// their four node planes with 16-byte stores. The exchange is double-buffered, so the next
// chunk's writes never meet this chunk's reads. A chunk runs in two phases that keep the
// register footprint to one pair of cells: (A) planes 0..2 -> cells 0, 1; (B) planes 2..4 ->
// cells 2, 3 (plane 2's modes formed in both). MODE 0 stores A u in out; modes 1..3 store a
// Chebyshev update instead (cheb_store; out unused).
template <int MODE>
__global__ void __launch_bounds__(TXC * TYC, 2)
k_apply_fine_x2(const __grid_constant__ TileMaps<float> maps, float* __restrict__ out,
                const uint8_t* __restrict__ mask, const KModal2 km2, const KModal<float> km, LpGrid g, int zch,
                int nchunks, int* __restrict__ err, const FineCheb ch) {
  extern __shared__ unsigned char smem_raw2[];
  const uint32_t raw_off = lp_smem_addr(smem_raw2);
  FineSmem2& sm = *reinterpret_cast<FineSmem2*>(smem_raw2 + ((128u - (raw_off & 127u)) & 127u));
  const int tid = threadIdx.x;
  const int i = tid % TXC, j = tid / TXC;
  const int x0 = blockIdx.x * (TXC - 1), y0 = blockIdx.y * (TYC - 1);
  const int c_begin = blockIdx.z * zch;
  const int c_end = min(c_begin + zch, nchunks);
  if (c_begin >= c_end) return;
  const int cstart = c_begin > 0 ? c_begin - 1 : 0;
  const int nload = min(c_end + 1, nchunks) - cstart;
  const int nproc = c_end - cstart;
  const int nx_ = x0 - 1 + i, ny_ = y0 - 1 + j;
  const bool writer = i >= 1 && j >= 1 && nx_ < g.NX() && ny_ < g.NY();
  const long long obase = writer ? g.node(nx_, ny_, 0) : 0;   // chunk c at obase + c * zcs
  const long long cs = g.comp_stride(), zcs = g.node_zc_stride();
  constexpr uint32_t UBYTES = 3 * BOX * BOX * 4 * sizeof(float);
  constexpr uint32_t EBYTES = BOX * BOX * 4 * sizeof(float);
  __shared__ int bad;
  if (tid == 0) {
    int code = 0;
    uint32_t so = 0;
    for (int s = 0; s < NST2; ++s) so |= lp_smem_addr(sm.u[s].v) | lp_smem_addr(sm.e[s].v);
    if (so & 127) code = 10;
    else if (reinterpret_cast<uintptr_t>(&maps.u) & 63) code = 11;
    else if (reinterpret_cast<uintptr_t>(&maps.e) & 63) code = 12;
    else if (MODE == 0 && (reinterpret_cast<uintptr_t>(out) & 15)) code = 13;
    else if (MODE != 0 && ((reinterpret_cast<uintptr_t>(ch.x) | reinterpret_cast<uintptr_t>(ch.r) |
                            reinterpret_cast<uintptr_t>(ch.d) | reinterpret_cast<uintptr_t>(ch.b) |
                            reinterpret_cast<uintptr_t>(ch.dinv)) & 15)) code = 14;
    else if (lp_smem_addr(&sm.full[0]) & 7) code = 15;
    else if (reinterpret_cast<uintptr_t>(mask) & 3) code = 16;
    bad = code;
    if (code) atomicExch(err, code);
  }
  __syncthreads();
  if (bad) return;
  float cs_s = 0.0f, cs_c1 = 0.0f, cs_c2 = 0.0f;
  if constexpr (MODE != 0) {
    cs_s = (float)ch.coef[1];
    cs_c1 = (float)ch.coef[2];
    cs_c2 = (float)ch.coef[3];
  }
  if (tid == 0) {
    for (int s = 0; s < NST2; ++s) lp_mbar_init(&sm.full[s], 1);
    lp_fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int k) {
    const int s = k % NST2;
    lp_mbar_expect_tx(&sm.full[s], UBYTES + EBYTES);
    lp_tma_load_4d(sm.u[s].v, &maps.u, 4 * (x0 - 1), y0 - 1, cstart + k, 0, &sm.full[s]);
    lp_tma_load_3d(sm.e[s].v, &maps.e, 4 * (x0 - 1), y0 - 1, cstart + k, &sm.full[s]);
  };
  if (tid == 0)
    for (int kk = 0; kk < NST2 - 1 && kk < nload; ++kk) issue(kk);
  float carry[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) carry[q][c] = 0.0f;

  for (int k = 0; k < nproc; ++k) {
    const int c = cstart + k;
    const bool halo = c < c_begin;
    const int s = k % NST2;
    // the stage refilled here was last read in the previous chunk, before its barrier
    if (tid == 0 && k + NST2 - 1 < nload) issue(k + NST2 - 1);
    const uint32_t mb4 = (writer && !halo) ? __ldg(reinterpret_cast<const uint32_t*>(mask + obase + c * zcs)) : 0u;
    bool ok = lp_mbar_wait(&sm.full[s], (k / NST2) & 1);
    const bool has_next = k + 1 < nload;
    if (has_next) ok = ok && lp_mbar_wait(&sm.full[(k + 1) % NST2], ((k + 1) / NST2) & 1);
    // a wait that gave up leaves stale but in-bounds data; the barrier below then stops the block
    const float* ecol = &sm.e[s].v[(j * BOX + i) * 4];
    f2_t m23[4][3];
    float m4[4][3];
    auto load_b = [&]() {
      f2_t p23[4][3];
      float p4[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const float2 v = *reinterpret_cast<const float2*>(u_at2(sm, s, cc, i + (q & 1), j + (q >> 1)) + 2);
          p23[q][cc] = pk2(v.x, v.y);
          p4[q][cc] = has_next ? *u_at2(sm, (k + 1) % NST2, cc, i + (q & 1), j + (q >> 1)) : 0.0f;
        }
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        f2_t v23[4] = {p23[0][cc], p23[1][cc], p23[2][cc], p23[3][cc]}, a23[4];
        float v4[4] = {p4[0][cc], p4[1][cc], p4[2][cc], p4[3][cc]}, a4[4];
        xy_modes2(v23, a23);
        xy_modes(v4, a4);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          m23[q][cc] = a23[q];
          m4[q][cc] = a4[q];
        }
      }
    };
    if (halo) {
      // only the chunk's last cell: its upper face starts the carry of the segment
      load_b();
      const float ew = ecol[3];
      float v[24], f[24];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const float lo = hi2(m23[q][cc]), hi = m4[q][cc];
          v[3 * q + cc] = (lo + hi) * ew;
          v[3 * (q + 4) + cc] = (hi - lo) * ew;
        }
      modal_product<float>(km, v, f);
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) carry[q][cc] = f[3 * q + cc] + f[3 * (q + 4) + cc];
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(err, 1);
          for (int kk = k; kk < min(k + NST2, nload); ++kk) lp_mbar_wait(&sm.full[kk % NST2], (kk / NST2) & 1);
        }
        break;
      }
      continue;
    }
    f2_t s0v[2][3];
    float2(*red)[3][TXC * TYC] = sm.red[k & 1];
    {
      f2_t m01[4][3];
      float m2[4][3];
      {
        f2_t p01[4][3];
        float p2[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const float4 v = *reinterpret_cast<const float4*>(u_at2(sm, s, cc, i + (q & 1), j + (q >> 1)));
            p01[q][cc] = pk2(v.x, v.y);
            p2[q][cc] = v.z;
          }
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          f2_t v01[4] = {p01[0][cc], p01[1][cc], p01[2][cc], p01[3][cc]}, a01[4];
          float v2[4] = {p2[0][cc], p2[1][cc], p2[2][cc], p2[3][cc]}, a2[4];
          xy_modes2(v01, a01);
          xy_modes(v2, a2);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            m01[q][cc] = a01[q];
            m2[q][cc] = a2[q];
          }
        }
      }
      const float2 e01 = *reinterpret_cast<const float2*>(ecol);
      f2_t fp[4][3];
      cell_pair(km2, m01, m2, pk2(e01.x, e01.y), carry, fp);
      plane_corners2(fp, s0v[0], red[0][0], tid);
    }
    {
      load_b();
      const float2 e23 = *reinterpret_cast<const float2*>(ecol + 2);
      f2_t fp[4][3];
      cell_pair(km2, m23, m4, pk2(e23.x, e23.y), carry, fp);
      plane_corners2(fp, s0v[1], red[1][0], tid);
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        for (int kk = k; kk < min(k + NST2, nload); ++kk) lp_mbar_wait(&sm.full[kk % NST2], (kk / NST2) & 1);
      }
      break;
    }
    if (writer) {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const float2 r01 = red[0][cc][tid - TXC], r23 = red[1][cc][tid - TXC];
        const f2_t o01 = add2(s0v[0][cc], pk2(r01.x, r01.y)), o23 = add2(s0v[1][cc], pk2(r23.x, r23.y));
        float4 o = make_float4(lo2(o01), hi2(o01), lo2(o23), hi2(o23));
        if (!((mb4 >> cc) & 1u)) o.x = 0.0f;
        if (!((mb4 >> (8 + cc)) & 1u)) o.y = 0.0f;
        if (!((mb4 >> (16 + cc)) & 1u)) o.z = 0.0f;
        if (!((mb4 >> (24 + cc)) & 1u)) o.w = 0.0f;
        if constexpr (MODE == 0) *reinterpret_cast<float4*>(out + cc * cs + obase + c * zcs) = o;
        else cheb_store<MODE>(ch, cc * cs + obase + c * zcs, o, cs_s, cs_c1, cs_c2);
      }
    }
  }
}

}  // namespace

static bool fine_args_ok(const LpGrid& g) { return lp_grid_ok(g) && g.pz % 4 == 0 && g.cpz == g.pz; }

// resident blocks of a kernel on this device at the given dynamic shared memory (and the
// attribute that allows it), looked up once per kernel
static long long resident_blocks(const void* kfn, int smem) {
  static std::mutex mu;
  static const void* keys[8];
  static long long vals[8];
  static int n = 0;
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < n; ++i)
    if (keys[i] == kfn) return vals[i];
  if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 0;
  int per_sm = 1, dev = 0, nsm = 148;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, TXC * TYC, smem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long v = (long long)(per_sm > 0 ? per_sm : 1) * nsm;
  if (n < 8) {
    keys[n] = kfn;
    vals[n] = v;
    ++n;
  }
  return v;
}

template <typename T>
static int launch_fine(T* out, const T* u, const T* e, const uint8_t* mask, const double* kmodal_host, int* err,
                       LpGrid g, cudaStream_t st, double* part = nullptr, long long part_len = 0,
                       double* dot_out = nullptr, int mode = 0, const FineCheb* ch = nullptr) {
  if (!fine_args_ok(g) || !out || !u || !e || !mask || !kmodal_host || !err || out == u) return LP_ERR_ARG;
  KModal<T> km;
  for (int i = 0; i < 45; ++i) km.c[i] = (T)kmodal_host[i];
  // float32: the packed-pair kernel
  const bool x2 = sizeof(T) == 4;
  if (mode != 0 && (!x2 || !ch || mode < 0 || mode > 3)) return LP_ERR_ARG;
  const uint32_t zc = 4;
  TileMaps<T> maps;
  const uint64_t nd[4] = {zc * (uint64_t)g.NX(), (uint64_t)g.NY(), (uint64_t)g.pz / zc, 3};
  const uint64_t cd[3] = {zc * (uint64_t)g.nx, (uint64_t)g.ny, (uint64_t)g.cpz / zc};
  const uint32_t bin[4] = {zc * BOX, BOX, 1, 3};
  const uint32_t be[3] = {zc * BOX, BOX, 1};
  const uint32_t bout[4] = {zc * (TXC - 1), TYC - 1, 1, 3};
  if (!lp_make_map(&maps.u, u, 4, nd, bin, sizeof(T)) || !lp_make_map(&maps.e, e, 3, cd, be, sizeof(T)) ||
      !lp_make_map(&maps.out, out, 4, nd, bout, sizeof(T)))
    return LP_ERR_ARG;
  const int smem = x2 ? (int)sizeof(FineSmem2) + 128 : (int)sizeof(FineSmem<T>) + 128;
  const void* x2fn = mode == 1   ? (const void*)k_apply_fine_x2<1>
                     : mode == 2 ? (const void*)k_apply_fine_x2<2>
                     : mode == 3 ? (const void*)k_apply_fine_x2<3>
                                 : (const void*)k_apply_fine_x2<0>;
  const void* kfn = x2 ? x2fn : (const void*)k_apply_fine<T>;
  const long long slots = resident_blocks(kfn, smem);
  if (!slots) return LP_ERR_LAUNCH;
  const int gx = (g.NX() + TXC - 2) / (TXC - 1), gy = (g.NY() + TYC - 2) / (TYC - 1);
  const int nchunks = g.pz / (int)zc;
  // z segments: balance the grid over the resident blocks; a segment recomputes one halo cell
  int best_zch = nchunks;
  double best = 1e30;
  for (int zch = 2; zch <= nchunks; ++zch) {
    const long long nseg = (nchunks + zch - 1) / zch;
    const long long units = (long long)gx * gy * nseg;
    const long long waves = (units + slots - 1) / slots;
    const double cost = (double)waves * (zch + (nseg > 1 ? 0.3 : 0.0));
    if (cost < best - 1e-9) { best = cost; best_zch = zch; }
  }
  const int tuned = lp_tune_lookup(sizeof(T) == 4 ? LP_KNOB_FINE_F32 : LP_KNOB_FINE_F64, g.nx, g.ny, g.nz);
  if (tuned >= 2 && tuned <= nchunks) best_zch = tuned;
  const int nseg = (nchunks + best_zch - 1) / best_zch;
  dim3 grid(gx, gy, nseg);
  if constexpr (sizeof(T) == 4) {
    if (x2) {
      KModal2 km2;
      for (int i = 0; i < 45; ++i) {
        const float c = (float)kmodal_host[i];
        uint32_t bits;
        memcpy(&bits, &c, 4);
        km2.c[i] = ((unsigned long long)bits << 32) | bits;
      }
      const FineCheb none{};
      const FineCheb& c = ch ? *ch : none;
      if (mode == 1) k_apply_fine_x2<1><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, km2, km, g, best_zch, nchunks, err, c);
      else if (mode == 2) k_apply_fine_x2<2><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, km2, km, g, best_zch, nchunks, err, c);
      else if (mode == 3) k_apply_fine_x2<3><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, km2, km, g, best_zch, nchunks, err, c);
      else k_apply_fine_x2<0><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, km2, km, g, best_zch, nchunks, err, c);
      LP_LAUNCH_CHECK();
      return LP_OK;
    }
  }
  if (part) {
    const long long nb = (long long)grid.x * grid.y * grid.z;
    if (nb > part_len) return LP_ERR_SIZE;
    k_apply_fine<T><<<grid, TXC * TYC, smem, st>>>(maps, mask, km, g, best_zch, nchunks, err, part);
    k_fine_dot_final<<<1, 1024, 0, st>>>(part, nb, dot_out);
  } else {
    k_apply_fine<T><<<grid, TXC * TYC, smem, st>>>(maps, mask, km, g, best_zch, nchunks, err, nullptr);
  }
  LP_LAUNCH_CHECK();
  return LP_OK;
}

extern "C" {

// Ke (24 x 24, row-major, float64) -> the 45 coefficients of T Ke T^T / 64 in the fixed
// pattern the kernel uses; -1 if Ke has weight outside the pattern (not an isotropic brick).
int lpb_modal_ke(const double* ke, double* kmodal_out) {
  static const int rows[LP_MODAL_NNZ] = LP_MODAL_ROWS;
  static const int cols[LP_MODAL_NNZ] = LP_MODAL_COLS;
  if (!ke || !kmodal_out) return LP_ERR_ARG;
  double kh[24][24];
  double amax = 0.0;
  for (int r = 0; r < 24; ++r)
    for (int c = 0; c < 24; ++c) {
      kh[r][c] = lp_modal_entry(ke, r, c);
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


int lpb_apply_fine_f32(float* out, const float* u, const float* e, const uint8_t* mask, const double* kmodal,
                       int* err, int nx, int ny, int nz, int pz, int cpz, void* stream) {
  return launch_fine<float>(out, u, e, mask, kmodal, err, lp_grid(nx, ny, nz, pz, cpz), (cudaStream_t)stream);
}

int lpb_apply_fine_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* kmodal,
                       int* err, int nx, int ny, int nz, int pz, int cpz, void* stream) {
  return launch_fine<double>(out, u, e, mask, kmodal, err, lp_grid(nx, ny, nz, pz, cpz), (cudaStream_t)stream);
}

// lpb_apply_fine_f32 with a degree-2 Chebyshev update formed where A u is stored: mode 1 (u = d)
// x = d + (c1 d + c2 dinv (b - A d)); mode 2 (u = x) r = b - A x, d = s dinv r; mode 3 (u = d)
// x = (x + d) + (c1 d + c2 dinv (r - A d)); coef: the level's Chebyshev coefficients (device);
// the fields a mode does not name may be NULL
int lpb_apply_fine_cheb_f32(int mode, float* x, float* r, float* d, const float* u, const float* b, const float* dinv,
                            const double* coef, const float* e, const uint8_t* mask, const double* kmodal, int* err,
                            int nx, int ny, int nz, int pz, int cpz, void* stream) {
  if (!u || !dinv || !coef) return LP_ERR_ARG;
  float* out = nullptr;
  if (mode == 1 && x && d && b && u == d && x != d) out = x;
  if (mode == 2 && r && d && b && u == x && r != u && d != u && r != d) out = r;
  if (mode == 3 && x && d && r && u == d && x != d && r != d && r != x) out = x;
  if (!out) return LP_ERR_ARG;
  const FineCheb ch{x, r, d, b, dinv, coef};
  return launch_fine<float>(out, u, e, mask, kmodal, err, lp_grid(nx, ny, nz, pz, cpz), (cudaStream_t)stream, nullptr,
                            0, nullptr, mode, &ch);
}

// lpb_apply_fine_f64 that also forms u . out over the level's nodes into *dot (float64, device):
// per-block partials in part (part_len doubles; -3 when the grid has more blocks), then an
// ordered sum, so the dot has the same bits every run
int lpb_apply_fine_dot_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* kmodal,
                           int* err, double* part, long long part_len, double* dot, int nx, int ny, int nz, int pz,
                           int cpz, void* stream) {
  if (!part || !dot || part_len <= 0) return LP_ERR_ARG;
  return launch_fine<double>(out, u, e, mask, kmodal, err, lp_grid(nx, ny, nz, pz, cpz), (cudaStream_t)stream, part,
                             part_len, dot);
}

}  // extern "C"
