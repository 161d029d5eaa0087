// Galerkin coarsening on the device (loadpath/mg.py:601-677) and the coarsest level's dense
// operator (loadpath/mg.py:708-766).
//
// Child prolongation: child k of a coarse cell is the fine cell at offset CORNERS[k]; its
// corner q is the fine node at CORNERS[k] + CORNERS[q] in {0, 1, 2}^3 inside the coarse cell,
// interpolated trilinearly from the coarse corners r (loadpath/mg.py:57-75):
//     W[k][q][r] = prod_a (r_a ? p_a / 2 : 1 - p_a / 2),  p = CORNERS[k] + CORNERS[q]
// The same weights act on each of the three components.
#include "lp_common.cuh"

namespace {

__device__ __forceinline__ double pw(int k, int q, int r) {
  double w = 1.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int p = ((k >> a) & 1) + ((q >> a) & 1);
    double t = 0.5 * p;
    w *= ((r >> a) & 1) ? t : 1.0 - t;
  }
  return w;
}

// w[k, C] = e[2C + CORNERS[k]] for C inside the fine grid's half, else 0 (loadpath/mg.py:617-620)
template <typename Te, typename Tw>
__global__ void k_weights_from_e(Tw* __restrict__ w, const Te* __restrict__ e, LpGrid gf, LpGrid gc) {
  const long long total = gc.cells_padded();
  const int hx = gf.nx / 2, hy = gf.ny / 2, hz = gf.nz / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int X, Y, Z;
    if (!gc.cell_at(t, X, Y, Z)) continue;
    long long c = gc.cell(X, Y, Z);
    bool in = X < hx && Y < hy && Z < hz;
    for (int k = 0; k < 8; ++k) {
      Tw v = Tw(0);
      if (in) v = (Tw)e[gf.cell(2 * X + cx_(k), 2 * Y + cy_(k), 2 * Z + cz_(k))];
      w[k * gc.cells_padded() + c] = v;
    }
  }
}

// coarse cells whose children touch a held node (alive and not solved) and carry stiffness
// (loadpath/mg.py:609-623)
template <typename Te>
__global__ void k_patch_flags(uint8_t* __restrict__ flag, const Te* __restrict__ e, const uint8_t* __restrict__ mf,
                              LpGrid gf, LpGrid gc) {
  const long long total = gc.cells_padded();
  const int hx = gf.nx / 2, hy = gf.ny / 2, hz = gf.nz / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int X, Y, Z;
    if (!gc.cell_at(t, X, Y, Z)) continue;
    uint8_t f = 0;
    if (X < hx && Y < hy && Z < hz) {
      for (int k = 0; k < 8 && !f; ++k) {
        int x = 2 * X + cx_(k), y = 2 * Y + cy_(k), z = 2 * Z + cz_(k);
        if (!(e[gf.cell(x, y, z)] > Te(0))) continue;
        for (int qq = 0; qq < 8; ++qq) {
          uint8_t mb = mf[gf.node(x + cx_(qq), y + cy_(qq), z + cz_(qq))];
          if (((mb >> 3) & ~mb) & 7) { f = 1; break; }
        }
      }
    }
    flag[gc.cell(X, Y, Z)] = f;
  }
}

// patch matrices: pk = sum_k P_k^T (e_child ke .* dm dm^T) P_k, one block per patch cell
// (loadpath/mg.py:627-638); the cell's weights are zeroed and its patch row recorded.
template <typename Te, typename Tw>
__global__ void k_patch_matrices(Tw* __restrict__ pk, Tw* __restrict__ w, int* __restrict__ patch_id,
                                 const long long* __restrict__ pcells, int npatch, const Te* __restrict__ e,
                                 const double* __restrict__ ke, const uint8_t* __restrict__ mf, LpGrid gf,
                                 LpGrid gc) {
  __shared__ double kc[576];
  __shared__ double tt[576];
  __shared__ double dm[24];
  int p = blockIdx.x;
  if (p >= npatch) return;
  const long long C = pcells[p];
  int X, Y, Z;
  gc.cell_at(C, X, Y, Z);
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;  // thread t handles outputs t, t+256, t+512
  for (int k = 0; k < 8; ++k) {
    int x = 2 * X + cx_(k), y = 2 * Y + cy_(k), z = 2 * Z + cz_(k);
    double ec = (double)e[gf.cell(x, y, z)];
    if (threadIdx.x < 24) {
      int qq = threadIdx.x / 3, c = threadIdx.x % 3;
      uint8_t mb = mf[gf.node(x + cx_(qq), y + cy_(qq), z + cz_(qq))];
      dm[threadIdx.x] = ((mb >> c) & 1) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 576; i += blockDim.x) kc[i] = ec * ke[i] * dm[i / 24] * dm[i % 24];
    __syncthreads();
    // tt[a][j] = sum_b kc[a][b] P[b][j]  (P[(q,c)][(r,c)] = W[k][q][r])
    for (int i = threadIdx.x; i < 576; i += blockDim.x) {
      int a = i / 24, j = i % 24, r = j / 3, c = j % 3;
      double s = 0.0;
      for (int qq = 0; qq < 8; ++qq) s += kc[a * 24 + 3 * qq + c] * pw(k, qq, r);
      tt[i] = s;
    }
    __syncthreads();
    for (int s = 0; s < 3; ++s) {
      int i = threadIdx.x + s * 256;
      if (i >= 576) break;
      int ii = i / 24, j = i % 24, r = ii / 3, c = ii % 3;
      double v = 0.0;
      for (int qq = 0; qq < 8; ++qq) v += pw(k, qq, r) * tt[(3 * qq + c) * 24 + j];
      if (s == 0) acc0 += v; else if (s == 1) acc1 += v; else acc2 += v;
    }
    __syncthreads();
  }
  for (int s = 0; s < 3; ++s) {
    int i = threadIdx.x + s * 256;
    if (i >= 576) break;
    pk[(long long)p * 576 + i] = (Tw)(s == 0 ? acc0 : s == 1 ? acc1 : acc2);
  }
  if (threadIdx.x < 8) w[threadIdx.x * gc.cells_padded() + C] = Tw(0);
  if (threadIdx.x == 0) patch_id[C] = p;
}

// explicit Galerkin level from a weights or explicit fine level (loadpath/mg.py:639-663);
// strict: the fine matrices masked by the fine level's own mask first (D K D).
// One block (256 threads) per coarse cell; accumulation in float64.
template <typename Tw>
__global__ void k_galerkin_explicit(Tw* __restrict__ kout, int fine_kind, const Tw* __restrict__ fw,
                                    const Tw* __restrict__ mcat, const int* __restrict__ patch_id,
                                    const Tw* __restrict__ patch_k, const Tw* __restrict__ fk,
                                    const uint8_t* __restrict__ mf, int strict, LpGrid gf, LpGrid gc) {
  __shared__ double kf[576];
  __shared__ double tt[576];
  __shared__ double dm[24];
  long long bid = blockIdx.x;
  const long long ncell = (long long)gc.nx * gc.ny * gc.nz;
  if (bid >= ncell) return;
  int Z = (int)(bid % gc.nz);
  long long q0 = bid / gc.nz;
  int Y = (int)(q0 % gc.ny);
  int X = (int)(q0 / gc.ny);
  long long C = gc.cell(X, Y, Z);
  const int hx = gf.nx / 2, hy = gf.ny / 2, hz = gf.nz / 2;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  if (X < hx && Y < hy && Z < hz) {
    for (int k = 0; k < 8; ++k) {
      int x = 2 * X + cx_(k), y = 2 * Y + cy_(k), z = 2 * Z + cz_(k);
      long long c = gf.cell(x, y, z);
      if (threadIdx.x < 24) {
        double v = 1.0;
        if (strict) {
          int qq = threadIdx.x / 3, cc = threadIdx.x % 3;
          uint8_t mb = mf[gf.node(x + cx_(qq), y + cy_(qq), z + cz_(qq))];
          v = ((mb >> cc) & 1) ? 1.0 : 0.0;
        }
        dm[threadIdx.x] = v;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < 576; i += blockDim.x) {
        double v;
        if (fine_kind == 1) {
          v = 0.0;
          for (int q = 0; q < 8; ++q) v += (double)mcat[q * 576 + i] * (double)fw[q * gf.cells_padded() + c];
          int p = patch_id ? patch_id[c] : -1;
          if (p >= 0) v += (double)patch_k[(long long)p * 576 + i];
        } else {
          v = (double)fk[c * 576 + i];
        }
        kf[i] = v * dm[i / 24] * dm[i % 24];
      }
      __syncthreads();
      for (int i = threadIdx.x; i < 576; i += blockDim.x) {
        int a = i / 24, j = i % 24, r = j / 3, cc = j % 3;
        double s = 0.0;
        for (int qq = 0; qq < 8; ++qq) s += kf[a * 24 + 3 * qq + cc] * pw(k, qq, r);
        tt[i] = s;
      }
      __syncthreads();
      for (int s = 0; s < 3; ++s) {
        int i = threadIdx.x + s * 256;
        if (i >= 576) break;
        int ii = i / 24, j = i % 24, r = ii / 3, cc = ii % 3;
        double v = 0.0;
        for (int qq = 0; qq < 8; ++qq) v += pw(k, qq, r) * tt[(3 * qq + cc) * 24 + j];
        if (s == 0) acc0 += v; else if (s == 1) acc1 += v; else acc2 += v;
      }
      __syncthreads();
    }
  }
  for (int s = 0; s < 3; ++s) {
    int i = threadIdx.x + s * 256;
    if (i >= 576) break;
    kout[C * 576 + i] = (Tw)(s == 0 ? acc0 : s == 1 ? acc1 : acc2);
  }
}

// strict hierarchy: held dofs injected down a level, and the share of a coarse dof's
// interpolation kept on solved fine dofs (restrict of the fine mask) (loadpath/mg.py:566-574)
__global__ void k_strict_held_kept(uint8_t* __restrict__ held_c, float* __restrict__ kept,
                                   const uint8_t* __restrict__ held_f, const uint8_t* __restrict__ mf, LpGrid gf,
                                   LpGrid gc) {
  const int FX = gf.NX(), FY = gf.NY(), FZ = gf.NZ();
  const long long total = gc.nodes_padded();
  const long long ccs = gc.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int X, Y, Z;
    if (!gc.node_at(t, X, Y, Z)) continue;
    const long long cn = t;
    uint8_t h = 0;
    if (2 * X < FX && 2 * Y < FY && 2 * Z < FZ) h = held_f[gf.node(2 * X, 2 * Y, 2 * Z)] & 7;
    held_c[cn] = h;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int a = -1; a <= 1; ++a) {
      int x = 2 * X + a;
      if (x < 0 || x >= FX) continue;
      double wa = a ? 0.5 : 1.0;
      for (int b = -1; b <= 1; ++b) {
        int y = 2 * Y + b;
        if (y < 0 || y >= FY) continue;
        double wb = wa * (b ? 0.5 : 1.0);
        for (int e = -1; e <= 1; ++e) {
          int z = 2 * Z + e;
          if (z < 0 || z >= FZ) continue;
          double we = wb * (e ? 0.5 : 1.0);
          uint8_t mb = mf[gf.node(x, y, z)];
          for (int i = 0; i < 3; ++i)
            if ((mb >> i) & 1) acc[i] += we;
        }
      }
    }
    for (int i = 0; i < 3; ++i) kept[i * ccs + cn] = (float)acc[i];
  }
}

// level-0 held bits: alive and fixed
__global__ void k_held0(uint8_t* __restrict__ held, const uint8_t* __restrict__ mask0,
                        const uint8_t* __restrict__ fixed_bits, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    held[i] = (uint8_t)(((mask0[i] >> 3) & fixed_bits[i]) & 7);
}

// one entry of the coarsest operator D K D + (I - D), symmetrised (loadpath/mg.py:735-740):
// row dof (ci at node ix, iy, iz), column dof (cj at node jx, jy, jz)
template <typename Tw>
__device__ __forceinline__ double coarse_entry(int kind, const Tw* __restrict__ w, const Tw* __restrict__ mcat,
                                               const int* __restrict__ patch_id, const Tw* __restrict__ patch_k,
                                               const Tw* __restrict__ k, const uint8_t* __restrict__ mask,
                                               const LpGrid& g, int ci, int ix, int iy, int iz, int cj, int jx,
                                               int jy, int jz) {
  double s = 0.0;
  if (abs(ix - jx) <= 1 && abs(iy - jy) <= 1 && abs(iz - jz) <= 1) {
    for (int kk = 0; kk < 8; ++kk) {
      int cx = ix - cx_(kk), cy = iy - cy_(kk), cz = iz - cz_(kk);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      int ox = jx - cx, oy = jy - cy, oz = jz - cz;
      if (ox < 0 || ox > 1 || oy < 0 || oy > 1 || oz < 0 || oz > 1) continue;
      int kj = ox | (oy << 1) | (oz << 2);
      long long c = g.cell(cx, cy, cz);
      int r1 = 3 * kk + ci, c1 = 3 * kj + cj;
      int e1 = r1 * 24 + c1, e2 = c1 * 24 + r1;
      double v1, v2;
      if (kind == 1) {
        v1 = v2 = 0.0;
        for (int q = 0; q < 8; ++q) {
          double wq = (double)w[q * g.cells_padded() + c];
          v1 += (double)mcat[q * 576 + e1] * wq;
          v2 += (double)mcat[q * 576 + e2] * wq;
        }
        int p = patch_id ? patch_id[c] : -1;
        if (p >= 0) {
          v1 += (double)patch_k[(long long)p * 576 + e1];
          v2 += (double)patch_k[(long long)p * 576 + e2];
        }
      } else {
        v1 = (double)k[c * 576 + e1];
        v2 = (double)k[c * 576 + e2];
      }
      s += 0.5 * (v1 + v2);
    }
  }
  double mi = ((mask[g.node(ix, iy, iz)] >> ci) & 1) ? 1.0 : 0.0;
  double mj = ((mask[g.node(jx, jy, jz)] >> cj) & 1) ? 1.0 : 0.0;
  double v = mi * s * mj;
  if (ci == cj && ix == jx && iy == jy && iz == jz) v += 1.0 - mi;
  return v;
}

// dense coarsest operator over every node of the level, dof (c, node) -> c * NN + node with
// node = (x * NY + y) * NZ + z
template <typename Tw>
__global__ void k_coarse_dense(double* __restrict__ a, int kind, const Tw* __restrict__ w,
                               const Tw* __restrict__ mcat, const int* __restrict__ patch_id,
                               const Tw* __restrict__ patch_k, const Tw* __restrict__ k,
                               const uint8_t* __restrict__ mask, LpGrid g) {
  const int NX = g.NX(), NY = g.NY(), NZ = g.NZ();
  const long long NN = (long long)NX * NY * NZ;
  const long long n = 3 * NN;
  (void)NX;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * n; t += (long long)gridDim.x * blockDim.x) {
    long long I = t / n, J = t % n;
    int ci = (int)(I / NN), cj = (int)(J / NN);
    long long ni = I % NN, nj = J % NN;
    int iz = (int)(ni % NZ), iy = (int)((ni / NZ) % NY), ix = (int)(ni / ((long long)NZ * NY));
    int jz = (int)(nj % NZ), jy = (int)((nj / NZ) % NY), jx = (int)(nj / ((long long)NZ * NY));
    a[t] = coarse_entry(kind, w, mcat, patch_id, patch_k, k, mask, g, ci, ix, iy, iz, cj, jx, jy, jz);
  }
}

// ---- the coarsest operator as a band (for lp_band.cu's Cholesky) ---------------------------
// Dofs are numbered 3 * node + component with the node's coordinates ordered so the longest
// axis varies slowest: the half-bandwidth is then 3 (N1 N2 + N2 + 1) + 2 for the two shorter
// extents N1 >= N2. The lower band is stored as 32 x 32 tiles: tile (R, d) holds rows
// 32R..32R+31, columns 32(R-d)..32(R-d)+31, row-major, at t + (R (D + 1) + d) 1024; dofs past n
// (padding to a multiple of 32) are identity rows.
template <typename Tw>
__global__ void k_coarse_band(double* __restrict__ t, int kind, const Tw* __restrict__ w, const Tw* __restrict__ mcat,
                              const int* __restrict__ patch_id, const Tw* __restrict__ patch_k,
                              const Tw* __restrict__ k, const uint8_t* __restrict__ mask, LpGrid g, LpBand bd) {
  const long long total = (long long)bd.nt * (bd.D + 1) * 1024;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int rc = (int)(e & 1023);
    const long long td = e >> 10;
    const int d = (int)(td % (bd.D + 1));
    const int R = (int)(td / (bd.D + 1));
    const long long i = 32LL * R + (rc >> 5), j = 32LL * (R - d) + (rc & 31);
    double v = 0.0;
    if (j >= 0 && j <= i) {
      if (i >= bd.n || j >= bd.n) {
        v = i == j ? 1.0 : 0.0;
      } else {
        int ix, iy, iz, jx, jy, jz;
        bd.coords(i / 3, ix, iy, iz);
        bd.coords(j / 3, jx, jy, jz);
        v = coarse_entry(kind, w, mcat, patch_id, patch_k, k, mask, g, (int)(i % 3), ix, iy, iz, (int)(j % 3), jx, jy,
                         jz);
      }
    }
    t[e] = v;
  }
}

// Level-2 Galerkin matrices from level-1 weights, plain hierarchy (loadpath/mg.py:639-663 with a
// weights fine level): K(C) = sum_k P_k^T (sum_q w_(k,q) M_q) P_k = sum_(k,q) w_(k,q) N_(k,q) with
// the 64 fixed products N_(k,q) = P_k^T M_q P_k (nkq: (64, 576), index 8 k + q), w_(k,q) the
// weight q of child k. A thread owns one of the 576 entries and keeps its 64 coefficients in
// registers; a block walks CB cells at a time (float64 accumulation). Children that carry a
// patch matrix (weights zero) are added by k_galerkin_patch_add.
template <typename Tw>
__global__ void __launch_bounds__(288, 1) k_galerkin_w2(Tw* __restrict__ kout, const Tw* __restrict__ w1,
                                                        const Tw* __restrict__ nkq, LpGrid gf, LpGrid gc) {
  constexpr int CB = 4;
  __shared__ __align__(16) double ws[CB][64];   // float64 here: the inner loop converts nothing
  const int e = blockIdx.y * 288 + threadIdx.x;
  double nr[64];
#pragma unroll
  for (int kq = 0; kq < 64; ++kq) nr[kq] = (double)__ldg(nkq + kq * 576 + e);
  const long long ncell = (long long)gc.nx * gc.ny * gc.nz;
  const long long ncp1 = gf.cells_padded();
  const int hx = gf.nx / 2, hy = gf.ny / 2, hz = gf.nz / 2;
  for (long long c0 = (long long)blockIdx.x * CB; c0 < ncell; c0 += (long long)gridDim.x * CB) {
    __syncthreads();
    for (int i = threadIdx.x; i < CB * 64; i += blockDim.x) {
      const int cb = i >> 6, kq = i & 63, k = kq >> 3, q = kq & 7;
      const long long cid = c0 + cb;
      double v = 0.0;
      if (cid < ncell) {
        const int Z = (int)(cid % gc.nz);
        const long long r = cid / gc.nz;
        const int Y = (int)(r % gc.ny), X = (int)(r / gc.ny);
        if (X < hx && Y < hy && Z < hz)
          v = (double)w1[q * ncp1 + gf.cell(2 * X + cx_(k), 2 * Y + cy_(k), 2 * Z + cz_(k))];
      }
      ws[cb][kq] = v;
    }
    __syncthreads();
#pragma unroll
    for (int cb = 0; cb < CB; ++cb) {
      const long long cid = c0 + cb;
      if (cid >= ncell) break;
      double a0 = 0.0, a1 = 0.0;
      const double2* w2 = reinterpret_cast<const double2*>(ws[cb]);
#pragma unroll
      for (int kk = 0; kk < 32; ++kk) {
        const double2 wv = w2[kk];
        a0 += nr[2 * kk] * wv.x;
        a1 += nr[2 * kk + 1] * wv.y;
      }
      const int Z = (int)(cid % gc.nz);
      const long long r = cid / gc.nz;
      const int Y = (int)(r % gc.ny), X = (int)(r / gc.ny);
      kout[gc.cell(X, Y, Z) * 576 + e] = (Tw)(a0 + a1);
    }
  }
}

// adds P_k^T patch P_k for every child k of coarse cell C that carries a patch matrix (after
// k_galerkin_w2); one block per coarse cell, most return at once
template <typename Tw>
__global__ void k_galerkin_patch_add(Tw* __restrict__ kout, const int* __restrict__ patch_id,
                                     const Tw* __restrict__ patch_k, LpGrid gf, LpGrid gc) {
  __shared__ double kf[576];
  __shared__ double tt[576];
  __shared__ int pids[8];
  const long long bid = blockIdx.x;
  const long long ncell = (long long)gc.nx * gc.ny * gc.nz;
  if (bid >= ncell) return;
  const int Z = (int)(bid % gc.nz);
  const long long q0 = bid / gc.nz;
  const int Y = (int)(q0 % gc.ny), X = (int)(q0 / gc.ny);
  const int hx = gf.nx / 2, hy = gf.ny / 2, hz = gf.nz / 2;
  if (!(X < hx && Y < hy && Z < hz)) return;
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    pids[k] = patch_id[gf.cell(2 * X + cx_(k), 2 * Y + cy_(k), 2 * Z + cz_(k))];
  }
  __syncthreads();
  bool any = false;
  for (int k = 0; k < 8; ++k) any = any || pids[k] >= 0;
  if (!any) return;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  for (int k = 0; k < 8; ++k) {
    const int p = pids[k];
    if (p < 0) continue;
    for (int i = threadIdx.x; i < 576; i += blockDim.x) kf[i] = (double)patch_k[(long long)p * 576 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < 576; i += blockDim.x) {
      const int a = i / 24, j = i % 24, r = j / 3, cc = j % 3;
      double sacc = 0.0;
      for (int qq = 0; qq < 8; ++qq) sacc += kf[a * 24 + 3 * qq + cc] * pw(k, qq, r);
      tt[i] = sacc;
    }
    __syncthreads();
    for (int sidx = 0; sidx < 3; ++sidx) {
      const int i = threadIdx.x + sidx * 256;
      if (i >= 576) break;
      const int ii = i / 24, j = i % 24, r = ii / 3, cc = ii % 3;
      double v = 0.0;
      for (int qq = 0; qq < 8; ++qq) v += pw(k, qq, r) * tt[(3 * qq + cc) * 24 + j];
      if (sidx == 0) acc0 += v; else if (sidx == 1) acc1 += v; else acc2 += v;
    }
    __syncthreads();
  }
  const long long C = gc.cell(X, Y, Z);
  for (int sidx = 0; sidx < 3; ++sidx) {
    const int i = threadIdx.x + sidx * 256;
    if (i >= 576) break;
    kout[C * 576 + i] += (Tw)(sidx == 0 ? acc0 : sidx == 1 ? acc1 : acc2);
  }
}

}  // namespace

#define LP_FC_ARGS int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz
#define LP_GF lp_grid(fnx, fny, fnz, fpz, fcpz)
#define LP_GC lp_grid(cnx, cny, cnz, cpz_, ccpz)
#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)

extern "C" {

int lpb_weights_from_e_f64_f32(float* w, const double* e, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !w || !e) return LP_ERR_ARG;
  long long total = gc.cells_padded();
  k_weights_from_e<double, float><<<lp_blocks(total, 256), 256, 0, LP_ST>>>(w, e, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_weights_from_e_f64_f64(double* w, const double* e, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !w || !e) return LP_ERR_ARG;
  long long total = gc.cells_padded();
  k_weights_from_e<double, double><<<lp_blocks(total, 256), 256, 0, LP_ST>>>(w, e, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_patch_flags(uint8_t* flag, const double* e, const uint8_t* mf, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !flag || !e || !mf) return LP_ERR_ARG;
  long long total = gc.cells_padded();
  k_patch_flags<double><<<lp_blocks(total, 256), 256, 0, LP_ST>>>(flag, e, mf, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_patch_matrices_f32(float* pk, float* w, int* patch_id, const long long* pcells, int npatch, const double* e,
                           const double* ke, const uint8_t* mf, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || npatch < 0) return LP_ERR_ARG;
  if (npatch == 0) return LP_OK;
  k_patch_matrices<double, float><<<npatch, 256, 0, LP_ST>>>(pk, w, patch_id, pcells, npatch, e, ke, mf, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_patch_matrices_f64(double* pk, double* w, int* patch_id, const long long* pcells, int npatch,
                           const double* e, const double* ke, const uint8_t* mf, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || npatch < 0) return LP_ERR_ARG;
  if (npatch == 0) return LP_OK;
  k_patch_matrices<double, double><<<npatch, 256, 0, LP_ST>>>(pk, w, patch_id, pcells, npatch, e, ke, mf, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// level-2 Galerkin matrices from level-1 weights, plain hierarchy: nkq (64 x 576, index 8k + q)
// = P_k^T M_q P_k; patch_id / patch_k may be NULL when the fine level has no patch cells
#define LP_GAL_W2(T, SFX)                                                                                      \
  int lpb_galerkin_w2_##SFX(T* kout, const T* w1, const T* nkq, const int* patch_id, const T* patch_k,      \
                            LP_FC_ARGS, void* stream) {                                                      \
    LpGrid gf = LP_GF, gc = LP_GC;                                                                          \
    if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !kout || !w1 || !nkq) return LP_ERR_ARG;                   \
    const long long ncell = (long long)gc.nx * gc.ny * gc.nz;                                               \
    long long nb = (ncell + 3) / 4;                                                                         \
    if (nb > 148 * 8) nb = 148 * 8;                                                                         \
    k_galerkin_w2<T><<<dim3((unsigned)nb, 2), 288, 0, LP_ST>>>(kout, w1, nkq, gf, gc);                      \
    if (patch_id && patch_k)                                                                                \
      k_galerkin_patch_add<T><<<(unsigned)ncell, 256, 0, LP_ST>>>(kout, patch_id, patch_k, gf, gc);          \
    LP_LAUNCH_CHECK();                                                                                      \
    return LP_OK;                                                                                           \
  }
LP_GAL_W2(float, f32)
LP_GAL_W2(double, f64)

int lpb_galerkin_explicit_f32(float* kout, int fine_kind, const float* fw, const float* mcat, const int* patch_id,
                              const float* patch_k, const float* fk, const uint8_t* mf, int strict, LP_FC_ARGS,
                              void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !kout) return LP_ERR_ARG;
  if (fine_kind == 1 && (!fw || !mcat)) return LP_ERR_ARG;
  if (fine_kind == 2 && !fk) return LP_ERR_ARG;
  long long ncell = (long long)gc.nx * gc.ny * gc.nz;
  k_galerkin_explicit<float><<<(unsigned)ncell, 256, 0, LP_ST>>>(kout, fine_kind, fw, mcat, patch_id, patch_k, fk, mf,
                                                                 strict, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_galerkin_explicit_f64(double* kout, int fine_kind, const double* fw, const double* mcat, const int* patch_id,
                              const double* patch_k, const double* fk, const uint8_t* mf, int strict, LP_FC_ARGS,
                              void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !kout) return LP_ERR_ARG;
  if (fine_kind == 1 && (!fw || !mcat)) return LP_ERR_ARG;
  if (fine_kind == 2 && !fk) return LP_ERR_ARG;
  long long ncell = (long long)gc.nx * gc.ny * gc.nz;
  k_galerkin_explicit<double><<<(unsigned)ncell, 256, 0, LP_ST>>>(kout, fine_kind, fw, mcat, patch_id, patch_k, fk,
                                                                  mf, strict, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_strict_held_kept(uint8_t* held_c, float* kept, const uint8_t* held_f, const uint8_t* mf, LP_FC_ARGS,
                         void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !held_c || !kept || !held_f || !mf) return LP_ERR_ARG;
  long long total = gc.nodes_padded();
  k_strict_held_kept<<<lp_blocks(total, 256), 256, 0, LP_ST>>>(held_c, kept, held_f, mf, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_held0(uint8_t* held, const uint8_t* mask0, const uint8_t* fixed_bits, long long n, void* stream) {
  if (!held || !mask0 || !fixed_bits) return LP_ERR_ARG;
  k_held0<<<lp_blocks(n, 256), 256, 0, LP_ST>>>(held, mask0, fixed_bits, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_coarse_dense_f32(double* a, int kind, const float* w, const float* mcat, const int* patch_id,
                         const float* patch_k, const float* k, const uint8_t* mask, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !a || !mask) return LP_ERR_ARG;
  long long n = 3LL * g.NX() * g.NY() * g.NZ();
  if (n > 40000) return LP_ERR_SIZE;
  k_coarse_dense<float><<<lp_blocks(n * n, 256), 256, 0, LP_ST>>>(a, kind, w, mcat, patch_id, patch_k, k, mask, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_coarse_dense_f64(double* a, int kind, const double* w, const double* mcat, const int* patch_id,
                         const double* patch_k, const double* k, const uint8_t* mask, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !a || !mask) return LP_ERR_ARG;
  long long n = 3LL * g.NX() * g.NY() * g.NZ();
  if (n > 40000) return LP_ERR_SIZE;
  k_coarse_dense<double><<<lp_blocks(n * n, 256), 256, 0, LP_ST>>>(a, kind, w, mcat, patch_id, patch_k, k, mask, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// f = ainv * f on the coarsest level; v: scratch of 3 * nodes doubles
// the coarsest operator as band tiles (layout: lpb_band_dims); t: nt (D + 1) x 1024 doubles
int lpb_coarse_band_f32(double* t, int kind, const float* w, const float* mcat, const int* patch_id,
                        const float* patch_k, const float* k, const uint8_t* mask, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !t || !mask || (kind == 1 && (!w || !mcat)) || (kind == 2 && !k)) return LP_ERR_ARG;
  const LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  const long long total = (long long)bd.nt * (bd.D + 1) * 1024;
  k_coarse_band<float><<<lp_blocks(total, 256), 256, 0, LP_ST>>>(t, kind, w, mcat, patch_id, patch_k, k, mask, g, bd);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_coarse_band_f64(double* t, int kind, const double* w, const double* mcat, const int* patch_id,
                        const double* patch_k, const double* k, const uint8_t* mask, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !t || !mask || (kind == 1 && (!w || !mcat)) || (kind == 2 && !k)) return LP_ERR_ARG;
  const LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  const long long total = (long long)bd.nt * (bd.D + 1) * 1024;
  k_coarse_band<double><<<lp_blocks(total, 256), 256, 0, LP_ST>>>(t, kind, w, mcat, patch_id, patch_k, k, mask, g,
                                                                  bd);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
