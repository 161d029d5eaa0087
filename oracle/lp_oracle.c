/* TEST INFRASTRUCTURE ONLY: C restatement of the reference's compiled CPU operator, used as
 * the CPU baseline (bench.py --impl reference, and bench.py's cpu_baseline) and as a checker.
 * Never linked into or called by the product (loadpath_b200).
 *
 * lpo_apply_masked_{f64,f32}: out = m * K (m * u) + (1 - m) * u on the node grid
 * (3, nx+1, ny+1, nz+1), K = sum over cells of e[c] * ke, in the reference's two passes
 * (loadpath/mgops.py:247-261): a product pass over blocks of cells gathering their 24 corner
 * values (mask read in the gather) and multiplying by ke (loadpath/mgops.py:66-103), then a
 * node pass summing each node's up-to-8 cells' rows and finishing with the mask
 * (loadpath/mgops.py:181-217). OpenMP threads over blocks / (x, y) node columns.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BLOCK 256

#define DEFINE_APPLY(T, SFX)                                                                        \
  int lpo_apply_masked_##SFX(T* out, const T* u, const T* e, const T* m, const double* ke64,       \
                             int nx, int ny, int nz, T* ft) {                                        \
    const long long NX = nx + 1, NY = ny + 1, NZ = nz + 1;                                           \
    const long long nn = NX * NY * NZ, ncell = (long long)nx * ny * nz;                              \
    T ke[576];                                                                                       \
    for (int i = 0; i < 576; ++i) ke[i] = (T)ke64[i];                                                \
    long long off[24];                                                                               \
    for (int k = 0; k < 8; ++k)                                                                      \
      for (int d = 0; d < 3; ++d)                                                                    \
        off[3 * k + d] = d * nn + (k & 1) * NY * NZ + ((k >> 1) & 1) * NZ + ((k >> 2) & 1);          \
    const long long nblk = (ncell + BLOCK - 1) / BLOCK;                                              \
    _Pragma("omp parallel for schedule(static)")                                                     \
    for (long long b = 0; b < nblk; ++b) {                                                          \
      T ubt[24][BLOCK];                                                                              \
      long long c0 = b * BLOCK;                                                                      \
      int cnt = (int)((ncell - c0) < BLOCK ? (ncell - c0) : BLOCK);                                  \
      long long base[BLOCK];                                                                         \
      for (int c = 0; c < cnt; ++c) {                                                                \
        long long cell = c0 + c;                                                                     \
        long long z = cell % nz, y = (cell / nz) % ny, x = cell / ((long long)nz * ny);              \
        base[c] = (x * NY + y) * NZ + z;                                                             \
      }                                                                                              \
      for (int i = 0; i < 24; ++i)                                                                   \
        for (int c = 0; c < cnt; ++c) {                                                              \
          long long k = base[c] + off[i];                                                            \
          ubt[i][c] = u[k] * m[k];                                                                   \
        }                                                                                            \
      for (int i = 0; i < 24; ++i) {                                                                 \
        T* fr = ft + (long long)i * ncell + c0;                                                      \
        for (int c = 0; c < cnt; ++c) fr[c] = 0;                                                     \
        for (int j = 0; j < 24; ++j) {                                                               \
          T kij = ke[i * 24 + j];                                                                    \
          for (int c = 0; c < cnt; ++c) fr[c] += kij * ubt[j][c];                                    \
        }                                                                                            \
        for (int c = 0; c < cnt; ++c) fr[c] *= e[c0 + c];                                            \
      }                                                                                              \
    }                                                                                                \
    _Pragma("omp parallel for schedule(static)")                                                     \
    for (long long xy = 0; xy < NX * NY; ++xy) {                                                     \
      long long x = xy / NY, y = xy % NY;                                                            \
      for (long long z = 0; z < NZ; ++z) {                                                           \
        T a[3] = {0, 0, 0};                                                                          \
        for (int k = 0; k < 8; ++k) {                                                                \
          long long cx = x - (k & 1), cy = y - ((k >> 1) & 1), cz = z - ((k >> 2) & 1);              \
          if (cx < 0 || cy < 0 || cz < 0 || cx >= nx || cy >= ny || cz >= nz) continue;              \
          long long r = (cx * ny + cy) * nz + cz;                                                    \
          for (int d = 0; d < 3; ++d) a[d] += ft[(long long)(3 * k + d) * ncell + r];                \
        }                                                                                            \
        long long n = (x * NY + y) * NZ + z;                                                         \
        for (int d = 0; d < 3; ++d) {                                                                \
          T md = m[d * nn + n];                                                                      \
          out[d * nn + n] = a[d] * md + (1 - md) * u[d * nn + n];                                    \
        }                                                                                            \
      }                                                                                              \
    }                                                                                                \
    return 0;                                                                                        \
  }

DEFINE_APPLY(double, f64)
DEFINE_APPLY(float, f32)

int lpo_threads(void) {
  int n = 1;
#ifdef _OPENMP
#pragma omp parallel
  {
#pragma omp single
    n = omp_get_num_threads();
  }
#endif
  return n;
}

/* lpo_apply_weights_f32: the level-1 ("weights") operator of the reference's hierarchy,
 * out = m * K1 (m * u) + (1 - m) * u on the coarse node grid, K1 = sum over cells of
 * sum_k w[k, c] M_k (M_k = P_k^T ke P_k, the eight children's Galerkin matrices) plus the patch
 * cells' explicit matrices (loadpath/mg.py:213-230, :251-276, :317-346; loadpath/mgops.py:247-261):
 * a product pass over blocks of cells (the masked corner values gathered once, the eight
 * children's products weighted and summed), the node pass, the patch cells' products added
 * node by node (serially, in the patch list's order), then the mask finish.
 * w: (8, cells) in C order over (x, y, z); mcat64: (8, 24, 24); pidx: (np, 24) flat
 * (component nn + node) dof indices of the patch cells; pk: (np, 24, 24). */
int lpo_apply_weights_f32(float* out, const float* u, const float* w, const double* mcat64, const float* m,
                          int nx, int ny, int nz, const long long* pidx, const float* pk, long long np,
                          float* ft) {
  const long long NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  const long long nn = NX * NY * NZ, ncell = (long long)nx * ny * nz;
  float mk[8 * 576];
  for (int i = 0; i < 8 * 576; ++i) mk[i] = (float)mcat64[i];
  long long off[24];
  for (int k = 0; k < 8; ++k)
    for (int d = 0; d < 3; ++d) off[3 * k + d] = d * nn + (k & 1) * NY * NZ + ((k >> 1) & 1) * NZ + ((k >> 2) & 1);
  const long long nblk = (ncell + BLOCK - 1) / BLOCK;
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < nblk; ++b) {
    float ubt[24][BLOCK], g[BLOCK];
    long long c0 = b * BLOCK;
    int cnt = (int)((ncell - c0) < BLOCK ? (ncell - c0) : BLOCK);
    long long base[BLOCK];
    for (int c = 0; c < cnt; ++c) {
      long long cell = c0 + c;
      long long z = cell % nz, y = (cell / nz) % ny, x = cell / ((long long)nz * ny);
      base[c] = (x * NY + y) * NZ + z;
    }
    for (int i = 0; i < 24; ++i)
      for (int c = 0; c < cnt; ++c) {
        long long k = base[c] + off[i];
        ubt[i][c] = u[k] * m[k];
      }
    for (int i = 0; i < 24; ++i) {
      float* fr = ft + (long long)i * ncell + c0;
      for (int c = 0; c < cnt; ++c) fr[c] = 0.0f;
      for (int k = 0; k < 8; ++k) {
        const float* wk = w + (long long)k * ncell + c0;
        for (int c = 0; c < cnt; ++c) g[c] = 0.0f;
        for (int j = 0; j < 24; ++j) {
          float kij = mk[(k * 24 + i) * 24 + j];
          for (int c = 0; c < cnt; ++c) g[c] += kij * ubt[j][c];
        }
        for (int c = 0; c < cnt; ++c) fr[c] += g[c] * wk[c];
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (long long xy = 0; xy < NX * NY; ++xy) {
    long long x = xy / NY, y = xy % NY;
    for (long long z = 0; z < NZ; ++z) {
      float a[3] = {0, 0, 0};
      for (int k = 0; k < 8; ++k) {
        long long cx = x - (k & 1), cy = y - ((k >> 1) & 1), cz = z - ((k >> 2) & 1);
        if (cx < 0 || cy < 0 || cz < 0 || cx >= nx || cy >= ny || cz >= nz) continue;
        long long r = (cx * ny + cy) * nz + cz;
        for (int d = 0; d < 3; ++d) a[d] += ft[(long long)(3 * k + d) * ncell + r];
      }
      long long n = (x * NY + y) * NZ + z;
      for (int d = 0; d < 3; ++d) out[d * nn + n] = a[d];
    }
  }
  for (long long p = 0; p < np; ++p) {
    const long long* id = pidx + p * 24;
    float ue[24];
    for (int j = 0; j < 24; ++j) ue[j] = u[id[j]] * m[id[j]];
    for (int i = 0; i < 24; ++i) {
      float s = 0.0f;
      for (int j = 0; j < 24; ++j) s += pk[(p * 24 + i) * 24 + j] * ue[j];
      out[id[i]] += s;
    }
  }
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < 3 * nn; ++i) out[i] = out[i] * m[i] + (1.0f - m[i]) * u[i];
  return 0;
}

/* lpo_coarse_residual_f32 / lpo_add_correction_f32: the V-cycle's transfers between a level and
 * the next coarser one in float32 (loadpath/mgops.py:666-711, :753-773). The coarse residual
 * rc = cm * R((b - ax) * m), R the transpose of trilinear prolongation over the fine nodes (a
 * coarse node sums the fine nodes within one step of its fine twin, weights 1, 1/2, 1/4, 1/8 by
 * the number of odd offsets; fine nodes past the fine grid count zero); the correction
 * x += m * P(cm * xc), a fine node taking its one to eight coarse neighbours' values at those
 * weights. Fields (3, n0, n1, n2) in C order; fine (3, F0, F1, F2), coarse (3, C0, C1, C2). */
int lpo_coarse_residual_f32(float* rc, const float* b, const float* ax, const float* m, const float* cm,
                            int F0, int F1, int F2, int C0, int C1, int C2) {
  const long long nf = (long long)F0 * F1 * F2, nc = (long long)C0 * C1 * C2;
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < 3 * nc; ++t) {
    const long long d = t / nc, r = t % nc;
    const long long I = r / ((long long)C1 * C2), J = (r / C2) % C1, K = r % C2;
    float s = 0.0f;
    for (int di = -1; di <= 1; ++di) {
      const long long i = 2 * I + di;
      if (i < 0 || i >= F0) continue;
      for (int dj = -1; dj <= 1; ++dj) {
        const long long j = 2 * J + dj;
        if (j < 0 || j >= F1) continue;
        for (int dk = -1; dk <= 1; ++dk) {
          const long long k = 2 * K + dk;
          if (k < 0 || k >= F2) continue;
          const float w = (di ? 0.5f : 1.0f) * (dj ? 0.5f : 1.0f) * (dk ? 0.5f : 1.0f);
          const long long f = d * nf + (i * F1 + j) * F2 + k;
          s += w * ((b[f] - ax[f]) * m[f]);
        }
      }
    }
    rc[t] = s * cm[t];
  }
  return 0;
}

int lpo_add_correction_f32(float* x, const float* xc, const float* cm, const float* m, int F0, int F1, int F2,
                           int C0, int C1, int C2) {
  const long long nf = (long long)F0 * F1 * F2, nc = (long long)C0 * C1 * C2;
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < 3 * nf; ++t) {
    const long long d = t / nf, r = t % nf;
    const long long i = r / ((long long)F1 * F2), j = (r / F2) % F1, k = r % F2;
    const long long i0 = i / 2, j0 = j / 2, k0 = k / 2;
    const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
    const float wi = (i & 1) ? 0.5f : 1.0f, wj = (j & 1) ? 0.5f : 1.0f, wk = (k & 1) ? 0.5f : 1.0f;
    float s = 0.0f;
    for (int a = 0; a < ni; ++a) {
      if (i0 + a >= C0) continue;
      for (int bb = 0; bb < nj; ++bb) {
        if (j0 + bb >= C1) continue;
        for (int c = 0; c < nk; ++c) {
          if (k0 + c >= C2) continue;
          const long long q = d * nc + ((i0 + a) * C1 + (j0 + bb)) * C2 + (k0 + c);
          s += wi * wj * wk * (xc[q] * cm[q]);
        }
      }
    }
    x[t] += s * m[t];
  }
  return 0;
}
