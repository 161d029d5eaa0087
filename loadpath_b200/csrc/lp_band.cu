// The coarsest level's direct solve (loadpath/mg.py:708-766: the reference factors D K D + (I - D)
// with SuperLU on the host, in symmetric mode without pivoting). Here the operator is a band (a
// 27-point block stencil whose nodes are numbered longest axis slowest, half-bandwidth
// 3 (N1 N2 + N2 + 1) + 2 dofs), so:
//   1. k_band_factor: signed Cholesky A = L S L^T (S = diag(+-1): a symmetric LU without pivoting,
//      failing only on an exactly zero pivot, as SuperLU does) of the band stored as 32 x 32
//      tiles (tile (R, d) = rows 32R.., columns 32(R - d)..), left-looking by tile rows as a
//      dataflow: each block owns tile rows and waits only on the progress counts of the rows it
//      reads (no grid-wide barrier). A diagonal tile is factored by one warp in registers; its
//      lower-triangular inverse (for step 2) is formed after the row is published.
//   2. k_band_inverse: A^-1 = L^-T S L^-1 applied to the identity, 32 columns per block: a
//      forward then a backward block substitution over the band tiles. Only the lower triangle
//      is needed (rows >= the block's first column); k_sym_lower copies it across.
//   3. per V-cycle: gather the level's field into the band numbering, one GEMV with the dense
//      inverse, scatter back (the inverse stays resident; a GEMV has no sequential chain).
// The factorisation costs O(n bw^2) instead of the dense O(n^3): at the 17 x 9 x 9-node coarsest
// level of a 256 x 128 x 128 grid, n = 4131 and bw = 275.
#include "lp_common.cuh"

#define LP_BAR_LIMIT (1u << 22)   // polls before a progress wait gives up and flags an error

namespace {

__device__ __forceinline__ double* tile_at(double* t, const LpBand& bd, int R, int d) {
  return t + ((long long)R * (bd.D + 1) + d) * 1024;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block-wide: wait until prog[row] > need (thread 0 polls with acquire loads, bounded); seen
// keeps the last value read (the same in every thread), so a later wait on the same row with a
// smaller need returns at once. False when a wait gave up (err is set).
__device__ bool wait_row(const unsigned* prog, int row, unsigned need, unsigned& seen, int* err) {
  __shared__ int ok_s;
  __shared__ unsigned seen_s;
  if (seen > need) return true;
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned v = ld_acquire(prog + row), it = 0;
    while (v <= need) {
      if (++it > LP_BAR_LIMIT) {
        ok = 0;
        atomicExch(err, 1);
        break;
      }
      if (it > 64) __nanosleep(32);
      v = ld_acquire(prog + row);
    }
    ok_s = ok;
    seen_s = v;
  }
  __syncthreads();
  seen = seen_s;
  const bool ok = ok_s != 0;
  __syncthreads();   // ok_s / seen_s are rewritten by the next wait
  return ok;
}

// row R of the factor now has its first v tile columns: tiles stored by every thread of the
// block are made visible before the count
__device__ __forceinline__ void publish_row(unsigned* prog, int row, unsigned v) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(prog + row, v);
  }
}

// Tiles another block wrote are read with ld.global.cg (L2, not a possibly stale L1 line).

// Signed Cholesky A = L S L^T (S = diag(+-1)) of one 32 x 32 diagonal tile (lower part read) by
// warp 0: lane i holds row i in registers. Each pivot p gives L_jj = sqrt|p| and S_j = sign(p),
// so negative pivots are factored as they are: a symmetric LU without pivoting, as the
// reference's SuperLU in symmetric mode (loadpath/mg.py:744-747). Writes L (upper part zero) over
// the tile and into sm, and S to sg[0..31]. A pivot that is exactly zero (or not finite) records
// its dof (1-based) in *info: the operator is singular; the arithmetic continues.
__device__ void factor_diag(double* __restrict__ tile, double* __restrict__ sg, long long row0, int* info,
                            double (*sm)[33]) {
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    double a[32];
    int bad = 0;
#pragma unroll
    for (int m = 0; m < 32; ++m) a[m] = m <= i ? __ldcg(tile + i * 32 + m) : 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const double p = __shfl_sync(0xffffffffu, a[j], j);
      if (!(fabs(p) > 0.0) && bad == 0) bad = (int)(row0 + j + 1);
      const double sj = p < 0.0 ? -1.0 : 1.0, ap = fabs(p);
      if (i == j) sg[j] = sj;
      // one reciprocal square root per pivot on the chain (not a square root and a division)
      const double rd = rsqrt(ap), d = ap * rd;
      const double l = i > j ? a[j] * rd * sj : (i == j ? d : 0.0);
      const double ls = l * sj;
      a[j] = l;
#pragma unroll
      for (int t = j + 1; t < 32; ++t) {   // entries above the diagonal of row i take garbage
        const double lt = __shfl_sync(0xffffffffu, l, t);   // here; a[t] is zeroed before use
        a[t] -= ls * lt;                                     // (l = 0 at pivot t > i)
      }
    }
    if (i == 0 && bad) atomicCAS(info, 0, bad);
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      const double v = m <= i ? a[m] : 0.0;
      tile[i * 32 + m] = v;
      sm[i][m] = v;
    }
    __syncwarp();
  }
}

// linv (row-major) = L^-1 of the diagonal factor in sm (factor_diag's copy), by warp 0: lane c
// forms column c, right-looking (the 32 row updates of a step are independent). The inverse is
// for k_band_inverse; the factorisation itself solves its panels against L.
__device__ void diag_inverse(double* __restrict__ linv, const double (*sm)[33]) {
  if (threadIdx.x < 32) {
    const int c = threadIdx.x;
    const double rd = 1.0 / sm[c][c];
    double x[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) x[r] = r == c ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      const double xm = x[m] * __shfl_sync(0xffffffffu, rd, m);
      x[m] = m >= c ? xm : 0.0;
#pragma unroll
      for (int r = m + 1; r < 32; ++r) x[r] -= sm[r][m] * x[m];
    }
#pragma unroll
    for (int r = 0; r < 32; ++r) linv[r * 32 + c] = x[r];
  }
}

// This thread's four entries x[q] of a 32 x 32 tile (entry e = threadIdx.x + 256 q, row e / 32,
// column e % 32) -= a S b^T, with a, b tiles in global memory (read through L2) and S the
// pivot signs of their column block.
__device__ void sub_product(double (&x)[4], const double* __restrict__ a, const double* __restrict__ b,
                            const double* __restrict__ sg, double (*sa)[33], double (*sb)[33]) {
  __syncthreads();   // the previous product is done with sa / sb
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    sa[e >> 5][e & 31] = __ldcg(a + e);
    sb[e >> 5][e & 31] = __ldcg(b + e) * __ldcg(sg + (e & 31));
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q, r = e >> 5, c = e & 31;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int m = 0; m < 32; m += 4) {
      s0 += sa[r][m] * sb[c][m];
      s1 += sa[r][m + 1] * sb[c][m + 1];
      s2 += sa[r][m + 2] * sb[c][m + 2];
      s3 += sa[r][m + 3] * sb[c][m + 3];
    }
    x[q] -= (s0 + s1) + (s2 + s3);
  }
}

// y -= l S l^T for the tile l this block holds in registers (four entries per thread, as x)
__device__ void sub_self_product(double (&y)[4], const double (&l)[4], const double* __restrict__ sg,
                                 double (*sa)[33], double (*sb)[33]) {
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q;
    sa[e >> 5][e & 31] = l[q];
    sb[e >> 5][e & 31] = l[q] * __ldcg(sg + (e & 31));
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + 256 * q, r = e >> 5, c = e & 31;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int m = 0; m < 32; m += 4) {
      s0 += sa[r][m] * sb[c][m];
      s1 += sa[r][m + 1] * sb[c][m + 1];
      s2 += sa[r][m + 2] * sb[c][m + 2];
      s3 += sa[r][m + 3] * sb[c][m + 3];
    }
    y[q] -= (s0 + s1) + (s2 + s3);
  }
}

// x = x L_cc^-T S_c (the panel solve L_Rc = X L_cc^-T S_c) by forward substitution against the
// diagonal factor tile lc: warp w holds rows w, w + 8, w + 16, w + 24 of x (x[q], the lane is the
// column), so each step is a shuffle and a multiply-add per row, no inverse on the chain.
__device__ void solve_panel(double (&x)[4], const double* __restrict__ lc, const double* __restrict__ sg,
                            double (*sb)[33]) {
  __syncthreads();
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) sb[e >> 5][e & 31] = __ldcg(lc + e);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const double rd = 1.0 / sb[lane][lane];
  double y[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    const double rm = __shfl_sync(0xffffffffu, rd, m);
    const double lm = sb[lane][m];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double ym = __shfl_sync(0xffffffffu, x[q], m) * rm;
      if (lane == m) y[q] = ym;
      if (lane > m) x[q] -= ym * lm;
    }
  }
  const double s = __ldcg(sg + lane);
#pragma unroll
  for (int q = 0; q < 4; ++q) x[q] = y[q] * s;
}

// Left-looking band factorisation by tile rows, as a dataflow: block b owns tile rows
// R = b, b + gridDim.x, ... and works through each row's tiles left to right,
//   L_Rc = (A_Rc - sum_j L_Rj S_j L_cj^T) L_cc^-T S_c     (c = R - D .. R - 1, j = max(R, c) - D .. c - 1)
//   L_RR S_R L_RR^T = A_RR - sum_j L_Rj S_j L_Rj^T         (factored by warp 0, factor_diag)
// publishing prog[R] = the number of tile columns of row R done after each tile. A tile waits
// only for the rows it reads (prog[c] > j for L_cj, prog[c] > c for L_cc^-1), so the chain from
// one row to the next is one panel solve (forward substitution against L_cc), one product and
// one diagonal factor; the diagonal tile's other terms are summed as the row's tiles come out. prog: nt zeroed words; every block
// must be resident (a cooperative launch); err: set when a wait gave up.
__global__ void __launch_bounds__(256, 1) k_band_factor(double* __restrict__ t, double* __restrict__ linv,
                                                        double* __restrict__ sg, LpBand bd, int* __restrict__ info,
                                                        unsigned* __restrict__ prog, int* __restrict__ err) {
  __shared__ double sa[32][33];
  __shared__ double sb[32][33];
  for (int R = blockIdx.x; R < bd.nt; R += gridDim.x) {
    const int c0 = R - bd.D > 0 ? R - bd.D : 0;
    double y[4];   // the diagonal tile, its terms subtracted as the row's tiles are formed
    const double* tr0 = tile_at(t, bd, R, 0);
#pragma unroll
    for (int q = 0; q < 4; ++q) y[q] = __ldcg(tr0 + threadIdx.x + 256 * q);
    for (int c = c0; c < R; ++c) {
      double* trc = tile_at(t, bd, R, R - c);
      double x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = __ldcg(trc + threadIdx.x + 256 * q);
      unsigned seen = 0;
      const int j0 = c - bd.D > c0 ? c - bd.D : c0;
      for (int j = j0; j < c; ++j) {
        if (!wait_row(prog, c, (unsigned)j, seen, err)) return;   // row c has its column j
        sub_product(x, tile_at(t, bd, R, R - j), tile_at(t, bd, c, c - j), sg + 32LL * j, sa, sb);
      }
      if (!wait_row(prog, c, (unsigned)c, seen, err)) return;     // row c's diagonal factor
      solve_panel(x, tile_at(t, bd, c, 0), sg + 32LL * c, sb);
#pragma unroll
      for (int q = 0; q < 4; ++q) trc[threadIdx.x + 256 * q] = x[q];
      publish_row(prog, R, (unsigned)(c + 1));
      sub_self_product(y, x, sg + 32LL * c, sa, sb);
    }
    double* tr0w = tile_at(t, bd, R, 0);
#pragma unroll
    for (int q = 0; q < 4; ++q) tr0w[threadIdx.x + 256 * q] = y[q];
    __syncthreads();
    factor_diag(tr0w, sg + 32LL * R, 32LL * R, info, sa);
    publish_row(prog, R, (unsigned)(R + 1));
    diag_inverse(linv + 1024LL * R, sa);   // off the chain: the next rows only need L
  }
}

// FP64 tensor-core MMA, m8n8k4 (row-major A 8 x 4, column-major B 4 x 8, C/D 8 x 8). Lane l holds
// A[l >> 2][l & 3], B[l & 3][l >> 2] and D[l >> 2][2 (l & 3) + i], i = 0, 1.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Columns j0..j0+31 of A^-1 (rows >= the first column's tile row) into ainv (n_pad x n_pad,
// row-major), A = L S L^T: Y = L^-1 E by forward substitution, then X = L^-T S Y backwards, one tile row per
// step. A step stages, in chunks of at most `chunk` pairs, its band tiles (8 KB each) with the
// matching earlier result blocks (read back from ainv through L2) in shared memory; each of 16
// warps forms one 8 x 8 block of the 32 x 32 result with FP64 MMAs:
//   forward  S = E - sum_d T_(k,d) Y_(k-d),      Y_k = L_kk^-1 S
//   backward S = S_k Y_k - sum_d T_(k+d,d)^T X_(k+d), X_k = L_kk^-T S   (S_k: the pivot signs)
// Shared row strides of 36 doubles spread each MMA operand load over all banks.
// 16-byte asynchronous copies global -> shared through L2 (cp.async.cg): a step issues all its
// loads at once and waits once, instead of a chain of dependent load rounds
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

constexpr int INV_COLS = 32;
constexpr int INV_LD = 36;
constexpr int INV_TILE = 32 * INV_LD;   // doubles per staged 32 x 32 block

__global__ void __launch_bounds__(512, 1) k_band_inverse(double* __restrict__ ainv, const double* __restrict__ t,
                                                         const double* __restrict__ linv, const double* __restrict__ sg,
                                                         LpBand bd, int chunk) {
  extern __shared__ __align__(16) double sm_inv[];
  double* tiles = sm_inv;                           // chunk band tiles
  double* blks = sm_inv + (long long)chunk * INV_TILE;  // chunk result blocks
  double* diag = blks + (long long)chunk * INV_TILE;    // L_kk^-1
  double* tmp = diag + INV_TILE;                         // S
  const int R1 = bd.D + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int row0 = 8 * (w >> 2), col0 = 8 * (w & 3);
  const int orow = row0 + g, ocol = col0 + 2 * q;   // this lane's two outputs: (orow, ocol + i)
  const long long np = 32LL * bd.nt;
  const int j0 = INV_COLS * blockIdx.x;
  const int kb = j0 >> 5;
  for (int pass = 0; pass < 2; ++pass) {
    const bool fwd = pass == 0;
    for (int step = 0; step < bd.nt - kb; ++step) {
      const int k = fwd ? kb + step : bd.nt - 1 - step;
      const int dm = fwd ? min(bd.D, k - kb) : min(bd.D, bd.nt - 1 - k);
      double p0 = 0.0, p1 = 0.0, r0 = 0.0, r1 = 0.0;
      for (int d0 = 1; d0 <= dm; d0 += chunk) {
        const int nc = min(chunk, dm - d0 + 1);
        // pairs of doubles: every offset below is a multiple of 16 bytes (row strides of 32 and
        // 36 doubles, n_pad a multiple of 32, j0 a multiple of 32, cc even)
        for (int e = threadIdx.x; e < nc * 512; e += blockDim.x) {
          const int d = d0 + (e >> 9), rr = (e >> 4) & 31, cc = 2 * (e & 15);
          const long long tk = fwd ? k : k + d;   // band tile (tk, d)
          const long long bk = fwd ? k - d : k + d;   // earlier result block
          cp_async16(tiles + (e >> 9) * INV_TILE + rr * INV_LD + cc, t + (tk * R1 + d) * 1024 + rr * 32 + cc);
          cp_async16(blks + (e >> 9) * INV_TILE + rr * INV_LD + cc, ainv + (32 * bk + rr) * np + j0 + cc);
        }
        if (d0 == 1)
          for (int e = threadIdx.x; e < 512; e += blockDim.x)
            cp_async16(diag + (e >> 4) * INV_LD + 2 * (e & 15), linv + (long long)k * 1024 + 2 * e);
        cp_async_wait_all();
        __syncthreads();
        for (int c = 0; c < nc; ++c) {
          const double* tc = tiles + c * INV_TILE;
          const double* yb = blks + c * INV_TILE + q * INV_LD + col0 + g;
          if (fwd) {
            const double* ta = tc + (row0 + g) * INV_LD + q;
#pragma unroll
            for (int m = 0; m < 32; m += 8) {
              dmma(p0, p1, ta[m], yb[m * INV_LD]);
              dmma(r0, r1, ta[m + 4], yb[(m + 4) * INV_LD]);
            }
          } else {
            const double* ta = tc + q * INV_LD + row0 + g;   // A[row][m] = T[m][row]
#pragma unroll
            for (int m = 0; m < 32; m += 8) {
              dmma(p0, p1, ta[m * INV_LD], yb[m * INV_LD]);
              dmma(r0, r1, ta[(m + 4) * INV_LD], yb[(m + 4) * INV_LD]);
            }
          }
        }
        __syncthreads();
      }
      if (dm == 0) {
        for (int e = threadIdx.x; e < 1024; e += blockDim.x)
          diag[(e >> 5) * INV_LD + (e & 31)] = __ldg(linv + (long long)k * 1024 + e);
      }
      double* out = ainv + (32LL * k + orow) * np + j0 + ocol;
      if (fwd) {
        const long long gr = 32LL * k + orow;
        tmp[orow * INV_LD + ocol] = (gr == j0 + ocol ? 1.0 : 0.0) - (p0 + r0);
        tmp[orow * INV_LD + ocol + 1] = (gr == j0 + ocol + 1 ? 1.0 : 0.0) - (p1 + r1);
      } else {
        const double2 yk = __ldcg(reinterpret_cast<const double2*>(out));
        const double sr = __ldg(sg + 32LL * k + orow);
        tmp[orow * INV_LD + ocol] = sr * yk.x - (p0 + r0);
        tmp[orow * INV_LD + ocol + 1] = sr * yk.y - (p1 + r1);
      }
      __syncthreads();
      double y0 = 0.0, y1 = 0.0;
      if (fwd) {
#pragma unroll
        for (int m = 0; m < 32; m += 4)
          dmma(y0, y1, diag[(row0 + g) * INV_LD + m + q], tmp[(m + q) * INV_LD + col0 + g]);
      } else {
#pragma unroll
        for (int m = 0; m < 32; m += 4)   // A = L_kk^-T
          dmma(y0, y1, diag[(m + q) * INV_LD + row0 + g], tmp[(m + q) * INV_LD + col0 + g]);
      }
      *reinterpret_cast<double2*>(out) = make_double2(y0, y1);
      __syncthreads();
    }
  }
}

// a[i][j] = a[j][i] for i < j (copy the lower triangle onto the upper), 32 x 32 tiles via
// shared memory; block (bi, bj) with bi <= bj writes tile (bi, bj)
__global__ void k_sym_lower(double* __restrict__ a, long long np) {
  __shared__ double s[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
  for (int r = ty; r < 32; r += 8) s[r][tx] = a[(32LL * bj + r) * np + 32LL * bi + tx];   // tile (bj, bi)
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long i = 32LL * bi + r, j = 32LL * bj + tx;
    if (i < j) a[i * np + j] = s[tx][r];
  }
}

// v[i] = field at band dof i (0 past n)
template <typename T>
__global__ void k_field_to_band(double* __restrict__ v, const T* __restrict__ f, LpGrid g, LpBand bd) {
  const long long np = 32LL * bd.nt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x) {
    double x = 0.0;
    if (i < bd.n) {
      int nx_, ny_, nz_;
      bd.coords(i / 3, nx_, ny_, nz_);
      x = (double)f[(i % 3) * g.comp_stride() + g.node(nx_, ny_, nz_)];
    }
    v[i] = x;
  }
}

// field at band dof i = row i of ainv . v, one warp per row
template <typename T>
__global__ void k_band_gemv_to_field(T* __restrict__ f, const double* __restrict__ a, const double* __restrict__ v,
                                     LpGrid g, LpBand bd) {
  const long long np = 32LL * bd.nt;
  const int lane = threadIdx.x & 31;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (row >= bd.n) return;
  const double* ar = a + row * np;
  double s = 0.0;
  for (long long j = lane; j < np; j += 32) s += ar[j] * v[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) {
    int nx_, ny_, nz_;
    bd.coords(row / 3, nx_, ny_, nz_);
    f[(row % 3) * g.comp_stride() + g.node(nx_, ny_, nz_)] = (T)s;
  }
}

// k right-hand sides at once (fields at column stride cstride, band vectors at stride np): one
// warp per row reads the row of ainv once for all k columns; each column's sum runs in the
// single-column kernel's order, so a column's result has the same bits as a lone solve
template <typename T, int K>
__global__ void k_band_gemm_to_field(T* __restrict__ f, long long cstride, const double* __restrict__ a,
                                     const double* __restrict__ v, LpGrid g, LpBand bd) {
  const long long np = 32LL * bd.nt;
  const int lane = threadIdx.x & 31;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (row >= bd.n) return;
  const double* ar = a + row * np;
  double s[K];
#pragma unroll
  for (int c = 0; c < K; ++c) s[c] = 0.0;
  for (long long j = lane; j < np; j += 32) {
    const double aj = ar[j];
#pragma unroll
    for (int c = 0; c < K; ++c) s[c] += aj * v[c * np + j];
  }
#pragma unroll
  for (int c = 0; c < K; ++c)
    for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_down_sync(0xffffffffu, s[c], o);
  if (lane == 0) {
    int nx_, ny_, nz_;
    bd.coords(row / 3, nx_, ny_, nz_);
    const long long at = (row % 3) * g.comp_stride() + g.node(nx_, ny_, nz_);
#pragma unroll
    for (int c = 0; c < K; ++c) f[c * cstride + at] = (T)s[c];
  }
}

template <typename T, int K>
void band_gemm_launch(T* f_out, long long cstride, const double* ainv, const double* v, LpGrid g, LpBand bd,
                      cudaStream_t st) {
  k_band_gemm_to_field<T, K><<<lp_blocks(bd.n * 32, 256), 256, 0, st>>>(f_out, cstride, ainv, v, g, bd);
}

template <typename T>
int band_solve_cols(T* f_out, const T* f_in, long long cstride, int ncol, const double* ainv, double* v, LpGrid g,
                    cudaStream_t st) {
  if (!lp_grid_ok(g) || !f_out || !f_in || !ainv || !v || ncol < 1 || cstride < g.comp_stride() * 3) return LP_ERR_ARG;
  const LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  const long long np = 32LL * bd.nt;
  for (int c = 0; c < ncol; ++c)
    k_field_to_band<T><<<lp_blocks(np, 256), 256, 0, st>>>(v + c * np, f_in + c * cstride, g, bd);
  for (int c0 = 0; c0 < ncol; c0 += 8) {
    const int k = ncol - c0 < 8 ? ncol - c0 : 8;
    T* fo = f_out + c0 * cstride;
    const double* vc = v + c0 * np;
    switch (k) {
      case 1: band_gemm_launch<T, 1>(fo, cstride, ainv, vc, g, bd, st); break;
      case 2: band_gemm_launch<T, 2>(fo, cstride, ainv, vc, g, bd, st); break;
      case 3: band_gemm_launch<T, 3>(fo, cstride, ainv, vc, g, bd, st); break;
      case 4: band_gemm_launch<T, 4>(fo, cstride, ainv, vc, g, bd, st); break;
      case 5: band_gemm_launch<T, 5>(fo, cstride, ainv, vc, g, bd, st); break;
      case 6: band_gemm_launch<T, 6>(fo, cstride, ainv, vc, g, bd, st); break;
      case 7: band_gemm_launch<T, 7>(fo, cstride, ainv, vc, g, bd, st); break;
      default: band_gemm_launch<T, 8>(fo, cstride, ainv, vc, g, bd, st); break;
    }
  }
  LP_LAUNCH_CHECK();
  return LP_OK;
}

template <typename T>
int band_solve(T* f_out, const T* f_in, const double* ainv, double* v, LpGrid g, cudaStream_t st) {
  if (!lp_grid_ok(g) || !f_out || !f_in || !ainv || !v) return LP_ERR_ARG;
  const LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  const long long np = 32LL * bd.nt;
  k_field_to_band<T><<<lp_blocks(np, 256), 256, 0, st>>>(v, f_in, g, bd);
  k_band_gemv_to_field<T><<<lp_blocks(bd.n * 32, 256), 256, 0, st>>>(f_out, ainv, v, g, bd);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)

extern "C" {

// the band layout of a level: out[0] = n (dofs), out[1] = nt (32-row tiles), out[2] = D
// (off-diagonal tiles per tile row), out[3] = half-bandwidth; returns the tile count nt (D + 1)
long long lpb_band_dims(int nx, int ny, int nz, long long* out) {
  if (nx < 1 || ny < 1 || nz < 1) return LP_ERR_ARG;
  const LpBand bd = lp_band(nx + 1, ny + 1, nz + 1);
  if (out) {
    out[0] = bd.n;
    out[1] = bd.nt;
    out[2] = bd.D;
    out[3] = 3LL * ((long long)bd.N1 * bd.N2 + bd.N2 + 1) + 2;
  }
  return (long long)bd.nt * (bd.D + 1);
}

// Signed Cholesky of the band in t (from lpb_coarse_band_*), in place; linv: nt x 1024 doubles
// (the inverses of the diagonal factor tiles); sgn: 32 nt doubles, the pivot signs; info: one
// device int, 0 or the first dof (1-based) whose pivot was exactly zero (or not finite); bar:
// max(64, nt) device words of scratch (the rows' progress counts); err: one device int, set when
// a wait gave up. One cooperative launch of up to 2 (D + 1) blocks, each owning tile rows.
int lpb_band_factor(double* t, double* linv, double* sgn, int* info, unsigned* bar, int* err, LP_GRID_ARGS,
                    void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !t || !linv || !sgn || !info || !bar || !err) return LP_ERR_ARG;
  LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  int dev = 0, nsm = 0, per_sm = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_band_factor, 256, 0);
  // D + 1 rows in flight hide each row's own products behind the chain from row to row; twice
  // that gives each block a row's worth of slack
  long long nblocks = 2LL * (bd.D + 1);
  if (nblocks > bd.nt) nblocks = bd.nt;
  const long long cap = (long long)per_sm * nsm;
  if (nblocks > cap) nblocks = cap;
  if (!coop || nblocks < 1) return LP_ERR_SIZE;
  const long long words = bd.nt > 64 ? bd.nt : 64;
  if (cudaMemsetAsync(bar, 0, words * sizeof(unsigned), LP_ST) != cudaSuccess) return LP_ERR_LAUNCH;
  if (cudaMemsetAsync(info, 0, sizeof(int), LP_ST) != cudaSuccess) return LP_ERR_LAUNCH;
  void* args[] = {&t, &linv, &sgn, &bd, &info, &bar, &err};
  if (cudaLaunchCooperativeKernel((const void*)k_band_factor, dim3((unsigned)nblocks), dim3(256), args, 0, LP_ST) !=
      cudaSuccess)
    return LP_ERR_LAUNCH;
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// ainv (32 nt x 32 nt doubles, row-major, band numbering) = A^-1 from the factor
int lpb_band_inverse(double* ainv, const double* t, const double* linv, const double* sgn, LP_GRID_ARGS,
                     void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !ainv || !t || !linv || !sgn) return LP_ERR_ARG;
  const LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  const long long np = 32LL * bd.nt;
  // as many (tile, block) pairs per chunk as fit in 227 KB next to the diagonal inverse and S
  int chunk = (int)((227 * 1024 / (INV_TILE * (long long)sizeof(double)) - 2) / 2);
  if (chunk > bd.D) chunk = bd.D;
  if (chunk < 1) return LP_ERR_SIZE;
  const long long smem = (2LL * chunk + 2) * INV_TILE * sizeof(double);
  if (cudaFuncSetAttribute(k_band_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return LP_ERR_SIZE;
  k_band_inverse<<<(unsigned)(np / INV_COLS), 512, (size_t)smem, LP_ST>>>(ainv, t, linv, sgn, bd, chunk);
  k_sym_lower<<<dim3(bd.nt, bd.nt), 256, 0, LP_ST>>>(ainv, np);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// f_out = A^-1 f_in on the coarsest level (fields of the level, any component masks already in
// the operator); v: 32 nt doubles of scratch
int lpb_band_solve_f32(float* f_out, const float* f_in, const double* ainv, double* v, LP_GRID_ARGS, void* stream) {
  return band_solve<float>(f_out, f_in, ainv, v, LP_GRID, LP_ST);
}

int lpb_band_solve_f64(double* f_out, const double* f_in, const double* ainv, double* v, LP_GRID_ARGS,
                       void* stream) {
  return band_solve<double>(f_out, f_in, ainv, v, LP_GRID, LP_ST);
}

// ncol right-hand sides at once: column c of f_in / f_out at element offset c * cstride (whole
// node fields, cstride >= 3 * the component stride); v: 32 nt * ncol doubles scratch
int lpb_band_solve_cols_f32(float* f_out, const float* f_in, long long cstride, int ncol, const double* ainv,
                            double* v, LP_GRID_ARGS, void* stream) {
  return band_solve_cols<float>(f_out, f_in, cstride, ncol, ainv, v, LP_GRID, LP_ST);
}

int lpb_band_solve_cols_f64(double* f_out, const double* f_in, long long cstride, int ncol, const double* ainv,
                            double* v, LP_GRID_ARGS, void* stream) {
  return band_solve_cols<double>(f_out, f_in, cstride, ncol, ainv, v, LP_GRID, LP_ST);
}

}  // extern "C"
