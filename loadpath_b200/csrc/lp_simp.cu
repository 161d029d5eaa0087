// SIMP-loop kernels: the cone density filter and its transpose (loadpath/simp.py:1143-1228,
// loadpath/benchmarks/reference.py:48-71), the SIMP law (loadpath/simp.py:1861), element
// strain energy u_e^T Ke v_e (loadpath/femops.py:51-78, loadpath/mg.py:975-988), sensitivities
// (loadpath/benchmarks/reference.py:89-99) and the OC volume pass (reference.py:100-110).
// All in float64.
#include <algorithm>

#include "lp_common.cuh"
#include "lp_modal.cuh"

#define LP_MAX_TAPS 1024
#define LP_MAX_LAMBDA 64

namespace {

// out[c] = sum_t w_t v[c + d_t] (zeros outside the grid); optional pre-division of v by hs
// and post-division of out by hs2; optional SIMP law on the result.
//   mode 0: out = H v
//   mode 1: out = H (v / hs_in)
//   mode 2: out = (H v) / hs_out ; e_out = emin + out^p (1 - emin) if e_out != null
// A block takes a tile of 32 x 8 cell columns times one z chunk (4 cells): it stages the tile with
// its halo of reach R (the largest |offset| of the taps, up to LP_FT_R) in shared memory, v / hs_in
// formed once per staged cell and zeros outside the grid, and each thread sums the taps for the 4
// cells of its column in the taps' order, so the sums are those of a gather cell by cell. The
// staging reads whole rows of chunks (32-byte sectors, contiguous along x). Taps reaching further
// than LP_FT_R are gathered from global memory instead, cell by cell.
#define LP_FT_X 32
#define LP_FT_Y 8
#define LP_FT_R 2
__global__ void __launch_bounds__(256) k_filter(double* __restrict__ out, const double* __restrict__ v,
                                                const int* __restrict__ toff, const double* __restrict__ tw,
                                                int ntaps, const double* __restrict__ hs_in,
                                                const double* __restrict__ hs_out, double* __restrict__ e_out,
                                                double penal, double emin, LpGrid g) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double tile[(4 + 2 * LP_FT_R) * (LP_FT_Y + 2 * LP_FT_R) * (LP_FT_X + 2 * LP_FT_R)];
  __shared__ int s_reach;
  int* so = reinterpret_cast<int*>(smem_raw);
  double* sw = reinterpret_cast<double*>(smem_raw + ((3 * ntaps * sizeof(int) + 15) & ~15));
  if (threadIdx.x == 0) s_reach = 0;
  __syncthreads();
  int reach = 0;
  for (int i = threadIdx.x; i < ntaps; i += blockDim.x) {
    const int dx = toff[3 * i], dy = toff[3 * i + 1], dz = toff[3 * i + 2];
    so[3 * i] = dx;
    so[3 * i + 1] = dy;
    so[3 * i + 2] = dz;
    sw[i] = tw[i];
    reach = max(reach, max(abs(dx), max(abs(dy), abs(dz))));
  }
  if (reach) atomicMax(&s_reach, reach);
  __syncthreads();
  const int R = s_reach;
  const int nbx = (g.nx + LP_FT_X - 1) / LP_FT_X, nby = (g.ny + LP_FT_Y - 1) / LP_FT_Y;
  const int bx = (int)(blockIdx.x % nbx), rest = (int)(blockIdx.x / nbx);
  const int by = rest % nby, cz = rest / nby;
  const int x0 = bx * LP_FT_X, y0 = by * LP_FT_Y;
  const int x = x0 + (int)(threadIdx.x & 31), y = y0 + (int)(threadIdx.x >> 5);
  const bool own = x < g.nx && y < g.ny;
  if (R > LP_FT_R) {
    if (!own) return;
    for (int zq = 0; zq < 4; ++zq) {
      const int z = 4 * cz + zq;
      if (z >= g.nz) break;
      double acc = 0.0;
      for (int i = 0; i < ntaps; ++i) {
        const int xx = x + so[3 * i], yy = y + so[3 * i + 1], zz = z + so[3 * i + 2];
        if (xx < 0 || yy < 0 || zz < 0 || xx >= g.nx || yy >= g.ny || zz >= g.nz) continue;
        const long long c = g.cell(xx, yy, zz);
        double vi = v[c];
        if (hs_in) vi = vi / hs_in[c];
        acc += sw[i] * vi;
      }
      const long long c = g.cell(x, y, z);
      if (hs_out) acc = acc / hs_out[c];
      out[c] = acc;
      if (e_out) e_out[c] = emin + pow(acc, penal) * (1.0 - emin);
    }
    return;
  }
  const int XH = LP_FT_X + 2 * R, YH = LP_FT_Y + 2 * R, ZH = 4 + 2 * R, P = XH * YH;
  const int CR = (R + 3) / 4;  // halo chunks on each side
  // the taps' offsets in the staged tile, written over their first coordinate
  for (int i = threadIdx.x; i < ntaps; i += blockDim.x) so[3 * i] += (so[3 * i + 2] * YH + so[3 * i + 1]) * XH;
  // a warp stages a (chunk, y) row at a time: 4 XH doubles contiguous in memory, lanes along it
  const int rowlen = 4 * XH, nrows = (2 * CR + 1) * YH;
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5), nwarps = (int)(blockDim.x >> 5);
  for (int row = warp; row < nrows; row += nwarps) {
    const int cr = row / YH, yl = row - cr * YH;
    const int gy = y0 - R + yl, zbase = 4 * (cz - CR + cr);
    const bool yok = gy >= 0 && gy < g.ny;
    for (int j = lane; j < rowlen; j += 32) {
      const int xl = j >> 2, gz = zbase + (j & 3);
      const int zl = gz - (4 * cz - R);
      if (zl < 0 || zl >= ZH) continue;
      const int gx = x0 - R + xl;
      double val = 0.0;
      if (yok && gx >= 0 && gx < g.nx && gz >= 0 && gz < g.nz) {
        const long long c = g.cell(gx, gy, gz);
        val = v[c];
        if (hs_in) val = val / hs_in[c];
      }
      tile[(zl * YH + yl) * XH + xl] = val;
    }
  }
  __syncthreads();
  if (!own) return;
  const int ctr = (R * YH + R + (int)(threadIdx.x >> 5)) * XH + R + (int)(threadIdx.x & 31);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = 0; i < ntaps; ++i) {
    const int o = ctr + so[3 * i];
    const double w = sw[i];
#pragma unroll
    for (int zq = 0; zq < 4; ++zq) acc[zq] += w * tile[o + zq * P];
  }
#pragma unroll
  for (int zq = 0; zq < 4; ++zq) {
    const int z = 4 * cz + zq;
    if (z >= g.nz) break;
    const long long c = g.cell(x, y, z);
    double r = acc[zq];
    if (hs_out) r = r / hs_out[c];
    out[c] = r;
    if (e_out) e_out[c] = emin + pow(r, penal) * (1.0 - emin);
  }
}

// e = emin + x^p (1 - emin) on the grid's cells (padding untouched)
__global__ void k_simp_law(double* __restrict__ e, const double* __restrict__ x, double penal, double emin, LpGrid g) {
  const long long total = g.cells_padded();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    const long long c = t;
    e[c] = emin + pow(x[c], penal) * (1.0 - emin);
  }
}

// per-cell u_e^T ke v_e on the node grid (v = u when v is null), float64. The product is taken in
// the corner-parity basis: u^ = T u_e, v^ = T v_e (eight-point Walsh transforms per component),
// u_e^T ke v_e = u^T K^ v^ with K^ = T ke T^T / 64 formed by each block from ke. When K^ has
// weight outside the 45-entry pattern (not an isotropic brick) the block takes the dense
// 21 x 21 modal product instead.
template <typename T>
__global__ void __launch_bounds__(128) k_element_energy(double* __restrict__ ce, const T* __restrict__ u,
                                                        const T* __restrict__ v, const double* __restrict__ ke,
                                                        LpGrid g) {
  __shared__ double kh[576];
  __shared__ double wmax[4];
  constexpr int rows[LP_MODAL_NNZ] = LP_MODAL_ROWS;
  constexpr int cols[LP_MODAL_NNZ] = LP_MODAL_COLS;
  double amax = 0.0;
  for (int i = threadIdx.x; i < 576; i += blockDim.x) {
    kh[i] = lp_modal_entry(ke, i / 24, i % 24);
    amax = fmax(amax, fabs(kh[i]));
  }
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = amax;
  __syncthreads();
  amax = fmax(fmax(wmax[0], wmax[1]), fmax(wmax[2], wmax[3]));
  int off = 0;
  for (int i = threadIdx.x; i < 576; i += blockDim.x) {
    bool in = false;
    for (int j = 0; j < LP_MODAL_NNZ; ++j) in |= (rows[j] * 24 + cols[j] == i);
    off |= (!in && fabs(kh[i]) > 1e-12 * amax);
  }
  const bool dense = __syncthreads_or(off) != 0;

  const long long total = g.cells_padded();
  const long long cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    long long nk[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) nk[k] = g.node(x + cx_(k), y + cy_(k), z + cz_(k));
    double uh[24], vh[24];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double a[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = (double)u[c * cs + nk[k]];
      lp_walsh8(a);
#pragma unroll
      for (int m = 0; m < 8; ++m) uh[3 * m + c] = vh[3 * m + c] = a[m];
    }
    if (v) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double a[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = (double)v[c * cs + nk[k]];
        lp_walsh8(a);
#pragma unroll
        for (int m = 0; m < 8; ++m) vh[3 * m + c] = a[m];
      }
    }
    double s = 0.0;
    if (!dense) {
#pragma unroll
      for (int j = 0; j < LP_MODAL_NNZ; ++j) s = fma(uh[rows[j]] * kh[rows[j] * 24 + cols[j]], vh[cols[j]], s);
    } else {
#pragma unroll
      for (int r = 3; r < 24; ++r) {
        double f = 0.0;
#pragma unroll
        for (int c = 3; c < 24; ++c) f = fma(kh[r * 24 + c], vh[c], f);
        s = fma(uh[r], f, s);
      }
    }
    ce[g.cell(x, y, z)] = s;
  }
}

// dc = -p (1 - emin) x^(p-1) ce * scale (accumulated into dc when accumulate != 0);
// partial compliance sum_c e_c ce_c into part[block]
__global__ void k_sensitivity(double* __restrict__ dc, const double* __restrict__ xphys, const double* __restrict__ ce,
                              const double* __restrict__ e, double penal, double emin, double scale, int accumulate,
                              LpGrid g, double* __restrict__ part) {
  __shared__ double sh[32];
  const long long total = g.cells_padded();
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    const long long c = t;
    double xv = xphys[c];
    double d = -penal * (1.0 - emin) * pow(xv, penal - 1.0) * ce[c] * scale;
    dc[c] = accumulate ? dc[c] + d : d;
    if (e) acc += e[c] * ce[c] * scale;
  }
  acc = lp_block_sum(acc, sh);
  if (part && threadIdx.x == 0) part[blockIdx.x] = acc;
}

// OC trial step for NL multipliers at once (the next levels of the bisection tree): for each
// lambda_j the step x sqrt(-dc / dv / lambda_j) clipped to [max(0, x - move), min(1, x + move)]
// (loadpath/benchmarks/reference.py:103), and partial sums of xnew * gv where gv = H (1 / hs)
// weighs a cell's share of the filtered volume. The step is formed as
// (x sqrt(-dc / dv)) / sqrt(lambda_j): one square root per cell; only the volume comparisons use
// it, the accepted step is recomputed with the reference's expression by k_oc_apply.
//
// The kernel is bound by latency and instruction issue, not by DRAM (32 bytes per cell): each
// thread loads its next cell's four values before working on the current one, the clip is two
// compare-and-selects (fmin / fmax on doubles take several instructions more; the selects give
// the same values, a NaN step clipping to the upper bound as fmin does), and the 1 / sqrt(lambda_j)
// are read from shared memory at each use (volatile loads, so that they take no registers: 114
// registers, two blocks per SM). The padding of the cell z pitch lies in the z chunks from nz / 4
// up, so comparisons of t with those chunks' starts stand for the division of LpGrid::cell_at.
__device__ __forceinline__ double lds_volatile_f64(const double* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}

template <int NL>
__global__ void __launch_bounds__(256, 2) k_oc_volumes(const double* __restrict__ x, const double* __restrict__ dc,
                                                       const double* __restrict__ dv, const double* __restrict__ gv,
                                                       const double* __restrict__ lam, double move, LpGrid g,
                                                       double* __restrict__ part) {
  __shared__ double s_isl[NL];
  __shared__ double sacc[NL][8];
  if (threadIdx.x < NL) s_isl[threadIdx.x] = 1.0 / sqrt(lam[threadIdx.x]);
  __syncthreads();
  double acc[NL];
#pragma unroll
  for (int j = 0; j < NL; ++j) acc[j] = 0.0;
  const long long total = g.cells_padded();
  // chunks below nz / 4 hold cells only; chunk nz / 4 holds nz % 4 cells at its start, the chunks
  // above it padding only
  const long long pad_from = (long long)(g.nz >> 2) * g.cell_zc_stride();
  const long long pad_all = pad_from + g.cell_zc_stride();
  const int zr = g.nz & 3;
  const long long step = (long long)gridDim.x * blockDim.x;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double nx_ = 0.0, ngw = 0.0, ndc = -1.0, ndv = 1.0;
  if (t < total) { nx_ = x[t]; ngw = gv[t]; ndc = dc[t]; ndv = dv[t]; }
  for (; t < total; t += step) {
    const double xv = nx_, gw = ngw, dcv = ndc, dvv = ndv;
    const long long tn = t + step;
    if (tn < total) { nx_ = x[tn]; ngw = gv[tn]; ndc = dc[tn]; ndv = dv[tn]; }
    if (t >= pad_from && (t >= pad_all || (int)(t & 3) >= zr)) continue;
    const double ts = xv * sqrt(-dcv / dvv);
    const double lo = fmax(0.0, xv - move), hi = fmin(1.0, xv + move);
#pragma unroll
    for (int j = 0; j < NL; ++j) {
      const double p = ts * lds_volatile_f64(&s_isl[j]);
      double v = p < hi ? p : hi;
      v = v > lo ? v : lo;
      acc[j] += v * gw;
    }
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NL; ++j) {
    double s = acc[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sacc[j][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < NL) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += sacc[threadIdx.x][w];
    part[(long long)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

// the nl volumes from the blocks' partial sums: one warp per multiplier, its lanes striding over
// the blocks, then a shuffle tree (a fixed order, so the sums are the same every run)
__global__ void k_oc_final(const double* __restrict__ part, int nblocks, int nl, double* __restrict__ out) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = threadIdx.x >> 5; j < nl; j += nw) {
    double s = 0.0;
    for (int i = lane; i < nblocks; i += 32) s += part[(long long)j * nblocks + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = s;
  }
}

// The top3d bisection on the volume multiplier walked on the device (the walk of
// loadpath_b200.simp.oc_bisection, loadpath/benchmarks/reference.py:100-110): state = {l1, l2,
// below (smallest multiplier seen with volume <= target), above (largest seen with volume >
// target), lmid, passes, done}. With absorb the 31 volumes of the last candidates are folded into
// below / above first; the walk then decides every midpoint the evaluations decide and stops at
// the first one they leave open, writing the next 31 candidates (the ladder l2 / 2^(2i+1) while l1 =
// 0, else the next five levels of the bisection tree below the open interval, breadth first), or
// finishes (done = 1, lmid the last midpoint). With a conditional handle (a graph WHILE node) the
// loop goes on while candidates are open.
__global__ void k_oc_walk(cudaGraphConditionalHandle handle, int use_handle, double* __restrict__ state,
                          const double* __restrict__ vols, double* __restrict__ cands, double target, double tol,
                          int absorb) {
  double l1 = state[0], l2 = state[1], below = state[2], above = state[3], lmid = state[4], passes = state[5];
  if (absorb) {
    for (int j = 0; j < 31; ++j) {
      if (vols[j] > target) above = fmax(above, cands[j]);
      else below = fmin(below, cands[j]);
    }
    passes += 1.0;
  }
  unsigned need = 0;
  while ((l2 - l1) / (l1 + l2) > tol) {
    const double m = 0.5 * (l2 + l1);
    if (m >= below) {
      lmid = l2 = m;
      continue;
    }
    if (m <= above) {
      lmid = l1 = m;
      continue;
    }
    if (l1 == 0.0) {
      for (int i = 0; i < 31; ++i) cands[i] = ldexp(l2, -(2 * i + 1));
    } else {
      double qa[63], qb[63];
      int head = 0, tail = 1;
      qa[0] = l1;
      qb[0] = l2;
      for (int n = 0; n < 31; ++n) {
        const double a = qa[head], b = qb[head];
        ++head;
        const double mm = 0.5 * (b + a);
        cands[n] = mm;
        qa[tail] = a;
        qb[tail] = mm;
        ++tail;
        qa[tail] = mm;
        qb[tail] = b;
        ++tail;
      }
    }
    need = 1;
    break;
  }
  state[0] = l1;
  state[1] = l2;
  state[2] = below;
  state[3] = above;
  state[4] = lmid;
  state[5] = passes;
  state[6] = need ? 0.0 : 1.0;
  if (use_handle) cudaGraphSetConditional(handle, need);
}

__global__ void k_oc_walk_init(double* __restrict__ state, double l2) {
  state[0] = 0.0;
  state[1] = l2;
  state[2] = __longlong_as_double(0x7ff0000000000000LL);    // +inf
  state[3] = -__longlong_as_double(0x7ff0000000000000LL);   // -inf
  state[4] = __longlong_as_double(0x7ff8000000000000LL);    // no midpoint yet
  state[5] = 0.0;
  state[6] = 0.0;
}

// the OC step at one multiplier (lam, or *lam_dev when given): xnew and the change max|xnew - x|
// partials
__global__ void k_oc_apply(double* __restrict__ xnew, const double* __restrict__ x, const double* __restrict__ dc,
                           const double* __restrict__ dv, double lam_h, const double* __restrict__ lam_dev,
                           double move, LpGrid g, double* __restrict__ part) {
  __shared__ double sh[32];
  const double lam = lam_dev ? *lam_dev : lam_h;
  const long long total = g.cells_padded();
  double mx = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    const long long c = t;
    double xv = x[c];
    double xn = xv * sqrt(-dc[c] / dv[c] / lam);
    xn = fmax(0.0, fmax(xv - move, fmin(1.0, fmin(xv + move, xn))));
    xnew[c] = xn;
    mx = fmax(mx, fabs(xn - xv));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
    part[blockIdx.x] = m;
  }
}

__global__ void k_max_final2(const double* __restrict__ part, int n, double* __restrict__ out) {
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, part[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    *out = r;
  }
}

__global__ void k_sum_final_s(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}


// ---- loadpath's own design update (loadpath/simp.py:1443-1450, :1775-1814, :2249-2376) --------
// Cell flags: bit 0 passive solid (pres: design and projection held at 1, derivative 0), bit 1
// passive void (held at 0).

// xp = (tanh(b eta) + tanh(b (xt - eta))) / den, den = tanh(b eta) + tanh(b (1 - eta)); dxp its
// derivative b (1 - tanh(b (xt - eta))^2) / den; held cells as the flags say; partial sums of
// xp * w into part[block] (w given)
__global__ void k_project(double* __restrict__ xp, double* __restrict__ dxp, const double* __restrict__ xt,
                          double beta, double eta, double tbe, double den, const uint8_t* __restrict__ flags,
                          const double* __restrict__ w, LpGrid g, double* __restrict__ part) {
  __shared__ double sh[32];
  const long long total = g.cells_padded();
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    const uint8_t fl = flags ? flags[t] : 0;
    const double th = tanh(beta * (xt[t] - eta));
    double p = (tbe + th) / den, dp = beta * (1.0 - th * th) / den;
    if (fl & 1) {
      p = 1.0;
      dp = 0.0;
    } else if (fl & 2) {
      p = 0.0;
      dp = 0.0;
    }
    if (xp) xp[t] = p;
    if (dxp) dxp[t] = dp;
    if (w) acc += p * w[t];
  }
  if (part) {
    acc = lp_block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
  }
}

// the OC step at multiplier lm: xn = clip(x sqrt(-dc / dv) / sqrt(lm), max(0, x - move),
// min(1, x + move)), held cells as the flags say
__global__ void k_oc_stepped(double* __restrict__ xn, const double* __restrict__ x, const double* __restrict__ dc,
                             const double* __restrict__ dv, double lm, double move, const uint8_t* __restrict__ flags,
                             LpGrid g) {
  const double sl = sqrt(lm);
  const long long total = g.cells_padded();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    const double xv = x[t];
    double v = fmin(fmax(xv * sqrt(-dc[t] / dv[t]) / sl, fmax(0.0, xv - move)), fmin(1.0, xv + move));
    const uint8_t fl = flags ? flags[t] : 0;
    if (fl & 1) v = 1.0;
    else if (fl & 2) v = 0.0;
    xn[t] = v;
  }
}

// out = a * b (zero where the flags hold a cell); with clip0, out = min(out, 0)
__global__ void k_cell_product(double* __restrict__ out, const double* __restrict__ a, const double* __restrict__ b,
                               const uint8_t* __restrict__ flags, int clip0, LpGrid g) {
  const long long total = g.cells_padded();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x_, y_, z;
    if (!g.cell_at(t, x_, y_, z)) continue;
    double v = b ? a[t] * b[t] : a[t];
    if (flags && (flags[t] & 3)) v = 0.0;
    if (clip0 == 1) v = fmin(v, 0.0);
    else if (clip0 == 2) v = fmax(v, 1e-12);
    out[t] = v;
  }
}

// v[c] = v[m(c)] = (v[c] + v[m(c)]) / 2 for every cell c and its mirror image m(c) across the
// grid's mid-plane normal to axis (loadpath/simp.py:1476-1482 `_symmetrize` on a box whose every cell
// has a mirror): one thread per pair, the cell below the mid-plane; the middle cell of an odd
// extent is its own image and keeps its value.
__global__ void k_mirror_average(double* __restrict__ v, int axis, LpGrid g) {
  const long long total = g.cells_padded();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.cell_at(t, x, y, z)) continue;
    int mx = x, my = y, mz = z;
    if (axis == 0) mx = g.nx - 1 - x;
    else if (axis == 1) my = g.ny - 1 - y;
    else mz = g.nz - 1 - z;
    const long long m = g.cell(mx, my, mz);
    if (m <= t) continue;
    const double a = v[t], b = v[m];
    const double h = 0.5 * (a + b);
    v[t] = h;
    v[m] = h;
  }
}

// ce[e] = u_e^T ke v_e over a general mesh, u_e the 24 values at edof[e, :] (femops.element_energy,
// loadpath/femops.py:236-242); v NULL: v = u. One thread per element, ke in shared memory; the
// caller has checked every index against the vectors' length.
__global__ void k_energy_edof(double* __restrict__ ce, const double* __restrict__ u, const double* __restrict__ v,
                              const long long* __restrict__ edof, const double* __restrict__ ke, long long ne) {
  __shared__ double sk[576];
  for (int i = threadIdx.x; i < 576; i += blockDim.x) sk[i] = ke[i];
  __syncthreads();
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    double ue[24], ve[24];
#pragma unroll
    for (int a = 0; a < 24; ++a) {
      const long long d = edof[e * 24 + a];
      ue[a] = u[d];
      ve[a] = v ? v[d] : ue[a];
    }
    double acc = 0.0;
#pragma unroll 4
    for (int j = 0; j < 24; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 24; ++k) s += sk[j * 24 + k] * ve[k];
      acc += ue[j] * s;
    }
    ce[e] = acc;
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)
#define LP_SIMP_BLOCKS 592
#define LP_ENERGY_BLOCKS 592  // 148 SMs x 4 resident blocks of 128 (128 registers)

extern "C" {

int lpb_filter(double* out, const double* v, const int* toff, const double* tw, int ntaps, const double* hs_in,
               const double* hs_out, double* e_out, double penal, double emin, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !v || !toff || !tw || ntaps < 1 || ntaps > LP_MAX_TAPS) return LP_ERR_ARG;
  if (out == v) return LP_ERR_ARG;
  size_t smem = ((3 * ntaps * sizeof(int) + 15) & ~(size_t)15) + ntaps * sizeof(double);
  const long long tiles = (long long)((g.nx + LP_FT_X - 1) / LP_FT_X) * ((g.ny + LP_FT_Y - 1) / LP_FT_Y) *
                          ((g.nz + 3) / 4);
  if (tiles > 2147483647LL) return LP_ERR_ARG;
  k_filter<<<(unsigned)tiles, 256, smem, LP_ST>>>(out, v, toff, tw, ntaps, hs_in, hs_out, e_out, penal, emin, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_simp_law(double* e, const double* x, double penal, double emin, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !e || !x) return LP_ERR_ARG;
  long long total = g.cells_padded();
  k_simp_law<<<lp_blocks(total, 256), 256, 0, LP_ST>>>(e, x, penal, emin, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_element_energy_edof(double* ce, const double* u, const double* v, const long long* edof, const double* ke,
                            long long ne, void* stream) {
  if (!ce || !u || !edof || !ke || ne < 0) return LP_ERR_ARG;
  if (ne == 0) return LP_OK;
  k_energy_edof<<<lp_blocks(ne, 128), 128, 0, LP_ST>>>(ce, u, v, edof, ke, ne);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_element_energy_f64(double* ce, const double* u, const double* v, const double* ke, LP_GRID_ARGS,
                           void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !ce || !u || !ke) return LP_ERR_ARG;
  long long total = g.cells_padded();
  k_element_energy<double><<<(int)std::min<long long>(lp_blocks(total, 128), LP_ENERGY_BLOCKS), 128, 0, LP_ST>>>(
      ce, u, v, ke, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_element_energy_f32(double* ce, const float* u, const float* v, const double* ke, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !ce || !u || !ke) return LP_ERR_ARG;
  long long total = g.cells_padded();
  k_element_energy<float><<<(int)std::min<long long>(lp_blocks(total, 128), LP_ENERGY_BLOCKS), 128, 0, LP_ST>>>(
      ce, u, v, ke, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// dc (+)= -p (1 - emin) x^(p-1) ce * scale; *comp = sum e * ce * scale (if e and comp given)
int lpb_sensitivity(double* dc, const double* xphys, const double* ce, const double* e, double penal, double emin,
                    double scale, int accumulate, double* part, double* comp, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !dc || !xphys || !ce || !part) return LP_ERR_ARG;
  k_sensitivity<<<LP_SIMP_BLOCKS, 256, 0, LP_ST>>>(dc, xphys, ce, e, penal, emin, scale, accumulate, g, part);
  if (comp) k_sum_final_s<<<1, 1024, 0, LP_ST>>>(part, LP_SIMP_BLOCKS, comp);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// the device walk of the bisection (k_oc_walk): init (state: 7 doubles, the first candidates in
// cands) and one step after a volumes pass; handle: the conditional of a graph WHILE node or 0
int lpb_oc_walk_init(double* state, double* cands, double l2, double target, double tol, void* stream) {
  if (!state || !cands || !(l2 > 0.0)) return LP_ERR_ARG;
  k_oc_walk_init<<<1, 1, 0, LP_ST>>>(state, l2);
  k_oc_walk<<<1, 1, 0, LP_ST>>>(cudaGraphConditionalHandle{}, 0, state, nullptr, cands, target, tol, 0);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_oc_walk(long long handle, double* state, const double* vols, double* cands, double target, double tol,
                void* stream) {
  if (!state || !vols || !cands) return LP_ERR_ARG;
  k_oc_walk<<<1, 1, 0, LP_ST>>>((cudaGraphConditionalHandle)handle, handle != 0, state, vols, cands, target, tol, 1);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// volumes[j] = sum_c xnew(lam[j])_c gv_c for nl = 31 multipliers; part: nl * 592 doubles
int lpb_oc_volumes(double* volumes, const double* x, const double* dc, const double* dv, const double* gv,
                   const double* lam, int nl, double move, double* part, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || nl < 1 || nl > LP_MAX_LAMBDA || !volumes || !x || !dc || !dv || !gv || !lam || !part)
    return LP_ERR_ARG;
  if (nl != 31) return LP_ERR_ARG;
  k_oc_volumes<31><<<LP_SIMP_BLOCKS, 256, 0, LP_ST>>>(x, dc, dv, gv, lam, move, g, part);
  k_oc_final<<<1, 1024, 0, LP_ST>>>(part, LP_SIMP_BLOCKS, nl, volumes);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_oc_apply(double* xnew, const double* x, const double* dc, const double* dv, double lam, double move,
                 double* part, double* change, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !xnew || !x || !dc || !dv || !part || !change) return LP_ERR_ARG;
  k_oc_apply<<<LP_SIMP_BLOCKS, 256, 0, LP_ST>>>(xnew, x, dc, dv, lam, nullptr, move, g, part);
  k_max_final2<<<1, 1024, 0, LP_ST>>>(part, LP_SIMP_BLOCKS, change);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// lpb_oc_apply at the multiplier *lam (device), e.g. the walk's lmid (state + 4)
int lpb_oc_apply_at(double* xnew, const double* x, const double* dc, const double* dv, const double* lam,
                    double move, double* part, double* change, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !xnew || !x || !dc || !dv || !lam || !part || !change) return LP_ERR_ARG;
  k_oc_apply<<<LP_SIMP_BLOCKS, 256, 0, LP_ST>>>(xnew, x, dc, dv, 0.0, lam, move, g, part);
  k_max_final2<<<1, 1024, 0, LP_ST>>>(part, LP_SIMP_BLOCKS, change);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// xp, dxp (either may be NULL) of the projection at (beta, eta); *vol = sum xp * w when w and vol
// are given (part: LP_SIMP_BLOCKS doubles)
int lpb_project(double* xp, double* dxp, const double* xt, double beta, double eta, const uint8_t* flags,
                const double* w, double* part, double* vol, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !xt || (w && (!part || !vol))) return LP_ERR_ARG;
  const double tbe = tanh(beta * eta), den = tbe + tanh(beta * (1.0 - eta));
  k_project<<<LP_SIMP_BLOCKS, 256, 0, LP_ST>>>(xp, dxp, xt, beta, eta, tbe, den, flags, w, g, w ? part : nullptr);
  if (w) k_sum_final_s<<<1, 1024, 0, LP_ST>>>(part, LP_SIMP_BLOCKS, vol);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_oc_stepped(double* xn, const double* x, const double* dc, const double* dv, double lm, double move,
                   const uint8_t* flags, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !xn || !x || !dc || !dv || !(lm > 0.0)) return LP_ERR_ARG;
  k_oc_stepped<<<lp_blocks(g.cells_padded(), 256), 256, 0, LP_ST>>>(xn, x, dc, dv, lm, move, flags, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// the mirror average across axis (0 x, 1 y, 2 z), in place
int lpb_mirror_average(double* v, int axis, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !v || axis < 0 || axis > 2) return LP_ERR_ARG;
  k_mirror_average<<<lp_blocks(g.cells_padded(), 256), 256, 0, LP_ST>>>(v, axis, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out = a * b (b NULL: a), zero on flagged cells, then min(., 0) (clip0 1) or max(., 1e-12) (clip0 2)
int lpb_cell_product(double* out, const double* a, const double* b, const uint8_t* flags, int clip0, LP_GRID_ARGS,
                     void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !a || clip0 < 0 || clip0 > 2) return LP_ERR_ARG;
  k_cell_product<<<lp_blocks(g.cells_padded(), 256), 256, 0, LP_ST>>>(out, a, b, flags, clip0, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
