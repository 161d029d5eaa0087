// The Method of Moving Asymptotes on the device (loadpath/mma.py:31-214, Svanberg's 2007
// formulation): the per-variable work of MMA.update and of its primal-dual interior-point
// subproblem solver, over n design variables and m <= 8 constraints, in float64.
//
//   lpb_mma_prepare   sanitised design and gradients, the moving asymptotes, move limits alfa /
//                     beta, p0 q0 P Q of the convex approximation and sum_j P_ij/ux_j + Q_ij/xl_j
//                     (loadpath/mma.py:57-103)
//   lpb_mma_sub_init  the subsolver's starting point x, xsi, eta (loadpath/mma.py:114-125)
//   lpb_mma_newton_a  one Newton step's n-sized terms: delx, diagx (kept) and the reductions
//                     gvec, GG (delx / diagx) and (GG / diagx) GG^T for the (m + 1) system
//   lpb_mma_newton_b  dx, dxsi, deta from dlam and the step-length maxima
//   lpb_mma_trial     x, xsi, eta = old + steg * d and the residual's n-sized parts at the new
//                     point (sum of squares, largest magnitude, gvec)
//   lpb_mma_finish    non-finite results back to the old design, clip to [alfa, beta]
// The host runs the loops, the m-sized parts of the residual and the (m + 1) x (m + 1) solve.
// Reductions go through fixed per-block partials summed in order (the same bits every run).
#include <math.h>

#include "lp_common.cuh"

#define LP_MMA_MAXM 8
#define LP_MMA_BLOCKS 592
#define LP_MMA_THREADS 256

namespace {

struct MVec {
  double v[LP_MMA_MAXM];
};

__device__ __forceinline__ double nan_to_num(double v, double nan, double big) {
  if (isnan(v)) return nan;
  if (isinf(v)) return v > 0 ? big : -big;
  return v;
}

// block reduction of K values per thread (sum or max per value) into part[k * nblocks + block]
template <int K>
__device__ __forceinline__ void block_reduce(double (&v)[K], const bool (&is_max)[K], double* __restrict__ part) {
  __shared__ double sh[LP_MMA_THREADS / 32][K > 0 ? K : 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = is_max[k] ? fmax(x, y) : x + y;
    }
    if (lane == 0) sh[w][k] = x;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double x = sh[0][k];
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) x = is_max[k] ? fmax(x, sh[ww][k]) : x + sh[ww][k];
    part[(long long)k * gridDim.x + blockIdx.x] = x;
  }
}

__global__ void k_mma_final(const double* __restrict__ part, int nblocks, int K, const int* __restrict__ maxmask,
                            double* __restrict__ out) {
  // one warp per value, blocks summed in a fixed order
  const int k = blockIdx.x;
  if (k >= K) return;
  const bool mx = maxmask[k] != 0;
  double x = mx ? -INFINITY : 0.0;
  for (int b = threadIdx.x; b < nblocks; b += 32) x = mx ? fmax(x, part[(long long)k * nblocks + b]) : x + part[(long long)k * nblocks + b];
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_down_sync(0xffffffffu, x, o);
    x = mx ? fmax(x, y) : x + y;
  }
  if (threadIdx.x == 0) out[k] = x;
}

// ---- update: asymptotes and the convex approximation (loadpath/mma.py:57-103) ---------------
template <int M>
__global__ void __launch_bounds__(LP_MMA_THREADS) k_mma_prepare(
    long long n, int m, double* __restrict__ x, const double* __restrict__ xmin, const double* __restrict__ xmax,
    double* __restrict__ low, double* __restrict__ upp, const double* __restrict__ xold1,
    const double* __restrict__ xold2, int init, double asyinit, double asyincr, double asydecr, double move,
    double* __restrict__ df0, double* __restrict__ df, double* __restrict__ alfa, double* __restrict__ beta,
    double* __restrict__ p0, double* __restrict__ q0, double* __restrict__ P, double* __restrict__ Q,
    double* __restrict__ part) {
  double acc[M];
  bool is_max[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    acc[i] = 0.0;
    is_max[i] = false;
  }
  const double raa0 = 1e-5, albefa = 0.1;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double lo_b = xmin[j], hi_b = xmax[j];
    const double xj = fmin(fmax(isnan(x[j]) ? 0.5 : x[j], lo_b), hi_b);
    x[j] = xj;
    const double span = hi_b - lo_b;
    double l, u;
    if (init) {
      l = xj - asyinit * span;
      u = xj + asyinit * span;
    } else {
      const double x1 = xold1[j], x2 = xold2[j];
      const double zzz = (xj - x1) * (x1 - x2);
      const double factor = zzz > 0 ? asyincr : (zzz < 0 ? asydecr : 1.0);
      l = xj - factor * (x1 - low[j]);
      u = xj + factor * (upp[j] - x1);
      l = fmin(fmax(l, xj - 10 * span), xj - 0.01 * span);
      u = fmin(fmax(u, xj + 0.01 * span), xj + 10 * span);
    }
    low[j] = l;
    upp[j] = u;
    alfa[j] = fmax(fmax(l + albefa * (xj - l), xj - move * span), lo_b);
    beta[j] = fmin(fmin(u - albefa * (u - xj), xj + move * span), hi_b);
    const double xmami = fmax(span, 1e-5);
    const double ux1 = u - xj, xl1 = xj - l, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    const double g0 = nan_to_num(df0[j], 0.0, 1e6);
    df0[j] = g0;
    const double pp = fmax(g0, 0.0), qq = fmax(-g0, 0.0), pq0 = 0.001 * (pp + qq) + raa0 / xmami;
    p0[j] = (pp + pq0) * ux2;
    q0[j] = (qq + pq0) * xl2;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (i >= m) break;
      const long long ij = (long long)i * n + j;
      const double gi = nan_to_num(df[ij], 0.0, 1e6);
      df[ij] = gi;
      const double Pp = fmax(gi, 0.0), Qq = fmax(-gi, 0.0), PQ = 0.001 * (Pp + Qq) + raa0 / xmami;
      const double Pij = (Pp + PQ) * ux2, Qij = (Qq + PQ) * xl2;
      P[ij] = Pij;
      Q[ij] = Qij;
      acc[i] += Pij / ux1 + Qij / xl1;
    }
  }
  block_reduce<M>(acc, is_max, part);
}

// ---- subsolver -------------------------------------------------------------------------------
__global__ void k_mma_sub_init(long long n, const double* __restrict__ alfa, const double* __restrict__ beta,
                               double* __restrict__ xs, double* __restrict__ xsi, double* __restrict__ eta) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double a = alfa[j], b = beta[j], x = 0.5 * (a + b);
    xs[j] = x;
    xsi[j] = fmax(1.0 / (x - a), 1.0);
    eta[j] = fmax(1.0 / (b - x), 1.0);
  }
}

struct MmaArrays {
  const double *low, *upp, *alfa, *beta, *p0, *q0, *P, *Q;
};

// reductions: gvec_i (M), bl_i = sum GG_ij delx_j / diagx_j (M), A_ik = sum GG_ij GG_kj / diagx_j
// for i <= k (M (M + 1) / 2, row-major upper triangle)
template <int M>
__global__ void __launch_bounds__(LP_MMA_THREADS) k_mma_newton_a(long long n, int m, MmaArrays A,
                                                                 const double* __restrict__ xs,
                                                                 const double* __restrict__ xsi,
                                                                 const double* __restrict__ eta, MVec lam,
                                                                 double epsi, double* __restrict__ delx,
                                                                 double* __restrict__ diagx,
                                                                 double* __restrict__ part) {
  constexpr int K = 2 * M + M * (M + 1) / 2;
  double acc[K];
  bool is_max[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc[k] = 0.0;
    is_max[k] = false;
  }
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double x = xs[j], ux1 = A.upp[j] - x, xl1 = x - A.low[j];
    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1, ux3 = ux1 * ux2, xl3 = xl1 * xl2;
    double plam = A.p0[j], qlam = A.q0[j];
    double gg[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      gg[i] = 0.0;
      if (i < m) {
        const double Pij = A.P[(long long)i * n + j], Qij = A.Q[(long long)i * n + j];
        plam += Pij * lam.v[i];
        qlam += Qij * lam.v[i];
        acc[i] += Pij / ux1 + Qij / xl1;
        gg[i] = Pij / ux2 - Qij / xl2;
      }
    }
    const double xa = x - A.alfa[j], bx = A.beta[j] - x;
    const double dpsidx = plam / ux2 - qlam / xl2;
    const double dx_ = dpsidx - epsi / xa + epsi / bx;
    const double dg = 2.0 * (plam / ux3 + qlam / xl3) + xsi[j] / xa + eta[j] / bx;
    delx[j] = dx_;
    diagx[j] = dg;
    int k = 2 * M;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      acc[M + i] += gg[i] * (dx_ / dg);
#pragma unroll
      for (int i2 = i; i2 < M; ++i2) acc[k++] += gg[i] * gg[i2] / dg;
    }
  }
  block_reduce<K>(acc, is_max, part);
}

// reductions (all maxima): -1.01 dxsi / xsi, -1.01 deta / eta, -1.01 dx / (x - alfa),
// 1.01 dx / (beta - x)
template <int M>
__global__ void __launch_bounds__(LP_MMA_THREADS) k_mma_newton_b(long long n, int m, MmaArrays A,
                                                                 const double* __restrict__ xs,
                                                                 const double* __restrict__ xsi,
                                                                 const double* __restrict__ eta,
                                                                 const double* __restrict__ delx,
                                                                 const double* __restrict__ diagx, MVec dlam,
                                                                 double epsi, double* __restrict__ dx,
                                                                 double* __restrict__ dxsi, double* __restrict__ deta,
                                                                 double* __restrict__ part) {
  double acc[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
  const bool is_max[4] = {true, true, true, true};
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double x = xs[j], ux1 = A.upp[j] - x, xl1 = x - A.low[j];
    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    double gtl = 0.0;   // (GG^T dlam)_j
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (i < m) gtl += (A.P[(long long)i * n + j] / ux2 - A.Q[(long long)i * n + j] / xl2) * dlam.v[i];
    const double dg = diagx[j];
    const double d = -delx[j] / dg - gtl / dg;
    const double xa = x - A.alfa[j], bx = A.beta[j] - x;
    const double s = xsi[j], e = eta[j];
    const double ds = -s + epsi / xa - s * d / xa;
    const double de = -e + epsi / bx + e * d / bx;
    dx[j] = d;
    dxsi[j] = ds;
    deta[j] = de;
    acc[0] = fmax(acc[0], -1.01 * ds / s);
    acc[1] = fmax(acc[1], -1.01 * de / e);
    acc[2] = fmax(acc[2], -1.01 * d / xa);
    acc[3] = fmax(acc[3], 1.01 * d / bx);
  }
  block_reduce<4>(acc, is_max, part);
}

// x, xsi, eta = old + steg * d; reductions at the new point: sum of squares of the n-sized
// residual parts (dpsidx - xsi + eta, xsi (x - alfa) - epsi, eta (beta - x) - epsi), their largest
// magnitude, and gvec_i (M)
template <int M>
__global__ void __launch_bounds__(LP_MMA_THREADS) k_mma_trial(long long n, int m, MmaArrays A,
                                                              const double* __restrict__ xs0,
                                                              const double* __restrict__ xsi0,
                                                              const double* __restrict__ eta0,
                                                              const double* __restrict__ dx,
                                                              const double* __restrict__ dxsi,
                                                              const double* __restrict__ deta, double steg, MVec lam,
                                                              double epsi, double* __restrict__ xs,
                                                              double* __restrict__ xsi, double* __restrict__ eta,
                                                              double* __restrict__ part) {
  constexpr int K = 2 + M;
  double acc[K];
  bool is_max[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc[k] = 0.0;
    is_max[k] = k == 1;
  }
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    double x = xs0[j], s = xsi0[j], e = eta0[j];
    if (dx) {
      x += steg * dx[j];
      s += steg * dxsi[j];
      e += steg * deta[j];
      xs[j] = x;
      xsi[j] = s;
      eta[j] = e;
    }
    const double ux1 = A.upp[j] - x, xl1 = x - A.low[j];
    double plam = A.p0[j], qlam = A.q0[j];
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (i < m) {
        const double Pij = A.P[(long long)i * n + j], Qij = A.Q[(long long)i * n + j];
        plam += Pij * lam.v[i];
        qlam += Qij * lam.v[i];
        acc[2 + i] += Pij / ux1 + Qij / xl1;
      }
    const double r1 = plam / (ux1 * ux1) - qlam / (xl1 * xl1) - s + e;
    const double r5 = s * (x - A.alfa[j]) - epsi;
    const double r6 = e * (A.beta[j] - x) - epsi;
    acc[0] += r1 * r1 + r5 * r5 + r6 * r6;
    acc[1] = fmax(acc[1], fmax(fabs(r1), fmax(fabs(r5), fabs(r6))));
  }
  block_reduce<K>(acc, is_max, part);
}

__global__ void k_mma_finish(long long n, const double* __restrict__ xs, const double* __restrict__ x,
                             const double* __restrict__ alfa, const double* __restrict__ beta,
                             double* __restrict__ xnew) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    double v = xs[j];
    if (!isfinite(v)) v = x[j];
    xnew[j] = fmin(fmax(v, alfa[j]), beta[j]);
  }
}

// which of a kernel's K reduced values are maxima: a small device table per layout
__device__ int g_mask_sum[64];                              // all zero: sums
__device__ int g_mask_max4[4] = {1, 1, 1, 1};
__device__ int g_mask_trial[2 + LP_MMA_MAXM] = {0, 1};   // [1]: the largest magnitude

static int final_reduce(const double* part, int K, const int* mask_dev, double* out, cudaStream_t st) {
  k_mma_final<<<K, 32, 0, st>>>(part, LP_MMA_BLOCKS, K, mask_dev, out);
  return LP_OK;
}

template <typename T>
static const int* dev_addr(T& sym) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, sym) != cudaSuccess) return nullptr;
  return static_cast<const int*>(p);
}

static int mma_m_template(int m) {
  if (m <= 1) return 1;
  if (m <= 2) return 2;
  if (m <= 4) return 4;
  return 8;
}

static MVec mvec(const double* h, int m) {
  MVec v;
  for (int i = 0; i < LP_MMA_MAXM; ++i) v.v[i] = (h && i < m) ? h[i] : 0.0;
  return v;
}

}  // namespace

#define LP_ST ((cudaStream_t)stream)
#define MMA_GRID LP_MMA_BLOCKS, LP_MMA_THREADS, 0, LP_ST
#define MMA_DISPATCH(KERNEL, ...)                                              \
  switch (mma_m_template(m)) {                                                  \
    case 1: KERNEL<1><<<MMA_GRID>>>(__VA_ARGS__); break;                        \
    case 2: KERNEL<2><<<MMA_GRID>>>(__VA_ARGS__); break;                        \
    case 4: KERNEL<4><<<MMA_GRID>>>(__VA_ARGS__); break;                        \
    default: KERNEL<8><<<MMA_GRID>>>(__VA_ARGS__); break;                       \
  }

extern "C" {

// part: scratch of at least lpb_mma_part_len(m) doubles: LP_MMA_BLOCKS partials for each value
// of the widest reduction any pass makes (prepare M, newton_a 2M + M(M+1)/2, newton_b 4,
// trial 2 + M, M = m rounded up to 1, 2, 4 or 8)
long long lpb_mma_part_len(int m) {
  const int M = mma_m_template(m);
  int K = 2 * M + M * (M + 1) / 2;
  if (K < 4) K = 4;
  if (K < 2 + M) K = 2 + M;
  return (long long)K * LP_MMA_BLOCKS;
}

int lpb_mma_prepare(long long n, int m, double* x, const double* xmin, const double* xmax, double* low, double* upp,
                    const double* xold1, const double* xold2, int init, double asyinit, double asyincr,
                    double asydecr, double move, double* df0, double* df, double* alfa, double* beta, double* p0,
                    double* q0, double* P, double* Q, double* part, double* bsum, void* stream) {
  if (n < 1 || m < 1 || m > LP_MMA_MAXM || !x || !xmin || !xmax || !low || !upp || !df0 || !df || !alfa || !beta ||
      !p0 || !q0 || !P || !Q || !part || !bsum)
    return LP_ERR_ARG;
  if (!init && (!xold1 || !xold2)) return LP_ERR_ARG;
  const int* mask = dev_addr(g_mask_sum);
  if (!mask) return LP_ERR_LAUNCH;
  MMA_DISPATCH(k_mma_prepare, n, m, x, xmin, xmax, low, upp, xold1, xold2, init, asyinit, asyincr, asydecr, move,
               df0, df, alfa, beta, p0, q0, P, Q, part)
  final_reduce(part, mma_m_template(m), mask, bsum, LP_ST);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_mma_sub_init(long long n, const double* alfa, const double* beta, double* xs, double* xsi, double* eta,
                     void* stream) {
  if (n < 1 || !alfa || !beta || !xs || !xsi || !eta) return LP_ERR_ARG;
  k_mma_sub_init<<<MMA_GRID>>>(n, alfa, beta, xs, xsi, eta);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out: gvec (M values), GG (delx / diagx) (M), (GG / diagx) GG^T upper triangle (M (M + 1) / 2),
// M = m rounded up to 1, 2, 4 or 8; lam: HOST pointer to m doubles
int lpb_mma_newton_a(long long n, int m, const double* low, const double* upp, const double* alfa,
                     const double* beta, const double* p0, const double* q0, const double* P, const double* Q,
                     const double* xs, const double* xsi, const double* eta, const double* lam, double epsi,
                     double* delx, double* diagx, double* part, double* out, void* stream) {
  if (n < 1 || m < 1 || m > LP_MMA_MAXM || !low || !upp || !alfa || !beta || !p0 || !q0 || !P || !Q || !xs || !xsi ||
      !eta || !lam || !delx || !diagx || !part || !out)
    return LP_ERR_ARG;
  const int* mask = dev_addr(g_mask_sum);
  if (!mask) return LP_ERR_LAUNCH;
  const MmaArrays A = {low, upp, alfa, beta, p0, q0, P, Q};
  const MVec lv = mvec(lam, m);
  MMA_DISPATCH(k_mma_newton_a, n, m, A, xs, xsi, eta, lv, epsi, delx, diagx, part)
  const int M = mma_m_template(m);
  final_reduce(part, 2 * M + M * (M + 1) / 2, mask, out, LP_ST);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out: the four step-length maxima; dlam: HOST pointer to m doubles
int lpb_mma_newton_b(long long n, int m, const double* low, const double* upp, const double* alfa,
                     const double* beta, const double* P, const double* Q, const double* xs, const double* xsi,
                     const double* eta, const double* delx, const double* diagx, const double* dlam, double epsi,
                     double* dx, double* dxsi, double* deta, double* part, double* out, void* stream) {
  if (n < 1 || m < 1 || m > LP_MMA_MAXM || !low || !upp || !alfa || !beta || !P || !Q || !xs || !xsi || !eta ||
      !delx || !diagx || !dlam || !dx || !dxsi || !deta || !part || !out)
    return LP_ERR_ARG;
  const int* mask = dev_addr(g_mask_max4);
  if (!mask) return LP_ERR_LAUNCH;
  const MmaArrays A = {low, upp, alfa, beta, nullptr, nullptr, P, Q};
  const MVec dl = mvec(dlam, m);
  MMA_DISPATCH(k_mma_newton_b, n, m, A, xs, xsi, eta, delx, diagx, dl, epsi, dx, dxsi, deta, part)
  final_reduce(part, 4, mask, out, LP_ST);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// x, xsi, eta = (x0, xsi0, eta0) + steg (dx, dxsi, deta) (dx NULL: the residual at x0, nothing
// written); out: sum of squares, largest magnitude, gvec (M); lam: HOST pointer to m doubles
int lpb_mma_trial(long long n, int m, const double* low, const double* upp, const double* alfa, const double* beta,
                  const double* p0, const double* q0, const double* P, const double* Q, const double* xs0,
                  const double* xsi0, const double* eta0, const double* dx, const double* dxsi, const double* deta,
                  double steg, const double* lam, double epsi, double* xs, double* xsi, double* eta, double* part,
                  double* out, void* stream) {
  if (n < 1 || m < 1 || m > LP_MMA_MAXM || !low || !upp || !alfa || !beta || !p0 || !q0 || !P || !Q || !xs0 ||
      !xsi0 || !eta0 || !lam || !part || !out)
    return LP_ERR_ARG;
  if (dx && (!dxsi || !deta || !xs || !xsi || !eta)) return LP_ERR_ARG;
  const int* mask = dev_addr(g_mask_trial);
  if (!mask) return LP_ERR_LAUNCH;
  const MmaArrays A = {low, upp, alfa, beta, p0, q0, P, Q};
  const MVec lv = mvec(lam, m);
  MMA_DISPATCH(k_mma_trial, n, m, A, xs0, xsi0, eta0, dx, dxsi, deta, steg, lv, epsi, xs, xsi, eta, part)
  final_reduce(part, 2 + mma_m_template(m), mask, out, LP_ST);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_mma_finish(long long n, const double* xs, const double* x, const double* alfa, const double* beta,
                   double* xnew, void* stream) {
  if (n < 1 || !xs || !x || !alfa || !beta || !xnew) return LP_ERR_ARG;
  k_mma_finish<<<MMA_GRID>>>(n, xs, x, alfa, beta, xnew);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
