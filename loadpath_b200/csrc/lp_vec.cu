// Vector passes of the V-cycle and the PCG (loadpath/mgops.py:302-360, :557-585, :593-773):
// Chebyshev updates, fused CG step with |r|^2, p = z + beta p, dots, casts, and the grid
// transfers (residual -> pad -> full-weighting restriction -> coarse mask; prolongation ->
// fine mask -> add).
//
// Reductions are deterministic: a fixed number of blocks (LP_RED_BLOCKS) each write a
// partial sum and one block adds the partials in order, so a given input always gives the
// same bits. Scalars the solver needs between kernels (rz, pap, |r|^2, alpha, beta) live in
// device memory so an iteration never waits on the host.
#include "lp_common.cuh"

#define LP_RED_BLOCKS 592   // 4 per SM on 148 SMs
#define LP_RED_THREADS 512
#define LP_CHEB_MAX_DEGREE 7   // coefficient block of 16 doubles per level

namespace {

template <typename T>
struct V4ld;
template <>
struct V4ld<float> {
  static __device__ __forceinline__ void ld(const float* p, float (&v)[4]) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  static __device__ __forceinline__ void st(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct V4ld<double> {
  static __device__ __forceinline__ void ld(const double* p, double (&v)[4]) {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  static __device__ __forceinline__ void st(double* p, const double (&v)[4]) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
  }
};


template <typename Ta, typename Tb>
__global__ void k_dot_partial(const Ta* __restrict__ a, const Tb* __restrict__ b, long long n,
                              double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// out[0] = sum(part); optional: out_sqrt = sqrt(sum)
__global__ void k_sum_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

// x += alpha p ; r -= alpha ap ; r32 = (float) r ; partial |r|^2. alpha = num / den.
__global__ void k_cg_step(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                          const double* __restrict__ ap, float* __restrict__ r32, long long n,
                          const double* __restrict__ num, const double* __restrict__ den, double* __restrict__ part) {
  __shared__ double sh[32];
  const double alpha = (*num) / (*den);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double ri = r[i] - alpha * ap[i];
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    s += ri * ri;
  }
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// p = z + (num / den) p, z in float32 or float64
template <typename Tz>
__global__ void k_xpby(double* __restrict__ p, const Tz* __restrict__ z, long long n, const double* __restrict__ num,
                       const double* __restrict__ den) {
  const double beta = (*num) / (*den);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = (double)z[i] + beta * p[i];
}

template <typename Ta, typename Tb>
__global__ void k_cast(Tb* __restrict__ out, const Ta* __restrict__ a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (Tb)a[i];
}

// out = a x + b y
template <typename T>
__global__ void k_axpby(T* __restrict__ out, T a, const T* __restrict__ x, T b, const T* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = a * x[i] + (y ? b * y[i] : T(0));
}

// Smoother coefficients live in device memory (written by k_cheb_coef after the power
// iteration), so a V-cycle never needs lmax on the host and a captured V-cycle stays valid when
// the hierarchy is rebuilt: coef[1] = 1 / theta, coef[2 + 2k], coef[3 + 2k] = c1, c2 of step k.

// Chebyshev start from zero: x = 0; r = b; d = (dinv b) s        (loadpath/mgops.py:321-328)
template <typename T>
__global__ void k_cheb_start(const T* __restrict__ b, const T* __restrict__ dinv, const double* __restrict__ coef,
                             T* __restrict__ x, T* __restrict__ r, T* __restrict__ d, long long n) {
  const T s = (T)coef[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T bi = b[i];
    x[i] = T(0);
    r[i] = bi;
    d[i] = (dinv[i] * bi) * s;
  }
}

// r = b - ax; d = s dinv r                                        (loadpath/mgops.py:314-319)
template <typename T>
__global__ void k_residual_scaled(const T* __restrict__ b, const T* __restrict__ ax, const T* __restrict__ dinv,
                                  const double* __restrict__ coef, T* __restrict__ r, T* __restrict__ d, long long n) {
  const T s = (T)coef[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T ri, di;
    lp_residual_scaled_v(b[i], ax[i], dinv[i], s, ri, di);
    r[i] = ri;
    d[i] = di;
  }
}

// x += d; unless last: r -= ad; d = c1 d + c2 dinv r             (loadpath/mgops.py:334-343)
template <typename T>
__global__ void k_cheb(T* __restrict__ x, T* __restrict__ d, T* __restrict__ r, const T* __restrict__ ad,
                       const T* __restrict__ dinv, const double* __restrict__ coef, int step, int last, long long n) {
  const T c1 = (T)coef[2 + 2 * step], c2 = (T)coef[3 + 2 * step];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T di = d[i];
    x[i] += di;
    if (!last) {
      T ri = r[i] - ad[i];
      r[i] = ri;
      d[i] = c1 * di + c2 * dinv[i] * ri;
    }
  }
}

// lmax and the Chebyshev coefficients from the power iteration's dots (loadpath/mg.py:771-794,
// :796-821): lmax = safety * max(v.Av of the last step, 1e-12), or 2 when some |v|^2 was 0;
// the interval is [lmax / 30, lmax]. One thread, float64 throughout.
__global__ void k_cheb_coef(double* __restrict__ coef, const double* __restrict__ vv, const double* __restrict__ vav,
                            int its, int degree, double safety) {
  bool zero = false;
  for (int k = 0; k < its; ++k) zero = zero || vv[k] == 0.0;
  const double lam = vav[its - 1];
  const double hi = zero ? 2.0 : safety * (lam > 1e-12 ? lam : 1e-12);
  const double lo = hi / 30.0;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  coef[0] = hi;
  coef[1] = 1.0 / theta;
  for (int k = 0; k < degree; ++k) {
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    coef[2 + 2 * k] = rho_new * rho;
    coef[3 + 2 * k] = 2.0 * rho_new / delta;
    rho = rho_new;
  }
}

// Degree-2 Chebyshev in two passes per smoothing (the reference's default degree). With
// d' = c1 d + c2 dinv (r - A d) (step 0's update) the two steps give x + d + d', formed here in
// the reference's order ((x + d) + d', and 0 + d = d exactly), so the result is the same bits as
// the step-by-step form while r and d are never rewritten.
// from zero, pass 1: d = (dinv b) s                               (loadpath/mgops.py:321-328)
template <typename T>
__global__ void k_cheb_d_start(const T* __restrict__ b, const T* __restrict__ dinv, const double* __restrict__ coef,
                               T* __restrict__ d, long long n) {
  const T s = (T)coef[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = (dinv[i] * b[i]) * s;
}

// from zero, pass 2 (ad = A d): x = d + (c1 d + c2 dinv (b - ad))
template <typename T>
__global__ void k_cheb2_zero(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ ad,
                             const T* __restrict__ d, const T* __restrict__ dinv, const double* __restrict__ coef,
                             long long n) {
  const T c1 = (T)coef[2], c2 = (T)coef[3];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = lp_cheb2_zero_v(d[i], b[i], ad[i], dinv[i], c1, c2);
}

// from x (after lpb_residual_scaled: r = b - A x, d = s dinv r; ad = A d):
// x = (x + d) + (c1 d + c2 dinv (r - ad))
template <typename T>
__global__ void k_cheb2(T* __restrict__ x, const T* __restrict__ d, const T* __restrict__ r, const T* __restrict__ ad,
                        const T* __restrict__ dinv, const double* __restrict__ coef, long long n) {
  const T c1 = (T)coef[2], c2 = (T)coef[3];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = lp_cheb2_v(x[i], d[i], r[i], ad[i], dinv[i], c1, c2);
}

// damped Jacobi: x += omega dinv (b - ax), x = 0 start handled by the caller
template <typename T>
__global__ void k_jacobi(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ ax,
                         const T* __restrict__ dinv, T omega, int from_zero, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (from_zero)
      x[i] = omega * dinv[i] * b[i];
    else
      x[i] += omega * dinv[i] * (b[i] - ax[i]);
  }
}

// ---- grid transfers by z chunks -----------------------------------------------------------
// One thread per (x, y) node column and chunk of four z planes (x fastest across threads), the
// chunk's values moved with 16-byte loads and stores, the trilinear weights applied separably
// (z inside a column first).

// rc = restrict(((b - ax) * m) zero-padded) * cm (loadpath/mgops.py:666-711). One warp per 15
// coarse columns X0..X0+14 of one coarse row Y and chunk C (coarse planes 4C..4C+3): lane l
// reads fine column x = 2 X0 - 1 + l (rows 2Y - 1 .. 2Y + 1, fine planes 8C - 1 .. 8C + 7), so a
// warp's loads are 32 consecutive 16-byte chunk rows; the lane restricts z and y in registers,
// and the odd lanes (x = 2X) finish x with their two neighbours' sums by shuffles and store.
constexpr int R4_COLS = 15;   // coarse columns per warp

template <typename T>
__global__ void k_restrict4(T* __restrict__ rc, const T* __restrict__ b, const T* __restrict__ ax,
                            const uint8_t* __restrict__ m, const uint8_t* __restrict__ cm, LpGrid gf, LpGrid gc) {
  const int CX = gc.NX(), CY = gc.NY(), CZ4 = gc.pz / 4;
  const int FX = gf.NX(), FY = gf.NY();
  const int ngx = (CX + R4_COLS - 1) / R4_COLS;
  const long long nwarps = (long long)ngx * CY * CZ4;
  const long long fcs = gf.comp_stride(), ccs = gc.comp_stride(), fzs = gf.node_zc_stride();
  const int lane = threadIdx.x & 31;
  const long long wstep = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < nwarps; w += wstep) {
    const int gx = (int)(w % ngx);
    const long long q = w / ngx;
    const int Y = (int)(q % CY), C = (int)(q / CY);
    const int X0 = gx * R4_COLS;
    const int x = 2 * X0 - 1 + lane;
    const int z0 = 8 * C;
    // a coarse level padded up past half the fine one reaches beyond the fine pitch: zeros
    const bool below = z0 >= 1 && z0 - 1 < gf.pz, lo = z0 < gf.pz, hi = z0 + 4 < gf.pz;
    T acc[3][4] = {};
    if (x >= 0 && x < FX) {
#pragma unroll 1
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = 2 * Y + dy;
        if (y < 0 || y >= FY) continue;
        const T wy = dy ? T(0.5) : T(1);
        const long long n_lo = lo ? gf.node(x, y, z0) : 0, n_hi = n_lo + fzs;
        const long long n_below = below ? gf.node(x, y, z0 - 1) : 0;
        uint8_t mz[9];
        mz[0] = below ? m[n_below] : 0;
        const uchar4 ma = lo ? *reinterpret_cast<const uchar4*>(m + n_lo) : make_uchar4(0, 0, 0, 0);
        const uchar4 mb = hi ? *reinterpret_cast<const uchar4*>(m + n_hi) : make_uchar4(0, 0, 0, 0);
        mz[1] = ma.x; mz[2] = ma.y; mz[3] = ma.z; mz[4] = ma.w;
        mz[5] = mb.x; mz[6] = mb.y; mz[7] = mb.z; mz[8] = mb.w;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T* bi = b + i * fcs;
          const T* ai = ax + i * fcs;
          T v[9];
          v[0] = below ? bi[n_below] - ai[n_below] : T(0);
          T b4[4], a4[4];
          if (lo) {
            V4ld<T>::ld(bi + n_lo, b4);
            V4ld<T>::ld(ai + n_lo, a4);
#pragma unroll
            for (int k = 0; k < 4; ++k) v[1 + k] = b4[k] - a4[k];
          } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) v[1 + k] = T(0);
          }
          if (hi) {
            V4ld<T>::ld(bi + n_hi, b4);
            V4ld<T>::ld(ai + n_hi, a4);
#pragma unroll
            for (int k = 0; k < 4; ++k) v[5 + k] = b4[k] - a4[k];
          } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) v[5 + k] = T(0);
          }
#pragma unroll
          for (int k = 0; k < 9; ++k) v[k] = ((mz[k] >> i) & 1) ? v[k] : T(0);
          // coarse Z = 4C + kk sums fine z = 2Z - 1, 2Z, 2Z + 1 = v[2kk], v[2kk + 1], v[2kk + 2]
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            acc[i][kk] += wy * (T(0.5) * v[2 * kk] + v[2 * kk + 1] + T(0.5) * v[2 * kk + 2]);
        }
      }
    }
    // x: coarse X = X0 + (lane - 1) / 2 on the odd lanes, from fine x - 1, x, x + 1
    const int X = X0 + ((lane - 1) >> 1);
    const bool out = (lane & 1) && lane <= 2 * R4_COLS - 1 && X < CX;
    T o[3][4];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const T l = __shfl_up_sync(0xffffffffu, acc[i][kk], 1);
        const T r = __shfl_down_sync(0xffffffffu, acc[i][kk], 1);
        o[i][kk] = T(0.5) * l + acc[i][kk] + T(0.5) * r;
      }
    if (out) {
      const long long cn = gc.node(X, Y, 4 * C);
      const uchar4 cmb = *reinterpret_cast<const uchar4*>(cm + cn);
      const uint8_t cms[4] = {cmb.x, cmb.y, cmb.z, cmb.w};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        T ov[4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) ov[kk] = ((cms[kk] >> i) & 1) ? o[i][kk] : T(0);
        V4ld<T>::st(rc + i * ccs + cn, ov);
      }
    }
  }
}

// x += prolong(xc * cm) * m for fine nodes (x, y, 4c..4c+3): coarse planes 2c, 2c + 1, 2c + 2 of
// the one, two or four coarse columns around (x / 2, y / 2)   (loadpath/mgops.py:714-750)
template <typename T>
__global__ void k_prolong4(T* __restrict__ xf, const T* __restrict__ xc, const uint8_t* __restrict__ cm,
                           const uint8_t* __restrict__ m, LpGrid gf, LpGrid gc) {
  const long long total = gf.nodes_padded() / 4;
  const long long fcs = gf.comp_stride(), ccs = gc.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, c;
    gf.node_at(4 * t, x, y, c);
    c >>= 2;
    const long long fn = 4 * t;
    const uchar4 mb = *reinterpret_cast<const uchar4*>(m + fn);
    const uint8_t ms[4] = {mb.x, mb.y, mb.z, mb.w};
    if (((mb.x | mb.y | mb.z | mb.w) & 7) == 0) continue;
    const int X0 = x >> 1, Y0 = y >> 1, ox = x & 1, oy = y & 1;
    const int Z0 = 2 * c;
    const int zmax = gc.pz - 1;
    T acc[3][4] = {};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (a && !ox) break;
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        if (bb && !oy) break;
        const T w = (ox ? T(0.5) : T(1)) * (oy ? T(0.5) : T(1));
        long long cn[3];
        uint8_t cmz[3];
        T cv[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          cn[k] = gc.node(X0 + a, Y0 + bb, min(Z0 + k, zmax));
          cmz[k] = cm[cn[k]];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const T v = xc[i * ccs + cn[k]];
            cv[i][k] = ((cmz[k] >> i) & 1) ? v : T(0);
          }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          acc[i][0] += w * cv[i][0];
          acc[i][1] += w * (T(0.5) * (cv[i][0] + cv[i][1]));
          acc[i][2] += w * cv[i][1];
          acc[i][3] += w * (T(0.5) * (cv[i][1] + cv[i][2]));
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T o[4];
      V4ld<T>::ld(xf + i * fcs + fn, o);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if ((ms[k] >> i) & 1) o[k] += acc[i][k];
      V4ld<T>::st(xf + i * fcs + fn, o);
    }
  }
}

// out = u * mask (per component bit); four nodes per step (the padded node count is a multiple
// of 4), the component found by comparison, not by a 64-bit division
template <typename T>
__global__ void k_mask_field(T* __restrict__ out, const T* __restrict__ u, const uint8_t* __restrict__ m, LpGrid g,
                             int bitshift) {
  const long long nq = g.nodes_padded() >> 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3 * nq; i += (long long)gridDim.x * blockDim.x) {
    const int c = i >= nq ? (i >= 2 * nq ? 2 : 1) : 0;
    const uchar4 mb = reinterpret_cast<const uchar4*>(m)[i - c * nq];
    const int sh = c + bitshift;
    T v[4];
    V4ld<T>::ld(u + 4 * i, v);
    if (!((mb.x >> sh) & 1)) v[0] = T(0);
    if (!((mb.y >> sh) & 1)) v[1] = T(0);
    if (!((mb.z >> sh) & 1)) v[2] = T(0);
    if (!((mb.w >> sh) & 1)) v[3] = T(0);
    V4ld<T>::st(out + 4 * i, v);
  }
}

// v *= 1 / sqrt(*nrm2) (power iteration normalisation); leaves v alone when the norm is 0
template <typename T>
__global__ void k_scale_rsqrt(T* __restrict__ v, long long n, const double* __restrict__ nrm2) {
  double s = *nrm2;
  if (s <= 0.0) return;
  T f = (T)(1.0 / sqrt(s));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = v[i] / (T)sqrt(s);
  (void)f;
}

// av = dinv * av * mask, four nodes per step as k_mask_field
template <typename T>
__global__ void k_dinv_mask(T* __restrict__ av, const T* __restrict__ dinv, const uint8_t* __restrict__ m, LpGrid g) {
  const long long nq = g.nodes_padded() >> 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3 * nq; i += (long long)gridDim.x * blockDim.x) {
    const int c = i >= nq ? (i >= 2 * nq ? 2 : 1) : 0;
    const uchar4 mb = reinterpret_cast<const uchar4*>(m)[i - c * nq];
    T v[4], d[4];
    V4ld<T>::ld(av + 4 * i, v);
    V4ld<T>::ld(dinv + 4 * i, d);
    v[0] = ((mb.x >> c) & 1) ? d[0] * v[0] : T(0);
    v[1] = ((mb.y >> c) & 1) ? d[1] * v[1] : T(0);
    v[2] = ((mb.z >> c) & 1) ? d[2] * v[2] : T(0);
    v[3] = ((mb.w >> c) & 1) ? d[3] * v[3] : T(0);
    V4ld<T>::st(av + 4 * i, v);
  }
}


// Warm start of the PCG on the device (loadpath/mg.py:878-895), so the solve never waits on
// the host before its first iteration. sc: [0] b.b, [5] x.Ax, [6] b.x, [7] |rs|^2.
//   s = b.x / x.Ax when x.Ax > 0, else 0;  rs = b - s Ax
__device__ __forceinline__ double lp_warm_scale(const double* sc) { return sc[5] > 0.0 ? sc[6] / sc[5] : 0.0; }

__global__ void k_warm_residual(double* __restrict__ rs, const double* __restrict__ b, const double* __restrict__ ax,
                                const double* __restrict__ sc, long long n) {
  const double s = lp_warm_scale(sc);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    rs[i] = b[i] - s * ax[i];
}

// keep the scaled warm start when s > 0 and |rs| < |b| (x = s x, r = rs), else x = 0, r = b
__global__ void k_warm_select(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ b,
                              const double* __restrict__ rs, const double* __restrict__ sc, long long n) {
  const double s = lp_warm_scale(sc);
  const bool keep = s > 0.0 && sqrt(sc[7]) < sqrt(sc[0]);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = keep ? x[i] * s : 0.0;
    r[i] = keep ? rs[i] : b[i];
  }
}

// The CG update split for fewer passes over the float64 fields: the step after A p only moves
// r (and its float32 copy) and forms |r|^2; x += alpha p is deferred to the pass that rebuilds p,
// which reads p anyway. alpha = rz / pap and beta = rz_new / rz are read on the device.
__global__ void k_cg_step_r(double* __restrict__ r, const double* __restrict__ ap, float* __restrict__ r32,
                            long long n, const double* __restrict__ num, const double* __restrict__ den,
                            double* __restrict__ part) {
  __shared__ double sh[32];
  const double alpha = (*num) / (*den);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ri = r[i] - alpha * ap[i];
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    s += ri * ri;
  }
  s = lp_block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// x += (rz / pap) p; p = z + (rz_new / rz) p
template <typename Tz>
__global__ void k_xpby_x(double* __restrict__ p, double* __restrict__ x, const Tz* __restrict__ z, long long n,
                         const double* __restrict__ rz, const double* __restrict__ pap,
                         const double* __restrict__ rz_new) {
  const double alpha = (*rz) / (*pap), beta = (*rz_new) / (*rz);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double pi = p[i];
    x[i] += alpha * pi;
    p[i] = (double)z[i] + beta * pi;
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)
#define LP_VEC_GRID(n) lp_blocks((n), 256) > 148 * 32 ? 148 * 32 : lp_blocks((n), 256), 256, 0, LP_ST

extern "C" {

int lpb_reduce_blocks(void) { return LP_RED_BLOCKS; }

// record a CUDA event on a stream; inside a stream capture it becomes an event-record node, so
// every replay of the graph records it again (for timing kernels inside graphs)
int lpb_event_record(void* event, void* stream) {
  if (!event) return LP_ERR_ARG;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(LP_ST, &cs) != cudaSuccess) return LP_ERR_LAUNCH;
  const cudaError_t e = cs == cudaStreamCaptureStatusActive
                            ? cudaEventRecordWithFlags((cudaEvent_t)event, LP_ST, cudaEventRecordExternal)
                            : cudaEventRecord((cudaEvent_t)event, LP_ST);
  return e == cudaSuccess ? LP_OK : LP_ERR_LAUNCH;
}

int lpb_dot_f64(const double* a, const double* b, long long n, double* part, double* out, void* stream) {
  if (!a || !b || !part || !out || n < 0) return LP_ERR_ARG;
  k_dot_partial<double, double><<<LP_RED_BLOCKS, LP_RED_THREADS, 0, LP_ST>>>(a, b, n, part);
  k_sum_final<<<1, 1024, 0, LP_ST>>>(part, LP_RED_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_dot_f32(const float* a, const float* b, long long n, double* part, double* out, void* stream) {
  if (!a || !b || !part || !out || n < 0) return LP_ERR_ARG;
  k_dot_partial<float, float><<<LP_RED_BLOCKS, LP_RED_THREADS, 0, LP_ST>>>(a, b, n, part);
  k_sum_final<<<1, 1024, 0, LP_ST>>>(part, LP_RED_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_dot_f64_f32(const double* a, const float* b, long long n, double* part, double* out, void* stream) {
  if (!a || !b || !part || !out || n < 0) return LP_ERR_ARG;
  k_dot_partial<double, float><<<LP_RED_BLOCKS, LP_RED_THREADS, 0, LP_ST>>>(a, b, n, part);
  k_sum_final<<<1, 1024, 0, LP_ST>>>(part, LP_RED_BLOCKS, out);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cg_step(double* x, double* r, const double* p, const double* ap, float* r32, long long n, const double* num,
                const double* den, double* part, double* rr, void* stream) {
  if (!x || !r || !p || !ap || !num || !den || !part || !rr) return LP_ERR_ARG;
  k_cg_step<<<LP_RED_BLOCKS, LP_RED_THREADS, 0, LP_ST>>>(x, r, p, ap, r32, n, num, den, part);
  k_sum_final<<<1, 1024, 0, LP_ST>>>(part, LP_RED_BLOCKS, rr);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_xpby_f32(double* p, const float* z, long long n, const double* num, const double* den, void* stream) {
  if (!p || !z || !num || !den) return LP_ERR_ARG;
  k_xpby<float><<<LP_VEC_GRID(n)>>>(p, z, n, num, den);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_xpby_f64(double* p, const double* z, long long n, const double* num, const double* den, void* stream) {
  if (!p || !z || !num || !den) return LP_ERR_ARG;
  k_xpby<double><<<LP_VEC_GRID(n)>>>(p, z, n, num, den);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_axpby_f64(double* out, double a, const double* x, double b, const double* y, long long n, void* stream) {
  if (!out || !x) return LP_ERR_ARG;
  k_axpby<double><<<LP_VEC_GRID(n)>>>(out, a, x, b, y, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_axpby_f32(float* out, float a, const float* x, float b, const float* y, long long n, void* stream) {
  if (!out || !x) return LP_ERR_ARG;
  k_axpby<float><<<LP_VEC_GRID(n)>>>(out, a, x, b, y, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cast_f64_f32(float* out, const double* a, long long n, void* stream) {
  if (!out || !a) return LP_ERR_ARG;
  k_cast<double, float><<<LP_VEC_GRID(n)>>>(out, a, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cast_f32_f64(double* out, const float* a, long long n, void* stream) {
  if (!out || !a) return LP_ERR_ARG;
  k_cast<float, double><<<LP_VEC_GRID(n)>>>(out, a, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cheb_coef(double* coef, const double* vv, const double* vav, int its, int degree, double safety,
                  void* stream) {
  if (!coef || !vv || !vav || its < 1 || degree < 1 || degree > LP_CHEB_MAX_DEGREE) return LP_ERR_ARG;
  k_cheb_coef<<<1, 1, 0, LP_ST>>>(coef, vv, vav, its, degree, safety);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cheb_start_f32(const float* b, const float* dinv, const double* coef, float* x, float* r, float* d,
                       long long n, void* stream) {
  if (!b || !dinv || !coef || !x || !r || !d) return LP_ERR_ARG;
  k_cheb_start<float><<<LP_VEC_GRID(n)>>>(b, dinv, coef, x, r, d, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cheb_start_f64(const double* b, const double* dinv, const double* coef, double* x, double* r, double* d,
                       long long n, void* stream) {
  if (!b || !dinv || !coef || !x || !r || !d) return LP_ERR_ARG;
  k_cheb_start<double><<<LP_VEC_GRID(n)>>>(b, dinv, coef, x, r, d, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_residual_scaled_f32(const float* b, const float* ax, const float* dinv, const double* coef, float* r,
                            float* d, long long n, void* stream) {
  if (!b || !ax || !dinv || !coef || !r || !d) return LP_ERR_ARG;
  k_residual_scaled<float><<<LP_VEC_GRID(n)>>>(b, ax, dinv, coef, r, d, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_residual_scaled_f64(const double* b, const double* ax, const double* dinv, const double* coef, double* r,
                            double* d, long long n, void* stream) {
  if (!b || !ax || !dinv || !coef || !r || !d) return LP_ERR_ARG;
  k_residual_scaled<double><<<LP_VEC_GRID(n)>>>(b, ax, dinv, coef, r, d, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cheb_f32(float* x, float* d, float* r, const float* ad, const float* dinv, const double* coef, int step,
                 int last, long long n, void* stream) {
  if (!x || !d || !r || !ad || !dinv || !coef || step < 0 || step >= LP_CHEB_MAX_DEGREE) return LP_ERR_ARG;
  k_cheb<float><<<LP_VEC_GRID(n)>>>(x, d, r, ad, dinv, coef, step, last, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_cheb_f64(double* x, double* d, double* r, const double* ad, const double* dinv, const double* coef, int step,
                 int last, long long n, void* stream) {
  if (!x || !d || !r || !ad || !dinv || !coef || step < 0 || step >= LP_CHEB_MAX_DEGREE) return LP_ERR_ARG;
  k_cheb<double><<<LP_VEC_GRID(n)>>>(x, d, r, ad, dinv, coef, step, last, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

#define LP_CHEB2_ENTRIES(T, SFX)                                                                            \
  int lpb_cheb_d_start_##SFX(const T* b, const T* dinv, const double* coef, T* d, long long n, void* stream) { \
    if (!b || !dinv || !coef || !d) return LP_ERR_ARG;                                                   \
    k_cheb_d_start<T><<<LP_VEC_GRID(n)>>>(b, dinv, coef, d, n);                                          \
    LP_LAUNCH_CHECK();                                                                                    \
    return LP_OK;                                                                                         \
  }                                                                                                       \
  int lpb_cheb2_zero_##SFX(T* x, const T* b, const T* ad, const T* d, const T* dinv, const double* coef,  \
                           long long n, void* stream) {                                                  \
    if (!x || !b || !ad || !d || !dinv || !coef) return LP_ERR_ARG;                                     \
    k_cheb2_zero<T><<<LP_VEC_GRID(n)>>>(x, b, ad, d, dinv, coef, n);                                     \
    LP_LAUNCH_CHECK();                                                                                    \
    return LP_OK;                                                                                         \
  }                                                                                                       \
  int lpb_cheb2_##SFX(T* x, const T* d, const T* r, const T* ad, const T* dinv, const double* coef,       \
                      long long n, void* stream) {                                                       \
    if (!x || !d || !r || !ad || !dinv || !coef) return LP_ERR_ARG;                                     \
    k_cheb2<T><<<LP_VEC_GRID(n)>>>(x, d, r, ad, dinv, coef, n);                                          \
    LP_LAUNCH_CHECK();                                                                                    \
    return LP_OK;                                                                                         \
  }
LP_CHEB2_ENTRIES(float, f32)
LP_CHEB2_ENTRIES(double, f64)

int lpb_cg_step_r(double* r, const double* ap, float* r32, long long n, const double* num, const double* den,
                  double* part, double* rr, void* stream) {
  if (!r || !ap || !num || !den || !part || !rr) return LP_ERR_ARG;
  k_cg_step_r<<<LP_RED_BLOCKS, LP_RED_THREADS, 0, LP_ST>>>(r, ap, r32, n, num, den, part);
  k_sum_final<<<1, 1024, 0, LP_ST>>>(part, LP_RED_BLOCKS, rr);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_xpby_x_f32(double* p, double* x, const float* z, long long n, const double* rz, const double* pap,
                   const double* rz_new, void* stream) {
  if (!p || !x || !z || !rz || !pap || !rz_new) return LP_ERR_ARG;
  k_xpby_x<float><<<LP_VEC_GRID(n)>>>(p, x, z, n, rz, pap, rz_new);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_xpby_x_f64(double* p, double* x, const double* z, long long n, const double* rz, const double* pap,
                   const double* rz_new, void* stream) {
  if (!p || !x || !z || !rz || !pap || !rz_new) return LP_ERR_ARG;
  k_xpby_x<double><<<LP_VEC_GRID(n)>>>(p, x, z, n, rz, pap, rz_new);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_jacobi_f32(float* x, const float* b, const float* ax, const float* dinv, float omega, int from_zero,
                   long long n, void* stream) {
  k_jacobi<float><<<LP_VEC_GRID(n)>>>(x, b, ax, dinv, omega, from_zero, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_jacobi_f64(double* x, const double* b, const double* ax, const double* dinv, double omega, int from_zero,
                   long long n, void* stream) {
  k_jacobi<double><<<LP_VEC_GRID(n)>>>(x, b, ax, dinv, omega, from_zero, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

#define LP_FC_ARGS int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz
#define LP_GF lp_grid(fnx, fny, fnz, fpz, fcpz)
#define LP_GC lp_grid(cnx, cny, cnz, cpz_, ccpz)

// a fine level and the level below it: on each axis the coarse cells are ceil(fine cells / 2),
// or one more when the coarse count is padded to even (loadpath/mg.py:607); the prolongation
// reads coarse nodes up to ceil(fine / 2), the restriction checks its fine reads against the fine
// grid
static bool lp_axis_ok(int f, int c) { return c >= (f + 1) / 2 && c <= (f + 1) / 2 + 1; }
static bool lp_pair_ok(const LpGrid& gf, const LpGrid& gc) {
  return lp_axis_ok(gf.nx, gc.nx) && lp_axis_ok(gf.ny, gc.ny) && lp_axis_ok(gf.nz, gc.nz);
}

int lpb_restrict_residual_f32(float* rc, const float* b, const float* ax, const uint8_t* m, const uint8_t* cm,
                              LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !rc || !b || !ax || !m || !cm) return LP_ERR_ARG;
  if (!lp_pair_ok(gf, gc)) return LP_ERR_ARG;
  const long long nw = (long long)((gc.NX() + R4_COLS - 1) / R4_COLS) * gc.NY() * (gc.pz / 4);
  k_restrict4<float><<<lp_blocks(32 * nw, 128), 128, 0, LP_ST>>>(rc, b, ax, m, cm, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_restrict_residual_f64(double* rc, const double* b, const double* ax, const uint8_t* m, const uint8_t* cm,
                              LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !rc || !b || !ax || !m || !cm) return LP_ERR_ARG;
  if (!lp_pair_ok(gf, gc)) return LP_ERR_ARG;
  const long long nw = (long long)((gc.NX() + R4_COLS - 1) / R4_COLS) * gc.NY() * (gc.pz / 4);
  k_restrict4<double><<<lp_blocks(32 * nw, 128), 128, 0, LP_ST>>>(rc, b, ax, m, cm, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_prolong_add_f32(float* x, const float* xc, const uint8_t* cm, const uint8_t* m, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !x || !xc || !m || !cm) return LP_ERR_ARG;
  if (!lp_pair_ok(gf, gc)) return LP_ERR_ARG;
  const long long t4 = gf.nodes_padded() / 4;
  k_prolong4<float><<<lp_blocks(t4, 128), 128, 0, LP_ST>>>(x, xc, cm, m, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_prolong_add_f64(double* x, const double* xc, const uint8_t* cm, const uint8_t* m, LP_FC_ARGS, void* stream) {
  LpGrid gf = LP_GF, gc = LP_GC;
  if (!lp_grid_ok(gf) || !lp_grid_ok(gc) || !x || !xc || !m || !cm) return LP_ERR_ARG;
  if (!lp_pair_ok(gf, gc)) return LP_ERR_ARG;
  const long long t4 = gf.nodes_padded() / 4;
  k_prolong4<double><<<lp_blocks(t4, 128), 128, 0, LP_ST>>>(x, xc, cm, m, gf, gc);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_mask_field_f32(float* out, const float* u, const uint8_t* m, LP_GRID_ARGS, int bitshift, void* stream) {
  LpGrid g = LP_GRID;
  long long n = 3 * g.nodes_padded();
  k_mask_field<float><<<LP_VEC_GRID(n / 4)>>>(out, u, m, g, bitshift);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_mask_field_f64(double* out, const double* u, const uint8_t* m, LP_GRID_ARGS, int bitshift, void* stream) {
  LpGrid g = LP_GRID;
  long long n = 3 * g.nodes_padded();
  k_mask_field<double><<<LP_VEC_GRID(n / 4)>>>(out, u, m, g, bitshift);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_scale_rsqrt_f32(float* v, long long n, const double* nrm2, void* stream) {
  k_scale_rsqrt<float><<<LP_VEC_GRID(n)>>>(v, n, nrm2);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_scale_rsqrt_f64(double* v, long long n, const double* nrm2, void* stream) {
  k_scale_rsqrt<double><<<LP_VEC_GRID(n)>>>(v, n, nrm2);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_dinv_mask_f32(float* av, const float* dinv, const uint8_t* m, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  long long n = 3 * g.nodes_padded();
  k_dinv_mask<float><<<LP_VEC_GRID(n / 4)>>>(av, dinv, m, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_dinv_mask_f64(double* av, const double* dinv, const uint8_t* m, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  long long n = 3 * g.nodes_padded();
  k_dinv_mask<double><<<LP_VEC_GRID(n / 4)>>>(av, dinv, m, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_warm_residual(double* rs, const double* b, const double* ax, const double* sc, long long n, void* stream) {
  if (!rs || !b || !ax || !sc || n < 0) return LP_ERR_ARG;
  k_warm_residual<<<LP_VEC_GRID(n)>>>(rs, b, ax, sc, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_warm_select(double* x, double* r, const double* b, const double* rs, const double* sc, long long n,
                    void* stream) {
  if (!x || !r || !b || !rs || !sc || n < 0) return LP_ERR_ARG;
  k_warm_select<<<LP_VEC_GRID(n)>>>(x, r, b, rs, sc, n);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
