// The corner-parity (Walsh) basis of a hex8 cell.
//
// A cell's eight corner values of one component c, u_(3k+c), map to the modes
// u^_(3m+c) = sum_k H[m][k] u_(3k+c), H[m][k] = prod over the axes a set in m of (2 bit_a(k) - 1),
// mode m = mx + 2 my + 4 mz. With T = kron(H, I3), T^T T = 8 I, so for K^ = T Ke T^T / 64
//   u^T Ke v = (T u)^T K^ (T v).
// For the plain and the incompatible-mode brick at any isotropic nu, K^ has 45 non-zeros at the
// fixed positions below (three decoupled blocks; rows and columns 0..2, the rigid translations,
// are zero).
#pragma once

#define LP_MODAL_NNZ 45
#define LP_MODAL_ROWS                                                                                       \
  {3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12, 13, 13, 14, 14, 14, 15, 15, 16, \
   16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21, 22, 23}
#define LP_MODAL_COLS                                                                                       \
  {3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12, 8, 13, 3, 7, 14, 15, 19, 11, \
   16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22, 23}

// H[m][k]
__host__ __device__ __forceinline__ double lp_walsh_h(int m, int k) {
  double v = 1.0;
  for (int a = 0; a < 3; ++a)
    if ((m >> a) & 1) v *= ((k >> a) & 1) ? 1.0 : -1.0;
  return v;
}

// entry (r, c) of K^ = T ke T^T / 64, ke 24 x 24 row-major
__host__ __device__ inline double lp_modal_entry(const double* ke, int r, int c) {
  const int mr = r / 3, cr = r % 3, mc = c / 3, cc = c % 3;
  double s = 0.0;
  for (int k1 = 0; k1 < 8; ++k1) {
    double t = 0.0;
    for (int k2 = 0; k2 < 8; ++k2) t += ke[(3 * k1 + cr) * 24 + 3 * k2 + cc] * lp_walsh_h(mc, k2);
    s += lp_walsh_h(mr, k1) * t;
  }
  return s / 64.0;
}

// In-place Walsh transform of one component's eight corner values: a[k] -> sum_k' H[k][k'] a[k'].
template <typename T>
__device__ __forceinline__ void lp_walsh8(T (&a)[8]) {
#pragma unroll
  for (int b = 1; b < 8; b <<= 1)
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (!(k & b)) {
        const T lo = a[k], hi = a[k | b];
        a[k] = lo + hi;
        a[k | b] = hi - lo;
      }
}
