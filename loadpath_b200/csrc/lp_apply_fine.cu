// Fine-level operator on the hot path: out = m * K(E) u + (1 - m) * u for u that is zero on
// masked dofs (every vector the solver makes), K = sum_cells E_c Ke
// (loadpath/mg.py:317-346 -> loadpath/mgops.py:86-103 + :181-217 with finish).
//
// Corner-parity basis. A cell's eight corner values of one component, rewritten in the modes
// {1, sx, sy, sxsy, sz, sxsz, sysz, sxsysz} (s = +-1 per axis), turn the 24 x 24 element matrix
// into one with 45 non-zeros (for the plain and the incompatible-mode brick alike, any isotropic
// nu): three decoupled blocks (linear, bilinear and trilinear modes). The unit brick's cubic
// symmetry leaves seven coefficient classes in those blocks (lpb_modal_sym), so with the cell's
// modulus folded into them a cell costs about 140 floating-point operations instead of the dense
// 1152:
//   linear normal   {(sx,x), (sy,y), (sz,z)}:      f = (a - b) v + b (v1 + v2 + v3)
//   linear shear    {(sx,y), (sy,x)} and its two axis permutations: f1 = f2 = d (v1 + v2)
//                   (the shear strain sees both modes alike: the block has rank one)
//   bilinear normal {(sxsy,z), (sxsz,y), (sysz,x)}: f = b2 v + b2 (v1 + v2 + v3)
//   bilinear shear  {(sxsy,x), (sysz,z)} and its two permutations: f1 = d2 v1 + e2 v2, f2 = e2 v1 + d2 v2
//   trilinear       (sxsysz, c):                  f = t v
//
// Work layout. A block owns a 15 x 15 patch of node columns and runs 16 x 16 threads, one per
// cell column of the patch plus a one-cell halo on the low x and y sides, lanes along x. It
// marches along z one chunk of four planes at a time: TMA brings the chunk's 17 x 17 node
// columns and 16 x 16 cell moduli into a ring of shared-memory stages; in the z-chunked field
// layout every box row is one contiguous run of columns x 4 planes. A thread forms its cells two
// at a time, cells (0, 1) then (2, 3) of the chunk, as pairs of values: the x-y modes of planes
// (0, 1) and (2, 3) come from one two-plane load per node column, the next chunk's planes (0, 1)
// are formed once and carried, and a pair of cells takes its upper planes (1, 2) or (3, 4) from
// those. A node plane's modal force is the upper face of the cell below plus the lower face of
// the cell above, both in this thread (a carry between chunks), so z needs no exchange; the four
// cell columns around a node column meet through warp shuffles (x) and shared memory (y), one
// block barrier per chunk. No atomics, no scatter: every output is written once by its owner.
// The pairs are plain registers and scalar instructions: a packed f32x2 form measured slower on
// B200 (58.8 against 55.3 us at 256 x 128 x 128), its repacking between pairs costing more issue
// slots than the packing saves.
//
// Requirements (checked by the host entry): pz % 4 == 0 and cpz == pz; u, e and the mask
// hold zeros in the z padding; u is zero on dofs whose mask bit is 0, so the identity rows
// (1 - m) u of the masked operator vanish and the kernel writes m * K u.
#include <cstring>
#include <initializer_list>
#include <mutex>

#include "lp_common.cuh"
#include "lp_modal.cuh"
#include "lp_tma.cuh"

namespace {

constexpr int TXC = 16;         // cell columns per block in x (15 owned node columns)
constexpr int TYC = 16;         // in y
constexpr int BOX = TXC + 1;    // 17 node columns per side in a loaded box
constexpr int NST = 3;          // TMA ring depth (chunks of four z planes; loads run NST - 1 ahead)

// every TMA destination starts on a 128-byte boundary
template <typename T, int N>
struct alignas(128) Slot {
  T v[(N * sizeof(T) + 127) / 128 * 128 / sizeof(T)];
};

// The fields as TMA tensors: a chunk's row of x columns (4 z values each) is the inner
// dimension, so every box row is one contiguous run.
struct FineMaps {
  CUtensorMap u;    // (4 NX, NY, pz / 4, 3), box (4 * 17, 17, 1, 3)
  CUtensorMap e;    // (4 nx, ny, cpz / 4),    box (4 * 16, 16, 1)
};

// two values of a field (two cells, or two planes of a node column) carried together
template <typename T>
struct Pair {
  T a, b;
};

template <typename T>
struct PairOps {
  typedef Pair<T> P;
  static __device__ __forceinline__ P mk(T a, T b) { return P{a, b}; }
  static __device__ __forceinline__ P add(P x, P y) { return P{x.a + y.a, x.b + y.b}; }
  static __device__ __forceinline__ P sub(P x, P y) { return P{x.a - y.a, x.b - y.b}; }
  static __device__ __forceinline__ P mul(P x, P y) { return P{x.a * y.a, x.b * y.b}; }
  static __device__ __forceinline__ P fma(P x, P y, P z) { return P{fmr(x.a, y.a, z.a), fmr(x.b, y.b, z.b)}; }
  static __device__ __forceinline__ P zero() { return P{T(0), T(0)}; }
  static __device__ __forceinline__ P shfl_up1(P v) {
    return P{__shfl_up_sync(0xffffffffu, v.a, 1, TXC), __shfl_up_sync(0xffffffffu, v.b, 1, TXC)};
  }
  // two consecutive values (an even offset into a 4-plane column)
  static __device__ __forceinline__ P lds2(const T* p);
  static __device__ __forceinline__ void sts(P* p, P v);
  static __device__ __forceinline__ float fmr(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ double fmr(double a, double b, double c) { return __fma_rn(a, b, c); }
};
template <>
__device__ __forceinline__ PairOps<float>::P PairOps<float>::lds2(const float* p) {
  const float2 v = *reinterpret_cast<const float2*>(p);
  return P{v.x, v.y};
}
template <>
__device__ __forceinline__ PairOps<double>::P PairOps<double>::lds2(const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return P{v.x, v.y};
}
template <>
__device__ __forceinline__ void PairOps<float>::sts(P* p, P v) {
  *reinterpret_cast<float2*>(p) = make_float2(v.a, v.b);
}
template <>
__device__ __forceinline__ void PairOps<double>::sts(P* p, P v) {
  *reinterpret_cast<double2*>(p) = make_double2(v.a, v.b);
}

// the seven coefficient classes of the symmetric product
template <typename T>
struct KSym {
  T c[7];   // a - b, b, d, b2, d2, e2, t
};

template <typename T>
struct FineSmem {
  Slot<T, 3 * BOX * BOX * 4> u[NST];                 // node values [comp][y][x][z]
  Slot<T, TXC * TYC * 4> e[NST];                     // cell moduli [y][x][z]
  Pair<T> red[2][2][3][TXC * TYC];                   // y exchange [chunk parity][plane pair][comp][thread]
  alignas(8) uint64_t full[NST];
};

template <typename T>
__device__ __forceinline__ const T* col_at(const FineSmem<T>& sm, int s, int c, int x, int y) {
  return &sm.u[s].v[((c * BOX + y) * BOX + x) * 4];
}

// x-y modes of two consecutive planes (zo = 0: planes 0, 1; zo = 2: planes 2, 3) of the thread's
// four node columns 00, 10, 01, 11: m[q][c], q = const, sx, sy, sxsy
template <typename T>
__device__ __forceinline__ void plane_modes(const FineSmem<T>& sm, int s, int i, int j, int zo, Pair<T> (&m)[4][3]) {
  typedef PairOps<T> O;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Pair<T> v0 = O::lds2(col_at(sm, s, c, i, j) + zo), v1 = O::lds2(col_at(sm, s, c, i + 1, j) + zo);
    const Pair<T> v2 = O::lds2(col_at(sm, s, c, i, j + 1) + zo), v3 = O::lds2(col_at(sm, s, c, i + 1, j + 1) + zo);
    const Pair<T> sx0 = O::add(v0, v1), dx0 = O::sub(v1, v0), sx1 = O::add(v2, v3), dx1 = O::sub(v3, v2);
    m[0][c] = O::add(sx0, sx1);
    m[1][c] = O::add(dx0, dx1);
    m[2][c] = O::sub(sx1, sx0);
    m[3][c] = O::sub(dx1, dx0);
  }
}

// One pair of cells: lower-plane modes lo, upper-plane modes hi, moduli E -> the node plane
// pair's forces in the x-y mode basis, F[q][c] = (carry + lower face of the first cell, upper
// face of the first + lower face of the second); carry becomes the second cell's upper face.
template <typename T>
__device__ __forceinline__ void cell_pair_sym(const KSym<T>& ks, const Pair<T> (&lo)[4][3], const Pair<T> (&hi)[4][3],
                                              Pair<T> E, T (&carry)[4][3], Pair<T> (&F)[4][3]) {
  typedef PairOps<T> O;
  typedef Pair<T> P;
  // z step: S[q][c] = lo + hi (q = 1..3; the constant mode carries no force), D[q][c] = hi - lo
  P S[4][3], D[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (q > 0) S[q][c] = O::add(lo[q][c], hi[q][c]);
      D[q][c] = O::sub(hi[q][c], lo[q][c]);
    }
  auto scaled = [&](T c) { return P{E.a * c, E.b * c}; };
  const P A = scaled(ks.c[0]), B = scaled(ks.c[1]), Dd = scaled(ks.c[2]), B2 = scaled(ks.c[3]);
  const P D2 = scaled(ks.c[4]), E2 = scaled(ks.c[5]), Tt = scaled(ks.c[6]);
  // fc[q][c]: force on mode (q, z-const) (q = 1..3); fo[q][c]: on mode (q, sz)
  P fc[4][3], fo[4][3];
  {  // linear normal: (sx,x) = S[1][0], (sy,y) = S[2][1], (sz,z) = D[0][2]
    const P bs = O::mul(B, O::add(O::add(S[1][0], S[2][1]), D[0][2]));
    fc[1][0] = O::fma(A, S[1][0], bs);
    fc[2][1] = O::fma(A, S[2][1], bs);
    fo[0][2] = O::fma(A, D[0][2], bs);
  }
  // linear shear: {(sx,y), (sy,x)}, {(sx,z), (sz,x)}, {(sy,z), (sz,y)}
  fc[1][1] = fc[2][0] = O::mul(Dd, O::add(S[1][1], S[2][0]));
  fc[1][2] = fo[0][0] = O::mul(Dd, O::add(S[1][2], D[0][0]));
  fc[2][2] = fo[0][1] = O::mul(Dd, O::add(S[2][2], D[0][1]));
  {  // bilinear normal: (sxsy,z) = S[3][2], (sxsz,y) = D[1][1], (sysz,x) = D[2][0]
    const P bs = O::mul(B2, O::add(O::add(S[3][2], D[1][1]), D[2][0]));
    fc[3][2] = O::fma(B2, S[3][2], bs);
    fo[1][1] = O::fma(B2, D[1][1], bs);
    fo[2][0] = O::fma(B2, D[2][0], bs);
  }
  // bilinear shear: {(sxsy,x), (sysz,z)}, {(sxsy,y), (sxsz,z)}, {(sxsz,x), (sysz,y)}
  fc[3][0] = O::fma(D2, S[3][0], O::mul(E2, D[2][2]));
  fo[2][2] = O::fma(D2, D[2][2], O::mul(E2, S[3][0]));
  fc[3][1] = O::fma(D2, S[3][1], O::mul(E2, D[1][2]));
  fo[1][2] = O::fma(D2, D[1][2], O::mul(E2, S[3][1]));
  fo[1][0] = O::fma(D2, D[1][0], O::mul(E2, D[2][1]));
  fo[2][1] = O::fma(D2, D[2][1], O::mul(E2, D[1][0]));
  // trilinear
#pragma unroll
  for (int c = 0; c < 3; ++c) fo[3][c] = O::mul(Tt, D[3][c]);
  // back along z: a cell's lower face is fc - fo, its upper face fc + fo (fc = 0 for q = 0)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    F[0][c] = O::sub(O::mk(carry[0][c], fo[0][c].a), fo[0][c]);
    carry[0][c] = fo[0][c].b;
#pragma unroll
    for (int q = 1; q < 4; ++q) {
      const P lw = O::sub(fc[q][c], fo[q][c]), up = O::add(fc[q][c], fo[q][c]);
      F[q][c] = O::add(O::mk(carry[q][c], up.a), lw);
      carry[q][c] = up.b;
    }
  }
}

// a node plane pair's x-y mode forces -> this thread's node column's share (own) and the share
// of the node column at y + 1 (published for that thread in red); x through shuffles
template <typename T>
__device__ __forceinline__ void plane_pair_back(const Pair<T> (&F)[4][3], Pair<T> (&own)[3], Pair<T>* red, int tid) {
  typedef PairOps<T> O;
  typedef Pair<T> P;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // corner (dx, dy) = P(dx) + sy(dy) Q(dx): P(0) = F0 - F1, P(1) = F0 + F1, Q likewise from F2, F3
    const P p0 = O::sub(F[0][c], F[1][c]), p1 = O::add(F[0][c], F[1][c]);
    const P q0 = O::sub(F[2][c], F[3][c]), q1 = O::add(F[2][c], F[3][c]);
    const P pn = O::add(p0, O::shfl_up1(p1)), qn = O::add(q0, O::shfl_up1(q1));
    own[c] = O::sub(pn, qn);
    O::sts(&red[c * TXC * TYC + tid], O::add(pn, qn));
  }
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

__device__ __forceinline__ void store4(float* p, const float (&o)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void store4(double* p, const double (&o)[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(o[2], o[3]);
}

// Persistent blocks, one barrier per chunk: each thread waits for its stages, forms its two pairs
// of cells, publishes its y shares into the exchange buffer of the chunk's parity, and the block
// meets once (which also settles a wait that gave up); the owners then add their -y neighbour's
// shares and store their four node planes. The exchange is double-buffered, so the next chunk's
// writes never meet this chunk's reads. The TMA ring runs over the block's loads of all its
// segments in order, so the next segment's first chunks load while this one finishes. MODE 0
// stores A u in out (float64: and, with dotp, the block's share of u . A u); modes 1..3 (float32)
// store a Chebyshev update instead (cheb_store; out unused).
template <typename T, int MODE>
__global__ void __launch_bounds__(TXC * TYC, (sizeof(T) == 4 ? 2 : 1))
k_apply_fine(const __grid_constant__ FineMaps maps, T* __restrict__ out, const uint8_t* __restrict__ mask,
             const KSym<T> ks, LpGrid g, int nchunks, int* __restrict__ err, const FineCheb ch,
             double* __restrict__ dotp) {
  typedef PairOps<T> O;
  typedef Pair<T> P;
  extern __shared__ unsigned char smem_raw[];
  // 128-byte alignment in the shared window (what TMA addresses), not in the generic space
  const uint32_t raw_off = lp_smem_addr(smem_raw);
  FineSmem<T>& sm = *reinterpret_cast<FineSmem<T>*>(smem_raw + ((128u - (raw_off & 127u)) & 127u));
  const int tid = threadIdx.x;
  const int i = tid % TXC, j = tid / TXC;
  const int gx = (g.NX() + TXC - 2) / (TXC - 1), gy = (g.NY() + TYC - 2) / (TYC - 1);
  const long long units = (long long)gx * gy * nchunks;
  const long long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
  const long long cs = g.comp_stride(), zcs = g.node_zc_stride();
  constexpr uint32_t UBYTES = 3 * BOX * BOX * 4 * sizeof(T);
  constexpr uint32_t EBYTES = TXC * TYC * 4 * sizeof(T);
  if (u0 >= u1) {
    if (dotp && tid == 0) dotp[blockIdx.x] = 0.0;
    return;
  }

  // alignment contract of every TMA operand and vector access, checked once per block: a
  // violation is recorded in *err (codes 10..17) and the block returns without touching memory
  __shared__ int bad;
  if (tid == 0) {
    int code = 0;
    uint32_t so = 0;
    for (int s = 0; s < NST; ++s) so |= lp_smem_addr(sm.u[s].v) | lp_smem_addr(sm.e[s].v);
    if (so & 127) code = 10;
    else if (reinterpret_cast<uintptr_t>(&maps.u) & 63) code = 11;
    else if (reinterpret_cast<uintptr_t>(&maps.e) & 63) code = 12;
    else if (MODE == 0 && (reinterpret_cast<uintptr_t>(out) & 15)) code = 13;
    else if (MODE != 0 && ((reinterpret_cast<uintptr_t>(ch.x) | reinterpret_cast<uintptr_t>(ch.r) |
                            reinterpret_cast<uintptr_t>(ch.d) | reinterpret_cast<uintptr_t>(ch.b) |
                            reinterpret_cast<uintptr_t>(ch.dinv)) & 15)) code = 14;
    else if (lp_smem_addr(&sm.full[0]) & 7) code = 15;
    else if (reinterpret_cast<uintptr_t>(mask) & 3) code = 16;
    else if (lp_smem_addr(&sm.red[0][0][0][0]) & 15) code = 17;
    bad = code;
    if (code) atomicExch(err, code);
  }
  __syncthreads();
  if (bad) {
    if (dotp && tid == 0) dotp[blockIdx.x] = 0.0;
    return;
  }
  float cs_s = 0.0f, cs_c1 = 0.0f, cs_c2 = 0.0f;
  if constexpr (MODE != 0) {
    cs_s = (float)ch.coef[1];
    cs_c1 = (float)ch.coef[2];
    cs_c2 = (float)ch.coef[3];
  }
  // the producer (thread 0) walks the block's loads: its segment, the loads issued in it and in all
  int total = 0;
  long long pu = u0;
  LpSeg ps = lp_seg(u0, u1, nchunks);
  int pk = 0, issued = 0, pst = 0;   // (pst: the stage of the next load issued)
  if (tid == 0) {
    for (long long u = u0; u < u1;) {
      const LpSeg q = lp_seg(u, u1, nchunks);
      total += q.nload;
      u += q.ce - q.cb;
    }
    for (int s = 0; s < NST; ++s) lp_mbar_init(&sm.full[s], 1);
    lp_fence_barrier_init();
  }
  __syncthreads();
  auto issue_next = [&]() {
    if (pk == ps.nload) {
      pu += ps.ce - ps.cb;
      ps = lp_seg(pu, u1, nchunks);
      pk = 0;
    }
    const int s = pst;
    pst = pst + 1 == NST ? 0 : pst + 1;
    const int x0 = (ps.tile % gx) * (TXC - 1), y0 = (ps.tile / gx) * (TYC - 1);
    lp_mbar_expect_tx(&sm.full[s], UBYTES + EBYTES);
    lp_tma_load_4d(sm.u[s].v, &maps.u, 4 * (x0 - 1), y0 - 1, ps.cstart + pk, 0, &sm.full[s]);
    lp_tma_load_3d(sm.e[s].v, &maps.e, 4 * (x0 - 1), y0 - 1, ps.cstart + pk, &sm.full[s]);
    ++pk;
    ++issued;
  };
  if (tid == 0)
    while (issued < NST - 1 && issued < total) issue_next();
  double pacc = 0.0;
  bool ok = true, failed = false;
  int n = 0;    // the block's load in hand (the chunk processed)
  int sn = 0;   // its stage, n % NST, and the parity of its phase, (n / NST) & 1, kept as they advance
  uint32_t pn = 0;
  auto advance = [](int& s, uint32_t& p) {
    if (++s == NST) {
      s = 0;
      p ^= 1u;
    }
  };
  int it = 0;   // chunks processed: the exchange buffer alternates with it
  for (long long u = u0; u < u1 && !failed;) {
    const LpSeg sg = lp_seg(u, u1, nchunks);
    u += sg.ce - sg.cb;
    const int x0 = (sg.tile % gx) * (TXC - 1), y0 = (sg.tile / gx) * (TYC - 1);
    const int nx_ = x0 - 1 + i, ny_ = y0 - 1 + j;
    const bool writer = i >= 1 && j >= 1 && nx_ < g.NX() && ny_ < g.NY();
    const long long obase = writer ? g.node(nx_, ny_, 0) : 0;   // chunk c at obase + c * zcs
    T carry[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) carry[q][c] = T(0);
    // modes of planes (0, 1) of the chunk in hand, formed by the iteration before
    P m01[4][3];
    ok = ok && lp_mbar_wait(&sm.full[sn], pn);
    plane_modes<T>(sm, sn, i, j, 0, m01);
    for (int k = 0; k < sg.nproc; ++k, ++n, ++it, advance(sn, pn)) {
      const int c = sg.cstart + k;
      const bool halo = c < sg.cb;
      const int s = sn;
      int s1 = sn;   // stage and phase of load n + 1
      uint32_t p1 = pn;
      advance(s1, p1);
      // the stages refilled here were last read before the previous chunk's barrier
      if (tid == 0)
        while (issued < n + NST && issued < total) issue_next();
      const uint32_t mb4 = (writer && !halo) ? __ldg(reinterpret_cast<const uint32_t*>(mask + obase + c * zcs)) : 0u;
      ok = ok && lp_mbar_wait(&sm.full[s], pn);
      const bool has_next = k + 1 < sg.nload;
      if (has_next) ok = ok && lp_mbar_wait(&sm.full[s1], p1);
      // a wait that gave up leaves stale but in-bounds data; the barrier below then stops the block
      const T* ecol = &sm.e[s].v[(j * TXC + i) * 4];
      P m23[4][3];
      plane_modes<T>(sm, s, i, j, 2, m23);
      P(*red)[3][TXC * TYC] = sm.red[it & 1];
      P own[2][3];
      T ucol[3][4];   // this node column's u (float64 dot), read before the barrier frees the stage
      if constexpr (MODE == 0 && sizeof(T) == 8) {
        if (dotp != nullptr && writer && !halo) {
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int t = 0; t < 4; ++t) ucol[cc][t] = col_at(sm, s, cc, i, j)[t];
        }
      }
      // cells (0, 1): planes (0, 1) and (1, 2). In a halo chunk only cell 3 matters (its upper
      // face starts the segment's carry), so the first pair is skipped there.
      if (!halo) {
        P hi[4][3], F[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) hi[q][cc] = O::mk(m01[q][cc].b, m23[q][cc].a);
        cell_pair_sym<T>(ks, m01, hi, O::lds2(ecol), carry, F);
        plane_pair_back<T>(F, own[0], &red[0][0][0], tid);
      }
      // the next chunk's planes (0, 1), kept for the next iteration
      if (has_next) {
        plane_modes<T>(sm, s1, i, j, 0, m01);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) m01[q][cc] = O::zero();
      }
      {
        // cells (2, 3): planes (2, 3) and (3, 4)
        P hi[4][3], F[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) hi[q][cc] = O::mk(m23[q][cc].b, m01[q][cc].a);
        if (halo) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) carry[q][cc] = T(0);
        }
        cell_pair_sym<T>(ks, m23, hi, O::lds2(ecol + 2), carry, F);
        if (!halo) plane_pair_back<T>(F, own[1], &red[1][0][0], tid);
      }
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(err, 1);
          // let the loads already issued land before the block exits (bounded as well)
          for (int kk = n; kk < issued; ++kk) lp_mbar_wait(&sm.full[kk % NST], (kk / NST) & 1);
        }
        failed = true;
        break;
      }
      if (halo) continue;   // uniform across the block
      if (writer) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const P a = O::add(own[0][cc], red[0][cc][tid - TXC]);
          const P b = O::add(own[1][cc], red[1][cc][tid - TXC]);
          T o[4] = {a.a, a.b, b.a, b.b};
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (!((mb4 >> (8 * t + cc)) & 1u)) o[t] = T(0);
          const long long idx = cc * cs + obase + c * zcs;
          if constexpr (MODE == 0) {
            store4(out + idx, o);
            if constexpr (sizeof(T) == 8) {
              if (dotp) {
#pragma unroll
                for (int t = 0; t < 4; ++t) pacc += o[t] * ucol[cc][t];
              }
            }
          } else if constexpr (sizeof(T) == 4) {
            cheb_store<MODE>(ch, idx, make_float4(o[0], o[1], o[2], o[3]), cs_s, cs_c1, cs_c2);
          }
        }
      }
    }
    // the segment's last load (the chunk above) was only read as the next chunk's planes
    if (!failed && sg.nload > sg.nproc) {
      ++n;
      advance(sn, pn);
    }
  }
  if (dotp) {
    __shared__ double sh[32];
    pacc = lp_block_sum(pacc, sh);
    if (tid == 0) dotp[blockIdx.x] = pacc;
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

// The seven coefficient classes of the cubic-symmetric modal matrix from lpb_modal_ke's 45
// values: {a - b, b, d, b2, d2, e2, t}. False when an entry strays from its class by more than
// 1e-9 of the largest, or the exact identities of the isotropic unit brick (the linear shear block
// has rank one, e = d; the bilinear normal block is b2 (I + 1 1^T), a2 = 2 b2) do not hold.
static bool modal_sym_classes(const double* km, double out[7]) {
  static const int rows[LP_MODAL_NNZ] = LP_MODAL_ROWS;
  static const int cols[LP_MODAL_NNZ] = LP_MODAL_COLS;
  auto in = [](int v, std::initializer_list<int> s) {
    for (int w : s)
      if (w == v) return true;
    return false;
  };
  auto pair_of = [](int v) -> int {   // the shear pairs: an id per pair, -1 when v is in none
    const int pl[3][2] = {{4, 6}, {5, 12}, {8, 13}}, pb[3][2] = {{9, 20}, {10, 17}, {15, 19}};
    for (int p = 0; p < 3; ++p) {
      if (v == pl[p][0] || v == pl[p][1]) return p;
      if (v == pb[p][0] || v == pb[p][1]) return 3 + p;
    }
    return -1;
  };
  // classes: 0 a, 1 b, 2 d, 3 e, 4 a2, 5 b2, 6 d2, 7 e2, 8 t
  double sum[9] = {}, lo[9], hi[9];
  int cnt[9] = {};
  for (int k = 0; k < 9; ++k) {
    lo[k] = 1e300;
    hi[k] = -1e300;
  }
  double amax = 0.0;
  for (int n = 0; n < LP_MODAL_NNZ; ++n) {
    const int r = rows[n], c = cols[n];
    int cl = -1;
    if (in(r, {3, 7, 14}) && in(c, {3, 7, 14})) cl = r == c ? 0 : 1;
    else if (in(r, {11, 16, 18}) && in(c, {11, 16, 18})) cl = r == c ? 4 : 5;
    else if (r >= 21 && r == c) cl = 8;
    else if (pair_of(r) >= 0 && pair_of(r) == pair_of(c)) cl = (pair_of(r) < 3 ? 2 : 6) + (r == c ? 0 : 1);
    if (cl < 0) return false;
    sum[cl] += km[n];
    cnt[cl] += 1;
    lo[cl] = fmin(lo[cl], km[n]);
    hi[cl] = fmax(hi[cl], km[n]);
    amax = fmax(amax, fabs(km[n]));
  }
  double m[9];
  for (int k = 0; k < 9; ++k) {
    if (!cnt[k] || hi[k] - lo[k] > 1e-9 * amax) return false;
    m[k] = sum[k] / cnt[k];
  }
  if (fabs(m[3] - m[2]) > 1e-9 * amax || fabs(m[4] - 2.0 * m[5]) > 1e-9 * amax) return false;
  out[0] = m[0] - m[1];
  out[1] = m[1];
  out[2] = m[2];
  out[3] = m[5];
  out[4] = m[6];
  out[5] = m[7];
  out[6] = m[8];
  return true;
}

template <typename T>
static int launch_fine(T* out, const T* u, const T* e, const uint8_t* mask, const double* kmodal_host, int* err,
                       LpGrid g, cudaStream_t st, double* part = nullptr, long long part_len = 0,
                       double* dot_out = nullptr, int mode = 0, const FineCheb* ch = nullptr) {
  if (!fine_args_ok(g) || !out || !u || !e || !mask || !kmodal_host || !err || out == u) return LP_ERR_ARG;
  if (mode != 0 && (sizeof(T) != 4 || !ch || mode < 0 || mode > 3)) return LP_ERR_ARG;
  double cls[7];
  if (!modal_sym_classes(kmodal_host, cls)) return LP_ERR_ARG;
  KSym<T> ks;
  for (int n = 0; n < 7; ++n) ks.c[n] = (T)cls[n];
  const uint32_t zc = 4;
  FineMaps maps;
  const uint64_t nd[4] = {zc * (uint64_t)g.NX(), (uint64_t)g.NY(), (uint64_t)g.pz / zc, 3};
  const uint64_t cd[3] = {zc * (uint64_t)g.nx, (uint64_t)g.ny, (uint64_t)g.cpz / zc};
  const uint32_t bin[4] = {zc * BOX, BOX, 1, 3};
  const uint32_t be[3] = {zc * TXC, TYC, 1};
  if (!lp_make_map(&maps.u, u, 4, nd, bin, sizeof(T)) || !lp_make_map(&maps.e, e, 3, cd, be, sizeof(T)))
    return LP_ERR_ARG;
  const int smem = (int)sizeof(FineSmem<T>) + 128;
  const void* kfn;
  if constexpr (sizeof(T) == 4) {
    kfn = mode == 1   ? (const void*)k_apply_fine<float, 1>
          : mode == 2 ? (const void*)k_apply_fine<float, 2>
          : mode == 3 ? (const void*)k_apply_fine<float, 3>
                      : (const void*)k_apply_fine<float, 0>;
  } else {
    kfn = (const void*)k_apply_fine<double, 0>;
  }
  const long long slots = resident_blocks(kfn, smem);
  if (!slots) return LP_ERR_LAUNCH;
  const int gx = (g.NX() + TXC - 2) / (TXC - 1), gy = (g.NY() + TYC - 2) / (TYC - 1);
  const int nchunks = g.pz / (int)zc;
  // persistent blocks: all resident blocks (or the tuned number per SM), each with an equal share
  // of the (tile, chunk) units
  long long nb = slots;
  const int tuned = lp_tune_lookup(sizeof(T) == 4 ? LP_KNOB_FINE_F32 : LP_KNOB_FINE_F64, g.nx, g.ny, g.nz);
  if (tuned >= 1) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((long long)tuned * nsm < nb) nb = (long long)tuned * nsm;
  }
  const long long units = (long long)gx * gy * nchunks;
  if (nb > units) nb = units;
  const FineCheb none{};
  const FineCheb& c = ch ? *ch : none;
  double* dp = nullptr;
  if (part) {
    if (nb > part_len) return LP_ERR_SIZE;
    dp = part;
  }
  const dim3 grid((unsigned)nb);
  if constexpr (sizeof(T) == 4) {
    if (mode == 1)
      k_apply_fine<float, 1><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, ks, g, nchunks, err, c, nullptr);
    else if (mode == 2)
      k_apply_fine<float, 2><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, ks, g, nchunks, err, c, nullptr);
    else if (mode == 3)
      k_apply_fine<float, 3><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, ks, g, nchunks, err, c, nullptr);
    else
      k_apply_fine<float, 0><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, ks, g, nchunks, err, c, nullptr);
  } else {
    k_apply_fine<double, 0><<<grid, TXC * TYC, smem, st>>>(maps, out, mask, ks, g, nchunks, err, c, dp);
  }
  if (dp) k_fine_dot_final<<<1, 1024, 0, st>>>(dp, nb, dot_out);
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

// lpb_modal_ke's 45 coefficients -> the seven classes the fine kernel's product uses
// {a - b, b, d, b2, d2, e2, t}; 7, or -1 when the coefficients lack the unit brick's symmetry
int lpb_modal_sym(const double* kmodal, double* classes_out) {
  if (!kmodal || !classes_out) return LP_ERR_ARG;
  return modal_sym_classes(kmodal, classes_out) ? 7 : -1;
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
