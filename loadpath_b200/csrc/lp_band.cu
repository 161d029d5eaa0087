// The coarsest level's direct solve (loadpath/mg.py:708-766: the reference factors D K D + (I - D)
// with SuperLU on the host, in symmetric mode without pivoting). Here the operator is a band (a
// 27-point block stencil whose nodes are numbered longest axis slowest, half-bandwidth
// 3 (N1 N2 + N2 + 1) + 2 dofs), so:
//   1. k_band_factor: signed Cholesky A = L S L^T (S = diag(+-1): a symmetric LU without pivoting,
//      failing only on an exactly zero pivot, as SuperLU does) of the band stored as 32 x 32
//      tiles (tile (R, d) = rows 32R.., columns 32(R - d)..), left-looking by tile rows as a
//      dataflow: helper blocks form each row's tiles up to three left of the diagonal and the
//      partial sums of the rest; one critical block finishes the rows in order, keeping the last
//      two rows on-chip. A diagonal tile is factored, and its factor inverted, by one warp in
//      registers; products run on the FP64 tensor cores.
//   2. k_band_inverse: A^-1 = L^-T S L^-1 applied to the identity, 32 columns per block: a
//      forward then a backward block substitution over the band tiles. Only the lower triangle
//      is needed (rows >= the block's first column); k_sym_lower copies it across.
//   3. per V-cycle: gather the level's field into the band numbering, one GEMV with the dense
//      inverse, scatter back (the inverse stays resident; a GEMV has no sequential chain).
// The factorisation costs O(n bw^2) instead of the dense O(n^3): at the 17 x 9 x 9-node coarsest
// level of a 256 x 128 x 128 grid, n = 4131 and bw = 275.
#include "lp_common.cuh"
#include "lp_tma.cuh"

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

// FP64 tensor-core MMA, m8n8k4 (row-major A 8 x 4, column-major B 4 x 8, C/D 8 x 8). Lane l holds
// A[l >> 2][l & 3], B[l & 3][l >> 2] and D[l >> 2][2 (l & 3) + i], i = 0, 1.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ---- 32 x 32 tiles in registers and shared memory ----
// NW warps (of a group starting at some warp) hold a tile 32 / NW entries per thread in the
// accumulator layout of the MMA: the sixteen 8 x 8 blocks are dealt out NB = 16 / NW per warp,
// block b = w NB + k of warp w in the group (row block b / 4, column block b % 4), and lane l
// (g = l / 4, q = l % 4) holds entries (8 (b / 4) + g, 8 (b % 4) + 2 q + i), i = 0, 1.
constexpr int FLD = 36;   // shared row stride: each MMA operand load spreads over all banks
typedef double FTile[32][FLD];

template <int NB>
__device__ __forceinline__ void frag_at(int w, int k, int& r, int& c) {
  const int b = w * NB + k, l = threadIdx.x & 31;
  r = 8 * (b >> 2) + (l >> 2);
  c = 8 * (b & 3) + 2 * (l & 3);
}
template <int NB>
__device__ __forceinline__ void frag_load(double (&v)[2 * NB], const double* __restrict__ t, int w) {
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    int r, c;
    frag_at<NB>(w, k, r, c);
    const double2 a = __ldcg(reinterpret_cast<const double2*>(t + r * 32 + c));
    v[2 * k] = a.x;
    v[2 * k + 1] = a.y;
  }
}
template <int NB>
__device__ __forceinline__ void frag_store(double* __restrict__ t, const double (&v)[2 * NB], int w) {
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    int r, c;
    frag_at<NB>(w, k, r, c);
    *reinterpret_cast<double2*>(t + r * 32 + c) = make_double2(v[2 * k], v[2 * k + 1]);
  }
}
// the tile into shared memory (row stride LD)
template <int NB, int LD>
__device__ __forceinline__ void frag_to_smem(double (&d)[32][LD], const double (&v)[2 * NB], int w) {
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    int r, c;
    frag_at<NB>(w, k, r, c);
    d[r][c] = v[2 * k];
    d[r][c + 1] = v[2 * k + 1];
  }
}
template <int NB, int LD>
__device__ __forceinline__ void smem_to_frag(double (&v)[2 * NB], const double (&d)[32][LD], int w) {
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    int r, c;
    frag_at<NB>(w, k, r, c);
    v[2 * k] = d[r][c];
    v[2 * k + 1] = d[r][c + 1];
  }
}
// p += A B^T over this thread's entries (A, B staged; FP64 tensor-core MMAs)
template <int NB>
__device__ __forceinline__ void mma_acc(double (&p)[2 * NB], const FTile& a, const FTile& b, int w) {
  const int l = threadIdx.x & 31, g = l >> 2, q = l & 3;
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    const int blk = w * NB + k, ar = 8 * (blk >> 2) + g, br = 8 * (blk & 3) + g;
#pragma unroll
    for (int kc = 0; kc < 32; kc += 4) dmma(p[2 * k], p[2 * k + 1], a[ar][kc + q], b[br][kc + q]);
  }
}
// p += A (B S)^T: B's column k times s[k] as it is read (s: 32 signs, shared)
template <int NB>
__device__ __forceinline__ void mma_acc_s(double (&p)[2 * NB], const FTile& a, const FTile& b, const double* s, int w) {
  const int l = threadIdx.x & 31, g = l >> 2, q = l & 3;
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    const int blk = w * NB + k, ar = 8 * (blk >> 2) + g, br = 8 * (blk & 3) + g;
#pragma unroll
    for (int kc = 0; kc < 32; kc += 4) dmma(p[2 * k], p[2 * k + 1], a[ar][kc + q], b[br][kc + q] * s[kc + q]);
  }
}
// 16-byte asynchronous copies global -> shared through L2: a batch of tiles is issued at once and
// waited for once
__device__ __forceinline__ void cpa16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
// a tile (row-major 32 x 32, global) into d by asynchronous copies of 256 threads (2 per thread)
__device__ __forceinline__ void stage_async(FTile& d, const double* __restrict__ g) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = threadIdx.x + 256 * h, r = e >> 4, c = 2 * (e & 15);
    cpa16(&d[r][c], g + r * 32 + c);
  }
}
// 32 doubles (global) into d by asynchronous copies of threads 0..15
__device__ __forceinline__ void stage_vec_async(double* d, const double* __restrict__ g) {
  if (threadIdx.x < 16) cpa16(d + 2 * threadIdx.x, g + 2 * threadIdx.x);
}

// a tile in global memory (row-major 32 x 32) into shared memory by nthr threads (t: this thread's
// index among them); colscale: column k times colscale[k] (global, may be NULL)
__device__ __forceinline__ void stage(FTile& d, const double* __restrict__ g, const double* __restrict__ colscale,
                                      int t, int nthr) {
  for (int e = t; e < 1024; e += nthr) {
    const int r = e >> 5, c = e & 31;
    double v = __ldcg(g + e);
    if (colscale) v *= __ldcg(colscale + c);
    d[r][c] = v;
  }
}

// Signed Cholesky A = L S L^T (S = diag(+-1)) of one 32 x 32 diagonal tile by the calling warp:
// lane i holds row i of the tile (from `in`, shared, lower part). Each pivot p gives
// L_jj = sqrt|p| and S_j = sign(p), so negative pivots are factored as they are: a symmetric LU
// without pivoting, as the reference's SuperLU in symmetric mode (loadpath/mg.py:744-747). A
// pivot's column goes to every lane through shared memory (col: two 32-double buffers, one read
// per pair of entries instead of a shuffle per entry), and the next pivot is broadcast from its
// own lane's update, so the chain per pivot is one shuffle, one reciprocal square root and three
// multiplies. Writes L (upper part zero) to dl, 1 / L_jj to rinv and S to sgs (shared). A pivot
// that is exactly zero (or not finite) records its dof (1-based) in *info: the operator is
// singular; the arithmetic continues.
__device__ __forceinline__ void factor_diag(const double (*in)[33], double (*dl)[33], double* rinv, double* sgs, double (*col)[32],
                            long long row0, int* info) {
  const int i = threadIdx.x & 31;
  double a[32];
  int bad = 0;
#pragma unroll
  for (int k = 0; k < 32; ++k) a[k] = k <= i ? in[i][k] : 0.0;
  double p = __shfl_sync(0xffffffffu, a[0], 0);
  double dii = 0.0;   // this lane's own L_ii
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (!(fabs(p) > 0.0) && bad == 0) bad = (int)(row0 + j + 1);
    const double sj = p < 0.0 ? -1.0 : 1.0, ap = fabs(p);
    // one reciprocal square root per pivot on the chain (not a square root and a division)
    const double rd = rsqrt(ap), d = ap * rd;
    const double l = i > j ? a[j] * rd * sj : (i == j ? d : 0.0);
    const double ls = l * sj;
    a[j] = l;
    if (i == j) sgs[j] = sj;
    dii = i == j ? d : dii;
    if (j < 31) p = __shfl_sync(0xffffffffu, a[j + 1] - ls * l, j + 1);   // lane j + 1's own update
    col[j & 1][i] = l;
    __syncwarp();
    // entries above the diagonal take garbage here (zeroed below); pairs of the column per read
    if ((j + 1) & 1) a[j + 1] -= ls * col[j & 1][j + 1];
#pragma unroll
    for (int t = (j + 2) & ~1; t < 32; t += 2) {
      const double2 c2 = *reinterpret_cast<const double2*>(&col[j & 1][t]);
      a[t] -= ls * c2.x;
      a[t + 1] -= ls * c2.y;
    }
  }
  if (i == 0 && bad) atomicCAS(info, 0, bad);
  rinv[i] = 1.0 / dii;   // 1 / L_ii, off the chain
#pragma unroll
  for (int k = 0; k < 32; ++k) dl[i][k] = k <= i ? a[k] : 0.0;
}

// x = x L^-T S (the panel solve L_Rc = X L_cc^-T S_c) by forward substitution, one warp: lane r
// holds row r of x (x[k] = X[r][k]), L the diagonal factor (shared), rinv its 1 / L_kk and s the
// signs S_c (shared): every row is its own chain, with no exchange between lanes. (Substitution,
// not a product with L_cc^-1: a diagonal tile with pivots near zero has an inverse too
// inaccurate to solve with.)
template <int LD>
__device__ __forceinline__ void solve_lane(double (&x)[32], const double (*L)[LD], const double* rinv, const double* s) {
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    const double ym = x[m] * rinv[m];
    x[m] = ym;
#pragma unroll
    for (int k = m + 1; k < 32; ++k) x[k] -= ym * L[k][m];
  }
#pragma unroll
  for (int k = 0; k < 32; ++k) x[k] *= s[k];
}

__device__ __forceinline__ void group_sync(int id, int nthr) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthr) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(lp_smem_addr(bar)) : "memory");
}

// Shared memory of k_band_factor. Helper blocks stage operand pairs of up to four products and a
// diagonal factor tile; the critical block keeps its ring of the last three rows (per row r:
// L_{r,r-1} S_{r-1} and L_{r,r-2} S_{r-2}, L_rr, S_r), the hand-over tiles between its two warp
// groups by row parity, their staging tiles and the mbarriers between them.
typedef double RTile[32][33];   // row stride 33: row-wise and column-wise reads spread over the banks
constexpr int NOWN = 8;   // a helper's ring of its row's last tiles; also its staging slots
struct HelperSmem {
  FTile own[NOWN];           // L_{R,c} of the helper's row, slot (c - c0) % NOWN
  FTile bst[NOWN];           // staged operands
  FTile dstage;              // L_cc for a panel solve
  RTile xbuf;                // the tile being solved
  alignas(16) double sgj[NOWN][32];   // the signs S_j of each staged product
  alignas(16) double rinv[32], sgn[32];
};
struct CriticalSmem {
  FTile ring[3][2];
  RTile ringd[3];
  alignas(16) double rinv[3][32], rsg[3][32];
  RTile hx1[2], hy[2];          // X_{R,R-1} (all its terms, not yet solved) and the diagonal tile
  FTile l1;                     // finisher: L_{R,R-1}
  FTile pa0, pa1, pl2;          // preparer: L_{R,R-3}, L_{R,R-4}, L_{R,R-2}
  RTile pbuf;                   // preparer: X_{R,R-2} for its solve
  alignas(16) double col[2][32];   // the finisher's pivot columns
  alignas(8) uint64_t hand[2], solved[2], fact[2];
};
union BandSmem {
  HelperSmem h;
  CriticalSmem c;
};

// the group's wait until *flag > need (its first thread polls with acquire loads, bounded); false
// when the wait gave up (err is set)
__device__ bool group_wait_flag(const unsigned* flag, unsigned need, int bar_id, bool leader, int* err, int* ok_s) {
  if (leader) {
    int ok = 1;
    unsigned v = ld_acquire(flag), it = 0;
    while (v <= need) {
      if (++it > LP_BAR_LIMIT) {
        ok = 0;
        atomicExch(err, 1);
        break;
      }
      if (it > 64) __nanosleep(32);
      v = ld_acquire(flag);
    }
    *ok_s = ok;
  }
  group_sync(bar_id, 128);
  const bool ok = *ok_s != 0;
  group_sync(bar_id, 128);
  return ok;
}

// the group's wait for the phase of an mbarrier (its first thread polls, backing off, bounded; the
// others wait at the group barrier, so no warp spins beside the ones doing the work); false when
// the wait gave up (err is set)
__device__ bool group_wait_mbar(uint64_t* bar, uint32_t parity, int bar_id, bool leader, int* err, int* ok_s) {
  if (leader) {
    int ok = 1;
    uint32_t it = 0;
    while (!lp_mbar_try_wait(bar, parity)) {
      if (++it > LP_BAR_LIMIT) {
        ok = 0;
        atomicExch(err, 1);
        break;
      }
      __nanosleep(20);
    }
    *ok_s = ok;
  }
  group_sync(bar_id, 128);
  const bool ok = *ok_s != 0;
  group_sync(bar_id, 128);
  return ok;
}

// The critical block: two groups of four warps, by row R in order.
// - The preparer (warps 4-7) waits for the helpers' partial sums of row R, adds the terms that
//   need the last two rows (j = R - 4, R - 3 to tile R - 2; j = R - 3, R - 2 to tile R - 1), solves
//   tile R - 2 against L_{R-2,R-2}, takes its term off the diagonal tile, and hands tile R - 1
//   (all but its solve) and the diagonal tile to the finisher.
// - The finisher (warps 0-3) solves tile R - 1 against L_{R-1,R-1}, takes its term off the
//   diagonal tile, factors it (warp 0), stores L_RR and S_R and publishes prog[R] = R + 1.
// The chain from row to row is the finisher's: one panel solve, one product, one diagonal factor;
// the preparer works on the next row meanwhile. The groups meet through mbarriers in shared
// memory (bounded waits): hand (row R's tiles ready), solved (L_{R,R-1} in the ring), fact
// (L_RR in the ring), one arrival per row each, indexed by row parity.
__device__ void critical_rows(double* __restrict__ t, double* __restrict__ sg, const LpBand& bd, int* info,
                              unsigned* prog, const unsigned* pdone, int* err, CriticalSmem& cs) {
  __shared__ int ok_f, ok_p;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; ++k) {
      lp_mbar_init(&cs.hand[k], 1);
      lp_mbar_init(&cs.solved[k], 1);
      lp_mbar_init(&cs.fact[k], 1);
    }
    lp_fence_barrier_init();
  }
  __syncthreads();
  if (warp < 4) {   // the finisher
    const int ft = threadIdx.x;
    // row r's L_rr and S_r to global memory by warps 1-3 (one row late, while warp 0 solves the
    // next row's tile); prog[r] = r + 1 follows from thread 32 while warp 0 factors
    auto store_row = [&](int r) {
      const int q = ft - 32, sr = r % 3;
      double* dg = tile_at(t, bd, r, 0);
      for (int e = q; e < 1024; e += 96) dg[e] = cs.ringd[sr][e >> 5][e & 31];
      if (q < 32) sg[32LL * r + q] = cs.rsg[sr][q];
    };
    auto release_row = [&](int r) {
      __threadfence();
      st_release(prog + r, (unsigned)(r + 1));
    };
    for (int R = 0; R < bd.nt; ++R) {
      const int c0 = R - bd.D > 0 ? R - bd.D : 0;
      const bool h1 = R - 1 >= c0;
      const int s0 = R % 3, s1 = (R + 2) % 3;
      if (!group_wait_mbar(&cs.hand[R & 1], (R >> 1) & 1, 1, ft == 0, err, &ok_f)) return;
      if (warp == 0) {
        if (h1) {   // L_{R,R-1} = X L_{R-1,R-1}^-T S_{R-1}, lane = row
          double x[32];
#pragma unroll
          for (int k = 0; k < 32; ++k) x[k] = cs.hx1[R & 1][lane][k];
          solve_lane(x, cs.ringd[s1], cs.rinv[s1], cs.rsg[s1]);
          double* tg = tile_at(t, bd, R, 1) + lane * 32;
#pragma unroll
          for (int k = 0; k < 32; k += 2) {
            cs.l1[lane][k] = x[k];
            cs.l1[lane][k + 1] = x[k + 1];
            cs.ring[s0][0][lane][k] = x[k] * cs.rsg[s1][k];
            cs.ring[s0][0][lane][k + 1] = x[k + 1] * cs.rsg[s1][k + 1];
            *reinterpret_cast<double2*>(tg + k) = make_double2(x[k], x[k + 1]);
          }
        }
      } else if (R >= 1) {
        store_row(R - 1);
      }
      group_sync(1, 128);
      if (ft == 0) mbar_arrive(&cs.solved[R & 1]);   // (every row, which keeps the phases in step)
      if (h1) {
        double y[8], p[8] = {};
        smem_to_frag<4, 33>(y, cs.hy[R & 1], warp);
        mma_acc<4>(p, cs.l1, cs.ring[s0][0], warp);
#pragma unroll
        for (int k = 0; k < 8; ++k) y[k] -= p[k];
        frag_to_smem<4, 33>(cs.hy[R & 1], y, warp);
        group_sync(1, 128);
      }
      if (warp == 0) factor_diag(cs.hy[R & 1], cs.ringd[s0], cs.rinv[s0], cs.rsg[s0], cs.col, 32LL * R, info);
      else if (ft == 32 && R >= 1) release_row(R - 1);   // its stores are ordered by the barriers above
      group_sync(1, 128);
      if (ft == 0) mbar_arrive(&cs.fact[R & 1]);
    }
    if (warp > 0) store_row(bd.nt - 1);
    group_sync(1, 128);
    if (ft == 32) release_row(bd.nt - 1);
    return;
  }
  // the preparer
  const int pt = threadIdx.x - 128, pw = warp - 4;
  for (int R = 0; R < bd.nt; ++R) {
    const int c0 = R - bd.D > 0 ? R - bd.D : 0;
    const bool h1 = R - 1 >= c0, h2 = R - 2 >= c0, h3 = R - 3 >= c0, h4 = R - 4 >= c0;
    const int s0 = R % 3, s1 = (R + 2) % 3, s2 = (R + 1) % 3;   // ring slots of rows R, R - 1, R - 2
    if (h3 && !group_wait_flag(pdone + R, 0u, 2, pt == 0, err, &ok_p)) return;   // the helper's sums
    // L_{R-2,R-2} is in the ring, and the finisher is done with row R - 2's hand-over tiles
    if (R >= 2 && !group_wait_mbar(&cs.fact[R & 1], ((R - 2) >> 1) & 1, 2, pt == 0, err, &ok_p)) return;
    double y[8], x1[8] = {}, x2[8] = {};
    frag_load<4>(y, tile_at(t, bd, R, 0), pw);
    if (h1) frag_load<4>(x1, tile_at(t, bd, R, 1), pw);
    if (h2) frag_load<4>(x2, tile_at(t, bd, R, 2), pw);
    if (h3) stage(cs.pa0, tile_at(t, bd, R, 3), nullptr, pt, 128);   // L_{R,R-3}
    if (h4) stage(cs.pa1, tile_at(t, bd, R, 4), nullptr, pt, 128);   // L_{R,R-4}
    group_sync(2, 128);
    if (h2) {   // L_{R,R-2}: X -= L_{R,R-4} S L_{R-2,R-4}^T + L_{R,R-3} S L_{R-2,R-3}^T, then the solve
      double p[8] = {};
      if (h4) mma_acc<4>(p, cs.pa1, cs.ring[s2][1], pw);
      if (h3) mma_acc<4>(p, cs.pa0, cs.ring[s2][0], pw);
#pragma unroll
      for (int k = 0; k < 8; ++k) x2[k] -= p[k];
      frag_to_smem<4, 33>(cs.pbuf, x2, pw);
      group_sync(2, 128);
      if (pw == 0) {
        double x[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) x[k] = cs.pbuf[lane][k];
        solve_lane(x, cs.ringd[s2], cs.rinv[s2], cs.rsg[s2]);
        double* tg = tile_at(t, bd, R, 2) + lane * 32;
#pragma unroll
        for (int k = 0; k < 32; k += 2) {
          cs.pl2[lane][k] = x[k];
          cs.pl2[lane][k + 1] = x[k + 1];
          cs.ring[s0][1][lane][k] = x[k] * cs.rsg[s2][k];
          cs.ring[s0][1][lane][k + 1] = x[k + 1] * cs.rsg[s2][k + 1];
          *reinterpret_cast<double2*>(tg + k) = make_double2(x[k], x[k + 1]);
        }
      }
      group_sync(2, 128);
      double qq[8] = {};
      mma_acc<4>(qq, cs.pl2, cs.ring[s0][1], pw);
#pragma unroll
      for (int k = 0; k < 8; ++k) y[k] -= qq[k];
    }
    if (h1) {   // X_{R,R-1} -= L_{R,R-3} S L_{R-1,R-3}^T + L_{R,R-2} S L_{R-1,R-2}^T
      double p[8] = {};
      if (h3) mma_acc<4>(p, cs.pa0, cs.ring[s1][1], pw);
      if (h2) {   // L_{R-1,R-2} S is in the ring once the finisher has solved row R - 1
        if (!group_wait_mbar(&cs.solved[(R - 1) & 1], ((R - 1) >> 1) & 1, 2, pt == 0, err, &ok_p)) return;
        mma_acc<4>(p, cs.pl2, cs.ring[s1][0], pw);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) x1[k] -= p[k];
      frag_to_smem<4, 33>(cs.hx1[R & 1], x1, pw);
    }
    frag_to_smem<4, 33>(cs.hy[R & 1], y, pw);
    __threadfence();   // this group's global stores (tile R - 2) before the finisher publishes
    group_sync(2, 128);
    if (pt == 0) mbar_arrive(&cs.hand[R & 1]);
  }
}

// Left-looking band factorisation by tile rows, as a dataflow between a critical block and helper
// blocks, with L_Rc = (A_Rc - sum_j L_Rj S_j L_cj^T) L_cc^-T S_c (c = R - D .. R - 1, j from
// R - D) and L_RR S_RR L_RR^T = A_RR - sum_j L_Rj S_j L_Rj^T:
// - helper blocks (1 .. gridDim.x - 1) own tile rows R (cyclically) and form the row's tiles
//   c <= R - 3, publishing prog[R] = c + 1 after each; with them they sum the diagonal tile's
//   terms j <= R - 3, tile R - 1's j <= R - 4 and tile R - 2's j <= R - 5 (terms between helper
//   tiles only), store the partial sums in place and set pdone[R];
// - the critical block (0) finishes the rows in order (critical_rows): the remaining terms
//   (which need the last two rows, kept in its shared memory), the panel solves of tiles R - 2
//   and R - 1, and the diagonal factor, then prog[R] = R + 1.
// A helper's row needs the critical block's rows up to R - 3, so the helpers run ahead of it.
// Products run on the FP64 tensor cores with their operands staged in shared memory. Every block
// must be resident (a cooperative launch); a wait that gives up sets err and its block returns.
__global__ void __launch_bounds__(256, 1) k_band_factor(double* __restrict__ t, double* __restrict__ sg, LpBand bd,
                                                        int* __restrict__ info, unsigned* __restrict__ prog,
                                                        unsigned* __restrict__ pdone, int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char band_smem_raw[];
  BandSmem& smu = *reinterpret_cast<BandSmem*>(band_smem_raw);
  if (blockIdx.x == 0) {
    critical_rows(t, sg, bd, info, prog, pdone, err, smu.c);
    return;
  }
  HelperSmem& sm = smu.h;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nh = gridDim.x - 1;
  for (int R = blockIdx.x - 1; R < bd.nt; R += nh) {
    const int c0 = R - bd.D > 0 ? R - bd.D : 0;
    if (c0 > R - 3) continue;   // the critical block does the whole row
    double y[4], x1[4], x2[4];
    frag_load<2>(y, tile_at(t, bd, R, 0), w);
    frag_load<2>(x1, tile_at(t, bd, R, 1), w);
    frag_load<2>(x2, tile_at(t, bd, R, 2), w);
    unsigned seen1 = 0, seen2 = 0;
    for (int c = c0; c <= R - 3; ++c) {
      double x[4], p[4] = {};
      frag_load<2>(x, tile_at(t, bd, R, R - c), w);
      unsigned seen = 0;
      // the terms j < c in batches of at most NOWN staged tiles: B = L_cj (and A = L_Rj when it
      // has left the ring of the row's own tiles)
      for (int j = c0; j < c;) {
        const int jb = j;
        int ns = 0;
        while (j < c) {
          const int need = c - j <= NOWN ? 1 : 2;
          if (ns + need > NOWN) break;
          ns += need;
          ++j;
        }
        if (!wait_row(prog, c, (unsigned)(j - 1), seen, err)) return;   // row c has its columns < j
        for (int jj = jb, sl = 0; jj < j; ++jj) {
          stage_async(sm.bst[sl], tile_at(t, bd, c, c - jj));
          stage_vec_async(sm.sgj[sl], sg + 32LL * jj);
          sl += 1;
          if (c - jj > NOWN) {
            stage_async(sm.bst[sl], tile_at(t, bd, R, R - jj));
            sl += 1;
          }
        }
        cpa_wait();
        __syncthreads();
        for (int jj = jb, sl = 0; jj < j; ++jj) {
          const bool in_ring = c - jj <= NOWN;
          const FTile& a = in_ring ? sm.own[(jj - c0) % NOWN] : sm.bst[sl + 1];
          mma_acc_s<2>(p, a, sm.bst[sl], sm.sgj[sl], w);
          sl += in_ring ? 1 : 2;
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) x[i] -= p[i];
      if (!wait_row(prog, c, (unsigned)c, seen, err)) return;   // row c's diagonal factor
      // the panel solve against L_cc by warp 0 (lane = row), through xbuf, into the own ring
      frag_to_smem<2, 33>(sm.xbuf, x, w);
      stage_async(sm.dstage, tile_at(t, bd, c, 0));
      stage_vec_async(sm.sgn, sg + 32LL * c);
      cpa_wait();
      __syncthreads();
      FTile& lo = sm.own[(c - c0) % NOWN];
      if (w == 0) {
        sm.rinv[lane] = 1.0 / sm.dstage[lane][lane];
        __syncwarp();
        double xr[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) xr[k] = sm.xbuf[lane][k];
        solve_lane(xr, sm.dstage, sm.rinv, sm.sgn);
        double* tg = tile_at(t, bd, R, R - c) + lane * 32;
#pragma unroll
        for (int k = 0; k < 32; k += 2) {
          lo[lane][k] = xr[k];
          lo[lane][k + 1] = xr[k + 1];
          *reinterpret_cast<double2*>(tg + k) = make_double2(xr[k], xr[k + 1]);
        }
      }
      publish_row(prog, R, (unsigned)(c + 1));   // (its barrier also makes the own tile visible)
      // the row's partial sums over j = c: A = L_Rc, B = L_Rc, L_{R-1,c}, L_{R-2,c}, all times S_c
      const bool t1 = c <= R - 4, t2 = c <= R - 5;
      if (t1 && !wait_row(prog, R - 1, (unsigned)c, seen1, err)) return;
      if (t2 && !wait_row(prog, R - 2, (unsigned)c, seen2, err)) return;
      if (t1) stage_async(sm.bst[0], tile_at(t, bd, R - 1, R - 1 - c));
      if (t2) stage_async(sm.bst[1], tile_at(t, bd, R - 2, R - 2 - c));
      cpa_wait();
      __syncthreads();
      double q0[4] = {}, q1[4] = {}, q2[4] = {};
      mma_acc_s<2>(q0, lo, lo, sm.sgn, w);
      if (t1) mma_acc_s<2>(q1, lo, sm.bst[0], sm.sgn, w);
      if (t2) mma_acc_s<2>(q2, lo, sm.bst[1], sm.sgn, w);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        y[i] -= q0[i];
        x1[i] -= q1[i];
        x2[i] -= q2[i];
      }
      __syncthreads();
    }
    frag_store<2>(tile_at(t, bd, R, 0), y, w);
    frag_store<2>(tile_at(t, bd, R, 1), x1, w);
    frag_store<2>(tile_at(t, bd, R, 2), x2, w);
    publish_row(pdone, R, 1u);
  }
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

// k_band_inverse for CB columns per block (4 CB / 8 warps, one 8 x 8 block of each step's 32 x CB
// result per warp), with the block's last D + 1 result blocks kept in shared memory (a ring; a
// step reads D of them) and each step's band tiles, L_kk^-1 and (backward) Y_k loaded by
// asynchronous copies while the step before finishes, so a step waits on no load of its own. A
// block's chain is its column's 2 (nt - kb) steps, each bound by the SM's FP64 tensor rate, so
// narrow column blocks (CB = 16) shorten the longest chain (column 0's). The same products in the
// same order as k_band_inverse, so the same bits. Bands of at most INV_RING_D tile diagonals.
constexpr int INV_RING_D = 9;
constexpr int INV_RING_CB = 16;

template <int CB>
struct InvRing {
  static constexpr int LDR = CB + 4;             // result block row stride
  static constexpr int RB = 32 * LDR;            // doubles per result block
  static constexpr int NW = 4 * CB / 8;          // warps
  static size_t smem(int D) {
    return ((size_t)(D + 1) * RB + (size_t)D * INV_TILE + 2 * (size_t)INV_TILE + 3 * (size_t)RB) * sizeof(double);
  }
};

template <int CB>
__global__ void __launch_bounds__(32 * InvRing<CB>::NW, 1)
k_band_inverse_ring(double* __restrict__ ainv, const double* __restrict__ t, const double* __restrict__ linv,
                    const double* __restrict__ sg, LpBand bd) {
  typedef InvRing<CB> IR;
  extern __shared__ __align__(16) double sm_inv[];
  const int D = bd.D, RS = D + 1, R1 = D + 1;
  double* ring = sm_inv;                   // result block k in slot k % RS
  double* tiles = ring + RS * IR::RB;      // the step's band tiles, d = 1 .. D
  double* diag = tiles + D * INV_TILE;     // L_kk^-1, by step parity
  double* ykb = diag + 2 * INV_TILE;       // Y_k of a backward step, by step parity
  double* tmp = ykb + 2 * IR::RB;          // S
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int row0 = 8 * (w / (CB / 8)), col0 = 8 * (w % (CB / 8));
  const int orow = row0 + g, ocol = col0 + 2 * q;   // this lane's two outputs: (orow, ocol + i)
  const long long np = 32LL * bd.nt;
  const int j0 = CB * blockIdx.x;
  const int kb = j0 >> 5;
  const int nfwd = bd.nt - kb, total = 2 * nfwd;
  const int nthr = 32 * IR::NW;
  // step s: forward k = kb + s (s < nfwd), backward k = nt - 1 - (s - nfwd)
  auto step_k = [&](int s) { return s < nfwd ? kb + s : bd.nt - 1 - (s - nfwd); };
  auto step_dm = [&](int s, int k) { return s < nfwd ? min(D, k - kb) : min(D, bd.nt - 1 - k); };
  // Y_k of a backward step is still in the ring when no later forward step reused its slot
  auto y_in_ring = [&](int k) { return k >= bd.nt - RS; };
  auto issue = [&](int s) {
    const bool fwd = s < nfwd;
    const int k = step_k(s), dm = step_dm(s, k);
    for (int e = threadIdx.x; e < dm * 512; e += nthr) {
      const int d = 1 + (e >> 9), rr = (e >> 4) & 31, cc = 2 * (e & 15);
      const long long tk = fwd ? k : k + d;   // band tile (tk, d)
      cp_async16(tiles + (d - 1) * INV_TILE + rr * INV_LD + cc, t + (tk * R1 + d) * 1024 + rr * 32 + cc);
    }
    for (int e = threadIdx.x; e < 512; e += nthr)
      cp_async16(diag + (s & 1) * INV_TILE + (e >> 4) * INV_LD + 2 * (e & 15), linv + (long long)k * 1024 + 2 * e);
    if (!fwd && !y_in_ring(k))
      for (int e = threadIdx.x; e < 16 * CB; e += nthr) {
        const int rr = e / (CB / 2), cc = 2 * (e % (CB / 2));
        cp_async16(ykb + (s & 1) * IR::RB + rr * IR::LDR + cc, ainv + (32LL * k + rr) * np + j0 + cc);
      }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  issue(0);
  for (int s = 0; s < total; ++s) {
    const bool fwd = s < nfwd;
    const int k = step_k(s), dm = step_dm(s, k);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    double p0 = 0.0, p1 = 0.0, r0 = 0.0, r1 = 0.0;
    for (int d = 1; d <= dm; ++d) {
      const double* tc = tiles + (d - 1) * INV_TILE;
      const int bk = fwd ? k - d : k + d;   // the earlier result block
      const double* yb = ring + (bk % RS) * IR::RB + q * IR::LDR + col0 + g;
      if (fwd) {
        const double* ta = tc + (row0 + g) * INV_LD + q;
#pragma unroll
        for (int m = 0; m < 32; m += 8) {
          dmma(p0, p1, ta[m], yb[m * IR::LDR]);
          dmma(r0, r1, ta[m + 4], yb[(m + 4) * IR::LDR]);
        }
      } else {
        const double* ta = tc + q * INV_LD + row0 + g;   // A[row][m] = T[m][row]
#pragma unroll
        for (int m = 0; m < 32; m += 8) {
          dmma(p0, p1, ta[m * INV_LD], yb[m * IR::LDR]);
          dmma(r0, r1, ta[(m + 4) * INV_LD], yb[(m + 4) * IR::LDR]);
        }
      }
    }
    __syncthreads();   // the band tiles are read: the next step's loads may land
    if (s + 1 < total) issue(s + 1);
    const double* dg = diag + (s & 1) * INV_TILE;
    double* out = ainv + (32LL * k + orow) * np + j0 + ocol;
    double* rs = ring + (k % RS) * IR::RB + orow * IR::LDR + ocol;
    if (fwd) {
      const long long gr = 32LL * k + orow;
      tmp[orow * IR::LDR + ocol] = (gr == j0 + ocol ? 1.0 : 0.0) - (p0 + r0);
      tmp[orow * IR::LDR + ocol + 1] = (gr == j0 + ocol + 1 ? 1.0 : 0.0) - (p1 + r1);
    } else {
      const double* yk = y_in_ring(k) ? rs : ykb + (s & 1) * IR::RB + orow * IR::LDR + ocol;
      const double sr = __ldg(sg + 32LL * k + orow);
      tmp[orow * IR::LDR + ocol] = sr * yk[0] - (p0 + r0);
      tmp[orow * IR::LDR + ocol + 1] = sr * yk[1] - (p1 + r1);
    }
    __syncthreads();
    double y0 = 0.0, y1 = 0.0;
    if (fwd) {
#pragma unroll
      for (int m = 0; m < 32; m += 4)
        dmma(y0, y1, dg[(row0 + g) * INV_LD + m + q], tmp[(m + q) * IR::LDR + col0 + g]);
    } else {
#pragma unroll
      for (int m = 0; m < 32; m += 4)   // A = L_kk^-T
        dmma(y0, y1, dg[(m + q) * INV_LD + row0 + g], tmp[(m + q) * IR::LDR + col0 + g]);
    }
    rs[0] = y0;
    rs[1] = y1;
    *reinterpret_cast<double2*>(out) = make_double2(y0, y1);
    __syncthreads();
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

// linv + 1024 R = the inverse of diagonal factor tile R (for k_band_inverse), one warp per tile:
// lane c forms column c, right-looking (the 32 row updates of a step are independent)
__global__ void k_diag_inverses(double* __restrict__ linv, const double* __restrict__ t, LpBand bd) {
  __shared__ double sm[32][33];
  const int R = blockIdx.x;
  const double* d = tile_at(const_cast<double*>(t), bd, R, 0);
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) sm[e >> 5][e & 31] = d[e];
  __syncwarp();
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
  for (int r = 0; r < 32; ++r) linv[(long long)R * 1024 + r * 32 + c] = x[r];
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
// 2 max(64, nt) device words of scratch (the rows' progress counts); err: one device int, set
// when a wait gave up. One cooperative launch (a critical block that finishes the rows in order
// and helper blocks that own tile rows), then one warp per diagonal tile for linv.
int lpb_band_factor(double* t, double* linv, double* sgn, int* info, unsigned* bar, int* err, LP_GRID_ARGS,
                    void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !t || !linv || !sgn || !info || !bar || !err) return LP_ERR_ARG;
  LpBand bd = lp_band(g.NX(), g.NY(), g.NZ());
  int dev = 0, nsm = 0, per_sm = 0, coop = 0;
  const int smem = (int)sizeof(BandSmem);
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_band_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return LP_ERR_SIZE;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_band_factor, 256, smem);
  // a helper holds its row while the critical block goes through about D rows; twice that many
  // helpers leave each one a row of slack
  long long nblocks = 1 + 2LL * (bd.D + 1);
  if (nblocks > 1 + (long long)bd.nt) nblocks = 1 + bd.nt;
  const long long cap = (long long)per_sm * nsm;
  if (nblocks > cap) nblocks = cap;
  if (!coop || nblocks < 2) return LP_ERR_SIZE;
  const long long words = bd.nt > 64 ? bd.nt : 64;
  unsigned* pdone = bar + words;
  if (cudaMemsetAsync(bar, 0, 2 * words * sizeof(unsigned), LP_ST) != cudaSuccess) return LP_ERR_LAUNCH;
  if (cudaMemsetAsync(info, 0, sizeof(int), LP_ST) != cudaSuccess) return LP_ERR_LAUNCH;
  void* args[] = {&t, &sgn, &bd, &info, &bar, &pdone, &err};
  if (cudaLaunchCooperativeKernel((const void*)k_band_factor, dim3((unsigned)nblocks), dim3(256), args, (size_t)smem,
                                  LP_ST) != cudaSuccess)
    return LP_ERR_LAUNCH;
  k_diag_inverses<<<bd.nt, 32, 0, LP_ST>>>(linv, t, bd);
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
  if (bd.D <= INV_RING_D) {
    typedef InvRing<INV_RING_CB> IR;
    const size_t smem = IR::smem(bd.D);
    if (cudaFuncSetAttribute(k_band_inverse_ring<INV_RING_CB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return LP_ERR_SIZE;
    k_band_inverse_ring<INV_RING_CB>
        <<<(unsigned)(np / INV_RING_CB), 32 * IR::NW, smem, LP_ST>>>(ainv, t, linv, sgn, bd);
    k_sym_lower<<<dim3(bd.nt, bd.nt), 256, 0, LP_ST>>>(ainv, np);
    LP_LAUNCH_CHECK();
    return LP_OK;
  }
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
