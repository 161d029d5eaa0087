/* loadpath_b200 — C ABI of the B200 (sm_100a) voxel SIMP inner loop.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream (void *, NULL = the
 * legacy default stream) and returns an int status: 0 ok, -1 bad arguments, -2 launch error,
 * -3 size beyond a kernel's limit. Nothing allocates: callers own every buffer.
 *
 * Layouts (C order): z is cut into chunks of four planes, the chunk index slowest, so that a
 * chunk's four planes of a row of x are contiguous (node (x, y, z) of a component at
 * ((z / 4 * (ny+1) + y) * (nx+1) + x) * 4 + z % 4):
 *   node field  (3, pz/4, ny+1, nx+1, 4)  pz >= nz+1, pz % 4 == 0
 *   cell field  (cpz/4, ny, nx, 4)        cpz >= nz, cpz % 4 == 0
 *   node mask   (pz/4, ny+1, nx+1, 4) uint8: bits 0..2 solved dof per component (alive and
 *               not held), bits 3..5 alive (carries stiffness) per component
 *   z padding (node z > nz, cell z >= nz) holds zeros
 *   cell matrices (cells, 24, 24), rows/cols ordered 3*corner + component, corner k at
 *               (k & 1, k >> 1 & 1, k >> 2 & 1)
 * `LP_GRID` below stands for the five ints  nx, ny, nz, pz, cpz  of one level;
 * `LP_FC` for the ten ints of a fine level then its coarse level.
 *
 * The reference interfaces cited are loadpath's (paths relative to its project root).
 */
#ifndef LOADPATH_B200_H
#define LOADPATH_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- level operators: out = m * K (m * u) + (1 - m) * u  (finish=1), or K (m * u) (finish=0).
 * mask_in=0 skips the input mask (callers whose u is zero on masked dofs).
 * Replaces mg._Level.apply / apply_k (loadpath/mg.py:251-346) and
 * mgops.apply_masked / apply_scaled / apply_weights / apply_explicit (loadpath/mgops.py:247-299). */
int lpb_apply_scaled_f32(float* out, const float* u, const float* e, const uint8_t* mask, const float* ke, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);
int lpb_apply_scaled_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* ke, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);
int lpb_apply_weights_f32(float* out, const float* u, const float* w, const float* mcat, const int* patch_id, const float* patch_k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);
int lpb_apply_weights_f64(double* out, const double* u, const double* w, const double* mcat, const int* patch_id, const double* patch_k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);
int lpb_apply_explicit_f32(float* out, const float* u, const float* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);
int lpb_apply_explicit_f64(double* out, const double* u, const double* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, int mask_in, int finish, void* stream);

/* ---- fine-level apply, TMA-tiled (the solver's hot path): same result as lpb_apply_scaled_* with
 * mask_in = 0 and finish = 1 on inputs that are zero on masked dofs; kmodal is a HOST pointer to
 * the 45 corner-parity coefficients (float64) from lpb_modal_ke (passed as kernel parameters);
 * err: device int the kernel sets to 1 if a shared-memory load wait gives up (never expected).
 * Needs pz % 4 == 0, cpz == pz and 16-byte aligned fields. Replaces mgops._product_scaled +
 * _scatter_into with finish (loadpath/mgops.py:86-103, :181-217). */
int lpb_apply_fine_f32(float* out, const float* u, const float* e, const uint8_t* mask, const double* kmodal, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* lpb_apply_fine_f32 with a degree-2 Chebyshev update formed where A u is stored (the V-cycle
 * smoothing of loadpath/mgops.py:312-343 as lpb_cheb2_zero / lpb_residual_scaled / lpb_cheb2
 * apply it, same bits): mode 1 (u = d) x = d + (c1 d + c2 dinv (b - A d)); mode 2 (u = x)
 * r = b - A x, d = s dinv r; mode 3 (u = d) x = (x + d) + (c1 d + c2 dinv (r - A d)). */
int lpb_apply_fine_cheb_f32(int mode, float* x, float* r, float* d, const float* u, const float* b, const float* dinv, const double* coef, const float* e, const uint8_t* mask, const double* kmodal, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_apply_fine_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* kmodal, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* the float64 fine apply that also forms u . out over the level's nodes into *dot (device),
 * for the PCG's p . A p: per-block partials in part (part_len doubles, -3 when short), summed in
 * a fixed order */
int lpb_apply_fine_dot_f64(double* out, const double* u, const double* e, const uint8_t* mask, const double* kmodal, int* err, double* part, long long part_len, double* dot, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* the element matrix (24 x 24, float64, host pointer) in the corner-parity basis that
 * lpb_apply_fine_* reads (45 coefficients, host pointer out); returns the count or < 0 */
int lpb_modal_ke(const double* ke, double* kmodal_out);
/* lpb_modal_ke's 45 coefficients -> the seven classes of the unit brick's cubic symmetry the fine
 * kernel's product uses {a - b, b, d, b2, d2, e2, t} (host pointers); 7, or -1 when the matrix
 * lacks that symmetry (the reference's element matrices, loadpath/fem.py:191-224, have it). */
int lpb_modal_sym(const double* kmodal, double* classes_out);

/* ---- coarse levels on the hot path (u zero on masked dofs; out = m K u):
 * level 1: z-marching kernel in the corner-parity basis; g1 is a HOST pointer to the 279
 * coefficients from lpb_modal_g1; pbox (HOST, 6 ints: x0, y0, z0, nx, ny, nz) bounds the nodes
 * touched by patch cells (patch_id/patch_k may be NULL when there are none). Needs pz % 4 == 0,
 * cpz == pz. Replaces mgops._product_weights + _scatter_into (loadpath/mgops.py:106-128, 181-217).
 * explicit levels: kp holds the 300 upper-triangle entries of each cell's symmetric matrix,
 * entry-major ((300, cells)); ft is caller scratch of 24 * cells values. Replaces
 * mgops._product_explicit + _scatter_into (loadpath/mgops.py:131-146, 181-217). */
int lpb_modal_g1(const double* ke, double* g1_out);
/* level 1, TMA-staged: the Walsh coefficients c = H w of each cell's child moduli in the
 * layout (cpz/4, ny, nx, 4, 8) from lpb_walsh_chunks_* (once per hierarchy, after the patch
 * cells' weights are zeroed), then the march with u arriving by TMA box loads into a 3-stage
 * mbarrier ring and outputs leaving by TMA stores; g1, pbox HOST; err: device int, set when a
 * bounded wait gave up (or to an alignment code 20..25) */
int lpb_walsh_chunks_f32(float* wc, const float* w, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_walsh_chunks_f64(double* wc, const double* w, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_apply_weights_tma_f32(float* out, const float* u, const float* wc, const int* patch_id, const float* patch_k, const uint8_t* mask, const double* g1, const int* pbox, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_apply_weights_tma_f64(double* out, const double* u, const double* wc, const int* patch_id, const double* patch_k, const uint8_t* mask, const double* g1, const int* pbox, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* explicit levels in the cell's corner-parity basis: K^ = T K T^T / 64 has the level-1 pattern
 * (150 upper entries) at every level of the plain hierarchy; lpb_pack_modal_f32 stores them
 * (km: (150, cells)) and lists the cells with off-pattern weight (children with masked patch
 * matrices; glist: up to `cells` ints, *gcount device int) with their 300 node-basis entries
 * (kpc: up to 300 * cells floats, cell-major by list slot); lpb_apply_explicit_modal_f32 applies
 * f = T^T K^ T u on the others and the node-basis entries on the listed ones (half the bytes of
 * lpb_apply_explicit_sym_f32). Same operator as loadpath/mgops.py:131-146 + 181-217. */
int lpb_pack_modal_f32(float* km, int* glist, int* gcount, float* kpc, const float* k, long long ncells, double tol, void* stream);
int lpb_apply_explicit_modal_f32(float* out, const float* u, const float* km, const float* kpc, const int* glist, const int* gcount, float* ft, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* The same with a degree-2 Chebyshev update formed in its gather (the smoothing of
 * loadpath/mgops.py:312-343 as lpb_cheb2_zero / lpb_residual_scaled / lpb_cheb2 apply it):
 * mode 1 (u = d) x = d + (c1 d + c2 dinv (b - A d)); mode 2 (u = x) r = b - A x, d = s dinv r;
 * mode 3 (u = d) x = (x + d) + (c1 d + c2 dinv (r - A d)); coef: the level's coefficients. */
int lpb_apply_explicit_modal_cheb_f32(int mode, float* x, float* r, float* d, const float* u, const float* b, const float* dinv, const double* coef, const float* km, const float* kpc, const int* glist, const int* gcount, float* ft, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_apply_explicit_sym_f32(float* out, const float* u, const float* kp, float* ft, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_apply_explicit_sym_f64(double* out, const double* u, const double* kp, double* ft, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* lpb_apply_explicit_sym_f32 for callers that cannot allocate device memory (a host that owns
 * every device allocation, or a loop that must not call cudaMalloc/cudaFree, which synchronize):
 * the (24, cells) intermediate lives in a 6 MB array inside the library instead of a caller
 * buffer. At most 65,536 padded cells (nx * ny * cpz) per call, else -3. The array's address is
 * looked up for the CURRENT device (cudaGetDevice), so the stream must belong to the current
 * device. The first call on a device looks the array up and should come before any stream
 * capture; the address is kept for the life of the process and is not looked up again after a
 * cudaDeviceReset (do not call this after resetting a device). Calls that overlap on the GPU
 * share the array and race. No counterpart in the reference. */
int lpb_apply_explicit_sym_noalloc_f32(float* out, const float* u, const float* kp, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* (cells, 24, 24) matrices -> packed symmetric entry-major (the mean of K and K^T) */
int lpb_pack_sym_f32(float* kp, const float* k, long long ncells, void* stream);
int lpb_pack_sym_f64(double* kp, const double* k, long long ncells, void* stream);

/* ---- diagonal of K in float64 (loadpath/mg.py:348-371) */
int lpb_diag_scaled_f64(double* d, const double* e, const double* ke, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_diag_weights_f32(double* d, const float* w, const float* mcat, const int* patch_id, const float* patch_k, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_diag_weights_f64(double* d, const double* w, const double* mcat, const int* patch_id, const double* patch_k, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_diag_explicit_f32(double* d, const float* k, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_diag_explicit_f64(double* d, const double* k, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- masks and inverse diagonal (loadpath/mg.py:537-550, :560-576): alive = d > alive_thr,
 * solved = d > live_thr and not held (held_bits may be NULL) and, when kept != NULL, kept >= 1;
 * dinv = solved ? 1/d : 1 (either dinv pointer may be NULL). With thr_scale != NULL (a device
 * scalar, e.g. the level's largest diagonal from lpb_max_f64) both thresholds are multiplied by
 * max(*thr_scale, 1e-300) on the device. */
int lpb_masks(uint8_t* mask, double* dinv64, float* dinv32, const double* d, const uint8_t* held_bits, const float* kept, int nx, int ny, int nz, int pz, int cpz, double alive_thr, double live_thr, const double* thr_scale, void* stream);
/* *out = max(a[0:n]); part: >= 1024 doubles of scratch (loadpath/mg.py:560) */
int lpb_max_f64(const double* a, long long n, double* part, double* out, void* stream);
/* max |a - b| over n doubles (the SIMP loop's design change, loadpath/simp.py:2379) */
int lpb_max_abs_diff_f64(const double* a, const double* b, long long n, double* part, double* out, void* stream);
/* counts into a device float64 scalar (exact), part: >= 592 doubles of scratch. Cells with
 * modulus > 0 (loadpath/mg.py:559), active cells of a level-1 (weights) or explicit level
 * (loadpath/mg.py:593-599: _active_cells), and positions where two byte arrays differ (the
 * hierarchy's reuse check: patch flags of a rebuild against the last build's). */
int lpb_count_positive_f64(const double* e, long long n, double* part, double* out, void* stream);
int lpb_count_active_weights_f32(const float* w, const int* patch_id, int nx, int ny, int nz, int pz, int cpz, double* part, double* out, void* stream);
int lpb_count_active_weights_f64(const double* w, const int* patch_id, int nx, int ny, int nz, int pz, int cpz, double* part, double* out, void* stream);
int lpb_count_active_explicit_f32(const float* k, int nx, int ny, int nz, int pz, int cpz, double* part, double* out, void* stream);
int lpb_count_active_explicit_f64(const double* k, int nx, int ny, int nz, int pz, int cpz, double* part, double* out, void* stream);
int lpb_count_ne_u8(const uint8_t* a, const uint8_t* b, long long n, double* part, double* out, void* stream);

/* ---- Galerkin coarsening (loadpath/mg.py:601-677) */
int lpb_weights_from_e_f64_f32(float* w, const double* e, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_weights_from_e_f64_f64(double* w, const double* e, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_patch_flags(uint8_t* flag, const double* e, const uint8_t* mf, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_patch_matrices_f32(float* pk, float* w, int* patch_id, const long long* pcells, int npatch, const double* e, const double* ke, const uint8_t* mf, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_patch_matrices_f64(double* pk, double* w, int* patch_id, const long long* pcells, int npatch, const double* e, const double* ke, const uint8_t* mf, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_galerkin_explicit_f32(float* kout, int fine_kind, const float* fw, const float* mcat, const int* patch_id, const float* patch_k, const float* fk, const uint8_t* mf, int strict, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_galerkin_explicit_f64(double* kout, int fine_kind, const double* fw, const double* mcat, const int* patch_id, const double* patch_k, const double* fk, const uint8_t* mf, int strict, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
/* level-2 Galerkin matrices from level-1 weights in the plain hierarchy, as 64 fixed products:
 * K(C) = sum_(k,q) w_(k,q) N_(k,q), N_(k,q) = P_k^T M_q P_k (nkq: 64 x 576, index 8k + q); children
 * with a patch matrix add P_k^T patch P_k (patch_id / patch_k NULL when there are none) */
int lpb_galerkin_w2_f32(float* kout, const float* w1, const float* nkq, const int* patch_id, const float* patch_k, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_galerkin_w2_f64(double* kout, const double* w1, const double* nkq, const int* patch_id, const double* patch_k, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
/* strict hierarchy: held dofs injected down a level and restrict(fine mask) (loadpath/mg.py:562-574) */
int lpb_strict_held_kept(uint8_t* held_c, float* kept, const uint8_t* held_f, const uint8_t* mf, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_held0(uint8_t* held, const uint8_t* mask0, const uint8_t* fixed_bits, long long n, void* stream);

/* ---- coarsest level (loadpath/mg.py:708-766): dense D K D + (I - D), symmetrised, over all
 * nodes of the level, dof (c, node) -> c * nodes + node (a check of the band path below) */
int lpb_coarse_dense_f32(double* a, int kind, const float* w, const float* mcat, const int* patch_id, const float* patch_k, const float* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_coarse_dense_f64(double* a, int kind, const double* w, const double* mcat, const int* patch_id, const double* patch_k, const double* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* ---- coarsest level as a band (loadpath/mg.py:708-766; the reference factors the same
 * operator with SuperLU on the host). Dofs numbered 3 * node + component with the longest
 * axis slowest, half-bandwidth bw = 3 (N1 N2 + N2 + 1) + 2 (N1 >= N2 the shorter node extents);
 * the lower band is stored as 32 x 32 tiles, tile (R, d) = rows 32R.., columns 32(R-d)..,
 * row-major at t + (R (D + 1) + d) * 1024, padding dofs past n as identity rows.
 * lpb_band_dims: out = {n, nt, D, bw}, returns the tile count nt (D + 1).
 * lpb_band_factor: in-place tiled signed Cholesky A = L S L^T, S = diag(+-1) (a symmetric LU
 *   without pivoting, as the reference's SuperLU in symmetric mode; one cooperative launch: helper
 *   blocks own tile rows, a critical block finishes the rows in order, all waiting on each other's
 *   progress counts with bounded waits); linv: nt * 1024 doubles, the inverses of the diagonal
 *   factor tiles; sgn: 32 nt doubles, the pivot signs; info: 0 or the 1-based band dof of the first
 *   exactly zero (or non-finite) pivot; bar: 2 max(64, nt) device words of scratch; err: set when
 *   a wait gave up.
 * lpb_band_inverse: ainv (32 nt x 32 nt, row-major, band numbering) = A^-1 from the factor.
 * lpb_band_solve_*: f_out = A^-1 f_in through the band numbering; v: 32 nt doubles scratch. */
int lpb_coarse_band_f32(double* t, int kind, const float* w, const float* mcat, const int* patch_id, const float* patch_k, const float* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_coarse_band_f64(double* t, int kind, const double* w, const double* mcat, const int* patch_id, const double* patch_k, const double* k, const uint8_t* mask, int nx, int ny, int nz, int pz, int cpz, void* stream);
long long lpb_band_dims(int nx, int ny, int nz, long long* out);
int lpb_band_factor(double* t, double* linv, double* sgn, int* info, unsigned* bar, int* err, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_band_inverse(double* ainv, const double* t, const double* linv, const double* sgn, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_band_solve_f32(float* f_out, const float* f_in, const double* ainv, double* v, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_band_solve_f64(double* f_out, const double* f_in, const double* ainv, double* v, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* The same for ncol right-hand sides of a block solve (no reference counterpart: the reference
 * solves its load cases one at a time, loadpath/mg.py:932-949): column c of f_in / f_out at element
 * offset c * cstride; the inverse is read once per 8 columns; v: 32 nt * ncol doubles. */
int lpb_band_solve_cols_f32(float* f_out, const float* f_in, long long cstride, int ncol, const double* ainv, double* v, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_band_solve_cols_f64(double* f_out, const double* f_in, long long cstride, int ncol, const double* ainv, double* v, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- Chebyshev smoother (loadpath/mg.py:771-821, loadpath/mgops.py:312-343) with its
 * coefficients in device memory: lpb_cheb_coef turns the power iteration's dots (vv[k] = |v|^2
 * before step k, vav[k] = v.D^-1 A v after it) into coef[0] = lmax (safety * max(vav[its-1],
 * 1e-12), or 2 when some vv[k] == 0), coef[1] = 1/theta, coef[2+2k], coef[3+2k] = the two
 * update coefficients of step k; degree <= 7 (16 doubles). The passes read coef on the device,
 * so no smoother step needs lmax on the host. */
int lpb_cheb_coef(double* coef, const double* vv, const double* vav, int its, int degree, double safety, void* stream);
int lpb_cheb_start_f32(const float* b, const float* dinv, const double* coef, float* x, float* r, float* d, long long n, void* stream);
int lpb_cheb_start_f64(const double* b, const double* dinv, const double* coef, double* x, double* r, double* d, long long n, void* stream);
int lpb_residual_scaled_f32(const float* b, const float* ax, const float* dinv, const double* coef, float* r, float* d, long long n, void* stream);
int lpb_residual_scaled_f64(const double* b, const double* ax, const double* dinv, const double* coef, double* r, double* d, long long n, void* stream);
int lpb_cheb_f32(float* x, float* d, float* r, const float* ad, const float* dinv, const double* coef, int step, int last, long long n, void* stream);
int lpb_cheb_f64(double* x, double* d, double* r, const double* ad, const double* dinv, const double* coef, int step, int last, long long n, void* stream);
/* degree-2 Chebyshev in two passes per smoothing (same bits as two lpb_cheb_* steps): from
 * zero, lpb_cheb_d_start (d = s dinv b), then with ad = A d lpb_cheb2_zero (x = d + d');
 * otherwise after lpb_residual_scaled and ad = A d, lpb_cheb2 (x = (x + d) + d'), where
 * d' = c1 d + c2 dinv (r - ad) with step 0's coefficients */
int lpb_cheb_d_start_f32(const float* b, const float* dinv, const double* coef, float* d, long long n, void* stream);
int lpb_cheb_d_start_f64(const double* b, const double* dinv, const double* coef, double* d, long long n, void* stream);
int lpb_cheb2_zero_f32(float* x, const float* b, const float* ad, const float* d, const float* dinv, const double* coef, long long n, void* stream);
int lpb_cheb2_zero_f64(double* x, const double* b, const double* ad, const double* d, const double* dinv, const double* coef, long long n, void* stream);
int lpb_cheb2_f32(float* x, const float* d, const float* r, const float* ad, const float* dinv, const double* coef, long long n, void* stream);
int lpb_cheb2_f64(double* x, const double* d, const double* r, const double* ad, const double* dinv, const double* coef, long long n, void* stream);
int lpb_jacobi_f32(float* x, const float* b, const float* ax, const float* dinv, float omega, int from_zero, long long n, void* stream);
int lpb_jacobi_f64(double* x, const double* b, const double* ax, const double* dinv, double omega, int from_zero, long long n, void* stream);

/* ---- grid transfers (loadpath/mgops.py:666-773: coarse_residual, add_correction) */
int lpb_restrict_residual_f32(float* rc, const float* b, const float* ax, const uint8_t* m, const uint8_t* cm, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_restrict_residual_f64(double* rc, const double* b, const double* ax, const uint8_t* m, const uint8_t* cm, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_prolong_add_f32(float* x, const float* xc, const uint8_t* cm, const uint8_t* m, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);
int lpb_prolong_add_f64(double* x, const double* xc, const uint8_t* cm, const uint8_t* m, int fnx, int fny, int fnz, int fpz, int fcpz, int cnx, int cny, int cnz, int cpz_, int ccpz, void* stream);

/* ---- PCG and power-iteration vector passes (loadpath/mgops.py:346-360, :557-585; mg.py:771-794,
 * :872-926). Reductions are deterministic: part needs lpb_reduce_blocks() doubles; results land
 * in device memory. alpha / beta are read as *num / *den on the device. */
int lpb_reduce_blocks(void);
/* record a CUDA event on a stream; inside a stream capture it is recorded with
 * cudaEventRecordExternal, so it becomes a graph node that every replay repeats (kernel timing
 * inside CUDA graphs) */
int lpb_event_record(void* event, void* stream);
int lpb_dot_f64(const double* a, const double* b, long long n, double* part, double* out, void* stream);
int lpb_dot_f32(const float* a, const float* b, long long n, double* part, double* out, void* stream);
int lpb_dot_f64_f32(const double* a, const float* b, long long n, double* part, double* out, void* stream);
int lpb_cg_step(double* x, double* r, const double* p, const double* ap, float* r32, long long n, const double* num, const double* den, double* part, double* rr, void* stream);
int lpb_xpby_f32(double* p, const float* z, long long n, const double* num, const double* den, void* stream);
int lpb_xpby_f64(double* p, const double* z, long long n, const double* num, const double* den, void* stream);
/* the CG update in two passes with x deferred: lpb_cg_step_r moves r (r -= alpha ap, its float32
 * copy, |r|^2 into *rr) and lpb_xpby_x_* then does x += (rz / pap) p and p = z + (rz_new / rz) p
 * (loadpath/mg.py:903-925; the same arithmetic, x updated one pass later) */
int lpb_cg_step_r(double* r, const double* ap, float* r32, long long n, const double* num, const double* den, double* part, double* rr, void* stream);
int lpb_xpby_x_f32(double* p, double* x, const float* z, long long n, const double* rz, const double* pap, const double* rz_new, void* stream);
int lpb_xpby_x_f64(double* p, double* x, const double* z, long long n, const double* rz, const double* pap, const double* rz_new, void* stream);
/* warm start of the PCG on the device (loadpath/mg.py:878-895); sc holds [0] b.b, [5] x.Ax,
 * [6] b.x, [7] |rs|^2 and s = b.x / x.Ax (0 unless x.Ax > 0). lpb_warm_residual: rs = b - s Ax;
 * lpb_warm_select: x = s x, r = rs when s > 0 and |rs| < |b|, else x = 0, r = b. */
int lpb_warm_residual(double* rs, const double* b, const double* ax, const double* sc, long long n, void* stream);
int lpb_warm_select(double* x, double* r, const double* b, const double* rs, const double* sc, long long n, void* stream);
int lpb_axpby_f64(double* out, double a, const double* x, double b, const double* y, long long n, void* stream);
int lpb_axpby_f32(float* out, float a, const float* x, float b, const float* y, long long n, void* stream);
int lpb_cast_f64_f32(float* out, const double* a, long long n, void* stream);
int lpb_cast_f32_f64(double* out, const float* a, long long n, void* stream);
int lpb_mask_field_f32(float* out, const float* u, const uint8_t* m, int nx, int ny, int nz, int pz, int cpz, int bitshift, void* stream);
int lpb_mask_field_f64(double* out, const double* u, const uint8_t* m, int nx, int ny, int nz, int pz, int cpz, int bitshift, void* stream);
int lpb_scale_rsqrt_f32(float* v, long long n, const double* nrm2, void* stream);
int lpb_scale_rsqrt_f64(double* v, long long n, const double* nrm2, void* stream);
int lpb_dinv_mask_f32(float* av, const float* dinv, const uint8_t* m, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_dinv_mask_f64(double* av, const double* dinv, const uint8_t* m, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- SIMP loop (loadpath/simp.py:1143-1228, :1861, :1901-1904, :2001;
 * loadpath/benchmarks/reference.py:48-110; loadpath/femops.py:51-78, loadpath/mg.py:975-988) */
int lpb_filter(double* out, const double* v, const int* toff, const double* tw, int ntaps, const double* hs_in, const double* hs_out, double* e_out, double penal, double emin, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_simp_law(double* e, const double* x, double penal, double emin, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_element_energy_f64(double* ce, const double* u, const double* v, const double* ke, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* femops.element_energy (loadpath/femops.py:236-242) on a general mesh: ce[e] = u_e^T ke v_e with
 * u_e = u[edof[e, 0..23]] (int64 indices, each < the vectors' length, checked by the caller);
 * v NULL: v = u; ke 24 x 24 float64 (device). */
int lpb_element_energy_edof(double* ce, const double* u, const double* v, const long long* edof, const double* ke, long long ne, void* stream);
int lpb_element_energy_f32(double* ce, const float* u, const float* v, const double* ke, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_sensitivity(double* dc, const double* xphys, const double* ce, const double* e, double penal, double emin, double scale, int accumulate, double* part, double* comp, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* volumes[j] of the clipped OC step at nl = 31 multipliers lam[j] (device), weights gv = H (1 / hs) */
int lpb_oc_volumes(double* volumes, const double* x, const double* dc, const double* dv, const double* gv, const double* lam, int nl, double move, double* part, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_oc_apply(double* xnew, const double* x, const double* dc, const double* dv, double lam, double move, double* part, double* change, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* top3d's bisection on the multiplier (loadpath/benchmarks/reference.py:100-110) walked on the
 * device, the host walk of simp.oc_bisection restated: state (7 doubles) = {l1, l2, below, above,
 * lmid, passes, done}; lpb_oc_walk_init starts it at (0, l2) and writes the first 31 candidates;
 * after each lpb_oc_volumes pass over the candidates lpb_oc_walk folds the volumes in, decides
 * what they decide and writes the next candidates, or finishes (done = 1, lmid the step's
 * multiplier). handle: a graph WHILE node's conditional (the loop runs while candidates are
 * open) or 0. lpb_oc_apply_at is lpb_oc_apply at a multiplier in device memory (state + 4). */
int lpb_oc_walk_init(double* state, double* cands, double l2, double target, double tol, void* stream);
int lpb_oc_walk(long long handle, double* state, const double* vols, double* cands, double target, double tol, void* stream);
int lpb_oc_apply_at(double* xnew, const double* x, const double* dc, const double* dv, const double* lam, double move, double* part, double* change, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* loadpath's own design update; flags: uint8 per cell, bit 0 passive solid, bit 1 passive void
 * (NULL: none). lpb_project: xp = (tanh(b eta) + tanh(b (xt - eta))) / den and its derivative dxp
 * (either NULL to skip), held cells 1 / 0 with derivative 0, and *vol = sum xp w when w is given
 * (part: 592 doubles)   (loadpath/simp.py:1443-1450 _project/_dproject, :1779-1785 physical,
 * :1809-1814 eroded) */
int lpb_project(double* xp, double* dxp, const double* xt, double beta, double eta, const uint8_t* flags, const double* w, double* part, double* vol, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* xn = clip(x sqrt(-dc / dv) / sqrt(lm), max(0, x - move), min(1, x + move)), held cells 1 / 0
 * (loadpath/simp.py:2314-2318, the optimality-criteria step at one volume multiplier) */
int lpb_oc_stepped(double* xn, const double* x, const double* dc, const double* dv, double lm, double move, const uint8_t* flags, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* out = a * b (b NULL: a), 0 on held cells, then min(out, 0) (clip0 1) or max(out, 1e-12) (clip0 2):
 * the products the filter chain rule feeds to H^T and its clips (loadpath/simp.py:2001, :2077, :2191,
 * :2204) */
int lpb_cell_product(double* out, const double* a, const double* b, const uint8_t* flags, int clip0, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* v = (v + v mirrored across the grid's mid-plane normal to axis) / 2 in place, axis 0 x, 1 y, 2 z
 * (loadpath/simp.py:1476-1482 `_symmetrize`, every cell of the box having its mirror image) */
int lpb_mirror_average(double* v, int axis, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- the minimum-mass loop's cell stresses (loadpath/constrained.py:597-652, corner points):
 * lpb_stress_pass over the cells that moved and are counted (counted: uint8 cell field, nonzero)
 * forms the corner stresses C B_k u_e (cb: 8 x 6 x 24 float64 on the device, corners x
 * outermost, already divided by the pitch), vm = sqrt(s . VM s) and r = xe vm / lim; mode 0:
 * *out = max r; mode 1: *out = sum (r / sc)^8; mode 2: gxe = sum_k w_k vm_k / lim per cell and fe
 * (cells_padded x 24) = sum_k w_k xe / (vm_k lim) B_k^T C VM s_k, w_k = kappa (r_k / pm)^7 / nc
 * (0 on inactive cells). part: 1184 doubles. lpb_cell_vectors_to_nodes sums each node's share of
 * the cells' 24-vectors into a node field (the adjoint right-hand side). */
int lpb_stress_pass(int mode, const double* u, const double* xe, const uint8_t* counted, const double* cb, double lim, double sc, double pm, double kappa, double nc, double* part, double* out, double* gxe, double* fe, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_cell_vectors_to_nodes(double* out, const double* fe, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- CUDA graphs of a stream's work (the solver records one CG iteration per solve) */
int lpb_capture_begin(void* stream);
int lpb_capture_end(void* stream, void** exec);
int lpb_graph_launch(void* exec, void* stream);
int lpb_graph_free(void* exec);
/* A device-side loop (no reference counterpart: loadpath/mg.py:872-926 tests convergence on the
 * host each iteration): lpb_while_begin starts capturing the body of a graph's WHILE node into
 * the stream, lpb_while_end instantiates it (an exec for lpb_graph_launch); the body's
 * lpb_cg_continue (sc: the PCG scalars, [0] |b|^2, [3] p.Ap, [4] |r|^2; state: iterations,
 * status) ends the loop once |r| <= rtol |b|, p.Ap <= 0, b = 0 or maxiter iterations ran. */
/* Launch-geometry tuning (no reference counterpart), per grid of nx x ny x nz cells: the
 * persistent blocks per SM of the fine float32 (knob 1) and float64 (2) apply, and the z-segment
 * length, in chunks of four planes, of the level-1 float32 (3) and float64 (4) apply; 0 clears it
 * (the launcher decides). Set by loadpath_b200.tune from timed candidates; results are the same
 * operator, the last bit of a float32 sum can differ at segment boundaries. */
int lpb_tune_set(int knob, int nx, int ny, int nz, int value);
int lpb_tune_get(int knob, int nx, int ny, int nz);
int lpb_while_begin(void* stream, long long* handle, void** graph);
int lpb_while_end(void* stream, void* graph, void** exec);
int lpb_cg_continue(long long handle, const double* sc, long long* state, double rtol, long long maxiter, void* stream);
/* The block solve's loop (k columns; sc (k, 8); state (k + 1, 2): per column the iteration it
 * stopped at and its status, then the iteration count): the loop runs while a column does;
 * lpb_snapshot_converged writes m x of column col into out in the iteration it converges. */
int lpb_cg_continue_cols(long long handle, const double* sc, long long* state, int k, double rtol, long long maxiter, void* stream);
int lpb_snapshot_converged(double* out, const double* x, const uint8_t* mask, const long long* state, int col, int k, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_memcpy_async(void* dst, const void* src, long long bytes, void* stream);
int lpb_memset_async(void* dst, int value, long long bytes, void* stream);

/* ---- the float32-only solve's pieces (loadpath/gpu.py:119-149 _two_sum/_rigid_free, :233-258
 * apply_rf, :429-481 solve_fp32). lpb_apply_rf_f32: out = m K (h + l) + (1 - m) h on the fine
 * level (float32 moduli e, float32 ke 24 x 24 on the device), each cell's matrix applied to its
 * corner displacements less the corner-0 translation and the mean rotation, formed in pair
 * (error-free) arithmetic; l may be NULL; ft: scratch of 24 * cells floats.
 * lpb_pair_residual_f32: r = (bh - ax) + bl. lpb_pair_add_f32: (xh, xl) += d in pair arithmetic. */
int lpb_apply_rf_f32(float* out, const float* h, const float* l, const uint8_t* mask, const float* e, const float* ke, float* ft, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_pair_residual_f32(float* r, const float* bh, const float* ax, const float* bl, long long n, void* stream);
int lpb_pair_add_f32(float* xh, float* xl, const float* d, long long n, void* stream);

/* ---- live-cell reduction (loadpath/simp.py:725 the alive set, :263-289 _connected, :795-826
 * _solve_mg): state (uint8 cell field) 0 dead, 1 alive, 2 alive and 26-connected to an alive cell
 * touching a support. flags: bit 0 the cell touches a support, bit 1 an anchor (alive whatever its
 * density). lpb_live_seed sets alive = xp > alive_thr or anchor and seeds the support cells
 * (*n_alive: the alive count, device); lpb_live_flood spreads the reached state one pass (the
 * caller zeroes *changed and repeats while a pass sets it); lpb_live_moduli keeps e on reached
 * cells only; lpb_dead_loads counts loaded dofs without stiffness (the reference then solves
 * the full grid). part: 592 doubles. */
int lpb_live_seed(uint8_t* state, const double* xp, const uint8_t* flags, double alive_thr, double* part, double* n_alive, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_live_flood(uint8_t* state, int* changed, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_live_moduli(double* e_out, const double* e, const uint8_t* state, int nx, int ny, int nz, int pz, int cpz, void* stream);
int lpb_dead_loads(const double* f, const uint8_t* mask, double* part, double* count, int nx, int ny, int nz, int pz, int cpz, void* stream);
/* *count = cells alive in a seeded state (nonzero) but not kept (2) in an earlier flooded state:
 * zero lets the direct solver's reduced system be reused (loadpath/simp.py:288-297) */
int lpb_live_outside(const uint8_t* state, const uint8_t* keep, double* part, double* count, int nx, int ny, int nz, int pz, int cpz, void* stream);

/* ---- MMA (loadpath/mma.py:31-214, MMA.update and MMA._subsolv): the n-sized work of one
 * update over n variables and m <= 8 constraints, float64, device arrays; P, Q, df are (m, n)
 * row-major. `part` is scratch of lpb_mma_part_len(m) doubles; each reduction writes its values to
 * `out` / `bsum` (device) with M = m rounded up to 1, 2, 4 or 8 entries per m-sized group.
 * lam / dlam are HOST pointers to m doubles. The host runs the interior-point loops and the
 * (m + 1) x (m + 1) Newton system (loadpath/mma.py:127-214). */
long long lpb_mma_part_len(int m);
/* sanitise x, df0, df in place (non-finite values as the reference reads them), move the
 * asymptotes (init: the first two iterations), alfa/beta, p0 q0 P Q; bsum[i] = sum_j P_ij / (upp_j -
 * x_j) + Q_ij / (x_j - low_j)   (loadpath/mma.py:57-103) */
int lpb_mma_prepare(long long n, int m, double* x, const double* xmin, const double* xmax, double* low, double* upp, const double* xold1, const double* xold2, int init, double asyinit, double asyincr, double asydecr, double move, double* df0, double* df, double* alfa, double* beta, double* p0, double* q0, double* P, double* Q, double* part, double* bsum, void* stream);
/* the subsolver's start: x = (alfa + beta) / 2, xsi = max(1 / (x - alfa), 1), eta = max(1 / (beta - x), 1) */
int lpb_mma_sub_init(long long n, const double* alfa, const double* beta, double* xs, double* xsi, double* eta, void* stream);
/* a Newton step's n-sized terms: delx, diagx; out = [gvec (M), GG (delx / diagx) (M),
 * (GG / diagx) GG^T upper triangle row by row (M (M + 1) / 2)] */
int lpb_mma_newton_a(long long n, int m, const double* low, const double* upp, const double* alfa, const double* beta, const double* p0, const double* q0, const double* P, const double* Q, const double* xs, const double* xsi, const double* eta, const double* lam, double epsi, double* delx, double* diagx, double* part, double* out, void* stream);
/* dx, dxsi, deta from dlam; out = [max -1.01 dxsi / xsi, max -1.01 deta / eta,
 * max -1.01 dx / (x - alfa), max 1.01 dx / (beta - x)] */
int lpb_mma_newton_b(long long n, int m, const double* low, const double* upp, const double* alfa, const double* beta, const double* P, const double* Q, const double* xs, const double* xsi, const double* eta, const double* delx, const double* diagx, const double* dlam, double epsi, double* dx, double* dxsi, double* deta, double* part, double* out, void* stream);
/* (xs, xsi, eta) = (xs0, xsi0, eta0) + steg (dx, dxsi, deta) (dx NULL: evaluate at xs0 only);
 * out = [sum of squares, largest magnitude of the residual's n-sized rows, gvec (M)] */
int lpb_mma_trial(long long n, int m, const double* low, const double* upp, const double* alfa, const double* beta, const double* p0, const double* q0, const double* P, const double* Q, const double* xs0, const double* xsi0, const double* eta0, const double* dx, const double* dxsi, const double* deta, double steg, const double* lam, double epsi, double* xs, double* xsi, double* eta, double* part, double* out, void* stream);
/* xnew = clip(finite(xs) ? xs : x, alfa, beta)   (loadpath/mma.py:104-108) */
int lpb_mma_finish(long long n, const double* xs, const double* x, const double* alfa, const double* beta, double* xnew, void* stream);


/* ---- the solver behind an opaque handle (loadpath/mg.py:411-988: GridElasticity(...),
 * .set_moduli, .solve_many), for hosts that are not Python. Fields are float64 device arrays in
 * the layout below; the handle owns its device memory (freed by lpb_mg_destroy) and must not be
 * used from two host threads at once. Given the same element matrix, a solve has the bits of
 * loadpath_b200.mg.GridElasticity.solve_device with convergence tested on the host.
 * lpb_mg_create: nx, ny, nz even cell counts; fixed: uint8 (NX, NY, NZ) host array in grid order,
 *   bit c set when component c of the node is held; ke: 24 x 24 element matrix at E = 1 (times the
 *   pitch), host; single: 1 for the float32 V-cycle (the mixed solve), 0 for float64; rtol,
 *   maxiter, coarse_cells as GridElasticity; *status 0 or < 0. Returns the handle or NULL.
 * lpb_mg_set_moduli: e, the fine cells' moduli (layout of lpb_layout_cells_f64): builds the
 *   hierarchy (the strict one when the coarsest factor is singular, loadpath/mg.py:586-591).
 * lpb_mg_solve: x = A^-1 b, b and x0 (may be NULL) masked first; the strict hierarchy when the
 *   plain one stalls (STALL = 100 CG iterations, loadpath/mg.py:951-965); returns 0, 1 when CG did
 *   not converge (loadpath/mg.py:945-946 raises there), < 0 on an error; *iters the CG count.
 * lpb_mg_levels / lpb_mg_strict: the depth and strictness of the current hierarchy. */
void* lpb_mg_create(int nx, int ny, int nz, const uint8_t* fixed, const double* ke, int single, double rtol, int maxiter, long long coarse_cells, int* status);
int lpb_mg_set_moduli(void* h, const double* e, void* stream);
int lpb_mg_solve(void* h, const double* b, const double* x0, double* x, int* iters, void* stream);
int lpb_mg_levels(void* h);
int lpb_mg_strict(void* h);
void lpb_mg_destroy(void* h);
/* host helpers of the handle (and of the Python class, which shares their bits):
 * lpb_hex8_ke: the hex8 element matrix at E = 1 on the unit cube (loadpath/fem.py:191-224),
 *   incompatible = 1 for Wilson's incompatible modes condensed ("im"), 0 for the plain brick;
 * lpb_level1_products: mcat (8 x 576) = P_k^T Ke P_k and nkq (64 x 576, 8 k + q) = P_k^T mcat_q P_k,
 *   P_k the child prolongations (loadpath/mg.py:57-75, 601-677);
 * lpb_uniform_numpy: numpy.random.default_rng(seed).random(n) (the power iteration's start,
 *   loadpath/mg.py:779-781);
 * lpb_layout_dims: {pz, cpz, node field entries, cell field entries, mask entries} of the layout;
 * lpb_layout_nodes_f64 / lpb_unlayout_nodes_f64 / lpb_layout_cells_f64: grid order (3, NX, NY, NZ)
 *   or (nx, ny, nz) <-> the device layout, host arrays. */
int lpb_hex8_ke(double nu, int incompatible, double* ke_out);
int lpb_level1_products(const double* ke, double* mcat, double* nkq);
int lpb_uniform_numpy(long long seed, long long n, double* out);
int lpb_layout_dims(int nx, int ny, int nz, long long* out);
int lpb_layout_nodes_f64(const double* grid, double* out, int nx, int ny, int nz);
int lpb_unlayout_nodes_f64(const double* dev_layout, double* grid, int nx, int ny, int nz);
int lpb_layout_cells_f64(const double* grid, double* out, int nx, int ny, int nz);

#ifdef __cplusplus
}
#endif
#endif /* LOADPATH_B200_H */
