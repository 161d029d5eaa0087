// The multigrid solver behind an opaque handle, for hosts that are not Python
// (loadpath/mg.py:411-988, GridElasticity: the constructor, set_moduli, solve_many).
//
// lpb_mg_create / lpb_mg_set_moduli / lpb_mg_solve / lpb_mg_destroy drive the same kernels in
// the same order as loadpath_b200.mg.GridElasticity (set_moduli_device, solve_device with the
// host-tested CG loop), so a solve through the handle has the bits of a solve through the Python
// class given the same element matrix: the Galerkin hierarchy (level-1 child moduli with patch
// matrices, explicit levels), masks and inverse diagonals, the coarsest level's band factor and
// dense inverse, twelve power iterations per level (the reference's random start,
// lpb_uniform_numpy, then warm-started from the last hierarchy), degree-2 Chebyshev smoothing,
// the float64 PCG with the energy-optimal warm start, and the strict hierarchy when the plain one
// stalls (STALL = 100 CG iterations) or its coarsest factor is singular. Fields live on the
// device in the z-chunked layout (lpb_layout_*). The handle allocates its own device memory and
// frees it in lpb_mg_destroy; one handle must not be used from two host threads at once.
//
// Also here, host code shared with the Python class: the element matrix (lpb_hex8_ke), the
// level-1 Galerkin products (lpb_level1_products), numpy's default_rng(seed).random()
// (lpb_uniform_numpy) and the layout conversions.
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "loadpath_b200.h"
#include "lp_common.cuh"

namespace {

// ---- numpy's default_rng(seed).random(): SeedSequence (one 32-bit word of entropy, a pool of
// four words) seeds PCG64 (128-bit LCG, XSL-RR output), doubles from the top 53 bits. Restated
// from the published algorithms of numpy.random.SeedSequence and PCG64.
typedef unsigned __int128 u128;

void seed_words(uint32_t seed, uint64_t out[4]) {
  const uint32_t INIT_A = 0x43b0d7e5u, MULT_A = 0x931e8875u, INIT_B = 0x8b51f9ddu, MULT_B = 0x58f38dedu;
  const uint32_t MIX_L = 0xca01f9ddu, MIX_R = 0x4973f715u;
  uint32_t hc = INIT_A;
  auto hashmix = [&](uint32_t v) {
    v ^= hc;
    hc *= MULT_A;
    v *= hc;
    v ^= v >> 16;
    return v;
  };
  auto mix = [](uint32_t x, uint32_t y) {
    uint32_t r = MIX_L * x - MIX_R * y;
    r ^= r >> 16;
    return r;
  };
  uint32_t pool[4];
  for (int i = 0; i < 4; ++i) pool[i] = hashmix(i == 0 ? seed : 0u);
  for (int s = 0; s < 4; ++s)
    for (int d = 0; d < 4; ++d)
      if (s != d) pool[d] = mix(pool[d], hashmix(pool[s]));
  uint32_t hb = INIT_B;
  uint32_t w[8];
  for (int i = 0; i < 8; ++i) {
    uint32_t v = pool[i % 4];
    v ^= hb;
    hb *= MULT_B;
    v *= hb;
    v ^= v >> 16;
    w[i] = v;
  }
  for (int i = 0; i < 4; ++i) out[i] = (uint64_t)w[2 * i] | ((uint64_t)w[2 * i + 1] << 32);
}

struct Pcg64 {
  u128 s, inc;
  uint64_t next() {
    static const u128 MULT = ((u128)0x2360ED051FC65DA4ull << 64) | 0x4385DF649FCCF645ull;
    s = s * MULT + inc;
    const uint64_t x = (uint64_t)(s >> 64) ^ (uint64_t)s;
    const unsigned rot = (unsigned)(s >> 122);
    return (x >> rot) | (x << ((64 - rot) & 63));
  }
};

void uniform_numpy(uint32_t seed, long long n, double* out) {
  uint64_t w[4];
  seed_words(seed, w);
  Pcg64 p;
  p.inc = ((((u128)w[2] << 64) | w[3]) << 1) | 1;
  p.s = 0;
  p.next();
  p.s += ((u128)w[0] << 64) | w[1];
  p.next();
  for (long long i = 0; i < n; ++i) out[i] = (double)(p.next() >> 11) * (1.0 / 9007199254740992.0);
}

// ---- the hex8 element (loadpath/fem.py:113-224): unit cube, E = 1, 2x2x2 Gauss points ----------
void strain_op(const double (*grads)[3], int n, double* b /* 6 x 3n */) {
  std::memset(b, 0, sizeof(double) * 6 * 3 * n);
  const int w = 3 * n;
  for (int k = 0; k < n; ++k) {
    const double gx = grads[k][0], gy = grads[k][1], gz = grads[k][2];
    const int c = 3 * k;
    b[0 * w + c] = gx;
    b[1 * w + c + 1] = gy;
    b[2 * w + c + 2] = gz;
    b[3 * w + c] = gy;
    b[3 * w + c + 1] = gx;
    b[4 * w + c + 1] = gz;
    b[4 * w + c + 2] = gy;
    b[5 * w + c] = gz;
    b[5 * w + c + 2] = gx;
  }
}

// out (m x n) += f * a^T c b, a: 6 x m, c: 6 x 6, b: 6 x n
void add_atcb(double* out, const double* a, int m, const double (*c)[6], const double* b, int n, double f) {
  for (int i = 0; i < m; ++i) {
    double ca[6];
    for (int r = 0; r < 6; ++r) {
      double s = 0.0;
      for (int q = 0; q < 6; ++q) s += a[q * m + i] * c[q][r];
      ca[r] = s;
    }
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int r = 0; r < 6; ++r) s += ca[r] * b[r * n + j];
      out[i * n + j] += f * s;
    }
  }
}

bool hex8_ke(double nu, int incompatible, double* ke) {
  if (!(nu > -1.0 && nu < 0.5)) return false;
  const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 0.5 / (1.0 + nu);
  double c[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c[i][j] = lam;
  for (int i = 0; i < 3; ++i) c[i][i] += 2.0 * mu;
  for (int i = 3; i < 6; ++i) c[i][i] = mu;
  static double kuu[24 * 24], kua[24 * 9], kaa[9 * 9];
  std::memset(kuu, 0, sizeof(kuu));
  std::memset(kua, 0, sizeof(kua));
  std::memset(kaa, 0, sizeof(kaa));
  const double g = 1.0 / std::sqrt(3.0);
  for (int ip = 0; ip < 8; ++ip) {
    const double pt[3] = {(ip >> 2) & 1 ? g : -g, (ip >> 1) & 1 ? g : -g, ip & 1 ? g : -g};
    double gr[8][3], gb[3][3] = {};
    for (int k = 0; k < 8; ++k) {
      const double s[3] = {(k & 1) ? 1.0 : -1.0, (k >> 1 & 1) ? 1.0 : -1.0, (k >> 2 & 1) ? 1.0 : -1.0};
      for (int a = 0; a < 3; ++a) {
        const int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
        gr[k][a] = 0.25 * s[a] * (1.0 + pt[o1] * s[o1]) * (1.0 + pt[o2] * s[o2]);
      }
    }
    for (int m = 0; m < 3; ++m) gb[m][m] = -4.0 * pt[m];
    double b[6 * 24], ba[6 * 9];
    strain_op(gr, 8, b);
    strain_op(gb, 3, ba);
    add_atcb(kuu, b, 24, c, b, 24, 0.125);
    add_atcb(kua, b, 24, c, ba, 9, 0.125);
    add_atcb(kaa, ba, 9, c, ba, 9, 0.125);
  }
  double k[24 * 24];
  std::memcpy(k, kuu, sizeof(k));
  if (incompatible) {
    // k = kuu - kua kaa^-1 kua^T, kaa symmetric positive definite (Cholesky)
    double l[9][9] = {};
    for (int i = 0; i < 9; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = kaa[i * 9 + j];
        for (int m = 0; m < j; ++m) s -= l[i][m] * l[j][m];
        if (i == j) {
          if (!(s > 0.0)) return false;
          l[i][i] = std::sqrt(s);
        } else {
          l[i][j] = s / l[j][j];
        }
      }
    for (int col = 0; col < 24; ++col) {
      double y[9];   // kaa^-1 kua^T[:, col]
      for (int i = 0; i < 9; ++i) {
        double s = kua[col * 9 + i];
        for (int m = 0; m < i; ++m) s -= l[i][m] * y[m];
        y[i] = s / l[i][i];
      }
      for (int i = 8; i >= 0; --i) {
        double s = y[i];
        for (int m = i + 1; m < 9; ++m) s -= l[m][i] * y[m];
        y[i] = s / l[i][i];
      }
      for (int row = 0; row < 24; ++row) {
        double s = 0.0;
        for (int m = 0; m < 9; ++m) s += kua[row * 9 + m] * y[m];
        k[row * 24 + col] -= s;
      }
    }
  }
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) ke[i * 24 + j] = 0.5 * (k[i * 24 + j] + k[j * 24 + i]);
  return true;
}

// P_k (coarse cell dofs -> child k's dofs, loadpath/mg.py:57-75), 8 x 24 x 24
void child_prolongations(double* pk) {
  std::memset(pk, 0, sizeof(double) * 8 * 576);
  for (int k = 0; k < 8; ++k)
    for (int q = 0; q < 8; ++q) {
      double p[3];
      for (int a = 0; a < 3; ++a) p[a] = 0.5 * (((k >> a) & 1) + ((q >> a) & 1));
      for (int r = 0; r < 8; ++r) {
        double w = 1.0;
        for (int a = 0; a < 3; ++a) w *= ((r >> a) & 1) ? p[a] : 1.0 - p[a];
        if (w != 0.0)
          for (int i = 0; i < 3; ++i) pk[k * 576 + (3 * q + i) * 24 + 3 * r + i] = w;
      }
    }
}

// out = P^T m P (24 x 24 each)
void ptmp(const double* p, const double* m, double* out) {
  double t[576];
  for (int a = 0; a < 24; ++a)
    for (int j = 0; j < 24; ++j) {
      double s = 0.0;
      for (int b = 0; b < 24; ++b) s += m[a * 24 + b] * p[b * 24 + j];
      t[a * 24 + j] = s;
    }
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) {
      double s = 0.0;
      for (int a = 0; a < 24; ++a) s += p[a * 24 + i] * t[a * 24 + j];
      out[i * 24 + j] = s;
    }
}

// ---- the handle ------------------------------------------------------------------------------
constexpr int STALL = 100;                    // loadpath/mg.py:930
constexpr double LMAX_SAFETY = 1.3;           // loadpath/mg.py:81
constexpr long long DENSE_COARSE_MAX = 12000;  // dofs of the coarsest level solved by the band factor
constexpr double MODAL_TOL = 1e-5;

enum { K_SCALED = 0, K_WEIGHTS = 1, K_EXPLICIT = 2 };

struct HGrid {
  int nx = 0, ny = 0, nz = 0, pz = 0, cpz = 0;
  int NX() const { return nx + 1; }
  int NY() const { return ny + 1; }
  int NZ() const { return nz + 1; }
  long long nnode() const { return 3LL * NX() * NY() * pz; }   // node field entries
  long long nmask() const { return (long long)NX() * NY() * pz; }
  long long ncell() const { return (long long)nx * ny * cpz; }
};
#define HG(g) (g).nx, (g).ny, (g).nz, (g).pz, (g).cpz

HGrid mkgrid(int nx, int ny, int nz) {
  HGrid g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.pz = (nz + 1 + 3) / 4 * 4;
  g.cpz = g.pz;
  return g;
}

struct Level {
  int kind = K_SCALED;
  HGrid g;
  bool f32 = false;
  void* e = nullptr;
  uint8_t* mask = nullptr;
  void* dinv = nullptr;
  void* w = nullptr;
  const void* mcat = nullptr;
  int* patch_id = nullptr;
  void* patch_k = nullptr;
  int npatch = 0;
  int pbox[6] = {0, 0, 0, 0, 0, 0};
  void* wc = nullptr;
  void* k = nullptr;
  void* ft = nullptr;
  void* kp = nullptr;
  void* km = nullptr;
  int* glist = nullptr;
  int* gcount = nullptr;
  void* kpc = nullptr;
  double* coef = nullptr;
  int dims_min() const { return std::min(g.nx, std::min(g.ny, g.nz)); }
};

struct Mg {
  HGrid g0;
  bool f32 = true;
  double rtol = 1e-6;
  int maxiter = 500;
  long long coarse_cells = 2000;
  int degree = 2;
  bool strict = false;
  int last_iters = 0;
  double ke[576], kmodal[45], g1[279];
  std::vector<double> mcat_h, nkq_h;
  std::map<std::string, std::pair<void*, size_t>> work;
  std::map<int, long long> lmax_init;   // level -> node entries of the start vector drawn
  std::vector<Level> levels;
  Level l0s;
  cudaStream_t st = nullptr;
  // fixed pieces
  uint8_t* fixed_bits = nullptr;
  double* ke64 = nullptr;
  float* ke32 = nullptr;
  void* mcat_d = nullptr;
  void* nkq_d = nullptr;
  int* err = nullptr;
  double* part = nullptr;
  long long part_len = 0;
  double *scal = nullptr, *chk = nullptr, *pw = nullptr, *coef = nullptr;
  double* host = nullptr;   // pinned: the CG scalars the host tests
  // coarsest level
  bool has_coarse = false;
  double* ainv = nullptr;
  double* cv = nullptr;
  int* info = nullptr;
  double* e0 = nullptr;     // the moduli of the last set_moduli (own copy)
  int status = LP_OK;       // the first error met (sticky until the next call)

  ~Mg() {
    for (auto& kv : work) cudaFree(kv.second.first);
    if (host) cudaFreeHost(host);
  }

  // a named device buffer of at least `bytes`, zeroed when created (the Python class's _buf / _tbuf)
  void* buf(const std::string& key, size_t bytes, int fill = 0) {
    auto it = work.find(key);
    if (it != work.end() && it->second.second >= bytes) return it->second.first;
    if (it != work.end()) {
      cudaFree(it->second.first);
      work.erase(it);
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
      status = LP_ERR_LAUNCH;
      return nullptr;
    }
    // on the handle's stream: it does not wait for the legacy default stream
    cudaMemsetAsync(p, fill, bytes ? bytes : 1, st);
    work[key] = {p, bytes};
    return p;
  }
  size_t vb() const { return f32 ? 4 : 8; }   // bytes of a V-cycle value
  void* field(const std::string& key, const HGrid& g, bool single) {
    return buf(key, (size_t)g.nnode() * (single ? 4 : 8));
  }
  void ok(int rc) {
    if (rc != LP_OK && status == LP_OK) status = rc < 0 ? rc : LP_ERR_LAUNCH;
  }
  double read(const double* p) {
    double v = 0.0;
    cudaMemcpyAsync(&v, p, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return v;
  }
  Level& op(int i) { return i == 0 ? l0s : levels[i]; }
};

// dispatch helpers over the V-cycle precision
int dot_v(bool f32, const void* a, const void* b, long long n, double* part, double* out, cudaStream_t st) {
  return f32 ? lpb_dot_f32((const float*)a, (const float*)b, n, part, out, st)
             : lpb_dot_f64((const double*)a, (const double*)b, n, part, out, st);
}

void apply(Mg& m, Level& lv, void* out, const void* u) {
  const HGrid& g = lv.g;
  if (lv.kind == K_SCALED) {
    m.ok(lv.f32 ? lpb_apply_fine_f32((float*)out, (const float*)u, (const float*)lv.e, lv.mask, m.kmodal, m.err, HG(g), m.st)
                : lpb_apply_fine_f64((double*)out, (const double*)u, (const double*)lv.e, lv.mask, m.kmodal, m.err, HG(g),
                                     m.st));
  } else if (lv.kind == K_WEIGHTS) {
    int* pid = lv.npatch ? lv.patch_id : nullptr;
    m.ok(lv.f32 ? lpb_apply_weights_tma_f32((float*)out, (const float*)u, (const float*)lv.wc, pid,
                                            (const float*)(lv.npatch ? lv.patch_k : nullptr), lv.mask, m.g1, lv.pbox,
                                            m.err, HG(g), m.st)
                : lpb_apply_weights_tma_f64((double*)out, (const double*)u, (const double*)lv.wc, pid,
                                            (const double*)(lv.npatch ? lv.patch_k : nullptr), lv.mask, m.g1, lv.pbox,
                                            m.err, HG(g), m.st));
  } else if (lv.km) {
    m.ok(lpb_apply_explicit_modal_f32((float*)out, (const float*)u, (const float*)lv.km, (const float*)lv.kpc,
                                      lv.glist, lv.gcount, (float*)lv.ft, lv.mask, HG(g), m.st));
  } else {
    m.ok(lv.f32 ? lpb_apply_explicit_sym_f32((float*)out, (const float*)u, (const float*)lv.kp, (float*)lv.ft, lv.mask,
                                             HG(g), m.st)
                : lpb_apply_explicit_sym_f64((double*)out, (const double*)u, (const double*)lv.kp, (double*)lv.ft,
                                             lv.mask, HG(g), m.st));
  }
}

void diagonal(Mg& m, Level& lv, double* d) {
  const HGrid& g = lv.g;
  if (lv.kind == K_WEIGHTS) {
    m.ok(lv.f32 ? lpb_diag_weights_f32(d, (const float*)lv.w, (const float*)lv.mcat, lv.patch_id,
                                       (const float*)lv.patch_k, HG(g), m.st)
                : lpb_diag_weights_f64(d, (const double*)lv.w, (const double*)lv.mcat, lv.patch_id,
                                       (const double*)lv.patch_k, HG(g), m.st));
  } else {
    m.ok(lv.f32 ? lpb_diag_explicit_f32(d, (const float*)lv.k, HG(g), m.st)
                : lpb_diag_explicit_f64(d, (const double*)lv.k, HG(g), m.st));
  }
}

void count_active(Mg& m, Level& lv, double* out) {
  const HGrid& g = lv.g;
  if (lv.kind == K_WEIGHTS) {
    int* pid = lv.npatch ? lv.patch_id : nullptr;
    m.ok(lv.f32 ? lpb_count_active_weights_f32((const float*)lv.w, pid, HG(g), m.part, out, m.st)
                : lpb_count_active_weights_f64((const double*)lv.w, pid, HG(g), m.part, out, m.st));
  } else {
    m.ok(lv.f32 ? lpb_count_active_explicit_f32((const float*)lv.k, HG(g), m.part, out, m.st)
                : lpb_count_active_explicit_f64((const double*)lv.k, HG(g), m.part, out, m.st));
  }
}

// Galerkin coarse level (loadpath/mg.py:601-677)
Level coarsen(Mg& m, Level& fine, int depth) {
  const HGrid& gf = fine.g;
  int h[3] = {gf.nx / 2, gf.ny / 2, gf.nz / 2};
  for (int a = 0; a < 3; ++a)
    if (h[a] > 1) h[a] += h[a] % 2;
  Level lv;
  lv.g = mkgrid(h[0], h[1], h[2]);
  lv.f32 = m.f32;
  const HGrid& gc = lv.g;
  const long long ncp = gc.ncell();
  const size_t vb = m.vb();
  if (depth == 1) {
    lv.kind = K_WEIGHTS;
    lv.w = m.buf("w1", vb * 8 * ncp);
    m.ok(m.f32 ? lpb_weights_from_e_f64_f32((float*)lv.w, (const double*)fine.e, HG(gf), HG(gc), m.st)
               : lpb_weights_from_e_f64_f64((double*)lv.w, (const double*)fine.e, HG(gf), HG(gc), m.st));
    lv.mcat = m.mcat_d;
    uint8_t* flag = (uint8_t*)m.buf("pflag", ncp);
    m.ok(lpb_patch_flags(flag, (const double*)fine.e, fine.mask, HG(gf), HG(gc), m.st));
    std::vector<uint8_t> fh(ncp);
    cudaMemcpyAsync(fh.data(), flag, ncp, cudaMemcpyDeviceToHost, m.st);
    cudaStreamSynchronize(m.st);
    std::vector<long long> pcells;
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-1, -1, -1};
    for (long long i = 0; i < ncp; ++i)
      if (fh[i]) {
        pcells.push_back(i);
        const long long col = i / 4;   // cell index -> (x, y, z), chunked layout
        const int x = (int)(col % gc.nx), y = (int)((col / gc.nx) % gc.ny), z = (int)(4 * (col / ((long long)gc.nx * gc.ny)) + i % 4);
        lo[0] = std::min(lo[0], x);
        lo[1] = std::min(lo[1], y);
        lo[2] = std::min(lo[2], z);
        hi[0] = std::max(hi[0], x + 2);
        hi[1] = std::max(hi[1], y + 2);
        hi[2] = std::max(hi[2], z + 2);
      }
    lv.npatch = (int)pcells.size();
    if (lv.npatch)
      for (int a = 0; a < 3; ++a) {
        lv.pbox[a] = lo[a];
        lv.pbox[3 + a] = hi[a] - lo[a];
      }
    lv.patch_id = (int*)m.buf("patch_id", 4 * ncp);
    cudaMemsetAsync(lv.patch_id, 0xff, 4 * ncp, m.st);   // -1: no patch matrix
    if (lv.npatch) {
      lv.patch_k = m.buf("patch_k", vb * 576 * (size_t)lv.npatch);
      long long* pc = (long long*)m.buf("pcells", 8 * (size_t)lv.npatch);
      cudaMemcpyAsync(pc, pcells.data(), 8 * (size_t)lv.npatch, cudaMemcpyHostToDevice, m.st);
      m.ok(m.f32 ? lpb_patch_matrices_f32((float*)lv.patch_k, (float*)lv.w, lv.patch_id, pc, lv.npatch,
                                          (const double*)fine.e, m.ke64, fine.mask, HG(gf), HG(gc), m.st)
                 : lpb_patch_matrices_f64((double*)lv.patch_k, (double*)lv.w, lv.patch_id, pc, lv.npatch,
                                          (const double*)fine.e, m.ke64, fine.mask, HG(gf), HG(gc), m.st));
      cudaStreamSynchronize(m.st);   // pcells' host copy is released below
    }
    lv.wc = m.buf("wc1", vb * 8 * ncp);
    m.ok(m.f32 ? lpb_walsh_chunks_f32((float*)lv.wc, (const float*)lv.w, HG(gc), m.st)
               : lpb_walsh_chunks_f64((double*)lv.wc, (const double*)lv.w, HG(gc), m.st));
    return lv;
  }
  lv.kind = K_EXPLICIT;
  const std::string d = std::to_string(depth);
  lv.k = m.buf("k" + d, vb * 576 * ncp);
  if (fine.kind == K_WEIGHTS && !m.strict) {
    const void* pid = fine.npatch ? fine.patch_id : nullptr;
    const void* pk = fine.npatch ? fine.patch_k : nullptr;
    m.ok(m.f32 ? lpb_galerkin_w2_f32((float*)lv.k, (const float*)fine.w, (const float*)m.nkq_d, (const int*)pid,
                                     (const float*)pk, HG(gf), HG(gc), m.st)
               : lpb_galerkin_w2_f64((double*)lv.k, (const double*)fine.w, (const double*)m.nkq_d, (const int*)pid,
                                     (const double*)pk, HG(gf), HG(gc), m.st));
  } else if (fine.kind == K_WEIGHTS) {
    m.ok(m.f32 ? lpb_galerkin_explicit_f32((float*)lv.k, 1, (const float*)fine.w, (const float*)fine.mcat,
                                           fine.patch_id, (const float*)fine.patch_k, nullptr, fine.mask,
                                           (int)m.strict, HG(gf), HG(gc), m.st)
               : lpb_galerkin_explicit_f64((double*)lv.k, 1, (const double*)fine.w, (const double*)fine.mcat,
                                           fine.patch_id, (const double*)fine.patch_k, nullptr, fine.mask,
                                           (int)m.strict, HG(gf), HG(gc), m.st));
  } else {
    m.ok(m.f32 ? lpb_galerkin_explicit_f32((float*)lv.k, 2, nullptr, nullptr, nullptr, nullptr, (const float*)fine.k,
                                           fine.mask, (int)m.strict, HG(gf), HG(gc), m.st)
               : lpb_galerkin_explicit_f64((double*)lv.k, 2, nullptr, nullptr, nullptr, nullptr,
                                           (const double*)fine.k, fine.mask, (int)m.strict, HG(gf), HG(gc), m.st));
  }
  lv.ft = m.buf("ft" + d, vb * 24 * ncp);
  if (!m.f32 || m.strict) {
    lv.kp = m.buf("kp" + d, vb * 300 * ncp);
    m.ok(m.f32 ? lpb_pack_sym_f32((float*)lv.kp, (const float*)lv.k, ncp, m.st)
               : lpb_pack_sym_f64((double*)lv.kp, (const double*)lv.k, ncp, m.st));
  } else {
    lv.km = m.buf("km" + d, 4 * 150 * ncp);
    lv.glist = (int*)m.buf("glist" + d, 4 * ncp);
    lv.gcount = (int*)m.buf("gcount" + d, 4);
    lv.kpc = m.buf("kpc" + d, 4 * 300 * ncp);
    m.ok(lpb_pack_modal_f32((float*)lv.km, lv.glist, lv.gcount, (float*)lv.kpc, (const float*)lv.k, ncp, MODAL_TOL,
                            m.st));
  }
  return lv;
}

// the coarsest level's band factor and dense inverse (loadpath/mg.py:708-754)
void build_coarse(Mg& m, Level& lv) {
  m.has_coarse = false;
  if (m.levels.size() < 2) return;
  const HGrid& g = lv.g;
  const long long n = 3LL * g.NX() * g.NY() * g.NZ();
  if (n > DENSE_COARSE_MAX) return;
  long long dims[4];
  const long long ntiles = lpb_band_dims(g.nx, g.ny, g.nz, dims);
  const long long nt = dims[1], npad = 32 * nt;
  double* t = (double*)m.buf("band_t", 8 * 1024 * (size_t)ntiles);
  if (lv.kind == K_WEIGHTS)
    m.ok(m.f32 ? lpb_coarse_band_f32(t, 1, (const float*)lv.w, (const float*)lv.mcat, lv.patch_id,
                                     (const float*)(lv.npatch ? lv.patch_k : nullptr), nullptr, lv.mask, HG(g), m.st)
               : lpb_coarse_band_f64(t, 1, (const double*)lv.w, (const double*)lv.mcat, lv.patch_id,
                                     (const double*)(lv.npatch ? lv.patch_k : nullptr), nullptr, lv.mask, HG(g), m.st));
  else
    m.ok(m.f32 ? lpb_coarse_band_f32(t, 2, nullptr, nullptr, nullptr, nullptr, (const float*)lv.k, lv.mask, HG(g), m.st)
               : lpb_coarse_band_f64(t, 2, nullptr, nullptr, nullptr, nullptr, (const double*)lv.k, lv.mask, HG(g),
                                     m.st));
  double* linv = (double*)m.buf("band_linv", 8 * 1024 * (size_t)nt);
  m.info = (int*)m.buf("band_info", 8);
  unsigned* bar = (unsigned*)m.buf("band_bar", 8 * (size_t)std::max(64LL, nt));
  m.ainv = (double*)m.buf("band_ainv", 8 * (size_t)npad * npad);
  double* sgn = (double*)m.buf("band_sgn", 8 * (size_t)npad);
  m.cv = (double*)m.buf("coarse_v", 8 * (size_t)npad);
  cudaMemsetAsync(m.info, 0, 8, m.st);
  m.ok(lpb_band_factor(t, linv, sgn, m.info, bar, m.info + 1, HG(g), m.st));
  m.ok(lpb_band_inverse(m.ainv, t, linv, sgn, HG(g), m.st));
  m.has_coarse = true;
}

// the power iteration's start vector: numpy's default_rng(level).random(node shape) - 0.5, drawn
// once per level shape, then the last hierarchy's vector (loadpath/mg.py:771-794)
void lmax_vectors(Mg& m, int i, void*& v, void*& av, void*& keep) {
  Level& lv = m.op(i);
  const HGrid& g = lv.g;
  const std::string s = std::to_string(i);
  v = m.field("pw_v" + s, g, lv.f32);
  av = m.field("pw_av" + s, g, lv.f32);
  keep = m.field("pw_keep" + s, g, lv.f32);
  const long long key = g.nnode() * (lv.f32 ? 1 : -1);
  auto it = m.lmax_init.find(i);
  if (it != m.lmax_init.end() && it->second == key) return;
  const long long nn = 3LL * g.NX() * g.NY() * g.NZ();
  std::vector<double> r(nn), lay(g.nnode());
  uniform_numpy((uint32_t)i, nn, r.data());
  for (auto& x : r) x -= 0.5;
  lpb_layout_nodes_f64(r.data(), lay.data(), g.nx, g.ny, g.nz);
  if (lv.f32) {
    std::vector<float> f(lay.begin(), lay.end());
    cudaMemcpyAsync(keep, f.data(), 4 * f.size(), cudaMemcpyHostToDevice, m.st);
    cudaStreamSynchronize(m.st);
  } else {
    cudaMemcpyAsync(keep, lay.data(), 8 * lay.size(), cudaMemcpyHostToDevice, m.st);
    cudaStreamSynchronize(m.st);
  }
  m.lmax_init[i] = key;
}

void estimate_lmax(Mg& m, int i, int its = 12) {
  Level& lv = m.op(i);
  const HGrid& g = lv.g;
  void *v, *av, *keep;
  lmax_vectors(m, i, v, av, keep);
  const bool f = lv.f32;
  m.ok(f ? lpb_mask_field_f32((float*)v, (const float*)keep, lv.mask, HG(g), 0, m.st)
         : lpb_mask_field_f64((double*)v, (const double*)keep, lv.mask, HG(g), 0, m.st));
  const long long n = g.nnode();
  double* pw = m.pw + 32 * i;
  for (int it = 0; it < its; ++it) {
    m.ok(dot_v(f, v, v, n, m.part, pw + it, m.st));
    m.ok(f ? lpb_scale_rsqrt_f32((float*)v, n, pw + it, m.st) : lpb_scale_rsqrt_f64((double*)v, n, pw + it, m.st));
    apply(m, lv, av, v);
    m.ok(f ? lpb_dinv_mask_f32((float*)av, (const float*)lv.dinv, lv.mask, HG(g), m.st)
           : lpb_dinv_mask_f64((double*)av, (const double*)lv.dinv, lv.mask, HG(g), m.st));
    m.ok(dot_v(f, v, av, n, m.part, pw + 16 + it, m.st));
    std::swap(v, av);
  }
  m.ok(f ? lpb_mask_field_f32((float*)keep, (const float*)v, lv.mask, HG(g), 0, m.st)
         : lpb_mask_field_f64((double*)keep, (const double*)v, lv.mask, HG(g), 0, m.st));
  m.ok(lpb_cheb_coef(m.coef + 16 * i, pw, pw + 16, its, std::max(m.degree, 1), LMAX_SAFETY, m.st));
}

// one hierarchy build (loadpath/mg.py:515-591); false when the coarsest factor is singular
bool build(Mg& m) {
  const HGrid& g0 = m.g0;
  Level l0;
  l0.kind = K_SCALED;
  l0.g = g0;
  l0.f32 = false;
  l0.e = m.e0;
  double* d0 = (double*)m.field("diag0", g0, false);
  m.ok(lpb_diag_scaled_f64(d0, m.e0, m.ke64, HG(g0), m.st));
  l0.mask = (uint8_t*)m.buf("mask0", g0.nmask());
  l0.dinv = m.field("dinv0_64", g0, false);
  float* dinv32 = m.f32 ? (float*)m.field("dinv0_32", g0, true) : nullptr;
  m.ok(lpb_masks(l0.mask, (double*)l0.dinv, dinv32, d0, m.fixed_bits, nullptr, HG(g0), 1e-300, 1e-300, nullptr, m.st));
  m.levels.clear();
  m.levels.push_back(l0);
  if (m.f32) {
    Level s = l0;
    s.f32 = true;
    s.e = m.buf("e0_32", 4 * g0.ncell());
    m.ok(lpb_cast_f64_f32((float*)s.e, m.e0, g0.ncell(), m.st));
    s.dinv = dinv32;
    m.l0s = s;
  } else {
    m.l0s = l0;
  }
  m.ok(lpb_count_positive_f64(m.e0, g0.ncell(), m.part, m.chk, m.st));
  double count = m.read(m.chk);
  uint8_t* held = nullptr;
  if (m.strict) {
    held = (uint8_t*)m.buf("held0", g0.nmask());
    m.ok(lpb_held0(held, l0.mask, m.fixed_bits, g0.nmask(), m.st));
  }
  int depth = 0;
  while (count > (double)m.coarse_cells && m.levels.back().dims_min() >= 2 && m.status == LP_OK) {
    ++depth;
    if (depth >= 30) {
      m.status = LP_ERR_SIZE;
      return true;
    }
    Level c = coarsen(m, m.levels.back(), depth);
    const HGrid& gc = c.g;
    const std::string s = std::to_string(depth);
    double* d = (double*)m.field("diag" + s, gc, false);
    diagonal(m, c, d);
    m.ok(lpb_max_f64(d, gc.nnode(), m.part, m.chk + 40 + depth, m.st));
    uint8_t* held_c = nullptr;
    float* kept = nullptr;
    if (m.strict) {
      held_c = (uint8_t*)m.buf("held" + s, gc.nmask());
      kept = (float*)m.field("kept" + s, gc, true);
      const HGrid& gf = m.levels.back().g;
      m.ok(lpb_strict_held_kept(held_c, kept, held, m.levels.back().mask, HG(gf), HG(gc), m.st));
      held = held_c;
    }
    c.mask = (uint8_t*)m.buf("mask" + s, gc.nmask());
    c.dinv = m.field("dinv" + s, gc, m.f32);
    m.ok(lpb_masks(c.mask, m.f32 ? nullptr : (double*)c.dinv, m.f32 ? (float*)c.dinv : nullptr, d, held_c, kept, HG(gc),
                   1e-12, 1e-12, m.chk + 40 + depth, m.st));
    count_active(m, c, m.chk + depth);
    count = m.read(m.chk + depth);
    m.levels.push_back(c);
  }
  build_coarse(m, m.levels.back());
  const int nl = (int)m.levels.size();
  for (int i = 0; i < nl; ++i) m.op(i).coef = m.coef + 16 * i;
  for (int i = 0; i < nl; ++i) estimate_lmax(m, i);
  if (m.has_coarse) {
    int st2[2] = {0, 0};
    cudaMemcpyAsync(st2, m.info, 8, cudaMemcpyDeviceToHost, m.st);
    cudaStreamSynchronize(m.st);
    if (st2[1]) {
      m.status = LP_ERR_LAUNCH;   // a wait of the factorisation gave up
      return true;
    }
    if (st2[0]) return false;
  }
  return true;
}

void set_moduli(Mg& m) {
  if (!build(m)) {
    // the coarsest factor is singular: the strict hierarchy (loadpath/mg.py:586-591)
    if (m.strict) {
      m.status = LP_ERR_ARG;
      return;
    }
    m.strict = true;
    if (!build(m)) m.status = LP_ERR_ARG;
  }
}

// Chebyshev smoothing of level i (degree 2; the fused forms of the Python class)
void smooth(Mg& m, int i, const void* b, void* x, bool from_zero) {
  Level& lv = m.op(i);
  const HGrid& g = lv.g;
  const bool f = lv.f32;
  const std::string s = std::to_string(i);
  void* r = m.field("r" + s, g, f);
  void* d = m.field("d" + s, g, f);
  void* t = m.field("t" + s, g, f);
  const long long n = g.nnode();
  const double* coef = lv.coef;
  if (lv.kind == K_SCALED && f) {
    auto fused = [&](int mode, const void* u) {
      m.ok(lpb_apply_fine_cheb_f32(mode, (float*)x, (float*)r, (float*)d, (const float*)u, (const float*)b,
                                   (const float*)lv.dinv, coef, (const float*)lv.e, lv.mask, m.kmodal, m.err, HG(g),
                                   m.st));
    };
    if (from_zero) {
      m.ok(lpb_cheb_d_start_f32((const float*)b, (const float*)lv.dinv, coef, (float*)d, n, m.st));
      fused(1, d);
    } else {
      fused(2, x);
      fused(3, d);
    }
    return;
  }
  if (lv.kind == K_EXPLICIT && lv.km) {
    auto fused = [&](int mode, const void* u) {
      m.ok(lpb_apply_explicit_modal_cheb_f32(mode, (float*)x, (float*)r, (float*)d, (const float*)u, (const float*)b,
                                             (const float*)lv.dinv, coef, (const float*)lv.km, (const float*)lv.kpc,
                                             lv.glist, lv.gcount, (float*)lv.ft, lv.mask, HG(g), m.st));
    };
    if (from_zero) {
      m.ok(lpb_cheb_d_start_f32((const float*)b, (const float*)lv.dinv, coef, (float*)d, n, m.st));
      fused(1, d);
    } else {
      fused(2, x);
      fused(3, d);
    }
    return;
  }
  if (from_zero) {
    m.ok(f ? lpb_cheb_d_start_f32((const float*)b, (const float*)lv.dinv, coef, (float*)d, n, m.st)
           : lpb_cheb_d_start_f64((const double*)b, (const double*)lv.dinv, coef, (double*)d, n, m.st));
    apply(m, lv, t, d);
    m.ok(f ? lpb_cheb2_zero_f32((float*)x, (const float*)b, (const float*)t, (const float*)d, (const float*)lv.dinv, coef,
                                n, m.st)
           : lpb_cheb2_zero_f64((double*)x, (const double*)b, (const double*)t, (const double*)d,
                                (const double*)lv.dinv, coef, n, m.st));
  } else {
    apply(m, lv, t, x);
    m.ok(f ? lpb_residual_scaled_f32((const float*)b, (const float*)t, (const float*)lv.dinv, coef, (float*)r, (float*)d, n,
                                     m.st)
           : lpb_residual_scaled_f64((const double*)b, (const double*)t, (const double*)lv.dinv, coef, (double*)r,
                                     (double*)d, n, m.st));
    apply(m, lv, t, d);
    m.ok(f ? lpb_cheb2_f32((float*)x, (const float*)d, (const float*)r, (const float*)t, (const float*)lv.dinv, coef, n,
                           m.st)
           : lpb_cheb2_f64((double*)x, (const double*)d, (const double*)r, (const double*)t, (const double*)lv.dinv,
                           coef, n, m.st));
  }
}

// x = V(b) on level i (loadpath/mg.py:837-860); with r64 also *dot = r64 . x
void* vcycle(Mg& m, int i, const void* b, const double* r64 = nullptr, double* dot = nullptr) {
  Level& lv = m.op(i);
  const HGrid& g = lv.g;
  const bool f = lv.f32;
  const std::string s = std::to_string(i);
  void* x = m.field("x" + s, g, f);
  if (i == (int)m.levels.size() - 1) {
    if (m.has_coarse) {
      m.ok(f ? lpb_band_solve_f32((float*)x, (const float*)b, m.ainv, m.cv, HG(g), m.st)
             : lpb_band_solve_f64((double*)x, (const double*)b, m.ainv, m.cv, HG(g), m.st));
    } else {
      smooth(m, i, b, x, true);
      smooth(m, i, b, x, false);
    }
    if (r64) m.ok(lpb_dot_f64_f32(r64, (const float*)x, g.nnode(), m.part, dot, m.st));
    return x;
  }
  smooth(m, i, b, x, true);
  void* t = m.field("t" + s, g, f);
  apply(m, lv, t, x);
  Level& nxt = m.op(i + 1);
  const HGrid& gc = nxt.g;
  void* bc = m.field("b" + std::to_string(i + 1), gc, f);
  m.ok(f ? lpb_restrict_residual_f32((float*)bc, (const float*)b, (const float*)t, lv.mask, nxt.mask, HG(g), HG(gc), m.st)
         : lpb_restrict_residual_f64((double*)bc, (const double*)b, (const double*)t, lv.mask, nxt.mask, HG(g), HG(gc),
                                     m.st));
  void* xc = vcycle(m, i + 1, bc);
  m.ok(f ? lpb_prolong_add_f32((float*)x, (const float*)xc, nxt.mask, lv.mask, HG(g), HG(gc), m.st)
         : lpb_prolong_add_f64((double*)x, (const double*)xc, nxt.mask, lv.mask, HG(g), HG(gc), m.st));
  smooth(m, i, b, x, false);
  if (r64) m.ok(lpb_dot_f64_f32(r64, (const float*)x, g.nnode(), m.part, dot, m.st));
  return x;
}

// z = V(r) with the casts to and from the V-cycle precision (loadpath/mg.py:862-864)
void precondition(Mg& m, const double* r64, double* z) {
  const HGrid& g = m.g0;
  const long long n = g.nnode();
  if (m.f32) {
    float* b = (float*)m.field("b0", g, true);
    m.ok(lpb_cast_f64_f32(b, r64, n, m.st));
    float* x = (float*)vcycle(m, 0, b);
    m.ok(lpb_cast_f32_f64(z, x, n, m.st));
  } else {
    double* b = (double*)m.field("b0", g, false);
    cudaMemcpyAsync(b, r64, 8 * n, cudaMemcpyDeviceToDevice, m.st);
    double* x = (double*)vcycle(m, 0, b);
    cudaMemcpyAsync(z, x, 8 * n, cudaMemcpyDeviceToDevice, m.st);
  }
}

// float64 PCG (loadpath/mg.py:872-926), the Python class's host-tested loop; b: the masked
// right-hand side in cg_b; x0 (masked) or null. Returns the iterate (cg_x).
double* pcg(Mg& m, const double* x0, int& iters, bool& ok) {
  const HGrid& g = m.g0;
  const long long n = g.nnode();
  const size_t nb = 8 * (size_t)n;
  Level& a = m.levels[0];
  double* sc = m.scal;
  double* x = (double*)m.field("cg_x", g, false);
  double* r = (double*)m.field("cg_r", g, false);
  double* p = (double*)m.field("cg_p", g, false);
  double* ap = (double*)m.field("cg_ap", g, false);
  double* z = (double*)m.field("cg_z", g, false);
  double* rs = (double*)m.field("cg_rs", g, false);
  float* r32 = m.f32 ? (float*)m.field("cg_r32", g, true) : nullptr;
  double* src = (double*)m.field("cg_b", g, false);
  if (x0) cudaMemcpyAsync(x, x0, nb, cudaMemcpyDeviceToDevice, m.st);
  // set-up: the warm start chosen on the device (loadpath/mg.py:880-896)
  m.ok(lpb_dot_f64(src, src, n, m.part, sc + 0, m.st));
  if (x0) {
    apply(m, a, ap, x);
    m.ok(lpb_dot_f64(x, ap, n, m.part, sc + 5, m.st));
    m.ok(lpb_dot_f64(src, x, n, m.part, sc + 6, m.st));
    m.ok(lpb_warm_residual(rs, src, ap, sc, n, m.st));
    m.ok(lpb_dot_f64(rs, rs, n, m.part, sc + 7, m.st));
    m.ok(lpb_warm_select(x, r, src, rs, sc, n, m.st));
  } else {
    cudaMemsetAsync(x, 0, nb, m.st);
    cudaMemcpyAsync(r, src, nb, cudaMemcpyDeviceToDevice, m.st);
  }
  precondition(m, r, z);
  cudaMemcpyAsync(p, z, nb, cudaMemcpyDeviceToDevice, m.st);
  m.ok(lpb_dot_f64(r, z, n, m.part, sc + 1, m.st));
  double tol = -1.0;
  cudaEvent_t ev;
  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  ok = false;
  iters = m.maxiter;
  for (int it = 1; it <= m.maxiter && m.status == LP_OK; ++it) {
    // head: ap = A p with p . A p, r -= alpha ap (and its float32 copy), |r|^2
    m.ok(lpb_apply_fine_dot_f64(ap, p, m.e0, a.mask, m.kmodal, m.err, m.part, m.part_len, sc + 3, HG(g), m.st));
    m.ok(lpb_cg_step_r(r, ap, r32, n, sc + 1, sc + 3, m.part, sc + 4, m.st));
    cudaMemcpyAsync(m.host, sc + 3, 16, cudaMemcpyDeviceToHost, m.st);
    cudaMemcpyAsync(m.host + 2, sc, 8, cudaMemcpyDeviceToHost, m.st);
    cudaEventRecord(ev, m.st);
    // tail, queued before the test: z = V(r), x += alpha p, p = z + beta p
    if (r32) {
      float* xv = (float*)vcycle(m, 0, r32, r, sc + 2);
      m.ok(lpb_xpby_x_f32(p, x, xv, n, sc + 1, sc + 3, sc + 2, m.st));
    } else {
      precondition(m, r, z);
      m.ok(lpb_dot_f64(r, z, n, m.part, sc + 2, m.st));
      m.ok(lpb_xpby_x_f64(p, x, z, n, sc + 1, sc + 3, sc + 2, m.st));
    }
    cudaMemcpyAsync(sc + 1, sc + 2, 8, cudaMemcpyDeviceToDevice, m.st);
    cudaEventSynchronize(ev);
    if (tol < 0.0) {
      const double bb = m.host[2];
      if (bb == 0.0) {
        cudaStreamSynchronize(m.st);
        cudaMemsetAsync(x, 0, nb, m.st);
        iters = 0;
        ok = true;
        break;
      }
      tol = m.rtol * std::sqrt(bb);
    }
    const double pap = m.host[0], rr = m.host[1];
    if (!(pap > 0.0)) {
      iters = it;
      break;
    }
    if (std::sqrt(rr) <= tol) {
      iters = it;
      ok = true;
      break;
    }
  }
  cudaStreamSynchronize(m.st);
  cudaEventDestroy(ev);
  return x;
}

}  // namespace

extern "C" {

// numpy.random.default_rng(seed).random(n) into out (host)
int lpb_uniform_numpy(long long seed, long long n, double* out) {
  if (seed < 0 || seed > 0xffffffffLL || n < 0 || (n && !out)) return LP_ERR_ARG;
  uniform_numpy((uint32_t)seed, n, out);
  return LP_OK;
}

// the hex8 element matrix at E = 1 on the unit cube (host, 24 x 24 row-major)
int lpb_hex8_ke(double nu, int incompatible, double* ke_out) {
  if (!ke_out) return LP_ERR_ARG;
  return hex8_ke(nu, incompatible, ke_out) ? LP_OK : LP_ERR_ARG;
}

// the level-1 Galerkin tables from the element matrix (host): mcat (8 x 576) = P_k^T Ke P_k and
// nkq (64 x 576, index 8 k + q) = P_k^T mcat_q P_k
int lpb_level1_products(const double* ke, double* mcat, double* nkq) {
  if (!ke || !mcat || !nkq) return LP_ERR_ARG;
  static double pk[8 * 576];
  child_prolongations(pk);
  for (int k = 0; k < 8; ++k) ptmp(pk + 576 * k, ke, mcat + 576 * k);
  for (int k = 0; k < 8; ++k)
    for (int q = 0; q < 8; ++q) ptmp(pk + 576 * k, mcat + 576 * q, nkq + 576 * (8 * k + q));
  return LP_OK;
}

// node field (3, NX, NY, NZ) in grid order <-> the device layout (3, pz/4, NY, NX, 4) (host arrays;
// the padding is written as zeros / skipped)
int lpb_layout_nodes_f64(const double* grid, double* out, int nx, int ny, int nz) {
  if (!grid || !out || nx < 1 || ny < 1 || nz < 1) return LP_ERR_ARG;
  const HGrid g = mkgrid(nx, ny, nz);
  const LpGrid lg = lp_grid(nx, ny, nz, g.pz, g.cpz);
  std::memset(out, 0, sizeof(double) * g.nnode());
  for (int c = 0; c < 3; ++c)
    for (int x = 0; x < g.NX(); ++x)
      for (int y = 0; y < g.NY(); ++y)
        for (int z = 0; z < g.NZ(); ++z)
          out[c * lg.comp_stride() + lg.node(x, y, z)] = grid[(((long long)c * g.NX() + x) * g.NY() + y) * g.NZ() + z];
  return LP_OK;
}

int lpb_unlayout_nodes_f64(const double* dev_layout, double* grid, int nx, int ny, int nz) {
  if (!grid || !dev_layout || nx < 1 || ny < 1 || nz < 1) return LP_ERR_ARG;
  const HGrid g = mkgrid(nx, ny, nz);
  const LpGrid lg = lp_grid(nx, ny, nz, g.pz, g.cpz);
  for (int c = 0; c < 3; ++c)
    for (int x = 0; x < g.NX(); ++x)
      for (int y = 0; y < g.NY(); ++y)
        for (int z = 0; z < g.NZ(); ++z)
          grid[(((long long)c * g.NX() + x) * g.NY() + y) * g.NZ() + z] = dev_layout[c * lg.comp_stride() + lg.node(x, y, z)];
  return LP_OK;
}

// cell field (nx, ny, nz) in grid order -> the device layout (cpz/4, ny, nx, 4), zero padding
int lpb_layout_cells_f64(const double* grid, double* out, int nx, int ny, int nz) {
  if (!grid || !out || nx < 1 || ny < 1 || nz < 1) return LP_ERR_ARG;
  const HGrid g = mkgrid(nx, ny, nz);
  const LpGrid lg = lp_grid(nx, ny, nz, g.pz, g.cpz);
  std::memset(out, 0, sizeof(double) * g.ncell());
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) out[lg.cell(x, y, z)] = grid[((long long)x * ny + y) * nz + z];
  return LP_OK;
}

// sizes of the device layout for nx x ny x nz cells: out = {pz, cpz, node field entries, cell
// field entries, mask entries}
int lpb_layout_dims(int nx, int ny, int nz, long long* out) {
  if (!out || nx < 1 || ny < 1 || nz < 1) return LP_ERR_ARG;
  const HGrid g = mkgrid(nx, ny, nz);
  out[0] = g.pz;
  out[1] = g.cpz;
  out[2] = g.nnode();
  out[3] = g.ncell();
  out[4] = g.nmask();
  return LP_OK;
}

void* lpb_mg_create(int nx, int ny, int nz, const uint8_t* fixed, const double* ke, int single, double rtol, int maxiter,
                    long long coarse_cells, int* status) {
  auto fail = [&](int code) -> void* {
    if (status) *status = code;
    return nullptr;
  };
  if (nx < 2 || ny < 2 || nz < 2 || (nx | ny | nz) & 1 || !fixed || !ke || !(rtol > 0.0) || maxiter < 1 ||
      coarse_cells < 1)
    return fail(LP_ERR_ARG);
  Mg* m = new Mg();
  m->g0 = mkgrid(nx, ny, nz);
  m->f32 = single != 0;
  m->rtol = rtol;
  m->maxiter = maxiter;
  m->coarse_cells = coarse_cells;
  std::memcpy(m->ke, ke, sizeof(m->ke));
  if (lpb_modal_ke(m->ke, m->kmodal) != 45 || lpb_modal_g1(m->ke, m->g1) != 279) {
    delete m;
    return fail(LP_ERR_ARG);
  }
  m->mcat_h.resize(8 * 576);
  m->nkq_h.resize(64 * 576);
  lpb_level1_products(m->ke, m->mcat_h.data(), m->nkq_h.data());
  if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost((void**)&m->host, 8 * sizeof(double)) != cudaSuccess) {
    delete m;
    return fail(LP_ERR_LAUNCH);
  }
  const HGrid& g = m->g0;
  // the held dofs as bits per node in the device layout (bit c = component c)
  std::vector<uint8_t> bits(g.nmask(), 0);
  const LpGrid lg = lp_grid(g.nx, g.ny, g.nz, g.pz, g.cpz);
  for (int x = 0; x < g.NX(); ++x)
    for (int y = 0; y < g.NY(); ++y)
      for (int z = 0; z < g.NZ(); ++z) bits[lg.node(x, y, z)] = fixed[((long long)x * g.NY() + y) * g.NZ() + z] & 7;
  m->fixed_bits = (uint8_t*)m->buf("fixed_bits", g.nmask());
  cudaMemcpyAsync(m->fixed_bits, bits.data(), g.nmask(), cudaMemcpyHostToDevice, m->st);
  m->ke64 = (double*)m->buf("ke64", 8 * 576);
  cudaMemcpyAsync(m->ke64, m->ke, 8 * 576, cudaMemcpyHostToDevice, m->st);
  std::vector<float> mc(m->mcat_h.begin(), m->mcat_h.end()), nk(m->nkq_h.begin(), m->nkq_h.end());
  if (m->f32) {
    m->mcat_d = m->buf("mcat", 4 * mc.size());
    m->nkq_d = m->buf("nkq", 4 * nk.size());
    cudaMemcpyAsync(m->mcat_d, mc.data(), 4 * mc.size(), cudaMemcpyHostToDevice, m->st);
    cudaMemcpyAsync(m->nkq_d, nk.data(), 4 * nk.size(), cudaMemcpyHostToDevice, m->st);
  } else {
    m->mcat_d = m->buf("mcat", 8 * m->mcat_h.size());
    m->nkq_d = m->buf("nkq", 8 * m->nkq_h.size());
    cudaMemcpyAsync(m->mcat_d, m->mcat_h.data(), 8 * m->mcat_h.size(), cudaMemcpyHostToDevice, m->st);
    cudaMemcpyAsync(m->nkq_d, m->nkq_h.data(), 8 * m->nkq_h.size(), cudaMemcpyHostToDevice, m->st);
  }
  m->err = (int*)m->buf("err", 4);
  const long long fine_blocks = ((g.NX() + 14) / 15) * (long long)((g.NY() + 14) / 15) * (g.pz / 4);
  m->part_len = std::max(std::max(2LL * lpb_reduce_blocks(), 2048LL), fine_blocks);
  m->part = (double*)m->buf("part", 8 * (size_t)m->part_len);
  m->scal = (double*)m->buf("scal", 8 * 64);
  m->chk = (double*)m->buf("chk", 8 * 64);
  m->pw = (double*)m->buf("pw", 8 * 32 * 32);
  m->coef = (double*)m->buf("coef", 8 * 16 * 32);
  m->e0 = (double*)m->buf("e0_64", 8 * g.ncell());
  cudaStreamSynchronize(m->st);   // the host arrays above are released on return
  if (m->status != LP_OK) {
    const int code = m->status;
    delete m;
    return fail(code);
  }
  if (status) *status = LP_OK;
  return m;
}

// e: the fine level's moduli, float64 device cell field in the layout (lpb_layout_cells_f64)
int lpb_mg_set_moduli(void* h, const double* e, void* stream) {
  Mg* m = static_cast<Mg*>(h);
  if (!m || !e) return LP_ERR_ARG;
  m->status = LP_OK;
  cudaEvent_t ev;   // the caller's stream's work on e comes first
  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEventRecord(ev, (cudaStream_t)stream);
  cudaStreamWaitEvent(m->st, ev, 0);
  cudaEventDestroy(ev);
  cudaMemcpyAsync(m->e0, e, 8 * m->g0.ncell(), cudaMemcpyDeviceToDevice, m->st);
  set_moduli(*m);
  cudaStreamSynchronize(m->st);
  return m->status;
}

// x = A^-1 b (float64 device node fields in the layout; x0 may be null): masked b and x0, the
// strict fallback when the plain hierarchy stalls (loadpath/mg.py:951-965). *iters: the CG
// iterations. Returns 0, 1 when CG did not converge, or < 0 on an error.
int lpb_mg_solve(void* h, const double* b, const double* x0, double* x, int* iters, void* stream) {
  Mg* m = static_cast<Mg*>(h);
  if (!m || !b || !x || m->levels.empty()) return LP_ERR_ARG;
  m->status = LP_OK;
  const HGrid& g = m->g0;
  cudaEvent_t ev;
  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEventRecord(ev, (cudaStream_t)stream);
  cudaStreamWaitEvent(m->st, ev, 0);
  double* bm = (double*)m->field("cg_b", g, false);
  m->ok(lpb_mask_field_f64(bm, b, m->levels[0].mask, HG(g), 0, m->st));
  double* x0m = nullptr;
  if (x0) {
    x0m = (double*)m->field("solve_x0", g, false);
    m->ok(lpb_mask_field_f64(x0m, x0, m->levels[0].mask, HG(g), 0, m->st));
  }
  int it = 0;
  bool ok = false;
  double* xs;
  if (m->strict || m->levels.size() < 2) {
    xs = pcg(*m, x0m, it, ok);
  } else {
    const int full = m->maxiter;
    m->maxiter = std::min(full, STALL);
    xs = pcg(*m, x0m, it, ok);
    m->maxiter = full;
    if (!ok && m->status == LP_OK) {
      m->strict = true;
      set_moduli(*m);
      int it2 = 0;
      // the strict build does not touch cg_b: the masked right-hand side is still there
      xs = pcg(*m, x0m, it2, ok);
      it += it2;
    }
  }
  m->last_iters = it;
  if (iters) *iters = it;
  int errflag = 0;
  cudaMemcpyAsync(&errflag, m->err, 4, cudaMemcpyDeviceToHost, m->st);
  m->ok(lpb_mask_field_f64(x, xs, m->levels[0].mask, HG(g), 0, m->st));
  cudaEventRecord(ev, m->st);
  cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
  cudaStreamSynchronize(m->st);
  cudaEventDestroy(ev);
  if (errflag) return LP_ERR_LAUNCH;
  if (m->status != LP_OK) return m->status;
  return ok ? LP_OK : 1;
}

// the hierarchy's depth and strictness after the last set_moduli / solve
int lpb_mg_levels(void* h) { return h ? (int)static_cast<Mg*>(h)->levels.size() : LP_ERR_ARG; }
int lpb_mg_strict(void* h) { return h ? (int)static_cast<Mg*>(h)->strict : LP_ERR_ARG; }

void lpb_mg_destroy(void* h) {
  Mg* m = static_cast<Mg*>(h);
  if (!m) return;
  if (m->st) {
    cudaStreamSynchronize(m->st);
    cudaStreamDestroy(m->st);
    m->st = nullptr;
  }
  delete m;
}

}  // extern "C"
