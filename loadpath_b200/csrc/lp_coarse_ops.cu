// Coarse-level operators on the solver's hot path (loadpath/mg.py:174-346 for the level kinds,
// loadpath/mgops.py:106-146 for the products they replace).
//
// Level 1 ("weights"): K_c = sum_k w[k, c] M_k with M_k = P_k^T Ke P_k, the reference's first
// Galerkin level. With the child moduli's Walsh transform c = H w, sum_k w_k M_k =
// sum_t c_t G_t, G_t = sum_k H[t, k] M_k / 8, and in the corner-parity basis of the coarse cell
// the eight G_t together have 279 non-zeros, each (row, col) entry belonging to exactly one t.
// The kernel marches z like the fine kernel (four cells per step, x neighbours by shuffles, y
// neighbours through shared memory) and forms each cell's product in that basis: ~450 flops
// against the 4608 of the dense sum. Cells touching held dofs ("patch" cells: weights zero,
// an explicit masked matrix instead) are added by a second, node-centric pass over the box of
// nodes they touch.
//
// Levels >= 2 ("explicit"): K_c stored per cell, symmetric, as the 300 upper-triangle entries
// in entry-major order (entry p of consecutive cells contiguous, so a warp's loads coalesce).
// Two passes: a cell pass forms the 24 corner forces f_c = K_c u_c into a caller-provided
// (24, cells) buffer, a node pass sums each node's eight cells' rows and applies the mask.
#include <cstring>

#include "lp_common.cuh"
#include "lp_tma.cuh"

#include <mutex>

namespace {

constexpr int TXC = 16, TYC = 16;

template <typename T>
struct G1 {
  T c[279];
};

// f = sum_t c_t G^_t v on the corner-parity modes (index 3 * mode + component)
template <typename T>
__device__ __forceinline__ void g1_product(const G1<T>& g, const T (&c)[8], const T (&v)[24], T (&f)[24]) {
  f[0] = f[1] = f[2] = T(0);
  f[3] = c[0] * (g.c[0] * v[3] + g.c[1] * v[7] + g.c[2] * v[14])
         + c[1] * (g.c[3] * v[10] + g.c[4] * v[17])
         + c[2] * (g.c[5] * v[9] + g.c[6] * v[20])
         + c[3] * (g.c[7] * v[23])
         + c[4] * (g.c[8] * v[15] + g.c[9] * v[19])
         + c[5] * (g.c[10] * v[22])
         + c[6] * (g.c[11] * v[21]);
  f[4] = c[0] * (g.c[12] * v[4] + g.c[13] * v[6])
         + c[1] * (g.c[14] * v[9])
         + c[2] * (g.c[15] * v[10])
         + c[4] * (g.c[16] * v[16] + g.c[17] * v[18])
         + c[5] * (g.c[18] * v[21])
         + c[6] * (g.c[19] * v[22]);
  f[5] = c[0] * (g.c[20] * v[5] + g.c[21] * v[12])
         + c[1] * (g.c[22] * v[15])
         + c[2] * (g.c[23] * v[11] + g.c[24] * v[18])
         + c[3] * (g.c[25] * v[21])
         + c[4] * (g.c[26] * v[17])
         + c[6] * (g.c[27] * v[23]);
  f[6] = c[0] * (g.c[28] * v[4] + g.c[29] * v[6])
         + c[1] * (g.c[30] * v[9])
         + c[2] * (g.c[31] * v[10])
         + c[4] * (g.c[32] * v[16] + g.c[33] * v[18])
         + c[5] * (g.c[34] * v[21])
         + c[6] * (g.c[35] * v[22]);
  f[7] = c[0] * (g.c[36] * v[3] + g.c[37] * v[7] + g.c[38] * v[14])
         + c[1] * (g.c[39] * v[10] + g.c[40] * v[17])
         + c[2] * (g.c[41] * v[9] + g.c[42] * v[20])
         + c[3] * (g.c[43] * v[23])
         + c[4] * (g.c[44] * v[15] + g.c[45] * v[19])
         + c[5] * (g.c[46] * v[22])
         + c[6] * (g.c[47] * v[21]);
  f[8] = c[0] * (g.c[48] * v[8] + g.c[49] * v[13])
         + c[1] * (g.c[50] * v[11] + g.c[51] * v[16])
         + c[2] * (g.c[52] * v[19])
         + c[3] * (g.c[53] * v[22])
         + c[4] * (g.c[54] * v[20])
         + c[5] * (g.c[55] * v[23]);
  f[9] = c[0] * (g.c[56] * v[9] + g.c[57] * v[20])
         + c[1] * (g.c[58] * v[4] + g.c[59] * v[6] + g.c[60] * v[23])
         + c[2] * (g.c[61] * v[3] + g.c[62] * v[7] + g.c[63] * v[14])
         + c[3] * (g.c[64] * v[10] + g.c[65] * v[17])
         + c[4] * (g.c[66] * v[21])
         + c[5] * (g.c[67] * v[16] + g.c[68] * v[18])
         + c[6] * (g.c[69] * v[15] + g.c[70] * v[19])
         + c[7] * (g.c[71] * v[22]);
  f[10] = c[0] * (g.c[72] * v[10] + g.c[73] * v[17])
         + c[1] * (g.c[74] * v[3] + g.c[75] * v[7] + g.c[76] * v[14])
         + c[2] * (g.c[77] * v[4] + g.c[78] * v[6] + g.c[79] * v[23])
         + c[3] * (g.c[80] * v[9] + g.c[81] * v[20])
         + c[4] * (g.c[82] * v[22])
         + c[5] * (g.c[83] * v[15] + g.c[84] * v[19])
         + c[6] * (g.c[85] * v[16] + g.c[86] * v[18])
         + c[7] * (g.c[87] * v[21]);
  f[11] = c[0] * (g.c[88] * v[11] + g.c[89] * v[16] + g.c[90] * v[18])
         + c[1] * (g.c[91] * v[8] + g.c[92] * v[13] + g.c[93] * v[21])
         + c[2] * (g.c[94] * v[5] + g.c[95] * v[12] + g.c[96] * v[22])
         + c[3] * (g.c[97] * v[15] + g.c[98] * v[19])
         + c[4] * (g.c[99] * v[23])
         + c[5] * (g.c[100] * v[20])
         + c[6] * (g.c[101] * v[17]);
  f[12] = c[0] * (g.c[102] * v[5] + g.c[103] * v[12])
         + c[1] * (g.c[104] * v[15])
         + c[2] * (g.c[105] * v[11] + g.c[106] * v[18])
         + c[3] * (g.c[107] * v[21])
         + c[4] * (g.c[108] * v[17])
         + c[6] * (g.c[109] * v[23]);
  f[13] = c[0] * (g.c[110] * v[8] + g.c[111] * v[13])
         + c[1] * (g.c[112] * v[11] + g.c[113] * v[16])
         + c[2] * (g.c[114] * v[19])
         + c[3] * (g.c[115] * v[22])
         + c[4] * (g.c[116] * v[20])
         + c[5] * (g.c[117] * v[23]);
  f[14] = c[0] * (g.c[118] * v[3] + g.c[119] * v[7] + g.c[120] * v[14])
         + c[1] * (g.c[121] * v[10] + g.c[122] * v[17])
         + c[2] * (g.c[123] * v[9] + g.c[124] * v[20])
         + c[3] * (g.c[125] * v[23])
         + c[4] * (g.c[126] * v[15] + g.c[127] * v[19])
         + c[5] * (g.c[128] * v[22])
         + c[6] * (g.c[129] * v[21]);
  f[15] = c[0] * (g.c[130] * v[15] + g.c[131] * v[19])
         + c[1] * (g.c[132] * v[5] + g.c[133] * v[12] + g.c[134] * v[22])
         + c[2] * (g.c[135] * v[21])
         + c[3] * (g.c[136] * v[11] + g.c[137] * v[18])
         + c[4] * (g.c[138] * v[3] + g.c[139] * v[7] + g.c[140] * v[14])
         + c[5] * (g.c[141] * v[10] + g.c[142] * v[17])
         + c[6] * (g.c[143] * v[9] + g.c[144] * v[20])
         + c[7] * (g.c[145] * v[23]);
  f[16] = c[0] * (g.c[146] * v[11] + g.c[147] * v[16] + g.c[148] * v[18])
         + c[1] * (g.c[149] * v[8] + g.c[150] * v[13] + g.c[151] * v[21])
         + c[2] * (g.c[152] * v[22])
         + c[3] * (g.c[153] * v[19])
         + c[4] * (g.c[154] * v[4] + g.c[155] * v[6] + g.c[156] * v[23])
         + c[5] * (g.c[157] * v[9] + g.c[158] * v[20])
         + c[6] * (g.c[159] * v[10]);
  f[17] = c[0] * (g.c[160] * v[10] + g.c[161] * v[17])
         + c[1] * (g.c[162] * v[3] + g.c[163] * v[7] + g.c[164] * v[14])
         + c[2] * (g.c[165] * v[23])
         + c[3] * (g.c[166] * v[9] + g.c[167] * v[20])
         + c[4] * (g.c[168] * v[5] + g.c[169] * v[12] + g.c[170] * v[22])
         + c[5] * (g.c[171] * v[15] + g.c[172] * v[19])
         + c[6] * (g.c[173] * v[11] + g.c[174] * v[18])
         + c[7] * (g.c[175] * v[21]);
  f[18] = c[0] * (g.c[176] * v[11] + g.c[177] * v[16] + g.c[178] * v[18])
         + c[1] * (g.c[179] * v[21])
         + c[2] * (g.c[180] * v[5] + g.c[181] * v[12] + g.c[182] * v[22])
         + c[3] * (g.c[183] * v[15])
         + c[4] * (g.c[184] * v[4] + g.c[185] * v[6] + g.c[186] * v[23])
         + c[5] * (g.c[187] * v[9])
         + c[6] * (g.c[188] * v[10] + g.c[189] * v[17]);
  f[19] = c[0] * (g.c[190] * v[15] + g.c[191] * v[19])
         + c[1] * (g.c[192] * v[22])
         + c[2] * (g.c[193] * v[8] + g.c[194] * v[13] + g.c[195] * v[21])
         + c[3] * (g.c[196] * v[11] + g.c[197] * v[16])
         + c[4] * (g.c[198] * v[3] + g.c[199] * v[7] + g.c[200] * v[14])
         + c[5] * (g.c[201] * v[10] + g.c[202] * v[17])
         + c[6] * (g.c[203] * v[9] + g.c[204] * v[20])
         + c[7] * (g.c[205] * v[23]);
  f[20] = c[0] * (g.c[206] * v[9] + g.c[207] * v[20])
         + c[1] * (g.c[208] * v[23])
         + c[2] * (g.c[209] * v[3] + g.c[210] * v[7] + g.c[211] * v[14])
         + c[3] * (g.c[212] * v[10] + g.c[213] * v[17])
         + c[4] * (g.c[214] * v[8] + g.c[215] * v[13] + g.c[216] * v[21])
         + c[5] * (g.c[217] * v[11] + g.c[218] * v[16])
         + c[6] * (g.c[219] * v[15] + g.c[220] * v[19])
         + c[7] * (g.c[221] * v[22]);
  f[21] = c[0] * (g.c[222] * v[21])
         + c[1] * (g.c[223] * v[11] + g.c[224] * v[16] + g.c[225] * v[18])
         + c[2] * (g.c[226] * v[15] + g.c[227] * v[19])
         + c[3] * (g.c[228] * v[5] + g.c[229] * v[12] + g.c[230] * v[22])
         + c[4] * (g.c[231] * v[9] + g.c[232] * v[20])
         + c[5] * (g.c[233] * v[4] + g.c[234] * v[6] + g.c[235] * v[23])
         + c[6] * (g.c[236] * v[3] + g.c[237] * v[7] + g.c[238] * v[14])
         + c[7] * (g.c[239] * v[10] + g.c[240] * v[17]);
  f[22] = c[0] * (g.c[241] * v[22])
         + c[1] * (g.c[242] * v[15] + g.c[243] * v[19])
         + c[2] * (g.c[244] * v[11] + g.c[245] * v[16] + g.c[246] * v[18])
         + c[3] * (g.c[247] * v[8] + g.c[248] * v[13] + g.c[249] * v[21])
         + c[4] * (g.c[250] * v[10] + g.c[251] * v[17])
         + c[5] * (g.c[252] * v[3] + g.c[253] * v[7] + g.c[254] * v[14])
         + c[6] * (g.c[255] * v[4] + g.c[256] * v[6] + g.c[257] * v[23])
         + c[7] * (g.c[258] * v[9] + g.c[259] * v[20]);
  f[23] = c[0] * (g.c[260] * v[23])
         + c[1] * (g.c[261] * v[9] + g.c[262] * v[20])
         + c[2] * (g.c[263] * v[10] + g.c[264] * v[17])
         + c[3] * (g.c[265] * v[3] + g.c[266] * v[7] + g.c[267] * v[14])
         + c[4] * (g.c[268] * v[11] + g.c[269] * v[16] + g.c[270] * v[18])
         + c[5] * (g.c[271] * v[8] + g.c[272] * v[13] + g.c[273] * v[21])
         + c[6] * (g.c[274] * v[5] + g.c[275] * v[12] + g.c[276] * v[22])
         + c[7] * (g.c[277] * v[15] + g.c[278] * v[19]);
}

// row r of the level-1 modal product (the rows g1_product forms together), so a caller can
// consume each row as it is produced
template <int R, typename T>
__device__ __forceinline__ T g1_row(const G1<T>& g, const T (&c)[8], const T (&v)[24]);
template <>
__device__ __forceinline__ float g1_row<0, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return 0.0f;
}
template <>
__device__ __forceinline__ double g1_row<0, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return 0.0;
}
template <>
__device__ __forceinline__ float g1_row<1, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return 0.0f;
}
template <>
__device__ __forceinline__ double g1_row<1, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return 0.0;
}
template <>
__device__ __forceinline__ float g1_row<2, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return 0.0f;
}
template <>
__device__ __forceinline__ double g1_row<2, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return 0.0;
}
template <>
__device__ __forceinline__ float g1_row<3, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[0] * v[3] + g.c[1] * v[7] + g.c[2] * v[14]) + c[1] * (g.c[3] * v[10] + g.c[4] * v[17]) + c[2] * (g.c[5] * v[9] + g.c[6] * v[20]) + c[3] * (g.c[7] * v[23]) + c[4] * (g.c[8] * v[15] + g.c[9] * v[19]) + c[5] * (g.c[10] * v[22]) + c[6] * (g.c[11] * v[21]);
}
template <>
__device__ __forceinline__ double g1_row<3, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[0] * v[3] + g.c[1] * v[7] + g.c[2] * v[14]) + c[1] * (g.c[3] * v[10] + g.c[4] * v[17]) + c[2] * (g.c[5] * v[9] + g.c[6] * v[20]) + c[3] * (g.c[7] * v[23]) + c[4] * (g.c[8] * v[15] + g.c[9] * v[19]) + c[5] * (g.c[10] * v[22]) + c[6] * (g.c[11] * v[21]);
}
template <>
__device__ __forceinline__ float g1_row<4, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[12] * v[4] + g.c[13] * v[6]) + c[1] * (g.c[14] * v[9]) + c[2] * (g.c[15] * v[10]) + c[4] * (g.c[16] * v[16] + g.c[17] * v[18]) + c[5] * (g.c[18] * v[21]) + c[6] * (g.c[19] * v[22]);
}
template <>
__device__ __forceinline__ double g1_row<4, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[12] * v[4] + g.c[13] * v[6]) + c[1] * (g.c[14] * v[9]) + c[2] * (g.c[15] * v[10]) + c[4] * (g.c[16] * v[16] + g.c[17] * v[18]) + c[5] * (g.c[18] * v[21]) + c[6] * (g.c[19] * v[22]);
}
template <>
__device__ __forceinline__ float g1_row<5, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[20] * v[5] + g.c[21] * v[12]) + c[1] * (g.c[22] * v[15]) + c[2] * (g.c[23] * v[11] + g.c[24] * v[18]) + c[3] * (g.c[25] * v[21]) + c[4] * (g.c[26] * v[17]) + c[6] * (g.c[27] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<5, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[20] * v[5] + g.c[21] * v[12]) + c[1] * (g.c[22] * v[15]) + c[2] * (g.c[23] * v[11] + g.c[24] * v[18]) + c[3] * (g.c[25] * v[21]) + c[4] * (g.c[26] * v[17]) + c[6] * (g.c[27] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<6, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[28] * v[4] + g.c[29] * v[6]) + c[1] * (g.c[30] * v[9]) + c[2] * (g.c[31] * v[10]) + c[4] * (g.c[32] * v[16] + g.c[33] * v[18]) + c[5] * (g.c[34] * v[21]) + c[6] * (g.c[35] * v[22]);
}
template <>
__device__ __forceinline__ double g1_row<6, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[28] * v[4] + g.c[29] * v[6]) + c[1] * (g.c[30] * v[9]) + c[2] * (g.c[31] * v[10]) + c[4] * (g.c[32] * v[16] + g.c[33] * v[18]) + c[5] * (g.c[34] * v[21]) + c[6] * (g.c[35] * v[22]);
}
template <>
__device__ __forceinline__ float g1_row<7, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[36] * v[3] + g.c[37] * v[7] + g.c[38] * v[14]) + c[1] * (g.c[39] * v[10] + g.c[40] * v[17]) + c[2] * (g.c[41] * v[9] + g.c[42] * v[20]) + c[3] * (g.c[43] * v[23]) + c[4] * (g.c[44] * v[15] + g.c[45] * v[19]) + c[5] * (g.c[46] * v[22]) + c[6] * (g.c[47] * v[21]);
}
template <>
__device__ __forceinline__ double g1_row<7, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[36] * v[3] + g.c[37] * v[7] + g.c[38] * v[14]) + c[1] * (g.c[39] * v[10] + g.c[40] * v[17]) + c[2] * (g.c[41] * v[9] + g.c[42] * v[20]) + c[3] * (g.c[43] * v[23]) + c[4] * (g.c[44] * v[15] + g.c[45] * v[19]) + c[5] * (g.c[46] * v[22]) + c[6] * (g.c[47] * v[21]);
}
template <>
__device__ __forceinline__ float g1_row<8, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[48] * v[8] + g.c[49] * v[13]) + c[1] * (g.c[50] * v[11] + g.c[51] * v[16]) + c[2] * (g.c[52] * v[19]) + c[3] * (g.c[53] * v[22]) + c[4] * (g.c[54] * v[20]) + c[5] * (g.c[55] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<8, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[48] * v[8] + g.c[49] * v[13]) + c[1] * (g.c[50] * v[11] + g.c[51] * v[16]) + c[2] * (g.c[52] * v[19]) + c[3] * (g.c[53] * v[22]) + c[4] * (g.c[54] * v[20]) + c[5] * (g.c[55] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<9, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[56] * v[9] + g.c[57] * v[20]) + c[1] * (g.c[58] * v[4] + g.c[59] * v[6] + g.c[60] * v[23]) + c[2] * (g.c[61] * v[3] + g.c[62] * v[7] + g.c[63] * v[14]) + c[3] * (g.c[64] * v[10] + g.c[65] * v[17]) + c[4] * (g.c[66] * v[21]) + c[5] * (g.c[67] * v[16] + g.c[68] * v[18]) + c[6] * (g.c[69] * v[15] + g.c[70] * v[19]) + c[7] * (g.c[71] * v[22]);
}
template <>
__device__ __forceinline__ double g1_row<9, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[56] * v[9] + g.c[57] * v[20]) + c[1] * (g.c[58] * v[4] + g.c[59] * v[6] + g.c[60] * v[23]) + c[2] * (g.c[61] * v[3] + g.c[62] * v[7] + g.c[63] * v[14]) + c[3] * (g.c[64] * v[10] + g.c[65] * v[17]) + c[4] * (g.c[66] * v[21]) + c[5] * (g.c[67] * v[16] + g.c[68] * v[18]) + c[6] * (g.c[69] * v[15] + g.c[70] * v[19]) + c[7] * (g.c[71] * v[22]);
}
template <>
__device__ __forceinline__ float g1_row<10, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[72] * v[10] + g.c[73] * v[17]) + c[1] * (g.c[74] * v[3] + g.c[75] * v[7] + g.c[76] * v[14]) + c[2] * (g.c[77] * v[4] + g.c[78] * v[6] + g.c[79] * v[23]) + c[3] * (g.c[80] * v[9] + g.c[81] * v[20]) + c[4] * (g.c[82] * v[22]) + c[5] * (g.c[83] * v[15] + g.c[84] * v[19]) + c[6] * (g.c[85] * v[16] + g.c[86] * v[18]) + c[7] * (g.c[87] * v[21]);
}
template <>
__device__ __forceinline__ double g1_row<10, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[72] * v[10] + g.c[73] * v[17]) + c[1] * (g.c[74] * v[3] + g.c[75] * v[7] + g.c[76] * v[14]) + c[2] * (g.c[77] * v[4] + g.c[78] * v[6] + g.c[79] * v[23]) + c[3] * (g.c[80] * v[9] + g.c[81] * v[20]) + c[4] * (g.c[82] * v[22]) + c[5] * (g.c[83] * v[15] + g.c[84] * v[19]) + c[6] * (g.c[85] * v[16] + g.c[86] * v[18]) + c[7] * (g.c[87] * v[21]);
}
template <>
__device__ __forceinline__ float g1_row<11, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[88] * v[11] + g.c[89] * v[16] + g.c[90] * v[18]) + c[1] * (g.c[91] * v[8] + g.c[92] * v[13] + g.c[93] * v[21]) + c[2] * (g.c[94] * v[5] + g.c[95] * v[12] + g.c[96] * v[22]) + c[3] * (g.c[97] * v[15] + g.c[98] * v[19]) + c[4] * (g.c[99] * v[23]) + c[5] * (g.c[100] * v[20]) + c[6] * (g.c[101] * v[17]);
}
template <>
__device__ __forceinline__ double g1_row<11, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[88] * v[11] + g.c[89] * v[16] + g.c[90] * v[18]) + c[1] * (g.c[91] * v[8] + g.c[92] * v[13] + g.c[93] * v[21]) + c[2] * (g.c[94] * v[5] + g.c[95] * v[12] + g.c[96] * v[22]) + c[3] * (g.c[97] * v[15] + g.c[98] * v[19]) + c[4] * (g.c[99] * v[23]) + c[5] * (g.c[100] * v[20]) + c[6] * (g.c[101] * v[17]);
}
template <>
__device__ __forceinline__ float g1_row<12, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[102] * v[5] + g.c[103] * v[12]) + c[1] * (g.c[104] * v[15]) + c[2] * (g.c[105] * v[11] + g.c[106] * v[18]) + c[3] * (g.c[107] * v[21]) + c[4] * (g.c[108] * v[17]) + c[6] * (g.c[109] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<12, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[102] * v[5] + g.c[103] * v[12]) + c[1] * (g.c[104] * v[15]) + c[2] * (g.c[105] * v[11] + g.c[106] * v[18]) + c[3] * (g.c[107] * v[21]) + c[4] * (g.c[108] * v[17]) + c[6] * (g.c[109] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<13, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[110] * v[8] + g.c[111] * v[13]) + c[1] * (g.c[112] * v[11] + g.c[113] * v[16]) + c[2] * (g.c[114] * v[19]) + c[3] * (g.c[115] * v[22]) + c[4] * (g.c[116] * v[20]) + c[5] * (g.c[117] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<13, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[110] * v[8] + g.c[111] * v[13]) + c[1] * (g.c[112] * v[11] + g.c[113] * v[16]) + c[2] * (g.c[114] * v[19]) + c[3] * (g.c[115] * v[22]) + c[4] * (g.c[116] * v[20]) + c[5] * (g.c[117] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<14, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[118] * v[3] + g.c[119] * v[7] + g.c[120] * v[14]) + c[1] * (g.c[121] * v[10] + g.c[122] * v[17]) + c[2] * (g.c[123] * v[9] + g.c[124] * v[20]) + c[3] * (g.c[125] * v[23]) + c[4] * (g.c[126] * v[15] + g.c[127] * v[19]) + c[5] * (g.c[128] * v[22]) + c[6] * (g.c[129] * v[21]);
}
template <>
__device__ __forceinline__ double g1_row<14, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[118] * v[3] + g.c[119] * v[7] + g.c[120] * v[14]) + c[1] * (g.c[121] * v[10] + g.c[122] * v[17]) + c[2] * (g.c[123] * v[9] + g.c[124] * v[20]) + c[3] * (g.c[125] * v[23]) + c[4] * (g.c[126] * v[15] + g.c[127] * v[19]) + c[5] * (g.c[128] * v[22]) + c[6] * (g.c[129] * v[21]);
}
template <>
__device__ __forceinline__ float g1_row<15, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[130] * v[15] + g.c[131] * v[19]) + c[1] * (g.c[132] * v[5] + g.c[133] * v[12] + g.c[134] * v[22]) + c[2] * (g.c[135] * v[21]) + c[3] * (g.c[136] * v[11] + g.c[137] * v[18]) + c[4] * (g.c[138] * v[3] + g.c[139] * v[7] + g.c[140] * v[14]) + c[5] * (g.c[141] * v[10] + g.c[142] * v[17]) + c[6] * (g.c[143] * v[9] + g.c[144] * v[20]) + c[7] * (g.c[145] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<15, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[130] * v[15] + g.c[131] * v[19]) + c[1] * (g.c[132] * v[5] + g.c[133] * v[12] + g.c[134] * v[22]) + c[2] * (g.c[135] * v[21]) + c[3] * (g.c[136] * v[11] + g.c[137] * v[18]) + c[4] * (g.c[138] * v[3] + g.c[139] * v[7] + g.c[140] * v[14]) + c[5] * (g.c[141] * v[10] + g.c[142] * v[17]) + c[6] * (g.c[143] * v[9] + g.c[144] * v[20]) + c[7] * (g.c[145] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<16, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[146] * v[11] + g.c[147] * v[16] + g.c[148] * v[18]) + c[1] * (g.c[149] * v[8] + g.c[150] * v[13] + g.c[151] * v[21]) + c[2] * (g.c[152] * v[22]) + c[3] * (g.c[153] * v[19]) + c[4] * (g.c[154] * v[4] + g.c[155] * v[6] + g.c[156] * v[23]) + c[5] * (g.c[157] * v[9] + g.c[158] * v[20]) + c[6] * (g.c[159] * v[10]);
}
template <>
__device__ __forceinline__ double g1_row<16, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[146] * v[11] + g.c[147] * v[16] + g.c[148] * v[18]) + c[1] * (g.c[149] * v[8] + g.c[150] * v[13] + g.c[151] * v[21]) + c[2] * (g.c[152] * v[22]) + c[3] * (g.c[153] * v[19]) + c[4] * (g.c[154] * v[4] + g.c[155] * v[6] + g.c[156] * v[23]) + c[5] * (g.c[157] * v[9] + g.c[158] * v[20]) + c[6] * (g.c[159] * v[10]);
}
template <>
__device__ __forceinline__ float g1_row<17, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[160] * v[10] + g.c[161] * v[17]) + c[1] * (g.c[162] * v[3] + g.c[163] * v[7] + g.c[164] * v[14]) + c[2] * (g.c[165] * v[23]) + c[3] * (g.c[166] * v[9] + g.c[167] * v[20]) + c[4] * (g.c[168] * v[5] + g.c[169] * v[12] + g.c[170] * v[22]) + c[5] * (g.c[171] * v[15] + g.c[172] * v[19]) + c[6] * (g.c[173] * v[11] + g.c[174] * v[18]) + c[7] * (g.c[175] * v[21]);
}
template <>
__device__ __forceinline__ double g1_row<17, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[160] * v[10] + g.c[161] * v[17]) + c[1] * (g.c[162] * v[3] + g.c[163] * v[7] + g.c[164] * v[14]) + c[2] * (g.c[165] * v[23]) + c[3] * (g.c[166] * v[9] + g.c[167] * v[20]) + c[4] * (g.c[168] * v[5] + g.c[169] * v[12] + g.c[170] * v[22]) + c[5] * (g.c[171] * v[15] + g.c[172] * v[19]) + c[6] * (g.c[173] * v[11] + g.c[174] * v[18]) + c[7] * (g.c[175] * v[21]);
}
template <>
__device__ __forceinline__ float g1_row<18, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[176] * v[11] + g.c[177] * v[16] + g.c[178] * v[18]) + c[1] * (g.c[179] * v[21]) + c[2] * (g.c[180] * v[5] + g.c[181] * v[12] + g.c[182] * v[22]) + c[3] * (g.c[183] * v[15]) + c[4] * (g.c[184] * v[4] + g.c[185] * v[6] + g.c[186] * v[23]) + c[5] * (g.c[187] * v[9]) + c[6] * (g.c[188] * v[10] + g.c[189] * v[17]);
}
template <>
__device__ __forceinline__ double g1_row<18, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[176] * v[11] + g.c[177] * v[16] + g.c[178] * v[18]) + c[1] * (g.c[179] * v[21]) + c[2] * (g.c[180] * v[5] + g.c[181] * v[12] + g.c[182] * v[22]) + c[3] * (g.c[183] * v[15]) + c[4] * (g.c[184] * v[4] + g.c[185] * v[6] + g.c[186] * v[23]) + c[5] * (g.c[187] * v[9]) + c[6] * (g.c[188] * v[10] + g.c[189] * v[17]);
}
template <>
__device__ __forceinline__ float g1_row<19, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[190] * v[15] + g.c[191] * v[19]) + c[1] * (g.c[192] * v[22]) + c[2] * (g.c[193] * v[8] + g.c[194] * v[13] + g.c[195] * v[21]) + c[3] * (g.c[196] * v[11] + g.c[197] * v[16]) + c[4] * (g.c[198] * v[3] + g.c[199] * v[7] + g.c[200] * v[14]) + c[5] * (g.c[201] * v[10] + g.c[202] * v[17]) + c[6] * (g.c[203] * v[9] + g.c[204] * v[20]) + c[7] * (g.c[205] * v[23]);
}
template <>
__device__ __forceinline__ double g1_row<19, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[190] * v[15] + g.c[191] * v[19]) + c[1] * (g.c[192] * v[22]) + c[2] * (g.c[193] * v[8] + g.c[194] * v[13] + g.c[195] * v[21]) + c[3] * (g.c[196] * v[11] + g.c[197] * v[16]) + c[4] * (g.c[198] * v[3] + g.c[199] * v[7] + g.c[200] * v[14]) + c[5] * (g.c[201] * v[10] + g.c[202] * v[17]) + c[6] * (g.c[203] * v[9] + g.c[204] * v[20]) + c[7] * (g.c[205] * v[23]);
}
template <>
__device__ __forceinline__ float g1_row<20, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[206] * v[9] + g.c[207] * v[20]) + c[1] * (g.c[208] * v[23]) + c[2] * (g.c[209] * v[3] + g.c[210] * v[7] + g.c[211] * v[14]) + c[3] * (g.c[212] * v[10] + g.c[213] * v[17]) + c[4] * (g.c[214] * v[8] + g.c[215] * v[13] + g.c[216] * v[21]) + c[5] * (g.c[217] * v[11] + g.c[218] * v[16]) + c[6] * (g.c[219] * v[15] + g.c[220] * v[19]) + c[7] * (g.c[221] * v[22]);
}
template <>
__device__ __forceinline__ double g1_row<20, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[206] * v[9] + g.c[207] * v[20]) + c[1] * (g.c[208] * v[23]) + c[2] * (g.c[209] * v[3] + g.c[210] * v[7] + g.c[211] * v[14]) + c[3] * (g.c[212] * v[10] + g.c[213] * v[17]) + c[4] * (g.c[214] * v[8] + g.c[215] * v[13] + g.c[216] * v[21]) + c[5] * (g.c[217] * v[11] + g.c[218] * v[16]) + c[6] * (g.c[219] * v[15] + g.c[220] * v[19]) + c[7] * (g.c[221] * v[22]);
}
template <>
__device__ __forceinline__ float g1_row<21, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[222] * v[21]) + c[1] * (g.c[223] * v[11] + g.c[224] * v[16] + g.c[225] * v[18]) + c[2] * (g.c[226] * v[15] + g.c[227] * v[19]) + c[3] * (g.c[228] * v[5] + g.c[229] * v[12] + g.c[230] * v[22]) + c[4] * (g.c[231] * v[9] + g.c[232] * v[20]) + c[5] * (g.c[233] * v[4] + g.c[234] * v[6] + g.c[235] * v[23]) + c[6] * (g.c[236] * v[3] + g.c[237] * v[7] + g.c[238] * v[14]) + c[7] * (g.c[239] * v[10] + g.c[240] * v[17]);
}
template <>
__device__ __forceinline__ double g1_row<21, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[222] * v[21]) + c[1] * (g.c[223] * v[11] + g.c[224] * v[16] + g.c[225] * v[18]) + c[2] * (g.c[226] * v[15] + g.c[227] * v[19]) + c[3] * (g.c[228] * v[5] + g.c[229] * v[12] + g.c[230] * v[22]) + c[4] * (g.c[231] * v[9] + g.c[232] * v[20]) + c[5] * (g.c[233] * v[4] + g.c[234] * v[6] + g.c[235] * v[23]) + c[6] * (g.c[236] * v[3] + g.c[237] * v[7] + g.c[238] * v[14]) + c[7] * (g.c[239] * v[10] + g.c[240] * v[17]);
}
template <>
__device__ __forceinline__ float g1_row<22, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[241] * v[22]) + c[1] * (g.c[242] * v[15] + g.c[243] * v[19]) + c[2] * (g.c[244] * v[11] + g.c[245] * v[16] + g.c[246] * v[18]) + c[3] * (g.c[247] * v[8] + g.c[248] * v[13] + g.c[249] * v[21]) + c[4] * (g.c[250] * v[10] + g.c[251] * v[17]) + c[5] * (g.c[252] * v[3] + g.c[253] * v[7] + g.c[254] * v[14]) + c[6] * (g.c[255] * v[4] + g.c[256] * v[6] + g.c[257] * v[23]) + c[7] * (g.c[258] * v[9] + g.c[259] * v[20]);
}
template <>
__device__ __forceinline__ double g1_row<22, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[241] * v[22]) + c[1] * (g.c[242] * v[15] + g.c[243] * v[19]) + c[2] * (g.c[244] * v[11] + g.c[245] * v[16] + g.c[246] * v[18]) + c[3] * (g.c[247] * v[8] + g.c[248] * v[13] + g.c[249] * v[21]) + c[4] * (g.c[250] * v[10] + g.c[251] * v[17]) + c[5] * (g.c[252] * v[3] + g.c[253] * v[7] + g.c[254] * v[14]) + c[6] * (g.c[255] * v[4] + g.c[256] * v[6] + g.c[257] * v[23]) + c[7] * (g.c[258] * v[9] + g.c[259] * v[20]);
}
template <>
__device__ __forceinline__ float g1_row<23, float>(const G1<float>& g, const float (&c)[8], const float (&v)[24]) {
  return c[0] * (g.c[260] * v[23]) + c[1] * (g.c[261] * v[9] + g.c[262] * v[20]) + c[2] * (g.c[263] * v[10] + g.c[264] * v[17]) + c[3] * (g.c[265] * v[3] + g.c[266] * v[7] + g.c[267] * v[14]) + c[4] * (g.c[268] * v[11] + g.c[269] * v[16] + g.c[270] * v[18]) + c[5] * (g.c[271] * v[8] + g.c[272] * v[13] + g.c[273] * v[21]) + c[6] * (g.c[274] * v[5] + g.c[275] * v[12] + g.c[276] * v[22]) + c[7] * (g.c[277] * v[15] + g.c[278] * v[19]);
}
template <>
__device__ __forceinline__ double g1_row<23, double>(const G1<double>& g, const double (&c)[8], const double (&v)[24]) {
  return c[0] * (g.c[260] * v[23]) + c[1] * (g.c[261] * v[9] + g.c[262] * v[20]) + c[2] * (g.c[263] * v[10] + g.c[264] * v[17]) + c[3] * (g.c[265] * v[3] + g.c[266] * v[7] + g.c[267] * v[14]) + c[4] * (g.c[268] * v[11] + g.c[269] * v[16] + g.c[270] * v[18]) + c[5] * (g.c[271] * v[8] + g.c[272] * v[13] + g.c[273] * v[21]) + c[6] * (g.c[274] * v[5] + g.c[275] * v[12] + g.c[276] * v[22]) + c[7] * (g.c[277] * v[15] + g.c[278] * v[19]);
}

// modes 1, s (per axis) of a pair: (a, b) -> (a + b, b - a)
template <typename T>
__device__ __forceinline__ void fwht8(const T (&w)[8], T (&c)[8]) {
  T a[8], b[8];
#pragma unroll
  for (int k = 0; k < 8; k += 2) { a[k] = w[k] + w[k + 1]; a[k + 1] = w[k + 1] - w[k]; }
#pragma unroll
  for (int k = 0; k < 8; k += 4) {
    b[k] = a[k] + a[k + 2]; b[k + 2] = a[k + 2] - a[k];
    b[k + 1] = a[k + 1] + a[k + 3]; b[k + 3] = a[k + 3] - a[k + 1];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) { c[k] = b[k] + b[k + 4]; c[k + 4] = b[k + 4] - b[k]; }
}

template <typename T>
__device__ __forceinline__ void xy4(T u00, T u10, T u01, T u11, T (&a)[4]) {
  T sx0 = u00 + u10, dx0 = u10 - u00, sx1 = u01 + u11, dx1 = u11 - u01;
  a[0] = sx0 + sx1;
  a[1] = dx0 + dx1;
  a[2] = sx1 - sx0;
  a[3] = dx1 - dx0;
}

// ---- level 1, TMA-staged march -------------------------------------------------------------
// The chunked Walsh layout: c = H w per cell (the coefficients of the eight G_t), stored
// (cpz / 4, ny, nx, 4, 8) so one cell column's four cells of a z chunk are 128 contiguous bytes
// (float32), each cell's eight coefficients 32 of them, and a row of x columns is one run.
// Formed once per hierarchy (after the patch cells' weights are zeroed).
template <typename T>
__global__ void k_walsh_chunks(T* __restrict__ wc, const T* __restrict__ w, LpGrid g) {
  const long long ncp = g.cells_padded();
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncp; c += (long long)gridDim.x * blockDim.x) {
    T wk[8], cw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) wk[k] = w[k * ncp + c];
    fwht8(wk, cw);
    T* dst = wc + (c >> 2) * 32 + (c & 3) * 8;
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[k] = cw[k];
  }
}

constexpr int WSTAGE = 3;
constexpr int WBOX = TXC + 1;

template <typename T, int N>
struct alignas(128) WSlot {
  T v[(N * sizeof(T) + 127) / 128 * 128 / sizeof(T)];
};

// float32: the Walsh coefficients of the block's 16 x 16 cell columns arrive by TMA with the
// node values, one 128-byte row per column in the 128-byte swizzle (a warp's 16-byte reads of
// eight consecutive rows then meet no bank twice); float64 reads them from global memory
template <typename T>
struct WCoef {
  static constexpr int N = sizeof(T) == 4 ? 32 * TXC * TYC : 32;
};

template <typename T>
struct WSmem {
  alignas(1024) T w[WSTAGE][WCoef<T>::N];            // Walsh coefficients [y][x][cell][t] (float32)
  WSlot<T, 3 * WBOX * WBOX * 4> u[WSTAGE];            // node values [comp][y][x][z]
  WSlot<T, 3 * (TXC - 1) * (TYC - 1) * 4> o[2];       // outputs staged for the TMA store [comp][y][x][z]
  T red[3][4][TXC * TYC];                             // corners 01 + 11 (to y + 1)
  T own[3][4][TXC * TYC];                             // corners 00 + 10 with the -x neighbour's
  alignas(8) uint64_t full[WSTAGE];
};

template <typename T>
struct WMaps {
  CUtensorMap u;    // (4 NX, NY, pz / 4, 3), box (4 * 17, 17, 1, 3)
  CUtensorMap out;  // (4 NX, NY, pz / 4, 3), box (4 * 15, 15, 1, 3)
  CUtensorMap w;    // float32 Walsh coefficients (32, nx, ny, cpz / 4), box (32, 16, 16, 1), 128-byte swizzle
};

// node-plane forces of one cell: rows (3q + cc, 3(q + 4) + cc) of the modal product give the
// lower face (f0 - f1) and upper face (f0 + f1) of mode (q, cc); fp = carry + lower face and the
// upper face becomes the next carry, row pair by row pair
template <int Q, int CC, typename T>
__device__ __forceinline__ void fold_pair(const G1<T>& g, const T (&c)[8], const T (&v)[24], T (&fp)[4][3],
                                          T (&up)[4][3]) {
  const T f0 = g1_row<3 * Q + CC, T>(g, c, v), f1 = g1_row<3 * (Q + 4) + CC, T>(g, c, v);
  fp[Q][CC] = up[Q][CC] + (f0 - f1);
  up[Q][CC] = f0 + f1;
}

template <typename T>
__device__ __forceinline__ void fold_rows(const G1<T>& g, const T (&c)[8], const T (&v)[24], T (&fp)[4][3],
                                          T (&up)[4][3]) {
  fold_pair<0, 0>(g, c, v, fp, up); fold_pair<0, 1>(g, c, v, fp, up); fold_pair<0, 2>(g, c, v, fp, up);
  fold_pair<1, 0>(g, c, v, fp, up); fold_pair<1, 1>(g, c, v, fp, up); fold_pair<1, 2>(g, c, v, fp, up);
  fold_pair<2, 0>(g, c, v, fp, up); fold_pair<2, 1>(g, c, v, fp, up); fold_pair<2, 2>(g, c, v, fp, up);
  fold_pair<3, 0>(g, c, v, fp, up); fold_pair<3, 1>(g, c, v, fp, up); fold_pair<3, 2>(g, c, v, fp, up);
}

// x-y modes of plane zz of this thread's four node columns, from a staged slot
template <typename T>
__device__ __forceinline__ void slot_modes(const T* __restrict__ slot, int i, int j, int zz, T (&a)[4][3]) {
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    const T* b = slot + cc * WBOX * WBOX * 4 + zz;
    T m[4];
    xy4(b[(j * WBOX + i) * 4], b[(j * WBOX + i + 1) * 4], b[((j + 1) * WBOX + i) * 4],
        b[((j + 1) * WBOX + i + 1) * 4], m);
#pragma unroll
    for (int q = 0; q < 4; ++q) a[q][cc] = m[q];
  }
}

// level-1 operator, u zero on masked dofs: out = m K u (the patch cells' rows are added by
// k_patch_add). One block per SM: the modal product keeps ~230 registers busy, and capping it at
// 168 or 128 (two blocks) spills and runs slower (65 us against 47 us at 128 x 64 x 64 cells).
// A block owns 15 x 15 node columns over a z segment and runs 16 x 16 threads,
// one per cell column plus a one-cell halo; u arrives by TMA into a 3-stage mbarrier ring
// (one chunk of 17 x 17 node columns x 3 components), the Walsh coefficients by 128-byte loads
// per cell column and chunk,
// the outputs leave by TMA stores. Waits are bounded and a block that gives up sets *err.
template <typename T>
__global__ void __launch_bounds__(TXC * TYC, 1)
k_weights_tma(const __grid_constant__ WMaps<T> maps, const T* __restrict__ wc, const uint8_t* __restrict__ mask,
              const G1<T> gc, LpGrid g, int zch, int nchunks, int* __restrict__ err) {
  extern __shared__ unsigned char wsm_raw[];
  const uint32_t raw_off = lp_smem_addr(wsm_raw);
  WSmem<T>& sm = *reinterpret_cast<WSmem<T>*>(wsm_raw + ((1024u - (raw_off & 1023u)) & 1023u));
  constexpr bool staged_w = sizeof(T) == 4;
  const int tid = threadIdx.x;
  const int i = tid % TXC, j = tid / TXC;
  const int x0 = blockIdx.x * (TXC - 1), y0 = blockIdx.y * (TYC - 1);
  const int c_begin = blockIdx.z * zch;
  const int c_end = min(c_begin + zch, nchunks);
  if (c_begin >= c_end) return;
  const int cstart = c_begin > 0 ? c_begin - 1 : 0;
  const int nload = min(c_end + 1, nchunks) - cstart;
  const int nproc = c_end - cstart;
  const bool own = i >= 1 && j >= 1;
  const int cx = x0 - 1 + i, cy = y0 - 1 + j;
  const bool cell_ok = cx >= 0 && cx < g.nx && cy >= 0 && cy < g.ny;
  const long long wstride = 32LL * g.nx * g.ny;   // one chunk of Walsh runs to the next
  const T* wcol = wc + (cell_ok ? ((long long)cy * g.nx + cx) * 32 : 0);
  constexpr uint32_t UBYTES = 3 * WBOX * WBOX * 4 * sizeof(T);
  constexpr uint32_t WBYTES = staged_w ? 32 * TXC * TYC * sizeof(T) : 0;
  __shared__ int bad;
  if (tid == 0) {
    int code = 0;
    uint32_t so = 0, sw = 0;
    for (int s = 0; s < WSTAGE; ++s) {
      so |= lp_smem_addr(sm.u[s].v);
      sw |= lp_smem_addr(sm.w[s]);
    }
    so |= lp_smem_addr(sm.o[0].v) | lp_smem_addr(sm.o[1].v);
    if ((so & 127) || (staged_w && (sw & 1023))) code = 20;
    else if (staged_w && (reinterpret_cast<uintptr_t>(&maps.w) & 63)) code = 26;
    else if (reinterpret_cast<uintptr_t>(&maps.u) & 63) code = 21;
    else if (reinterpret_cast<uintptr_t>(&maps.out) & 63) code = 22;
    else if (lp_smem_addr(&sm.full[0]) & 7) code = 23;
    else if (reinterpret_cast<uintptr_t>(mask) & 3) code = 24;
    else if (reinterpret_cast<uintptr_t>(wc) & 15) code = 25;
    bad = code;
    if (code) atomicExch(err, code);
  }
  __syncthreads();
  if (bad) return;
  if (tid == 0) {
    for (int s = 0; s < WSTAGE; ++s) lp_mbar_init(&sm.full[s], 1);
    lp_fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int k) {
    const int s = k % WSTAGE;
    lp_mbar_expect_tx(&sm.full[s], UBYTES + WBYTES);
    lp_tma_load_4d(sm.u[s].v, &maps.u, 4 * (x0 - 1), y0 - 1, cstart + k, 0, &sm.full[s]);
    if constexpr (staged_w) lp_tma_load_4d(sm.w[s], &maps.w, 0, x0 - 1, y0 - 1, cstart + k, &sm.full[s]);
  };
  if (tid == 0) {
    issue(0);
    if (nload > 1) issue(1);
  }
  T up_carry[4][3], a_lo[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) up_carry[q][c] = a_lo[q][c] = T(0);

  for (int k = 0; k < nproc; ++k) {
    const int c = cstart + k;
    const bool halo = c < c_begin;
    const int s = k % WSTAGE;
    if (tid == 0) {
      if (k + 2 < nload) issue(k + 2);
      lp_bulk_wait_read<1>();
    }
    bool ok = lp_mbar_wait(&sm.full[s], (k / WSTAGE) & 1);
    const bool has_next = k + 1 < nload;
    if (has_next) ok = ok && lp_mbar_wait(&sm.full[(k + 1) % WSTAGE], ((k + 1) / WSTAGE) & 1);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        for (int kk = k; kk < min(k + 3, nload); ++kk) lp_mbar_wait(&sm.full[kk % WSTAGE], (kk / WSTAGE) & 1);
      }
      break;
    }
    const T* us = sm.u[s].v;
    const T* un = sm.u[(k + 1) % WSTAGE].v;
    if (k == 0) slot_modes(us, i, j, halo ? 3 : 0, a_lo);
    const T* wch = wcol + (long long)c * wstride;   // this chunk's Walsh run (128 bytes in float32)
#pragma unroll 1
    for (int t = halo ? 3 : 0; t < 4; ++t) {
      T a_hi[4][3];
      if (t < 3) {
        slot_modes(us, i, j, t + 1, a_hi);
      } else if (has_next) {
        slot_modes(un, i, j, 0, a_hi);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) a_hi[q][cc] = T(0);
      }
      T v[24], cw[8];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const T lo = a_lo[q][cc], hi = a_hi[q][cc];
          v[3 * q + cc] = lo + hi;
          v[3 * (q + 4) + cc] = hi - lo;
          a_lo[q][cc] = hi;
        }
      if constexpr (staged_w) {
        // this cell's eight coefficients: two 16-byte reads of the column's swizzled row
        const uint32_t row = (uint32_t)(j * TXC + i);
        const unsigned char* wb = reinterpret_cast<const unsigned char*>(sm.w[s]);
        const float4 c0 = *reinterpret_cast<const float4*>(wb + lp_swz128(row * 128u + (uint32_t)t * 32u));
        const float4 c1 = *reinterpret_cast<const float4*>(wb + lp_swz128(row * 128u + (uint32_t)t * 32u + 16u));
        cw[0] = c0.x; cw[1] = c0.y; cw[2] = c0.z; cw[3] = c0.w;
        cw[4] = c1.x; cw[5] = c1.y; cw[6] = c1.z; cw[7] = c1.w;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) cw[kk] = cell_ok ? cw[kk] : T(0);
      } else {
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) cw[kk] = cell_ok ? __ldg(wch + t * 8 + kk) : T(0);
      }
      T fp[4][3];
      fold_rows<T>(gc, cw, v, fp, up_carry);
      if (!halo) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const T t0 = fp[0][cc] - fp[2][cc], t1 = fp[1][cc] - fp[3][cc];
          const T t2 = fp[0][cc] + fp[2][cc], t3 = fp[1][cc] + fp[3][cc];
          const T c10 = __shfl_up_sync(0xffffffffu, t0 + t1, 1, TXC);
          const T c11 = __shfl_up_sync(0xffffffffu, t2 + t3, 1, TXC);
          sm.own[cc][t][tid] = (t0 - t1) + c10;
          sm.red[cc][t][tid] = (t2 - t3) + c11;
        }
      }
    }
    if (halo) {
      __syncthreads();
      continue;
    }
    __syncthreads();
    if (own) {
      const bool inside = cx < g.NX() && cy < g.NY();
      uint8_t mbs[4] = {0, 0, 0, 0};
      if (inside) {
        const uchar4 mb = *reinterpret_cast<const uchar4*>(mask + g.node(cx, cy, 4 * c));
        mbs[0] = mb.x; mbs[1] = mb.y; mbs[2] = mb.z; mbs[3] = mb.w;
      }
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        T o[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const T v = sm.own[cc][t][tid] + sm.red[cc][t][tid - TXC];
          o[t] = ((mbs[t] >> cc) & 1) ? v : T(0);
        }
        T* dst = &sm.o[k & 1].v[((cc * (TYC - 1) + (j - 1)) * (TXC - 1) + (i - 1)) * 4];
#pragma unroll
        for (int t = 0; t < 4; ++t) dst[t] = o[t];
      }
    }
    lp_fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      lp_tma_store_4d(&maps.out, 4 * x0, y0, c, 0, sm.o[k & 1].v);
      lp_bulk_commit();
    }
  }
  if (tid == 0) lp_bulk_wait_all();
}

// patch cells (weights zero, an explicit masked matrix): out += m * sum of their rows times
// u, node by node over the box of nodes they touch (one warp per node: the lanes split the
// 8 cells x 24 columns); runs after k_weights_tma
template <typename T>
__global__ void k_patch_add(T* __restrict__ out, const T* __restrict__ u, const int* __restrict__ pid,
                            const T* __restrict__ pk, const uint8_t* __restrict__ mask, LpGrid g, int bx0, int by0,
                            int bz0, int bnx, int bny, int bnz) {
  const long long total = (long long)bnx * bny * bnz;
  const long long cs = g.comp_stride();
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (warp >= total) return;
  const int z = bz0 + (int)(warp % bnz);
  const long long q = warp / bnz;
  const int y = by0 + (int)(q % bny), x = bx0 + (int)(q / bny);
  // a node with no solved component keeps its output (the held nodes of a support face are
  // half of a patch box): the whole warp leaves
  const uint8_t mb0 = mask[g.node(x, y, z)];
  if (!(mb0 & 7)) return;
  // lane -> (cell corner kk = lane / 4, column block of 6 = lane % 4)
  const int kk = lane >> 2, cb = lane & 3;
  T a[3] = {T(0), T(0), T(0)};
  const int cx = x - cx_(kk), cy = y - cy_(kk), cz = z - cz_(kk);
  int p = -1;
  if (cx >= 0 && cy >= 0 && cz >= 0 && cx < g.nx && cy < g.ny && cz < g.nz) p = pid[g.cell(cx, cy, cz)];
  if (p >= 0) {
    const T* kp = pk + (long long)p * 576;
#pragma unroll
    for (int c6 = 0; c6 < 6; ++c6) {
      const int col = 6 * cb + c6, q2 = col / 3, c2 = col % 3;
      const T uv = u[c2 * cs + g.node(cx + cx_(q2), cy + cy_(q2), cz + cz_(q2))];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) a[cc] += kp[(3 * kk + cc) * 24 + col] * uv;
    }
  }
  const unsigned any = __ballot_sync(0xffffffffu, p >= 0);
  if (!any) return;
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
    for (int o = 16; o > 0; o >>= 1) a[cc] += __shfl_down_sync(0xffffffffu, a[cc], o);
  if (lane == 0) {
    const long long n = g.node(x, y, z);
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
      if ((mb0 >> cc) & 1) out[cc * cs + n] += a[cc];
  }
}

// ---- explicit levels: packed symmetric matrices, entry-major ---------------------------------
__host__ __device__ __forceinline__ int sym_index(int i, int j) {  // i <= j
  return i * 24 - (i * (i - 1)) / 2 + (j - i);
}

// One thread per cell, its 300 matrix entries streamed (entry p of consecutive cells coalesced).
// The kernel is bound by how many of those loads are in flight: under a (128, 4) register bound
// the compiler hoists them (a few spilled bytes), which measured 1.3x faster at 64 x 32 x 32
// cells than the unbounded build (96 registers, loads issued as used) and 2x faster than a
// grid-stride form.
template <typename T>
__global__ void __launch_bounds__(128, 4)
k_explicit_cells(T* __restrict__ ft, const T* __restrict__ u, const T* __restrict__ kp, LpGrid g) {
  const long long ncp = g.cells_padded();
  const long long cs = g.comp_stride();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ncp) return;
  int x, y, z;
  if (!g.cell_at(t, x, y, z)) return;
  const long long c = t;
  // corner k at n0 + x step (4) + y step (4 NX) + z step (1, or to the next chunk)
  const long long n0 = g.node(x, y, z);
  const long long oy = 4LL * g.NX(), oz = (z & 3) == 3 ? g.node_zc_stride() - 3 : 1;
  T uc[24], f[24];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const long long n = n0 + (k & 1 ? 4 : 0) + (k & 2 ? oy : 0) + (k & 4 ? oz : 0);
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) uc[3 * k + cc] = u[cc * cs + n];
  }
#pragma unroll
  for (int r = 0; r < 24; ++r) f[r] = T(0);
  const T* kc = kp + c;
#pragma unroll
  for (int a = 0; a < 24; ++a) {
#pragma unroll
    for (int b = a; b < 24; ++b) {
      const T kab = __ldg(kc + (long long)sym_index(a, b) * ncp);
      f[a] += kab * uc[b];
      if (b != a) f[b] += kab * uc[a];
    }
  }
#pragma unroll
  for (int r = 0; r < 24; ++r) ft[(long long)r * ncp + c] = f[r];
}

// ---- explicit levels in the corner-parity basis ------------------------------------------------
// A Galerkin level's cell matrix K, in the modes of its cell (K^ = T K T^T / 64, T = kron(H, I3)),
// has the level-1 pattern: 279 non-zeros, 150 in the upper triangle, at every level of the plain
// hierarchy (the pattern is kept by the child Galerkin product). Those cells are stored as the
// 150 entries (entry-major, (150, cells)) and applied as f = T^T (K^ (T u)): half the bytes of the
// 300-entry node-basis form. Cells with weight off the pattern (children carrying masked patch
// matrices) are listed and applied from the node-basis form.
constexpr int MODAL_UP = 150;
__constant__ int c_mup_r[MODAL_UP] = {3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, 8, 8, 8, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 12, 12, 12, 12, 12, 12, 13, 13, 13, 13, 13, 13, 14, 14, 14, 14, 14, 14, 14, 14, 15, 15, 15, 15, 15, 15, 15, 15, 16, 16, 16, 16, 16, 16, 16, 17, 17, 17, 17, 17, 17, 17, 18, 18, 18, 18, 19, 19, 19, 19, 19, 20, 20, 20, 20, 21, 21, 21, 22, 22, 23};
__constant__ int c_mup_c[MODAL_UP] = {3, 7, 9, 10, 14, 15, 17, 19, 20, 21, 22, 23, 4, 6, 9, 10, 16, 18, 21, 22, 5, 11, 12, 15, 17, 18, 21, 23, 6, 9, 10, 16, 18, 21, 22, 7, 9, 10, 14, 15, 17, 19, 20, 21, 22, 23, 8, 11, 13, 16, 19, 20, 22, 23, 9, 10, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 10, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 11, 12, 13, 15, 16, 17, 18, 19, 20, 21, 22, 23, 12, 15, 17, 18, 21, 23, 13, 16, 19, 20, 22, 23, 14, 15, 17, 19, 20, 21, 22, 23, 15, 17, 18, 19, 20, 21, 22, 23, 16, 18, 19, 20, 21, 22, 23, 17, 18, 19, 20, 21, 22, 23, 18, 21, 22, 23, 19, 20, 21, 22, 23, 20, 21, 22, 23, 21, 22, 23, 22, 23, 23};
// bit i % 32 of word i / 32: entry i = 24 r + c of K^ is on the pattern
__constant__ unsigned c_mpat[18] = {0x00000000u, 0x00000000u, 0xfac68800u, 0x20650650u, 0x0650a698u, 0xfac68865u, 0xd8d92900u, 0xc6d8ffc6u, 0xffb920ffu, 0x00a69820u, 0xc688d929u, 0xfedea8fau, 0xa8fd2f50u, 0x9e70fedeu, 0xfbef88e7u, 0xf8fbef88u, 0xefd8ffdeu, 0xffffa8ffu};
#define MUP_ROWS {3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, 8, 8, 8, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 12, 12, 12, 12, 12, 12, 13, 13, 13, 13, 13, 13, 14, 14, 14, 14, 14, 14, 14, 14, 15, 15, 15, 15, 15, 15, 15, 15, 16, 16, 16, 16, 16, 16, 16, 17, 17, 17, 17, 17, 17, 17, 18, 18, 18, 18, 19, 19, 19, 19, 19, 20, 20, 20, 20, 21, 21, 21, 22, 22, 23}
#define MUP_COLS {3, 7, 9, 10, 14, 15, 17, 19, 20, 21, 22, 23, 4, 6, 9, 10, 16, 18, 21, 22, 5, 11, 12, 15, 17, 18, 21, 23, 6, 9, 10, 16, 18, 21, 22, 7, 9, 10, 14, 15, 17, 19, 20, 21, 22, 23, 8, 11, 13, 16, 19, 20, 22, 23, 9, 10, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 10, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 11, 12, 13, 15, 16, 17, 18, 19, 20, 21, 22, 23, 12, 15, 17, 18, 21, 23, 13, 16, 19, 20, 22, 23, 14, 15, 17, 19, 20, 21, 22, 23, 15, 17, 18, 19, 20, 21, 22, 23, 16, 18, 19, 20, 21, 22, 23, 17, 18, 19, 20, 21, 22, 23, 18, 21, 22, 23, 19, 20, 21, 22, 23, 20, 21, 22, 23, 21, 22, 23, 22, 23, 23}

__device__ __forceinline__ float walsh_h(int m, int k) {
  float v = 1.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if ((m >> a) & 1) v *= ((k >> a) & 1) ? 1.0f : -1.0f;
  return v;
}

// one warp per cell: K^ of the cell's (24 x 24) matrix in float64, its symmetric part on the
// pattern into km; a cell with off-pattern weight above tol of its largest entry is listed
template <typename Ti>
__global__ void __launch_bounds__(128) k_pack_modal(float* __restrict__ km, int* __restrict__ glist,
                                                    int* __restrict__ gcount, float* __restrict__ kpc,
                                                    const Ti* __restrict__ k, long long ncp, double tol) {
  __shared__ double sk[4][576];
  __shared__ double sa[4][576];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* K = sk[w];
  double* A = sa[w];
  for (long long cell = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; cell < ncp;
       cell += (long long)gridDim.x * (blockDim.x >> 5)) {
    for (int i = lane; i < 576; i += 32) K[i] = (double)k[cell * 576 + i];
    __syncwarp();
    // A = T K
    for (int i = lane; i < 576; i += 32) {
      const int r = i / 24, c = i % 24, mr = r / 3, cr = r % 3;
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) s += (double)walsh_h(mr, q) * K[(3 * q + cr) * 24 + c];
      A[i] = s;
    }
    __syncwarp();
    // K^ = A T^T / 64 into K (reused)
    double amax = 0.0, off = 0.0;
    for (int i = lane; i < 576; i += 32) {
      const int r = i / 24, c = i % 24, mc = c / 3, cc = c % 3;
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) s += A[r * 24 + 3 * q + cc] * (double)walsh_h(mc, q);
      s /= 64.0;
      K[i] = s;
      amax = fmax(amax, fabs(s));
    }
    __syncwarp();
    for (int i = lane; i < 576; i += 32)
      if (!((c_mpat[i >> 5] >> (i & 31)) & 1u)) off = fmax(off, fabs(K[i]));
    for (int o = 16; o > 0; o >>= 1) {
      amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
      off = fmax(off, __shfl_xor_sync(0xffffffffu, off, o));
    }
    const bool general = off > tol * amax;
    for (int p = lane; p < MODAL_UP; p += 32) {
      const int r = c_mup_r[p], c = c_mup_c[p];
      // a listed cell's entries are zero, its entry 0 a NaN marker the apply skips it by
      km[(long long)p * ncp + cell] =
          general ? (p == 0 ? __int_as_float(0x7fc00001) : 0.0f) : (float)(0.5 * (K[r * 24 + c] + K[c * 24 + r]));
    }
    if (general) {   // listed: the node-basis symmetric part, cell-major, at the cell's slot
      int slot = 0;
      if (lane == 0) slot = atomicAdd(gcount, 1);
      slot = __shfl_sync(0xffffffffu, slot, 0);
      if (lane == 0) glist[slot] = (int)cell;
      for (int p = lane; p < 300; p += 32) {
        int a = 0, rem = p;
        while (rem >= 24 - a) { rem -= 24 - a; ++a; }
        const int b2 = a + rem;
        kpc[(long long)slot * 300 + p] =
            (float)(0.5 * ((double)k[cell * 576 + a * 24 + b2] + (double)k[cell * 576 + b2 * 24 + a]));
      }
    }
    __syncwarp();
  }
}

// in-place a[k] <- sum_m H[m][k] a[m] (the transpose of lp's Walsh transform H a)
__device__ __forceinline__ void walsh8t(float (&a)[8]) {
#pragma unroll
  for (int b = 1; b < 8; b <<= 1)
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (!(k & b)) {
        const float lo = a[k], hi = a[k | b];
        a[k] = lo - hi;
        a[k | b] = lo + hi;
      }
}

__device__ __forceinline__ void walsh8(float (&a)[8]) {
#pragma unroll
  for (int b = 1; b < 8; b <<= 1)
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (!(k & b)) {
        const float lo = a[k], hi = a[k | b];
        a[k] = lo + hi;
        a[k | b] = hi - lo;
      }
}

// ft (24, cells) = T^T (K^ (T u_c)) for every cell (listed cells are rewritten afterwards)
__device__ __forceinline__ void modal_cell(float* __restrict__ ft, const float* __restrict__ u,
                                           const float* __restrict__ km, const LpGrid& g, long long t) {
  const long long ncp = g.cells_padded();
  const long long cs = g.comp_stride();
  if (t >= ncp) return;
  int x, y, z;
  if (!g.cell_at(t, x, y, z)) return;
  if (isnan(__ldg(km + t))) return;                // a listed cell (its entry 0 holds the marker)
  const long long n0 = g.node(x, y, z);
  const long long oy = 4LL * g.NX(), oz = (z & 3) == 3 ? g.node_zc_stride() - 3 : 1;
  constexpr int MUP_R[MODAL_UP] = MUP_ROWS;
  constexpr int MUP_C[MODAL_UP] = MUP_COLS;
  float uh[24], fh[24];
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    float a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
      a[q] = u[cc * cs + n0 + (q & 1 ? 4 : 0) + (q & 2 ? oy : 0) + (q & 4 ? oz : 0)];
    walsh8(a);
#pragma unroll
    for (int m = 0; m < 8; ++m) uh[3 * m + cc] = a[m];
  }
#pragma unroll
  for (int r = 0; r < 24; ++r) fh[r] = 0.0f;
  const float* kc = km + t;
#pragma unroll
  for (int p = 0; p < MODAL_UP; ++p) {
    const float v = __ldg(kc + (long long)p * ncp);
    fh[MUP_R[p]] += v * uh[MUP_C[p]];
    if (MUP_R[p] != MUP_C[p]) fh[MUP_C[p]] += v * uh[MUP_R[p]];
  }
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    float a[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) a[m] = fh[3 * m + cc];
    walsh8t(a);
#pragma unroll
    for (int q = 0; q < 8; ++q) ft[(long long)(3 * q + cc) * ncp + t] = a[q];
  }
}

// the listed cells from their node-basis entries (kpc: 300 per listed cell, cell-major): one warp
// per cell, its 300 entries and 24 corner values staged in shared memory, lane r < 24 forms row r
__device__ __forceinline__ void listed_cells(float* __restrict__ ft, const float* __restrict__ u,
                                             const float* __restrict__ kpc, const int* __restrict__ glist,
                                             const int* __restrict__ gcount, const LpGrid& g, int block, int nblocks,
                                             float (*sk)[300], float (*su)[24]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long ncp = g.cells_padded();
  const long long cs = g.comp_stride();
  const int cnt = *gcount;
  for (int slot = (block * blockDim.x + threadIdx.x) >> 5; slot < cnt; slot += (nblocks * blockDim.x) >> 5) {
    const long long c = glist[slot];
    int x, y, z;
    g.cell_at(c, x, y, z);
    for (int p = lane; p < 300; p += 32) sk[w][p] = __ldg(kpc + (long long)slot * 300 + p);
    if (lane < 24) {
      const int q = lane / 3, cc = lane % 3;
      su[w][lane] = u[cc * cs + g.node(x + cx_(q), y + cy_(q), z + cz_(q))];
    }
    __syncwarp();
    if (lane < 24) {
      float f = 0.0f;
#pragma unroll
      for (int b = 0; b < 24; ++b) {
        const int lo = lane < b ? lane : b, hi = lane < b ? b : lane;
        f += sk[w][sym_index(lo, hi)] * su[w][b];
      }
      ft[(long long)lane * ncp + c] = f;
    }
    __syncwarp();
  }
}

// the cell rows of an explicit level in one launch: blocks below modal_blocks apply the modal
// form to one cell per thread (listed cells skipped), the blocks past them the listed cells
__global__ void __launch_bounds__(128, 4) k_explicit_modal_cells(float* __restrict__ ft, const float* __restrict__ u,
                                                                const float* __restrict__ km,
                                                                const float* __restrict__ kpc,
                                                                const int* __restrict__ glist,
                                                                const int* __restrict__ gcount, LpGrid g,
                                                                int modal_blocks) {
  __shared__ float sk[4][300];
  __shared__ float su[4][24];
  if ((int)blockIdx.x < modal_blocks) {
    modal_cell(ft, u, km, g, blockIdx.x * (long long)blockDim.x + threadIdx.x);
  } else {
    listed_cells(ft, u, kpc, glist, gcount, g, blockIdx.x - modal_blocks, gridDim.x - modal_blocks, sk, su);
  }
}

template <typename T>
__global__ void k_explicit_gather(T* __restrict__ out, const T* __restrict__ ft, const uint8_t* __restrict__ mask,
                                  LpGrid g) {
  const long long total = g.nodes_padded();
  const long long ncp = g.cells_padded(), cs = g.comp_stride();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    T a[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int cx = x - cx_(k), cy = y - cy_(k), cz = z - cz_(k);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      const long long c = g.cell(cx, cy, cz);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) a[cc] += ft[(long long)(3 * k + cc) * ncp + c];
    }
    const long long n = g.node(x, y, z);
    const uint8_t mb = mask[n];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) out[cc * cs + n] = ((mb >> cc) & 1) ? a[cc] : T(0);
  }
}

// The explicit gather with a degree-2 Chebyshev update applied to each node's A u as it is formed
// (the standalone kernels' expressions): mode 1 x = d + (c1 d + c2 dinv (b - A d)); mode 2 r = b - A x,
// d = s dinv r; mode 3 x = (x + d) + (c1 d + c2 dinv (r - A d)). Padding is left as it is (zero).
struct ChebArgs {
  float* x;
  float* r;
  float* d;
  const float* b;
  const float* dinv;
  const double* coef;
};

template <int MODE>
__global__ void k_explicit_gather_cheb(const float* __restrict__ ft, const uint8_t* __restrict__ mask, LpGrid g,
                                       ChebArgs a) {
  const long long total = g.nodes_padded();
  const long long ncp = g.cells_padded(), cs = g.comp_stride();
  const float s = (float)a.coef[1], c1 = (float)a.coef[2], c2 = (float)a.coef[3];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!g.node_at(t, x, y, z)) continue;
    float acc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int cx = x - cx_(k), cy = y - cy_(k), cz = z - cz_(k);
      if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) continue;
      const long long c = g.cell(cx, cy, cz);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) acc[cc] += ft[(long long)(3 * k + cc) * ncp + c];
    }
    const long long n = g.node(x, y, z);
    const uint8_t mb = mask[n];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const long long i = cc * cs + n;
      const float adi = ((mb >> cc) & 1) ? acc[cc] : 0.0f;
      if (MODE == 1) {
        a.x[i] = lp_cheb2_zero_v(a.d[i], a.b[i], adi, a.dinv[i], c1, c2);
      } else if (MODE == 2) {
        float ri, di;
        lp_residual_scaled_v(a.b[i], adi, a.dinv[i], s, ri, di);
        a.r[i] = ri;
        a.d[i] = di;
      } else {
        a.x[i] = lp_cheb2_v(a.x[i], a.d[i], a.r[i], adi, a.dinv[i], c1, c2);
      }
    }
  }
}

// full (cells, 576) matrices -> packed symmetric entry-major (the average of K and K^T)
template <typename Ti, typename To>
__global__ void k_pack_sym(To* __restrict__ kp, const Ti* __restrict__ k, long long ncp) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 300 * ncp; t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / ncp);
    const long long c = t % ncp;
    int a = 0, rem = p;
    while (rem >= 24 - a) { rem -= 24 - a; ++a; }
    const int b = a + rem;
    kp[t] = (To)(0.5 * ((double)k[c * 576 + a * 24 + b] + (double)k[c * 576 + b * 24 + a]));
  }
}

}  // namespace

#define LP_GRID_ARGS int nx, int ny, int nz, int pz, int cpz
#define LP_GRID lp_grid(nx, ny, nz, pz, cpz)
#define LP_ST ((cudaStream_t)stream)

static double pw_host(int k, int q, int r) {
  double w = 1.0;
  for (int a = 0; a < 3; ++a) {
    const int p = ((k >> a) & 1) + ((q >> a) & 1);
    const double t = 0.5 * p;
    w *= ((r >> a) & 1) ? t : 1.0 - t;
  }
  return w;
}

static const int G1_ROWS[279] = {3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, 8, 8, 8, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 12, 12, 12, 12, 12, 12, 12, 12, 13, 13, 13, 13, 13, 13, 13, 13, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 20, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 21, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 22, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23, 23};
static const int G1_TS[279] = {0, 0, 0, 1, 1, 2, 2, 3, 4, 4, 5, 6, 0, 0, 1, 2, 4, 4, 5, 6, 0, 0, 1, 2, 2, 3, 4, 6, 0, 0, 1, 2, 4, 4, 5, 6, 0, 0, 0, 1, 1, 2, 2, 3, 4, 4, 5, 6, 0, 0, 1, 1, 2, 3, 4, 5, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 5, 6, 6, 7, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 5, 6, 6, 7, 0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 6, 0, 0, 1, 2, 2, 3, 4, 6, 0, 0, 1, 1, 2, 3, 4, 5, 0, 0, 0, 1, 1, 2, 2, 3, 4, 4, 5, 6, 0, 0, 1, 1, 1, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 0, 0, 0, 1, 1, 1, 2, 3, 4, 4, 4, 5, 5, 6, 0, 0, 1, 1, 1, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 0, 0, 0, 1, 2, 2, 2, 3, 4, 4, 4, 5, 6, 6, 0, 0, 1, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 0, 0, 1, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 7, 0, 1, 1, 1, 2, 2, 3, 3, 3, 4, 4, 5, 5, 5, 6, 6, 6, 7, 7, 0, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 5, 5, 5, 6, 6, 6, 7, 7, 0, 1, 1, 2, 2, 3, 3, 3, 4, 4, 4, 5, 5, 5, 6, 6, 6, 7, 7};
static const int G1_COLS[279] = {3, 7, 14, 10, 17, 9, 20, 23, 15, 19, 22, 21, 4, 6, 9, 10, 16, 18, 21, 22, 5, 12, 15, 11, 18, 21, 17, 23, 4, 6, 9, 10, 16, 18, 21, 22, 3, 7, 14, 10, 17, 9, 20, 23, 15, 19, 22, 21, 8, 13, 11, 16, 19, 22, 20, 23, 9, 20, 4, 6, 23, 3, 7, 14, 10, 17, 21, 16, 18, 15, 19, 22, 10, 17, 3, 7, 14, 4, 6, 23, 9, 20, 22, 15, 19, 16, 18, 21, 11, 16, 18, 8, 13, 21, 5, 12, 22, 15, 19, 23, 20, 17, 5, 12, 15, 11, 18, 21, 17, 23, 8, 13, 11, 16, 19, 22, 20, 23, 3, 7, 14, 10, 17, 9, 20, 23, 15, 19, 22, 21, 15, 19, 5, 12, 22, 21, 11, 18, 3, 7, 14, 10, 17, 9, 20, 23, 11, 16, 18, 8, 13, 21, 22, 19, 4, 6, 23, 9, 20, 10, 10, 17, 3, 7, 14, 23, 9, 20, 5, 12, 22, 15, 19, 11, 18, 21, 11, 16, 18, 21, 5, 12, 22, 15, 4, 6, 23, 9, 10, 17, 15, 19, 22, 8, 13, 21, 11, 16, 3, 7, 14, 10, 17, 9, 20, 23, 9, 20, 23, 3, 7, 14, 10, 17, 8, 13, 21, 11, 16, 15, 19, 22, 21, 11, 16, 18, 15, 19, 5, 12, 22, 9, 20, 4, 6, 23, 3, 7, 14, 10, 17, 22, 15, 19, 11, 16, 18, 8, 13, 21, 10, 17, 3, 7, 14, 4, 6, 23, 9, 20, 23, 9, 20, 10, 17, 3, 7, 14, 11, 16, 18, 8, 13, 21, 5, 12, 22, 15, 19};

template <typename T>
static int launch_weights_tma(T* out, const T* u, const T* wc, const int* pid, const T* pk, const uint8_t* mask,
                              const double* g1_host, const int* pbox, int* err, LpGrid g, cudaStream_t st) {
  if (!lp_grid_ok(g) || g.pz % 4 || g.cpz != g.pz || !out || !u || !wc || !mask || !g1_host || !err || out == u)
    return LP_ERR_ARG;
  G1<T> gc;
  for (int i = 0; i < 279; ++i) gc.c[i] = (T)g1_host[i];
  WMaps<T> maps;
  const uint64_t nd[4] = {4 * (uint64_t)g.NX(), (uint64_t)g.NY(), (uint64_t)g.pz / 4, 3};
  const uint32_t bin[4] = {4 * WBOX, WBOX, 1, 3};
  const uint32_t bout[4] = {4 * (TXC - 1), TYC - 1, 1, 3};
  if (!lp_make_map(&maps.u, u, 4, nd, bin, sizeof(T)) || !lp_make_map(&maps.out, out, 4, nd, bout, sizeof(T)))
    return LP_ERR_ARG;
  memset(&maps.w, 0, sizeof(maps.w));
  if (sizeof(T) == 4) {
    const uint64_t wd[4] = {32, (uint64_t)g.nx, (uint64_t)g.ny, (uint64_t)g.cpz / 4};
    const uint32_t wb[4] = {32, TXC, TYC, 1};
    if (!lp_make_map(&maps.w, wc, 4, wd, wb, sizeof(T), 128)) return LP_ERR_ARG;
  }
  const int smem = (int)sizeof(WSmem<T>) + 1024;
  static long long slots = 0;   // resident blocks on the device (queried once per process)
  if (!slots) {
    if (cudaFuncSetAttribute(k_weights_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return LP_ERR_LAUNCH;
    int per_sm = 1, dev = 0, nsm = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_weights_tma<T>, TXC * TYC, smem);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    slots = (long long)(per_sm > 0 ? per_sm : 1) * nsm;
  }
  const int gx = (g.NX() + TXC - 2) / (TXC - 1), gy = (g.NY() + TYC - 2) / (TYC - 1);
  const int nchunks = g.pz / 4;
  int best = nchunks;
  double bc = 1e30;
  for (int zch = 1; zch <= nchunks; ++zch) {
    const long long nseg = (nchunks + zch - 1) / zch, units = (long long)gx * gy * nseg;
    const double cost = (double)((units + slots - 1) / slots) * (zch + (nseg > 1 ? 0.3 : 0.0));
    if (cost < bc - 1e-9) { bc = cost; best = zch; }
  }
  const int tuned = lp_tune_lookup(sizeof(T) == 4 ? LP_KNOB_L1_F32 : LP_KNOB_L1_F64, g.nx, g.ny, g.nz);
  if (tuned >= 1 && tuned <= nchunks) best = tuned;
  dim3 grid(gx, gy, (nchunks + best - 1) / best);
  k_weights_tma<T><<<grid, TXC * TYC, smem, st>>>(maps, wc, mask, gc, g, best, nchunks, err);
  if (pid && pk && pbox && pbox[3] > 0 && pbox[4] > 0 && pbox[5] > 0) {
    const long long nb = (long long)pbox[3] * pbox[4] * pbox[5];
    k_patch_add<T><<<lp_blocks(nb * 32, 256), 256, 0, st>>>(out, u, pid, pk, mask, g, pbox[0], pbox[1], pbox[2],
                                                            pbox[3], pbox[4], pbox[5]);
  }
  LP_LAUNCH_CHECK();
  return LP_OK;
}

template <typename T>
static int launch_explicit(T* out, const T* u, const T* kp, T* ft, const uint8_t* mask, LpGrid g, cudaStream_t st) {
  if (!lp_grid_ok(g) || !out || !u || !kp || !ft || !mask || out == u) return LP_ERR_ARG;
  k_explicit_cells<T><<<lp_blocks(g.cells_padded(), 128), 128, 0, st>>>(ft, u, kp, g);
  k_explicit_gather<T><<<lp_blocks(g.nodes_padded(), 256), 256, 0, st>>>(out, ft, mask, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// ---- the explicit-level apply without caller scratch -----------------------------------------
// For callers that cannot allocate device memory: a host application or language binding that
// owns every device allocation and hands this library only the pointers it needs, or a loop
// that must never call cudaMalloc / cudaFree (they synchronize the device). The cell pass's
// (24, cells) intermediate lives in this file-scope array instead of a caller buffer. Every GPU
// that loads the library holds it (6 MB) until the process exits.
#define LP_NOALLOC_MAX_CELLS (1 << 16)   // padded cells (nx * ny * cpz) one call may cover
#define LP_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) float g_explicit_scratch[24 * LP_NOALLOC_MAX_CELLS];

// the array's device address on the current device, looked up once per device ordinal and kept
// for the life of the process: the caller's stream must belong to the current device, and a
// cudaDeviceReset invalidates the kept address (callers must not reset a device they use it on)
static float* explicit_scratch_address() {
  static std::mutex mu;
  static float* addr[LP_NOALLOC_MAX_DEVICES] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= LP_NOALLOC_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_explicit_scratch) != cudaSuccess || !p) return nullptr;
    addr[dev] = static_cast<float*>(p);
  }
  return addr[dev];
}

extern "C" {

// the 279 corner-parity coefficients of the eight G_t = sum_k H[t, k] P_k^T Ke P_k / 8 (host)
int lpb_modal_g1(const double* ke, double* g1_out) {
  if (!ke || !g1_out) return LP_ERR_ARG;
  double h[8][8];
  for (int m = 0; m < 8; ++m)
    for (int k = 0; k < 8; ++k) {
      double v = 1.0;
      for (int a = 0; a < 3; ++a)
        if ((m >> a) & 1) v *= ((k >> a) & 1) ? 1.0 : -1.0;
      h[m][k] = v;
    }
  // M_k = P_k^T Ke P_k
  static double mk[8][24][24];
  for (int k = 0; k < 8; ++k)
    for (int i = 0; i < 24; ++i)
      for (int jj = 0; jj < 24; ++jj) {
        const int ri = i / 3, ci = i % 3, rj = jj / 3, cj = jj % 3;
        double s = 0.0;
        for (int q1 = 0; q1 < 8; ++q1) {
          const double p1 = pw_host(k, q1, ri);
          if (p1 == 0.0) continue;
          for (int q2 = 0; q2 < 8; ++q2) {
            const double p2 = pw_host(k, q2, rj);
            if (p2 == 0.0) continue;
            s += p1 * ke[(3 * q1 + ci) * 24 + 3 * q2 + cj] * p2;
          }
        }
        mk[k][i][jj] = s;
      }
  double amax = 0.0;
  static double gh[8][24][24];
  for (int t = 0; t < 8; ++t)
    for (int r = 0; r < 24; ++r)
      for (int c = 0; c < 24; ++c) {
        const int mr = r / 3, cr = r % 3, mc = c / 3, cc = c % 3;
        double s = 0.0;
        for (int k1 = 0; k1 < 8; ++k1)
          for (int k2 = 0; k2 < 8; ++k2) {
            double gsum = 0.0;
            for (int k = 0; k < 8; ++k) gsum += h[t][k] * mk[k][3 * k1 + cr][3 * k2 + cc];
            s += h[mr][k1] * gsum * h[mc][k2];
          }
        gh[t][r][c] = s / (8.0 * 64.0);
        if (fabs(gh[t][r][c]) > amax) amax = fabs(gh[t][r][c]);
      }
  static bool used[8][24][24];
  for (int t = 0; t < 8; ++t)
    for (int r = 0; r < 24; ++r)
      for (int c = 0; c < 24; ++c) used[t][r][c] = false;
  for (int i = 0; i < 279; ++i) used[G1_TS[i]][G1_ROWS[i]][G1_COLS[i]] = true;
  for (int t = 0; t < 8; ++t)
    for (int r = 0; r < 24; ++r)
      for (int c = 0; c < 24; ++c)
        if (!used[t][r][c] && fabs(gh[t][r][c]) > 1e-12 * amax) return -1;
  for (int i = 0; i < 279; ++i) g1_out[i] = gh[G1_TS[i]][G1_ROWS[i]][G1_COLS[i]];
  return 279;
}

// pbox (host, 6 ints): node box x0, y0, z0, nx, ny, nz holding every node a patch cell touches
int lpb_walsh_chunks_f32(float* wc, const float* w, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || g.cpz % 4 || !wc || !w) return LP_ERR_ARG;
  k_walsh_chunks<float><<<lp_blocks(g.cells_padded(), 256), 256, 0, LP_ST>>>(wc, w, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_walsh_chunks_f64(double* wc, const double* w, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || g.cpz % 4 || !wc || !w) return LP_ERR_ARG;
  k_walsh_chunks<double><<<lp_blocks(g.cells_padded(), 256), 256, 0, LP_ST>>>(wc, w, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// level-1 apply, TMA-staged (same result as lpb_apply_weights_march_*): wc from
// lpb_walsh_chunks_*; g1 and pbox are HOST arrays; err: a device int set when a wait gave up
// (or to an alignment code, 20..25)
int lpb_apply_weights_tma_f32(float* out, const float* u, const float* wc, const int* patch_id, const float* patch_k,
                              const uint8_t* mask, const double* g1, const int* pbox, int* err, LP_GRID_ARGS,
                              void* stream) {
  return launch_weights_tma<float>(out, u, wc, patch_id, patch_k, mask, g1, pbox, err, LP_GRID, LP_ST);
}

int lpb_apply_weights_tma_f64(double* out, const double* u, const double* wc, const int* patch_id,
                              const double* patch_k, const uint8_t* mask, const double* g1, const int* pbox, int* err,
                              LP_GRID_ARGS, void* stream) {
  return launch_weights_tma<double>(out, u, wc, patch_id, patch_k, mask, g1, pbox, err, LP_GRID, LP_ST);
}

int lpb_apply_explicit_sym_f32(float* out, const float* u, const float* kp, float* ft, const uint8_t* mask,
                               LP_GRID_ARGS, void* stream) {
  return launch_explicit<float>(out, u, kp, ft, mask, LP_GRID, LP_ST);
}

int lpb_apply_explicit_sym_f64(double* out, const double* u, const double* kp, double* ft, const uint8_t* mask,
                               LP_GRID_ARGS, void* stream) {
  return launch_explicit<double>(out, u, kp, ft, mask, LP_GRID, LP_ST);
}

// lpb_apply_explicit_sym_f32 with its (24, cells) scratch in the library's static array: no
// allocation by the caller or the library. Grids with more than LP_NOALLOC_MAX_CELLS padded
// cells return LP_ERR_SIZE. The first call on a device looks the array's address up (it should
// come before any stream capture); calls that overlap on the GPU share the array and race. The
// cell pass writes every entry the node pass reads, so stale contents from an earlier call are
// never used and nothing needs clearing.
int lpb_apply_explicit_sym_noalloc_f32(float* out, const float* u, const float* kp, const uint8_t* mask, LP_GRID_ARGS,
                                       void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g)) return LP_ERR_ARG;
  if (g.cells_padded() > LP_NOALLOC_MAX_CELLS) return LP_ERR_SIZE;
  float* ft = explicit_scratch_address();
  if (!ft) return LP_ERR_LAUNCH;
  return launch_explicit<float>(out, u, kp, ft, mask, g, LP_ST);
}

// km (150, ncells) = the pattern entries of each cell's K^ = T K T^T / 64 (symmetric part); cells
// with off-pattern weight above tol of their largest entry get zeros and are listed in glist
// (*gcount of them), their 300 node-basis symmetric entries in kpc at their list slot (glist and
// kpc hold up to ncells cells)
int lpb_pack_modal_f32(float* km, int* glist, int* gcount, float* kpc, const float* k, long long ncells, double tol,
                       void* stream) {
  if (!km || !glist || !gcount || !kpc || !k || ncells < 1) return LP_ERR_ARG;
  if (cudaMemsetAsync(gcount, 0, sizeof(int), LP_ST) != cudaSuccess) return LP_ERR_LAUNCH;
  const long long blocks = (ncells + 3) / 4;
  k_pack_modal<float><<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 128, 0, LP_ST>>>(km, glist, gcount, kpc,
                                                                                          k, ncells, tol);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// out = m K u on an explicit level from the modal form km and, for the listed cells, their
// node-basis entries kpc (both from lpb_pack_modal_f32); ft: 24 * cells scratch
int lpb_apply_explicit_modal_f32(float* out, const float* u, const float* km, const float* kpc, const int* glist,
                                 const int* gcount, float* ft, const uint8_t* mask, LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !out || !u || !km || !kpc || !glist || !gcount || !ft || !mask || out == u) return LP_ERR_ARG;
  const int modal_blocks = lp_blocks(g.cells_padded(), 128);
  k_explicit_modal_cells<<<modal_blocks + 148, 128, 0, LP_ST>>>(ft, u, km, kpc, glist, gcount, g, modal_blocks);
  k_explicit_gather<float><<<lp_blocks(g.nodes_padded(), 256), 256, 0, LP_ST>>>(out, ft, mask, g);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

// the explicit level's A u (modal form, as lpb_apply_explicit_modal_f32) with a degree-2 Chebyshev
// update in its gather: mode 1 (u = d) x = d + (c1 d + c2 dinv (b - A d)); mode 2 (u = x)
// r = b - A x, d = s dinv r; mode 3 (u = d) x = (x + d) + (c1 d + c2 dinv (r - A d)); the fields
// a mode does not name may be NULL; coef: the level's Chebyshev coefficients (device)
int lpb_apply_explicit_modal_cheb_f32(int mode, float* x, float* r, float* d, const float* u, const float* b,
                                      const float* dinv, const double* coef, const float* km, const float* kpc,
                                      const int* glist, const int* gcount, float* ft, const uint8_t* mask,
                                      LP_GRID_ARGS, void* stream) {
  LpGrid g = LP_GRID;
  if (!lp_grid_ok(g) || !u || !km || !kpc || !glist || !gcount || !ft || !mask || !dinv || !coef) return LP_ERR_ARG;
  if (mode == 1 && (!x || !d || !b || u != d || x == d)) return LP_ERR_ARG;
  if (mode == 2 && (!r || !d || !b || u == r || u == d || r == d)) return LP_ERR_ARG;
  if (mode == 3 && (!x || !d || !r || u != d || x == d)) return LP_ERR_ARG;
  if (mode < 1 || mode > 3) return LP_ERR_ARG;
  const int modal_blocks = lp_blocks(g.cells_padded(), 128);
  k_explicit_modal_cells<<<modal_blocks + 148, 128, 0, LP_ST>>>(ft, u, km, kpc, glist, gcount, g, modal_blocks);
  const ChebArgs a{x, r, d, b, dinv, coef};
  const int nb = lp_blocks(g.nodes_padded(), 256);
  if (mode == 1) k_explicit_gather_cheb<1><<<nb, 256, 0, LP_ST>>>(ft, mask, g, a);
  else if (mode == 2) k_explicit_gather_cheb<2><<<nb, 256, 0, LP_ST>>>(ft, mask, g, a);
  else k_explicit_gather_cheb<3><<<nb, 256, 0, LP_ST>>>(ft, mask, g, a);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_pack_sym_f32(float* kp, const float* k, long long ncells, void* stream) {
  if (!kp || !k || ncells < 0) return LP_ERR_ARG;
  k_pack_sym<float, float><<<lp_blocks(300 * ncells, 256), 256, 0, LP_ST>>>(kp, k, ncells);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

int lpb_pack_sym_f64(double* kp, const double* k, long long ncells, void* stream) {
  if (!kp || !k || ncells < 0) return LP_ERR_ARG;
  k_pack_sym<double, double><<<lp_blocks(300 * ncells, 256), 256, 0, LP_ST>>>(kp, k, ncells);
  LP_LAUNCH_CHECK();
  return LP_OK;
}

}  // extern "C"
