// tp_elem.cuh -- P1-tetrahedron element arithmetic shared by the assembly kernels.
//
// The element entries follow the reference kernel's operation order
// (gpu/gpu_assembler.py:104-132) with every product and sum rounded separately
// (__dmul_rn/__dadd_rn/__ddiv_rn: no FMA contraction), so that a row summed over its
// cells in ascending cell order equals the reference kernel executed in cell order.
#pragma once
#include "tp_common.cuh"

namespace tp {

struct GeoRec {
  double G00, G01, G02, G11, G12, G22, dJ;
};

__device__ __forceinline__ GeoRec load_geo(const double* __restrict__ geo, int64_t c) {
  const double4* g = reinterpret_cast<const double4*>(geo) + 2 * c;
  const double4 a = ldg_d4(g), b = ldg_d4(g + 1);
  return GeoRec{a.x, a.y, a.z, a.w, b.x, b.y, b.z};
}

// Row li of K / ((dJ De)/6), K_li,j for j = 0..3, in the reference's order
// (gpu_assembler.py:108-119): with reference gradients g_0 = (-1,-1,-1), g_k = e_{k-1},
// every product is exact and
//   Gg_j[a] = -((G[a][0] + G[a][1]) + G[a][2])  (j = 0),   G[a][j-1]  (j > 0)
//   K_ij    = -((Gg_j[0] + Gg_j[1]) + Gg_j[2])  (i = 0),   Gg_j[i-1]  (i > 0)
// G is symmetric, so the column sums of the first row are the row sums
// S[a] = (G[a][0] + G[a][1]) + G[a][2] (same operands, same order).  li is a runtime
// value: the row comes from selects, not from an indexed array (which would live in
// local memory).
__device__ __forceinline__ void kref_row(int li, const GeoRec& g, double k[4]) {
  const double S0 = __dadd_rn(__dadd_rn(g.G00, g.G01), g.G02);
  const double S1 = __dadd_rn(__dadd_rn(g.G01, g.G11), g.G12);
  const double S2 = __dadd_rn(__dadd_rn(g.G02, g.G12), g.G22);
  const double T = __dadd_rn(__dadd_rn(S0, S1), S2);
  const bool l0 = li == 0, l1 = li == 1, l2 = li == 2;
  k[0] = l0 ? T : -(l1 ? S0 : (l2 ? S1 : S2));
  k[1] = l0 ? -S0 : (l1 ? g.G00 : (l2 ? g.G01 : g.G02));
  k[2] = l0 ? -S1 : (l1 ? g.G01 : (l2 ? g.G11 : g.G12));
  k[3] = l0 ? -S2 : (l1 ? g.G02 : (l2 ? g.G12 : g.G22));
}

// Entry (i, j) of the cell's operator in the reference's rounding:
//   MODE FULL:  (K_ij (dJ De)/6) + ((inv_dt + alpha) M_ij)
//   MODE STIFF: K_ij (dJ De)/6
//   MODE MASS:  M_ij
// with M the lumped (dJ 5/120 on the diagonal) or consistent (dJ (1 + d_ij)/120) mass.
// kr = kref_row(i), ks = (dJ De)/6, react = inv_dt + alpha.  K and M are symmetric
// bit for bit (kref_row(i)[j] == kref_row(j)[i]), so entry (i, j) == entry (j, i).
template <int MODE>
__device__ __forceinline__ double elem_entry(const double kr[4], int i, int j, double dJ,
                                             double ks, double react, int lumped) {
  double a = 0.0;
  if (MODE != TP_ASM_MASS) a = __dmul_rn(kr[j], ks);
  if (MODE != TP_ASM_STIFF) {
    double M;
    if (lumped)
      M = (i == j) ? __ddiv_rn(__dmul_rn(dJ, 5.0), 120.0) : 0.0;
    else
      M = __ddiv_rn(__dmul_rn(dJ, (i == j) ? 2.0 : 1.0), 120.0);
    a = (MODE == TP_ASM_FULL) ? __dadd_rn(a, __dmul_rn(react, M)) : M;
  }
  return a;
}

// position of entry (i, j) in the 10 upper-triangle values of a symmetric 4x4 block,
// row by row: (0,0..3) 0-3, (1,1..3) 4-6, (2,2..3) 7-8, (3,3) 9
__device__ __forceinline__ int tri_index(int i, int j) {
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  return (lo == 0 ? 0 : (lo == 1 ? 4 : (lo == 2 ? 7 : 9))) + (hi - lo);
}

}  // namespace tp
