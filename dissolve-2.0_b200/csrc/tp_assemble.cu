// tp_assemble.cu -- per-step assembly of the P1-tet backward-Euler operators.
//
// Reference: gpu/gpu_assembler.py assembles with one thread per cell and 16 FP64
// atomicAdds into the CSR values (:60-139), one atomicAdd per vertex for the RHS
// (:176-221) and four for the nodal gradient (:251-304).  Here every output row is
// owned by one thread, which walks the row's incident cells (vertex->cell lists in
// ascending cell order) and accumulates in shared memory: no atomics, deterministic,
// and -- because the walk follows cell order and every product/sum is rounded
// separately (__dmul_rn/__dadd_rn, no FMA contraction) in the reference's operation
// order -- equal to the reference kernel executed in cell order.
#include <algorithm>
#include <mutex>

#include "tp_elem.cuh"
#include "tp_tiles.cuh"

namespace tp {

// ----------------------------------------------------------------- CSR assembly
// Optional extras of the same row walk (the stiffness of the batched step): the per-column
// lumped diagonal of tp_lumped_diag, and the FP32 values in SELL-32 order for the solver.
struct RowExtras {
  int S, ld;
  const double* alpha;  // (n_cells, ld) or NULL
  double4 shift;
  double* d64;
  float* d32;
  const int32_t* slice_ptr;  // with sell32: SELL-32 slice offsets (rows in CSR order)
  float* sell32;
};

// One thread per row; the block's rows are written back coalesced from shared memory.
// DIAG: the row also sums its lumped diagonal, in the order of k_lumped_diag.
template <int MODE, bool DIAG>
__global__ void __launch_bounds__(128) k_assemble_rows(
    int64_t nv, const int32_t* __restrict__ v2c_ptr, const int32_t* __restrict__ v2c,
    const uint32_t* __restrict__ slots, const double* __restrict__ geo,
    const double* __restrict__ De, const double* __restrict__ alpha, double inv_dt, int lumped,
    const uint8_t* __restrict__ bc_mask, const int32_t* __restrict__ indptr,
    const int32_t* __restrict__ indices, double* __restrict__ out64,
    float* __restrict__ out32, RowExtras ex) {
  constexpr int B = 128;
  // [max_row_len][B + 1]: the odd row stride puts consecutive slots of one row in
  // different banks (the write-back reads them with consecutive lanes); the walk's
  // accesses (one row per lane, the same slot on every lane of a structured mesh) stay
  // conflict-free
  constexpr int BS = B + 1;
  extern __shared__ double acc[];
  __shared__ int32_t s_ptr[B + 1];
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * B;
  const int64_t r = r0 + tid;
  const bool valid = r < nv;
  const int64_t rend = (r0 + B < nv) ? r0 + B : nv;
  const int nrows = (int)(rend - r0);
  if (tid < nrows) s_ptr[tid] = indptr[r0 + tid];
  if (tid == 0) s_ptr[nrows] = indptr[rend];
  __syncthreads();
  const int len = valid ? s_ptr[tid + 1] - s_ptr[tid] : 0;
  for (int s = 0; s < len; s++) acc[s * BS + tid] = 0.0;
  const bool is_bc = valid && bc_mask && bc_mask[r];
  double dacc[4] = {0.0, 0.0, 0.0, 0.0};
  const double dsh[4] = {ex.shift.x, ex.shift.y, ex.shift.z, ex.shift.w};
  if (valid && !is_bc) {
    // incident cells in ascending order, fetched PF at a time so their loads overlap;
    // accumulation stays in cell order
    constexpr int PF = 4;
    const int kbeg = v2c_ptr[r], kend = v2c_ptr[r + 1];
    for (int k0 = kbeg; k0 < kend; k0 += PF) {
      int32_t ev[PF];
      uint32_t sv[PF];
#pragma unroll
      for (int u = 0; u < PF; u++) {
        const bool ok = k0 + u < kend;
        ev[u] = ok ? __ldg(v2c + k0 + u) : 0;
        sv[u] = ok ? __ldg(slots + k0 + u) : 0u;
      }
      GeoRec gv[PF];
      double dev[PF], alv[PF];
#pragma unroll
      for (int u = 0; u < PF; u++) {
        const int64_t c = ev[u] >> 2;
        gv[u] = load_geo(geo, c);
        dev[u] = (MODE == TP_ASM_MASS) ? 0.0 : __ldg(De + c);
        alv[u] = (MODE == TP_ASM_FULL && alpha) ? __ldg(alpha + c) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < PF; u++) {
        if (k0 + u >= kend) break;
        const int li = ev[u] & 3;
        const GeoRec& g = gv[u];
        if constexpr (DIAG) {
          const int64_t c = ev[u] >> 2;
          const double Ld = __dmul_rn(__ddiv_rn(g.dJ, 120.0), 5.0);
#pragma unroll
          for (int s = 0; s < 4; s++) {
            if (s < ex.S) {
              const double w = __dadd_rn(dsh[s], ex.alpha ? ex.alpha[c * ex.ld + s] : 0.0);
              dacc[s] = __dadd_rn(dacc[s], __dmul_rn(w, Ld));
            }
          }
        }
        double kr[4];
        kref_row(li, g, kr);
        const double kscale = (MODE == TP_ASM_MASS) ? 0.0
                                                    : __ddiv_rn(__dmul_rn(g.dJ, dev[u]), 6.0);
        const double react = (MODE == TP_ASM_FULL) ? __dadd_rn(inv_dt, alv[u]) : 1.0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double a = elem_entry<MODE>(kr, li, j, g.dJ, kscale, react, lumped);
          const int slot = (sv[u] >> (8 * j)) & 0xff;
          if (slot < len) acc[slot * BS + tid] = __dadd_rn(acc[slot * BS + tid], a);
        }
      }
    }
  }
  if constexpr (DIAG) {
    if (valid) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        if (s < ex.ld) {
          const double v = is_bc ? 1.0 : (s < ex.S ? dacc[s] : 0.0);
          if (ex.d64) ex.d64[r * ex.ld + s] = v;
          if (ex.d32) ex.d32[r * ex.ld + s] = (float)v;
        }
      }
    }
  }
  __syncthreads();
  const int pbeg = s_ptr[0], pend = s_ptr[nrows];
  for (int p = pbeg + tid; p < pend; p += B) {
    int lo = 0, hi = nrows;  // find row: s_ptr[lo] <= p < s_ptr[lo+1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_ptr[mid] <= p)
        lo = mid;
      else
        hi = mid;
    }
    const int slot = p - s_ptr[lo];
    double v = acc[slot * BS + lo];
    if (bc_mask && bc_mask[r0 + lo]) v = (indices[p] == r0 + lo) ? 1.0 : 0.0;
    if (out64) out64[p] = v;
    if (out32) out32[p] = (float)v;
  }
  if (ex.sell32) {
    // SELL-32: the block's 128 rows are four whole slices; warp w writes slice r0/32 + w,
    // entry k of its lane's row at slice_ptr[slice] + 32 k + lane (padding entries 0), so
    // every store is one coalesced 128-byte line
    const int wsl = tid >> 5, ln = tid & 31;
    if (r0 + wsl * 32 < nv) {
      const int64_t sl = (r0 >> 5) + wsl;
      const int base = ex.slice_ptr[sl], width = (ex.slice_ptr[sl + 1] - base) >> 5;
      const int lr = wsl * 32 + ln;
      const bool rv = lr < nrows;
      const int rlen = rv ? s_ptr[lr + 1] - s_ptr[lr] : 0;
      const bool rbc = rv && bc_mask && bc_mask[r0 + lr];
      for (int k = 0; k < width; k++) {
        float f = 0.f;
        if (k < rlen) {
          double v = acc[k * BS + lr];
          if (rbc) v = (indices[s_ptr[lr] + k] == r0 + lr) ? 1.0 : 0.0;
          f = (float)v;
        }
        ex.sell32[base + k * 32 + ln] = f;
      }
    }
  }
}

// ----------------------------------------------------------------- tiled CSR assembly
// One CTA per row tile (tp_tiles.cu).  Phase A: the records of the tile's distinct cells
// are copied into shared memory with asynchronous copies, all in flight together; each
// cell's 10 upper-triangle entries (elem_entry, the reference's rounding) and, with DIAG,
// its S lumped-diagonal terms replace its record in place (odd slot stride: the cells the
// lanes of a warp read fall in different banks).  Phase B: each
// tile row sums its diagonal over its cells in ascending order, each owned edge sums its
// cells in ascending order, in registers, and writes (r, v) and (v, r) -- the same
// ordered sums as the row walk of k_assemble_rows, bit for bit.
constexpr int TILE_BLOCK = 256;

// Shared-memory slot of one cell: ew doubles, ew = 10 or 14 (80 or 112 bytes: 5 or 7
// sixteen-byte units, so 16-byte accesses of 8 consecutive slots fall in 8 different
// bank groups).  First the raw record as copied -- the 64-byte geometry record
// (G00 G01 G02 G11 G12 G22 |detJ| 0) at 0..7, De at 8, alpha at 9 or the DIAG alpha
// columns at 9..9+ld-1 -- then, computed in place by one thread, the 10 upper-triangle
// entries at 0..9 and, with DIAG, the S lumped-diagonal column terms at 10..10+S-1.
__device__ __forceinline__ void lds2(const double* p, double& a, double& b) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void sts2(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

// CMP (compact, DIAG without per-cell alpha): ew = 11, the slot keeps only the cell's
// lumped-mass factor Ld at 10 (each column's term shift_s Ld is formed where it is summed,
// with the same rounding); the odd stride leaves slots 8-byte aligned only, so every
// access is a single double.
template <int MODE, bool DIAG, bool CMP = false>
__device__ __forceinline__ void tile_cell_entries(double* slot, bool has_alpha, double inv_dt,
                                                  int lumped, const RowExtras& ex,
                                                  const double dsh[4]) {
  // the whole raw record first (the entries overwrite it)
  double r[10];
  if constexpr (CMP) {
#pragma unroll
    for (int k = 0; k < 10; k++) r[k] = slot[k];
  } else {
#pragma unroll
    for (int k = 0; k < 5; k++) lds2(slot + 2 * k, r[2 * k], r[2 * k + 1]);
  }
  double alc[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (DIAG && !CMP) {
    if (ex.alpha) {
      alc[0] = r[9];
#pragma unroll
      for (int s = 1; s < 4; s++)
        if (s < ex.ld) alc[s] = slot[9 + s];
    }
  }
  const GeoRec g{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
  const double de = (MODE == TP_ASM_MASS) ? 0.0 : r[8];
  const double al = (MODE == TP_ASM_FULL && has_alpha) ? r[9] : 0.0;
  const double ks = (MODE == TP_ASM_MASS) ? 0.0 : __ddiv_rn(__dmul_rn(g.dJ, de), 6.0);
  const double react = (MODE == TP_ASM_FULL) ? __dadd_rn(inv_dt, al) : 1.0;
  double e[10];
#pragma unroll
  for (int li = 0; li < 4; li++) {
    double kr[4];
    kref_row(li, g, kr);
#pragma unroll
    for (int j = li; j < 4; j++)
      e[tri_index(li, j)] = elem_entry<MODE>(kr, li, j, g.dJ, ks, react, lumped);
  }
  if constexpr (CMP) {
#pragma unroll
    for (int k = 0; k < 10; k++) slot[k] = e[k];
  } else {
#pragma unroll
    for (int k = 0; k < 5; k++) sts2(slot + 2 * k, e[2 * k], e[2 * k + 1]);
  }
  if constexpr (DIAG && CMP) {
    slot[10] = __dmul_rn(__ddiv_rn(g.dJ, 120.0), 5.0);
  } else if constexpr (DIAG) {
    const double Ld = __dmul_rn(__ddiv_rn(g.dJ, 120.0), 5.0);
    double dt[4];
#pragma unroll
    for (int s = 0; s < 4; s++)
      dt[s] = (s < ex.S) ? __dmul_rn(__dadd_rn(dsh[s], alc[s]), Ld) : 0.0;
    sts2(slot + 10, dt[0], dt[1]);
    sts2(slot + 12, dt[2], dt[3]);
  }
}

__device__ __forceinline__ void sell_put(const RowExtras& ex, int64_t row, int slot, float v) {
  const int64_t sl = row >> 5;
  ex.sell32[ex.slice_ptr[sl] + (int64_t)slot * 32 + (row & 31)] = v;
}

// term k (0..7) of 8 packed 16-bit terms
__device__ __forceinline__ uint32_t term_of(const uint4& v, int k) {
  const uint32_t w = (k < 2) ? v.x : (k < 4) ? v.y : (k < 6) ? v.z : v.w;
  return (k & 1) ? (w >> 16) : (w & 0xffffu);
}

template <int MODE, bool DIAG, bool CMP = false>
__global__ void __launch_bounds__(TILE_BLOCK, 3) k_assemble_tiles(
    TileView tv, const double* __restrict__ geo, const double* __restrict__ De,
    const double* __restrict__ alpha, double inv_dt, int lumped,
    const uint8_t* __restrict__ bc_mask, const int32_t* __restrict__ indptr,
    double* __restrict__ out64, float* __restrict__ out32, RowExtras ex, int ew, int64_t nv) {
  extern __shared__ double sm_tiles[];
  const int R = tv.R, T = blockDim.x;
  const int t = blockIdx.x, tid = threadIdx.x;
  const int c0 = __ldg(tv.cell_ptr + t), m = __ldg(tv.cell_ptr + t + 1) - c0;
  double* E = sm_tiles;
  const double dsh[4] = {ex.shift.x, ex.shift.y, ex.shift.z, ex.shift.w};
  const uint4 none4 = make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);

  // ---- phase A: every record of the tile copied into shared memory at once: the ids
  // first, then the 64-byte geometry records as 16-byte chunks (four lanes per record,
  // consecutive records on consecutive lanes), De and alpha as 8-byte copies ...
  {
    constexpr int MAXC = 4;
    const int lane = tid & 31;
    int64_t cid[MAXC];
#pragma unroll
    for (int u = 0; u < MAXC; u++) {
      const int i = tid + u * T;
      cid[u] = (i < m) ? (int64_t)__ldg(tv.cells + c0 + i) : -1;
    }
#pragma unroll
    for (int u = 0; u < MAXC; u++) {
      const int ib = (tid & ~31) + u * T;  // the warp's first cell of this round
      if (ib >= m) break;
      const int h = lane & 3;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int j = (lane >> 2) + 8 * k;
        const int64_t c = __shfl_sync(0xffffffffu, cid[u], j);
        if (ib + j < m) {
          if constexpr (CMP) {
            cp_async<8>(E + (size_t)(ib + j) * ew + 2 * h, geo + 8 * c + 2 * h);
            cp_async<8>(E + (size_t)(ib + j) * ew + 2 * h + 1, geo + 8 * c + 2 * h + 1);
          } else {
            cp_async<16>(E + (size_t)(ib + j) * ew + 2 * h, geo + 8 * c + 2 * h);
          }
        }
      }
      if (cid[u] >= 0) {
        double* slot = E + (size_t)(ib + lane) * ew;
        const int64_t c = cid[u];
        if (MODE != TP_ASM_MASS) cp_async<8>(slot + 8, De + c);
        if (MODE == TP_ASM_FULL && alpha) cp_async<8>(slot + 9, alpha + c);
        if constexpr (DIAG && !CMP) {
          if (ex.alpha)
            for (int s = 0; s < ex.ld; s++) cp_async<8>(slot + 9 + s, ex.alpha + c * ex.ld + s);
        }
      }
    }
    for (int i = tid + MAXC * T; i < m; i += T) {  // tiles of more than MAXC * T cells
      const int64_t c = __ldg(tv.cells + c0 + i);
      double* slot = E + (size_t)i * ew;
      if constexpr (CMP) {
#pragma unroll
        for (int h = 0; h < 8; h++) cp_async<8>(slot + h, geo + 8 * c + h);
      } else {
#pragma unroll
        for (int h = 0; h < 4; h++) cp_async<16>(slot + 2 * h, geo + 8 * c + 2 * h);
      }
      if (MODE != TP_ASM_MASS) cp_async<8>(slot + 8, De + c);
      if (MODE == TP_ASM_FULL && alpha) cp_async<8>(slot + 9, alpha + c);
      if constexpr (DIAG && !CMP) {
        if (ex.alpha)
          for (int s = 0; s < ex.ld; s++) cp_async<8>(slot + 9 + s, ex.alpha + c * ex.ld + s);
      }
    }
  }
  // ... while they fly, the phase-B inputs of this thread: its row's first 24 diagonal
  // terms and its first two edges with their first 8 terms ...
  int64_t r = -1;
  int pd = 0, KD = 0;
  const uint4* dv = nullptr;
  uint4 dq[3] = {none4, none4, none4};
  if (tid < R) {
    r = __ldg(tv.rows + (int64_t)t * R + tid);
    pd = __ldg(tv.diag_pos + (int64_t)t * R + tid);
    const int d0 = __ldg(tv.dterm_ptr + t);
    KD = (__ldg(tv.dterm_ptr + t + 1) - d0) / R;
    dv = reinterpret_cast<const uint4*>(tv.dterms + d0 + (int64_t)tid * KD);
#pragma unroll
    for (int u = 0; u < 3; u++)
      if (8 * u < KD) dq[u] = __ldg(dv + u);
  }
  const int eb = __ldg(tv.edge_ptr + t), ne = __ldg(tv.edge_ptr + t + 1) - eb;
  const int tb = __ldg(tv.eterm_ptr + t);
  const int KE = ne ? (__ldg(tv.eterm_ptr + t + 1) - tb) / ne : 0;
  // the diagonal threads take the last edges of a round, the others the first
  const int q0 = (tid >= R) ? tid - R : T - R + tid;
  int2 ep[2];
  uint4 eq[2] = {none4, none4};
#pragma unroll
  for (int u = 0; u < 2; u++) {
    const int q = q0 + u * T;
    if (q < ne) {
      ep[u] = __ldg(tv.edge_pos + eb + q);
      eq[u] = __ldg(reinterpret_cast<const uint4*>(tv.eterms + tb + (int64_t)q * KE));
    }
  }
  // ... and each thread turns the records it copied into element entries in place
  cp_async_wait_all();
  for (int i = tid; i < m; i += T)
    tile_cell_entries<MODE, DIAG, CMP>(E + (size_t)i * ew, alpha != nullptr, inv_dt, lumped, ex,
                                       dsh);
  __syncthreads();

  // ---- phase B1: the diagonal of each tile row
  if (tid < R && r >= 0) {
    const bool is_bc = bc_mask && bc_mask[r];
    double dacc = 0.0, dg[4] = {0.0, 0.0, 0.0, 0.0};
    if (!is_bc) {
      auto group = [&](const uint4& g8) -> bool {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint32_t tm = term_of(g8, k);
          if (tm == TILE_TERM_NONE) return false;
          const int loc = tm & ((1 << TILE_LOC_BITS) - 1), li = tm >> TILE_LOC_BITS;
          const double* e = E + (size_t)loc * ew;
          dacc = __dadd_rn(dacc, e[tri_index(li, li)]);
          if constexpr (DIAG && CMP) {
            // the term tile_cell_entries forms without per-cell alpha, (shift_s + 0) Ld
#pragma unroll
            for (int s = 0; s < 4; s++)
              if (s < ex.S) dg[s] = __dadd_rn(dg[s], __dmul_rn(__dadd_rn(dsh[s], 0.0), e[10]));
          } else if constexpr (DIAG) {
#pragma unroll
            for (int s = 0; s < 4; s++)
              if (s < ex.S) dg[s] = __dadd_rn(dg[s], e[10 + s]);
          }
        }
        return true;
      };
      bool more = group(dq[0]) && group(dq[1]) && group(dq[2]);
      for (int g = 3; more && 8 * g < KD; g++) more = group(__ldg(dv + g));
    }
    const double v = is_bc ? 1.0 : dacc;
    if (out64) out64[pd] = v;
    if (out32) out32[pd] = (float)v;
    if (ex.sell32) {
      // the diagonal, then the row's padding entries of its SELL-32 slice
      const int p0 = __ldg(indptr + r), len = __ldg(indptr + r + 1) - p0;
      const int64_t sl = r >> 5;
      const int base = ex.slice_ptr[sl], width = (ex.slice_ptr[sl + 1] - base) >> 5;
      float* col = ex.sell32 + base + (r & 31);
      col[(int64_t)(pd - p0) * 32] = (float)v;
      for (int k = len; k < width; k++) col[(int64_t)k * 32] = 0.f;
    }
    if constexpr (DIAG) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        if (s < ex.ld) {
          const double dv2 = is_bc ? 1.0 : (s < ex.S ? dg[s] : 0.0);
          if (ex.d64) ex.d64[r * ex.ld + s] = dv2;
          if (ex.d32) ex.d32[r * ex.ld + s] = (float)dv2;
        }
      }
    }
  }

  // ---- phase B2: the tile's edges, (r, v) and (v, r) from one ordered sum
  auto edge = [&](int q, int2 pp, const uint4& g0) {
    double acc = 0.0;
    auto group = [&](const uint4& g8) -> bool {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t tm = term_of(g8, k);
        if (tm == TILE_TERM_NONE) return false;
        const int loc = tm & ((1 << TILE_LOC_BITS) - 1), tq = tm >> TILE_LOC_BITS;
        acc = __dadd_rn(acc, E[(size_t)loc * ew + tq]);
      }
      return true;
    };
    bool more = group(g0);
    for (int g = 1; more && 8 * g < KE; g++)
      more = group(__ldg(reinterpret_cast<const uint4*>(tv.eterms + tb + (int64_t)q * KE) + g));
    double a_rv = acc, a_vr = acc;
    if (bc_mask || ex.sell32) {
      const int2 rv = __ldg(tv.edge_rv + eb + q);
      if (bc_mask) {
        if (bc_mask[rv.x]) a_rv = 0.0;
        if (bc_mask[rv.y]) a_vr = 0.0;
      }
      if (ex.sell32) {
        sell_put(ex, rv.x, pp.x - __ldg(indptr + rv.x), (float)a_rv);
        sell_put(ex, rv.y, pp.y - __ldg(indptr + rv.y), (float)a_vr);
      }
    }
    if (out64) {
      out64[pp.x] = a_rv;
      out64[pp.y] = a_vr;
    }
    if (out32) {
      out32[pp.x] = (float)a_rv;
      out32[pp.y] = (float)a_vr;
    }
  };
  if (q0 < ne) edge(q0, ep[0], eq[0]);
  if (q0 + T < ne) edge(q0 + T, ep[1], eq[1]);
  for (int q = q0 + 2 * T; q < ne; q += T)
    edge(q, __ldg(tv.edge_pos + eb + q),
         __ldg(reinterpret_cast<const uint4*>(tv.eterms + tb + (int64_t)q * KE)));
  if (ex.sell32 && t == 0 && (nv & 31)) {
    // the lanes of the last slice past the last row: padding, 0
    const int64_t sl = nv >> 5;
    const int base = ex.slice_ptr[sl], width = (ex.slice_ptr[sl + 1] - base) >> 5;
    for (int q = tid; q < width * 32; q += T)
      if ((q & 31) >= (nv & 31)) ex.sell32[base + q] = 0.f;
  }
}

// gpu_assembler.py:147-165
__global__ void k_dirichlet_rows(int64_t n_bc, const int32_t* __restrict__ bc, int64_t nv,
                                 const int32_t* __restrict__ indptr,
                                 const int32_t* __restrict__ indices, double* __restrict__ data) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_bc) return;
  const int row = bc[k];
  if (row < 0 || row >= nv) return;
  for (int j = indptr[row]; j < indptr[row + 1]; j++) data[j] = (indices[j] == row) ? 1.0 : 0.0;
}

__global__ void k_bc_mask(int64_t n_bc, const int32_t* __restrict__ bc, int64_t nv,
                          uint8_t* __restrict__ mask, int32_t* __restrict__ flags) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_bc) return;
  const int v = bc[k];
  if (v < 0 || v >= nv) {
    atomicOr(flags, FLAG_BCINDEX);
    return;
  }
  mask[v] = 1;
}

// gpu_assembler.py:465-466: d[elem_nodes].reshape(n, 4).mean(axis=1)
__global__ void k_cell_average(int64_t n, const int4* __restrict__ cells,
                               const double* __restrict__ vv, double* __restrict__ out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const double s = __dadd_rn(__dadd_rn(__dadd_rn(vv[v.x], vv[v.y]), vv[v.z]), vv[v.w]);
    out[c] = __ddiv_rn(s, 4.0);
  }
}

// lumped diagonal per column (no reference counterpart on its own: the lumped mass +
// reaction terms of gpu_assembler.py:122-132 for the split operator)
__global__ void k_lumped_diag(int64_t nv, int S, int ld, const int32_t* __restrict__ v2c_ptr,
                              const int32_t* __restrict__ v2c, const double* __restrict__ geo,
                              const double* __restrict__ alpha, double4 shift,
                              const uint8_t* __restrict__ bc_mask, double* __restrict__ d64,
                              float* __restrict__ d32) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
       r += (int64_t)gridDim.x * blockDim.x) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const double sh[4] = {shift.x, shift.y, shift.z, shift.w};
    const bool is_bc = bc_mask && bc_mask[r];
    if (!is_bc) {
      constexpr int PF = 8;
      const int kbeg = v2c_ptr[r], kend = v2c_ptr[r + 1];
      for (int k0 = kbeg; k0 < kend; k0 += PF) {
        int64_t cv[PF];
        double dJ[PF];
#pragma unroll
        for (int u = 0; u < PF; u++) cv[u] = (k0 + u < kend) ? (v2c[k0 + u] >> 2) : 0;
#pragma unroll
        for (int u = 0; u < PF; u++) dJ[u] = geo[8 * cv[u] + 6];
#pragma unroll
        for (int u = 0; u < PF; u++) {
          if (k0 + u >= kend) break;
          const double Ld = __dmul_rn(__ddiv_rn(dJ[u], 120.0), 5.0);
#pragma unroll
          for (int s = 0; s < 4; s++) {
            if (s < S) {
              const double w = __dadd_rn(sh[s], alpha ? alpha[cv[u] * ld + s] : 0.0);
              acc[s] = __dadd_rn(acc[s], __dmul_rn(w, Ld));
            }
          }
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; s++) {
      if (s < ld) {
        const double v = is_bc ? 1.0 : (s < S ? acc[s] : 0.0);
        if (d64) d64[r * ld + s] = v;
        if (d32) d32[r * ld + s] = (float)v;
      }
    }
  }
}

// ----------------------------------------------------------------- RHS
// gpu_assembler.py:176-221 row-gathered; columns interleaved with stride ld
__global__ void k_rhs_rows(int64_t nv, int S, int ld, const int32_t* __restrict__ cells,
                           const int32_t* __restrict__ v2c_ptr, const int32_t* __restrict__ v2c,
                           const double* __restrict__ geo, const double* __restrict__ u,
                           const double* __restrict__ f, double inv_dt, int lumped,
                           double* __restrict__ b) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
       r += (int64_t)gridDim.x * blockDim.x) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    double ur[4], fr[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      ur[s] = (s < S) ? u[r * ld + s] : 0.0;
      fr[s] = (s < S && f) ? f[r * ld + s] : 0.0;
    }
    constexpr int PF = 8;
    const int kbeg = v2c_ptr[r], kend = v2c_ptr[r + 1];
    for (int k0 = kbeg; k0 < kend; k0 += PF) {
      int64_t cvv[PF];
      double dJv[PF];
#pragma unroll
      for (int q = 0; q < PF; q++) cvv[q] = (k0 + q < kend) ? (v2c[k0 + q] >> 2) : 0;
#pragma unroll
      for (int q = 0; q < PF; q++) dJv[q] = geo[8 * cvv[q] + 6];
#pragma unroll
      for (int q = 0; q < PF; q++) {
        if (k0 + q >= kend) break;
        const int64_t c = cvv[q];
        const double base = __ddiv_rn(dJv[q], 120.0);
        if (lumped) {
          const double Ld = __dmul_rn(base, 5.0);
#pragma unroll
          for (int s = 0; s < 4; s++)
            if (s < S)
              acc[s] = __dadd_rn(acc[s],
                                 __dmul_rn(Ld, __dadd_rn(__dmul_rn(inv_dt, ur[s]), fr[s])));
        } else {
          const int4 cv = reinterpret_cast<const int4*>(cells)[c];
          const double mdt = __dmul_rn(base, inv_dt);
#pragma unroll
          for (int s = 0; s < 4; s++) {
            if (s >= S) continue;
            const double su = __dadd_rn(
                __dadd_rn(__dadd_rn(u[(int64_t)cv.x * ld + s], u[(int64_t)cv.y * ld + s]),
                          u[(int64_t)cv.z * ld + s]),
                u[(int64_t)cv.w * ld + s]);
            double sf = 0.0;
            if (f)
              sf = __dadd_rn(
                  __dadd_rn(__dadd_rn(f[(int64_t)cv.x * ld + s], f[(int64_t)cv.y * ld + s]),
                            f[(int64_t)cv.z * ld + s]),
                  f[(int64_t)cv.w * ld + s]);
            acc[s] = __dadd_rn(acc[s], __dadd_rn(__dmul_rn(mdt, __dadd_rn(su, ur[s])),
                                                 __dmul_rn(base, __dadd_rn(sf, fr[s]))));
          }
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; s++)
      if (s < ld) b[r * ld + s] = (s < S) ? acc[s] : 0.0;
  }
}

// Right-hand side on row tiles: the tile's cells' factors in shared memory, then each
// tile row sums its cells in ascending order -- the same ordered sums, with the same
// rounding, as k_rhs_rows.  Lumped: one slot per cell, Ld = (|detJ| / 120) 5, and the row
// adds Ld (inv_dt u + f).  Consistent: a slot of CW = 6 (10 with f) doubles per cell,
// [base dt^-1, base, sum of u over the cell's vertices (4 columns), the same for f], base =
// |detJ| / 120, and the row adds base dt^-1 (su + u_r) + base (sf + f_r).
template <bool LUMPED>
__global__ void __launch_bounds__(256) k_rhs_tiles(TileView tv, int S, int ld,
                                                   const int32_t* __restrict__ cells,
                                                   const double* __restrict__ geo,
                                                   const double* __restrict__ u,
                                                   const double* __restrict__ f, double inv_dt,
                                                   double* __restrict__ b) {
  extern __shared__ double sm_ld[];
  const int R = tv.R, T = blockDim.x, t = blockIdx.x, tid = threadIdx.x;
  const int c0 = __ldg(tv.cell_ptr + t), m = __ldg(tv.cell_ptr + t + 1) - c0;
  const int CW = LUMPED ? 1 : (f ? 10 : 6);
  {
    constexpr int MAXC = 4;
    int64_t cid[MAXC];
    double dj[MAXC];
    int4 cv[MAXC];
#pragma unroll
    for (int k = 0; k < MAXC; k++) {
      const int i = tid + k * T;
      cid[k] = (i < m) ? (int64_t)__ldg(tv.cells + c0 + i) : -1;
    }
#pragma unroll
    for (int k = 0; k < MAXC; k++) {
      dj[k] = (cid[k] >= 0) ? __ldg(geo + 8 * cid[k] + 6) : 0.0;
      if constexpr (!LUMPED)
        cv[k] = (cid[k] >= 0) ? __ldg(reinterpret_cast<const int4*>(cells) + cid[k])
                              : make_int4(0, 0, 0, 0);
    }
    auto put = [&](int i, double djv, const int4& c4) {
      double* slot = sm_ld + (size_t)i * CW;
      if constexpr (LUMPED) {
        slot[0] = __dmul_rn(__ddiv_rn(djv, 120.0), 5.0);
      } else {
        const double base = __ddiv_rn(djv, 120.0);
        slot[0] = __dmul_rn(base, inv_dt);
        slot[1] = base;
#pragma unroll
        for (int s = 0; s < 4; s++) {
          if (s >= S) break;
          slot[2 + s] = __dadd_rn(
              __dadd_rn(__dadd_rn(__ldg(u + (int64_t)c4.x * ld + s), __ldg(u + (int64_t)c4.y * ld + s)),
                        __ldg(u + (int64_t)c4.z * ld + s)),
              __ldg(u + (int64_t)c4.w * ld + s));
          if (f)
            slot[6 + s] = __dadd_rn(
                __dadd_rn(__dadd_rn(__ldg(f + (int64_t)c4.x * ld + s), __ldg(f + (int64_t)c4.y * ld + s)),
                          __ldg(f + (int64_t)c4.z * ld + s)),
                __ldg(f + (int64_t)c4.w * ld + s));
        }
      }
    };
#pragma unroll
    for (int k = 0; k < MAXC; k++)
      if (cid[k] >= 0) put(tid + k * T, dj[k], cv[k]);
    for (int i = tid + MAXC * T; i < m; i += T) {
      const int64_t c = __ldg(tv.cells + c0 + i);
      put(i, __ldg(geo + 8 * c + 6),
          LUMPED ? make_int4(0, 0, 0, 0) : __ldg(reinterpret_cast<const int4*>(cells) + c));
    }
  }
  // the row's first 24 terms and its u, f are loaded before the barrier (in flight with
  // the loads above)
  int64_t r = -1;
  double w[4] = {0.0, 0.0, 0.0, 0.0}, fr[4] = {0.0, 0.0, 0.0, 0.0};
  const uint4* dv = nullptr;
  int KD = 0;
  const uint4 none4 = make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);
  uint4 dq[3] = {none4, none4, none4};
  if (tid < R) {
    r = __ldg(tv.rows + (int64_t)t * R + tid);
    const int d0 = __ldg(tv.dterm_ptr + t);
    KD = (__ldg(tv.dterm_ptr + t + 1) - d0) / R;
    dv = reinterpret_cast<const uint4*>(tv.dterms + d0 + (int64_t)tid * KD);
#pragma unroll
    for (int g = 0; g < 3; g++)
      if (8 * g < KD) dq[g] = __ldg(dv + g);
    if (r >= 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        if (s >= S) continue;
        if constexpr (LUMPED) {
          w[s] = __dadd_rn(__dmul_rn(inv_dt, u[r * ld + s]), f ? f[r * ld + s] : 0.0);
        } else {
          w[s] = u[r * ld + s];  // u_r
          fr[s] = f ? f[r * ld + s] : 0.0;
        }
      }
    }
  }
  __syncthreads();
  if (r < 0) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  auto group = [&](const uint4& g8) -> bool {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t tm = term_of(g8, k);
      if (tm == TILE_TERM_NONE) return false;
      const double* slot = sm_ld + (size_t)(tm & ((1 << TILE_LOC_BITS) - 1)) * CW;
      if constexpr (LUMPED) {
        const double Ld = slot[0];
#pragma unroll
        for (int s = 0; s < 4; s++)
          if (s < S) acc[s] = __dadd_rn(acc[s], __dmul_rn(Ld, w[s]));
      } else {
        const double mdt = slot[0], base = slot[1];
#pragma unroll
        for (int s = 0; s < 4; s++) {
          if (s >= S) continue;
          const double sf = f ? slot[6 + s] : 0.0;
          acc[s] = __dadd_rn(acc[s], __dadd_rn(__dmul_rn(mdt, __dadd_rn(slot[2 + s], w[s])),
                                               __dmul_rn(base, __dadd_rn(sf, fr[s]))));
        }
      }
    }
    return true;
  };
  bool more = group(dq[0]) && group(dq[1]) && group(dq[2]);
  for (int g = 3; more && 8 * g < KD; g++) more = group(__ldg(dv + g));
#pragma unroll
  for (int s = 0; s < 4; s++)
    if (s < ld) b[r * ld + s] = (s < S) ? acc[s] : 0.0;
}

// lumped right-hand side from the per-vertex lumped mass: b = m (inv_dt u + f) per column
__global__ void k_lumped_rhs(int64_t nv, int S, int ld, const double* __restrict__ mass,
                             const double* __restrict__ u, const double* __restrict__ f,
                             double inv_dt, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv * ld;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = i / ld;
    const int s = (int)(i - v * ld);
    double r = 0.0;
    if (s < S) r = __dmul_rn(mass[v], __dadd_rn(__dmul_rn(inv_dt, u[i]), f ? f[i] : 0.0));
    b[i] = r;
  }
}

// gpu_assembler.py:228-239
__global__ void k_rhs_bc(int64_t n_bc, const int32_t* __restrict__ bc, int64_t nv, int S,
                         int ld, double4 val, double* __restrict__ b) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_bc) return;
  const int64_t v0 = bc[k];
  if (v0 < 0 || v0 >= nv) return;  // ids are validated by tp_bc_mask; never write outside b
  const double v[4] = {val.x, val.y, val.z, val.w};
  for (int s = 0; s < S; s++) b[v0 * ld + s] = v[s];
}

// ----------------------------------------------------------------- nodal gradient
// gpu_assembler.py:251-304 + :672, row-gathered
__global__ void k_nodal_gradient(int64_t nv, const int32_t* __restrict__ cells,
                                 const int32_t* __restrict__ v2c_ptr,
                                 const int32_t* __restrict__ v2c, const double* __restrict__ geo,
                                 const double* __restrict__ JinvT,
                                 const double* __restrict__ coords4, const double* __restrict__ u,
                                 double* __restrict__ grad) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
       r += (int64_t)gridDim.x * blockDim.x) {
    double gx = 0.0, gy = 0.0, gz = 0.0, ws = 0.0;
    for (int k = v2c_ptr[r]; k < v2c_ptr[r + 1]; k++) {
      const int64_t c = v2c[k] >> 2;
      const int4 cv = reinterpret_cast<const int4*>(cells)[c];
      const double u0 = u[cv.x], u1 = u[cv.y], u2 = u[cv.z], u3 = u[cv.w];
      const double g0 = __dadd_rn(-u0, u1), g1 = __dadd_rn(-u0, u2), g2 = __dadd_rn(-u0, u3);
      double JT[9];
      if (JinvT) {
#pragma unroll
        for (int q = 0; q < 9; q++) JT[q] = JinvT[9 * c + q];
      } else {
        const double4* X = reinterpret_cast<const double4*>(coords4);
        const double4 x0 = X[cv.x], x1 = X[cv.y], x2 = X[cv.z], x3 = X[cv.w];
        const double e[3][3] = {{x1.x - x0.x, x1.y - x0.y, x1.z - x0.z},
                                {x2.x - x0.x, x2.y - x0.y, x2.z - x0.z},
                                {x3.x - x0.x, x3.y - x0.y, x3.z - x0.z}};
        double cr[3][3];
        cr[0][0] = e[1][1] * e[2][2] - e[1][2] * e[2][1];
        cr[0][1] = e[1][2] * e[2][0] - e[1][0] * e[2][2];
        cr[0][2] = e[1][0] * e[2][1] - e[1][1] * e[2][0];
        cr[1][0] = e[2][1] * e[0][2] - e[2][2] * e[0][1];
        cr[1][1] = e[2][2] * e[0][0] - e[2][0] * e[0][2];
        cr[1][2] = e[2][0] * e[0][1] - e[2][1] * e[0][0];
        cr[2][0] = e[0][1] * e[1][2] - e[0][2] * e[1][1];
        cr[2][1] = e[0][2] * e[1][0] - e[0][0] * e[1][2];
        cr[2][2] = e[0][0] * e[1][1] - e[0][1] * e[1][0];
        const double inv =
            1.0 / (e[0][0] * cr[0][0] + e[0][1] * cr[0][1] + e[0][2] * cr[0][2]);
        // J^-T[a][b] = J^-1[b][a] = cr[b][a] / det
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int bb = 0; bb < 3; bb++) JT[3 * a + bb] = cr[bb][a] * inv;
      }
      const double px = __dadd_rn(__dadd_rn(__dmul_rn(JT[0], g0), __dmul_rn(JT[1], g1)),
                                  __dmul_rn(JT[2], g2));
      const double py = __dadd_rn(__dadd_rn(__dmul_rn(JT[3], g0), __dmul_rn(JT[4], g1)),
                                  __dmul_rn(JT[5], g2));
      const double pz = __dadd_rn(__dadd_rn(__dmul_rn(JT[6], g0), __dmul_rn(JT[7], g1)),
                                  __dmul_rn(JT[8], g2));
      const double w = __ddiv_rn(geo[8 * c + 6], 6.0);
      gx = __dadd_rn(gx, __dmul_rn(w, px));
      gy = __dadd_rn(gy, __dmul_rn(w, py));
      gz = __dadd_rn(gz, __dmul_rn(w, pz));
      ws = __dadd_rn(ws, w);
    }
    grad[3 * r + 0] = __ddiv_rn(gx, ws);
    grad[3 * r + 1] = __ddiv_rn(gy, ws);
    grad[3 * r + 2] = __ddiv_rn(gz, ws);
  }
}

// ----------------------------------------------------------------- scaffold volume
// gpu_assembler.py:605-644: sum_c mean_q H_eps(phi_q) |detJ|/6, deterministic two-level
__global__ void k_scaffold_volume(int64_t n, const int4* __restrict__ cells,
                                  const double* __restrict__ geo, const double* __restrict__ phi,
                                  double eps, double qa, double qb, double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  const double pi = 3.141592653589793;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const double p[4] = {phi[v.x], phi[v.y], phi[v.z], phi[v.w]};
    const double ps = ((p[0] + p[1]) + p[2]) + p[3];
    double hs = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double pq = (qa - qb) * p[q] + qb * ps;
      double h;
      if (pq < -eps)
        h = 0.0;
      else if (pq > eps)
        h = 1.0;
      else
        h = 0.5 * (1.0 + pq / eps + sin(pi * pq / eps) / pi);
      hs += h;
    }
    s += (hs / 4.0) * (geo[8 * c + 6] / 6.0);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_sum_parts(int n, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *out = s;
}

// ----------------------------------------------------------------- species coefficients
__device__ __forceinline__ double delta_eps(double phi, double eps) {
  const double pi = 3.141592653589793;
  return (fabs(phi) < eps) ? (1.0 / (2.0 * eps)) * (1.0 + cos(pi * phi / eps)) : 0.0;
}

__global__ void k_o2_alpha(int64_t n, const double* __restrict__ phi,
                           const double* __restrict__ ng, double eps, double k_orr,
                           double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = delta_eps(phi[i], eps) * ng[i] * k_orr;
}

__global__ void k_oh_source(int64_t n, const double* __restrict__ phi,
                            const double* __restrict__ ng, const double* __restrict__ F,
                            const double* __restrict__ Cl, const double* __restrict__ O2,
                            double eps, double kd, double k_orr, double fac,
                            double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double medium = (phi[i] <= 0.0) ? 1.0 : 0.0;
    out[i] = medium * kd * F[i] * (Cl[i] * Cl[i]) +
             fac * delta_eps(phi[i], eps) * ng[i] * k_orr * O2[i];
  }
}


// ----------------------------------------------------------------- coupled gyroid step
// Smoothed Heaviside of the scaffold indicator (the integrand of tp_scaffold_volume).
__device__ __forceinline__ double heaviside_eps(double phi, double eps) {
  const double pi = 3.141592653589793;
  if (phi < -eps) return 0.0;
  if (phi > eps) return 1.0;
  return 0.5 * (1.0 + phi / eps + sin(pi * phi / eps) / pi);
}

// hv = k_orr H_eps(phi); ngphi = |grad phi| (grad may be NULL); f[:, col_oh] = orr_factor
// hv U[:, col_o2], other columns of f zero
__global__ void k_interface_terms(int64_t n, const double* __restrict__ phi,
                                  const double* __restrict__ grad, double eps, double k_orr,
                                  double orr_factor, int ld, const double* __restrict__ U,
                                  int col_o2, int col_oh, double* __restrict__ f,
                                  double* __restrict__ hv, double* __restrict__ ngphi) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double h = k_orr * heaviside_eps(phi[i], eps);
    if (hv) hv[i] = h;
    if (ngphi && grad) {
      const double gx = grad[3 * i], gy = grad[3 * i + 1], gz = grad[3 * i + 2];
      ngphi[i] = sqrt(gx * gx + gy * gy + gz * gz);
    }
    if (f) {
      for (int s = 0; s < ld; s++) f[i * ld + s] = 0.0;
      f[i * ld + col_oh] = orr_factor * h * U[i * ld + col_o2];
    }
  }
}

// out[c, col] (leading dim ld) = mean of the 4 vertex values (gpu_assembler.py:465-466)
__global__ void k_cell_average_col(int64_t n, const int4* __restrict__ cells,
                                   const double* __restrict__ vv, int ld, int col,
                                   double* __restrict__ out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const double s = __dadd_rn(__dadd_rn(__dadd_rn(vv[v.x], vv[v.y]), vv[v.z]), vv[v.w]);
    out[c * ld + col] = __ddiv_rn(s, 4.0);
  }
}

// phi -= dt rate (1 + gain U[:, col])
__global__ void k_levelset_advance(int64_t n, double* __restrict__ phi, int ld,
                                   const double* __restrict__ U, int col, double dt, double rate,
                                   double gain) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    phi[i] -= dt * rate * (1.0 + gain * U[i * ld + col]);
}


// ----------------------------------------------------------------- film / Zn / level set
// interface_velocity.py:90-155 (compute_effective_diffusion), per vertex:
//   sat = clip(F / max(Fmax, 1e-20), 0, 1), ff = (1 - sat) + sat floor,
//   De_Zn = D_Zn ff, De_s = D_s ff [phi <= 0] for Cl-, OH-, O2;
// flags |= 1 on a non-finite result, 2 on a negative one
__global__ void k_effective_diffusion(int64_t n, const double* __restrict__ phi,
                                      const double* __restrict__ F, double Fmax, double floor_,
                                      double4 d0, double* __restrict__ zn, double* __restrict__ cl,
                                      double* __restrict__ oh, double* __restrict__ o2,
                                      int32_t* __restrict__ flags) {
  const double fm = fmax(Fmax, 1e-20);
  int bad = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = F[i] / fm;
    const double sat = (x < 0.0) ? 0.0 : ((x > 1.0) ? 1.0 : x);  // clip; NaN stays NaN
    const double ff = (1.0 - sat) + sat * floor_;
    const double med = (phi[i] <= 0.0) ? 1.0 : 0.0;
    const double v[4] = {d0.x * ff, d0.y * ff * med, d0.z * ff * med, d0.w * ff * med};
    double* out[4] = {zn, cl, oh, o2};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (!isfinite(v[k])) bad |= 1;
      if (v[k] < 0.0) bad |= 2;
      if (out[k]) out[k][i] = v[k];
    }
  }
  if (bad) atomicOr(flags, bad);
}

// dissolve.py:746-755: medium = [phi <= 0]; alpha = medium kf (1 - F / Fmax);
// f = medium kd F Cl^2
__global__ void k_zn_coefficients(int64_t n, const double* __restrict__ phi,
                                  const double* __restrict__ F, const double* __restrict__ Cl,
                                  double kf, double kd, double Fmax, double* __restrict__ alpha,
                                  double* __restrict__ src) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double med = (phi[i] <= 0.0) ? 1.0 : 0.0;
    if (alpha) alpha[i] = med * kf * (1.0 - F[i] / Fmax);
    if (src) src[i] = med * kd * F[i] * (Cl[i] * Cl[i]);
  }
}

// mesh_utils.py:478-484: s = phi0 / sqrt(phi0^2 + eps_sign^2), 0 inside the frozen band
// |phi0| < band (the update there is exactly zero in the reference too)
__global__ void k_redistance_init(int64_t n, const double* __restrict__ phi, double band,
                                  double eps_sign, double* __restrict__ s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double p = phi[i];
    s[i] = (fabs(p) < band) ? 0.0 : p / sqrt(p * p + eps_sign * eps_sign);
  }
}

// mesh_utils.py:515-519: gm = sqrt(|grad|^2 + 1e-12), dtau = h/2 / max(gm, 1/2),
// phi += dtau s (1 - gm)
__global__ void k_redistance_update(int64_t n, double* __restrict__ phi,
                                    const double* __restrict__ grad,
                                    const double* __restrict__ s, double h) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double gx = grad[3 * i], gy = grad[3 * i + 1], gz = grad[3 * i + 2];
    const double gm = sqrt(gx * gx + gy * gy + gz * gz + 1e-12);
    const double dtau = 0.5 * h / fmax(gm, 0.5);
    if (s[i] != 0.0) phi[i] += dtau * s[i] * (1.0 - gm);
  }
}

// longest edge of every cell (the cell diameter of a tetrahedron), summed per block
__global__ void k_cell_diameter(int64_t n, const int4* __restrict__ cells,
                                const double4* __restrict__ X, double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const double4 p[4] = {X[v.x], X[v.y], X[v.z], X[v.w]};
    double h2 = 0.0;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = a + 1; b < 4; b++) {
        const double dx = p[a].x - p[b].x, dy = p[a].y - p[b].y, dz = p[a].z - p[b].z;
        h2 = fmax(h2, dx * dx + dy * dy + dz * dz);
      }
    s += sqrt(h2);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b,
                        double* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// state advance after a solve: d = x - u, u_prev = u, u = x (one pass)
__global__ void k_advance(int64_t n, const double* __restrict__ x, double* __restrict__ u,
                          double* __restrict__ u_prev, double* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double xv = x[i], uv = u[i];
    d[i] = xv - uv;
    u_prev[i] = uv;
    u[i] = xv;
  }
}

// the same with a history of step increments in fixed buffers, shifted in place (newest
// first): hist[k] = hist[k - 1] for k = H - 1 .. 1, hist[0] = x - u (graph-replayable)
struct HistPtrs {
  double* h[8];
  double* g[8];  // optional second ring shifted alongside (slot 0 left as it is)
};
__global__ void k_advance_hist(int64_t n, int H, const double* __restrict__ x,
                               double* __restrict__ u, double* __restrict__ u_prev,
                               HistPtrs hp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double xv = x[i], uv = u[i];
    for (int k = H - 1; k >= 1; k--) hp.h[k][i] = hp.h[k - 1][i];
    if (hp.g[0])
      for (int k = H - 1; k >= 1; k--) hp.g[k][i] = hp.g[k - 1][i];
    hp.h[0][i] = xv - uv;
    u_prev[i] = uv;
    u[i] = xv;
  }
}

// (n, S) contiguous <-> (n, ld) interleaved with zero padding
__global__ void k_pack(int64_t n, int S, int ld, const double* __restrict__ src,
                       double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * ld;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / ld;
    const int s = (int)(i - r * ld);
    dst[i] = (s < S) ? src[r * S + s] : 0.0;
  }
}

__global__ void k_unpack(int64_t n, int S, int ld, const double* __restrict__ src,
                         double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * S;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / S;
    const int s = (int)(i - r * S);
    dst[i] = src[r * ld + s];
  }
}

}  // namespace tp

using namespace tp;

extern "C" int tp_pack_columns(int64_t n, int S, int ld, const double* src, double* dst,
                               void* stream) {
  TP_REQUIRE(src && dst && S >= 1 && ld >= S, "bad argument");
  if (n == 0) return TP_OK;
  k_pack<<<grid_for(n * ld, 256, 65535), 256, 0, as_stream(stream)>>>(n, S, ld, src, dst);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_unpack_columns(int64_t n, int S, int ld, const double* src, double* dst,
                                 void* stream) {
  TP_REQUIRE(src && dst && S >= 1 && ld >= S, "bad argument");
  if (n == 0) return TP_OK;
  k_unpack<<<grid_for(n * S, 256, 65535), 256, 0, as_stream(stream)>>>(n, S, ld, src, dst);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

// geo and coords4 rows are read with 32-byte loads
static bool mesh_ok(const tp_mesh* m) {
  return m && m->cells && m->geo && m->v2c_ptr && m->v2c && m->indptr &&
         (reinterpret_cast<uintptr_t>(m->geo) & 31) == 0 &&
         (reinterpret_cast<uintptr_t>(m->coords4) & 31) == 0;
}

extern "C" int tp_cell_average(int64_t n_cells, const int32_t* cells, const double* vert_vals,
                               double* cell_vals, void* stream) {
  TP_REQUIRE(cells && vert_vals && cell_vals, "null pointer");
  if (n_cells == 0) return TP_OK;
  k_cell_average<<<grid_for(n_cells, 256, 65535), 256, 0, as_stream(stream)>>>(
      n_cells, reinterpret_cast<const int4*>(cells), vert_vals, cell_vals);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_bc_mask(int64_t n_bc, const int32_t* bc_dofs, int64_t n_verts, uint8_t* mask,
                          int32_t* flags_dev, void* stream) {
  TP_REQUIRE(mask && flags_dev && (n_bc == 0 || bc_dofs), "null pointer");
  cudaStream_t st = as_stream(stream);
  TP_CUDA_TRY(cudaMemsetAsync(mask, 0, (size_t)n_verts, st));
  TP_CUDA_TRY(cudaMemsetAsync(flags_dev, 0, sizeof(int32_t), st));
  if (n_bc > 0) {
    k_bc_mask<<<grid_for(n_bc, 256), 256, 0, st>>>(n_bc, bc_dofs, n_verts, mask, flags_dev);
    TP_LAUNCH_CHECK();
  }
  int32_t f = 0;
  TP_CUDA_TRY(cudaMemcpyAsync(&f, flags_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  if (f) {
    set_error("a Dirichlet dof is outside [0, %lld)", (long long)n_verts);
    return TP_ERR_INDEX;
  }
  return TP_OK;
}

template <int MODE, bool DIAG>
static int launch_tiles(const tp_mesh* m, const double* De, const double* alpha, double inv_dt,
                        int lumped, const uint8_t* bc_mask, double* out64, float* out32,
                        const RowExtras& ex, cudaStream_t st, bool* used) {
  *used = false;
  if (!m->tiles) return TP_OK;
  const TileView& tv = m->tiles->v;
  // slot of 5 or 7 sixteen-byte units (tile_cell_entries), or 11 doubles for DIAG without
  // per-cell alpha (three CTAs of the largest tiles per SM instead of two)
  const bool cmp = DIAG && ex.alpha == nullptr;
  const int ew = DIAG ? (cmp ? 11 : 14) : 10;
  const size_t smem = sizeof(double) * (size_t)tv.max_cells * ew;
  int dev = 0, optin = 0;
  TP_CUDA_TRY(cudaGetDevice(&dev));
  TP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > (size_t)optin || tv.R > TILE_BLOCK || tv.n_tiles == 0) return TP_OK;
  auto fn = k_assemble_tiles<MODE, DIAG, false>;
  if constexpr (DIAG) {
    if (cmp) fn = k_assemble_tiles<MODE, DIAG, true>;
  }
  if (smem > 48 * 1024)
    TP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (cmp)
    TP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
  fn<<<tv.n_tiles, TILE_BLOCK, smem, st>>>(tv, m->geo, De, alpha, inv_dt, lumped, bc_mask,
                                           m->indptr, out64, out32, ex, ew, m->n_verts);
  TP_LAUNCH_CHECK();
  *used = true;
  return TP_OK;
}

extern "C" int tp_assemble_csr(const tp_mesh* m, const double* De_cell, const double* alpha_cell,
                               double inv_dt, int lumped, int mode, const uint8_t* bc_mask,
                               double* out64, float* out32, void* stream) {
  TP_REQUIRE(mesh_ok(m) && m->v2c_slots && m->indices, "incomplete mesh");
  TP_REQUIRE(mode == TP_ASM_MASS || De_cell, "De_cell is required");
  TP_REQUIRE(out64 || out32, "no output");
  TP_REQUIRE(m->max_row_len >= 1 && m->max_row_len <= 255, "bad max_row_len");
  if (m->n_verts == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  const size_t smem = sizeof(double) * 129 * (size_t)m->max_row_len;
  const int grid = grid_for(m->n_verts, 128);
  const RowExtras ex{};
  {
    bool used = false;
    int rc = TP_OK;
    if (mode == TP_ASM_FULL)
      rc = launch_tiles<TP_ASM_FULL, false>(m, De_cell, alpha_cell, inv_dt, lumped, bc_mask,
                                            out64, out32, ex, st, &used);
    else if (mode == TP_ASM_STIFF)
      rc = launch_tiles<TP_ASM_STIFF, false>(m, De_cell, alpha_cell, inv_dt, lumped, bc_mask,
                                             out64, out32, ex, st, &used);
    else if (mode == TP_ASM_MASS)
      rc = launch_tiles<TP_ASM_MASS, false>(m, De_cell, alpha_cell, inv_dt, lumped, bc_mask,
                                            out64, out32, ex, st, &used);
    if (rc != TP_OK || used) return rc;
  }
#define TP_ASM_LAUNCH(MD)                                                                 \
  do {                                                                                    \
    if (smem > 48 * 1024)                                                                 \
      TP_CUDA_TRY(cudaFuncSetAttribute(k_assemble_rows<MD, false>,                        \
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                       (int)smem));                                       \
    k_assemble_rows<MD, false><<<grid, 128, smem, st>>>(                                  \
        m->n_verts, m->v2c_ptr, m->v2c, m->v2c_slots, m->geo, De_cell, alpha_cell, inv_dt, \
        lumped, bc_mask, m->indptr, m->indices, out64, out32, ex);                        \
  } while (0)
  switch (mode) {
    case TP_ASM_FULL:
      TP_ASM_LAUNCH(TP_ASM_FULL);
      break;
    case TP_ASM_STIFF:
      TP_ASM_LAUNCH(TP_ASM_STIFF);
      break;
    case TP_ASM_MASS:
      TP_ASM_LAUNCH(TP_ASM_MASS);
      break;
    default:
      set_error("unknown assembly mode %d", mode);
      return TP_ERR_ARG;
  }
#undef TP_ASM_LAUNCH
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_dirichlet_rows(int64_t n_bc, const int32_t* bc_dofs, int64_t n_rows,
                                 const int32_t* indptr, const int32_t* indices, double* data,
                                 void* stream) {
  TP_REQUIRE(indptr && indices && data && (n_bc == 0 || bc_dofs), "null pointer");
  if (n_bc == 0) return TP_OK;
  k_dirichlet_rows<<<grid_for(n_bc, 128), 128, 0, as_stream(stream)>>>(n_bc, bc_dofs, n_rows,
                                                                        indptr, indices, data);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_lumped_diag(const tp_mesh* m, int S, int ld, const double* alpha,
                              const double* shift, const uint8_t* bc_mask, double* diag64,
                              float* diag32, void* stream) {
  TP_REQUIRE(mesh_ok(m), "incomplete mesh");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && ld >= S && ld <= TP_MAX_COLS, "bad S/ld");
  TP_REQUIRE(diag64 || diag32, "no output");
  double sh[4] = {0, 0, 0, 0};
  for (int s = 0; s < S; s++) sh[s] = shift ? shift[s] : 0.0;
  if (m->n_verts == 0) return TP_OK;
  k_lumped_diag<<<grid_for(m->n_verts, 128, 65535), 128, 0, as_stream(stream)>>>(
      m->n_verts, S, ld, m->v2c_ptr, m->v2c, m->geo, alpha, make_double4(sh[0], sh[1], sh[2], sh[3]),
      bc_mask, diag64, diag32);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_assemble_stiffness_diag(const tp_mesh* m, const double* De_cell, int S,
                                          int ld, const double* alpha, const double* shift,
                                          const uint8_t* bc_mask, double* out64, float* out32,
                                          const int32_t* slice_ptr, float* sell32,
                                          double* diag64, float* diag32, void* stream) {
  TP_REQUIRE(mesh_ok(m) && m->v2c_slots && m->indices && De_cell, "incomplete mesh or De");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && ld >= S && ld <= TP_MAX_COLS, "bad S/ld");
  TP_REQUIRE(out64 || out32 || sell32, "no operator output");
  TP_REQUIRE(diag64 || diag32, "no diagonal output");
  TP_REQUIRE(!sell32 || slice_ptr, "sell32 needs slice_ptr");
  TP_REQUIRE(m->max_row_len >= 1 && m->max_row_len <= 255, "bad max_row_len");
  if (m->n_verts == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  double sh[4] = {0, 0, 0, 0};
  for (int s = 0; s < S; s++) sh[s] = shift ? shift[s] : 0.0;
  RowExtras ex{S, ld, alpha, make_double4(sh[0], sh[1], sh[2], sh[3]), diag64, diag32,
               slice_ptr, sell32};
  {
    bool used = false;
    const int rc = launch_tiles<TP_ASM_STIFF, true>(m, De_cell, nullptr, 0.0, 1, bc_mask, out64,
                                                    out32, ex, st, &used);
    if (rc != TP_OK || used) return rc;
  }
  const size_t smem = sizeof(double) * 129 * (size_t)m->max_row_len;
  const int grid = grid_for(m->n_verts, 128);
  if (smem > 48 * 1024)
    TP_CUDA_TRY(cudaFuncSetAttribute(k_assemble_rows<TP_ASM_STIFF, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_assemble_rows<TP_ASM_STIFF, true><<<grid, 128, smem, st>>>(
      m->n_verts, m->v2c_ptr, m->v2c, m->v2c_slots, m->geo, De_cell, nullptr, 0.0, 1, bc_mask,
      m->indptr, m->indices, out64, out32, ex);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_assemble_rhs(const tp_mesh* m, int S, int ld, const double* u_old,
                               const double* f, double inv_dt, int lumped, int64_t n_bc,
                               const int32_t* bc_dofs, const double* bc_value, double* b,
                               void* stream) {
  TP_REQUIRE(mesh_ok(m) && u_old && b, "null pointer");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && ld >= S && ld <= TP_MAX_COLS, "bad S/ld");
  cudaStream_t st = as_stream(stream);
  int optin = 0;
  if (m->n_verts > 0 && m->tiles && m->tiles->v.n_tiles > 0 && m->tiles->v.R <= 256) {
    int dev = 0;
    TP_CUDA_TRY(cudaGetDevice(&dev));
    TP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  }
  const size_t cw = lumped ? 1 : (f ? 10 : 6);  // k_rhs_tiles' slot width
  const size_t smem_t = m->tiles ? sizeof(double) * cw * (size_t)std::max(m->tiles->v.max_cells, 1) : 0;
  if (m->n_verts > 0 && m->tiles && m->tiles->v.n_tiles > 0 && m->tiles->v.R <= 256 &&
      smem_t <= (size_t)optin) {
    const TileView& tv = m->tiles->v;
    auto fn = lumped ? k_rhs_tiles<true> : k_rhs_tiles<false>;
    if (smem_t > 48 * 1024)
      TP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t));
    fn<<<tv.n_tiles, 256, smem_t, st>>>(tv, S, ld, m->cells, m->geo, u_old, f, inv_dt, b);
    TP_LAUNCH_CHECK();
  } else if (m->n_verts > 0) {
    k_rhs_rows<<<grid_for(m->n_verts, 128, 65535), 128, 0, st>>>(
        m->n_verts, S, ld, m->cells, m->v2c_ptr, m->v2c, m->geo, u_old, f, inv_dt, lumped, b);
    TP_LAUNCH_CHECK();
  }
  if (n_bc > 0 && bc_dofs) {
    double v[4] = {0, 0, 0, 0};
    for (int s = 0; s < S; s++) v[s] = bc_value ? bc_value[s] : 0.0;
    k_rhs_bc<<<grid_for(n_bc, 128), 128, 0, st>>>(n_bc, bc_dofs, m->n_verts, S, ld,
                                                  make_double4(v[0], v[1], v[2], v[3]), b);
    TP_LAUNCH_CHECK();
  }
  return TP_OK;
}

extern "C" int tp_lumped_rhs(int64_t n_verts, int S, int ld, const double* mass,
                             const double* u_old, const double* f, double inv_dt, int64_t n_bc,
                             const int32_t* bc_dofs, const double* bc_value, double* b,
                             void* stream) {
  TP_REQUIRE(mass && u_old && b, "null pointer");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && ld >= S && ld <= TP_MAX_COLS, "bad S/ld");
  cudaStream_t st = as_stream(stream);
  if (n_verts > 0) {
    k_lumped_rhs<<<grid_for(n_verts * ld, 256, sm_count() * 8), 256, 0, st>>>(
        n_verts, S, ld, mass, u_old, f, inv_dt, b);
    TP_LAUNCH_CHECK();
  }
  if (n_bc > 0 && bc_dofs) {
    double v[4] = {0, 0, 0, 0};
    for (int s = 0; s < S; s++) v[s] = bc_value ? bc_value[s] : 0.0;
    k_rhs_bc<<<grid_for(n_bc, 128), 128, 0, st>>>(n_bc, bc_dofs, n_verts, S, ld,
                                                  make_double4(v[0], v[1], v[2], v[3]), b);
    TP_LAUNCH_CHECK();
  }
  return TP_OK;
}

extern "C" int tp_nodal_gradient(const tp_mesh* m, const double* JinvT, const double* u,
                                 double* grad, void* stream) {
  TP_REQUIRE(mesh_ok(m) && u && grad, "null pointer");
  TP_REQUIRE(JinvT || m->coords4, "need JinvT or coords4");
  if (m->n_verts == 0) return TP_OK;
  k_nodal_gradient<<<grid_for(m->n_verts, 128, 65535), 128, 0, as_stream(stream)>>>(
      m->n_verts, m->cells, m->v2c_ptr, m->v2c, m->geo, JinvT, m->coords4, u, grad);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_scaffold_volume(const tp_mesh* m, const double* phi, double eps,
                                  double* out_dev, void* scratch, void* stream) {
  TP_REQUIRE(mesh_ok(m) && phi && out_dev && scratch, "null pointer");
  TP_REQUIRE(eps > 0.0, "epsilon must be positive");
  cudaStream_t st = as_stream(stream);
  const int grid = grid_for(m->n_cells, 256, 1024);
  double* part = static_cast<double*>(scratch);
  const double qa = (5.0 + 3.0 * sqrt(5.0)) / 20.0, qb = (5.0 - sqrt(5.0)) / 20.0;
  k_scaffold_volume<<<grid, 256, 0, st>>>(m->n_cells, reinterpret_cast<const int4*>(m->cells),
                                          m->geo, phi, eps, qa, qb, part);
  TP_LAUNCH_CHECK();
  k_sum_parts<<<1, 256, 0, st>>>(grid, part, out_dev);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

// ----------------------------------------------------------------- scaffold volume, fixed scratch
// tp_scaffold_volume_static keeps its block partials in this module-resident array instead
// of a caller buffer.  The launch uses at most kSvMaxParts blocks (grid_for caps the grid;
// the kernel strides over the cells), so every mesh size fits; nothing in the array has to
// start at zero because every partial is written before the second kernel reads it.  One
// array per device, shared by all callers: calls that overlap on one device (two streams,
// two host threads) race on it.
static constexpr int kSvMaxParts = 1024;  // 8 KiB of doubles
static constexpr int kSvMaxDevices = 64;
static __device__ __align__(256) double g_sv_parts[kSvMaxParts];
static std::mutex g_sv_mu;
static double* g_sv_ptr[kSvMaxDevices] = {};

// Device address of g_sv_parts on the current device.  Outside a stream capture it is
// looked up on every call (cheap after the first), so a device reset or another context
// never leaves a stale address behind; inside a capture the address kept by an earlier
// call on this device is used (no lookup while a graph is being recorded).
static int sv_parts_on_current_device(cudaStream_t st, double** out) {
  int dev = -1;
  TP_CUDA_TRY(cudaGetDevice(&dev));
  TP_REQUIRE(dev >= 0 && dev < kSvMaxDevices,
             "tp_scaffold_volume_static: device ordinal %d beyond the %d supported", dev,
             kSvMaxDevices);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TP_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  std::lock_guard<std::mutex> lock(g_sv_mu);
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    TP_CUDA_TRY(cudaGetSymbolAddress(&p, g_sv_parts));
    g_sv_ptr[dev] = static_cast<double*>(p);
  }
  TP_REQUIRE(g_sv_ptr[dev] != nullptr,
             "tp_scaffold_volume_static: the first call on device %d was inside a stream "
             "capture; call it once on that device before capturing", dev);
  *out = g_sv_ptr[dev];
  return TP_OK;
}

extern "C" int tp_scaffold_volume_static(const tp_mesh* m, const double* phi, double eps,
                                         double* out_dev, void* stream) {
  TP_REQUIRE(mesh_ok(m) && phi && out_dev, "null pointer");
  TP_REQUIRE(eps > 0.0, "epsilon must be positive");
  cudaStream_t st = as_stream(stream);
  const int grid = grid_for(m->n_cells, 256, kSvMaxParts);  // at most kSvMaxParts partials
  double* part = nullptr;
  const int rc = sv_parts_on_current_device(st, &part);
  if (rc != TP_OK) return rc;
  const double qa = (5.0 + 3.0 * sqrt(5.0)) / 20.0, qb = (5.0 - sqrt(5.0)) / 20.0;
  k_scaffold_volume<<<grid, 256, 0, st>>>(m->n_cells, reinterpret_cast<const int4*>(m->cells),
                                          m->geo, phi, eps, qa, qb, part);
  TP_LAUNCH_CHECK();
  k_sum_parts<<<1, 256, 0, st>>>(grid, part, out_dev);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_o2_alpha(int64_t n, const double* phi, const double* normgradphi, double eps,
                           double k_orr, double* alpha, void* stream) {
  TP_REQUIRE(phi && normgradphi && alpha, "null pointer");
  if (n == 0) return TP_OK;
  k_o2_alpha<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(n, phi, normgradphi, eps,
                                                                      k_orr, alpha);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_oh_source(int64_t n, const double* phi, const double* normgradphi,
                            const double* F, const double* Cl, const double* O2, double eps,
                            double kd, double k_orr, double orr_factor, double* f, void* stream) {
  TP_REQUIRE(phi && normgradphi && F && Cl && O2 && f, "null pointer");
  if (n == 0) return TP_OK;
  k_oh_source<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(
      n, phi, normgradphi, F, Cl, O2, eps, kd, k_orr, orr_factor, f);
  TP_LAUNCH_CHECK();
  return TP_OK;
}


extern "C" int tp_interface_terms(int64_t n, const double* phi, const double* grad, double eps,
                                  double k_orr, double orr_factor, int ld, const double* U,
                                  int col_o2, int col_oh, double* f, double* hv, double* ngphi,
                                  void* stream) {
  TP_REQUIRE(phi, "null pointer");
  TP_REQUIRE(eps > 0.0, "epsilon must be positive");
  TP_REQUIRE(!f || (U && ld >= 1 && ld <= TP_MAX_COLS && col_o2 >= 0 && col_o2 < ld &&
                    col_oh >= 0 && col_oh < ld),
             "bad column layout");
  if (n == 0) return TP_OK;
  k_interface_terms<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(
      n, phi, grad, eps, k_orr, orr_factor, ld, U, col_o2, col_oh, f, hv, ngphi);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_cell_average_col(int64_t n_cells, const int32_t* cells, const double* vert_vals,
                                   int ld, int col, double* out, void* stream) {
  TP_REQUIRE(cells && vert_vals && out, "null pointer");
  TP_REQUIRE(ld >= 1 && col >= 0 && col < ld, "bad column");
  if (n_cells == 0) return TP_OK;
  k_cell_average_col<<<grid_for(n_cells, 256, 65535), 256, 0, as_stream(stream)>>>(
      n_cells, reinterpret_cast<const int4*>(cells), vert_vals, ld, col, out);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_levelset_advance(int64_t n, double* phi, int ld, const double* U, int col,
                                   double dt, double rate, double gain, void* stream) {
  TP_REQUIRE(phi && U, "null pointer");
  TP_REQUIRE(ld >= 1 && col >= 0 && col < ld, "bad column");
  if (n == 0) return TP_OK;
  k_levelset_advance<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(n, phi, ld, U, col,
                                                                          dt, rate, gain);
  TP_LAUNCH_CHECK();
  return TP_OK;
}


extern "C" int tp_effective_diffusion(int64_t n, const double* phi, const double* F, double Fmax,
                                      double film_floor, const double* D0, double* De_zn,
                                      double* De_cl, double* De_oh, double* De_o2,
                                      int32_t* flags_dev, void* stream) {
  TP_REQUIRE(phi && F && D0 && flags_dev, "null pointer");
  if (n == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  TP_CUDA_TRY(cudaMemsetAsync(flags_dev, 0, sizeof(int32_t), st));
  k_effective_diffusion<<<grid_for(n, 256, 65535), 256, 0, st>>>(
      n, phi, F, Fmax, film_floor, make_double4(D0[0], D0[1], D0[2], D0[3]), De_zn, De_cl, De_oh,
      De_o2, flags_dev);
  TP_LAUNCH_CHECK();
  int32_t fl = 0;
  TP_CUDA_TRY(cudaMemcpyAsync(&fl, flags_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  if (fl & 1) {
    set_error("effective diffusion contains NaN/Inf (check F against Fmax)");
    return TP_ERR_NONFINITE;
  }
  if (fl & 2) {
    set_error("effective diffusion has negative values (unphysical film saturation)");
    return TP_ERR_ARG;
  }
  return TP_OK;
}

extern "C" int tp_zn_coefficients(int64_t n, const double* phi, const double* F, const double* Cl,
                                  double kf, double kd, double Fmax, double* alpha, double* src,
                                  void* stream) {
  TP_REQUIRE(phi && F && (Cl || !src), "null pointer");
  if (n == 0) return TP_OK;
  k_zn_coefficients<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(n, phi, F, Cl, kf, kd,
                                                                         Fmax, alpha, src);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" size_t tp_redistance_scratch_bytes(int64_t n_verts) {
  return sizeof(double) * 4 * (size_t)n_verts;
}

extern "C" int tp_redistance(const tp_mesh* m, double* phi, int iters, double h_avg,
                             double band_factor, double eps_factor, void* scratch,
                             void* stream) {
  TP_REQUIRE(mesh_ok(m) && m->coords4 && phi && scratch, "null pointer");
  TP_REQUIRE(iters >= 0 && h_avg > 0.0, "bad redistancing parameters");
  if (m->n_verts == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  double* grad = static_cast<double*>(scratch);
  double* s = grad + 3 * m->n_verts;
  const int g = grid_for(m->n_verts, 256, 65535);
  k_redistance_init<<<g, 256, 0, st>>>(m->n_verts, phi, band_factor * h_avg, eps_factor * h_avg, s);
  TP_LAUNCH_CHECK();
  for (int k = 0; k < iters; k++) {
    const int rc = tp_nodal_gradient(m, nullptr, phi, grad, stream);
    if (rc != TP_OK) return rc;
    k_redistance_update<<<g, 256, 0, st>>>(m->n_verts, phi, grad, s, h_avg);
    TP_LAUNCH_CHECK();
  }
  return TP_OK;
}

// ----------------------------------------------------------------- level set from regions
// domain/mesh_utils.py:367-449 (_init_phi_from_regions): a vertex of any cell with the
// scaffold label is inside (+1), every other vertex outside (-1); the interface vertices
// are those of at least one scaffold cell and one other cell; phi = sign * the distance to
// the nearest interface vertex, or sign * 0.5 when there is none.  Distances are
// sqrt((dx dx + dy dy) + dz dz) in FP64 with every operation rounded once, and the minimum
// over all interface vertices is exact and order-free, as the reference's KD-tree query.
__global__ void k_region_marks(int64_t n, const int4* __restrict__ cells,
                               const int32_t* __restrict__ regions, int label,
                               int32_t* __restrict__ marks) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const int mk = (regions[c] == label) ? 1 : 2;
    atomicOr(marks + v.x, mk);
    atomicOr(marks + v.y, mk);
    atomicOr(marks + v.z, mk);
    atomicOr(marks + v.w, mk);
  }
}

// coordinates of the interface vertices (marks 3) appended to list; count in *count
__global__ void k_interface_list(int64_t nv, const int32_t* __restrict__ marks,
                                 const double4* __restrict__ X, double4* __restrict__ list,
                                 int32_t* __restrict__ count) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    if (marks[v] == 3) list[atomicAdd(count, 1)] = X[v];
  }
}

constexpr int PHI_CHUNK = 1024;  // interface points staged per round (32 KB)

__global__ void __launch_bounds__(256) k_phi_nearest(int64_t nv, const int32_t* __restrict__ marks,
                                                     const double4* __restrict__ X,
                                                     const double4* __restrict__ list,
                                                     const int32_t* __restrict__ count,
                                                     double* __restrict__ phi) {
  __shared__ double4 s_pts[PHI_CHUNK];
  const int ni = *count;
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool in = v < nv;
  const double sign = (in && (marks[v] & 1)) ? 1.0 : -1.0;
  const double4 x = in ? X[v] : make_double4(0.0, 0.0, 0.0, 0.0);
  double best = INFINITY;
  for (int b = 0; b < ni; b += PHI_CHUNK) {
    const int m = min(PHI_CHUNK, ni - b);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) s_pts[i] = list[b + i];
    __syncthreads();
    for (int i = 0; i < m; i++) {
      const double4 p = s_pts[i];
      const double dx = __dsub_rn(x.x, p.x), dy = __dsub_rn(x.y, p.y), dz = __dsub_rn(x.z, p.z);
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      best = fmin(best, d2);
    }
  }
  if (in) phi[v] = (ni == 0) ? sign * 0.5 : sign * __dsqrt_rn(best);
}

extern "C" size_t tp_phi_from_regions_scratch_bytes(int64_t n_verts) {
  const auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return a256(sizeof(int32_t) * (size_t)n_verts) + 256 + sizeof(double4) * (size_t)n_verts;
}

extern "C" int tp_phi_from_regions(const tp_mesh* m, const int32_t* regions, int scaffold_label,
                                   double* phi, void* scratch, void* stream) {
  TP_REQUIRE(mesh_ok(m) && m->coords4 && regions && phi && scratch, "null pointer");
  if (m->n_verts == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  const size_t mb = (sizeof(int32_t) * (size_t)m->n_verts + 255) & ~(size_t)255;
  int32_t* marks = static_cast<int32_t*>(scratch);
  int32_t* count = reinterpret_cast<int32_t*>(static_cast<char*>(scratch) + mb);
  double4* list = reinterpret_cast<double4*>(static_cast<char*>(scratch) + mb + 256);
  TP_CUDA_TRY(cudaMemsetAsync(scratch, 0, mb + 256, st));
  if (m->n_cells > 0)
    k_region_marks<<<grid_for(m->n_cells, 256, 65535), 256, 0, st>>>(
        m->n_cells, reinterpret_cast<const int4*>(m->cells), regions, scaffold_label, marks);
  const double4* X = reinterpret_cast<const double4*>(m->coords4);
  k_interface_list<<<grid_for(m->n_verts, 256, 65535), 256, 0, st>>>(m->n_verts, marks, X, list,
                                                                     count);
  k_phi_nearest<<<grid_for(m->n_verts, 256), 256, 0, st>>>(m->n_verts, marks, X, list, count,
                                                          phi);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_mean_cell_diameter(const tp_mesh* m, double* out_dev, void* scratch,
                                     void* stream) {
  TP_REQUIRE(mesh_ok(m) && m->coords4 && out_dev && scratch, "null pointer");
  if (m->n_cells == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  const int grid = grid_for(m->n_cells, 256, 1024);
  double* part = static_cast<double*>(scratch);
  k_cell_diameter<<<grid, 256, 0, st>>>(m->n_cells, reinterpret_cast<const int4*>(m->cells),
                                        reinterpret_cast<const double4*>(m->coords4), part);
  TP_LAUNCH_CHECK();
  k_sum_parts<<<1, 256, 0, st>>>(grid, part, out_dev);  // the sum; the caller divides by n
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_advance_state(int64_t n, const double* x, double* u, double* u_prev,
                                double* d, void* stream) {
  TP_REQUIRE(x && u && u_prev && d, "null pointer");
  if (n == 0) return TP_OK;
  k_advance<<<grid_for(n, 256, sm_count() * 8), 256, 0, as_stream(stream)>>>(n, x, u, u_prev, d);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_advance_history(int64_t n, const double* x, double* u, double* u_prev,
                                  int n_hist, double* const* hist, double* const* ring2,
                                  void* stream) {
  TP_REQUIRE(x && u && u_prev && hist && n_hist >= 1 && n_hist <= 8, "bad arguments");
  HistPtrs hp{};
  for (int k = 0; k < n_hist; k++) {
    TP_REQUIRE(hist[k] && (!ring2 || ring2[k]), "null history buffer");
    hp.h[k] = hist[k];
    hp.g[k] = ring2 ? ring2[k] : nullptr;
  }
  if (n == 0) return TP_OK;
  k_advance_hist<<<grid_for(n, 256, sm_count() * 8), 256, 0, as_stream(stream)>>>(
      n, n_hist, x, u, u_prev, hp);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream) {
  TP_REQUIRE(x && y, "null pointer");
  if (n == 0) return TP_OK;
  k_axpby<<<grid_for(n, 256, 65535), 256, 0, as_stream(stream)>>>(n, a, x, b, y);
  TP_LAUNCH_CHECK();
  return TP_OK;
}
