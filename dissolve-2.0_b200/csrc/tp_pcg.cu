// tp_pcg.cu -- persistent Jacobi-PCG: one cooperative launch per solve.
//
// The problem sizes of the transport step (a few 100k rows, operator and vectors
// resident in the 126 MB L2) make a Krylov iteration latency-bound: what costs is the
// number of dependent launches, dependent memory round trips and reduction tails, not
// bytes.  This engine runs the whole solve in ONE cooperative kernel with one CTA group
// per SM:
//
//   init  I1 Jacobi diagonal, Dirichlet values into x      | barrier
//         I2 r = b - A64 x, z = D^-1 r, p = z, norms        | barrier -> lane state
//   loop  A  p = z + beta p (recomputed at every gathered neighbour), q = A p, p.q
//                                                            | barrier -> alpha
//         B  xi += alpha p, r -= alpha q, z = D^-1 r, r.z, r.r | barrier -> beta, trigger
//         RU (FP32 inner only, when triggered) x += xi        | barrier
//            r = b - A64 x in FP64, replace r, z             | barrier -> converge / keep
//   final x += xi | barrier | r = b - A64 x -> true residual norms
//
// Layout.  z and p of a row sit side by side in one record [z_0..z_{LD-1} | p_0..p_{LD-1}]
// (32 bytes for 4 FP32 columns: one sector per gathered neighbour), double-buffered: phase
// A of iteration k reads record k and writes p into record k+1, phase B writes z into
// record k+1.  Every CTA owns a contiguous range of 32-row slices (its slice offsets are
// staged in shared memory at launch).
//
// Phase A walks a warp's (slice, group-of-U-entries) sequence as one flat loop and loads
// the SELL stream (column, value) of the NEXT group before gathering the records of the
// current one, so the dependent chain per group is one gather, not a stream load followed
// by a gather.  Phase B handles two rows per thread per step so their loads overlap.
//
// Reductions.  Each dot product is one FP64 partial per CTA; after the barrier every CTA
// sums all partials in the same fixed order, so all CTAs hold bit-identical scalars and
// take the same branches (deterministic for a given grid).
//
// Barrier.  A monotonic arrival counter: each CTA adds 1 (release) and waits until the
// counter reaches (barriers so far) x gridDim.  The wait is bounded in time (2 s of
// %globaltimer by default, tp_pcg_set_wait_limit); a CTA that gives up raises an abort
// flag that every other wait also watches, so a lost CTA ends the kernel with
// TP_ERR_TIMEOUT instead of a hang.
//
// Reliable updates (FP32 inner solve).  When any lane's recurrence residual has dropped
// by delta since its last refresh (or reached the tolerance), every active lane is
// refreshed in the same pass: the FP64 residual costs one operator sweep whatever the
// number of lanes, and refreshing together keeps the number of sweeps at that of the
// fastest-converging lane.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tp_ops.cuh"

namespace tp {

struct PBar {
  unsigned int count;  // arrivals since the launch (reset by tp_pcg_run)
  unsigned int abort;
  unsigned int pad[2];
};

struct POut {
  int32_t iterations, n_reliable, status, timeouts;
  int32_t lane_iters[4], lane_status[4];
  double lane_rtrue[4], lane_bb[4];
};

template <typename VT>
struct PArgs {
  int64_t n;
  int S, ns, max_it;
  double delta2;
  // inner operator, SELL-32
  const int32_t* slice_ptr;
  const int32_t* sell_col;
  const VT* sK;
  const VT* sM;
  const VT* diag;
  // outer operator, FP64 CSR
  CsrView<double> A64;
  double dscale[4], cscale[4];
  const uint8_t* bc;
  const double* b;
  double* x;
  const double* rtol;
  VT *rec0, *rec1;  // [z | p] records, double-buffered
  VT *q, *r, *xi, *dinv;
  VT *u, *w, *p, *s;  // window engine (Chronopoulos-Gear CG): u = D^-1 r, w = A u
  // window engine: per-CTA halo lists and window-local SELL columns
  const int32_t* halo_ptr;  // gridDim.x + 1
  const int32_t* halo;      // sorted columns outside each CTA's row range
  const uint16_t* loc_col;  // (n_entries) window-local column of every SELL entry
  int sp_cap, halo_cap, col_cap;  // shared-memory capacities (entries)
  int win_cap;                    // window entries (own rows + halo) of the largest CTA
  int reg_values;                 // every slice at most 16 wide: values via registers
  int tmem_values;                // FP32 values resident in tensor memory for the solve
  // pipelined engine: the halo of each CTA as bulk-copy runs (int4 {global row, window
  // slot past the own rows, entries, 0}) and the entries left to single copies (halo
  // positions), per CTA ranges in run_ptr / single_ptr
  const int4* runs;
  const int32_t* run_ptr;
  const uint16_t* single;
  const int32_t* single_ptr;
  int single_cap;                 // shared-memory capacity of the single list (entries)
  double* part;  // gridDim.x * 32: two rows of 16 partial sums per CTA
  PBar* bar;
  POut* out;
  unsigned long long* prof;  // optional: gridDim.x * 8 phase times (ns)
  // barrier wait bound, and arrivals every barrier waits for beyond the grid's own (0 in
  // production; > 0 only to make the waits run out on purpose, which exercises the
  // timeout path).  Kernel arguments: reading them costs no memory access per barrier.
  unsigned long long wait_limit_ns;
  unsigned int wait_missing;
};

constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // default barrier bound: 2 s

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Read-only matrix stream: no L1 allocation, so the L1 keeps the gathered records.
__device__ __forceinline__ int ld_na(const int32_t* p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_na(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_na(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Phase clock of thread 0 (profiled runs only): adds now - last to slot k of a shared
// array (kept out of registers: the solve loop needs them).
struct PhaseClock {
  unsigned long long last = 0;
  unsigned long long* acc = nullptr;
  bool on = false;
  __device__ __forceinline__ void start(bool enable, unsigned long long* sacc) {
    on = enable && threadIdx.x == 0;
    acc = sacc;
    if (on) {
      for (int k = 0; k < 8; k++) acc[k] = 0;
      last = gtime();
    }
  }
  __device__ __forceinline__ void lap(int k) {
    if (on) {
      const unsigned long long t = gtime();
      acc[k] += t - last;
      last = t;
    }
  }
};

// Grid barrier; returns false in every thread of the CTA when the grid has aborted.
// `target` (thread 0 only) counts the arrivals this CTA has waited for so far.  The CTA's
// writes are ordered by __syncthreads and published by thread 0's gpu-scope release add;
// the acquire poll and the closing __syncthreads make the other CTAs' writes visible.
__device__ __forceinline__ bool grid_sync(PBar* bar, unsigned int& target,
                                          unsigned long long limit_ns, unsigned int missing) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    target += gridDim.x + missing;
    red_release_add(&bar->count, 1u);
    unsigned int spins = 0;
    unsigned long long t0 = 0;
    while ((int)(ld_acquire(&bar->count) - target) < 0) {
      if ((++spins & 31u) == 0u) {
        if (ld_acquire(&bar->abort)) {
          ok = 0;
          break;
        }
        const unsigned long long t = gtime();
        if (t0 == 0) {
          t0 = t;
        } else if (t - t0 > limit_ns) {
          atomicExch(&bar->abort, 1u);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum slots K0 .. K0+NV-1 of every CTA's partial row (fixed order) into s_tot[K0 ..] for
// all threads.  Thread (group g, slot k) adds the partials of CTAs g, g + groups, ... (a
// half-warp reads one CTA's 16 slots: one 128-byte line; the first 8 loads are issued
// together), then warp k sums slot k over the groups with a fixed shuffle tree; every
// CTA computes the same bits.
template <int NV, int K0 = 0>
__device__ __forceinline__ void grid_totals(const double* part, double* s_tot, double* s_buf) {
  const int T = blockDim.x;
  const int groups = T / 16;  // blockDim multiple of 16
  const int k = threadIdx.x % 16, g = threadIdx.x / 16;
  const int nb = (int)gridDim.x;
  double v = 0.0;
  if (k >= K0 && k < K0 + NV) {
    constexpr int Q = 8;
    double x[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const int b = g + q * groups;
      x[q] = (b < nb) ? __ldcg(part + (int64_t)b * 16 + k) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < Q; q++)
      if (g + q * groups < nb) v += x[q];
    for (int b = g + Q * groups; b < nb; b += groups) v += __ldcg(part + (int64_t)b * 16 + k);
  }
  s_buf[threadIdx.x] = v;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= K0 && w < K0 + NV) {
    double t = 0.0;
    for (int gg = lane; gg < groups; gg += 32) t += s_buf[gg * 16 + w];
    t = warp_sum(t);
    if (lane == 0) s_tot[w] = t;
  }
  __syncthreads();
}

template <int NV>
__device__ __forceinline__ void block_partial(double v[NV], double* part, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) sh[k * 32 + w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int ww = 0; ww < nw; ww++) t += sh[threadIdx.x * 32 + ww];
    part[(int64_t)blockIdx.x * 16 + threadIdx.x] = t;
  }
}

struct LaneState {
  double rz[4], alpha[4], beta[4], rr[4], rmax2[4], tol2[4], bb[4], rtrue[4];
  // frozen (window engine): the lane's recurrence residual reached the tolerance; it takes
  // no further steps and is confirmed by the next FP64 sweep
  int active[4], trigger[4], status[4], iters[4], frozen[4];
};

// z and p of row j from a [z | p] record buffer (plain loads: written by this kernel)
template <typename VT, int LD>
__device__ __forceinline__ void ld_rec(const VT* rec, int64_t j, VT z[LD], VT p[LD]) {
  constexpr int NB = 2 * LD * (int)sizeof(VT);
  VT t[2 * LD];
  const VT* src = rec + j * 2 * LD;
  if constexpr (NB == 8) {
    const uint2 u = *reinterpret_cast<const uint2*>(src);
    memcpy(t, &u, 8);
  } else {
    uint4 u[NB / 16];
#pragma unroll
    for (int i = 0; i < NB / 16; i++) u[i] = reinterpret_cast<const uint4*>(src)[i];
    memcpy(t, u, NB);
  }
#pragma unroll
  for (int s = 0; s < LD; s++) {
    z[s] = t[s];
    p[s] = t[LD + s];
  }
}

// SELL stream of entries k .. k+U-1 of a slice (base, width w) for this lane; entries past
// the width read the slice's last column with value 0.
template <typename VT, int U, bool HASM>
__device__ __forceinline__ void stage_group(const PArgs<VT>& a, int base, int w, int k, int lane,
                                            int cc[U], VT vv[U], VT mm[]) {
#pragma unroll
  for (int u = 0; u < U; u++) {
    const bool in = k + u < w;
    const int pos = base + (in ? k + u : w - 1) * 32 + lane;
    cc[u] = (w > 0) ? ld_na(a.sell_col + pos) : 0;
    vv[u] = in ? ld_na(a.sK + pos) : VT(0);
    if constexpr (HASM) mm[u] = in ? ld_na(a.sM + pos) : VT(0);
  }
}

// LD values of entry i of a shared-memory window
template <typename VT, int LD>
__device__ __forceinline__ void ld_win(const VT* w, int i, VT v[LD]) {
  constexpr int NB = LD * (int)sizeof(VT);
  const VT* src = w + i * LD;
  if constexpr (NB == 4 || NB == 8) {
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = src[s];
  } else {
    VT t[LD];
    uint4 u[NB / 16];
#pragma unroll
    for (int k = 0; k < NB / 16; k++) u[k] = reinterpret_cast<const uint4*>(src)[k];
    memcpy(t, u, NB);
#pragma unroll
    for (int s = 0; s < LD; s++) v[s] = t[s];
  }
}

// store LD values into entry i of a shared-memory window
template <typename VT, int LD>
__device__ __forceinline__ void st_win(VT* w, int i, const VT v[LD]) {
  constexpr int NB = LD * (int)sizeof(VT);
  VT* dst = w + i * LD;
  if constexpr (NB == 4 || NB == 8) {
#pragma unroll
    for (int s = 0; s < LD; s++) dst[s] = v[s];
  } else {
    uint4 u[NB / 16];
    memcpy(u, v, NB);
#pragma unroll
    for (int k = 0; k < NB / 16; k++) reinterpret_cast<uint4*>(dst)[k] = u[k];
  }
}

// values only of entries k .. k+U-1 of a slice (the window engine reads its columns from
// shared memory); entries past the width are 0 and not loaded
template <typename VT, int U, bool HASM>
__device__ __forceinline__ void stage_values(const PArgs<VT>& a, int base, int w, int k, int lane,
                                             VT vv[U], VT mm[]) {
#pragma unroll
  for (int u = 0; u < U; u++) {
    const bool in = k + u < w;
    const int pos = base + (k + u) * 32 + lane;
    vv[u] = in ? ld_na(a.sK + pos) : VT(0);
    if constexpr (HASM) mm[u] = in ? ld_na(a.sM + pos) : VT(0);
  }
}

template <typename VT, int LD>
__device__ __forceinline__ void csr64_residual(const PArgs<VT>& a, int64_t row, double r64[LD]) {
  double ax[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) ax[s] = 0.0;
  const bool bcr = a.bc && a.bc[row];
  double xr[LD];
  ldv_cg<double, LD>(a.x, row, xr);
  if (bcr) {
#pragma unroll
    for (int s = 0; s < LD; s++) ax[s] = xr[s];
  } else {
    double ak[LD], am[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) ak[s] = am[s] = 0.0;
    const int beg = a.A64.indptr[row], end = a.A64.indptr[row + 1];
    // RP entries at a time: their index, value and x loads are in flight together; the
    // sums still run entry by entry in CSR order
    constexpr int RP = (LD == 4) ? 2 : 4;
    for (int p0 = beg; p0 < end; p0 += RP) {
      int jj[RP];
      double kv[RP], mv[RP], xv[RP][LD];
#pragma unroll
      for (int u = 0; u < RP; u++) {
        const bool in = p0 + u < end;
        jj[u] = in ? __ldg(a.A64.indices + p0 + u) : (int)row;
        kv[u] = in ? __ldg(a.A64.K + p0 + u) : 0.0;
        mv[u] = (in && a.A64.M) ? __ldg(a.A64.M + p0 + u) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < RP; u++) ldv_cg<double, LD>(a.x, jj[u], xv[u]);
#pragma unroll
      for (int u = 0; u < RP; u++) {
        if (p0 + u >= end) break;
#pragma unroll
        for (int s = 0; s < LD; s++) ak[s] += kv[u] * xv[u][s];
        if (a.A64.M) {
#pragma unroll
          for (int s = 0; s < LD; s++) am[s] += mv[u] * xv[u][s];
        }
      }
    }
    double dr[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) dr[s] = 0.0;
    if (a.A64.diag) ldv<double, LD>(a.A64.diag, row, dr);
#pragma unroll
    for (int s = 0; s < LD; s++) ax[s] = a.dscale[s] * ak[s] + a.cscale[s] * am[s] + dr[s] * xr[s];
  }
  double bv[LD];
  ldv_cg<double, LD>(a.b, row, bv);
#pragma unroll
  for (int s = 0; s < LD; s++) r64[s] = (s < a.S) ? bv[s] - ax[s] : 0.0;
}

template <typename VT, int LD, int U, int MINB, bool HASM>
__global__ void __launch_bounds__(512, MINB) k_pcg(PArgs<VT> a) {
  extern __shared__ int32_t s_sp[];  // slice offsets of this CTA's range, se - sb + 1
  __shared__ double sh[32 * 12];
  __shared__ double s_buf[512];
  __shared__ double s_tot[16];
  __shared__ LaneState L;
  __shared__ int s_anytrig;
  __shared__ unsigned long long s_clk[8];
  unsigned int target = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int sb = (int)((int64_t)blockIdx.x * a.ns / gridDim.x);
  const int se = (int)((int64_t)(blockIdx.x + 1) * a.ns / gridDim.x);
  const int S = a.S;
  PhaseClock clk;
  clk.start(a.prof != nullptr, s_clk);
  // read only after the first barrier (whose __syncthreads orders these stores)
  for (int i = threadIdx.x; i <= se - sb; i += blockDim.x) s_sp[i] = a.slice_ptr[sb + i];

#define FOR_OWN_ROWS                                              \
  for (int sl = sb + warp; sl < se; sl += nwarps)                 \
    for (int64_t row = (int64_t)sl * 32 + lane; row < a.n; row = a.n)

  // ---- I1: Jacobi diagonal (FP64 values), Dirichlet values into x
  FOR_OWN_ROWS {
    VT dv[LD];
    const bool bcr = a.bc && a.bc[row];
    if (bcr) {
#pragma unroll
      for (int s = 0; s < LD; s++) {
        dv[s] = VT(0);
        a.x[row * LD + s] = a.b[row * LD + s];
      }
    } else {
      const int lo = a.A64.indptr[row], hi = a.A64.indptr[row + 1];
      int l = lo, h = hi;
      while (l < h) {
        const int mid = (l + h) >> 1;
        if (a.A64.indices[mid] < row)
          l = mid + 1;
        else
          h = mid;
      }
      const bool found = l < hi && a.A64.indices[l] == row;
      const double kd = found ? a.A64.K[l] : 0.0;
      const double md = (a.A64.M && found) ? a.A64.M[l] : 0.0;
#pragma unroll
      for (int s = 0; s < LD; s++) {
        double d = a.dscale[s] * kd + a.cscale[s] * md;
        if (a.A64.diag) d += a.A64.diag[row * LD + s];
        dv[s] = (s < S && d != 0.0) ? VT(1.0 / d) : VT(0);
      }
    }
    stv<VT, LD>(a.dinv, row, dv);
  }
  bool ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);

  // ---- I2: r = b - A x, z = D^-1 r, record 0 = [z | z], xi = 0; rr, rz, bb
  {
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = 0.0;
    if (ok) {
      FOR_OWN_ROWS {
        double r64[LD];
        csr64_residual<VT, LD>(a, row, r64);
        VT rv[LD], dv[LD], zv[LD], zero[LD];
        ldv_cg<VT, LD>(a.dinv, row, dv);
        double bv[LD];
        ldv_cg<double, LD>(a.b, row, bv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          rv[s] = (VT)r64[s];
          zv[s] = dv[s] * rv[s];
          zero[s] = VT(0);
          acc[s] += r64[s] * r64[s];
          acc[4 + s] += (double)rv[s] * (double)zv[s];
          acc[8 + s] += (s < S) ? bv[s] * bv[s] : 0.0;
        }
        stv<VT, LD>(a.r, row, rv);
        stv<VT, LD>(a.rec0, 2 * row, zv);
        stv<VT, LD>(a.rec0, 2 * row + 1, zv);
        stv<VT, LD>(a.xi, row, zero);
      }
    }
    block_partial<12>(acc, a.part, sh);
  }
  ok = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok) grid_totals<12>(a.part, s_tot, s_buf);
  if (threadIdx.x == 0) {
    for (int s = 0; s < 4; s++) {
      const bool use = s < S && ok;
      const double rr = use ? s_tot[s] : 0.0, rz = use ? s_tot[4 + s] : 0.0;
      const double bb = use ? s_tot[8 + s] : 0.0;
      const double rt = use ? a.rtol[s] : 0.0;
      L.bb[s] = bb;
      L.tol2[s] = rt * rt * bb;
      L.rr[s] = rr;
      L.rtrue[s] = rr;
      L.rmax2[s] = rr;
      L.rz[s] = rz;
      L.alpha[s] = 0.0;
      L.beta[s] = 0.0;
      L.trigger[s] = 0;
      L.iters[s] = 0;
      const bool fin = isfinite(rr) && isfinite(rz);
      const bool act = use && fin && rr > L.tol2[s];
      L.active[s] = act;
      L.status[s] = !use ? TP_OK : (!fin ? TP_ERR_NONFINITE : (act ? -1 : TP_OK));
    }
  }
  __syncthreads();

  clk.lap(7);  // init phases
  int it = 0, n_rel = 0, par = 0;
  while (ok && it < a.max_it) {
    int nact = 0;
#pragma unroll
    for (int s = 0; s < 4; s++) nact += L.active[s];
    if (!nact) break;
    const VT* __restrict__ rec_o = par ? a.rec1 : a.rec0;
    VT* rec_n = par ? a.rec0 : a.rec1;
    // ---- A: p = z + beta p_old for own rows and, on the fly, for every gathered
    //         neighbour; q = A p; p.q
    {
      VT be[LD];
      bool act[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) {
        act[s] = (s < S) && L.active[s];
        be[s] = act[s] ? (VT)L.beta[s] : VT(0);
      }
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      int sl = sb + warp;
      if (sl < se) {
        int base = s_sp[sl - sb], w = (s_sp[sl - sb + 1] - base) >> 5, k = 0;
        int cc[U];
        VT vv[U], mm[HASM ? U : 1];
        stage_group<VT, U, HASM>(a, base, w, 0, lane, cc, vv, mm);
        VT ak[LD], am[LD];
#pragma unroll
        for (int s = 0; s < LD; s++) ak[s] = am[s] = VT(0);
        while (true) {
          const bool last = k + U >= w;  // last group of this slice
          const int nsl = last ? sl + nwarps : sl;
          const int nk = last ? 0 : k + U;
          const bool more = nsl < se;
          int nbase = base, nw = w;
          if (last && more) {
            nbase = s_sp[nsl - sb];
            nw = (s_sp[nsl - sb + 1] - nbase) >> 5;
          }
          int cn[U];
          VT vn[U], mn[HASM ? U : 1];
          if (more) stage_group<VT, U, HASM>(a, nbase, nw, nk, lane, cn, vn, mn);
          const int64_t row = (int64_t)sl * 32 + lane;
          const bool own = last && row < a.n;
          VT zr[LD], por[LD], dr[LD];
#pragma unroll
          for (int s = 0; s < LD; s++) zr[s] = por[s] = dr[s] = VT(0);
          bool bcr = false;
          if (own) {
            ld_rec<VT, LD>(rec_o, row, zr, por);
            if (a.diag) ldv<VT, LD>(a.diag, row, dr);
            bcr = a.bc && a.bc[row];
          }
          VT zg[U][LD], pg[U][LD];
#pragma unroll
          for (int u = 0; u < U; u++) ld_rec<VT, LD>(rec_o, cc[u], zg[u], pg[u]);
#pragma unroll
          for (int u = 0; u < U; u++) {
#pragma unroll
            for (int s = 0; s < LD; s++) {
              const VT pj = act[s] ? zg[u][s] + be[s] * pg[u][s] : pg[u][s];
              ak[s] += vv[u] * pj;
              if constexpr (HASM) am[s] += mm[u] * pj;
            }
          }
          if (last) {
            if (own) {
              VT pr[LD], qv[LD];
#pragma unroll
              for (int s = 0; s < LD; s++) pr[s] = act[s] ? zr[s] + be[s] * por[s] : por[s];
              stv<VT, LD>(rec_n, 2 * row + 1, pr);
#pragma unroll
              for (int s = 0; s < LD; s++) {
                const VT v = VT(a.dscale[s]) * ak[s] + VT(a.cscale[s]) * am[s] + dr[s] * pr[s];
                qv[s] = bcr ? pr[s] : v;
                acc[s] += (double)pr[s] * (double)qv[s];
              }
              stv<VT, LD>(a.q, row, qv);
            }
#pragma unroll
            for (int s = 0; s < LD; s++) ak[s] = am[s] = VT(0);
          }
          if (!more) break;
          sl = nsl;
          k = nk;
          base = nbase;
          w = nw;
#pragma unroll
          for (int u = 0; u < U; u++) {
            cc[u] = cn[u];
            vv[u] = vn[u];
            if constexpr (HASM) mm[u] = mn[u];
          }
        }
      }
      block_partial<4>(acc, a.part, sh);
    }
    clk.lap(0);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
    clk.lap(1);
    if (!ok) break;
    grid_totals<4>(a.part, s_tot, s_buf);
    if (threadIdx.x == 0) {
      for (int s = 0; s < S; s++) {
        if (!L.active[s]) {
          L.alpha[s] = 0.0;
          continue;
        }
        const double pq = s_tot[s];
        if (!isfinite(pq) || !(pq > 0.0)) {
          L.alpha[s] = 0.0;
          L.active[s] = 0;
          L.status[s] = isfinite(pq) ? TP_ERR_BREAKDOWN : TP_ERR_NONFINITE;
          L.iters[s] = it;
          continue;
        }
        L.alpha[s] = L.rz[s] / pq;
      }
    }
    __syncthreads();
    // ---- B: xi += alpha p, r -= alpha q, z = D^-1 r; r.z, r.r
    {
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; k++) acc[k] = 0.0;
      VT al[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) al[s] = (s < S) ? (VT)L.alpha[s] : VT(0);
      constexpr int RS = (LD * sizeof(VT) <= 8) ? 2 : 1;  // rows per step (registers)
      for (int sl = sb + warp; sl < se; sl += RS * nwarps) {
        const int sl1 = (RS == 2) ? sl + nwarps : se;
        const int64_t rw[2] = {(int64_t)sl * 32 + lane, (int64_t)sl1 * 32 + lane};
        const bool vr[2] = {rw[0] < a.n, sl1 < se && rw[1] < a.n};
        VT pv[2][LD], qv[2][LD], rv[2][LD], xv[2][LD], dv[2][LD];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          if (vr[h]) {
            ldv_cg<VT, LD>(rec_n, 2 * rw[h] + 1, pv[h]);
            ldv_cg<VT, LD>(a.q, rw[h], qv[h]);
            ldv_cg<VT, LD>(a.r, rw[h], rv[h]);
            ldv_cg<VT, LD>(a.xi, rw[h], xv[h]);
            ldv_cg<VT, LD>(a.dinv, rw[h], dv[h]);
          }
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          if (vr[h]) {
            VT zv[LD];
#pragma unroll
            for (int s = 0; s < LD; s++) {
              xv[h][s] += al[s] * pv[h][s];
              rv[h][s] -= al[s] * qv[h][s];
              zv[s] = dv[h][s] * rv[h][s];
              acc[s] += (double)rv[h][s] * (double)zv[s];
              acc[4 + s] += (double)rv[h][s] * (double)rv[h][s];
            }
            stv<VT, LD>(a.xi, rw[h], xv[h]);
            stv<VT, LD>(a.r, rw[h], rv[h]);
            stv<VT, LD>(rec_n, 2 * rw[h], zv);
          }
        }
      }
      block_partial<8>(acc, a.part, sh);
    }
    clk.lap(2);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
    clk.lap(3);
    if (!ok) break;
    grid_totals<8>(a.part, s_tot, s_buf);
    if (threadIdx.x == 0) {
      int any = 0;
      for (int s = 0; s < S; s++) {
        L.trigger[s] = 0;
        if (!L.active[s]) {
          L.beta[s] = 0.0;
          continue;
        }
        const double rz = s_tot[s], rr = s_tot[4 + s];
        if (!isfinite(rz) || !isfinite(rr)) {
          L.active[s] = 0;
          L.status[s] = TP_ERR_NONFINITE;
          L.iters[s] = it + 1;
          continue;
        }
        const double old = L.rz[s];
        L.beta[s] = (old != 0.0) ? rz / old : 0.0;
        L.rz[s] = rz;
        L.rr[s] = rr;
        const bool trig = (rr <= L.tol2[s]) || (a.delta2 > 0.0 && rr < a.delta2 * L.rmax2[s]);
        any |= trig;
      }
      // one FP64 sweep refreshes every active lane
      if (any)
        for (int s = 0; s < S; s++) L.trigger[s] = L.active[s];
      s_anytrig = any;
    }
    __syncthreads();
    it++;
    clk.lap(4);  // scalar updates
    if (s_anytrig) {
      // ---- RU1: x += xi on trigger lanes
      int tr[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) tr[s] = (s < S) ? L.trigger[s] : 0;
      FOR_OWN_ROWS {
        VT xv[LD];
        ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (tr[s]) {
            a.x[row * LD + s] += (double)xv[s];
            xv[s] = VT(0);
          }
        }
        stv<VT, LD>(a.xi, row, xv);
      }
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      // ---- RU2: FP64 residual on trigger lanes, replace r and z (z of the next record)
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; k++) acc[k] = 0.0;
      FOR_OWN_ROWS {
        double r64[LD];
        csr64_residual<VT, LD>(a, row, r64);
        VT rv[LD], dv[LD], zv[LD];
        ldv_cg<VT, LD>(a.r, row, rv);
        ldv_cg<VT, LD>(a.dinv, row, dv);
        ldv_cg<VT, LD>(rec_n, 2 * row, zv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (tr[s]) {
            rv[s] = (VT)r64[s];
            zv[s] = dv[s] * rv[s];
            acc[s] += r64[s] * r64[s];
            acc[4 + s] += (double)rv[s] * (double)zv[s];
          }
        }
        stv<VT, LD>(a.r, row, rv);
        stv<VT, LD>(rec_n, 2 * row, zv);
      }
      block_partial<8>(acc, a.part, sh);
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      grid_totals<8>(a.part, s_tot, s_buf);
      if (threadIdx.x == 0) {
        n_rel++;
        for (int s = 0; s < S; s++) {
          if (!L.trigger[s]) continue;
          L.trigger[s] = 0;
          const double rr = s_tot[s], rz = s_tot[4 + s];
          L.rtrue[s] = rr;
          if (!isfinite(rr)) {
            L.active[s] = 0;
            L.status[s] = TP_ERR_NONFINITE;
            L.iters[s] = it;
          } else if (rr <= L.tol2[s]) {
            L.active[s] = 0;
            L.status[s] = TP_OK;
            L.iters[s] = it;
          } else {
            L.rz[s] = rz;
            L.rr[s] = rr;
            L.rmax2[s] = rr;
          }
        }
      }
      __syncthreads();
      clk.lap(5);  // reliable update
    }
    par ^= 1;
  }

  // ---- final: x += xi, true residual norms
  FOR_OWN_ROWS {
    VT xv[LD];
    ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
    for (int s = 0; s < LD; s++) {
      if (s < S) a.x[row * LD + s] += (double)xv[s];
      xv[s] = VT(0);
    }
    stv<VT, LD>(a.xi, row, xv);
  }
  bool ok2 = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok2) {
      FOR_OWN_ROWS {
        double r64[LD];
        csr64_residual<VT, LD>(a, row, r64);
#pragma unroll
        for (int s = 0; s < LD; s++) acc[s] += r64[s] * r64[s];
      }
    }
    block_partial<4>(acc, a.part, sh);
  }
  ok2 = ok2 && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok2) grid_totals<4>(a.part, s_tot, s_buf);
  if (clk.on) {
    clk.lap(6);
#pragma unroll
    for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // a CTA that gave up at the last barrier leaves only the flag behind
    if (ld_acquire(&a.bar->abort)) ok2 = false;
    int status = TP_OK;
    for (int s = 0; s < 4; s++) {
      if (s < S) {
        if (ok2) L.rtrue[s] = s_tot[s];
        if (L.status[s] == -1) {
          L.status[s] = (ok2 && L.rtrue[s] <= L.tol2[s]) ? TP_OK : TP_ERR_NOT_CONVERGED;
          L.iters[s] = it;
        }
        if (!ok2) L.status[s] = TP_ERR_TIMEOUT;
        if (L.status[s] != TP_OK && status == TP_OK) status = L.status[s];
      }
      a.out->lane_iters[s] = L.iters[s];
      a.out->lane_status[s] = L.status[s];
      a.out->lane_rtrue[s] = L.rtrue[s];
      a.out->lane_bb[s] = L.bb[s];
    }
    a.out->iterations = it;
    a.out->n_reliable = n_rel;
    a.out->status = status;
    a.out->timeouts = ok2 ? 0 : 1;
  }
#undef FOR_OWN_ROWS
}

// ================================================================= window engine
// Chronopoulos-Gear form of the same Jacobi-PCG: one operator product and one reduction
// step per iteration, algebraically the same iterates as the standard recurrences:
//   u = D^-1 r, w = A u, gamma = r.u, delta = w.u,
//   beta = gamma / gamma_old, alpha = gamma / (delta - beta gamma / alpha_old),
//   p = u + beta p, s = w + beta s, xi += alpha p, r -= alpha s.
// The only vector another CTA reads is u.  Every other vector is touched by its owning
// CTA only, and the operator product runs from shared memory: each CTA copies u of its
// own rows plus its halo (the columns outside its row range that its rows reference) into
// a shared-memory window with asynchronous copies, and reads the window through CTA-local
// 16-bit column indices that stay resident for the whole solve.  The SELL values are
// staged in registers, MAXS slices per warp at a time (one memory round trip for all).
//
//   init  I1 Jacobi diagonal, Dirichlet values, p = s = xi = 0 | barrier
//         I2 r = b - A64 x, u = D^-1 r, publish u; r.u, r.r, b.b | barrier
//         W  w = A u; w.u                                    | barrier -> alpha, beta = 0
//   loop  P  p = u + beta p, s = w + beta s, xi += alpha p, r -= alpha s, u = D^-1 r,
//            publish u; r.u, r.r                             | barrier
//         W  w = A u; w.u                                    | barrier -> convergence /
//                                                              trigger, beta, alpha
//         RU (when triggered) x += xi | barrier | r = b - A64 x, u = D^-1 r; r.u, r.r |
//            barrier | W | barrier -> convergence on the FP64 residual, beta, alpha
//   final x += xi | barrier | r = b - A64 x -> true residual norms

// beta = gamma / gamma_old, alpha = gamma / (delta - beta gamma / alpha_old).  The
// denominator equals p.Ap; when rounding makes the difference non-positive the direction
// restarts (beta = 0, alpha = gamma / delta); delta = u.Au itself not positive means the
// operator is not SPD on the free dofs.
__device__ __forceinline__ void cg_coefficients(LaneState& L, int s, double gm, double dl,
                                                int it) {
  if (!(dl > 0.0)) {
    L.active[s] = 0;
    L.status[s] = TP_ERR_BREAKDOWN;
    L.iters[s] = it;
    return;
  }
  double beta = (L.rz[s] != 0.0) ? gm / L.rz[s] : 0.0;
  double den = (L.alpha[s] != 0.0) ? dl - beta * gm / L.alpha[s] : dl;
  if (!(den > 0.0)) {
    beta = 0.0;
    den = dl;
  }
  L.beta[s] = beta;
  L.alpha[s] = gm / den;
  L.rz[s] = gm;
}

// lane results and status (block 0, thread 0); s_tot holds the final true r.r
// have_final: s_tot holds the final FP64 residual norms of every lane (else each lane's
// rtrue is the one of the sweep that confirmed it)
template <typename VT>
__device__ void write_result(const PArgs<VT>& a, LaneState& L, bool ok2, const double* s_tot,
                             int it, int n_rel, bool have_final = true) {
  // a CTA that gave up at the last barrier leaves only the flag behind
  if (ld_acquire(&a.bar->abort)) ok2 = false;
  int status = TP_OK;
  for (int s = 0; s < 4; s++) {
    if (s < a.S) {
      if (ok2 && have_final) L.rtrue[s] = s_tot[s];
      if (L.status[s] == -1) {
        L.status[s] = (ok2 && L.rtrue[s] <= L.tol2[s]) ? TP_OK : TP_ERR_NOT_CONVERGED;
        L.iters[s] = it;
      }
      if (!ok2) L.status[s] = TP_ERR_TIMEOUT;
      if (L.status[s] != TP_OK && status == TP_OK) status = L.status[s];
    }
    a.out->lane_iters[s] = L.iters[s];
    a.out->lane_status[s] = L.status[s];
    a.out->lane_rtrue[s] = L.rtrue[s];
    a.out->lane_bb[s] = L.bb[s];
  }
  a.out->iterations = it;
  a.out->n_reliable = n_rel;
  a.out->status = status;
  a.out->timeouts = ok2 ? 0 : 1;
}

// Tensor memory (256 KB per SM) as an on-chip home for the operator values of a solve:
// one warp allocates, every warp stores the values of its slices into its own lane
// quarter (warp w reaches lanes 32 (w % 4) .. 32 (w % 4) + 31: one lane per row of a
// 32-row slice) and reads them back with one 16-column load per slice per product.
__device__ __forceinline__ void tm_alloc(uint32_t* slot, uint32_t ncols) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(slot);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tm_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tm_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tm_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tm_st16(uint32_t taddr, const uint32_t v[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15,%16};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
      "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
      "r"(v[15])
      : "memory");
}
__device__ __forceinline__ void tm_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// 16 consecutive 32-bit columns of this thread's lane; complete after tm_wait_ld()
__device__ __forceinline__ void tm_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tm_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
constexpr uint32_t TM_COLS = 256;  // 4 column blocks of 64: warps w and w + 4k share lanes

template <typename VT, int LD, int U, bool HASM>
__global__ void __launch_bounds__(512, 1) k_cgw(PArgs<VT> a) {
  // dynamic shared memory: slice offsets (sp_cap), halo list (halo_cap), window-local
  // columns (col_cap), then the window of u (own rows, then halo; LD values each)
  extern __shared__ __align__(16) unsigned char s_dyn[];
  int32_t* s_sp = reinterpret_cast<int32_t*>(s_dyn);
  int32_t* s_halo = s_sp + a.sp_cap;
  uint16_t* s_col = reinterpret_cast<uint16_t*>(s_halo + a.halo_cap);
  VT* s_win = reinterpret_cast<VT*>(
      s_dyn + ((4 * (size_t)(a.sp_cap + a.halo_cap) + 2 * (size_t)a.col_cap + 15) & ~(size_t)15));
  VT* s_w = s_win + (size_t)a.win_cap * LD;  // w = A u of the own rows
  __shared__ double sh[32 * 12];
  __shared__ double s_buf[512];
  __shared__ double s_tot[16];
  __shared__ LaneState L;
  __shared__ int s_anytrig;
  __shared__ unsigned long long s_clk[8];
  constexpr int WMAX = 16;  // register-staged slices: at most WMAX entries per row
  constexpr int MAXS = std::max(1, 64 / (WMAX * (int)sizeof(VT) / 4 * (HASM ? 2 : 1)));
  constexpr int RB = LD * (int)sizeof(VT);  // bytes of one row of u
  unsigned int target = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int sb = (int)((int64_t)blockIdx.x * a.ns / gridDim.x);
  const int se = (int)((int64_t)(blockIdx.x + 1) * a.ns / gridDim.x);
  const int S = a.S;
  const int r0 = sb * 32;
  const int nown = (se > sb) ? (int)(min((int64_t)se * 32, a.n) - r0) : 0;
  const int nhalo = a.halo_ptr[blockIdx.x + 1] - a.halo_ptr[blockIdx.x];
  PhaseClock clk;
  clk.start(a.prof != nullptr, s_clk);
  // resident tables; read only after the first barrier (whose __syncthreads orders them)
  for (int i = threadIdx.x; i <= se - sb; i += blockDim.x) s_sp[i] = a.slice_ptr[sb + i];
  {
    const int hb = a.halo_ptr[blockIdx.x];
    for (int i = threadIdx.x; i < nhalo; i += blockDim.x) s_halo[i] = a.halo[hb + i];
    if (se > sb) {
      // this CTA's SELL columns: a multiple of 32 entries starting at a multiple of 32
      const int e0 = a.slice_ptr[sb], ne = a.slice_ptr[se] - e0;
      const uint4* src = reinterpret_cast<const uint4*>(a.loc_col + e0);
      uint4* dst = reinterpret_cast<uint4*>(s_col);
      for (int i = threadIdx.x; i < ne / 8; i += blockDim.x) dst[i] = src[i];
    }
  }
  // FP32 values into tensor memory (the host enables this only for 16 warps, slices of at
  // most 16 entries and at most MAXS slices per warp): warp w, its j-th slice sb + w + 16 j
  // at lanes 32 (w % 4).., columns 64 (w / 4) + 16 j
  __shared__ uint32_t s_taddr;
  uint32_t tm_warp = 0;
  const bool use_tm = sizeof(VT) == 4 && !HASM && a.tmem_values;
  if (use_tm) {
    if (warp == 0) tm_alloc(&s_taddr, TM_COLS);
    tm_fence_before();
    __syncthreads();
    tm_fence_after();
    tm_warp = s_taddr + ((uint32_t)(32 * (warp & 3)) << 16) + 64u * (uint32_t)(warp >> 2);
#pragma unroll
    for (int j = 0; j < MAXS; j++) {
      const int sl = sb + warp + j * nwarps;
      uint32_t v[16];
      const int base = (sl < se) ? a.slice_ptr[sl] : 0;
      const int w = (sl < se) ? (a.slice_ptr[sl + 1] - base) >> 5 : 0;
#pragma unroll
      for (int k = 0; k < 16; k++)
        v[k] = (k < w) ? __float_as_uint((float)ld_na(a.sK + base + k * 32 + lane)) : 0u;
      tm_st16(tm_warp + 16u * (uint32_t)j, v);
    }
    tm_wait_st();
  }
  auto tm_release = [&]() {
    if (use_tm) {
      tm_fence_before();
      __syncthreads();
      if (warp == 0) tm_dealloc(s_taddr, TM_COLS);
    }
  };

#define FOR_OWN_ROWS                                              \
  for (int sl = sb + warp; sl < se; sl += nwarps)                 \
    for (int64_t row = (int64_t)sl * 32 + lane; row < a.n; row = a.n)

  // w = A u for the own rows from the window; w.u partials into acc.  fill_window issues
  // the copies (own_done: the own rows of the window already hold u -- the P phase wrote
  // them -- only the halo is copied); product_rows waits for them and multiplies.
  auto fill_window = [&](bool own_done) {
    const int W = nown + nhalo;
    for (int i = (own_done ? nown : 0) + threadIdx.x; i < W; i += blockDim.x) {
      const int64_t g = (i < nown) ? (int64_t)(r0 + i) : (int64_t)s_halo[i - nown];
      const VT* src = a.u + g * LD;
      VT* dst = s_win + (size_t)i * LD;
      if constexpr (RB <= 16) {
        cp_async<RB>(dst, src);
      } else {
        constexpr int E = 16 / (int)sizeof(VT);
#pragma unroll
        for (int k = 0; k < RB / 16; k++) cp_async<16>(dst + k * E, src + k * E);
      }
    }
  };
  auto product_rows = [&](double acc[4]) {
    cp_async_wait_all();
    __syncthreads();
    const int e0 = s_sp[0];
    // dr: the row's diagonal (loaded by the caller)
    auto row_done = [&](int sl, const VT ak[LD], const VT am[LD], const VT dr[LD]) {
      const int64_t row = (int64_t)sl * 32 + lane;
      if (row < a.n) {
        VT ur[LD], wv[LD];
        ld_win<VT, LD>(s_win, (int)(row - r0), ur);
        const bool bcr = a.bc && a.bc[row];
#pragma unroll
        for (int s = 0; s < LD; s++) {
          const VT v = VT(a.dscale[s]) * ak[s] + VT(a.cscale[s]) * am[s] + dr[s] * ur[s];
          wv[s] = bcr ? ur[s] : v;
          acc[s] += (double)wv[s] * (double)ur[s];
        }
        st_win<VT, LD>(s_w, (int)(row - r0), wv);
      }
    };
    if (a.reg_values) {
      for (int slb = sb + warp; slb < se; slb += MAXS * nwarps) {
        VT vals[MAXS][WMAX];
        VT mvals[HASM ? MAXS : 1][HASM ? WMAX : 1];
        if constexpr (sizeof(VT) == 4 && !HASM && WMAX == 16) {
          if (use_tm) {
            // one round per warp (slb == sb + warp): the values of its slices, on chip
#pragma unroll
            for (int j = 0; j < MAXS; j++)
              tm_ld16(tm_warp + 16u * (uint32_t)j, reinterpret_cast<float*>(vals[j]));
            tm_wait_ld();
          }
        }
#pragma unroll
        for (int j = 0; j < MAXS; j++) {
          if (use_tm) break;
          const int sl = slb + j * nwarps;
          const int base = (sl < se) ? s_sp[sl - sb] : 0;
          const int w = (sl < se) ? (s_sp[sl - sb + 1] - base) >> 5 : 0;
#pragma unroll
          for (int k = 0; k < WMAX; k++) {
            vals[j][k] = (k < w) ? ld_na(a.sK + base + k * 32 + lane) : VT(0);
            if constexpr (HASM) mvals[j][k] = (k < w) ? ld_na(a.sM + base + k * 32 + lane) : VT(0);
          }
        }
        // the slab rows' diagonals: issued with the values for rows of at most 8 bytes
        // (wider rows have no registers to spare and load them per slice)
        constexpr bool DPRE = RB <= 8;
        VT dgs[MAXS][LD];
        auto load_diag = [&](int j) {
          const int64_t row = (int64_t)(slb + j * nwarps) * 32 + lane;
#pragma unroll
          for (int s = 0; s < LD; s++) dgs[j][s] = VT(0);
          if (a.diag && slb + j * nwarps < se && row < a.n) ldv<VT, LD>(a.diag, row, dgs[j]);
        };
        if constexpr (DPRE) {
#pragma unroll
          for (int j = 0; j < MAXS; j++) load_diag(j);
        }
#pragma unroll
        for (int j = 0; j < MAXS; j++) {
          const int sl = slb + j * nwarps;
          if (sl < se) {
            const int base = s_sp[sl - sb], w = (s_sp[sl - sb + 1] - base) >> 5;
            const int lb = base - e0;
            // wider FP32 rows without a mass matrix: the slice's diagonal is issued before
            // its gathers, which hide the load (the other forms have no registers left)
            constexpr bool DEARLY = !DPRE && !HASM && sizeof(VT) == 4;
            if constexpr (DEARLY) load_diag(j);
            VT ak[LD], am[LD];
#pragma unroll
            for (int s = 0; s < LD; s++) ak[s] = am[s] = VT(0);
#pragma unroll
            for (int k = 0; k < WMAX; k++) {
              if (k < w) {
                VT pv[LD];
                ld_win<VT, LD>(s_win, s_col[lb + k * 32 + lane], pv);
#pragma unroll
                for (int s = 0; s < LD; s++) {
                  ak[s] += vals[j][k] * pv[s];
                  if constexpr (HASM) am[s] += mvals[j][k] * pv[s];
                }
              }
            }
            if constexpr (!DPRE && !DEARLY) load_diag(j);
            row_done(sl, ak, am, dgs[j]);
          }
        }
      }
    } else {
      for (int sl = sb + warp; sl < se; sl += nwarps) {
        const int base = s_sp[sl - sb], w = (s_sp[sl - sb + 1] - base) >> 5;
        const int lb = base - e0;
        VT ak[LD], am[LD];
#pragma unroll
        for (int s = 0; s < LD; s++) ak[s] = am[s] = VT(0);
        VT vv[U], mm[HASM ? U : 1];
        stage_values<VT, U, HASM>(a, base, w, 0, lane, vv, mm);
        for (int k = 0; k < w; k += U) {
          VT vn[U], mn[HASM ? U : 1];
          if (k + U < w) stage_values<VT, U, HASM>(a, base, w, k + U, lane, vn, mn);
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (k + u < w) {
              VT pv[LD];
              ld_win<VT, LD>(s_win, s_col[lb + (k + u) * 32 + lane], pv);
#pragma unroll
              for (int s = 0; s < LD; s++) {
                ak[s] += vv[u] * pv[s];
                if constexpr (HASM) am[s] += mm[u] * pv[s];
              }
            }
          }
#pragma unroll
          for (int u = 0; u < U; u++) {
            vv[u] = vn[u];
            if constexpr (HASM) mm[u] = mn[u];
          }
        }
        VT dr[LD];
#pragma unroll
        for (int s = 0; s < LD; s++) dr[s] = VT(0);
        if (a.diag && (int64_t)sl * 32 + lane < a.n) ldv<VT, LD>(a.diag, (int64_t)sl * 32 + lane, dr);
        row_done(sl, ak, am, dr);
      }
    }
  };

  auto product = [&](double acc[4], bool own_done) {
    fill_window(own_done);
    product_rows(acc);
  };

  // residual refresh of the lanes in tr: r = b - A64 x (FP64), u = D^-1 r, publish u;
  // partials [r.u | r.r (FP64) | b.b]
  auto refresh = [&](const int tr[LD], double acc[12]) {
    FOR_OWN_ROWS {
      double r64[LD];
      csr64_residual<VT, LD>(a, row, r64);
      VT rv[LD], dv[LD], uv[LD];
      ldv_cg<VT, LD>(a.r, row, rv);
      ldv_cg<VT, LD>(a.dinv, row, dv);
      ldv_cg<VT, LD>(a.u, row, uv);
      double bv[LD];
      ldv_cg<double, LD>(a.b, row, bv);
#pragma unroll
      for (int s = 0; s < LD; s++) {
        if (tr[s]) {
          rv[s] = (VT)r64[s];
          uv[s] = dv[s] * rv[s];
          acc[s] += (double)rv[s] * (double)uv[s];
          acc[4 + s] += r64[s] * r64[s];
          acc[8 + s] += (s < S) ? bv[s] * bv[s] : 0.0;
        }
      }
      stv<VT, LD>(a.r, row, rv);
      stv<VT, LD>(a.u, row, uv);
    }
  };

  // The FP64 residual with x read through the shared-memory window (own rows + halo at
  // their window-local columns) instead of CSR gathers from global memory.  x is FP64, so
  // a window entry holds CP = RB / 8 of its columns and the own rows are walked LD / CP
  // times.  Each row sums its CSR entries in order (the SELL entries k < row length of a
  // row are its CSR entries, in order), as csr64_residual does.
  //   final = false: the refresh above (lanes in tr): r, u and partials [r.u | r.r | b.b]
  //   final = true:  partials r.r of every lane into acc[0..3], nothing written
  constexpr int CP = (RB >= 8) ? RB / 8 : 1;
  constexpr bool WINRES = (RB % 8 == 0) && (LD % CP == 0);
  auto refresh_win = [&](const int tr[LD], double* acc, bool final) {
    const int W = nown + nhalo;
    const int e0 = s_sp[0];
    double* s_x = reinterpret_cast<double*>(s_win);  // entry i: CP doubles at s_x + i CP
#pragma unroll
    for (int c0 = 0; c0 < LD; c0 += CP) {
      __syncthreads();  // the window may still be read (previous pass or product)
      for (int i = threadIdx.x; i < W; i += blockDim.x) {
        const int64_t g = (i < nown) ? (int64_t)(r0 + i) : (int64_t)s_halo[i - nown];
        double* dst = s_x + (size_t)i * CP;
        const double* src = a.x + g * LD + c0;
        if constexpr (CP == 1) {
          cp_async<8>(dst, src);
        } else {
#pragma unroll
          for (int k = 0; k < CP / 2; k++) cp_async<16>(dst + 2 * k, src + 2 * k);
        }
      }
      cp_async_wait_all();
      __syncthreads();
      FOR_OWN_ROWS {
        const int lr = (int)(row - r0);
        double xo[CP], ax[CP];
#pragma unroll
        for (int c = 0; c < CP; c++) xo[c] = s_x[lr * CP + c];
        const bool bcr = a.bc && a.bc[row];
        if (bcr) {
#pragma unroll
          for (int c = 0; c < CP; c++) ax[c] = xo[c];
        } else {
          double ak[CP], am[CP];
#pragma unroll
          for (int c = 0; c < CP; c++) ak[c] = am[c] = 0.0;
          const int p0 = a.A64.indptr[row], len = a.A64.indptr[row + 1] - p0;
          const int lb = s_sp[sl - sb] - e0;
#pragma unroll 4
          for (int k = 0; k < len; k++) {
            const int loc = s_col[lb + k * 32 + lane];
            const double kv = __ldg(a.A64.K + p0 + k);
            const double mv = a.A64.M ? __ldg(a.A64.M + p0 + k) : 0.0;
#pragma unroll
            for (int c = 0; c < CP; c++) {
              const double xv = s_x[loc * CP + c];
              ak[c] += kv * xv;
              if (a.A64.M) am[c] += mv * xv;
            }
          }
#pragma unroll
          for (int c = 0; c < CP; c++) {
            const double dr = a.A64.diag ? a.A64.diag[row * LD + c0 + c] : 0.0;
            ax[c] = a.dscale[c0 + c] * ak[c] + a.cscale[c0 + c] * am[c] + dr * xo[c];
          }
        }
#pragma unroll
        for (int c = 0; c < CP; c++) {
          const int s = c0 + c;
          const double bv = (s < S) ? a.b[row * LD + s] : 0.0;
          const double r64 = (s < S) ? bv - ax[c] : 0.0;
          if (final) {
            acc[s] += r64 * r64;
          } else if (tr[s]) {
            const VT rv = (VT)r64;
            const VT uv = a.dinv[row * LD + s] * rv;
            acc[s] += (double)rv * (double)uv;
            acc[4 + s] += r64 * r64;
            acc[8 + s] += bv * bv;
            a.r[row * LD + s] = rv;
            a.u[row * LD + s] = uv;
          }
        }
      }
    }
  };

  // ---- I1: Jacobi diagonal (FP64 values), Dirichlet values into x, p = s = xi = 0
  FOR_OWN_ROWS {
    VT dv[LD], zero[LD], rz[LD];
    const bool bcr = a.bc && a.bc[row];
#pragma unroll
    for (int s = 0; s < LD; s++) zero[s] = rz[s] = VT(0);
    if (bcr) {
#pragma unroll
      for (int s = 0; s < LD; s++) {
        dv[s] = VT(0);
        a.x[row * LD + s] = a.b[row * LD + s];
      }
    } else {
      const int lo = a.A64.indptr[row], hi = a.A64.indptr[row + 1];
      int l = lo, h = hi;
      while (l < h) {
        const int mid = (l + h) >> 1;
        if (a.A64.indices[mid] < row)
          l = mid + 1;
        else
          h = mid;
      }
      const bool found = l < hi && a.A64.indices[l] == row;
      const double kd = found ? a.A64.K[l] : 0.0;
      const double md = (a.A64.M && found) ? a.A64.M[l] : 0.0;
#pragma unroll
      for (int s = 0; s < LD; s++) {
        double d = a.dscale[s] * kd + a.cscale[s] * md;
        if (a.A64.diag) d += a.A64.diag[row * LD + s];
        dv[s] = (s < S && d != 0.0) ? VT(1.0 / d) : VT(0);
      }
    }
    stv<VT, LD>(a.dinv, row, dv);
    stv<VT, LD>(a.p, row, zero);
    stv<VT, LD>(a.s, row, zero);
    stv<VT, LD>(a.xi, row, zero);
    stv<VT, LD>(a.r, row, rz);
    stv<VT, LD>(a.u, row, rz);
  }
  bool ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);

  // ---- I2: r = b - A x, u = D^-1 r; r.u, r.r, b.b
  {
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = 0.0;
    int tr[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) tr[s] = 1;
    if (ok) {
      if constexpr (WINRES)
        refresh_win(tr, acc, false);
      else
        refresh(tr, acc);
    }
    block_partial<12>(acc, a.part, sh);
  }
  ok = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok) grid_totals<12>(a.part, s_tot, s_buf);
  if (threadIdx.x == 0) {
    for (int s = 0; s < 4; s++) {
      const bool use = s < S && ok;
      const double rz = use ? s_tot[s] : 0.0, rr = use ? s_tot[4 + s] : 0.0;
      const double bb = use ? s_tot[8 + s] : 0.0;
      const double rt = use ? a.rtol[s] : 0.0;
      L.bb[s] = bb;
      L.tol2[s] = rt * rt * bb;
      L.rr[s] = rr;
      L.rtrue[s] = rr;
      L.rmax2[s] = rr;
      L.rz[s] = rz;
      L.alpha[s] = 0.0;
      L.beta[s] = 0.0;
      L.trigger[s] = 0;
      L.frozen[s] = 0;
      L.iters[s] = 0;
      const bool fin = isfinite(rr) && isfinite(rz);
      const bool act = use && fin && rr > L.tol2[s];
      L.active[s] = act;
      L.status[s] = !use ? TP_OK : (!fin ? TP_ERR_NONFINITE : (act ? -1 : TP_OK));
    }
  }
  // ---- W: w = A u; w.u -> alpha = r.u / w.u
  {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok) product(acc, false);
    block_partial<4>(acc, a.part, sh);
  }
  ok = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok) grid_totals<4>(a.part, s_tot, s_buf);
  if (threadIdx.x == 0 && ok) {
    for (int s = 0; s < S; s++) {
      if (!L.active[s]) continue;
      const double dl = s_tot[s];
      if (!isfinite(dl)) {
        L.active[s] = 0;
        L.status[s] = TP_ERR_NONFINITE;
        continue;
      }
      const double gm = L.rz[s];
      L.rz[s] = 0.0;  // no previous gamma: beta = 0
      L.alpha[s] = 0.0;
      cg_coefficients(L, s, gm, dl, 0);
    }
  }
  __syncthreads();

  clk.lap(7);  // init phases
  int it = 0, n_rel = 0;
  while (ok && it < a.max_it) {
    int nact = 0;
#pragma unroll
    for (int s = 0; s < 4; s++) nact += L.active[s];
    if (!nact) break;
    // ---- P: p = u + beta p, s = w + beta s, xi += alpha p, r -= alpha s, u = D^-1 r;
    //         partials r.u, r.r into slots 0..7
    {
      VT al[LD], be[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) {
        const bool act = (s < S) && L.active[s] && !L.frozen[s];  // frozen lanes stand still
        al[s] = act ? (VT)L.alpha[s] : VT(0);
        be[s] = act ? (VT)L.beta[s] : VT(0);
      }
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; k++) acc[k] = 0.0;
      // distinct arrays: declared non-aliasing so loads of the next row may be issued
      // before the stores of this one
      VT* __restrict__ pP = a.p;
      VT* __restrict__ pS = a.s;
      VT* __restrict__ pX = a.xi;
      VT* __restrict__ pR = a.r;
      VT* __restrict__ pU = a.u;
      const VT* __restrict__ pD = a.dinv;
#pragma unroll 2
      for (int sl = sb + warp; sl < se; sl += nwarps) {
        const int64_t row = (int64_t)sl * 32 + lane;
        if (row >= a.n) continue;
        const int lr = (int)(row - r0);
        VT uv[LD], wv[LD], pv[LD], sv[LD], xv[LD], rv[LD], dv[LD];
        ldv_cg<VT, LD>(pP, row, pv);
        ldv_cg<VT, LD>(pS, row, sv);
        ldv_cg<VT, LD>(pX, row, xv);
        ldv_cg<VT, LD>(pR, row, rv);
        ldv_cg<VT, LD>(pD, row, dv);
        ld_win<VT, LD>(s_win, lr, uv);  // u of the own rows, last window
        ld_win<VT, LD>(s_w, lr, wv);    // w = A u of the own rows, last product
#pragma unroll
        for (int s = 0; s < LD; s++) {
          pv[s] = uv[s] + be[s] * pv[s];
          sv[s] = wv[s] + be[s] * sv[s];
          xv[s] += al[s] * pv[s];
          rv[s] -= al[s] * sv[s];
          uv[s] = dv[s] * rv[s];
          acc[s] += (double)rv[s] * (double)uv[s];
          acc[4 + s] += (double)rv[s] * (double)rv[s];
        }
        stv<VT, LD>(pP, row, pv);
        stv<VT, LD>(pS, row, sv);
        stv<VT, LD>(pX, row, xv);
        stv<VT, LD>(pR, row, rv);
        stv<VT, LD>(pU, row, uv);
        st_win<VT, LD>(s_win, lr, uv);  // the next product reads it from here
      }
      block_partial<8>(acc, a.part, sh);
    }
    clk.lap(2);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);  // u published
    clk.lap(3);
    if (!ok) break;
    // ---- W: w = A u; w.u into slots 8..11.  The three sums are read together below.
    {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      fill_window(true);
      grid_totals<8, 0>(a.part, s_tot, s_buf);  // r.u, r.r of this P phase: final already
      product_rows(acc);
      block_partial<4>(acc, a.part + 8, sh);
    }
    clk.lap(0);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
    clk.lap(1);
    if (!ok) break;
    grid_totals<4, 8>(a.part, s_tot, s_buf);
    it++;
    // lanes in parallel: thread s owns lane s.  A lane whose recurrence residual reaches
    // the tolerance freezes (its columns of the next steps are no-ops) instead of asking for
    // a sweep at once: the lanes converge at different iterations, and one sweep then
    // confirms them together.
    int trig = 0;
    if (threadIdx.x < S) {
      const int s = threadIdx.x;
      L.trigger[s] = 0;
      if (L.active[s] && !L.frozen[s]) {
        const double gm = s_tot[s], rr = s_tot[4 + s], dl = s_tot[8 + s];
        if (!isfinite(gm) || !isfinite(rr) || !isfinite(dl)) {
          L.active[s] = 0;
          L.status[s] = TP_ERR_NONFINITE;
          L.iters[s] = it;
        } else {
          L.rr[s] = rr;
          if (rr <= L.tol2[s])
            L.frozen[s] = 1;
          else
            trig = a.delta2 > 0.0 && rr < a.delta2 * L.rmax2[s];
        }
      }
    }
    // one FP64 sweep refreshes every active lane when any lane asks for it, or when every
    // lane still active is frozen (the same decision in every CTA: same totals)
    int any = __syncthreads_or(trig);
    if (!any) {
      int running = 0, pending = 0;
      for (int s = 0; s < S; s++) {
        running |= L.active[s] && !L.frozen[s];
        pending |= L.active[s] && L.frozen[s];
      }
      any = pending && !running;
    }
    if (threadIdx.x < S && L.active[threadIdx.x]) {
      const int s = threadIdx.x;
      if (any)
        L.trigger[s] = 1;
      else if (!L.frozen[s])
        cg_coefficients(L, s, s_tot[s], s_tot[8 + s], it);
    }
    if (threadIdx.x == 0) s_anytrig = any;
    __syncthreads();
    clk.lap(4);  // scalar updates
    if (s_anytrig) {
      // ---- RU: x += xi, then the FP64 residual replaces r, u, w and gamma, delta
      int tr[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) tr[s] = (s < S) ? L.trigger[s] : 0;
      FOR_OWN_ROWS {
        VT xv[LD];
        ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (tr[s]) {
            a.x[row * LD + s] += (double)xv[s];
            xv[s] = VT(0);
          }
        }
        stv<VT, LD>(a.xi, row, xv);
      }
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      {
        double acc[12];
#pragma unroll
        for (int k = 0; k < 12; k++) acc[k] = 0.0;
        if constexpr (WINRES)
          refresh_win(tr, acc, false);
        else
          refresh(tr, acc);
        block_partial<12>(acc, a.part, sh);  // slots 8..11 (b.b) are replaced by w.u
      }
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      // the FP64 residual sums first: when no triggered lane goes on (all converged or
      // failed) the product is skipped.  Every CTA reads the same totals, so every CTA
      // takes the same branch and the barrier counts stay equal.
      grid_totals<8, 0>(a.part, s_tot, s_buf);
      if (threadIdx.x == 0) {
        int cont = 0;
        for (int s = 0; s < S; s++)
          if (L.trigger[s] && isfinite(s_tot[s]) && isfinite(s_tot[4 + s]) &&
              s_tot[4 + s] > L.tol2[s])
            cont = 1;
        s_anytrig = cont;
        if (!cont)
          for (int s = 0; s < 4; s++) s_tot[8 + s] = 0.0;  // w.u not needed
      }
      __syncthreads();
      if (s_anytrig) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        product(acc, false);
        block_partial<4>(acc, a.part + 8, sh);
        ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
        if (!ok) break;
        grid_totals<4, 8>(a.part, s_tot, s_buf);
      }
      if (threadIdx.x == 0) {
        n_rel++;
        for (int s = 0; s < S; s++) {
          if (!L.trigger[s]) continue;
          L.trigger[s] = 0;
          L.frozen[s] = 0;
          const double gm = s_tot[s], rr = s_tot[4 + s], dl = s_tot[8 + s];
          L.rtrue[s] = rr;
          if (!isfinite(rr) || !isfinite(gm) || !isfinite(dl)) {
            L.active[s] = 0;
            L.status[s] = TP_ERR_NONFINITE;
            L.iters[s] = it;
          } else if (rr <= L.tol2[s]) {
            L.active[s] = 0;
            L.status[s] = TP_OK;
            L.iters[s] = it;
          } else {
            L.rr[s] = rr;
            L.rmax2[s] = rr;
            cg_coefficients(L, s, gm, dl, it);
          }
        }
      }
      __syncthreads();
      clk.lap(5);  // reliable update
    }
  }

  // ---- final: x += xi, true residual norms.  When every lane was confirmed by a sweep
  // (converged there, or before the first iteration), x holds its solution already (xi
  // was added and zeroed then, and the lane took no step after) and rtrue its FP64
  // residual: the pass is skipped (the same decision in every CTA).
  bool all_confirmed = true;
  for (int s = 0; s < S; s++) all_confirmed &= !L.active[s] && L.status[s] == TP_OK;
  if (ok && all_confirmed) {
    if (clk.on) {
      clk.lap(6);
#pragma unroll
      for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, true, s_tot, it, n_rel, false);
    tm_release();
    return;
  }
  FOR_OWN_ROWS {
    VT xv[LD];
    ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
    for (int s = 0; s < LD; s++) {
      if (s < S) a.x[row * LD + s] += (double)xv[s];
      xv[s] = VT(0);
    }
    stv<VT, LD>(a.xi, row, xv);
  }
  bool ok2 = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok2) {
      if constexpr (WINRES) {
        int none[LD];
#pragma unroll
        for (int s = 0; s < LD; s++) none[s] = 0;
        refresh_win(none, acc, true);
      } else {
        FOR_OWN_ROWS {
          double r64[LD];
          csr64_residual<VT, LD>(a, row, r64);
#pragma unroll
          for (int s = 0; s < LD; s++) acc[s] += r64[s] * r64[s];
        }
      }
    }
    block_partial<4>(acc, a.part, sh);
  }
  ok2 = ok2 && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok2) grid_totals<4>(a.part, s_tot, s_buf);
  if (clk.on) {
    clk.lap(6);
#pragma unroll
    for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, ok2, s_tot, it, n_rel);
  tm_release();
#undef FOR_OWN_ROWS
}

// ----------------------------------------------------------------- tensor-memory engine
// k_cgt: the window engine's FP32 solve (no mass matrix; slices of at most 16 entries; at
// most 4 slices per warp, i.e. 2048 rows per CTA) with every per-row vector of the
// recurrence on chip.  The SM's 512 tensor-memory columns hold, for warp w (lanes
// 32 (w % 4) .., columns 128 (w / 4) ..), the FP32 values of its slices (16 columns per
// slice) and one 16-column record per slice row, [p | s | xi | r] (4 columns each, the
// first LD used); D^-1 of the own rows sits in shared memory where k_cgw keeps w, and u
// in the window as before.  The only per-iteration global traffic left is the halo of u
// (written by the P phase, copied by the other CTAs) and the row diagonals.
//
// Iteration: the Chronopoulos-Gear recurrences of k_cgw, with the direction update moved
// into the product.  beta = gamma / gamma_old only needs the P-phase sums, which every CTA
// holds right after barrier B, so the product of row i also forms p_i = u_i + beta p_i and
// s_i = w_i + beta s_i, and w never leaves registers:
//
//   barrier B | halo copies in flight, gamma and r.r totals, lane decisions, beta
//             | w = A u, p = u + beta p, s = w + beta s, w.u
//   barrier A | delta total, alpha = gamma / (delta - beta gamma / alpha_old)
//             | xi += alpha p, r -= alpha s, u = D^-1 r (window and global), r.u, r.r
//   barrier B ...
//
// Partial slots per CTA: r.u 0-3, r.r 4-7, w.u 8-11, b.b 12-15 (written only by the FP64
// refreshes), so no slot is rewritten while another CTA may still read it.  A lane whose
// alpha denominator is not positive (rounding) takes no step and restarts through an FP64
// refresh (beta = 0 after it), as does a lane that was frozen.
constexpr int CGT_MAXS = 4;
constexpr int CGT_WARPS = 16;
constexpr uint32_t CGT_COLS = 512;

template <int LD>
__global__ void __launch_bounds__(512, 1) k_cgt(PArgs<float> a) {
  using VT = float;
  static_assert(LD == 2 || LD == 4, "FP64 residual windows hold LD / 2 doubles per entry");
  constexpr int CP = LD / 2;  // FP64 columns per window entry in the residual passes
  extern __shared__ __align__(16) unsigned char s_dyn[];
  int32_t* s_sp = reinterpret_cast<int32_t*>(s_dyn);
  int32_t* s_halo = s_sp + a.sp_cap;
  uint16_t* s_col = reinterpret_cast<uint16_t*>(s_halo + a.halo_cap);
  VT* s_win = reinterpret_cast<VT*>(
      s_dyn + ((4 * (size_t)(a.sp_cap + a.halo_cap) + 2 * (size_t)a.col_cap + 15) & ~(size_t)15));
  VT* s_dinv = s_win + (size_t)a.win_cap * LD;  // D^-1 of the own rows
  __shared__ double sh[32 * 12];
  __shared__ double s_buf[512];
  __shared__ double s_tot[16];
  __shared__ LaneState L;
  __shared__ double s_gm[4], s_step[4];
  __shared__ int s_restart[4];
  __shared__ uint32_t s_taddr;
  __shared__ unsigned long long s_clk[8];
  unsigned int target = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sb = (int)((int64_t)blockIdx.x * a.ns / gridDim.x);
  const int se = (int)((int64_t)(blockIdx.x + 1) * a.ns / gridDim.x);
  const int S = a.S;
  const int r0 = sb * 32;
  const int nown = (se > sb) ? (int)(min((int64_t)se * 32, a.n) - r0) : 0;
  const int nhalo = a.halo_ptr[blockIdx.x + 1] - a.halo_ptr[blockIdx.x];
  PhaseClock clk;
  clk.start(a.prof != nullptr, s_clk);
  for (int i = threadIdx.x; i <= se - sb; i += blockDim.x) s_sp[i] = a.slice_ptr[sb + i];
  {
    const int hb = a.halo_ptr[blockIdx.x];
    for (int i = threadIdx.x; i < nhalo; i += blockDim.x) s_halo[i] = a.halo[hb + i];
    if (se > sb) {
      const int e0 = a.slice_ptr[sb], ne = a.slice_ptr[se] - e0;
      const uint4* src = reinterpret_cast<const uint4*>(a.loc_col + e0);
      uint4* dst = reinterpret_cast<uint4*>(s_col);
      for (int i = threadIdx.x; i < ne / 8; i += blockDim.x) dst[i] = src[i];
    }
  }
  if (threadIdx.x < 4) s_restart[threadIdx.x] = 0;
  // ---- tensor memory: the whole of it; values of slice j at tw + 16 j, records at
  // tw + 64 + 16 j
  if (warp == 0) tm_alloc(&s_taddr, CGT_COLS);
  tm_fence_before();
  __syncthreads();
  tm_fence_after();
  const uint32_t tw = s_taddr + ((uint32_t)(32 * (warp & 3)) << 16) + 128u * (uint32_t)(warp >> 2);
  auto rec_ld = [&](int j, float rc[16]) { tm_ld16(tw + 64u + 16u * (uint32_t)j, rc); };
  auto rec_st = [&](int j, const float rc[16]) {
    uint32_t v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __float_as_uint(rc[k]);
    tm_st16(tw + 64u + 16u * (uint32_t)j, v);
  };
#pragma unroll
  for (int j = 0; j < CGT_MAXS; j++) {
    const int sl = sb + warp + j * CGT_WARPS;
    uint32_t v[16];
    const int base = (sl < se) ? a.slice_ptr[sl] : 0;
    const int w = (sl < se) ? (a.slice_ptr[sl + 1] - base) >> 5 : 0;
#pragma unroll
    for (int k = 0; k < 16; k++)
      v[k] = (k < w) ? __float_as_uint(ld_na(a.sK + base + k * 32 + lane)) : 0u;
    tm_st16(tw + 16u * (uint32_t)j, v);
  }
  tm_wait_st();

  // window of u: own rows (unless the P phase wrote them) and halo, asynchronously
  auto fill_window = [&](bool own_done) {
    const int W = nown + nhalo;
    for (int i = (own_done ? nown : 0) + threadIdx.x; i < W; i += blockDim.x) {
      const int64_t g = (i < nown) ? (int64_t)(r0 + i) : (int64_t)s_halo[i - nown];
      cp_async<LD * 4>(s_win + (size_t)i * LD, a.u + g * LD);
    }
  };

  // ---- w = A u of the own rows; p = u + beta p, s = w + beta s; w.u into acc
  auto product_rows = [&](const float be[LD], double acc[4]) {
    // the row diagonals and Dirichlet flags of this warp's rows, in flight while the
    // window copies land
    float dg[CGT_MAXS][LD];
    bool bcm[CGT_MAXS];
#pragma unroll
    for (int j = 0; j < CGT_MAXS; j++) {
      const int64_t row = (int64_t)(sb + warp + j * CGT_WARPS) * 32 + lane;
      const bool in = sb + warp + j * CGT_WARPS < se && row < a.n;
#pragma unroll
      for (int s = 0; s < LD; s++) dg[j][s] = 0.f;
      if (in && a.diag) ldv<VT, LD>(a.diag, row, dg[j]);
      bcm[j] = in && a.bc && a.bc[row];
    }
    cp_async_wait_all();
    __syncthreads();
    const int e0 = s_sp[0];
#pragma unroll
    for (int j = 0; j < CGT_MAXS; j++) {
      const int sl = sb + warp + j * CGT_WARPS;
      if (sl >= se) break;
      float vals[16], rc[16];
      tm_ld16(tw + 16u * (uint32_t)j, vals);
      rec_ld(j, rc);
      tm_wait_ld();
      const int64_t row = (int64_t)sl * 32 + lane;
      const int base = s_sp[sl - sb], w = (s_sp[sl - sb + 1] - base) >> 5;
      const int lb = base - e0;
      float ak[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) ak[s] = 0.f;
#pragma unroll
      for (int k = 0; k < 16; k++) {
        if (k < w) {
          float pv[LD];
          ld_win<VT, LD>(s_win, s_col[lb + k * 32 + lane], pv);
#pragma unroll
          for (int s = 0; s < LD; s++) ak[s] += vals[k] * pv[s];
        }
      }
      if (row < a.n) {
        float ur[LD];
        ld_win<VT, LD>(s_win, (int)(row - r0), ur);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          const float v = (float)a.dscale[s] * ak[s] + dg[j][s] * ur[s];
          const float wv = bcm[j] ? ur[s] : v;
          acc[s] += (double)wv * (double)ur[s];
          rc[s] = ur[s] + be[s] * rc[s];
          rc[4 + s] = wv + be[s] * rc[4 + s];
        }
      }
      rec_st(j, rc);
    }
    tm_wait_st();
  };

  // ---- xi += alpha p, r -= alpha s, u = D^-1 r (window and global); r.u, r.r into acc
  auto p_rows = [&](const float al[LD], double acc[8]) {
#pragma unroll
    for (int j = 0; j < CGT_MAXS; j++) {
      const int sl = sb + warp + j * CGT_WARPS;
      if (sl >= se) break;
      float rc[16];
      rec_ld(j, rc);
      tm_wait_ld();
      const int64_t row = (int64_t)sl * 32 + lane;
      if (row < a.n) {
        const int lr = (int)(row - r0);
        float dv[LD], uv[LD];
        ld_win<VT, LD>(s_dinv, lr, dv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          rc[8 + s] += al[s] * rc[s];
          rc[12 + s] -= al[s] * rc[4 + s];
          uv[s] = dv[s] * rc[12 + s];
          acc[s] += (double)rc[12 + s] * (double)uv[s];
          acc[4 + s] += (double)rc[12 + s] * (double)rc[12 + s];
        }
        st_win<VT, LD>(s_win, lr, uv);
        stv<VT, LD>(a.u, row, uv);
      }
      rec_st(j, rc);
    }
    tm_wait_st();
  };

  // ---- x += xi for the lanes in tr (xi of those lanes back to 0)
  auto add_xi = [&](const int tr[LD]) {
#pragma unroll
    for (int j = 0; j < CGT_MAXS; j++) {
      const int sl = sb + warp + j * CGT_WARPS;
      if (sl >= se) break;
      float rc[16];
      rec_ld(j, rc);
      tm_wait_ld();
      const int64_t row = (int64_t)sl * 32 + lane;
      if (row < a.n) {
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (tr[s]) {
            a.x[row * LD + s] += (double)rc[8 + s];
            rc[8 + s] = 0.f;
          }
        }
      }
      rec_st(j, rc);
    }
    tm_wait_st();
  };

  // ---- FP64 residual r64 = b - A64 x with x read through the window (CP columns per
  // pass).  final = false: for the lanes in tr, r = (float) r64 into the records, u =
  // D^-1 r into global memory (the next product refills the whole window), partials r.u
  // 0-3, r.r 4-7, b.b 8-11 of acc; final = true: r.r of every lane into acc[0..3].
  auto refresh = [&](const int tr[LD], double* acc, bool final) {
    const int W = nown + nhalo;
    const int e0 = s_sp[0];
    double* s_x = reinterpret_cast<double*>(s_win);
#pragma unroll
    for (int c0 = 0; c0 < LD; c0 += CP) {
      bool any_c = false;
#pragma unroll
      for (int c = 0; c < CP; c++) any_c |= final ? (c0 + c < S) : (tr[c0 + c] != 0);
      if (!any_c) continue;
      cp_async_wait_all();
      __syncthreads();  // the window may still be read (previous pass or product)
      for (int i = threadIdx.x; i < W; i += blockDim.x) {
        const int64_t g = (i < nown) ? (int64_t)(r0 + i) : (int64_t)s_halo[i - nown];
        cp_async<CP * 8>(s_x + (size_t)i * CP, a.x + g * LD + c0);
      }
      cp_async_wait_all();
      __syncthreads();
#pragma unroll
      for (int j = 0; j < CGT_MAXS; j++) {
        const int sl = sb + warp + j * CGT_WARPS;
        if (sl >= se) break;
        float rc[16];
        if (!final) {
          rec_ld(j, rc);
          tm_wait_ld();
        }
        const int64_t row = (int64_t)sl * 32 + lane;
        if (row < a.n) {
          const int lr = (int)(row - r0);
          double xo[CP], ax[CP];
#pragma unroll
          for (int c = 0; c < CP; c++) xo[c] = s_x[lr * CP + c];
          const bool bcr = a.bc && a.bc[row];
          if (bcr) {
#pragma unroll
            for (int c = 0; c < CP; c++) ax[c] = xo[c];
          } else {
            double ak[CP];
#pragma unroll
            for (int c = 0; c < CP; c++) ak[c] = 0.0;
            const int p0 = a.A64.indptr[row], len = a.A64.indptr[row + 1] - p0;
            const int lb = s_sp[sl - sb] - e0;
            // eight entries at a time: their value loads are in flight together; the sums
            // run entry by entry in CSR order
            for (int k0 = 0; k0 < len; k0 += 8) {
              double kv[8];
              int loc[8];
#pragma unroll
              for (int u = 0; u < 8; u++) {
                const bool in = k0 + u < len;
                kv[u] = in ? __ldg(a.A64.K + p0 + k0 + u) : 0.0;
                loc[u] = in ? s_col[lb + (k0 + u) * 32 + lane] : 0;
              }
#pragma unroll
              for (int u = 0; u < 8; u++) {
                if (k0 + u < len) {
#pragma unroll
                  for (int c = 0; c < CP; c++) ak[c] += kv[u] * s_x[loc[u] * CP + c];
                }
              }
            }
#pragma unroll
            for (int c = 0; c < CP; c++) {
              const double dr = a.A64.diag ? a.A64.diag[row * LD + c0 + c] : 0.0;
              ax[c] = a.dscale[c0 + c] * ak[c] + dr * xo[c];
            }
          }
          float dv[LD];
          ld_win<VT, LD>(s_dinv, lr, dv);
#pragma unroll
          for (int c = 0; c < CP; c++) {
            const int s = c0 + c;
            const double bv = (s < S) ? a.b[row * LD + s] : 0.0;
            const double r64 = (s < S) ? bv - ax[c] : 0.0;
            if (final) {
              acc[s] += r64 * r64;
            } else if (tr[s]) {
              const VT rv = (VT)r64;
              const VT uv = dv[s] * rv;
              acc[s] += (double)rv * (double)uv;
              acc[4 + s] += r64 * r64;
              acc[8 + s] += bv * bv;
              rc[12 + s] = rv;
              a.u[row * LD + s] = uv;
            }
          }
        }
        if (!final) rec_st(j, rc);
      }
      if (!final) tm_wait_st();
    }
  };

  auto release = [&]() {
    tm_fence_before();
    __syncthreads();
    if (warp == 0) tm_dealloc(s_taddr, CGT_COLS);
  };

  // ---- I1: Jacobi diagonal (FP64 values) into shared memory, Dirichlet values into x,
  // records zero
#pragma unroll
  for (int j = 0; j < CGT_MAXS; j++) {
    const int sl = sb + warp + j * CGT_WARPS;
    if (sl >= se) break;
    const int64_t row = (int64_t)sl * 32 + lane;
    if (row < a.n) {
      VT dv[LD];
      if (a.bc && a.bc[row]) {
#pragma unroll
        for (int s = 0; s < LD; s++) {
          dv[s] = VT(0);
          a.x[row * LD + s] = a.b[row * LD + s];
        }
      } else {
        const int lo = a.A64.indptr[row], hi = a.A64.indptr[row + 1];
        int l = lo, h = hi;
        while (l < h) {
          const int mid = (l + h) >> 1;
          if (a.A64.indices[mid] < row)
            l = mid + 1;
          else
            h = mid;
        }
        const bool found = l < hi && a.A64.indices[l] == row;
        const double kd = found ? a.A64.K[l] : 0.0;
#pragma unroll
        for (int s = 0; s < LD; s++) {
          double d = a.dscale[s] * kd;
          if (a.A64.diag) d += a.A64.diag[row * LD + s];
          dv[s] = (s < S && d != 0.0) ? VT(1.0 / d) : VT(0);
        }
      }
      st_win<VT, LD>(s_dinv, (int)(row - r0), dv);
    }
    float z[16];
#pragma unroll
    for (int k = 0; k < 16; k++) z[k] = 0.f;
    rec_st(j, z);
  }
  tm_wait_st();
  bool ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);

  // ---- I2: r = b - A x, u = D^-1 r for every lane; r.u, r.r, b.b
  {
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = 0.0;
    int tr[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) tr[s] = 1;
    if (ok) refresh(tr, acc, false);
    block_partial<8>(acc, a.part, sh);
    block_partial<4>(acc + 8, a.part + 12, sh);
  }
  ok = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok) {
    fill_window(false);
    grid_totals<8, 0>(a.part, s_tot, s_buf);
    grid_totals<4, 12>(a.part, s_tot, s_buf);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < 4; s++) {
      const bool use = s < S && ok;
      const double rz = use ? s_tot[s] : 0.0, rr = use ? s_tot[4 + s] : 0.0;
      const double bb = use ? s_tot[12 + s] : 0.0;
      const double rt = use ? a.rtol[s] : 0.0;
      L.bb[s] = bb;
      L.tol2[s] = rt * rt * bb;
      L.rr[s] = rr;
      L.rtrue[s] = rr;
      L.rmax2[s] = rr;
      L.rz[s] = 0.0;  // no previous gamma: beta = 0 in the first product
      L.alpha[s] = 0.0;
      L.beta[s] = 0.0;
      L.trigger[s] = 0;
      L.frozen[s] = 0;
      L.iters[s] = 0;
      s_gm[s] = rz;
      const bool fin = isfinite(rr) && isfinite(rz);
      const bool act = use && fin && rr > L.tol2[s];
      L.active[s] = act;
      L.status[s] = !use ? TP_OK : (!fin ? TP_ERR_NONFINITE : (act ? -1 : TP_OK));
    }
  }
  __syncthreads();
  clk.lap(7);  // init phases

  int it = 0, n_rel = 0;
  bool decided = true;  // the lane state is set for this pass (the init above)
  while (ok) {
    if (!decided) {
      // ---- lane decisions on gamma = r.u and r.r of the last P phase or FP64 refresh.
      // A lane whose recurrence residual reaches the tolerance freezes (its columns stand
      // still) until the next FP64 sweep confirms it; a sweep runs for every active lane
      // when any lane asks for one (its residual dropped by delta, or a restart) or when
      // every lane still active is frozen.  Every CTA holds the same totals and decides
      // the same.
      int want = 0;
      if (threadIdx.x < S) {
        const int s = threadIdx.x;
        if (L.active[s]) {
          const double gm = s_tot[s], rr = s_tot[4 + s];
          if (L.trigger[s]) {  // refreshed in FP64 just now
            L.trigger[s] = 0;
            L.rtrue[s] = rr;
            if (!isfinite(rr) || !isfinite(gm)) {
              L.active[s] = 0;
              L.status[s] = TP_ERR_NONFINITE;
              L.iters[s] = it;
            } else if (rr <= L.tol2[s]) {
              L.active[s] = 0;
              L.status[s] = TP_OK;
              L.iters[s] = it;
            } else {
              L.rr[s] = rr;
              L.rmax2[s] = rr;
              s_gm[s] = gm;
              if (L.frozen[s] || s_restart[s]) L.rz[s] = 0.0;  // restart: beta = 0
              L.frozen[s] = 0;
              s_restart[s] = 0;
            }
          } else if (!L.frozen[s]) {
            if (!isfinite(gm) || !isfinite(rr)) {
              L.active[s] = 0;
              L.status[s] = TP_ERR_NONFINITE;
              L.iters[s] = it;
            } else {
              L.rr[s] = rr;
              s_gm[s] = gm;
              if (s_restart[s])
                want = 1;
              else if (rr <= L.tol2[s])
                L.frozen[s] = 1;
              else
                want = a.delta2 > 0.0 && rr < a.delta2 * L.rmax2[s];
            }
          }
        }
      }
      int any = __syncthreads_or(want);
      if (!any) {
        int running = 0, pending = 0;
        for (int s = 0; s < S; s++) {
          running |= L.active[s] && !L.frozen[s];
          pending |= L.active[s] && L.frozen[s];
        }
        any = pending && !running;
      }
      clk.lap(4);
      if (any) {
        // ---- RU: x += xi, then the FP64 residual replaces r and u of every active lane
        int tr[LD];
#pragma unroll
        for (int s = 0; s < LD; s++) tr[s] = (s < S) ? L.active[s] : 0;
        __syncthreads();  // every thread has read L.active
        if (threadIdx.x < S) L.trigger[threadIdx.x] = L.active[threadIdx.x];
        cp_async_wait_all();  // the halo copies issued after the last barrier
        add_xi(tr);
        ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
        if (!ok) break;
        {
          double acc[12];
#pragma unroll
          for (int k = 0; k < 12; k++) acc[k] = 0.0;
          refresh(tr, acc, false);
          block_partial<8>(acc, a.part, sh);
        }
        ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
        if (!ok) break;
        fill_window(false);
        grid_totals<8, 0>(a.part, s_tot, s_buf);
        n_rel++;
        clk.lap(5);  // reliable update
        continue;
      }
    }
    decided = false;
    int nact = 0;
#pragma unroll
    for (int s = 0; s < 4; s++) nact += L.active[s];
    if (!nact || it >= a.max_it) break;
    // ---- beta of every running lane (0 for frozen lanes and after a restart)
    __syncthreads();  // every thread has counted the active lanes
    if (threadIdx.x < S) {
      const int s = threadIdx.x;
      const bool run = L.active[s] && !L.frozen[s];
      L.beta[s] = (run && L.rz[s] != 0.0) ? s_gm[s] / L.rz[s] : 0.0;
    }
    __syncthreads();
    clk.lap(4);
    {
      VT be[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) be[s] = (s < S) ? (VT)L.beta[s] : VT(0);
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      product_rows(be, acc);
      block_partial<4>(acc, a.part + 8, sh);
    }
    clk.lap(0);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
    clk.lap(1);
    if (!ok) break;
    grid_totals<4, 8>(a.part, s_tot, s_buf);
    // ---- alpha of every running lane
    if (threadIdx.x < S) {
      const int s = threadIdx.x;
      double step = 0.0;
      if (L.active[s] && !L.frozen[s]) {
        const double dl = s_tot[8 + s], gm = s_gm[s], beta = L.beta[s];
        if (!isfinite(dl)) {
          L.active[s] = 0;
          L.status[s] = TP_ERR_NONFINITE;
          L.iters[s] = it;
        } else if (!(dl > 0.0)) {
          L.active[s] = 0;
          L.status[s] = TP_ERR_BREAKDOWN;
          L.iters[s] = it;
        } else {
          const double den =
              (beta != 0.0 && L.alpha[s] != 0.0) ? dl - beta * gm / L.alpha[s] : dl;
          if (den > 0.0) {
            L.alpha[s] = gm / den;
            L.rz[s] = gm;
            step = L.alpha[s];
          } else {
            s_restart[s] = 1;  // no step; an FP64 refresh restarts the lane
          }
        }
      }
      s_step[s] = step;
    }
    __syncthreads();
    clk.lap(4);
    {
      VT al[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) al[s] = (s < S) ? (VT)s_step[s] : VT(0);
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; k++) acc[k] = 0.0;
      p_rows(al, acc);
      block_partial<8>(acc, a.part, sh);
    }
    it++;
    clk.lap(2);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);  // u published
    clk.lap(3);
    if (!ok) break;
    fill_window(true);
    grid_totals<8, 0>(a.part, s_tot, s_buf);
  }
  cp_async_wait_all();

  // ---- final: x += xi and the FP64 residual norms, unless every lane was confirmed by
  // a sweep (then x and the residual norms are final already; the same decision in every
  // CTA)
  bool all_confirmed = true;
  for (int s = 0; s < S; s++) all_confirmed &= !L.active[s] && L.status[s] == TP_OK;
  if (ok && all_confirmed) {
    if (clk.on) {
      clk.lap(6);
#pragma unroll
      for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, true, s_tot, it, n_rel, false);
    release();
    return;
  }
  if (ok) {
    int all[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) all[s] = s < S;
    add_xi(all);
  }
  bool ok2 = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok2) {
      int none[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) none[s] = 0;
      refresh(none, acc, true);
    }
    block_partial<4>(acc, a.part, sh);
  }
  ok2 = ok2 && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok2) grid_totals<4>(a.part, s_tot, s_buf);
  if (clk.on) {
    clk.lap(6);
#pragma unroll
    for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, ok2, s_tot, it, n_rel);
  release();
}

// ----------------------------------------------------------------- pipelined engine
// k_pcgp: Jacobi-preconditioned pipelined CG (Ghysels-Vanroose) with one grid barrier per
// iteration.  The standard and Chronopoulos-Gear forms need two global synchronisations
// per iteration -- the dot products that give alpha, and the exchange of the new vector the
// product reads -- and on this problem size each costs a barrier plus an L2 round trip for
// the partial sums.  The pipelined form carries the next product's input m = D^-1 w
// through recurrences, so one barrier publishes m and the partial sums together, and the
// reduction's round trip and the lane decisions overlap the halo copies that the product
// n = A m waits for:
//
//   barrier | halo copies of m and the partial-sum loads in flight;
//           | gamma = r.u, delta = w.u, r.r totals; lane decisions; alpha, beta (while
//           | the halo copies land); n = A m (registers)
//           | z = n + beta z, s = w + beta s, p = u + beta p, xi += alpha p,
//           | r -= alpha s, w -= alpha z, u = D^-1 r, m = D^-1 w (window and global);
//           | partials of the next gamma, delta, r.r
//   barrier | ...
//
// With a diagonal preconditioner q = D^-1 s and u = D^-1 r exactly, so the state per row
// and column is r, w, z, s, p (in tensor memory: one 16-column record per slice row next
// to the 16 value columns, CW = 3 (LD 4) or LD columns each) and xi (global memory, read
// ahead of its update).  m is double-buffered in global memory and the partial sums in
// the partial rows (a single barrier per iteration: a CTA may write the next ones while
// another still reads the last).
//
// FP32 recurrences of the pipelined form drift faster than the two-barrier forms, so the
// FP64 refresh (x += xi, r = b - A64 x) restarts every refreshed lane (beta = 0); a lane
// whose recurrence residual grows by 1e4 over its last refresh is refreshed too, and a
// lane whose sums turn non-finite drops its increment since the last refresh and is
// refreshed (a second time in a row it fails with TP_ERR_NONFINITE).  Convergence is
// only ever declared on the FP64 residual.
constexpr int PGP_MAXS = 4;
constexpr int PGP_WARPS = 16;
constexpr uint32_t PGP_COLS = 512;
constexpr int PGP_RUNS_SMEM = 32;  // = PGP_RUNCAP of the host tables

// bulk copy global -> shared (no multicast) completing on an mbarrier; both addresses on
// 16-byte boundaries, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(d), "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(b)
      : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
               : "memory");
}
// bounded wait for the completion of phase `parity`; false when limit_ns ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          unsigned long long limit_ns) {
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  unsigned long long t0 = 0;
  for (uint32_t spins = 1;; spins++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
    if ((spins & 63u) == 0u) {
      const unsigned long long t = gtime();
      if (t0 == 0)
        t0 = t;
      else if (t - t0 > limit_ns)
        return false;
    }
  }
}

struct PgpLanes {
  int poisoned[4];  // the lane's sums were not finite: its xi is dropped at the refresh
  int fails[4];     // refreshes in a row forced by non-finite sums
};

template <int LD>
__global__ void __launch_bounds__(512, 1) k_pcgp(PArgs<float> a) {
  using VT = float;
  static_assert(LD == 2 || LD == 4, "FP64 residual windows hold LD / 2 doubles per entry");
  constexpr int CP = LD / 2;
  constexpr int CW = (LD == 4) ? 3 : LD;  // record columns per vector (S <= CW)
  // record layout: z 0, s CW, p 2 CW, r 3 CW, w 4 CW
  extern __shared__ __align__(16) unsigned char s_dyn[];
  int32_t* s_sp = reinterpret_cast<int32_t*>(s_dyn);
  int32_t* s_halo = s_sp + a.sp_cap;
  uint16_t* s_col = reinterpret_cast<uint16_t*>(s_halo + a.halo_cap);
  VT* s_win = reinterpret_cast<VT*>(
      s_dyn + ((4 * (size_t)(a.sp_cap + a.halo_cap) + 2 * (size_t)a.col_cap + 15) & ~(size_t)15));
  VT* s_dinv = s_win + (size_t)a.win_cap * LD;
  // halo runs and single entries after D^-1
  int4* s_runs = reinterpret_cast<int4*>(
      s_dyn + ((((4 * (size_t)(a.sp_cap + a.halo_cap) + 2 * (size_t)a.col_cap + 15) & ~(size_t)15) +
                ((size_t)a.win_cap + 32 * (size_t)a.sp_cap) * LD * sizeof(VT) + 15) &
               ~(size_t)15));
  uint16_t* s_single = reinterpret_cast<uint16_t*>(s_runs + PGP_RUNS_SMEM);
  __shared__ __align__(8) uint64_t s_mbar;
  __shared__ uint32_t s_halo_bytes;
  __shared__ double sh[32 * 12];
  __shared__ double s_buf[512];
  __shared__ double s_tot[16];
  __shared__ LaneState L;
  __shared__ PgpLanes P;
  __shared__ float s_al[4], s_be[4];
  __shared__ double s_nalpha[4], s_nbeta[4], s_ngm[4];
  __shared__ int s_commit[4];
  __shared__ uint32_t s_taddr;
  __shared__ unsigned long long s_clk[8];
  unsigned int target = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sb = (int)((int64_t)blockIdx.x * a.ns / gridDim.x);
  const int se = (int)((int64_t)(blockIdx.x + 1) * a.ns / gridDim.x);
  const int S = a.S;
  const int r0 = sb * 32;
  const int nown = (se > sb) ? (int)(min((int64_t)se * 32, a.n) - r0) : 0;
  const int nhalo = a.halo_ptr[blockIdx.x + 1] - a.halo_ptr[blockIdx.x];
  // double buffers: m (and u in the refresh) alternate between a.u and a.w, the partial
  // rows between a.part and a.part + 16 gridDim.x
  auto mbuf = [&](int k) { return k ? a.w : a.u; };
  int vp = 0;  // buffer of the last published vector
  int pp = 0;  // partial rows of the last published sums
  auto part_of = [&](int k) { return a.part + (size_t)k * 16 * gridDim.x; };
  PhaseClock clk;
  clk.start(a.prof != nullptr, s_clk);
  for (int i = threadIdx.x; i <= se - sb; i += blockDim.x) s_sp[i] = a.slice_ptr[sb + i];
  {
    const int hb = a.halo_ptr[blockIdx.x];
    for (int i = threadIdx.x; i < nhalo; i += blockDim.x) s_halo[i] = a.halo[hb + i];
    if (se > sb) {
      const int e0 = a.slice_ptr[sb], ne = a.slice_ptr[se] - e0;
      const uint4* src = reinterpret_cast<const uint4*>(a.loc_col + e0);
      uint4* dst = reinterpret_cast<uint4*>(s_col);
      for (int i = threadIdx.x; i < ne / 8; i += blockDim.x) dst[i] = src[i];
    }
  }
  if (threadIdx.x < 4) {
    P.poisoned[threadIdx.x] = 0;
    P.fails[threadIdx.x] = 0;
  }
  constexpr int EB = LD * (int)sizeof(VT);  // bytes of one window entry
  const int run0 = a.run_ptr[blockIdx.x], nrun = a.run_ptr[blockIdx.x + 1] - run0;
  const int sg0 = a.single_ptr[blockIdx.x], nsingle = a.single_ptr[blockIdx.x + 1] - sg0;
  for (int i = threadIdx.x; i < nrun; i += blockDim.x) s_runs[i] = a.runs[run0 + i];
  for (int i = threadIdx.x; i < nsingle; i += blockDim.x) s_single[i] = a.single[sg0 + i];
  if (threadIdx.x == 0) {
    uint32_t hb = 0;
    for (int q = 0; q < nrun; q++) hb += (uint32_t)a.runs[run0 + q].z * EB;
    s_halo_bytes = hb;
    mbar_init(&s_mbar);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  const int own_bulk_rows = (int)(((int64_t)nown * EB & ~(int64_t)15) / EB);
  uint32_t mphase = 0;
  // ---- tensor memory: slice j of warp w: values at tw + 32 j, record at tw + 32 j + 16
  if (warp == 0) tm_alloc(&s_taddr, PGP_COLS);
  tm_fence_before();
  __syncthreads();
  tm_fence_after();
  const uint32_t tw = s_taddr + ((uint32_t)(32 * (warp & 3)) << 16) + 128u * (uint32_t)(warp >> 2);
  auto rec_ld = [&](int j, float rc[16]) { tm_ld16(tw + 32u * (uint32_t)j + 16u, rc); };
  auto rec_st = [&](int j, const float rc[16]) {
    uint32_t v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __float_as_uint(rc[k]);
    tm_st16(tw + 32u * (uint32_t)j + 16u, v);
  };
#pragma unroll
  for (int j = 0; j < PGP_MAXS; j++) {
    const int sl = sb + warp + j * PGP_WARPS;
    uint32_t v[16];
    const int base = (sl < se) ? a.slice_ptr[sl] : 0;
    const int w = (sl < se) ? (a.slice_ptr[sl + 1] - base) >> 5 : 0;
#pragma unroll
    for (int k = 0; k < 16; k++)
      v[k] = (k < w) ? __float_as_uint(ld_na(a.sK + base + k * 32 + lane)) : 0u;
    tm_st16(tw + 32u * (uint32_t)j, v);
  }
  tm_wait_st();

  // window fill: the halo runs (and the own rows unless the update wrote them) as bulk
  // copies issued by thread 0 on the mbarrier, the rest as single asynchronous copies;
  // returns whether bulk copies were issued (the same in every thread)
  auto fill_window = [&](bool own_done, const VT* src) -> bool {
    const bool own_bulk = !own_done && own_bulk_rows > 0;
    const bool bulk = nrun > 0 || own_bulk;
    if (threadIdx.x == 0 && bulk) {
      const uint32_t bytes = s_halo_bytes + (own_bulk ? (uint32_t)own_bulk_rows * EB : 0u);
      asm volatile("fence.proxy.async;" ::: "memory");
      mbar_expect_tx(&s_mbar, bytes);
      if (own_bulk) bulk_g2s(s_win, src + (int64_t)r0 * LD, (uint32_t)own_bulk_rows * EB, &s_mbar);
      for (int q = 0; q < nrun; q++) {
        const int4 r = s_runs[q];
        bulk_g2s(s_win + (size_t)(nown + r.y) * LD, src + (int64_t)r.x * LD, (uint32_t)r.z * EB,
                 &s_mbar);
      }
    }
    if (!own_done)
      for (int i = own_bulk_rows + threadIdx.x; i < nown; i += blockDim.x)
        cp_async<EB>(s_win + (size_t)i * LD, src + (int64_t)(r0 + i) * LD);
    for (int i = threadIdx.x; i < nsingle; i += blockDim.x) {
      const int k = s_single[i];
      cp_async<EB>(s_win + (size_t)(nown + k) * LD, src + (int64_t)s_halo[k] * LD);
    }
    return bulk;
  };
  // every copy of the last fill landed (false in every thread when the bulk copies did
  // not complete within the wait bound: the grid aborts)
  auto wait_window = [&](bool bulk) -> bool {
    cp_async_wait_all();
    bool ok_w = true;
    if (bulk) {
      // a second bounded wait after a first that ran out: the copies in flight land before
      // the CTA gives up
      ok_w = mbar_wait(&s_mbar, mphase, a.wait_limit_ns);
      if (!ok_w) mbar_wait(&s_mbar, mphase, a.wait_limit_ns);
      mphase ^= 1u;
    }
    const int bad = __syncthreads_or(!ok_w);
    if (bad && threadIdx.x == 0) atomicExch(&a.bar->abort, 1u);
    return !bad;
  };

  // partial-sum loads of slots 0..11 (gamma, delta, r.r) of every CTA, issued right after
  // the barrier and summed in the fixed order of grid_totals
  auto totals_load = [&](const double* part, double x[5]) {
    const int k = threadIdx.x % 16, g = threadIdx.x / 16;
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const int b = g + q * 32;
      x[q] = (k < 12 && b < (int)gridDim.x) ? __ldcg(part + (int64_t)b * 16 + k) : 0.0;
    }
  };
  // ---- n = A src (the window) of this warp's rows into nr (registers).  The row
  // diagonals of all four slices (diag_load) are loaded while the copies into the window
  // land; a Dirichlet row (identity, D^-1 = 0 in every column) is recognised by its D^-1.  (A
  // split into the own-column terms, summed while the halo copies land, and the halo
  // terms after them was measured slower: 10.4 against 3.2 us per product.)
  auto diag_load = [&](float dgs[PGP_MAXS][CW]) {
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j++) {
      const int64_t row = (int64_t)(sb + warp + j * PGP_WARPS) * 32 + lane;
      float dg[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) dg[s] = 0.f;
      if (sb + warp + j * PGP_WARPS < se && row < a.n && a.diag) ldv<VT, LD>(a.diag, row, dg);
#pragma unroll
      for (int c = 0; c < CW; c++) dgs[j][c] = dg[c];
    }
  };
  auto product_rows = [&](float nr[PGP_MAXS][CW], const float dgs[PGP_MAXS][CW],
                          bool bulk) -> bool {
    if (!wait_window(bulk)) return false;
    clk.lap(3);
    const int e0 = s_sp[0];
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j++) {
      const int sl = sb + warp + j * PGP_WARPS;
#pragma unroll
      for (int c = 0; c < CW; c++) nr[j][c] = 0.f;
      if (sl >= se) continue;
      const int64_t row = (int64_t)sl * 32 + lane;
      const bool in = row < a.n;
      const bool bcr = in && a.bc && s_dinv[(row - r0) * LD] == 0.f;
      float vals[16];
      tm_ld16(tw + 32u * (uint32_t)j, vals);
      tm_wait_ld();
      const int base = s_sp[sl - sb], w = (s_sp[sl - sb + 1] - base) >> 5;
      const int lb = base - e0;
      float ak[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) ak[s] = 0.f;
#pragma unroll
      for (int k = 0; k < 16; k++) {
        if (k < w) {
          float pv[LD];
          ld_win<VT, LD>(s_win, s_col[lb + k * 32 + lane], pv);
#pragma unroll
          for (int s = 0; s < LD; s++) ak[s] += vals[k] * pv[s];
        }
      }
      if (in) {
        float mr[LD];
        ld_win<VT, LD>(s_win, (int)(row - r0), mr);
#pragma unroll
        for (int c = 0; c < CW; c++) {
          const float v = (float)a.dscale[c] * ak[c] + dgs[j][c] * mr[c];
          nr[j][c] = bcr ? mr[c] : v;
        }
      }
    }
    return true;
  };

  // ---- the update pass (see the header); partials gamma 0-3, delta 4-7, r.r 8-11.  The
  // records of two slices are read per tensor-memory round.
  auto update_rows = [&](const float nr[PGP_MAXS][CW], const float xr[PGP_MAXS][LD],
                         double acc[12], VT* mdst) {
    float al[CW], be[CW];
#pragma unroll
    for (int c = 0; c < CW; c++) {
      al[c] = s_al[c];
      be[c] = s_be[c];
    }
    auto one = [&](int j, float rc[16]) {
      const int64_t row = (int64_t)(sb + warp + j * PGP_WARPS) * 32 + lane;
      if (row >= a.n) return;
      const int lr = (int)(row - r0);
      float dv[LD], mv[LD], xv[LD];
      ld_win<VT, LD>(s_dinv, lr, dv);
#pragma unroll
      for (int s = 0; s < LD; s++) {
        mv[s] = 0.f;
        xv[s] = xr[j][s];
      }
#pragma unroll
      for (int c = 0; c < CW; c++) {
        float& z = rc[c];
        float& sv = rc[CW + c];
        float& p = rc[2 * CW + c];
        float& r = rc[3 * CW + c];
        float& w = rc[4 * CW + c];
        z = nr[j][c] + be[c] * z;
        sv = w + be[c] * sv;
        p = dv[c] * r + be[c] * p;
        xv[c] += al[c] * p;
        r -= al[c] * sv;
        w -= al[c] * z;
        const float u = dv[c] * r;
        mv[c] = dv[c] * w;
        acc[c] += (double)r * (double)u;
        acc[4 + c] += (double)w * (double)u;
        acc[8 + c] += (double)r * (double)r;
      }
      st_win<VT, LD>(s_win, lr, mv);
      stv<VT, LD>(mdst, row, mv);
      stv<VT, LD>(a.xi, row, xv);
    };
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j += 2) {
      const bool h0 = sb + warp + j * PGP_WARPS < se;
      const bool h1 = sb + warp + (j + 1) * PGP_WARPS < se;
      if (!h0) break;
      float rc0[16], rc1[16];
      rec_ld(j, rc0);
      if (h1) rec_ld(j + 1, rc1);
      tm_wait_ld();
      one(j, rc0);
      rec_st(j, rc0);
      if (h1) {
        one(j + 1, rc1);
        rec_st(j + 1, rc1);
      }
    }
    tm_wait_st();
  };

  // ---- x += xi for the lanes in tr (dropped for poisoned lanes), xi = 0 for them
  auto add_xi = [&](const int tr[LD], const int drop[LD]) {
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j++) {
      const int sl = sb + warp + j * PGP_WARPS;
      if (sl >= se) break;
      const int64_t row = (int64_t)sl * 32 + lane;
      if (row < a.n) {
        VT xv[LD];
        ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (tr[s]) {
            if (!drop[s]) a.x[row * LD + s] += (double)xv[s];
            xv[s] = VT(0);
          }
        }
        stv<VT, LD>(a.xi, row, xv);
      }
    }
  };

  // ---- FP64 residual through the window (as k_cgt): final = false: for the lanes in tr
  // r = (float) r64 into the records and u = D^-1 r into udst; partials r.u 0-3, r.r 8-11,
  // b.b 12-15 (r.r in the slot the decisions read); final = true: r.r of every lane in
  // acc[0..3]
  auto refresh = [&](const int tr[LD], double* acc, bool final, VT* udst) {
    const int W = nown + nhalo;
    const int e0 = s_sp[0];
    double* s_x = reinterpret_cast<double*>(s_win);
#pragma unroll
    for (int c0 = 0; c0 < LD; c0 += CP) {
      bool any_c = false;
#pragma unroll
      for (int c = 0; c < CP; c++) any_c |= final ? (c0 + c < S) : (tr[c0 + c] != 0);
      if (!any_c) continue;
      cp_async_wait_all();
      __syncthreads();
      for (int i = threadIdx.x; i < W; i += blockDim.x) {
        const int64_t g = (i < nown) ? (int64_t)(r0 + i) : (int64_t)s_halo[i - nown];
        cp_async<CP * 8>(s_x + (size_t)i * CP, a.x + g * LD + c0);
      }
      cp_async_wait_all();
      __syncthreads();
#pragma unroll
      for (int j = 0; j < PGP_MAXS; j++) {
        const int sl = sb + warp + j * PGP_WARPS;
        if (sl >= se) break;
        float rc[16];
        if (!final) {
          rec_ld(j, rc);
          tm_wait_ld();
        }
        const int64_t row = (int64_t)sl * 32 + lane;
        if (row < a.n) {
          const int lr = (int)(row - r0);
          double xo[CP], ax[CP];
#pragma unroll
          for (int c = 0; c < CP; c++) xo[c] = s_x[lr * CP + c];
          const bool bcr = a.bc && a.bc[row];
          if (bcr) {
#pragma unroll
            for (int c = 0; c < CP; c++) ax[c] = xo[c];
          } else {
            double ak[CP];
#pragma unroll
            for (int c = 0; c < CP; c++) ak[c] = 0.0;
            const int p0 = a.A64.indptr[row], len = a.A64.indptr[row + 1] - p0;
            const int lb = s_sp[sl - sb] - e0;
            for (int k0 = 0; k0 < len; k0 += 8) {
              double kv[8];
              int loc[8];
#pragma unroll
              for (int u = 0; u < 8; u++) {
                const bool in = k0 + u < len;
                kv[u] = in ? __ldg(a.A64.K + p0 + k0 + u) : 0.0;
                loc[u] = in ? s_col[lb + (k0 + u) * 32 + lane] : 0;
              }
#pragma unroll
              for (int u = 0; u < 8; u++) {
                if (k0 + u < len) {
#pragma unroll
                  for (int c = 0; c < CP; c++) ak[c] += kv[u] * s_x[loc[u] * CP + c];
                }
              }
            }
#pragma unroll
            for (int c = 0; c < CP; c++) {
              const double dr = a.A64.diag ? a.A64.diag[row * LD + c0 + c] : 0.0;
              ax[c] = a.dscale[c0 + c] * ak[c] + dr * xo[c];
            }
          }
          float dv[LD];
          ld_win<VT, LD>(s_dinv, lr, dv);
#pragma unroll
          for (int c = 0; c < CP; c++) {
            const int s = c0 + c;
            const double bv = (s < S) ? a.b[row * LD + s] : 0.0;
            const double r64 = (s < S) ? bv - ax[c] : 0.0;
            if (final) {
              acc[s] += r64 * r64;
            } else if (tr[s]) {
              const VT rv = (VT)r64;
              const VT uv = dv[s] * rv;
              acc[s] += (double)rv * (double)uv;
              acc[8 + s] += r64 * r64;
              acc[12 + s] += bv * bv;
              if (s < CW) rc[3 * CW + s] = rv;
              udst[row * LD + s] = uv;
            }
          }
        }
        if (!final) rec_st(j, rc);
      }
      if (!final) tm_wait_st();
    }
  };

  // ---- w = A u after a refresh (u in the window): w into the records of the lanes in tr,
  // m = D^-1 w into the window and mdst, partials gamma, delta, r.r of the new state
  auto restart_rows = [&](const int tr[LD], double acc[12], VT* mdst, bool bulk) -> bool {
    float nr[PGP_MAXS][CW], dgs[PGP_MAXS][CW];
    diag_load(dgs);
    if (!product_rows(nr, dgs, bulk)) return false;
    __syncthreads();  // every warp has read the window: m may replace u in it
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j++) {
      const int sl = sb + warp + j * PGP_WARPS;
      if (sl >= se) break;
      float rc[16];
      rec_ld(j, rc);
      tm_wait_ld();
      const int64_t row = (int64_t)sl * 32 + lane;
      if (row < a.n) {
        const int lr = (int)(row - r0);
        float dv[LD], mv[LD];
        ld_win<VT, LD>(s_dinv, lr, dv);
#pragma unroll
        for (int s = 0; s < LD; s++) mv[s] = 0.f;
#pragma unroll
        for (int c = 0; c < CW; c++) {
          float& r = rc[3 * CW + c];
          float& w = rc[4 * CW + c];
          if (tr[c]) w = nr[j][c];
          const float u = dv[c] * r;
          mv[c] = dv[c] * w;
          acc[c] += (double)r * (double)u;
          acc[4 + c] += (double)w * (double)u;
          acc[8 + c] += (double)r * (double)r;
        }
        st_win<VT, LD>(s_win, lr, mv);
        stv<VT, LD>(mdst, row, mv);
      }
      rec_st(j, rc);
    }
    tm_wait_st();
    return true;
  };

  auto release = [&]() {
    tm_fence_before();
    __syncthreads();
    if (warp == 0) tm_dealloc(s_taddr, PGP_COLS);
  };

  // this CTA's partial row of gamma, delta, r.r: a shuffle tree per warp, then warp k
  // sums slot k over the 16 warps with a second fixed tree.  Every caller comes after a
  // CTA barrier that follows the last reads of sh.
  auto publish12 = [&](double acc[12], double* part) {
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = warp_sum(acc[k]);
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < 12; k++) sh[k * 32 + warp] = acc[k];
    }
    __syncthreads();
    if (warp < 12) {
      const double t = warp_sum(lane < PGP_WARPS ? sh[warp * 32 + lane] : 0.0);
      if (lane == 0) part[(int64_t)blockIdx.x * 16 + warp] = t;
    }
  };

  // ---- I1: Jacobi diagonal into shared memory, Dirichlet values into x, records and xi 0
#pragma unroll
  for (int j = 0; j < PGP_MAXS; j++) {
    const int sl = sb + warp + j * PGP_WARPS;
    if (sl >= se) break;
    const int64_t row = (int64_t)sl * 32 + lane;
    if (row < a.n) {
      VT dv[LD], zero[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) zero[s] = VT(0);
      if (a.bc && a.bc[row]) {
#pragma unroll
        for (int s = 0; s < LD; s++) {
          dv[s] = VT(0);
          a.x[row * LD + s] = a.b[row * LD + s];
        }
      } else {
        const int lo = a.A64.indptr[row], hi = a.A64.indptr[row + 1];
        int l = lo, h = hi;
        while (l < h) {
          const int mid = (l + h) >> 1;
          if (a.A64.indices[mid] < row)
            l = mid + 1;
          else
            h = mid;
        }
        const bool found = l < hi && a.A64.indices[l] == row;
        const double kd = found ? a.A64.K[l] : 0.0;
#pragma unroll
        for (int s = 0; s < LD; s++) {
          double d = a.dscale[s] * kd;
          if (a.A64.diag) d += a.A64.diag[row * LD + s];
          dv[s] = (s < S && d != 0.0) ? VT(1.0 / d) : VT(0);
        }
      }
      st_win<VT, LD>(s_dinv, (int)(row - r0), dv);
      stv<VT, LD>(a.xi, row, zero);
    }
    float z[16];
#pragma unroll
    for (int k = 0; k < 16; k++) z[k] = 0.f;
    rec_st(j, z);
  }
  tm_wait_st();
  bool ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);

  // ---- the lane state from an FP64 refresh of the lanes in tr (all lanes at the start):
  // the residuals were published in partial rows pp and u in buffer vp.  Lanes below the
  // tolerance are done; the others restart (beta = 0) from w = A u.  Returns false when
  // no lane goes on.
  int tr_all[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) tr_all[s] = 1;
  int it = 0, n_rel = 0;
  bool first = true;
  bool wfail = false;  // a window fill did not land within the wait bound
  auto after_refresh = [&](const int tr[LD]) -> bool {
    const bool bulk = fill_window(false, mbuf(vp));
    grid_totals<8, 0>(part_of(pp), s_tot, s_buf);
    grid_totals<8, 8>(part_of(pp), s_tot, s_buf);
    if (threadIdx.x < 4) {
      const int s = threadIdx.x;
      const double gm = s_tot[s], rr = s_tot[8 + s], bb = s_tot[12 + s];
      if (first) {
        const bool use = s < S;
        const double rt = use ? a.rtol[s] : 0.0;
        L.bb[s] = use ? bb : 0.0;
        L.tol2[s] = rt * rt * L.bb[s];
        L.rr[s] = L.rtrue[s] = L.rmax2[s] = use ? rr : 0.0;
        L.rz[s] = L.alpha[s] = L.beta[s] = 0.0;
        L.trigger[s] = L.frozen[s] = L.iters[s] = 0;
        const bool fin = isfinite(rr) && isfinite(gm) && isfinite(bb);
        const bool act = use && fin && rr > L.tol2[s];
        L.active[s] = act;
        L.status[s] = !use ? TP_OK : (!fin ? TP_ERR_NONFINITE : (act ? -1 : TP_OK));
      } else if (s < S && tr[s] && L.active[s]) {
        L.rtrue[s] = rr;
        L.frozen[s] = 0;
        L.rz[s] = 0.0;  // restart: beta = 0
        if (!isfinite(rr) || !isfinite(gm)) {
          L.active[s] = 0;
          L.status[s] = TP_ERR_NONFINITE;
          L.iters[s] = it;
        } else if (rr <= L.tol2[s]) {
          L.active[s] = 0;
          L.status[s] = TP_OK;
          L.iters[s] = it;
        } else {
          L.rr[s] = rr;
          L.rmax2[s] = rr;
          if (!P.poisoned[s]) P.fails[s] = 0;
        }
        P.poisoned[s] = 0;
      }
    }
    first = false;
    __syncthreads();
    int nact = 0;
    for (int s = 0; s < S; s++) nact += L.active[s];
    if (!nact) return false;
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = 0.0;
    if (!restart_rows(tr, acc, mbuf(vp ^ 1), bulk)) {
      wfail = true;
      return false;
    }
    vp ^= 1;
    pp ^= 1;
    publish12(acc, part_of(pp));
    return true;
  };

  // ---- I2: r = b - A x, u = D^-1 r for every lane, then w = A u
  if (ok) {
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    refresh(tr_all, acc, false, mbuf(vp));
    block_partial<8>(acc, part_of(pp), sh);
    block_partial<8>(acc + 8, part_of(pp) + 8, sh);
  }
  ok = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  bool going = ok && after_refresh(tr_all);
  ok = ok && !wfail && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  clk.lap(7);

  while (ok && going) {
    // ---- after the barrier: m of the halo and the partial sums in flight.  The totals
    // and lane decisions need only the partial sums, so they run while the halo copies
    // land; the product waits for the window after them.
    const bool bulk = fill_window(true, mbuf(vp));
    double tx[5];
    totals_load(part_of(pp), tx);
    float dgs[PGP_MAXS][CW];
    diag_load(dgs);
    // ---- totals and lane decisions with two CTA barriers: warp s sums lane s's partial
    // sums (gamma, delta, r.r; the fixed order of grid_totals) and its lane 0 decides for
    // the lane and forms alpha and beta tentatively; the lane state of alpha, beta and
    // gamma_old is committed only when no lane asks for a refresh.  Every CTA holds the
    // same totals and decides the same.
    {
      const int k = threadIdx.x % 16, g = threadIdx.x / 16;
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < 5; q++)
        if (g + q * 32 < (int)gridDim.x) v += tx[q];
      for (int bb = g + 5 * 32; bb < (int)gridDim.x; bb += 32)
        if (k < 12) v += __ldcg(part_of(pp) + (int64_t)bb * 16 + k);
      s_buf[threadIdx.x] = v;
    }
    __syncthreads();
    int want = 0;
    if (warp < 4) {
      const int s = warp;
      double gm = 0.0, dl = 0.0, rr = 0.0;
      if (s < S) {
        gm = warp_sum(s_buf[lane * 16 + s]);
        dl = warp_sum(s_buf[lane * 16 + 4 + s]);
        rr = warp_sum(s_buf[lane * 16 + 8 + s]);
      }
      if (lane == 0) {
        float al = 0.f, be = 0.f;
        s_commit[s] = 0;
        if (s < S && L.active[s] && !L.frozen[s]) {
          if (!isfinite(gm) || !isfinite(dl) || !isfinite(rr)) {
            if (++P.fails[s] >= 2) {
              L.active[s] = 0;
              L.status[s] = TP_ERR_NONFINITE;
              L.iters[s] = it;
            } else {
              P.poisoned[s] = 1;
              want = 1;
            }
          } else if (!(dl > 0.0)) {
            // w.u = u.Au is exact right after a restart: not positive there means the
            // operator is not positive definite; later it is recurrence drift
            if (L.rz[s] == 0.0) {
              L.active[s] = 0;
              L.status[s] = TP_ERR_BREAKDOWN;
              L.iters[s] = it;
            } else {
              want = 1;
            }
          } else {
            L.rr[s] = rr;
            if (rr <= L.tol2[s])
              L.frozen[s] = 1;
            else if (rr > 1e4 * L.rmax2[s])
              want = 1;  // the recurrences drifted off: refresh and restart
            else
              want = a.delta2 > 0.0 && rr < a.delta2 * L.rmax2[s];
            if (!L.frozen[s] && !want) {
              double beta = (L.rz[s] != 0.0) ? gm / L.rz[s] : 0.0;
              double den = (beta != 0.0 && L.alpha[s] != 0.0) ? dl - beta * gm / L.alpha[s] : dl;
              if (!(den > 0.0)) {  // rounding: restart the direction
                beta = 0.0;
                den = dl;
              }
              s_nbeta[s] = beta;
              s_nalpha[s] = gm / den;
              s_ngm[s] = gm;
              s_commit[s] = 1;
              al = (float)s_nalpha[s];
              be = (float)beta;
            }
          }
        }
        s_al[s] = al;
        s_be[s] = be;
      }
    }
    int any = __syncthreads_or(want);
    if (!any) {
      int running = 0, pending = 0;
      for (int s = 0; s < S; s++) {
        running |= L.active[s] && !L.frozen[s];
        pending |= L.active[s] && L.frozen[s];
      }
      any = pending && !running;
    }
    if (!any && it >= a.max_it) {
      // the window's copies land before the final refresh reuses the window
      if (!wait_window(bulk)) ok = false;
      break;
    }
    if (any) {
      // ---- RU: x += xi, FP64 residual, restart from w = A u (after the window's copies
      // landed: the refresh reuses the window)
      clk.lap(4);
      if (!wait_window(bulk)) {
        ok = false;
        break;
      }
      int tr[LD], drop[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) {
        tr[s] = (s < S) ? L.active[s] : 0;
        drop[s] = (s < S) ? P.poisoned[s] : 0;
      }
      __syncthreads();
      add_xi(tr, drop);
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      {
        double acc[16];
#pragma unroll
        for (int k = 0; k < 16; k++) acc[k] = 0.0;
        refresh(tr, acc, false, mbuf(vp ^ 1));
        pp ^= 1;
        block_partial<8>(acc, part_of(pp), sh);
        block_partial<8>(acc + 8, part_of(pp) + 8, sh);
      }
      vp ^= 1;
      ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      if (!ok) break;
      n_rel++;
      going = after_refresh(tr);
      ok = !wfail && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
      clk.lap(5);
      continue;
    }
    // ---- commit alpha, beta, gamma_old of the lanes that step (read again only after
    // the barriers of the update)
    if (threadIdx.x < S && s_commit[threadIdx.x]) {
      const int s = threadIdx.x;
      L.beta[s] = s_nbeta[s];
      L.alpha[s] = s_nalpha[s];
      L.rz[s] = s_ngm[s];
    }
    clk.lap(4);
    float nr[PGP_MAXS][CW];
    if (!product_rows(nr, dgs, bulk)) {
      ok = false;
      break;
    }
    clk.lap(0);
    // xi of the own rows, read ahead of the update
    float xr[PGP_MAXS][LD];
#pragma unroll
    for (int j = 0; j < PGP_MAXS; j++) {
      const int64_t row = (int64_t)(sb + warp + j * PGP_WARPS) * 32 + lane;
#pragma unroll
      for (int s = 0; s < LD; s++) xr[j][s] = 0.f;
      if (sb + warp + j * PGP_WARPS < se && row < a.n) ldv_cg<VT, LD>(a.xi, row, xr[j]);
    }
    __syncthreads();  // every warp has read the window: the update may replace m in it
    {
      double acc[12];
#pragma unroll
      for (int k = 0; k < 12; k++) acc[k] = 0.0;
      update_rows(nr, xr, acc, mbuf(vp ^ 1));
      vp ^= 1;
      pp ^= 1;
      publish12(acc, part_of(pp));
    }
    it++;
    clk.lap(2);
    ok = grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
    clk.lap(1);
  }
  cp_async_wait_all();

  bool all_confirmed = true;
  for (int s = 0; s < S; s++) all_confirmed &= !L.active[s] && L.status[s] == TP_OK;
  if (ok && all_confirmed) {
    if (clk.on) {
      clk.lap(6);
#pragma unroll
      for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, true, s_tot, it, n_rel, false);
    release();
    return;
  }
  if (ok) {
    int all[LD], none[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) {
      all[s] = s < S;
      none[s] = 0;
    }
    add_xi(all, none);
  }
  bool ok2 = ok && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  pp ^= 1;
  {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (ok2) {
      int none[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) none[s] = 0;
      refresh(none, acc, true, nullptr);
    }
    block_partial<4>(acc, part_of(pp), sh);
  }
  ok2 = ok2 && grid_sync(a.bar, target, a.wait_limit_ns, a.wait_missing);
  if (ok2) grid_totals<4>(part_of(pp), s_tot, s_buf);
  if (clk.on) {
    clk.lap(6);
#pragma unroll
    for (int k = 0; k < 8; k++) a.prof[blockIdx.x * 8 + k] = clk.acc[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) write_result(a, L, ok2, s_tot, it, n_rel);
  release();
}

// ----------------------------------------------------------------- SELL-32 build
__global__ void k_slice_width(int64_t n, const int32_t* __restrict__ indptr, int ns,
                              int32_t* __restrict__ width) {
  const int sl = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (sl >= ns) return;
  const int64_t row = (int64_t)sl * 32 + lane;
  int len = (row < n) ? indptr[row + 1] - indptr[row] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
  if (lane == 0) width[sl] = len;
}

__global__ void k_sell_fill_pattern(int64_t n, const int32_t* __restrict__ indptr,
                                    const int32_t* __restrict__ indices, int ns,
                                    const int32_t* __restrict__ slice_ptr,
                                    int32_t* __restrict__ sell_col,
                                    int32_t* __restrict__ csr2sell) {
  const int sl = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (sl >= ns) return;
  const int64_t row = (int64_t)sl * 32 + lane;
  const int base = slice_ptr[sl], w = (slice_ptr[sl + 1] - base) >> 5;
  const int beg = row < n ? indptr[row] : 0, len = row < n ? indptr[row + 1] - beg : 0;
  const int own = (int)(row < n ? row : n - 1);
  for (int k = 0; k < w; k++) {
    const int pos = base + k * 32 + lane;
    if (k < len) {
      sell_col[pos] = indices[beg + k];
      csr2sell[beg + k] = pos;
    } else {
      sell_col[pos] = own;  // padding: own column, value 0
    }
  }
}

template <typename T>
__global__ void k_sell_scatter(int64_t nnz, const int32_t* __restrict__ csr2sell,
                               const double* __restrict__ v, T* __restrict__ out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz;
       p += (int64_t)gridDim.x * blockDim.x)
    out[csr2sell[p]] = (T)v[p];
}

}  // namespace tp

using namespace tp;

extern "C" int tp_sell_build(int64_t n_rows, const int32_t* indptr, const int32_t* indices,
                             int32_t* slice_ptr, int32_t* sell_col, int32_t* csr2sell,
                             int64_t* n_entries, void* stream) {
  TP_REQUIRE(indptr && slice_ptr && n_entries, "null pointer");
  cudaStream_t st = as_stream(stream);
  const int ns = (int)((n_rows + 31) / 32);
  std::vector<int32_t> w(ns), sp(ns + 1, 0);
  if (ns > 0) {
    int32_t* dw = slice_ptr;  // scratch: slice_ptr has ns + 1 entries
    k_slice_width<<<(ns + 7) / 8, 256, 0, st>>>(n_rows, indptr, ns, dw);
    TP_LAUNCH_CHECK();
    TP_CUDA_TRY(cudaMemcpyAsync(w.data(), dw, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, st));
    TP_CUDA_TRY(cudaStreamSynchronize(st));
  }
  int64_t tot = 0;
  for (int s = 0; s < ns; s++) {
    sp[s] = (int32_t)tot;
    tot += 32 * (int64_t)w[s];
    if (tot > INT32_MAX) {
      set_error("SELL storage exceeds int32 offsets");
      return TP_ERR_CAPACITY;
    }
  }
  sp[ns] = (int32_t)tot;
  *n_entries = tot;
  TP_CUDA_TRY(cudaMemcpyAsync(slice_ptr, sp.data(), sizeof(int32_t) * (ns + 1),
                              cudaMemcpyHostToDevice, st));
  if (sell_col && csr2sell && ns > 0) {
    k_sell_fill_pattern<<<(ns + 7) / 8, 256, 0, st>>>(n_rows, indptr, indices, ns, slice_ptr,
                                                      sell_col, csr2sell);
    TP_LAUNCH_CHECK();
  }
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  return TP_OK;
}

extern "C" int tp_sell_scatter(int64_t nnz, const int32_t* csr2sell, const double* csr_vals,
                               float* sell32, double* sell64, void* stream) {
  TP_REQUIRE(csr2sell && csr_vals && (sell32 || sell64), "null pointer");
  if (nnz == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  const int grid = grid_for(nnz, 256, sm_count() * 16);
  if (sell32) k_sell_scatter<float><<<grid, 256, 0, st>>>(nnz, csr2sell, csr_vals, sell32);
  if (sell64) k_sell_scatter<double><<<grid, 256, 0, st>>>(nnz, csr2sell, csr_vals, sell64);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

// ----------------------------------------------------------------- persistent handle
struct tp_pcg_handle {
  int fp32, ld, grid, block, window;
  size_t dyn_smem;  // slice offsets (+ window engine tables and window) per CTA
  void* fn;
  tp::PArgs<float> af;
  tp::PArgs<double> ad;
  tp::POut* out;
  tp::PBar* bar;
  // window engine tables (owned by the handle)
  int32_t* d_halo_ptr = nullptr;
  int32_t* d_halo = nullptr;
  uint16_t* d_loc_col = nullptr;
  // pipelined engine: bulk-copy runs and single entries of the halo
  void* d_runs = nullptr;
  ~tp_pcg_handle() {
    if (d_halo_ptr) cudaFree(d_halo_ptr);
    if (d_halo) cudaFree(d_halo);
    if (d_loc_col) cudaFree(d_loc_col);
    if (d_runs) cudaFree(d_runs);
  }
};

namespace tp {
// SELL entries per pipelined group: the current and next group's stream entries and the
// current group's gathered records stay in registers (about 48 per thread: 2 to 8
// entries).  Two CTAs per SM (64 registers) only for records of at most 16 bytes.  The
// window engine (k_cgw) runs one CTA per SM.
template <typename VT, int LD>
static void* pick_kernel(int minb, bool hasM, bool win) {
  constexpr int RB = 2 * LD * (int)sizeof(VT);
  constexpr int cost = 2 * (1 + (int)sizeof(VT) / 4) + RB / 4;  // registers per entry
  constexpr int U = std::max(2, std::min(8, 48 / cost));
  if (win) return hasM ? (void*)k_cgw<VT, LD, U, true> : (void*)k_cgw<VT, LD, U, false>;
  if constexpr (RB <= 16) {
    if (minb >= 2) return hasM ? (void*)k_pcg<VT, LD, U, 2, true> : (void*)k_pcg<VT, LD, U, 2, false>;
  }
  return hasM ? (void*)k_pcg<VT, LD, U, 1, true> : (void*)k_pcg<VT, LD, U, 1, false>;
}

// CTAs per SM: 1 (up to 128 registers per thread) or 2 (64 registers)
static void* pcg_kernel(int fp32, int ld, int minb, bool hasM, bool win = false) {
  if (fp32) {
    if (ld == 1) return pick_kernel<float, 1>(minb, hasM, win);
    if (ld == 2) return pick_kernel<float, 2>(minb, hasM, win);
    if (ld == 4) return pick_kernel<float, 4>(minb, hasM, win);
  } else {
    if (ld == 1) return pick_kernel<double, 1>(minb, hasM, win);
    if (ld == 2) return pick_kernel<double, 2>(minb, hasM, win);
    if (ld == 4) return pick_kernel<double, 4>(minb, hasM, win);
  }
  return nullptr;
}

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
static size_t a16(size_t x) { return (x + 15) & ~(size_t)15; }

template <typename VT>
static void fill_pargs(PArgs<VT>& a, const tp_csr_op* op, const tp_sell* sl, const double* b,
                       double* x, const double* rtol, int max_it, double delta, char* ws,
                       size_t vec_bytes, int grid) {
  a.n = op->n_rows;
  a.S = op->S;
  a.ns = (int)((op->n_rows + 31) / 32);
  a.max_it = max_it;
  a.delta2 = delta * delta;
  a.slice_ptr = sl->slice_ptr;
  a.sell_col = sl->sell_col;
  if constexpr (sizeof(VT) == 4) {
    a.sK = sl->sK32;
    a.sM = sl->sM32;
    a.diag = op->diag32;
  } else {
    a.sK = sl->sK64;
    a.sM = sl->sM64;
    a.diag = op->diag64;
  }
  a.A64.indptr = op->indptr;
  a.A64.indices = op->indices;
  a.A64.K = op->K64;
  a.A64.M = op->M64;
  a.A64.diag = op->diag64;
  a.A64.bc = op->bc_mask;
  for (int s = 0; s < 4; s++) {
    a.dscale[s] = a.A64.dscale[s] = s < op->S ? op->dscale[s] : 0.0;
    a.cscale[s] = a.A64.cscale[s] = s < op->S ? op->cscale[s] : 0.0;
  }
  a.bc = op->bc_mask;
  a.b = b;
  a.x = x;
  a.rtol = rtol;
  char* p = ws;
  VT** v[4] = {&a.q, &a.r, &a.xi, &a.dinv};
  for (int i = 0; i < 4; i++) {
    *v[i] = reinterpret_cast<VT*>(p);
    p += vec_bytes;
  }
  a.rec0 = reinterpret_cast<VT*>(p);
  p += 2 * vec_bytes;
  a.rec1 = reinterpret_cast<VT*>(p);
  p += 2 * vec_bytes;
  // the window engine's vectors share the record buffers
  a.p = a.rec0;
  a.s = a.rec0 + vec_bytes / sizeof(VT);
  a.u = a.rec1;
  a.w = a.rec1 + vec_bytes / sizeof(VT);
  a.halo_ptr = nullptr;
  a.halo = nullptr;
  a.loc_col = nullptr;
  a.sp_cap = a.halo_cap = a.col_cap = a.win_cap = 0;
  a.reg_values = 0;
  a.tmem_values = 0;
  a.runs = nullptr;
  a.run_ptr = nullptr;
  a.single = nullptr;
  a.single_ptr = nullptr;
  a.single_cap = 0;
  a.wait_limit_ns = WAIT_LIMIT_NS;
  a.wait_missing = 0;
  // two rows of 16 partial sums per CTA: the pipelined engine alternates between them
  a.part = reinterpret_cast<double*>(p);
  p += a256(sizeof(double) * 2 * 16 * grid);
  a.bar = reinterpret_cast<PBar*>(p);
  p += a256(sizeof(PBar));
  a.out = reinterpret_cast<POut*>(p);
}
static int round4(int64_t x) { return (int)((x + 3) & ~(int64_t)3); }

// Window tables for a grid of `grid` CTAs over contiguous slice ranges: for CTA c (rows
// [r0, r1)) the sorted columns outside [r0, r1) that its rows reference (its halo) and
// every SELL entry's column as a window index (own rows 0 .. r1-r0-1, then the halo in
// order).  ok = false (no error) when a window would exceed 65535 entries.
struct WinTables {
  std::vector<int32_t> halo_ptr, halo;
  std::vector<uint16_t> loc_col;
  int sp_cap = 0, halo_cap = 0, col_cap = 0, win_cap = 0, max_width = 0;
  // bulk-copy runs of the halo and the entries left to single copies (build_runs)
  std::vector<int4> runs;
  std::vector<int32_t> run_ptr, single_ptr;
  std::vector<uint16_t> single;
  int single_cap = 0;
};

constexpr int PGP_RUNCAP = 32;  // bulk runs per CTA (shared-memory list)
constexpr double PGP_MIN_DELTA = 1e-3;  // the pipelined engine's largest refresh interval
constexpr int PGP_MINRUN = 8;   // shortest run copied in bulk (entries)

// The halo of every CTA (sorted global rows, window slots nown + k) split into runs of
// consecutive rows.  A run of at least PGP_MINRUN entries whose source and destination
// start on 16-byte boundaries and whose length is a multiple of 16 bytes is one bulk copy
// (entry bytes eb = 16: always; eb = 8: the even-aligned middle of the run), at most
// PGP_RUNCAP per CTA; every other entry is a single copy.
static void build_runs(WinTables& w, int grid, int64_t n, int ns, int eb) {
  w.runs.clear();
  w.single.clear();
  w.run_ptr.assign(grid + 1, 0);
  w.single_ptr.assign(grid + 1, 0);
  int max_single = 0;
  for (int c = 0; c < grid; c++) {
    const int sb = (int)((int64_t)c * ns / grid), se = (int)((int64_t)(c + 1) * ns / grid);
    const int64_t r0 = (int64_t)sb * 32, r1 = std::min<int64_t>((int64_t)se * 32, n);
    const int64_t nown = se > sb ? r1 - r0 : 0;
    const int h0 = w.halo_ptr[c], h1 = w.halo_ptr[c + 1];
    int nr = 0;
    const size_t s0 = w.single.size();
    for (int k = h0; k < h1;) {
      int e = k + 1;
      while (e < h1 && w.halo[e] == w.halo[e - 1] + 1) e++;
      // run of halo positions [k, e): rows halo[k] .., window slots nown + (k - h0) ..
      int a = k, b = e;
      if (eb == 8) {
        const int64_t g = w.halo[k], slot = nown + (k - h0);
        if (((g ^ slot) & 1) != 0) {
          a = b = k;  // source and destination parities differ: no bulk part
        } else {
          if (g & 1) a++;
          if ((b - a) & 1) b--;
        }
      }
      if (b - a >= PGP_MINRUN && nr < PGP_RUNCAP) {
        w.runs.push_back(make_int4(w.halo[a], (int)(a - h0), b - a, 0));
        nr++;
      } else {
        a = b = k;
      }
      for (int q = k; q < e; q++)
        if (q < a || q >= b) w.single.push_back((uint16_t)(q - h0));
      k = e;
    }
    w.run_ptr[c + 1] = (int32_t)w.runs.size();
    w.single_ptr[c + 1] = (int32_t)w.single.size();
    max_single = std::max(max_single, (int)(w.single.size() - s0));
  }
  w.single_cap = (max_single + 7) & ~7;
}

static int build_window(const tp_sell* sell, int grid, cudaStream_t st, WinTables& w, bool* ok) {
  *ok = false;
  const int64_t n = sell->n_rows;
  const int ns = (int)((n + 31) / 32);
  std::vector<int32_t> sp(ns + 1);
  std::vector<int32_t> col(sell->n_entries);
  TP_CUDA_TRY(cudaMemcpyAsync(sp.data(), sell->slice_ptr, sizeof(int32_t) * (ns + 1),
                              cudaMemcpyDeviceToHost, st));
  if (sell->n_entries > 0)
    TP_CUDA_TRY(cudaMemcpyAsync(col.data(), sell->sell_col, sizeof(int32_t) * sell->n_entries,
                                cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<int32_t> mark(n, -1), pos(n, 0);
  w.halo_ptr.assign(grid + 1, 0);
  w.halo.clear();
  w.loc_col.assign(sell->n_entries, 0);
  int max_sl = 0, max_h = 0, max_e = 0, max_w = 0;
  for (int s = 0; s < ns; s++) w.max_width = std::max(w.max_width, (sp[s + 1] - sp[s]) / 32);
  for (int c = 0; c < grid; c++) {
    const int sb = (int)((int64_t)c * ns / grid), se = (int)((int64_t)(c + 1) * ns / grid);
    const int64_t r0 = (int64_t)sb * 32, r1 = std::min<int64_t>((int64_t)se * 32, n);
    const int e0 = sp[sb], e1 = sp[se];
    const size_t h0 = w.halo.size();
    for (int e = e0; e < e1; e++) {
      const int j = col[e];
      if ((j < r0 || j >= r1) && mark[j] != c) {
        mark[j] = c;
        w.halo.push_back(j);
      }
    }
    std::sort(w.halo.begin() + h0, w.halo.end());
    const int64_t nown = se > sb ? r1 - r0 : 0;
    const int64_t nh = (int64_t)(w.halo.size() - h0);
    if (nown + nh > 65535) return TP_OK;  // *ok stays false
    for (int64_t k = 0; k < nh; k++) pos[w.halo[h0 + k]] = (int32_t)(nown + k);
    for (int e = e0; e < e1; e++) {
      const int j = col[e];
      w.loc_col[e] = (uint16_t)((j >= r0 && j < r1) ? j - r0 : pos[j]);
    }
    w.halo_ptr[c + 1] = (int32_t)w.halo.size();
    max_sl = std::max(max_sl, se - sb + 1);
    max_h = std::max(max_h, (int)nh);
    max_e = std::max(max_e, e1 - e0);
    max_w = std::max(max_w, (int)(nown + nh));
  }
  w.sp_cap = round4(max_sl);
  w.halo_cap = round4(max_h);
  w.col_cap = max_e;  // a multiple of 32
  w.win_cap = max_w;
  *ok = true;
  return TP_OK;
}
}  // namespace tp

static int default_minb(int) { return 1; }

// Kernel attributes are per function and shared by every handle, so they only ever grow:
// the dynamic shared-memory limit to the largest request so far, the shared-memory
// carveout to what `ctas` CTAs of that size need (the rest of the unified storage stays
// L1).  Set before occupancy queries so cooperative grids match the launches.
static cudaError_t raise_smem_limits(void* fn, size_t dyn, int ctas) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  if ((int)dyn > fa.maxDynamicSharedSizeBytes) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
  }
  const size_t per_sm = (fa.sharedSizeBytes + dyn + 1024) * ctas;
  const int pct = (int)std::min<size_t>(100, (per_sm * 100 + 228 * 1024 - 1) / (228 * 1024));
  if (pct > fa.preferredShmemCarveout)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  return e;
}

// Grid of `minb` CTAs per SM (fewer if they do not fit) and the dynamic shared memory
// (slice offsets of one CTA's range) for n_rows rows.
static int pcg_grid(int fp32, int ld, int minb, bool hasM, int block, int64_t n_rows, int* grid,
                    size_t* dyn) {
  const int64_t ns = (n_rows + 31) / 32;
  for (int m = minb; m >= 1; m--) {
    void* fn = pcg_kernel(fp32, ld, m, hasM);
    if (!fn) return TP_ERR_ARG;
    const int g = sm_count() * m;
    const size_t d = sizeof(int32_t) * (size_t)((ns + g - 1) / g + 2);
    if (d > 160 * 1024) {
      set_error("persistent CG: %lld rows exceed the slice table of one CTA", (long long)n_rows);
      return TP_ERR_CAPACITY;
    }
    TP_CUDA_TRY(raise_smem_limits(fn, d, m));
    int occ = 0;
    TP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, d));
    if (occ >= m) {
      *grid = g;
      *dyn = d;
      return TP_OK;
    }
  }
  set_error("persistent CG kernel does not fit on an SM");
  return TP_ERR_CAPACITY;
}

extern "C" size_t tp_pcg_workspace_bytes(const tp_csr_op* op, int inner_fp32) {
  if (!op) return 0;
  // partial rows for the largest grid (2 CTAs per SM)
  const int grid = 2 * sm_count();
  const size_t vt = inner_fp32 ? 4 : 8;
  return 8 * a256(vt * op->ld * (size_t)op->n_rows) + a256(sizeof(double) * 2 * 16 * grid) +
         a256(sizeof(PBar)) + a256(sizeof(POut));
}

static int getenv_flag(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

// Window engine for a one-CTA-per-SM grid when its tables and window fit in shared
// memory; leaves h on the streaming engine otherwise.  DISSOLVE_PCG_ENGINE=stream at
// create keeps the streaming engine.
static int try_window(tp_pcg_handle* h, const tp_sell* sell, bool hasM, cudaStream_t st) {
  const char* env = getenv("DISSOLVE_PCG_ENGINE");
  if (env && strcmp(env, "stream") == 0) return TP_OK;
  if (h->grid != sm_count()) return TP_OK;
  WinTables w;
  bool ok = false;
  int rc = build_window(sell, h->grid, st, w, &ok);
  if (rc != TP_OK || !ok) return rc;
  const size_t vt = h->fp32 ? 4 : 8;
  const size_t head = (4 * (size_t)(w.sp_cap + w.halo_cap) + 2 * (size_t)w.col_cap + 15) & ~(size_t)15;
  // window (own rows + halo), then w of the own rows (at most 32 per slice)
  const size_t d = head + ((size_t)w.win_cap + 32 * (size_t)w.sp_cap) * h->ld * vt;
  // tensor-memory engine (k_cgt): FP32 without a mass matrix, 16 warps with at most 4
  // slices each, slices of at most 16 entries, 2 or 4 columns; DISSOLVE_PCG_CGT=0 keeps
  // k_cgw
  const int ns = (int)((sell->n_rows + 31) / 32);
  const int max_sl = (ns + h->grid - 1) / h->grid;
  const bool tm_fit = h->fp32 && !hasM && h->block == 512 && w.max_width <= 16 && max_sl <= 64;
  const bool cgt = tm_fit && (h->ld == 2 || h->ld == 4) && h->af.A64.M == nullptr &&
                   getenv_flag("DISSOLVE_PCG_CGT", 1) != 0;
  // pipelined form (k_pcgp): the same conditions, at most 3 columns (5 record vectors of
  // 3 columns next to the 16 value columns); DISSOLVE_PCG_PIPE=0 keeps k_cgt
  const int S = h->af.S;
  const bool pipe = cgt && S <= (h->ld == 4 ? 3 : h->ld) && getenv_flag("DISSOLVE_PCG_PIPE", 1) != 0;
  void* fn = pipe  ? (h->ld == 4 ? (void*)k_pcgp<4> : (void*)k_pcgp<2>)
             : cgt ? (h->ld == 4 ? (void*)k_cgt<4> : (void*)k_cgt<2>)
                   : pcg_kernel(h->fp32, h->ld, 1, hasM, true);
  // the pipelined engine's halo runs and single entries, after D^-1 in shared memory
  size_t d_pipe = d;
  if (pipe) {
    build_runs(w, h->grid, sell->n_rows, ns, h->ld * 4);
    d_pipe = a16(d) + 16 * (size_t)PGP_RUNCAP + 2 * (size_t)w.single_cap;
  }
  cudaFuncAttributes fa;
  TP_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
  int optin = 0, dev = 0;
  TP_CUDA_TRY(cudaGetDevice(&dev));
  TP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (fa.sharedSizeBytes + d_pipe + 1024 > (size_t)optin) return TP_OK;  // does not fit
  TP_CUDA_TRY(raise_smem_limits(fn, d_pipe, 1));
  int occ = 0;
  TP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, h->block, d_pipe));
  if (occ < 1) return TP_OK;
  TP_CUDA_TRY(cudaMalloc(&h->d_halo_ptr, sizeof(int32_t) * w.halo_ptr.size()));
  TP_CUDA_TRY(cudaMalloc(&h->d_halo, sizeof(int32_t) * std::max<size_t>(w.halo.size(), 1)));
  TP_CUDA_TRY(cudaMalloc(&h->d_loc_col, sizeof(uint16_t) * std::max<size_t>(w.loc_col.size(), 8)));
  TP_CUDA_TRY(cudaMemcpyAsync(h->d_halo_ptr, w.halo_ptr.data(),
                              sizeof(int32_t) * w.halo_ptr.size(), cudaMemcpyHostToDevice, st));
  if (!w.halo.empty())
    TP_CUDA_TRY(cudaMemcpyAsync(h->d_halo, w.halo.data(), sizeof(int32_t) * w.halo.size(),
                                cudaMemcpyHostToDevice, st));
  if (!w.loc_col.empty())
    TP_CUDA_TRY(cudaMemcpyAsync(h->d_loc_col, w.loc_col.data(),
                                sizeof(uint16_t) * w.loc_col.size(), cudaMemcpyHostToDevice, st));
  if (pipe) {
    // one allocation: runs (int4), run_ptr, single_ptr (int32), single (uint16)
    const size_t b_runs = a256(sizeof(int4) * std::max<size_t>(w.runs.size(), 1));
    const size_t b_ptr = a256(sizeof(int32_t) * w.run_ptr.size());
    const size_t b_single = a256(sizeof(uint16_t) * std::max<size_t>(w.single.size(), 8));
    TP_CUDA_TRY(cudaMalloc(&h->d_runs, b_runs + 2 * b_ptr + b_single));
    char* base = static_cast<char*>(h->d_runs);
    if (!w.runs.empty())
      TP_CUDA_TRY(cudaMemcpyAsync(base, w.runs.data(), sizeof(int4) * w.runs.size(),
                                  cudaMemcpyHostToDevice, st));
    TP_CUDA_TRY(cudaMemcpyAsync(base + b_runs, w.run_ptr.data(),
                                sizeof(int32_t) * w.run_ptr.size(), cudaMemcpyHostToDevice, st));
    TP_CUDA_TRY(cudaMemcpyAsync(base + b_runs + b_ptr, w.single_ptr.data(),
                                sizeof(int32_t) * w.single_ptr.size(), cudaMemcpyHostToDevice,
                                st));
    if (!w.single.empty())
      TP_CUDA_TRY(cudaMemcpyAsync(base + b_runs + 2 * b_ptr, w.single.data(),
                                  sizeof(uint16_t) * w.single.size(), cudaMemcpyHostToDevice,
                                  st));
    h->af.runs = reinterpret_cast<const int4*>(base);
    h->af.run_ptr = reinterpret_cast<const int32_t*>(base + b_runs);
    h->af.single_ptr = reinterpret_cast<const int32_t*>(base + b_runs + b_ptr);
    h->af.single = reinterpret_cast<const uint16_t*>(base + b_runs + 2 * b_ptr);
    h->af.single_cap = w.single_cap;
  }
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  auto set = [&](auto& a) {
    a.halo_ptr = h->d_halo_ptr;
    a.halo = h->d_halo;
    a.loc_col = h->d_loc_col;
    a.sp_cap = w.sp_cap;
    a.halo_cap = w.halo_cap;
    a.col_cap = w.col_cap;
    a.win_cap = w.win_cap;
    a.reg_values = w.max_width <= 16 ? 1 : 0;  // the kernel's register-staging width
    // FP32 values in tensor memory: 16 warps, one round of at most 4 slices per warp
    // (k_cgw's MAXS for FP32 without a mass matrix), slices of at most 16 entries
    a.tmem_values = (tm_fit && getenv_flag("DISSOLVE_PCG_TMEM", 1)) ? 1 : 0;
  };
  if (h->fp32)
    set(h->af);
  else
    set(h->ad);
  h->fn = fn;
  h->dyn_smem = d_pipe;
  h->window = pipe ? 3 : (cgt ? 2 : 1);
  // the pipelined recurrences run at most three decades between FP64 refreshes: at 1e-4
  // a refresh threshold let their FP32 drift stall a solve on the benchmark mesh
  if (pipe) h->af.delta2 = std::max(h->af.delta2, PGP_MIN_DELTA * PGP_MIN_DELTA);
  return TP_OK;
}

extern "C" int tp_pcg_create(const tp_csr_op* op, const tp_sell* sell, int max_it,
                             int inner_fp32, double delta, int ctas_per_sm, const double* b,
                             double* x, const double* rtol, void* workspace,
                             size_t workspace_bytes, void* stream, tp_pcg_handle** out) {
  TP_REQUIRE(op && sell && b && x && rtol && workspace && out, "null pointer");
  TP_REQUIRE(op->n_systems <= 1, "the persistent engine solves one system (use tp_cg_*)");
  TP_REQUIRE(op->S >= 1 && op->S <= 4 && (op->ld == 1 || op->ld == 2 || op->ld == 4) &&
                 op->ld >= op->S,
             "bad S/ld");
  TP_REQUIRE(op->indptr && op->indices && op->K64, "operator needs the FP64 CSR values");
  TP_REQUIRE(sell->slice_ptr && sell->sell_col && (inner_fp32 ? sell->sK32 != nullptr : sell->sK64 != nullptr),
             "SELL operator incomplete");
  TP_REQUIRE(!inner_fp32 || !op->diag64 || op->diag32, "FP32 inner solve needs diag32");
  TP_REQUIRE(!sell->sM64 || op->M64, "SELL mass values need the CSR mass values");
  TP_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  TP_REQUIRE(workspace_bytes >= tp_pcg_workspace_bytes(op, inner_fp32), "workspace too small");
  TP_REQUIRE(max_it >= 0, "max_it < 0");
  tp_pcg_handle* h = new tp_pcg_handle();
  h->fp32 = inner_fp32 ? 1 : 0;
  h->ld = op->ld;
  h->block = 512;
  h->window = 0;
  TP_REQUIRE(sell->n_rows == op->n_rows, "SELL and CSR row counts differ");
  const int minb = ctas_per_sm > 0 ? std::min(ctas_per_sm, 2) : default_minb(op->ld);
  const bool hasM = inner_fp32 ? sell->sM32 != nullptr : sell->sM64 != nullptr;
  int rc = pcg_grid(h->fp32, h->ld, minb, hasM, h->block, op->n_rows, &h->grid, &h->dyn_smem);
  if (rc) {
    delete h;
    return rc;
  }
  h->fn = pcg_kernel(h->fp32, h->ld, h->grid / sm_count(), hasM);
  const size_t vt = inner_fp32 ? 4 : 8;
  const size_t vec = a256(vt * op->ld * (size_t)op->n_rows);
  const double d = inner_fp32 ? (delta > 0 ? delta : 0.01) : 0.0;
  char* ws = static_cast<char*>(workspace);
  if (h->fp32)
    fill_pargs(h->af, op, sell, b, x, rtol, max_it, d, ws, vec, h->grid);
  else
    fill_pargs(h->ad, op, sell, b, x, rtol, max_it, d, ws, vec, h->grid);
  h->bar = h->fp32 ? h->af.bar : h->ad.bar;
  h->out = h->fp32 ? h->af.out : h->ad.out;
  cudaStream_t st = as_stream(stream);
  rc = try_window(h, sell, hasM, st);
  if (rc != TP_OK) {
    delete h;
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(h->bar, 0, sizeof(PBar), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->out, 0, sizeof(POut), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error("pcg setup failed: %s", cudaGetErrorString(e));
    delete h;
    return TP_ERR_CUDA;
  }
  *out = h;
  return TP_OK;
}

extern "C" int tp_pcg_run(tp_pcg_handle* h, void* stream) {
  TP_REQUIRE(h, "null handle");
  cudaStream_t st = as_stream(stream);
  // a previous run that timed out leaves the abort flag set: clear the barrier first
  TP_CUDA_TRY(cudaMemsetAsync(h->bar, 0, sizeof(PBar), st));
  void* arg = h->fp32 ? (void*)&h->af : (void*)&h->ad;
  void* args[1] = {arg};
  TP_CUDA_TRY(cudaLaunchCooperativeKernel(h->fn, dim3(h->grid), dim3(h->block), args,
                                          h->dyn_smem, st));
  return TP_OK;
}

extern "C" int tp_pcg_result_get(tp_pcg_handle* h, tp_cg_result* res, int32_t* lane_iters,
                                 int32_t* lane_status, double* lane_rnorm, double* lane_bnorm,
                                 void* stream) {
  TP_REQUIRE(h, "null handle");
  cudaStream_t st = as_stream(stream);
  POut o;
  TP_CUDA_TRY(cudaMemcpyAsync(&o, h->out, sizeof(POut), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  const int S = h->fp32 ? h->af.S : h->ad.S;
  for (int s = 0; s < S; s++) {
    if (lane_iters) lane_iters[s] = o.lane_iters[s];
    if (lane_status) lane_status[s] = o.lane_status[s];
    if (lane_rnorm) lane_rnorm[s] = sqrt(std::max(o.lane_rtrue[s], 0.0));
    if (lane_bnorm) lane_bnorm[s] = sqrt(std::max(o.lane_bb[s], 0.0));
  }
  if (res) {
    res->status = o.status;
    res->iterations = o.iterations;
    res->n_reliable = o.n_reliable;
    res->n_lanes = S;
  }
  return TP_OK;
}

extern "C" int tp_pcg_grid(tp_pcg_handle* h, int* grid, int* block) {
  TP_REQUIRE(h, "null handle");
  if (grid) *grid = h->grid;
  if (block) *block = h->block;
  return TP_OK;
}

extern "C" int tp_pcg_engine(tp_pcg_handle* h, int* window, size_t* smem_bytes) {
  TP_REQUIRE(h, "null handle");
  if (window) *window = h->window;
  if (smem_bytes) *smem_bytes = h->dyn_smem;
  return TP_OK;
}

extern "C" int tp_pcg_set_profile(tp_pcg_handle* h, unsigned long long* prof) {
  TP_REQUIRE(h, "null handle");
  h->af.prof = prof;
  h->ad.prof = prof;
  return TP_OK;
}

extern "C" int tp_pcg_set_wait_limit(tp_pcg_handle* h, unsigned long long limit_ns,
                                     unsigned int missing_arrivals) {
  TP_REQUIRE(h, "null handle");
  TP_REQUIRE(missing_arrivals <= 1024, "missing_arrivals above 1024");
  const unsigned long long lim = limit_ns ? limit_ns : WAIT_LIMIT_NS;
  h->af.wait_limit_ns = h->ad.wait_limit_ns = lim;
  h->af.wait_missing = h->ad.wait_missing = missing_arrivals;
  return TP_OK;
}

extern "C" int tp_pcg_destroy(tp_pcg_handle* h) {
  delete h;
  return TP_OK;
}
