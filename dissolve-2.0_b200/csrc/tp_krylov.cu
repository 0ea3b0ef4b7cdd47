// tp_krylov.cu -- Jacobi-preconditioned CG over many (system, column) lanes, run as one
// CUDA graph with a device-side while loop (conditional node), FP64 or FP32-inner with
// FP64 reliable updates.
//
// Replaces the per-species PETSc KSP(gmres, restart 50) + PC(bjacobi) solve of
// numerics/solvers.py:322-335, 369, whose every inner product returns to the host.
// Here nothing returns to the host until the solve ends.
//
// Work is cut into tiles of rows that never straddle two systems.  Every reduction is
// per tile (one block reduces one tile in a fixed tree), and the last block of each
// kernel (atomic ticket) sums the tile partials of each lane in tile order, so results
// do not depend on the grid size or on block scheduling.
//
// Iteration (lanes l = system * S + column):
//   B1  q = A p,              pq_l = p.q                 -> alpha_l = rz_l / pq_l
//   B2  xi += alpha p, r -= alpha q, z = D^-1 r, rz, rr   -> beta_l, reliable trigger
//   IF  any trigger:  RU1  x += xi, xi = 0 (trigger lanes)
//                     RU2  r = b - A64 x (FP64), z = D^-1 r -> converge / replace
//   B4  p = z + beta p; set the while condition (active lanes and iter < max_it)
// The FP64 path uses the same sequence with the trigger reduced to "recurrence residual
// below tolerance", so convergence is always confirmed on b - A x in FP64.
#include <cuda.h>

#include <algorithm>
#include <vector>

#include "tp_ops.cuh"

namespace tp {

enum LaneStatus : int32_t {
  LS_RUNNING = -1,
  LS_OK = TP_OK,
  LS_MAXIT = TP_ERR_NOT_CONVERGED,
  LS_BREAKDOWN = TP_ERR_BREAKDOWN,
  LS_NONFINITE = TP_ERR_NONFINITE
};

struct Lanes {
  double *rz, *alpha, *beta, *rr, *rmax2, *tol2, *bb, *rtrue;
  int32_t *active, *trigger, *status, *iters;
};

struct Glob {
  int32_t iter, max_it, n_trigger, n_reliable, n_active, cont, timing, pad1;
  uint32_t ticket[8];
  double delta2;
};

constexpr int PQ = 12;  // partial slots per tile: 3 quantities x 4 columns
constexpr int CHUNK = 32;  // tiles per first-level reduction chunk
enum Kind { K_I2 = 0, K_B1 = 1, K_B2 = 2, K_RU2 = 3, K_F2 = 4, N_KINDS = 5 };

template <typename VT>
struct Args {
  int64_t n;
  int S, ld, NL, nsys, ntiles;
  CsrView<VT> Ain;
  CsrView<double> A64;
  const int64_t* tile_row0;
  const int32_t* tile_sys;
  const int32_t* sys_tile_ptr;
  const int32_t* tile_chunk;     // ntiles
  const int32_t* chunk_tile_ptr; // nchunks + 1
  const int32_t* sys_chunk_ptr;  // nsys + 1
  int nchunks;
  double* chunk_part;            // nchunks * PQ
  uint32_t* chunk_ticket;        // N_KINDS * nchunks
  VT *p, *q, *r, *z, *xi, *dinv;
  double* x;
  const double* b;
  const double* rtol;
  double* part;
  Lanes L;
  int32_t* sys_active;
  int32_t* sys_trig;
  uint32_t* sys_ticket;  // N_KINDS * nsys
  Glob* g;
  cudaGraphConditionalHandle h_while, h_if;
};

// ----------------------------------------------------------------- reductions
template <int NV>
__device__ __forceinline__ void block_sum_vec(double v[NV], double* sh /* 32*NV */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) sh[k * 32 + w] = v[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = (lane < nw) ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Called by every thread after thread 0 wrote tile t's partials (slots 0..PQ-1).
// Two-level, fixed-order reduction: the block completing the last tile of a chunk sums
// the chunk's tiles in order into chunk_part; the block completing the last chunk of a
// system returns true (in every thread) and then calls reduce_system.
template <typename VT>
__device__ __forceinline__ bool finish_tile(const Args<VT>& a, int t, int sys, int kind) {
  __shared__ int s_flag;
  const int c = a.tile_chunk[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t ntl = (uint32_t)(a.chunk_tile_ptr[c + 1] - a.chunk_tile_ptr[c]);
    const uint32_t k = atomicAdd(&a.chunk_ticket[kind * a.nchunks + c], 1u);
    s_flag = (k == ntl - 1);
    if (s_flag) a.chunk_ticket[kind * a.nchunks + c] = 0u;
  }
  __syncthreads();
  if (!s_flag) return false;
  __threadfence();
  if (threadIdx.x < PQ) {
    const int t0 = a.chunk_tile_ptr[c], t1 = a.chunk_tile_ptr[c + 1];
    double v = 0.0;
#pragma unroll 8
    for (int u = t0; u < t1; u++) v += __ldcg(a.part + (int64_t)u * PQ + threadIdx.x);
    a.chunk_part[(int64_t)c * PQ + threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t nch = (uint32_t)(a.sys_chunk_ptr[sys + 1] - a.sys_chunk_ptr[sys]);
    const uint32_t k = atomicAdd(&a.sys_ticket[kind * a.nsys + sys], 1u);
    s_flag = (k == nch - 1);
    if (s_flag) a.sys_ticket[kind * a.nsys + sys] = 0u;
  }
  __syncthreads();
  const bool last = s_flag;
  if (last) __threadfence();
  return last;
}

// true in every thread of the block that finished last in the grid
__device__ __forceinline__ bool global_last(uint32_t* ticket) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1);
    if (s_last) *ticket = 0u;
  }
  __syncthreads();
  const bool last = s_last;
  if (last) __threadfence();
  return last;
}

// Fixed-order sum of the system's chunk partials: NQ quantities x 4 columns, result in
// tot (valid in thread 0).
template <int NQ, typename VT>
__device__ __forceinline__ void reduce_system(const Args<VT>& a, int sys, double tot[NQ * 4]) {
  __shared__ double s_tot[PQ];
  if (threadIdx.x < NQ * 4) {
    const int c0 = a.sys_chunk_ptr[sys], c1 = a.sys_chunk_ptr[sys + 1];
    double v = 0.0;
#pragma unroll 8
    for (int c = c0; c < c1; c++) v += __ldcg(a.chunk_part + (int64_t)c * PQ + threadIdx.x);
    s_tot[threadIdx.x] = v;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NQ * 4; k++) tot[k] = s_tot[k];
  __syncthreads();
}

template <typename VT, int LD>
__device__ __forceinline__ void lane_vals(const double* arr, const Args<VT>& a, int sys,
                                          double out[LD]) {
#pragma unroll
  for (int s = 0; s < LD; s++) out[s] = (s < a.S) ? arr[sys * a.S + s] : 0.0;
}

template <typename VT>
__device__ __forceinline__ void set_inactive(const Args<VT>& a, int l, int status, int it) {
  a.L.active[l] = 0;
  a.L.status[l] = status;
  a.L.iters[l] = it;
  atomicSub(&a.g->n_active, 1);
}

template <typename VT>
__device__ __forceinline__ void refresh_system(const Args<VT>& a, int sys) {
  int act = 0;
  for (int s = 0; s < a.S; s++) act |= a.L.active[sys * a.S + s];
  a.sys_active[sys] = act;
}

// ----------------------------------------------------------------- init
// I1: Jacobi diagonal from the current FP64 values, Dirichlet values into x, counters
template <typename VT, int LD>
__global__ void k_i1(Args<VT> a) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.g->iter = 0;
    a.g->n_active = 0;
    a.g->n_trigger = 0;
    a.g->n_reliable = 0;
  }
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < a.n;
       row += (int64_t)gridDim.x * blockDim.x) {
    VT dv[LD];
    const bool bc = a.A64.bc && a.A64.bc[row];
    if (bc) {
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
        double d = a.A64.dscale[s] * kd + a.A64.cscale[s] * md;
        if (a.A64.diag) d += a.A64.diag[row * LD + s];
        dv[s] = (s < a.S && d != 0.0) ? VT(1.0 / d) : VT(0);
      }
    }
    stv<VT, LD>(a.dinv, row, dv);
  }
}

// FP64 residual r64 = b - A64 x of one row (all G lanes call it)
template <typename VT, int LD, int G>
__device__ __forceinline__ void residual64(const Args<VT>& a, int64_t rr, int gl,
                                           double r64[LD]) {
  double ax[LD];
  csr_row<double, LD, G, false>(a.A64, rr, gl, a.x, ax);
  double bv[LD];
  ldv_cg<double, LD>(a.b, rr, bv);
#pragma unroll
  for (int s = 0; s < LD; s++) r64[s] = (s < a.S) ? bv[s] - ax[s] : 0.0;
}

// I2: r = b - A x, z = D^-1 r, p = z, xi = 0; per system rr, rz, bb -> lane state
template <typename VT, int LD, int G, bool COND>
__global__ void __launch_bounds__(256) k_i2(Args<VT> a) {
  __shared__ double sh[32 * 3 * LD];
  const int gl = threadIdx.x % G;
  const int rpb = blockDim.x / G;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    double acc[3 * LD];
#pragma unroll
    for (int k = 0; k < 3 * LD; k++) acc[k] = 0.0;
    for (int64_t base = r0; base < r1; base += rpb) {
      const int64_t row = base + threadIdx.x / G;
      const int64_t rr = row < r1 ? row : r1 - 1;
      double r64[LD];
      residual64<VT, LD, G>(a, rr, gl, r64);
      if (row < r1 && gl == 0) {
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
          acc[LD + s] += (double)rv[s] * (double)zv[s];
          acc[2 * LD + s] += (s < a.S) ? bv[s] * bv[s] : 0.0;
        }
        stv<VT, LD>(a.r, row, rv);
        stv<VT, LD>(a.z, row, zv);
        stv<VT, LD>(a.p, row, zv);
        stv<VT, LD>(a.xi, row, zero);
      }
    }
    block_sum_vec<3 * LD>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        a.part[(int64_t)t * PQ + 0 + s] = s < LD ? acc[s] : 0.0;
        a.part[(int64_t)t * PQ + 4 + s] = s < LD ? acc[LD + s] : 0.0;
        a.part[(int64_t)t * PQ + 8 + s] = s < LD ? acc[2 * LD + s] : 0.0;
      }
    }
    if (finish_tile(a, t, sys, K_I2)) {
      double tot[12];
      reduce_system<3>(a, sys, tot);
      if (threadIdx.x == 0) {
        int act_all = 0;
        for (int s = 0; s < a.S; s++) {
          const int l = sys * a.S + s;
          const double rr = tot[s], rz = tot[4 + s], bb = tot[8 + s];
          const double rt = a.rtol[l];
          a.L.bb[l] = bb;
          a.L.tol2[l] = rt * rt * bb;
          a.L.rr[l] = rr;
          a.L.rtrue[l] = rr;
          a.L.rmax2[l] = rr;
          a.L.rz[l] = rz;
          a.L.alpha[l] = 0.0;
          a.L.beta[l] = 0.0;
          a.L.trigger[l] = 0;
          a.L.iters[l] = 0;
          const bool fin = isfinite(rr) && isfinite(rz);
          const bool act = fin && rr > a.L.tol2[l];
          a.L.active[l] = act;
          a.L.status[l] = !fin ? LS_NONFINITE : (act ? LS_RUNNING : LS_OK);
          act_all += act;
        }
        a.sys_active[sys] = act_all > 0;
        a.sys_trig[sys] = 0;
        if (act_all) atomicAdd(&a.g->n_active, act_all);
      }
    }
  }
  if (global_last(&a.g->ticket[K_I2]) && threadIdx.x == 0) {
    const int cont = (a.g->n_active > 0) && (a.g->max_it > 0);
    a.g->cont = cont;
    if constexpr (COND) cudaGraphSetConditional(a.h_while, cont);
  }
}

// ----------------------------------------------------------------- iteration
// B1: q = A p, pq per lane -> alpha
template <typename VT, int LD, int G>
__global__ void __launch_bounds__(256) k_b1(Args<VT> a) {
  __shared__ double sh[32 * LD];
  const int gl = threadIdx.x % G;
  const int rpb = blockDim.x / G;
  const VT* __restrict__ P = a.p;
  VT* __restrict__ Q = a.q;
  const bool timing = a.g->timing != 0;  // autotuner / roofline timing: all tiles, no lane updates
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    if (!timing && !a.sys_active[sys]) continue;
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    double acc[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) acc[s] = 0.0;
    for (int64_t base = r0; base < r1; base += rpb) {
      const int64_t row = base + threadIdx.x / G;
      const int64_t rr = row < r1 ? row : r1 - 1;
      VT qv[LD];
      csr_row<VT, LD, G, true>(a.Ain, rr, gl, P, qv);
      if (row < r1 && gl == 0) {
        stv<VT, LD>(Q, row, qv);
        VT pv[LD];
        ldv<VT, LD>(P, row, pv);
#pragma unroll
        for (int s = 0; s < LD; s++) acc[s] += (double)pv[s] * (double)qv[s];
      }
    }
    block_sum_vec<LD>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) a.part[(int64_t)t * PQ + s] = s < LD ? acc[s] : 0.0;
    }
    if (finish_tile(a, t, sys, K_B1)) {
      double tot[4];
      reduce_system<1>(a, sys, tot);
      if (threadIdx.x == 0 && !timing) {
        for (int s = 0; s < a.S; s++) {
          const int l = sys * a.S + s;
          if (!a.L.active[l]) {
            a.L.alpha[l] = 0.0;
            continue;
          }
          const double pq = tot[s];
          if (!isfinite(pq) || !(pq > 0.0)) {
            a.L.alpha[l] = 0.0;
            set_inactive(a, l, isfinite(pq) ? LS_BREAKDOWN : LS_NONFINITE, a.g->iter);
            continue;
          }
          a.L.alpha[l] = a.L.rz[l] / pq;
        }
        refresh_system(a, sys);
      }
    }
  }
}

// B2: xi += alpha p, r -= alpha q, z = D^-1 r; rz, rr per lane -> beta, trigger
template <typename VT, int LD, bool COND>
__global__ void __launch_bounds__(256) k_b2(Args<VT> a) {
  __shared__ double sh[32 * 2 * LD];
  const VT* __restrict__ P = a.p;
  const VT* __restrict__ Q = a.q;
  const VT* __restrict__ DI = a.dinv;
  VT* __restrict__ R = a.r;
  VT* __restrict__ XI = a.xi;
  VT* __restrict__ Z = a.z;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    if (!a.sys_active[sys]) continue;
    double al[LD];
    lane_vals<VT, LD>(a.L.alpha, a, sys, al);
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    double acc[2 * LD];
#pragma unroll
    for (int k = 0; k < 2 * LD; k++) acc[k] = 0.0;
    for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
      VT pv[LD], qv[LD], rv[LD], xv[LD], dv[LD], zv[LD];
      ldv_cg<VT, LD>(P, row, pv);
      ldv_cg<VT, LD>(Q, row, qv);
      ldv_cg<VT, LD>(R, row, rv);
      ldv_cg<VT, LD>(XI, row, xv);
      ldv<VT, LD>(DI, row, dv);
#pragma unroll
      for (int s = 0; s < LD; s++) {
        if (al[s] != 0.0) {
          const VT as = (VT)al[s];
          xv[s] += as * pv[s];
          rv[s] -= as * qv[s];
        }
        zv[s] = dv[s] * rv[s];
        acc[s] += (double)rv[s] * (double)zv[s];
        acc[LD + s] += (double)rv[s] * (double)rv[s];
      }
      stv<VT, LD>(XI, row, xv);
      stv<VT, LD>(R, row, rv);
      stv<VT, LD>(Z, row, zv);
    }
    block_sum_vec<2 * LD>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        a.part[(int64_t)t * PQ + s] = s < LD ? acc[s] : 0.0;
        a.part[(int64_t)t * PQ + 4 + s] = s < LD ? acc[LD + s] : 0.0;
      }
    }
    if (finish_tile(a, t, sys, K_B2)) {
      double tot[8];
      reduce_system<2>(a, sys, tot);
      if (threadIdx.x == 0) {
        const int it = a.g->iter + 1;
        int ntrig = 0;
        for (int s = 0; s < a.S; s++) {
          const int l = sys * a.S + s;
          if (!a.L.active[l]) {
            a.L.beta[l] = 0.0;
            a.L.trigger[l] = 0;
            continue;
          }
          const double rz = tot[s], rr = tot[4 + s];
          if (!isfinite(rz) || !isfinite(rr)) {
            a.L.trigger[l] = 0;
            set_inactive(a, l, LS_NONFINITE, it);
            continue;
          }
          const double old = a.L.rz[l];
          a.L.beta[l] = (old != 0.0) ? rz / old : 0.0;
          a.L.rz[l] = rz;
          a.L.rr[l] = rr;
          const bool trig = (rr <= a.L.tol2[l]) ||
                            (a.g->delta2 > 0.0 && rr < a.g->delta2 * a.L.rmax2[l]);
          a.L.trigger[l] = trig;
          ntrig += trig;
        }
        a.sys_trig[sys] = ntrig > 0;
        if (ntrig) atomicAdd(&a.g->n_trigger, ntrig);
        refresh_system(a, sys);
      }
    }
  }
  if (global_last(&a.g->ticket[K_B2]) && threadIdx.x == 0) {
    a.g->iter += 1;
    if constexpr (COND) cudaGraphSetConditional(a.h_if, a.g->n_trigger > 0 ? 1u : 0u);
  }
}

// RU1: fold the inner correction of trigger lanes into x (FP64)
template <typename VT, int LD>
__global__ void k_ru1(Args<VT> a) {
  if (a.g->n_trigger == 0) return;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    if (!a.sys_trig[sys]) continue;
    int trig[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) trig[s] = (s < a.S) ? a.L.trigger[sys * a.S + s] : 0;
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
      VT xv[LD];
      ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
      for (int s = 0; s < LD; s++) {
        if (trig[s]) {
          a.x[row * LD + s] += (double)xv[s];
          xv[s] = VT(0);
        }
      }
      stv<VT, LD>(a.xi, row, xv);
    }
  }
}

// RU2: FP64 residual of trigger lanes; converge or replace the inner residual
template <typename VT, int LD, int G>
__global__ void __launch_bounds__(256) k_ru2(Args<VT> a) {
  __shared__ double sh[32 * 2 * LD];
  if (a.g->n_trigger == 0) return;
  const int gl = threadIdx.x % G;
  const int rpb = blockDim.x / G;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    if (!a.sys_trig[sys]) continue;
    int trig[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) trig[s] = (s < a.S) ? a.L.trigger[sys * a.S + s] : 0;
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    double acc[2 * LD];
#pragma unroll
    for (int k = 0; k < 2 * LD; k++) acc[k] = 0.0;
    for (int64_t base = r0; base < r1; base += rpb) {
      const int64_t row = base + threadIdx.x / G;
      const int64_t rr = row < r1 ? row : r1 - 1;
      double r64[LD];
      residual64<VT, LD, G>(a, rr, gl, r64);
      if (row < r1 && gl == 0) {
        VT rv[LD], dv[LD], zv[LD];
        ldv_cg<VT, LD>(a.r, row, rv);
        ldv<VT, LD>(a.dinv, row, dv);
        ldv_cg<VT, LD>(a.z, row, zv);
#pragma unroll
        for (int s = 0; s < LD; s++) {
          if (trig[s]) {
            rv[s] = (VT)r64[s];
            zv[s] = dv[s] * rv[s];
            acc[s] += r64[s] * r64[s];
            acc[LD + s] += (double)rv[s] * (double)zv[s];
          }
        }
        stv<VT, LD>(a.r, row, rv);
        stv<VT, LD>(a.z, row, zv);
      }
    }
    block_sum_vec<2 * LD>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) {
        a.part[(int64_t)t * PQ + s] = s < LD ? acc[s] : 0.0;
        a.part[(int64_t)t * PQ + 4 + s] = s < LD ? acc[LD + s] : 0.0;
      }
    }
    if (finish_tile(a, t, sys, K_RU2)) {
      double tot[8];
      reduce_system<2>(a, sys, tot);
      if (threadIdx.x == 0) {
        const int it = a.g->iter;
        for (int s = 0; s < a.S; s++) {
          const int l = sys * a.S + s;
          if (!a.L.trigger[l]) continue;
          a.L.trigger[l] = 0;
          const double rr = tot[s], rz = tot[4 + s];
          a.L.rtrue[l] = rr;
          if (!isfinite(rr)) {
            set_inactive(a, l, LS_NONFINITE, it);
          } else if (rr <= a.L.tol2[l]) {
            set_inactive(a, l, LS_OK, it);
          } else {
            a.L.rz[l] = rz;
            a.L.rr[l] = rr;
            a.L.rmax2[l] = rr;
          }
        }
        a.sys_trig[sys] = 0;
        refresh_system(a, sys);
      }
    }
  }
  if (global_last(&a.g->ticket[K_RU2]) && threadIdx.x == 0) {
    a.g->n_reliable += 1;
    a.g->n_trigger = 0;
  }
}

// B4: p = z + beta p; decide whether the loop continues
template <typename VT, int LD, bool COND>
__global__ void __launch_bounds__(256) k_b4(Args<VT> a) {
  const VT* __restrict__ Z = a.z;
  VT* __restrict__ P = a.p;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    if (!a.sys_active[sys]) continue;
    double be[LD];
    lane_vals<VT, LD>(a.L.beta, a, sys, be);
    int act[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) act[s] = (s < a.S) ? a.L.active[sys * a.S + s] : 0;
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
      VT pv[LD], zv[LD];
      ldv_cg<VT, LD>(P, row, pv);
      ldv_cg<VT, LD>(Z, row, zv);
#pragma unroll
      for (int s = 0; s < LD; s++)
        if (act[s]) pv[s] = zv[s] + (VT)be[s] * pv[s];
      stv<VT, LD>(P, row, pv);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int cont = (a.g->n_active > 0) && (a.g->iter < a.g->max_it);
    a.g->cont = cont;
    if constexpr (COND) cudaGraphSetConditional(a.h_while, cont);
  }
}

// F1: fold what is left of xi into x
template <typename VT, int LD>
__global__ void k_f1(Args<VT> a) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < a.n;
       row += (int64_t)gridDim.x * blockDim.x) {
    VT xv[LD];
    ldv_cg<VT, LD>(a.xi, row, xv);
#pragma unroll
    for (int s = 0; s < LD; s++) {
      if (s < a.S) a.x[row * LD + s] += (double)xv[s];
      xv[s] = VT(0);
    }
    stv<VT, LD>(a.xi, row, xv);
  }
}

// F2: true residual of every lane; final lane status
template <typename VT, int LD, int G>
__global__ void __launch_bounds__(256) k_f2(Args<VT> a) {
  __shared__ double sh[32 * LD];
  const int gl = threadIdx.x % G;
  const int rpb = blockDim.x / G;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const int sys = a.tile_sys[t];
    const int64_t r0 = a.tile_row0[t], r1 = a.tile_row0[t + 1];
    double acc[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) acc[s] = 0.0;
    for (int64_t base = r0; base < r1; base += rpb) {
      const int64_t row = base + threadIdx.x / G;
      const int64_t rr = row < r1 ? row : r1 - 1;
      double r64[LD];
      residual64<VT, LD, G>(a, rr, gl, r64);
      if (row < r1 && gl == 0) {
#pragma unroll
        for (int s = 0; s < LD; s++) acc[s] += r64[s] * r64[s];
      }
    }
    block_sum_vec<LD>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < 4; s++) a.part[(int64_t)t * PQ + s] = s < LD ? acc[s] : 0.0;
    }
    if (finish_tile(a, t, sys, K_F2)) {
      double tot[4];
      reduce_system<1>(a, sys, tot);
      if (threadIdx.x == 0) {
        const int it = a.g->iter;
        for (int s = 0; s < a.S; s++) {
          const int l = sys * a.S + s;
          a.L.rtrue[l] = tot[s];
          if (a.L.status[l] == LS_RUNNING) {
            a.L.status[l] = (tot[s] <= a.L.tol2[l]) ? LS_OK : LS_MAXIT;
            a.L.iters[l] = it;
            a.L.active[l] = 0;
          }
        }
      }
    }
  }
}

// ----------------------------------------------------------------- host side
static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
  size_t vec, part, lanes_d, lanes_i, sysact, systrig, systicket, glob, trow, tsys, sptr,
      tchunk, cptr, schptr, cpart, cticket, total;
};

// Row tiles (never straddling two systems) and chunks of up to CHUNK tiles of one system.
struct Tiles {
  std::vector<int64_t> row0;
  std::vector<int32_t> tsys, sptr, tchunk, cptr, schptr;
  int64_t nt = 0, nch = 0;
};

static Tiles make_tiles(const tp_csr_op* op, int rpt) {
  Tiles T;
  const int nsys = op->n_systems > 0 ? op->n_systems : 1;
  T.sptr.push_back(0);
  T.cptr.push_back(0);
  T.schptr.push_back(0);
  for (int m = 0; m < nsys; m++) {
    const int64_t a = op->sys_row_ptr ? op->sys_row_ptr[m] : 0;
    const int64_t b = op->sys_row_ptr ? op->sys_row_ptr[m + 1] : op->n_rows;
    int64_t in_chunk = 0;
    for (int64_t r = a; r < b; r += rpt) {
      if (in_chunk == CHUNK) {
        T.cptr.push_back((int32_t)T.nt);
        T.nch++;
        in_chunk = 0;
      }
      T.row0.push_back(r);
      T.tsys.push_back(m);
      T.tchunk.push_back((int32_t)T.nch);
      T.nt++;
      in_chunk++;
    }
    if (in_chunk > 0) {
      T.cptr.push_back((int32_t)T.nt);
      T.nch++;
    }
    T.sptr.push_back((int32_t)T.nt);
    T.schptr.push_back((int32_t)T.nch);
  }
  T.row0.push_back(op->n_rows);
  return T;
}

static int64_t count_tiles(const tp_csr_op* op, int rpt, int64_t* nch) {
  const Tiles T = make_tiles(op, rpt);
  if (nch) *nch = T.nch;
  return T.nt;
}

static Layout layout(const tp_csr_op* op, const tp_cg_config* cfg) {
  const int nsys = op->n_systems > 0 ? op->n_systems : 1;
  const int NL = nsys * op->S;
  const size_t vt = cfg->inner_fp32 ? 4 : 8;
  int64_t nch = 0;
  const int64_t nt = count_tiles(op, cfg->rows_per_tile, &nch);
  const size_t nt1 = (size_t)std::max<int64_t>(nt, 1), nc1 = (size_t)std::max<int64_t>(nch, 1);
  Layout L;
  L.vec = al256(vt * op->ld * (size_t)op->n_rows);
  L.part = al256(sizeof(double) * PQ * nt1);
  L.lanes_d = al256(sizeof(double) * NL);
  L.lanes_i = al256(sizeof(int32_t) * NL);
  L.sysact = al256(sizeof(int32_t) * nsys);
  L.systrig = al256(sizeof(int32_t) * nsys);
  L.systicket = al256(sizeof(uint32_t) * N_KINDS * nsys);
  L.glob = al256(sizeof(Glob));
  L.trow = al256(sizeof(int64_t) * (nt + 1));
  L.tsys = al256(sizeof(int32_t) * nt1);
  L.sptr = al256(sizeof(int32_t) * (nsys + 1));
  L.tchunk = al256(sizeof(int32_t) * nt1);
  L.cptr = al256(sizeof(int32_t) * (nc1 + 1));
  L.schptr = al256(sizeof(int32_t) * (nsys + 1));
  L.cpart = al256(sizeof(double) * PQ * nc1);
  L.cticket = al256(sizeof(uint32_t) * N_KINDS * nc1);
  L.total = 6 * L.vec + L.part + 8 * L.lanes_d + 4 * L.lanes_i + L.sysact + L.systrig +
            L.systicket + L.glob + L.trow + L.tsys + L.sptr + L.tchunk + L.cptr + L.schptr +
            L.cpart + L.cticket;
  return L;
}

}  // namespace tp

struct tp_cg_handle {
  int vt_fp32, ld, G, block, grid, row_grid, ntiles, NL, max_it, use_cond;
  tp::Args<float> af;
  tp::Args<double> ad;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // host-loop variant
  cudaGraph_t g_init = nullptr, g_iter = nullptr, g_fin = nullptr;
  cudaGraphExec_t e_init = nullptr, e_iter = nullptr, e_fin = nullptr;
  tp::Glob* glob;
  tp::Lanes lanes;
  int32_t* sys_active;
};

namespace tp {

using KFn = void*;

struct KernelSet {
  KFn i1, i2, b1, b2, ru1, ru2, b4, f1, f2;
};

// COND: the variant that drives the graph's conditional nodes; the host-loop variant
// carries no device-side conditional call (profilers can then see every kernel node).
template <typename VT, int LD, int G, bool COND>
static KernelSet kset() {
  KernelSet k;
  k.i1 = (KFn)k_i1<VT, LD>;
  k.i2 = (KFn)k_i2<VT, LD, G, COND>;
  k.b1 = (KFn)k_b1<VT, LD, G>;
  k.b2 = (KFn)k_b2<VT, LD, COND>;
  k.ru1 = (KFn)k_ru1<VT, LD>;
  k.ru2 = (KFn)k_ru2<VT, LD, G>;
  k.b4 = (KFn)k_b4<VT, LD, COND>;
  k.f1 = (KFn)k_f1<VT, LD>;
  k.f2 = (KFn)k_f2<VT, LD, G>;
  return k;
}

template <typename VT, int LD, bool COND>
static bool kset_gc(int G, KernelSet* k) {
  switch (G) {
    case 1: *k = kset<VT, LD, 1, COND>(); return true;
    case 2: *k = kset<VT, LD, 2, COND>(); return true;
    case 4: *k = kset<VT, LD, 4, COND>(); return true;
    case 8: *k = kset<VT, LD, 8, COND>(); return true;
    default: return false;
  }
}

template <typename VT, int LD>
static bool kset_g(int G, bool cond, KernelSet* k) {
  return cond ? kset_gc<VT, LD, true>(G, k) : kset_gc<VT, LD, false>(G, k);
}

static bool get_kernels(int fp32, int ld, int G, bool cond, KernelSet* k) {
  if (fp32) {
    if (ld == 1) return kset_g<float, 1>(G, cond, k);
    if (ld == 2) return kset_g<float, 2>(G, cond, k);
    if (ld == 4) return kset_g<float, 4>(G, cond, k);
  } else {
    if (ld == 1) return kset_g<double, 1>(G, cond, k);
    if (ld == 2) return kset_g<double, 2>(G, cond, k);
    if (ld == 4) return kset_g<double, 4>(G, cond, k);
  }
  return false;
}

static int add_kernel(cudaGraph_t g, const cudaGraphNode_t* deps, size_t nd, KFn fn, int grid,
                      int block, void* arg, cudaGraphNode_t* out) {
  cudaKernelNodeParams p = {};
  p.func = fn;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(block);
  p.sharedMemBytes = 0;
  void* args[1] = {arg};
  p.kernelParams = args;
  TP_CUDA_TRY(cudaGraphAddKernelNode(out, g, deps, nd, &p));
  return TP_OK;
}

#define TP_TRY(x)          \
  do {                     \
    int _rc = (x);         \
    if (_rc) return _rc;   \
  } while (0)

static void set_handles(tp_cg_handle* h, cudaGraphConditionalHandle hw,
                        cudaGraphConditionalHandle hi) {
  if (h->vt_fp32) {
    h->af.h_while = hw;
    h->af.h_if = hi;
  } else {
    h->ad.h_while = hw;
    h->ad.h_if = hi;
  }
}

// Kernel node parameters are copied when a node is added, so both conditional handles
// are created (and stored in the argument struct) before the first kernel node.
static int build_graphs(tp_cg_handle* h, const KernelSet& K, void* arg) {
  const int G = h->grid, B = h->block, RG = h->row_grid;
  if (h->use_cond) {
    TP_CUDA_TRY(cudaGraphCreate(&h->graph, 0));
    cudaGraph_t g = h->graph;
    cudaGraphConditionalHandle hw, hi;
    TP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t n_w;
    TP_CUDA_TRY(cudaGraphAddNode(&n_w, g, nullptr, 0, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    TP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hi, body, 0, cudaGraphCondAssignDefault));
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hi;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    set_handles(h, hw, hi);
    // main graph: I1 -> I2 -> while -> F1 -> F2
    cudaGraphNode_t n_i1, n_i2, n_f1, n_f2;
    TP_TRY(add_kernel(g, nullptr, 0, K.i1, RG, B, arg, &n_i1));
    TP_TRY(add_kernel(g, &n_i1, 1, K.i2, G, B, arg, &n_i2));
    TP_CUDA_TRY(cudaGraphAddDependencies(g, &n_i2, &n_w, 1));
    TP_TRY(add_kernel(g, &n_w, 1, K.f1, RG, B, arg, &n_f1));
    TP_TRY(add_kernel(g, &n_f1, 1, K.f2, G, B, arg, &n_f2));
    // body: B1 -> B2 -> if(RU1 -> RU2) -> B4
    cudaGraphNode_t n_b1, n_b2, n_if, n_b4, n_r1, n_r2;
    TP_TRY(add_kernel(body, nullptr, 0, K.b1, G, B, arg, &n_b1));
    TP_TRY(add_kernel(body, &n_b1, 1, K.b2, G, B, arg, &n_b2));
    TP_CUDA_TRY(cudaGraphAddNode(&n_if, body, &n_b2, 1, &ip));
    cudaGraph_t ifb = ip.conditional.phGraph_out[0];
    TP_TRY(add_kernel(ifb, nullptr, 0, K.ru1, G, B, arg, &n_r1));
    TP_TRY(add_kernel(ifb, &n_r1, 1, K.ru2, G, B, arg, &n_r2));
    TP_TRY(add_kernel(body, &n_if, 1, K.b4, G, B, arg, &n_b4));
    TP_CUDA_TRY(cudaGraphInstantiate(&h->exec, g, 0));
    return TP_OK;
  }
  // host loop: init, one iteration (RU kernels exit early without a trigger), final
  cudaGraphNode_t a0, a1, b1, b2, r1, r2, b4, f1, f2;
  TP_CUDA_TRY(cudaGraphCreate(&h->g_init, 0));
  TP_TRY(add_kernel(h->g_init, nullptr, 0, K.i1, RG, B, arg, &a0));
  TP_TRY(add_kernel(h->g_init, &a0, 1, K.i2, G, B, arg, &a1));
  TP_CUDA_TRY(cudaGraphCreate(&h->g_iter, 0));
  TP_TRY(add_kernel(h->g_iter, nullptr, 0, K.b1, G, B, arg, &b1));
  TP_TRY(add_kernel(h->g_iter, &b1, 1, K.b2, G, B, arg, &b2));
  TP_TRY(add_kernel(h->g_iter, &b2, 1, K.ru1, G, B, arg, &r1));
  TP_TRY(add_kernel(h->g_iter, &r1, 1, K.ru2, G, B, arg, &r2));
  TP_TRY(add_kernel(h->g_iter, &r2, 1, K.b4, G, B, arg, &b4));
  TP_CUDA_TRY(cudaGraphCreate(&h->g_fin, 0));
  TP_TRY(add_kernel(h->g_fin, nullptr, 0, K.f1, RG, B, arg, &f1));
  TP_TRY(add_kernel(h->g_fin, &f1, 1, K.f2, G, B, arg, &f2));
  TP_CUDA_TRY(cudaGraphInstantiate(&h->e_init, h->g_init, 0));
  TP_CUDA_TRY(cudaGraphInstantiate(&h->e_iter, h->g_iter, 0));
  TP_CUDA_TRY(cudaGraphInstantiate(&h->e_fin, h->g_fin, 0));
  return TP_OK;
}

template <typename VT>
static void fill_args(Args<VT>& a, const tp_csr_op* op, const tp_cg_config* cfg, char* ws,
                      const Layout& L, int64_t nt, int64_t nch, const double* b, double* x,
                      const double* rtol, int use_cond) {
  const int nsys = op->n_systems > 0 ? op->n_systems : 1;
  a.n = op->n_rows;
  a.S = op->S;
  a.ld = op->ld;
  a.nsys = nsys;
  a.NL = nsys * op->S;
  a.ntiles = (int)nt;
  a.nchunks = (int)nch;
  (void)use_cond;
  a.Ain.indptr = a.A64.indptr = op->indptr;
  a.Ain.indices = a.A64.indices = op->indices;
  a.Ain.bc = a.A64.bc = op->bc_mask;
  for (int s = 0; s < 4; s++) {
    const double d = s < op->S ? op->dscale[s] : 0.0, c = s < op->S ? op->cscale[s] : 0.0;
    a.Ain.dscale[s] = a.A64.dscale[s] = d;
    a.Ain.cscale[s] = a.A64.cscale[s] = c;
  }
  a.A64.K = op->K64;
  a.A64.M = op->M64;
  a.A64.diag = op->diag64;
  if constexpr (sizeof(VT) == 4) {
    a.Ain.K = op->K32;
    a.Ain.M = op->M32;
    a.Ain.diag = op->diag32;
  } else {
    a.Ain.K = op->K64;
    a.Ain.M = op->M64;
    a.Ain.diag = op->diag64;
  }
  (void)cfg;
  char* p = ws;
  VT** vecs[6] = {&a.p, &a.q, &a.r, &a.z, &a.xi, &a.dinv};
  for (int i = 0; i < 6; i++) {
    *vecs[i] = reinterpret_cast<VT*>(p);
    p += L.vec;
  }
  a.part = reinterpret_cast<double*>(p);
  p += L.part;
  double** ld_[8] = {&a.L.rz, &a.L.alpha, &a.L.beta, &a.L.rr, &a.L.rmax2, &a.L.tol2, &a.L.bb,
                     &a.L.rtrue};
  for (int i = 0; i < 8; i++) {
    *ld_[i] = reinterpret_cast<double*>(p);
    p += L.lanes_d;
  }
  int32_t** li_[4] = {&a.L.active, &a.L.trigger, &a.L.status, &a.L.iters};
  for (int i = 0; i < 4; i++) {
    *li_[i] = reinterpret_cast<int32_t*>(p);
    p += L.lanes_i;
  }
  a.sys_active = reinterpret_cast<int32_t*>(p);
  p += L.sysact;
  a.sys_trig = reinterpret_cast<int32_t*>(p);
  p += L.systrig;
  a.sys_ticket = reinterpret_cast<uint32_t*>(p);
  p += L.systicket;
  a.g = reinterpret_cast<Glob*>(p);
  p += L.glob;
  a.tile_row0 = reinterpret_cast<const int64_t*>(p);
  p += L.trow;
  a.tile_sys = reinterpret_cast<const int32_t*>(p);
  p += L.tsys;
  a.sys_tile_ptr = reinterpret_cast<const int32_t*>(p);
  p += L.sptr;
  a.tile_chunk = reinterpret_cast<const int32_t*>(p);
  p += L.tchunk;
  a.chunk_tile_ptr = reinterpret_cast<const int32_t*>(p);
  p += L.cptr;
  a.sys_chunk_ptr = reinterpret_cast<const int32_t*>(p);
  p += L.schptr;
  a.chunk_part = reinterpret_cast<double*>(p);
  p += L.cpart;
  a.chunk_ticket = reinterpret_cast<uint32_t*>(p);
  a.x = x;
  a.b = b;
  a.rtol = rtol;
  a.h_while = 0;
  a.h_if = 0;
}

}  // namespace tp

using namespace tp;

extern "C" size_t tp_cg_workspace_bytes(const tp_csr_op* op, const tp_cg_config* cfg) {
  if (!op || !cfg || cfg->rows_per_tile <= 0) return 0;
  return layout(op, cfg).total;
}

extern "C" int tp_cg_create(const tp_csr_op* op, const tp_cg_config* cfg, const double* b,
                            double* x, const double* rtol, void* workspace,
                            size_t workspace_bytes, void* stream, tp_cg_handle** out) {
  TP_REQUIRE(op && cfg && b && x && rtol && workspace && out, "null pointer");
  TP_REQUIRE(op->indptr && op->indices && op->K64, "operator needs indptr, indices, K64");
  TP_REQUIRE(op->S >= 1 && op->S <= TP_MAX_COLS, "S must be 1..4");
  TP_REQUIRE(op->ld == 1 || op->ld == 2 || op->ld == 4, "ld must be 1, 2 or 4");
  TP_REQUIRE(op->ld >= op->S, "ld < S");
  TP_REQUIRE(!cfg->inner_fp32 || op->K32, "FP32 inner solve needs K32");
  TP_REQUIRE(!op->M64 || !cfg->inner_fp32 || op->M32, "FP32 inner solve needs M32");
  TP_REQUIRE(!op->diag64 || !cfg->inner_fp32 || op->diag32, "FP32 inner solve needs diag32");
  TP_REQUIRE(cfg->block == 128 || cfg->block == 256, "block must be 128 or 256");
  TP_REQUIRE(cfg->group == 1 || cfg->group == 2 || cfg->group == 4 || cfg->group == 8,
             "group must be 1, 2, 4 or 8");
  TP_REQUIRE(cfg->rows_per_tile >= cfg->block && cfg->rows_per_tile % cfg->block == 0,
             "rows_per_tile must be a positive multiple of block");
  TP_REQUIRE(cfg->max_it >= 0, "max_it < 0");
  const int nsys = op->n_systems > 0 ? op->n_systems : 1;
  TP_REQUIRE(nsys == 1 || op->sys_row_ptr, "sys_row_ptr required for several systems");
  TP_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  TP_REQUIRE(((uintptr_t)b & 31) == 0 && ((uintptr_t)x & 31) == 0, "b, x must be 32-byte aligned");
  const Layout L = layout(op, cfg);
  TP_REQUIRE(workspace_bytes >= L.total, "workspace too small (%zu < %zu)", workspace_bytes,
             L.total);
  const Tiles T = make_tiles(op, cfg->rows_per_tile);
  const int64_t nt = T.nt;
  TP_REQUIRE(nt < INT32_MAX, "too many tiles");
  KernelSet K;
  if (!get_kernels(cfg->inner_fp32, op->ld, cfg->group, cfg->use_graph_loop != 0, &K)) {
    set_error("no kernel for fp32=%d ld=%d group=%d", cfg->inner_fp32, op->ld, cfg->group);
    return TP_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  tp_cg_handle* h = new tp_cg_handle();
  h->vt_fp32 = cfg->inner_fp32;
  h->ld = op->ld;
  h->G = cfg->group;
  h->block = cfg->block;
  h->ntiles = (int)nt;
  h->NL = nsys * op->S;
  h->max_it = cfg->max_it;
  h->use_cond = cfg->use_graph_loop ? 1 : 0;
  int occ = 0;
  cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)K.b1,
                                                                 cfg->block, 0);
  if (oe != cudaSuccess || occ < 1) occ = 1;
  const int64_t cap = (int64_t)sm_count() * occ;
  // one tile per block up to 16 resident waves; beyond that blocks loop over tiles
  h->grid = (int)std::max<int64_t>(1, std::min<int64_t>(nt, 16 * cap));
  h->row_grid = (int)std::max<int64_t>(1, std::min<int64_t>((op->n_rows + cfg->block - 1) / cfg->block, cap));
  char* ws = static_cast<char*>(workspace);
  if (h->vt_fp32)
    fill_args(h->af, op, cfg, ws, L, nt, T.nch, b, x, rtol, h->use_cond);
  else
    fill_args(h->ad, op, cfg, ws, L, nt, T.nch, b, x, rtol, h->use_cond);
  Glob* gp = h->vt_fp32 ? h->af.g : h->ad.g;
  h->glob = gp;
  h->lanes = h->vt_fp32 ? h->af.L : h->ad.L;
  h->sys_active = h->vt_fp32 ? h->af.sys_active : h->ad.sys_active;
  Glob g0 = {};
  g0.max_it = cfg->max_it;
  const double delta = cfg->inner_fp32 ? (cfg->delta > 0 ? cfg->delta : 0.1) : 0.0;
  g0.delta2 = delta * delta;
  struct Copy {
    const void* dst;
    const void* src;
    size_t bytes;
  };
  const bool f = h->vt_fp32 != 0;
  const Copy copies[] = {
      {f ? (const void*)h->af.tile_row0 : (const void*)h->ad.tile_row0, T.row0.data(),
       sizeof(int64_t) * T.row0.size()},
      {f ? (const void*)h->af.tile_sys : (const void*)h->ad.tile_sys, T.tsys.data(),
       sizeof(int32_t) * T.tsys.size()},
      {f ? (const void*)h->af.sys_tile_ptr : (const void*)h->ad.sys_tile_ptr, T.sptr.data(),
       sizeof(int32_t) * T.sptr.size()},
      {f ? (const void*)h->af.tile_chunk : (const void*)h->ad.tile_chunk, T.tchunk.data(),
       sizeof(int32_t) * T.tchunk.size()},
      {f ? (const void*)h->af.chunk_tile_ptr : (const void*)h->ad.chunk_tile_ptr, T.cptr.data(),
       sizeof(int32_t) * T.cptr.size()},
      {f ? (const void*)h->af.sys_chunk_ptr : (const void*)h->ad.sys_chunk_ptr, T.schptr.data(),
       sizeof(int32_t) * T.schptr.size()},
  };
  uint32_t* d_tick = f ? h->af.sys_ticket : h->ad.sys_ticket;
  uint32_t* d_ctick = f ? h->af.chunk_ticket : h->ad.chunk_ticket;
  int rc = TP_OK;
  cudaError_t e = cudaMemcpyAsync(gp, &g0, sizeof(Glob), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d_tick, 0, sizeof(uint32_t) * N_KINDS * nsys, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d_ctick, 0, sizeof(uint32_t) * N_KINDS * std::max<int64_t>(T.nch, 1), st);
  for (const Copy& c : copies) {
    if (e != cudaSuccess) break;
    if (c.bytes) e = cudaMemcpyAsync((void*)c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error("cg setup copy failed: %s", cudaGetErrorString(e));
    delete h;
    return TP_ERR_CUDA;
  }
  void* arg = h->vt_fp32 ? (void*)&h->af : (void*)&h->ad;
  rc = build_graphs(h, K, arg);
  if (rc) {
    tp_cg_destroy(h);
    return rc;
  }
  *out = h;
  return TP_OK;
}

extern "C" int tp_cg_run(tp_cg_handle* h, void* stream) {
  TP_REQUIRE(h, "null handle");
  cudaStream_t st = as_stream(stream);
  if (h->use_cond) {
    TP_CUDA_TRY(cudaGraphLaunch(h->exec, st));
    return TP_OK;
  }
  TP_CUDA_TRY(cudaGraphLaunch(h->e_init, st));
  int cont = 1;
  int it = 0;
  const int chunk = 8;
  while (cont && it < h->max_it) {
    for (int k = 0; k < chunk && it < h->max_it; k++, it++)
      TP_CUDA_TRY(cudaGraphLaunch(h->e_iter, st));
    TP_CUDA_TRY(cudaMemcpyAsync(&cont, &h->glob->cont, sizeof(int), cudaMemcpyDeviceToHost, st));
    TP_CUDA_TRY(cudaStreamSynchronize(st));
  }
  TP_CUDA_TRY(cudaGraphLaunch(h->e_fin, st));
  return TP_OK;
}

extern "C" int tp_cg_result_get(tp_cg_handle* h, tp_cg_result* res, int32_t* lane_iters,
                                int32_t* lane_status, double* lane_rnorm, double* lane_bnorm,
                                void* stream) {
  TP_REQUIRE(h, "null handle");
  cudaStream_t st = as_stream(stream);
  Glob g;
  const int NL = h->NL;
  std::vector<int32_t> it(NL), stt(NL);
  std::vector<double> rt(NL), bb(NL);
  TP_CUDA_TRY(cudaMemcpyAsync(&g, h->glob, sizeof(Glob), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaMemcpyAsync(it.data(), h->lanes.iters, sizeof(int32_t) * NL,
                              cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaMemcpyAsync(stt.data(), h->lanes.status, sizeof(int32_t) * NL,
                              cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaMemcpyAsync(rt.data(), h->lanes.rtrue, sizeof(double) * NL,
                              cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaMemcpyAsync(bb.data(), h->lanes.bb, sizeof(double) * NL,
                              cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  int status = TP_OK, maxit = 0;
  for (int l = 0; l < NL; l++) {
    maxit = std::max(maxit, it[l]);
    if (stt[l] != TP_OK && status == TP_OK) status = stt[l] < 0 ? TP_ERR_NOT_CONVERGED : stt[l];
    if (lane_iters) lane_iters[l] = it[l];
    if (lane_status) lane_status[l] = stt[l];
    if (lane_rnorm) lane_rnorm[l] = sqrt(std::max(rt[l], 0.0));
    if (lane_bnorm) lane_bnorm[l] = sqrt(std::max(bb[l], 0.0));
  }
  if (res) {
    res->status = status;
    res->iterations = maxit;
    res->n_reliable = g.n_reliable;
    res->n_lanes = NL;
  }
  return TP_OK;
}

extern "C" int tp_cg_destroy(tp_cg_handle* h) {
  if (!h) return TP_OK;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->e_init) cudaGraphExecDestroy(h->e_init);
  if (h->e_iter) cudaGraphExecDestroy(h->e_iter);
  if (h->e_fin) cudaGraphExecDestroy(h->e_fin);
  if (h->g_init) cudaGraphDestroy(h->g_init);
  if (h->g_iter) cudaGraphDestroy(h->g_iter);
  if (h->g_fin) cudaGraphDestroy(h->g_fin);
  delete h;
  return TP_OK;
}

extern "C" int tp_cg_time_spmv(tp_cg_handle* h, int reps, float* ms, void* stream) {
  TP_REQUIRE(h && ms && reps > 0, "bad argument");
  cudaStream_t st = as_stream(stream);
  KernelSet K;
  if (!get_kernels(h->vt_fp32, h->ld, h->G, h->use_cond != 0, &K)) return TP_ERR_ARG;
  // timing mode: B1 processes every tile and leaves the lane state alone
  static const int32_t on = 1, off = 0;
  TP_CUDA_TRY(cudaMemcpyAsync(&h->glob->timing, &on, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  void* arg = h->vt_fp32 ? (void*)&h->af : (void*)&h->ad;
  void* args[1] = {arg};
  cudaEvent_t e0, e1;
  TP_CUDA_TRY(cudaEventCreate(&e0));
  TP_CUDA_TRY(cudaEventCreate(&e1));
  TP_CUDA_TRY(cudaLaunchKernel(K.b1, dim3(h->grid), dim3(h->block), args, 0, st));
  TP_CUDA_TRY(cudaEventRecord(e0, st));
  for (int i = 0; i < reps; i++)
    TP_CUDA_TRY(cudaLaunchKernel(K.b1, dim3(h->grid), dim3(h->block), args, 0, st));
  TP_CUDA_TRY(cudaEventRecord(e1, st));
  TP_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0;
  TP_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  TP_CUDA_TRY(cudaMemcpyAsync(&h->glob->timing, &off, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  *ms = t / reps;
  return TP_OK;
}
