// tp_apply.cu -- matrix-free operator apply and the standalone multi-column CSR apply.
//
// Matrix-free (replaces gpu/ceed_operators.py CeedDiffusionMassOp / DiffMassBilinear,
// :87-108, 247-353): one thread per cell gathers its 4 vertex coordinates with
// 32-byte loads, recomputes J, det J and the cofactor rows c_k = (J^-1 row k) det J in
// FP64, and applies, for every column s,
//     y_i += scale (c_i . w) + react M_e u,    w = sum_k (u_k - u_0) c_k
// with scale = De/(6|det J|) (exact P1 stiffness) or 4 De/det^2 (legacy: the reference
// QFunction drops wdetJ), and consistent (|det|/120 (1+d_ij)) or lumped (|det|/24) mass.
// Contributions land with hardware atomics (FP32 columns as one 16-byte vector atomic),
// so the result's last bits depend on arrival order, as in the reference.  A warp takes
// 32 consecutive cells.  Scalar atomics (FP64, FP32 rows narrower than 16 bytes) are
// grouped: for each local vertex slot, a run of consecutive lanes whose cells have the
// same vertex in that slot sums its contributions through shared memory and the run's
// first lane issues the atomics.  The six cells of a Kuhn cube share their first and last
// vertex (runs of six) and pairs of them their second (runs of two): 11 atomics per cube
// instead of 24; on any other ordering the runs are single lanes.  A 16-byte FP32 row
// goes out as one vector atomic per lane, where the grouping does not pay.
#include "tp_ops.cuh"

namespace tp {

// CS columns of LD are used (compile time, so the column loops carry no predicates).
template <typename T, int LD, int CS>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 3 : 4) k_matfree(
    int64_t n, const int4* __restrict__ cells, const double4* __restrict__ X,
    const double* __restrict__ De, const double* __restrict__ alpha, double4 dsc, double4 shf,
    double inv_dt, int lumped, int legacy, const T* __restrict__ x, T* __restrict__ y) {
  constexpr bool VEC = sizeof(T) == 4 && LD == 4;  // one 16-byte vector atomic per row
  constexpr int WPB = 256 / 32;
  __shared__ T s_val[VEC ? 1 : WPB][32][CS];  // one contribution per lane, for the run head
  const double dscale[4] = {dsc.x, dsc.y, dsc.z, dsc.w};
  const double shift[4] = {shf.x, shf.y, shf.z, shf.w};
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t wstride = (int64_t)gridDim.x * WPB * 32;
  // the loop trip count is uniform over the warp: lanes past n compute a copy of the
  // last cell and add nothing
  for (int64_t base = ((int64_t)blockIdx.x * WPB + wib) * 32; base < n; base += wstride) {
    const int64_t c0 = base + lane;
    const bool valid = c0 < n;
    const int64_t c = valid ? c0 : n - 1;
    const int4 v = cells[c];
    const double4 x0 = ldg_d4(X + v.x), x1 = ldg_d4(X + v.y), x2 = ldg_d4(X + v.z),
                  x3 = ldg_d4(X + v.w);
    T xv[4][LD];
    ldv<T, LD>(x, v.x, xv[0]);
    ldv<T, LD>(x, v.y, xv[1]);
    ldv<T, LD>(x, v.z, xv[2]);
    ldv<T, LD>(x, v.w, xv[3]);
    const double De_c = De[c];
    const double al = alpha ? alpha[c] : 0.0;
    const double e[3][3] = {{x1.x - x0.x, x1.y - x0.y, x1.z - x0.z},
                            {x2.x - x0.x, x2.y - x0.y, x2.z - x0.z},
                            {x3.x - x0.x, x3.y - x0.y, x3.z - x0.z}};
    double cr[3][3];  // cr[k] = row k of adj(J): e2 x e3, e3 x e1, e1 x e2
    cr[0][0] = e[1][1] * e[2][2] - e[1][2] * e[2][1];
    cr[0][1] = e[1][2] * e[2][0] - e[1][0] * e[2][2];
    cr[0][2] = e[1][0] * e[2][1] - e[1][1] * e[2][0];
    cr[1][0] = e[2][1] * e[0][2] - e[2][2] * e[0][1];
    cr[1][1] = e[2][2] * e[0][0] - e[2][0] * e[0][2];
    cr[1][2] = e[2][0] * e[0][1] - e[2][1] * e[0][0];
    cr[2][0] = e[0][1] * e[1][2] - e[0][2] * e[1][1];
    cr[2][1] = e[0][2] * e[1][0] - e[0][0] * e[1][2];
    cr[2][2] = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    const double det = e[0][0] * cr[0][0] + e[0][1] * cr[0][1] + e[0][2] * cr[0][2];
    const double adet = fabs(det);
    // one division: De/(6|det|), or 4 De/det^2 for the legacy QFunction
    const double kbase = legacy ? (4.0 * De_c) / (det * det) : De_c / (6.0 * adet);
    const double mbase = adet * (lumped ? 1.0 / 24.0 : 1.0 / 120.0);
    T c_[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) c_[a][b] = (T)cr[a][b];
    T out[4][CS];
#pragma unroll
    for (int s = 0; s < CS; s++) {
      const T ks = (T)(kbase * dscale[s]);
      const T ms = (T)(mbase * (inv_dt + al + shift[s]));
      const T d1 = xv[1][s] - xv[0][s], d2 = xv[2][s] - xv[0][s], d3 = xv[3][s] - xv[0][s];
      T w[3];
#pragma unroll
      for (int b = 0; b < 3; b++) w[b] = d1 * c_[0][b] + d2 * c_[1][b] + d3 * c_[2][b];
      T yk[4];
#pragma unroll
      for (int i = 1; i < 4; i++)
        yk[i] = ks * (c_[i - 1][0] * w[0] + c_[i - 1][1] * w[1] + c_[i - 1][2] * w[2]);
      yk[0] = -(yk[1] + yk[2] + yk[3]);
      if (lumped) {
#pragma unroll
        for (int i = 0; i < 4; i++) out[i][s] = yk[i] + ms * xv[i][s];
      } else {
        const T su = xv[0][s] + xv[1][s] + xv[2][s] + xv[3][s];
#pragma unroll
        for (int i = 0; i < 4; i++) out[i][s] = yk[i] + ms * (su + xv[i][s]);
      }
    }
    const int vid[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      T* dst = y + (int64_t)vid[i] * LD;
      if constexpr (VEC) {
        if (valid) {
          float4 o;
          o.x = out[i][0];
          o.y = CS > 1 ? out[i][CS > 1 ? 1 : 0] : 0.f;
          o.z = CS > 2 ? out[i][CS > 2 ? 2 : 0] : 0.f;
          o.w = CS > 3 ? out[i][CS > 3 ? 3 : 0] : 0.f;
          atomicAdd(reinterpret_cast<float4*>(dst), o);
        }
        continue;
      }
      // vertex ids are >= 0, so the keys of lanes past n are unique (runs of one)
      const int key = valid ? vid[i] : -1 - lane;
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      const bool head = lane == 0 || prev != key;
      const unsigned above = (__ballot_sync(0xffffffffu, head) >> lane) >> 1;
      const int end = above ? lane + __ffs(above) : 32;  // run = lanes [lane, end)
      if (!head) {
#pragma unroll
        for (int s = 0; s < CS; s++) s_val[wib][lane][s] = out[i][s];
      }
      __syncwarp();
      if (head && valid) {
        T acc[CS];
#pragma unroll
        for (int s = 0; s < CS; s++) acc[s] = out[i][s];
        for (int l = lane + 1; l < end; l++) {
#pragma unroll
          for (int s = 0; s < CS; s++) acc[s] += s_val[wib][l][s];
        }
#pragma unroll
        for (int s = 0; s < CS; s++) atomicAdd(dst + s, acc[s]);
      }
      __syncwarp();
    }
  }
}

template <typename T, int LD, int G>
__global__ void __launch_bounds__(256) k_csr_apply(int64_t n, CsrView<T> A,
                                                   const T* __restrict__ x, T* __restrict__ y) {
  const int gl = threadIdx.x % G;
  const int64_t rpb = blockDim.x / G;
  for (int64_t base = blockIdx.x * rpb; base < n; base += (int64_t)gridDim.x * rpb) {
    const int64_t row = base + threadIdx.x / G;
    const int64_t rr = row < n ? row : n - 1;
    T out[LD];
    csr_row<T, LD, G, true>(A, rr, gl, x, out);
    if (row < n && gl == 0) stv<T, LD>(y, row, out);
  }
}

// y1 = D K x1 and y2 = D K (x1 - x2) in one pass over the CSR operator (no mass, no
// diagonal, no identity rows): the stiffness images of u^n and of the last increment.
// G lanes per row, FP64.  W256: 4-column rows of x1 and x2 are gathered with one 256-bit
// load each (both bases 32-byte aligned, checked by the caller).
template <int LD, int G, bool W256 = false>
__global__ void __launch_bounds__(256) k_csr_images(int64_t n, const int32_t* __restrict__ indptr,
                                                    const int32_t* __restrict__ indices,
                                                    const double* __restrict__ K, double4 dsc,
                                                    const double* __restrict__ x1,
                                                    const double* __restrict__ x2,
                                                    double* __restrict__ y1,
                                                    double* __restrict__ y2) {
  const double dscale[4] = {dsc.x, dsc.y, dsc.z, dsc.w};
  const int gl = threadIdx.x % G;
  const int64_t rpb = blockDim.x / G;
  for (int64_t base = blockIdx.x * rpb; base < n; base += (int64_t)gridDim.x * rpb) {
    const int64_t row = base + threadIdx.x / G;
    const int64_t rr = row < n ? row : n - 1;
    double a1[LD], a2[LD];
#pragma unroll
    for (int s = 0; s < LD; s++) a1[s] = a2[s] = 0.0;
    const int beg = indptr[rr], end = indptr[rr + 1];
    // the index and value loads of up to RP entries per lane in flight before their gathers
    constexpr int RP = 4;
    for (int p0 = beg + gl; p0 < end; p0 += G * RP) {
      int jj[RP];
      double kv[RP];
#pragma unroll
      for (int v = 0; v < RP; v++) {
        const int p = p0 + v * G;
        jj[v] = p < end ? __ldg(indices + p) : 0;
        kv[v] = p < end ? __ldg(K + p) : 0.0;
      }
#pragma unroll
      for (int v = 0; v < RP; v++) {
        if (p0 + v * G >= end) break;
        double u[LD], up[LD];
        if constexpr (W256 && LD == 4) {
          const double4 a = ldg_d4(reinterpret_cast<const double4*>(x1) + jj[v]);
          const double4 c = ldg_d4(reinterpret_cast<const double4*>(x2) + jj[v]);
          u[0] = a.x, u[1] = a.y, u[2] = a.z, u[3] = a.w;
          up[0] = c.x, up[1] = c.y, up[2] = c.z, up[3] = c.w;
        } else {
          ldv<double, LD>(x1, jj[v], u);
          ldv<double, LD>(x2, jj[v], up);
        }
#pragma unroll
        for (int s = 0; s < LD; s++) {
          a1[s] += kv[v] * u[s];
          a2[s] += kv[v] * (u[s] - up[s]);
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
#pragma unroll
      for (int s = 0; s < LD; s++) {
        a1[s] += __shfl_xor_sync(0xffffffffu, a1[s], o, G);
        a2[s] += __shfl_xor_sync(0xffffffffu, a2[s], o, G);
      }
    }
    if (row < n && gl == 0) {
      double o1[LD], o2[LD];
#pragma unroll
      for (int s = 0; s < LD; s++) {
        o1[s] = dscale[s] * a1[s];
        o2[s] = dscale[s] * a2[s];
      }
      stv<double, LD>(y1, row, o1);
      stv<double, LD>(y2, row, o2);
    }
  }
}

// ---------------------------------------------------------------- guess projection
// The initial guess projected in the energy norm.  With A = D K + diag (identity rows
// where bc), u = u^n and M <= GP_MAXD directions d_k (increments of past steps, the
// network's correction), the guess is x = u + sum_k c_k d_k on the free rows, c per column
// from the Galerkin system  G c = h,  G_kl = d_k . A d_l,  h_k = d_k . (b - A u),  which
// minimises the A-norm of the error over u + span{d_k}: the guess is never worse than u^n
// in that norm.  Sums run over the free rows; every direction is taken as zero on the
// Dirichlet rows, which keep x = b.
constexpr int GP_MAXD = 6;
constexpr int GP_BLOCKS = 592;

struct GuessDirs {
  const double* d[GP_MAXD];
  const double* img[GP_MAXD];  // D K d[k] precomputed (no Dirichlet rows), or NULL
};

template <int M>
__host__ __device__ constexpr int gp_nq() {
  return M * (M + 1) / 2 + M;  // upper triangle of G, then h
}
constexpr int GP_SLOTS = gp_nq<GP_MAXD>() * 4;

// A d_k for the first NG directions by one CSR walk per row (the others come with their
// images d.img[k]).  A group of LD lanes per row; lane s feeds column s.  With NG <= 2 the
// group walks the row together: lane s takes entries s, s + LD, ... and gathers whole
// LD-column rows of the directions, the index and value loads of up to 4 LD entries in
// flight before their gathers, and a shuffle tree over the group gives every column's sum.
// With more gathered directions each lane walks the whole row for its own column.  One row
// of GP_SLOTS partials per block (slot q * 4 + s), summed over the warps in a fixed order.
template <int LD, int M, int NG>
__global__ void __launch_bounds__(256) k_guess_dots(
    int64_t n, int S, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
    const double* __restrict__ K, double4 dsc, const double* __restrict__ diag,
    const uint8_t* __restrict__ bc, const double* __restrict__ b, const double* __restrict__ U,
    const double* __restrict__ opU, GuessDirs dirs, double* __restrict__ part) {
  constexpr int NQ = gp_nq<M>();
  constexpr bool COOP = NG >= 1 && NG <= 2;
  constexpr int NGA = NG > 0 ? NG : 1;
  __shared__ double red[8][NQ * 4];  // blockDim 256: 8 warps
  const double dscale[4] = {dsc.x, dsc.y, dsc.z, dsc.w};
  const int s = threadIdx.x % LD;
  double dsc_s = dscale[0];
#pragma unroll
  for (int c = 1; c < LD; c++)
    if (c == s) dsc_s = dscale[c];
  const int64_t rpb = blockDim.x / LD;
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  for (int64_t base = blockIdx.x * rpb; base < n; base += (int64_t)gridDim.x * rpb) {
    const int64_t row = base + threadIdx.x / LD;
    // the same in every lane of the row's group (the group's shuffles need all of it)
    const bool live = row < n && !(bc && bc[row]);
    const bool act = live && s < S;
    if (!COOP && !act) continue;
    // the row's vector entries first: they do not depend on the CSR walk, so their loads
    // are in flight during it
    const int64_t i = (live ? row : 0) * LD + s;
    double u = 0.0, dg = 0.0, bi = 0.0, ou = 0.0, dv[M], im[M];
#pragma unroll
    for (int k = 0; k < M; k++) dv[k] = im[k] = 0.0;
    if (act) {
      u = U[i], dg = diag[i], bi = b[i], ou = opU[i];
#pragma unroll
      for (int k = 0; k < M; k++) {
        dv[k] = dirs.d[k][i];
        im[k] = k < NG ? 0.0 : dirs.img[k][i];
      }
    }
    double kd[NGA];
#pragma unroll
    for (int k = 0; k < NGA; k++) kd[k] = 0.0;
    if constexpr (COOP) {
      double kg[NGA][LD];
#pragma unroll
      for (int k = 0; k < NGA; k++)
#pragma unroll
        for (int c = 0; c < LD; c++) kg[k][c] = 0.0;
      if (live) {
        const int beg = indptr[row], end = indptr[row + 1];
        constexpr int RP = 4;
        for (int p0 = beg; p0 < end; p0 += LD * RP) {
          int jj[RP];
          double kv[RP];
#pragma unroll
          for (int v = 0; v < RP; v++) {
            const int p = p0 + s + v * LD;
            const bool in = p < end;
            jj[v] = in ? __ldg(indices + p) : 0;
            kv[v] = (in && !(bc && bc[jj[v]])) ? __ldg(K + p) : 0.0;
          }
#pragma unroll
          for (int v = 0; v < RP; v++) {
            if (p0 + s + v * LD < end) {
#pragma unroll
              for (int k = 0; k < NGA; k++) {
                double g[LD];
                ldv<double, LD>(dirs.d[k], jj[v], g);
#pragma unroll
                for (int c = 0; c < LD; c++) kg[k][c] += kv[v] * g[c];
              }
            }
          }
        }
      }
#pragma unroll
      for (int o = 1; o < LD; o <<= 1)
#pragma unroll
        for (int k = 0; k < NGA; k++)
#pragma unroll
          for (int c = 0; c < LD; c++) kg[k][c] += __shfl_xor_sync(0xffffffffu, kg[k][c], o);
      if (!act) continue;
#pragma unroll
      for (int k = 0; k < NGA; k++)
#pragma unroll
        for (int c = 0; c < LD; c++)
          if (c == s) kd[k] = kg[k][c];
    } else {
      const int beg = indptr[row], end = indptr[row + 1];
      // four entries at a time: their index, value and gathers in flight together; the
      // sums still run entry by entry in CSR order
      constexpr int RP = 4;
      for (int p0 = beg; p0 < end; p0 += RP) {
        int64_t jj[RP];
        double kv[RP], dvv[RP][NGA];
#pragma unroll
        for (int v = 0; v < RP; v++) {
          const bool in = p0 + v < end;
          const int j = in ? __ldg(indices + p0 + v) : 0;
          kv[v] = (in && !(bc && bc[j])) ? __ldg(K + p0 + v) : 0.0;
          jj[v] = (int64_t)j * LD + s;
        }
#pragma unroll
        for (int v = 0; v < RP; v++)
#pragma unroll
          for (int k = 0; k < NG; k++) dvv[v][k] = __ldg(dirs.d[k] + jj[v]);
#pragma unroll
        for (int v = 0; v < RP; v++) {
          if (p0 + v >= end) break;
#pragma unroll
          for (int k = 0; k < NG; k++) kd[k] += kv[v] * dvv[v][k];
        }
      }
    }
    const double r0 = bi - (ou + dg * u);
    double Ad[M];
#pragma unroll
    for (int k = 0; k < M; k++) Ad[k] = (k < NG ? dsc_s * kd[k < NG ? k : 0] : im[k]) + dg * dv[k];
    int q = 0;
#pragma unroll
    for (int k = 0; k < M; k++)
#pragma unroll
      for (int l = k; l < M; l++) acc[q++] += dv[k] * Ad[l];
#pragma unroll
    for (int k = 0; k < M; k++) acc[q++] += dv[k] * r0;
  }
  // lanes of one column within the warp, then the warps in order
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    double v = acc[q];
#pragma unroll
    for (int o = LD; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < 4) red[w][q * 4 + lane] = (lane < LD) ? v : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NQ * 4; k += blockDim.x) {
    double v = 0.0;
    for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) v += red[ww][k];
    part[(int64_t)blockIdx.x * GP_SLOTS + k] = v;
  }
}

// One block: the sums over the partial rows in a fixed order, then per column the M x M
// solve by a Cholesky factorisation that drops a direction whose pivot falls below 1e-12
// of its diagonal (numerically in the span of the earlier ones): coef[s * GP_MAXD + k].
template <int M>
__global__ void __launch_bounds__(1024) k_guess_coeffs(int nparts, int S,
                                                       const double* __restrict__ part,
                                                       double* __restrict__ coef) {
  constexpr int NQ = gp_nq<M>();
  __shared__ double tot[NQ * 4];
  // warp w sums slots w, w + 32, ...: lane l adds partial rows l, l + 32, ... (all loads
  // in flight together), then a fixed shuffle tree
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = w; k < NQ * 4; k += nw) {
    constexpr int QN = (GP_BLOCKS + 31) / 32;
    double xq[QN];
#pragma unroll
    for (int q = 0; q < QN; q++) {
      const int bl = lane + 32 * q;
      xq[q] = (bl < nparts) ? part[(int64_t)bl * GP_SLOTS + k] : 0.0;
    }
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < QN; q++) v += xq[q];
    v = warp_sum(v);
    if (lane == 0) tot[k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int s = threadIdx.x;
    double c[M];
#pragma unroll
    for (int k = 0; k < M; k++) c[k] = 0.0;
    if (s < S) {
      double Gm[M][M], h[M], L[M][M];
      int q = 0;
#pragma unroll
      for (int k = 0; k < M; k++)
#pragma unroll
        for (int l = k; l < M; l++) {
          Gm[k][l] = tot[q * 4 + s];
          Gm[l][k] = Gm[k][l];
          q++;
        }
#pragma unroll
      for (int k = 0; k < M; k++) h[k] = tot[(q + k) * 4 + s];
      bool keep[M];
#pragma unroll
      for (int k = 0; k < M; k++) {
        double p = Gm[k][k];
#pragma unroll
        for (int j = 0; j < k; j++) p -= L[k][j] * L[k][j];
        keep[k] = Gm[k][k] > 0.0 && p > 1e-12 * Gm[k][k] && isfinite(p);
        const double lk = keep[k] ? sqrt(p) : 0.0;
        L[k][k] = lk;
#pragma unroll
        for (int i = k + 1; i < M; i++) {
          double v = Gm[i][k];
#pragma unroll
          for (int j = 0; j < k; j++) v -= L[i][j] * L[k][j];
          L[i][k] = keep[k] ? v / lk : 0.0;
        }
      }
      double y[M];
#pragma unroll
      for (int k = 0; k < M; k++) {
        double v = h[k];
#pragma unroll
        for (int j = 0; j < k; j++) v -= L[k][j] * y[j];
        y[k] = keep[k] ? v / L[k][k] : 0.0;
      }
#pragma unroll
      for (int k = M - 1; k >= 0; k--) {
        double v = y[k];
#pragma unroll
        for (int j = k + 1; j < M; j++) v -= L[j][k] * c[j];
        c[k] = keep[k] ? v / L[k][k] : 0.0;
      }
      bool fin = true;
#pragma unroll
      for (int k = 0; k < M; k++) fin = fin && isfinite(c[k]);
      if (!fin)
#pragma unroll
        for (int k = 0; k < M; k++) c[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < M; k++) coef[s * GP_MAXD + k] = c[k];
  }
}

template <int LD, int M>
__global__ void k_guess_update(int64_t n, int S, const double* __restrict__ coef,
                               const uint8_t* __restrict__ bc, const double* __restrict__ b,
                               const double* __restrict__ U, GuessDirs dirs,
                               double* __restrict__ x) {
  __shared__ double cs[4 * GP_MAXD];
  if (threadIdx.x < 4 * GP_MAXD) cs[threadIdx.x] = coef[threadIdx.x];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * LD;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / LD;
    const int s = (int)(i - row * LD);
    double v = U[i];
    if (bc && bc[row]) {
      v = (s < S) ? b[i] : v;
    } else if (s < S) {
#pragma unroll
      for (int k = 0; k < M; k++) v += cs[s * GP_MAXD + k] * dirs.d[k][i];
    }
    x[i] = v;
  }
}

template <typename T, int LD, int CS>
static void launch_matfree_cs(const tp_mesh* m, const double* De, const double* al, double4 dsc,
                              double4 shf, double inv_dt, int lumped, int legacy, const void* x,
                              void* y, cudaStream_t st) {
  const int grid = grid_for(m->n_cells, 256, sm_count() * 8);
  k_matfree<T, LD, CS><<<grid, 256, 0, st>>>(
      m->n_cells, reinterpret_cast<const int4*>(m->cells),
      reinterpret_cast<const double4*>(m->coords4), De, al, dsc, shf, inv_dt, lumped, legacy,
      static_cast<const T*>(x), static_cast<T*>(y));
}

template <typename T>
static int launch_matfree(const tp_mesh* m, int S, int ld, const double* De, const double* al,
                          double4 dsc, double4 shf, double inv_dt, int lumped, int legacy,
                          const void* x, void* y, cudaStream_t st) {
#define TP_MF(LD_, CS_) \
  launch_matfree_cs<T, LD_, CS_>(m, De, al, dsc, shf, inv_dt, lumped, legacy, x, y, st)
  if (ld == 1) {
    TP_MF(1, 1);
  } else if (ld == 2) {
    if (S == 1) TP_MF(2, 1); else TP_MF(2, 2);
  } else if (ld == 4) {
    if (S == 1) TP_MF(4, 1);
    else if (S == 2) TP_MF(4, 2);
    else if (S == 3) TP_MF(4, 3);
    else TP_MF(4, 4);
  } else {
    set_error("ld must be 1, 2 or 4");
    return TP_ERR_ARG;
  }
#undef TP_MF
  TP_LAUNCH_CHECK();
  return TP_OK;
}

template <typename T>
static CsrView<T> make_view(const tp_csr_op* op, bool fp32) {
  CsrView<T> v;
  v.indptr = op->indptr;
  v.indices = op->indices;
  if constexpr (sizeof(T) == 4) {
    v.K = op->K32;
    v.M = op->M32;
    v.diag = op->diag32;
  } else {
    v.K = op->K64;
    v.M = op->M64;
    v.diag = op->diag64;
  }
  (void)fp32;
  v.bc = op->bc_mask;
  for (int s = 0; s < 4; s++) {
    v.dscale[s] = s < op->S ? op->dscale[s] : 0.0;
    v.cscale[s] = s < op->S ? op->cscale[s] : 0.0;
  }
  return v;
}

template <typename T, int LD>
static void launch_csr(const tp_csr_op* op, const void* x, void* y, cudaStream_t st) {
  constexpr int G = 4;
  const int64_t n = op->n_rows;
  const int grid = grid_for(n * G, 256, sm_count() * 8);
  k_csr_apply<T, LD, G><<<grid, 256, 0, st>>>(n, make_view<T>(op, sizeof(T) == 4),
                                              static_cast<const T*>(x), static_cast<T*>(y));
}

}  // namespace tp

using namespace tp;

extern "C" int tp_matfree_apply(const tp_mesh* m, int S, int ld, int fp32, const double* De_cell,
                                const double* alpha_cell, const double* diff_scale,
                                const double* shift, double inv_dt, int lumped, int legacy,
                                const void* x, void* y, void* stream) {
  TP_REQUIRE(m && m->cells && m->coords4 && De_cell && x && y, "null pointer");
  TP_REQUIRE((reinterpret_cast<uintptr_t>(m->coords4) & 31) == 0, "coords4 not 32-byte aligned");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && (ld == 1 || ld == 2 || ld == 4) && ld >= S,
             "bad S/ld");
  cudaStream_t st = as_stream(stream);
  const size_t esz = fp32 ? 4 : 8;
  TP_CUDA_TRY(cudaMemsetAsync(y, 0, esz * ld * (size_t)m->n_verts, st));
  if (m->n_cells == 0) return TP_OK;
  double d[4] = {1, 1, 1, 1}, s[4] = {0, 0, 0, 0};
  for (int i = 0; i < S; i++) {
    if (diff_scale) d[i] = diff_scale[i];
    if (shift) s[i] = shift[i];
  }
  const double4 dsc = make_double4(d[0], d[1], d[2], d[3]);
  const double4 shf = make_double4(s[0], s[1], s[2], s[3]);
  if (fp32)
    return launch_matfree<float>(m, S, ld, De_cell, alpha_cell, dsc, shf, inv_dt, lumped, legacy,
                                 x, y, st);
  return launch_matfree<double>(m, S, ld, De_cell, alpha_cell, dsc, shf, inv_dt, lumped, legacy,
                                x, y, st);
}

extern "C" int tp_csr_apply(const tp_csr_op* op, int fp32, const void* x, void* y, void* stream) {
  TP_REQUIRE(op && op->indptr && op->indices && x && y, "null pointer");
  TP_REQUIRE(fp32 ? (op->K32 != nullptr) : (op->K64 != nullptr), "operator values missing");
  TP_REQUIRE(op->ld == 1 || op->ld == 2 || op->ld == 4, "ld must be 1, 2 or 4");
  if (op->n_rows == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  if (fp32) {
    if (op->ld == 1) launch_csr<float, 1>(op, x, y, st);
    else if (op->ld == 2) launch_csr<float, 2>(op, x, y, st);
    else launch_csr<float, 4>(op, x, y, st);
  } else {
    if (op->ld == 1) launch_csr<double, 1>(op, x, y, st);
    else if (op->ld == 2) launch_csr<double, 2>(op, x, y, st);
    else launch_csr<double, 4>(op, x, y, st);
  }
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_csr_images(const tp_csr_op* op, const double* x1, const double* x2,
                             double* y1, double* y2, void* stream) {
  TP_REQUIRE(op && op->indptr && op->indices && op->K64 && x1 && x2 && y1 && y2,
             "null pointer");
  TP_REQUIRE(op->ld == 1 || op->ld == 2 || op->ld == 4, "ld must be 1, 2 or 4");
  if (op->n_rows == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  constexpr int G = 4;
  const int grid = grid_for(op->n_rows, 256 / G, sm_count() * 16);
  const double4 dsc = make_double4(op->S > 0 ? op->dscale[0] : 0.0, op->S > 1 ? op->dscale[1] : 0.0,
                                   op->S > 2 ? op->dscale[2] : 0.0, op->S > 3 ? op->dscale[3] : 0.0);
  if (op->ld == 1)
    k_csr_images<1, G><<<grid, 256, 0, st>>>(op->n_rows, op->indptr, op->indices, op->K64, dsc,
                                             x1, x2, y1, y2);
  else if (op->ld == 2)
    k_csr_images<2, G><<<grid, 256, 0, st>>>(op->n_rows, op->indptr, op->indices, op->K64, dsc,
                                             x1, x2, y1, y2);
  else if (((reinterpret_cast<uintptr_t>(x1) | reinterpret_cast<uintptr_t>(x2)) & 31) == 0)
    k_csr_images<4, G, true><<<grid, 256, 0, st>>>(op->n_rows, op->indptr, op->indices, op->K64,
                                                   dsc, x1, x2, y1, y2);
  else
    k_csr_images<4, G><<<grid, 256, 0, st>>>(op->n_rows, op->indptr, op->indices, op->K64, dsc,
                                             x1, x2, y1, y2);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" size_t tp_guess_project_workspace_doubles(void) {
  return (size_t)GP_BLOCKS * GP_SLOTS + 4 * GP_MAXD;
}

extern "C" int tp_guess_project(const tp_csr_op* op, const double* diag, const uint8_t* bc_mask,
                                const double* b, const double* U, const double* opU,
                                int n_dirs, const double* const* dirs,
                                const double* const* imgs, double* x, double* work,
                                void* stream) {
  TP_REQUIRE(op && op->indptr && op->indices && op->K64 && diag && b && U && opU && x && work,
             "null pointer");
  TP_REQUIRE(op->ld == 1 || op->ld == 2 || op->ld == 4, "ld must be 1, 2 or 4");
  TP_REQUIRE(op->S >= 1 && op->S <= op->ld, "bad S");
  TP_REQUIRE(n_dirs >= 0 && n_dirs <= GP_MAXD && (n_dirs == 0 || dirs), "0 to 6 directions");
  for (int k = 0; k < n_dirs; k++) TP_REQUIRE(dirs[k], "null direction");
  // directions without an image first (gathered), then those with one; other counts of
  // gathered directions than 1, 2 or all gather everything
  int ng = n_dirs;
  bool split = false;
  if (imgs && !bc_mask) {
    int cnt = 0;
    for (int k = 0; k < n_dirs; k++) cnt += imgs[k] ? 0 : 1;
    split = (cnt == 1 || cnt == 2) && cnt < n_dirs;
    if (split) ng = cnt;
  }
  GuessDirs gd{};
  {
    int q = 0;
    for (int k = 0; k < n_dirs; k++)
      if (!split || !imgs[k]) gd.d[q++] = dirs[k];
    if (split)
      for (int k = 0; k < n_dirs; k++)
        if (imgs[k]) {
          gd.img[q] = imgs[k];
          gd.d[q++] = dirs[k];
        }
  }
  if (op->n_rows == 0) return TP_OK;
  cudaStream_t st = as_stream(stream);
  if (n_dirs == 0) {
    TP_CUDA_TRY(cudaMemcpyAsync(x, U, sizeof(double) * op->n_rows * op->ld,
                                cudaMemcpyDeviceToDevice, st));
    return TP_OK;
  }
  const double4 dsc = make_double4(op->S > 0 ? op->dscale[0] : 0.0, op->S > 1 ? op->dscale[1] : 0.0,
                                   op->S > 2 ? op->dscale[2] : 0.0, op->S > 3 ? op->dscale[3] : 0.0);
  const int64_t n = op->n_rows;
  double* part = work;
  double* coef = work + (size_t)GP_BLOCKS * GP_SLOTS;
#define TP_GP(LDV, MV)                                                                       \
  do {                                                                                       \
    const int nb = (int)std::min<int64_t>(GP_BLOCKS / 2, (n + 256 / LDV - 1) / (256 / LDV)); \
    if (ng == 1)                                                                             \
      k_guess_dots<LDV, MV, (MV < 1 ? MV : 1)><<<nb, 256, 0, st>>>(                          \
          n, op->S, op->indptr, op->indices, op->K64, dsc, diag, bc_mask, b, U, opU, gd, part); \
    else if (ng == 2)                                                                        \
      k_guess_dots<LDV, MV, (MV < 2 ? MV : 2)><<<nb, 256, 0, st>>>(                          \
          n, op->S, op->indptr, op->indices, op->K64, dsc, diag, bc_mask, b, U, opU, gd, part); \
    else                                                                                     \
      k_guess_dots<LDV, MV, MV><<<nb, 256, 0, st>>>(n, op->S, op->indptr, op->indices,       \
                                                    op->K64, dsc, diag, bc_mask, b, U, opU,  \
                                                    gd, part);                               \
    k_guess_coeffs<MV><<<1, 1024, 0, st>>>(nb, op->S, part, coef);                           \
    k_guess_update<LDV, MV><<<grid_for(n * LDV, 256, sm_count() * 8), 256, 0, st>>>(         \
        n, op->S, coef, bc_mask, b, U, gd, x);                                               \
  } while (0)
#define TP_GP_M(LDV)                 \
  do {                               \
    switch (n_dirs) {                \
      case 1: TP_GP(LDV, 1); break;  \
      case 2: TP_GP(LDV, 2); break;  \
      case 3: TP_GP(LDV, 3); break;  \
      case 4: TP_GP(LDV, 4); break;  \
      case 5: TP_GP(LDV, 5); break;  \
      default: TP_GP(LDV, 6); break; \
    }                                \
  } while (0)
  if (op->ld == 1)
    TP_GP_M(1);
  else if (op->ld == 2)
    TP_GP_M(2);
  else
    TP_GP_M(4);
#undef TP_GP_M
#undef TP_GP
  TP_LAUNCH_CHECK();
  return TP_OK;
}

// ================================================================= matrix-free Krylov solve
// Jacobi-preconditioned CG whose product is the matrix-free apply above (k_matfree): the
// operator is never assembled, every product recomputes the P1 gradients from the
// coordinates.  This is the solve of the reference's MatShell branch
// (numerics/solvers.py:172-203, 375-404: PETSc KSP around CeedDiffusionMassOp) on the GPU.
// FP64, S columns of LD; Dirichlet rows are identity rows (x = b there, the
// preconditioner zero), as in the CSR engines.  Reductions are one FP64 partial per block
// summed in block order by the last block to finish (atomic ticket): deterministic for a
// given grid.
namespace tp {

struct MfState {
  double rz[4], alpha[4], beta[4], rr[4], bb[4], tol2[4], rtrue[4];
  int32_t active[4], iters[4], status[4];
  int32_t it, max_it, done, pad;
  uint32_t ticket;
};

constexpr int MF_BLOCK = 256;

// The operator's diagonal, per cell from the same arithmetic as k_matfree: stiffness
// ks |c_{i-1}|^2 (|c_0 + c_1 + c_2|^2 for local vertex 0), mass ms (lumped) or 2 ms.
template <int LD>
__global__ void __launch_bounds__(256) k_mf_diag(int64_t n, const int4* __restrict__ cells,
                                                 const double4* __restrict__ X,
                                                 const double* __restrict__ De,
                                                 const double* __restrict__ alpha, double4 dsc,
                                                 double4 shf, double inv_dt, int lumped,
                                                 int legacy, int S, double* __restrict__ diag) {
  const double dscale[4] = {dsc.x, dsc.y, dsc.z, dsc.w};
  const double shift[4] = {shf.x, shf.y, shf.z, shf.w};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const double4 x0 = ldg_d4(X + v.x), x1 = ldg_d4(X + v.y), x2 = ldg_d4(X + v.z),
                  x3 = ldg_d4(X + v.w);
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
    const double det = e[0][0] * cr[0][0] + e[0][1] * cr[0][1] + e[0][2] * cr[0][2];
    const double adet = fabs(det);
    const double De_c = De[c];
    const double al = alpha ? alpha[c] : 0.0;
    const double kbase = legacy ? (4.0 * De_c) / (det * det) : De_c / (6.0 * adet);
    const double mbase = adet * (lumped ? 1.0 / 24.0 : 1.0 / 120.0);
    double kd[4];
    const double g[3] = {cr[0][0] + cr[1][0] + cr[2][0], cr[0][1] + cr[1][1] + cr[2][1],
                         cr[0][2] + cr[1][2] + cr[2][2]};
    kd[0] = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
#pragma unroll
    for (int i = 1; i < 4; i++)
      kd[i] = cr[i - 1][0] * cr[i - 1][0] + cr[i - 1][1] * cr[i - 1][1] +
              cr[i - 1][2] * cr[i - 1][2];
    const int vid[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int s = 0; s < 4; s++) {
      if (s >= S) break;
      const double ks = kbase * dscale[s];
      const double ms = mbase * (inv_dt + al + shift[s]);
      const double md = lumped ? ms : 2.0 * ms;
#pragma unroll
      for (int i = 0; i < 4; i++) atomicAdd(diag + (int64_t)vid[i] * LD + s, ks * kd[i] + md);
    }
  }
}

// per-block partial sums of NQ quantities, then the last block sums them: thread t adds
// the partials of blocks t, t + blockDim, ... and a fixed block tree sums the threads (the
// same order on every run; one round trip for the partials instead of one per block)
template <int NQ>
__device__ __forceinline__ bool mf_reduce(double v[NQ], double* part, uint32_t* ticket,
                                          double out[NQ]) {
  __shared__ double sh[32];
  __shared__ bool s_last;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    const double t = block_sum(v[q], sh);
    if (threadIdx.x == 0) part[blockIdx.x * 16 + q] = t;
  }
  __threadfence();
  if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NQ; q++) acc[q] += __ldcg(part + b * 16 + q);
  }
#pragma unroll
  for (int q = 0; q < NQ; q++) out[q] = block_sum(acc[q], sh);
  if (threadIdx.x == 0) *ticket = 0;
  return true;
}

#define MF_ROWS for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; \
                     i += (int64_t)gridDim.x * blockDim.x)

// dinv = 1 / diag on free rows (0 on Dirichlet rows and zero diagonals); x = b on
// Dirichlet rows
template <int LD>
__global__ void k_mf_prep(int64_t n, int S, const uint8_t* __restrict__ bc,
                          const double* __restrict__ b, double* __restrict__ x,
                          double* __restrict__ dinv) {
  MF_ROWS {
    const bool br = bc && bc[i];
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const double d = dinv[i * LD + s];
      dinv[i * LD + s] = (br || s >= S || d == 0.0) ? 0.0 : 1.0 / d;
      if (br && s < S) x[i * LD + s] = b[i * LD + s];
    }
  }
}

// r = b - q (q = A x; r = 0 on Dirichlet rows), z = D^-1 r, p = z; r.z, r.r, b.b
template <int LD>
__global__ void __launch_bounds__(MF_BLOCK) k_mf_start(int64_t n, int S, const uint8_t* bc,
                                                       const double* b, const double* q,
                                                       const double* dinv, double* r,
                                                       double* z, double* p, double* part,
                                                       MfState* st, double4 rtol) {
  double acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = 0.0;
  MF_ROWS {
    const bool br = bc && bc[i];
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const int64_t k = i * LD + s;
      const double bv = (s < S) ? b[k] : 0.0;
      const double rv = (br || s >= S) ? 0.0 : bv - q[k];
      const double zv = dinv[k] * rv;
      r[k] = rv;
      z[k] = zv;
      p[k] = zv;
      acc[s] += rv * zv;
      acc[4 + s] += rv * rv;
      acc[8 + s] += bv * bv;
    }
  }
  double tot[12];
  if (!mf_reduce<12>(acc, part, &st->ticket, tot) || threadIdx.x != 0) return;
  const double rt[4] = {rtol.x, rtol.y, rtol.z, rtol.w};
  for (int s = 0; s < 4; s++) {
    st->rz[s] = tot[s];
    st->rr[s] = tot[4 + s];
    st->bb[s] = tot[8 + s];
    st->tol2[s] = rt[s] * rt[s] * tot[8 + s];
    st->alpha[s] = st->beta[s] = 0.0;
    st->iters[s] = 0;
    const bool fin = isfinite(tot[s]) && isfinite(tot[4 + s]);
    const bool act = s < S && fin && tot[4 + s] > st->tol2[s];
    st->active[s] = act;
    st->status[s] = (s < S && !fin) ? TP_ERR_NONFINITE : (act ? -1 : TP_OK);
  }
  st->it = 0;
  st->done = 0;
  for (int s = 0; s < S; s++) st->done |= st->active[s];
  st->done = !st->done;
}

// q = A p with Dirichlet rows as identity rows (p = 0 there); p.q -> alpha
template <int LD>
__global__ void __launch_bounds__(MF_BLOCK) k_mf_alpha(int64_t n, int S, const uint8_t* bc,
                                                       const double* p, double* q,
                                                       double* part, MfState* st) {
  if (st->done) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  MF_ROWS {
    const bool br = bc && bc[i];
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const int64_t k = i * LD + s;
      const double qv = br ? p[k] : q[k];
      if (br) q[k] = qv;
      acc[s] += p[k] * qv;
    }
  }
  double tot[4];
  if (!mf_reduce<4>(acc, part, &st->ticket, tot) || threadIdx.x != 0) return;
  for (int s = 0; s < 4; s++) {
    st->alpha[s] = 0.0;
    if (!st->active[s]) continue;
    if (!(tot[s] > 0.0)) {
      st->active[s] = 0;
      st->status[s] = isfinite(tot[s]) ? TP_ERR_BREAKDOWN : TP_ERR_NONFINITE;
      st->iters[s] = st->it;
      continue;
    }
    st->alpha[s] = st->rz[s] / tot[s];
  }
}

// x += alpha p, r -= alpha q, z = D^-1 r; r.z, r.r -> beta, convergence of each lane
template <int LD>
__global__ void __launch_bounds__(MF_BLOCK) k_mf_update(int64_t n, int S, const double* p,
                                                        const double* q, const double* dinv,
                                                        double* x, double* r, double* z,
                                                        double* part, MfState* st) {
  if (st->done) return;
  double al[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) al[s] = st->alpha[s];
  double acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = 0.0;
  MF_ROWS {
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const int64_t k = i * LD + s;
      if (al[s] != 0.0) {
        x[k] += al[s] * p[k];
        r[k] -= al[s] * q[k];
      }
      const double rv = r[k], zv = dinv[k] * rv;
      z[k] = zv;
      acc[s] += rv * zv;
      acc[4 + s] += rv * rv;
    }
  }
  double tot[8];
  if (!mf_reduce<8>(acc, part, &st->ticket, tot) || threadIdx.x != 0) return;
  st->it++;
  int any = 0;
  for (int s = 0; s < S; s++) {
    st->beta[s] = 0.0;
    if (!st->active[s]) continue;
    const double rz = tot[s], rr = tot[4 + s];
    if (!isfinite(rz) || !isfinite(rr)) {
      st->active[s] = 0;
      st->status[s] = TP_ERR_NONFINITE;
      st->iters[s] = st->it;
      continue;
    }
    st->rr[s] = rr;
    if (rr <= st->tol2[s]) {
      st->active[s] = 0;
      st->status[s] = TP_OK;
      st->iters[s] = st->it;
      continue;
    }
    st->beta[s] = (st->rz[s] != 0.0) ? rz / st->rz[s] : 0.0;
    st->rz[s] = rz;
    any = 1;
  }
  if (any && st->it >= st->max_it) {
    for (int s = 0; s < S; s++) {
      if (st->active[s]) {
        st->active[s] = 0;
        st->status[s] = TP_ERR_NOT_CONVERGED;
        st->iters[s] = st->it;
      }
    }
    any = 0;
  }
  st->done = !any;
}

// p = z + beta p (the lanes still active; a converged lane's p is left as it is)
template <int LD>
__global__ void k_mf_dir(int64_t n, const double* z, double* p, const MfState* st) {
  double be[LD];
  int act[LD];
#pragma unroll
  for (int s = 0; s < LD; s++) {
    be[s] = st->beta[s];
    act[s] = st->active[s];
  }
  MF_ROWS {
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const int64_t k = i * LD + s;
      if (act[s]) p[k] = z[k] + be[s] * p[k];
    }
  }
}

// true residual ||b - A x||^2 per lane (q = A x; Dirichlet rows contribute b - x = 0)
template <int LD>
__global__ void __launch_bounds__(MF_BLOCK) k_mf_true(int64_t n, int S, const uint8_t* bc,
                                                      const double* b, const double* q,
                                                      double* part, MfState* st) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  MF_ROWS {
    if (bc && bc[i]) continue;
#pragma unroll
    for (int s = 0; s < LD; s++) {
      const int64_t k = i * LD + s;
      const double d = (s < S) ? b[k] - q[k] : 0.0;
      acc[s] += d * d;
    }
  }
  double tot[4];
  if (!mf_reduce<4>(acc, part, &st->ticket, tot) || threadIdx.x != 0) return;
  for (int s = 0; s < 4; s++) st->rtrue[s] = tot[s];
}
#undef MF_ROWS

template <int LD>
static int mf_solve(const tp_mesh* m, int S, const double* De, const double* alpha,
                    const double* dscale, const double* shift, double inv_dt, int lumped,
                    int legacy, const uint8_t* bc, const double* b, double* x, double4 rtol,
                    int max_it, char* ws, tp_mfcg_result* res, cudaStream_t st) {
  const int64_t n = m->n_verts;
  const size_t vec = ((sizeof(double) * LD * (size_t)n) + 255) & ~(size_t)255;
  double* r = reinterpret_cast<double*>(ws);
  double* z = reinterpret_cast<double*>(ws + vec);
  double* p = reinterpret_cast<double*>(ws + 2 * vec);
  double* q = reinterpret_cast<double*>(ws + 3 * vec);
  double* dinv = reinterpret_cast<double*>(ws + 4 * vec);
  const int G = 2 * sm_count();
  double* part = reinterpret_cast<double*>(ws + 5 * vec);
  MfState* sd = reinterpret_cast<MfState*>(ws + 5 * vec + ((sizeof(double) * 16 * G + 255) & ~(size_t)255));
  double d4[4] = {1, 1, 1, 1}, s4[4] = {0, 0, 0, 0};
  for (int i = 0; i < S; i++) {
    if (dscale) d4[i] = dscale[i];
    if (shift) s4[i] = shift[i];
  }
  // Jacobi diagonal, Dirichlet values into x
  TP_CUDA_TRY(cudaMemsetAsync(dinv, 0, sizeof(double) * LD * n, st));
  TP_CUDA_TRY(cudaMemsetAsync(sd, 0, sizeof(MfState), st));
  MfState h{};
  h.max_it = max_it;
  TP_CUDA_TRY(cudaMemcpyAsync(&sd->max_it, &h.max_it, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  k_mf_diag<LD><<<grid_for(m->n_cells, 256, sm_count() * 8), 256, 0, st>>>(
      m->n_cells, reinterpret_cast<const int4*>(m->cells),
      reinterpret_cast<const double4*>(m->coords4), De, alpha,
      make_double4(d4[0], d4[1], d4[2], d4[3]), make_double4(s4[0], s4[1], s4[2], s4[3]),
      inv_dt, lumped, legacy, S, dinv);
  TP_LAUNCH_CHECK();
  k_mf_prep<LD><<<G, MF_BLOCK, 0, st>>>(n, S, bc, b, x, dinv);
  TP_LAUNCH_CHECK();
  auto apply = [&](const double* in, double* out) -> int {
    return tp_matfree_apply(m, S, LD, 0, De, alpha, d4, s4, inv_dt, lumped, legacy, in, out,
                            st);
  };
  int rc = apply(x, q);
  if (rc != TP_OK) return rc;
  k_mf_start<LD><<<G, MF_BLOCK, 0, st>>>(n, S, bc, b, q, dinv, r, z, p, part, sd, rtol);
  TP_LAUNCH_CHECK();
  // iterations in batches, the done flag read between batches (a batch past convergence
  // is a string of no-op launches)
  constexpr int BATCH = 8;
  int32_t done = 0;
  for (int it = 0; it < max_it && !done; it += BATCH) {
    for (int k = 0; k < BATCH; k++) {
      rc = apply(p, q);
      if (rc != TP_OK) return rc;
      k_mf_alpha<LD><<<G, MF_BLOCK, 0, st>>>(n, S, bc, p, q, part, sd);
      k_mf_update<LD><<<G, MF_BLOCK, 0, st>>>(n, S, p, q, dinv, x, r, z, part, sd);
      k_mf_dir<LD><<<G, MF_BLOCK, 0, st>>>(n, z, p, sd);
      TP_LAUNCH_CHECK();
    }
    TP_CUDA_TRY(cudaMemcpyAsync(&done, &sd->done, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    TP_CUDA_TRY(cudaStreamSynchronize(st));
  }
  rc = apply(x, q);
  if (rc != TP_OK) return rc;
  k_mf_true<LD><<<G, MF_BLOCK, 0, st>>>(n, S, bc, b, q, part, sd);
  TP_LAUNCH_CHECK();
  TP_CUDA_TRY(cudaMemcpyAsync(&h, sd, sizeof(MfState), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  int status = TP_OK;
  for (int s = 0; s < S; s++) {
    int ls = h.status[s];
    if (ls == -1) ls = TP_ERR_NOT_CONVERGED;
    // the recurrence residual stopped the lane; the true residual confirms it
    if (ls == TP_OK && !(h.rtrue[s] <= h.tol2[s] * 1.0000001)) ls = TP_ERR_NOT_CONVERGED;
    res->lane_status[s] = ls;
    res->lane_iters[s] = h.iters[s];
    res->lane_rnorm[s] = sqrt(std::max(h.rtrue[s], 0.0));
    res->lane_bnorm[s] = sqrt(std::max(h.bb[s], 0.0));
    if (ls != TP_OK && status == TP_OK) status = ls;
  }
  res->status = status;
  res->iterations = h.it;
  return TP_OK;
}

}  // namespace tp

extern "C" size_t tp_mfcg_workspace_bytes(int64_t n_verts, int ld) {
  const size_t vec = ((sizeof(double) * (size_t)ld * (size_t)n_verts) + 255) & ~(size_t)255;
  const size_t part = ((sizeof(double) * 16 * 2 * (size_t)tp::sm_count()) + 255) & ~(size_t)255;
  return 5 * vec + part + ((sizeof(tp::MfState) + 255) & ~(size_t)255);
}

extern "C" int tp_mfcg_solve(const tp_mesh* m, int S, int ld, const double* De_cell,
                             const double* alpha_cell, const double* diff_scale,
                             const double* shift, double inv_dt, int lumped, int legacy,
                             const uint8_t* bc_mask, const double* b, double* x,
                             const double* rtol, int max_it, void* workspace,
                             size_t workspace_bytes, tp_mfcg_result* res, void* stream) {
  TP_REQUIRE(m && m->cells && m->coords4 && De_cell && b && x && rtol && workspace && res,
             "null pointer");
  TP_REQUIRE(S >= 1 && S <= TP_MAX_COLS && (ld == 1 || ld == 2 || ld == 4) && ld >= S,
             "bad S/ld");
  TP_REQUIRE(max_it >= 0, "max_it < 0");
  TP_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  TP_REQUIRE(workspace_bytes >= tp_mfcg_workspace_bytes(m->n_verts, ld), "workspace too small");
  *res = tp_mfcg_result{};
  if (m->n_verts == 0) return TP_OK;
  double rt[4] = {0, 0, 0, 0};
  for (int s = 0; s < S; s++) rt[s] = rtol[s];
  const double4 r4 = make_double4(rt[0], rt[1], rt[2], rt[3]);
  char* ws = static_cast<char*>(workspace);
  cudaStream_t st = as_stream(stream);
  if (ld == 1)
    return mf_solve<1>(m, S, De_cell, alpha_cell, diff_scale, shift, inv_dt, lumped, legacy,
                       bc_mask, b, x, r4, max_it, ws, res, st);
  if (ld == 2)
    return mf_solve<2>(m, S, De_cell, alpha_cell, diff_scale, shift, inv_dt, lumped, legacy,
                       bc_mask, b, x, r4, max_it, ws, res, st);
  return mf_solve<4>(m, S, De_cell, alpha_cell, diff_scale, shift, inv_dt, lumped, legacy,
                     bc_mask, b, x, r4, max_it, ws, res, st);
}
