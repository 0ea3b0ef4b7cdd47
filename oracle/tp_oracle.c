/*
 * tp_oracle.c -- CPU oracle for the P1-tet reaction-diffusion transport path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain sequential C, the
 * arithmetic of the reference's GPU assembler and the Krylov semantics of its
 * solver layer.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs load it, always as the checker or as the timed CPU baseline,
 * never as part of the product path.
 *
 * Restated reference code (paths inside the reference project):
 *   or_assemble           gpu/gpu_assembler.py:60-139   (assemble_p1_tet kernel)
 *   or_dirichlet_rows     gpu/gpu_assembler.py:147-165  (apply_dirichlet_rows)
 *   or_assemble_rhs       gpu/gpu_assembler.py:176-221  (assemble_rhs_p1_tet)
 *   or_dirichlet_rhs      gpu/gpu_assembler.py:228-239  (apply_dirichlet_rhs)
 *   or_nodal_gradient     gpu/gpu_assembler.py:251-304, 646-673
 *   or_matfree_apply      gpu/ceed_operators.py:87-108 (DiffMassBilinear), with the
 *                         stiffness weighted by wdetJ (intended) or not (legacy)
 *   or_gmres_bjacobi      numerics/solvers.py:322-335, 369 (KSP gmres restart 50,
 *                         PC bjacobi, whose per-block sub-PC is ILU(0) in PETSc)
 *   or_pcg_jacobi         the configs' Jacobi-PCG, with the stopping rule
 *                         ||b - A x||_2 <= rtol ||b||_2 used throughout this project
 *
 * Accumulation runs in cell order with no fused multiply-add (built with
 * -ffp-contract=off), so results are a fixed function of the inputs.  The
 * reference accumulates with atomicAdd in an order the GPU chooses.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

static const double REF_GRAD[4][3] = {
    {-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
static const double MUNIT[4][4] = {
    {2.0, 1.0, 1.0, 1.0}, {1.0, 2.0, 1.0, 1.0}, {1.0, 1.0, 2.0, 1.0}, {1.0, 1.0, 1.0, 2.0}};

EXPORT int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

EXPORT void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* element matrix entry exactly as gpu_assembler.py:104-132 writes it */
static inline double elem_entry(int i, int j, double dJ, double De, double a_,
                                const double G[3][3], double inv_dt, int lumped) {
  double Gg[3] = {0.0, 0.0, 0.0};
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) Gg[a] += G[a][b] * REF_GRAD[j][b];
  double K = 0.0;
  for (int a = 0; a < 3; a++) K += REF_GRAD[i][a] * Gg[a];
  K *= (dJ * De) / 6.0;
  double M;
  if (lumped)
    M = (i == j) ? (dJ * 5.0 / 120.0) : 0.0;
  else
    M = dJ * MUNIT[i][j] / 120.0;
  return K + (inv_dt + a_) * M;
}

/* gpu_assembler.py:60-139 + :488 (data zeroed first) */
EXPORT void or_assemble(int64_t n_cells, const double* detJ, const double* Gflat,
                        const double* De_cell, const double* alpha_cell, double inv_dt,
                        int lumped, const int32_t* scatter_map, int64_t nnz, double* data) {
  memset(data, 0, sizeof(double) * (size_t)nnz);
  for (int64_t c = 0; c < n_cells; c++) {
    const double dJ = detJ[c], De = De_cell[c], a_ = alpha_cell[c];
    double G[3][3];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) G[a][b] = Gflat[c * 9 + a * 3 + b];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++)
        data[scatter_map[c * 16 + i * 4 + j]] +=
            elem_entry(i, j, dJ, De, a_, G, inv_dt, lumped);
  }
}

/* gpu_assembler.py:147-165 */
EXPORT void or_dirichlet_rows(int64_t n_bc, const int32_t* bc, const int32_t* indptr,
                              const int32_t* indices, double* data) {
  for (int64_t k = 0; k < n_bc; k++) {
    const int row = bc[k];
    for (int p = indptr[row]; p < indptr[row + 1]; p++)
      data[p] = (indices[p] == row) ? 1.0 : 0.0;
  }
}

/* gpu_assembler.py:176-221 + :575 (b zeroed first) */
EXPORT void or_assemble_rhs(int64_t n_cells, int64_t n_dofs, const int32_t* elem,
                            const double* detJ, const double* u_old, const double* f,
                            double inv_dt, int lumped, double* b) {
  memset(b, 0, sizeof(double) * (size_t)n_dofs);
  for (int64_t c = 0; c < n_cells; c++) {
    const int n0 = elem[c * 4 + 0], n1 = elem[c * 4 + 1], n2 = elem[c * 4 + 2],
              n3 = elem[c * 4 + 3];
    const double dJ = detJ[c];
    const double u0 = u_old[n0], u1 = u_old[n1], u2 = u_old[n2], u3 = u_old[n3];
    const double f0 = f[n0], f1 = f[n1], f2 = f[n2], f3 = f[n3];
    const double sum_u = u0 + u1 + u2 + u3;
    const double sum_f = f0 + f1 + f2 + f3;
    const double base = dJ / 120.0;
    const double mdt = base * inv_dt;
    const double mf = base;
    if (lumped) {
      const double Ld = base * 5.0;
      b[n0] += Ld * (inv_dt * u0 + f0);
      b[n1] += Ld * (inv_dt * u1 + f1);
      b[n2] += Ld * (inv_dt * u2 + f2);
      b[n3] += Ld * (inv_dt * u3 + f3);
    } else {
      b[n0] += mdt * (sum_u + u0) + mf * (sum_f + f0);
      b[n1] += mdt * (sum_u + u1) + mf * (sum_f + f1);
      b[n2] += mdt * (sum_u + u2) + mf * (sum_f + f2);
      b[n3] += mdt * (sum_u + u3) + mf * (sum_f + f3);
    }
  }
}

/* gpu_assembler.py:228-239 */
EXPORT void or_dirichlet_rhs(int64_t n_bc, const int32_t* bc, double value, double* b) {
  for (int64_t k = 0; k < n_bc; k++) b[bc[k]] = value;
}

/* gpu_assembler.py:251-304 and the division at :672 */
EXPORT void or_nodal_gradient(int64_t n_cells, int64_t n_dofs, const int32_t* elem,
                              const double* detJ, const double* JinvT, const double* u,
                              double* grad /* (n_dofs,3) */, double* wsum) {
  memset(grad, 0, sizeof(double) * 3 * (size_t)n_dofs);
  memset(wsum, 0, sizeof(double) * (size_t)n_dofs);
  for (int64_t c = 0; c < n_cells; c++) {
    int gn[4];
    double uu[4];
    for (int a = 0; a < 4; a++) {
      gn[a] = elem[c * 4 + a];
      uu[a] = u[gn[a]];
    }
    double gr[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 4; a++) {
      gr[0] += uu[a] * REF_GRAD[a][0];
      gr[1] += uu[a] * REF_GRAD[a][1];
      gr[2] += uu[a] * REF_GRAD[a][2];
    }
    const double* JT = JinvT + c * 9;
    double gp[3];
    gp[0] = JT[0] * gr[0] + JT[1] * gr[1] + JT[2] * gr[2];
    gp[1] = JT[3] * gr[0] + JT[4] * gr[1] + JT[5] * gr[2];
    gp[2] = JT[6] * gr[0] + JT[7] * gr[1] + JT[8] * gr[2];
    const double w = detJ[c] / 6.0;
    for (int i = 0; i < 4; i++) {
      const int d = gn[i];
      grad[d * 3 + 0] += w * gp[0];
      grad[d * 3 + 1] += w * gp[1];
      grad[d * 3 + 2] += w * gp[2];
      wsum[d] += w;
    }
  }
  for (int64_t d = 0; d < n_dofs; d++)
    for (int k = 0; k < 3; k++) grad[d * 3 + k] = grad[d * 3 + k] / wsum[d];
}

/*
 * Matrix-free operator of gpu/ceed_operators.py:87-108 applied to S interleaved
 * columns: y[:, s] = sum_e [ De_e K_e + (inv_dt + alpha_e + shift_s) M_e ] x_e[:, s].
 * De, alpha per cell (alpha may be NULL); mass consistent (degree-2 quadrature is
 * exact for P1 x P1) or lumped; legacy != 0 reproduces the reference QFunction,
 * whose stiffness omits wdetJ (sum over 4 points of De G -> 4 De instead of
 * |detJ|/6 De).  diff_scale[s] multiplies De for column s (NULL -> 1).
 */
EXPORT void or_matfree_apply(int64_t n_cells, int64_t n_dofs, int S, const int32_t* elem,
                             const double* detJ, const double* Gflat, const double* De_cell,
                             const double* alpha_cell, const double* diff_scale,
                             const double* shift, double inv_dt, int lumped, int legacy,
                             const double* x, double* y) {
  memset(y, 0, sizeof(double) * (size_t)n_dofs * S);
  for (int64_t c = 0; c < n_cells; c++) {
    const double dJ = detJ[c];
    double G[3][3];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) G[a][b] = Gflat[c * 9 + a * 3 + b];
    double Kref[4][4];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        double Gg[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) Gg[a] += G[a][b] * REF_GRAD[j][b];
        double K = 0.0;
        for (int a = 0; a < 3; a++) K += REF_GRAD[i][a] * Gg[a];
        Kref[i][j] = K;
      }
    const double kscale = legacy ? 4.0 : dJ / 6.0;
    for (int s = 0; s < S; s++) {
      const double De = De_cell[c] * (diff_scale ? diff_scale[s] : 1.0);
      const double react = inv_dt + (alpha_cell ? alpha_cell[c] : 0.0) + (shift ? shift[s] : 0.0);
      for (int i = 0; i < 4; i++) {
        double acc = 0.0;
        for (int j = 0; j < 4; j++) {
          const double M = lumped ? ((i == j) ? dJ * 5.0 / 120.0 : 0.0) : dJ * MUNIT[i][j] / 120.0;
          acc += (De * kscale * Kref[i][j] + react * M) * x[(int64_t)elem[c * 4 + j] * S + s];
        }
        y[(int64_t)elem[c * 4 + i] * S + s] += acc;
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* sparse kernels and Krylov solvers                                   */
/* ------------------------------------------------------------------ */

EXPORT void or_spmv(int64_t n, const int32_t* indptr, const int32_t* indices,
                    const double* data, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    double s = 0.0;
    for (int p = indptr[i]; p < indptr[i + 1]; p++) s += data[p] * x[indices[p]];
    y[i] = s;
  }
}

/* fixed-order parallel dot: per-thread static chunks summed in thread order */
static double dot_fixed(int64_t n, const double* a, const double* b) {
  int nt = or_num_threads();
  double part[512];
  if (nt > 512) nt = 512;
#pragma omp parallel num_threads(nt)
  {
    int t = 0, T = 1;
#ifdef _OPENMP
    t = omp_get_thread_num();
    T = omp_get_num_threads();
#endif
    int64_t lo = n * t / T, hi = n * (t + 1) / T;
    double s = 0.0;
    for (int64_t i = lo; i < hi; i++) s += a[i] * b[i];
    part[t] = s;
  }
  double s = 0.0;
  for (int t = 0; t < nt; t++) s += part[t];
  return s;
}

/*
 * Jacobi-PCG on the row-eliminated system.  Rows with bc_mask != 0 are identity
 * rows: x keeps its value there, the preconditioner is zero there, so every
 * search direction vanishes on them and CG runs on the symmetric free block.
 * Stops when ||b - A x||_2 <= rtol ||b||_2 (recurrence residual, confirmed by a
 * true residual).  Returns iterations; *status: 0 converged, 1 max_it,
 * 2 breakdown (p.Ap <= 0), 3 non-finite.
 */
EXPORT int or_pcg_jacobi(int64_t n, const int32_t* indptr, const int32_t* indices,
                         const double* data, const uint8_t* bc_mask, const double* b,
                         double* x, double rtol, int max_it, int* status, double* rnorm_out) {
  double *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n),
         *p = malloc(sizeof(double) * n), *q = malloc(sizeof(double) * n),
         *dinv = malloc(sizeof(double) * n);
  for (int64_t i = 0; i < n; i++) {
    double d = 0.0;
    for (int k = indptr[i]; k < indptr[i + 1]; k++)
      if (indices[k] == i) d = data[k];
    dinv[i] = (bc_mask && bc_mask[i]) ? 0.0 : 1.0 / d;
  }
  const double bnorm = sqrt(dot_fixed(n, b, b));
  const double tol = rtol * bnorm;
  or_spmv(n, indptr, indices, data, x, q);
  for (int64_t i = 0; i < n; i++) {
    r[i] = b[i] - q[i];
    z[i] = dinv[i] * r[i];
    p[i] = z[i];
  }
  double rz = dot_fixed(n, r, z);
  double rr = dot_fixed(n, r, r);
  int it = 0;
  *status = 1;
  while (it < max_it) {
    if (sqrt(rr) <= tol) {
      /* confirm with the true residual */
      or_spmv(n, indptr, indices, data, x, q);
      for (int64_t i = 0; i < n; i++) r[i] = b[i] - q[i];
      rr = dot_fixed(n, r, r);
      if (sqrt(rr) <= tol) {
        *status = 0;
        break;
      }
      for (int64_t i = 0; i < n; i++) {
        z[i] = dinv[i] * r[i];
        p[i] = z[i];
      }
      rz = dot_fixed(n, r, z);
    }
    or_spmv(n, indptr, indices, data, p, q);
    const double pq = dot_fixed(n, p, q);
    if (!(pq > 0.0)) {
      *status = isfinite(pq) ? 2 : 3;
      break;
    }
    const double alpha = rz / pq;
    for (int64_t i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = dinv[i] * r[i];
    }
    const double rz_new = dot_fixed(n, r, z);
    rr = dot_fixed(n, r, r);
    const double beta = rz_new / rz;
    rz = rz_new;
    for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    it++;
    if (!isfinite(rr)) {
      *status = 3;
      break;
    }
  }
  if (*status == 1 && sqrt(rr) <= tol) *status = 0;
  if (rnorm_out) *rnorm_out = sqrt(rr);
  free(r);
  free(z);
  free(p);
  free(q);
  free(dinv);
  return it;
}

/* ---- ILU(0) restricted to diagonal blocks (PCBJACOBI with sub-PC ILU) ---- */

typedef struct {
  int64_t n;
  const int32_t* indptr;
  const int32_t* indices;
  double* lu;       /* factored values on the block-restricted pattern */
  int32_t* diag;    /* position of the diagonal in each row */
  int32_t* blk_lo;  /* block start row per row */
  int32_t* blk_hi;
} ilu_t;

static void ilu0_factor_block(ilu_t* F, int64_t lo, int64_t hi) {
  const int32_t* ip = F->indptr;
  const int32_t* ix = F->indices;
  double* a = F->lu;
  for (int64_t i = lo; i < hi; i++) {
    for (int p = ip[i]; p < ip[i + 1]; p++) {
      const int k = ix[p];
      if (k < lo || k >= i) continue;
      const double akk = a[F->diag[k]];
      a[p] = a[p] / akk;
      const double aik = a[p];
      /* a_ij -= a_ik a_kj for j > k present in both rows (sorted merge) */
      int q = F->diag[k] + 1;
      int r = p + 1;
      while (q < ip[k + 1] && r < ip[i + 1]) {
        const int jk = ix[q], ji = ix[r];
        if (jk >= hi) break;
        if (jk == ji) {
          a[r] -= aik * a[q];
          q++;
          r++;
        } else if (jk < ji) {
          q++;
        } else {
          r++;
        }
      }
    }
  }
}

static void ilu0_solve_block(const ilu_t* F, int64_t lo, int64_t hi, const double* rhs,
                             double* out) {
  const int32_t* ip = F->indptr;
  const int32_t* ix = F->indices;
  const double* a = F->lu;
  for (int64_t i = lo; i < hi; i++) {
    double s = rhs[i];
    for (int p = ip[i]; p < F->diag[i]; p++) {
      const int k = ix[p];
      if (k >= lo) s -= a[p] * out[k];
    }
    out[i] = s;
  }
  for (int64_t i = hi - 1; i >= lo; i--) {
    double s = out[i];
    for (int p = F->diag[i] + 1; p < ip[i + 1]; p++) {
      const int k = ix[p];
      if (k < hi) s -= a[p] * out[k];
    }
    out[i] = s / a[F->diag[i]];
  }
}

/*
 * Restarted GMRES(m), right-preconditioned by block-Jacobi ILU(0) with nblocks
 * contiguous row blocks (PETSc PCBJACOBI gives one block per MPI rank, each
 * factored by ILU(0)).  Classical Gram-Schmidt as in PETSc's default
 * orthogonalisation.  Right preconditioning makes the Arnoldi residual the true
 * residual, so the stop rule ||b - A x|| <= rtol ||b|| matches or_pcg_jacobi.
 * Returns the total iteration count.
 */
EXPORT int or_gmres_bjacobi(int64_t n, const int32_t* indptr, const int32_t* indices,
                            const double* data, const double* b, double* x, double rtol,
                            int max_it, int restart, int nblocks, int* status,
                            double* rnorm_out) {
  const int m = restart;
  ilu_t F;
  F.n = n;
  F.indptr = indptr;
  F.indices = indices;
  const int64_t nnz = indptr[n];
  F.lu = malloc(sizeof(double) * nnz);
  memcpy(F.lu, data, sizeof(double) * nnz);
  F.diag = malloc(sizeof(int32_t) * n);
  for (int64_t i = 0; i < n; i++) {
    F.diag[i] = indptr[i];
    for (int p = indptr[i]; p < indptr[i + 1]; p++)
      if (indices[p] == i) F.diag[i] = p;
  }
  if (nblocks < 1) nblocks = 1;
  if (nblocks > n) nblocks = (int)n;
#pragma omp parallel for schedule(static, 1)
  for (int bk = 0; bk < nblocks; bk++) ilu0_factor_block(&F, n * bk / nblocks, n * (bk + 1) / nblocks);

  double* V = malloc(sizeof(double) * n * (m + 1));
  double* Z = malloc(sizeof(double) * n * m);
  double* H = calloc((size_t)(m + 1) * m, sizeof(double));
  double *cs = malloc(sizeof(double) * m), *sn = malloc(sizeof(double) * m),
         *g = malloc(sizeof(double) * (m + 1)), *yv = malloc(sizeof(double) * m);
  double* w = malloc(sizeof(double) * n);
  const double bnorm = sqrt(dot_fixed(n, b, b));
  const double tol = rtol * bnorm;
  int it = 0;
  double beta = 0.0;
  *status = 1;
  for (;;) {
    or_spmv(n, indptr, indices, data, x, w);
    for (int64_t i = 0; i < n; i++) V[i] = b[i] - w[i];
    beta = sqrt(dot_fixed(n, V, V));
    if (beta <= tol) {
      *status = 0;
      break;
    }
    if (it >= max_it) break;
    for (int64_t i = 0; i < n; i++) V[i] /= beta;
    memset(g, 0, sizeof(double) * (m + 1));
    g[0] = beta;
    int j = 0;
    for (; j < m && it < max_it; j++, it++) {
      double* vj = V + (int64_t)j * n;
      double* zj = Z + (int64_t)j * n;
#pragma omp parallel for schedule(static, 1)
      for (int bk = 0; bk < nblocks; bk++)
        ilu0_solve_block(&F, n * bk / nblocks, n * (bk + 1) / nblocks, vj, zj);
      or_spmv(n, indptr, indices, data, zj, w);
      for (int k = 0; k <= j; k++) H[k * m + j] = dot_fixed(n, w, V + (int64_t)k * n);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; i++) {
        double s = w[i];
        for (int k = 0; k <= j; k++) s -= H[k * m + j] * V[(int64_t)k * n + i];
        w[i] = s;
      }
      const double hn = sqrt(dot_fixed(n, w, w));
      H[(j + 1) * m + j] = hn;
      double* vn = V + (int64_t)(j + 1) * n;
      for (int64_t i = 0; i < n; i++) vn[i] = (hn > 0.0) ? w[i] / hn : 0.0;
      for (int k = 0; k < j; k++) {
        const double t = cs[k] * H[k * m + j] + sn[k] * H[(k + 1) * m + j];
        H[(k + 1) * m + j] = -sn[k] * H[k * m + j] + cs[k] * H[(k + 1) * m + j];
        H[k * m + j] = t;
      }
      const double h0 = H[j * m + j], h1 = H[(j + 1) * m + j];
      const double den = sqrt(h0 * h0 + h1 * h1);
      cs[j] = (den > 0.0) ? h0 / den : 1.0;
      sn[j] = (den > 0.0) ? h1 / den : 0.0;
      H[j * m + j] = den;
      H[(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (fabs(g[j + 1]) <= tol || hn == 0.0) {
        j++;
        it++;
        break;
      }
    }
    /* back-substitute and update x += Z y */
    for (int k = j - 1; k >= 0; k--) {
      double s = g[k];
      for (int l = k + 1; l < j; l++) s -= H[k * m + l] * yv[l];
      yv[k] = s / H[k * m + k];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      double s = 0.0;
      for (int k = 0; k < j; k++) s += yv[k] * Z[(int64_t)k * n + i];
      x[i] += s;
    }
  }
  if (rnorm_out) *rnorm_out = beta;
  free(F.lu);
  free(F.diag);
  free(V);
  free(Z);
  free(H);
  free(cs);
  free(sn);
  free(g);
  free(yv);
  free(w);
  return it;
}

/* row sums of the consistent mass = lumped nodal mass |detJ|/24 per incident cell
   (gpu_assembler.py:122-129) */
EXPORT void or_lumped_mass(int64_t n_cells, int64_t n_dofs, const int32_t* elem,
                           const double* detJ, double* m) {
  memset(m, 0, sizeof(double) * (size_t)n_dofs);
  for (int64_t c = 0; c < n_cells; c++)
    for (int i = 0; i < 4; i++) m[elem[c * 4 + i]] += detJ[c] * 5.0 / 120.0;
}
