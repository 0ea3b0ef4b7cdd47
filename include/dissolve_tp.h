/*
 * dissolve_tp.h -- C ABI of the B200 P1-tetrahedral reaction-diffusion transport path.
 *
 * Plain C: every pointer is device memory owned by the caller unless marked (host),
 * sizes are int64_t, `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).  Every entry point returns TP_OK or a TP_ERR_* code;
 * tp_last_error() gives the detail text of the last failure on the calling thread.
 * Functions marked [sync] synchronise `stream` before returning (they validate
 * input on the device and report through the return code); all others only
 * enqueue work on `stream`.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   gpu/gpu_assembler.py   GPUSparseAssembler and its five NVRTC kernels
 *   gpu/ceed_operators.py  CeedDiffusionMassOp (libCEED matrix-free operator)
 *   numerics/solvers.py    _solve_gpu_asm's PETSc KSP solve
 *   dissolve.py            per-species coefficient builders (CuPy elementwise)
 * The Python module dissolve_tp (dissolve-2.0_b200/) binds these through ctypes and
 * keeps the reference's Python call signatures on top.
 */
#ifndef DISSOLVE_TP_H
#define DISSOLVE_TP_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TP_API __attribute__((visibility("default")))
#else
#define TP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define TP_OK 0
#define TP_ERR_ARG 1          /* invalid argument (null pointer, size, option)        */
#define TP_ERR_CUDA 2         /* CUDA runtime error                                   */
#define TP_ERR_INDEX 3        /* a vertex or dof id outside [0, n_verts)              */
#define TP_ERR_DEGENERATE 4   /* a cell with det J == 0 or non-finite coordinates     */
#define TP_ERR_CAPACITY 5     /* a CSR row or vertex degree beyond the kernel limits  */
#define TP_ERR_NOT_CONVERGED 6 /* Krylov solve stopped at max_it                      */
#define TP_ERR_BREAKDOWN 7    /* p.Ap <= 0: operator not SPD on the free dofs         */
#define TP_ERR_NONFINITE 8    /* NaN/Inf in a Krylov scalar                           */
#define TP_ERR_TIMEOUT 9      /* a bounded device-side wait gave up (grid barrier)     */

/* assembly modes for tp_assemble_csr */
#define TP_ASM_FULL 0   /* De K + (inv_dt + alpha) M  (gpu_assembler.py:60-139)      */
#define TP_ASM_STIFF 1  /* De K only (shared stiffness for multi-species operators) */
#define TP_ASM_MASS 2   /* M only, coefficient 1 (consistent or lumped)             */

#define TP_MAX_COLS 4   /* right-hand sides per multi-column operator/solve          */

TP_API int tp_version(void);
TP_API const char* tp_status_string(int status);
TP_API const char* tp_last_error(void);
TP_API int tp_device_sm_count(void);

/* ------------------------------------------------------------------ mesh on device */
/* Row tiles of a mesh (opaque; tp_tiles_create).  No reference counterpart: the tables
 * that let the row-owned kernels load every cell record of a group of nearby rows once. */
typedef struct tp_tiles tp_tiles;

/* Device-resident mesh: the state GPUSparseAssembler keeps between calls
 * (gpu_assembler.py:323-326, 350-367).  Built once by the setup calls below. */
typedef struct tp_mesh {
  int64_t n_cells;
  int64_t n_verts;
  int64_t nnz;
  int32_t max_row_len;        /* longest CSR row (<= 255)                            */
  int32_t max_degree;         /* most cells sharing one vertex                       */
  const int32_t* cells;       /* (n_cells, 4) vertex ids = P1 dofs                   */
  const double* coords4;      /* (n_verts, 4) x, y, z, 0 (32-byte rows, 32-byte base) */
  const double* geo;          /* (n_cells, 8) G00 G01 G02 G11 G12 G22 |detJ| 0, 32-byte base */
  const int32_t* v2c_ptr;     /* (n_verts + 1) incidence offsets                     */
  const int32_t* v2c;         /* (4 n_cells) cell*4 + local index, ascending cell    */
  const uint32_t* v2c_slots;  /* (4 n_cells) row-local CSR slot of the cell's 4 vertices,
                                 byte j = slot of vertex j in the incidence row      */
  const int32_t* indptr;      /* (n_verts + 1) CSR row offsets                       */
  const int32_t* indices;     /* (nnz) sorted column ids                             */
  const tp_tiles* tiles;      /* row tiles (tp_tiles_create) or NULL: the kernels that
                                 have a tiled form use it when set (same results)     */
} tp_mesh;

/* [sync] Per-cell geometry of gpu_assembler.py:380-393: J = [x1-x0 | x2-x0 | x3-x0],
 * detJ = |det J|, G = J^-1 J^-T and J^-T, all row-major, plus the compact 64-byte record
 * `geo` and the padded coordinate copy `coords4` the kernels read.  detJ, Gflat, JinvT
 * and coords4 may be NULL.  flags_dev: 1 int32 of device scratch.
 * Returns TP_ERR_INDEX / TP_ERR_DEGENERATE on bad cells. */
TP_API int tp_cell_geometry(int64_t n_cells, int64_t n_verts, const int32_t* cells,
                     const double* coords, double* coords4, double* geo, double* detJ,
                     double* Gflat, double* JinvT, int32_t* flags_dev, void* stream);

/* [sync] Compact record from the reference-layout arrays (detJ (n), Gflat (n, 9)), so the
 * assembly can run on geometry computed elsewhere (gpu_assembler.py:380-386 numpy). */
TP_API int tp_pack_geometry(int64_t n_cells, const double* detJ, const double* Gflat, double* geo,
                     void* stream);

/* bytes of device scratch the setup calls below need */
TP_API size_t tp_setup_scratch_bytes(int64_t n_cells, int64_t n_verts);

/* [sync] Vertex -> cell incidence (ascending cell id per vertex).  Replaces the
 * per-row Python sets of gpu_assembler.py:396-400. */
TP_API int tp_incidence(int64_t n_cells, int64_t n_verts, const int32_t* cells, int32_t* v2c_ptr,
                 int32_t* v2c, void* scratch, int32_t* max_degree_out /* host */,
                 void* stream);

/* [sync] CSR sparsity of gpu_assembler.py:396-410: row r = sorted set of every vertex
 * sharing a cell with r, r included.  Call once with indices == NULL (fills indptr,
 * returns nnz), then with indices allocated to nnz. */
TP_API int tp_pattern(int64_t n_cells, int64_t n_verts, const int32_t* cells, const int32_t* v2c_ptr,
               const int32_t* v2c, int32_t max_degree, int32_t* indptr, int32_t* indices,
               void* scratch, int64_t* nnz_out /* host */,
               int32_t* max_row_len_out /* host */, void* stream);

/* gpu_assembler.py:419-438: scatter_map[c*16 + i*4 + j] = CSR position of
 * (cells[c,i], cells[c,j]). */
TP_API int tp_scatter_map(int64_t n_cells, const int32_t* cells, const int32_t* indptr,
                   const int32_t* indices, int32_t* scatter_map, void* stream);

/* [sync] Row-local slots of every incidence entry (no reference counterpart: this is
 * the element-to-nonzero map the atomics-free row assembly reads instead of the
 * reference's scatter_map + atomicAdd). */
TP_API int tp_incidence_slots(const tp_mesh* m, uint32_t* slots, int32_t* flags_dev, void* stream);

/* [sync] Row tiles for the tiled kernels (no reference counterpart): the rows are cut by
 * recursive coordinate bisection into tiles of rows_per_tile (64) nearby rows; per tile
 * the ascending list of the distinct cells its rows touch and, per incidence entry of its
 * rows (row-major [entry k][row]), the cell's tile-local index, the row's local vertex
 * and the four CSR slots of tp_incidence_slots.  Needs a complete mesh (coords4, v2c,
 * v2c_slots, indptr); built on the host from copies of those arrays, device tables owned
 * by the returned handle.  TP_ERR_CAPACITY if a tile touches more than 16383 cells. */
TP_API int tp_tiles_create(const tp_mesh* m, int rows_per_tile, void* stream, tp_tiles** out);
/* size of the tiling (any pointer may be NULL) */
TP_API int tp_tiles_info(const tp_tiles* t, int32_t* n_tiles, int32_t* rows_per_tile,
                         int32_t* max_cells, int64_t* n_entries, size_t* device_bytes);
TP_API int tp_tiles_destroy(tp_tiles* t);

/* ------------------------------------------------------------------ per-step kernels */
/* gpu_assembler.py:452-470 (_to_cell_avg, per-vertex branch): mean of 4 vertex values */
TP_API int tp_cell_average(int64_t n_cells, const int32_t* cells, const double* vert_vals,
                    double* cell_vals, void* stream);

/* [sync] mask[v] = 1 for v in bc_dofs, 0 elsewhere (mask is cleared first).
 * TP_ERR_INDEX if a dof is outside [0, n_verts). */
TP_API int tp_bc_mask(int64_t n_bc, const int32_t* bc_dofs, int64_t n_verts, uint8_t* mask,
               int32_t* flags_dev, void* stream);

/* gpu_assembler.py:60-139 (+ :147-165 when bc_mask != NULL) without atomics: each CSR
 * row sums its incident cells in ascending cell order, in the reference's operation
 * order, so the result equals the reference kernel run in cell order.  mode TP_ASM_*;
 * De_cell per cell; alpha_cell per cell or NULL (0).  out64 / out32: either may be NULL. */
TP_API int tp_assemble_csr(const tp_mesh* m, const double* De_cell, const double* alpha_cell,
                    double inv_dt, int lumped, int mode, const uint8_t* bc_mask,
                    double* out64, float* out32, void* stream);

/* gpu_assembler.py:147-165 on its own: rows of bc_dofs become identity rows (ids outside
 * [0, n_rows) are skipped) */
TP_API int tp_dirichlet_rows(int64_t n_bc, const int32_t* bc_dofs, int64_t n_rows,
                             const int32_t* indptr, const int32_t* indices, double* data,
                             void* stream);

/* Lumped-mass diagonal per column: diag[v, s] = sum_{c at v} (shift[s] + alpha[c, s])
 * |detJ_c|/24; alpha (n_cells, ld) or NULL; shift (host, S).  diag64/diag32 (n_verts, ld),
 * either may be NULL; bc rows (bc_mask != 0) get 1. */
TP_API int tp_lumped_diag(const tp_mesh* m, int S, int ld, const double* alpha, const double* shift,
                   const uint8_t* bc_mask, double* diag64, float* diag32, void* stream);

/* The shared stiffness of the batched step and its per-column lumped diagonal in one row
 * walk (no reference counterpart as one call: gpu_assembler.py:60-139 in TP_ASM_STIFF mode
 * plus tp_lumped_diag): out64 / out32 (CSR order) as tp_assemble_csr(mode TP_ASM_STIFF,
 * lumped) and diag64 / diag32 as tp_lumped_diag, both bit-identical to those calls;
 * optionally the FP32 values in the SELL-32 order of tp_sell_build (slice_ptr: its slice
 * offsets; entry k of row r at slice_ptr[r / 32] + 32 k + r % 32, padding entries 0), the
 * values tp_sell_scatter writes from out64. */
TP_API int tp_assemble_stiffness_diag(const tp_mesh* m, const double* De_cell, int S, int ld,
                                      const double* alpha, const double* shift,
                                      const uint8_t* bc_mask, double* out64, float* out32,
                                      const int32_t* slice_ptr, float* sell32, double* diag64,
                                      float* diag32, void* stream);

/* gpu_assembler.py:176-221 + :228-239 for S columns (interleaved, leading dim ld):
 * b = M (inv_dt u_old + f) lumped or consistent, then b[bc_dofs, s] = bc_value[s]
 * (host array of S values; bc_dofs may be NULL).  f may be NULL (zero source). */
TP_API int tp_assemble_rhs(const tp_mesh* m, int S, int ld, const double* u_old, const double* f,
                    double inv_dt, int lumped, int64_t n_bc, const int32_t* bc_dofs,
                    const double* bc_value, double* b, void* stream);

/* The lumped right-hand side of tp_assemble_rhs (lumped = 1) from a precomputed lumped
 * mass per vertex (mass = tp_lumped_diag with S = 1, shift 1, no alpha): b = mass (inv_dt
 * u_old + f) per column, one element-wise pass (no reference counterpart as such; it
 * differs from the cell-order sums of tp_assemble_rhs by rounding only, ~1e-16 relative). */
TP_API int tp_lumped_rhs(int64_t n_verts, int S, int ld, const double* mass, const double* u_old,
                         const double* f, double inv_dt, int64_t n_bc, const int32_t* bc_dofs,
                         const double* bc_value, double* b, void* stream);

/* gpu_assembler.py:251-304, 646-673: volume-weighted vertex average of the cellwise
 * gradient.  JinvT (n_cells, 9) as the reference stores it, or NULL to recompute J^-T
 * from coords4.  grad (n_verts, 3). */
TP_API int tp_nodal_gradient(const tp_mesh* m, const double* JinvT, const double* u, double* grad,
                      void* stream);

/* gpu_assembler.py:605-644: integral of the smoothed Heaviside H_eps(phi) with the
 * 4-point degree-2 rule.  out_dev: 1 double (device). scratch >= tp_setup_scratch_bytes. */
TP_API int tp_scaffold_volume(const tp_mesh* m, const double* phi, double eps, double* out_dev,
                       void* scratch, void* stream);

/* tp_scaffold_volume without the scratch argument: it allocates no device memory and needs
 * no buffer from the caller (no counterpart in the reference, whose volume integral runs
 * through CuPy's allocator).  For callers that cannot hand over a device temporary: hosts
 * that bind plain pointers and own no device allocator (a cgo/JNI/FFI embedding that only
 * passes the mesh and phi it already holds), and per-step loops that must not call
 * cudaMalloc/cudaFree, which synchronise the device.
 * Scratch: a fixed 8 KiB array compiled into this library, one per device, holding the
 * block partials; the launch is capped at 1024 blocks (grid-stride over the cells), so
 * every mesh size fits.  Nothing in it has to start at zero.  Outside a stream capture
 * every call looks up the array's address (cudaGetSymbolAddress) with the calling device
 * current and keeps it for that device; inside a capture the kept address is used, so a
 * caller that records calls into a stream capture makes one call on that device before the
 * capture begins (a call in a capture without one is rejected with TP_ERR_ARG).  Calls
 * that overlap on one device (two streams, or two host threads) share the array and race:
 * serialise them.  Result as tp_scaffold_volume. */
TP_API int tp_scaffold_volume_static(const tp_mesh* m, const double* phi, double eps,
                              double* out_dev, void* stream);

/* dissolve.py:866-875: alpha_O2 = delta_eps(phi) |grad phi| k_orr (per vertex) */
TP_API int tp_o2_alpha(int64_t n, const double* phi, const double* normgradphi, double eps,
                double k_orr, double* alpha, void* stream);

/* dissolve.py:923-936: f_OH = [phi <= 0] kd F Cl^2 + orr_factor delta_eps |grad phi| k_orr O2 */
TP_API int tp_oh_source(int64_t n, const double* phi, const double* normgradphi, const double* F,
                 const double* Cl, const double* O2, double eps, double kd, double k_orr,
                 double orr_factor, double* f, void* stream);

/* Interface reaction of the gyroid-scaffold step (the per-vertex analogue of
 * dissolve.py:866-875 and :923-936 with the smoothed Heaviside H_eps of
 * gpu_assembler.py:605-644 in place of delta_eps |grad phi|):
 * hv = k_orr H_eps(phi); ngphi = |grad phi| (grad (n, 3), may be NULL); f (n, ld) =
 * 0 except f[:, col_oh] = orr_factor hv U[:, col_o2] (explicit OH- production from O2).
 * f, hv, ngphi may each be NULL. */
TP_API int tp_interface_terms(int64_t n, const double* phi, const double* grad, double eps,
                              double k_orr, double orr_factor, int ld, const double* U,
                              int col_o2, int col_oh, double* f, double* hv, double* ngphi,
                              void* stream);

/* tp_cell_average into column `col` of an (n_cells, ld) array (per-cell, per-column
 * reaction for tp_lumped_diag). */
TP_API int tp_cell_average_col(int64_t n_cells, const int32_t* cells, const double* vert_vals,
                               int ld, int col, double* out, void* stream);

/* [sync] physics/interface_velocity.py:90-155 (compute_effective_diffusion) per vertex:
 * sat = clip(F / max(Fmax, 1e-20), 0, 1), ff = (1 - sat) + sat film_floor
 * (film_floor = porosity constrictivity / tortuosity^2); De_Zn = D0[0] ff and, where
 * phi <= 0 (medium), De_Cl/OH/O2 = D0[1..3] ff (0 in the scaffold).  Any output may be
 * NULL.  TP_ERR_NONFINITE on NaN/Inf, TP_ERR_ARG on a negative value (the reference's
 * RuntimeErrors).  flags_dev: 1 int32 of device scratch. */
TP_API int tp_effective_diffusion(int64_t n, const double* phi, const double* F, double Fmax,
                                  double film_floor, const double* D0 /* host, 4 */,
                                  double* De_zn, double* De_cl, double* De_oh, double* De_o2,
                                  int32_t* flags_dev, void* stream);

/* dissolve.py:746-755, Zn transport coefficients per vertex: medium = [phi <= 0],
 * alpha = medium kf (1 - F / Fmax), src = medium kd F Cl^2 (either output may be NULL).
 * The scaffold vertices (phi > 0) are the Dirichlet set of the Zn solve (dissolve.py:
 * 745, 764-770). */
TP_API int tp_zn_coefficients(int64_t n, const double* phi, const double* F, const double* Cl,
                              double kf, double kd, double Fmax, double* alpha, double* src,
                              void* stream);

/* domain/mesh_utils.py:450-542 (redistance, GPU branch): `iters` Sussman pseudo-time steps
 * psi += dtau sign(phi0) (1 - |grad psi|), sign(phi0) = phi0 / sqrt(phi0^2 + (eps_factor
 * h_avg)^2), dtau = h_avg / 2 / max(|grad psi|, 1/2), nodes with |phi0| < band_factor h_avg
 * frozen; |grad psi| from tp_nodal_gradient (volume-weighted, coords4).  In place on phi.
 * scratch >= tp_redistance_scratch_bytes(n_verts).  The reference uses band_factor 3 and
 * eps_factor 1.5. */
TP_API size_t tp_redistance_scratch_bytes(int64_t n_verts);
TP_API int tp_redistance(const tp_mesh* m, double* phi, int iters, double h_avg,
                         double band_factor, double eps_factor, void* scratch, void* stream);

/* domain/mesh_utils.py:367-449 (_init_phi_from_regions): the level set from cell region
 * labels (regions: n_cells int32; the scaffold cells carry scaffold_label).  Vertices of a
 * scaffold cell are inside (+), the others outside (-); phi (n_verts) = sign times the
 * distance to the nearest interface vertex (a vertex of a scaffold cell and of another
 * cell), or sign times 0.5 when there is none.  FP64 distances, each operation rounded
 * once; the nearest search is exhaustive.  scratch >= tp_phi_from_regions_scratch_bytes. */
TP_API size_t tp_phi_from_regions_scratch_bytes(int64_t n_verts);
TP_API int tp_phi_from_regions(const tp_mesh* m, const int32_t* regions, int scaffold_label,
                               double* phi, void* scratch, void* stream);

/* Sum over cells of the cell diameter (longest edge), into out_dev (1 double); divided by
 * n_cells it is the h_avg of domain/mesh_utils.py:559-575 (dolfinx mesh.h).
 * scratch >= 1024 doubles. */
TP_API int tp_mean_cell_diameter(const tp_mesh* m, double* out_dev, void* scratch, void* stream);

/* Level-set update phi -= dt rate (1 + gain U[:, col]) (the algebraic part of the
 * level-set step, dissolve.py:684-730, with the configured dissolution law). */
TP_API int tp_levelset_advance(int64_t n, double* phi, int ld, const double* U, int col,
                               double dt, double rate, double gain, void* stream);

/* y = a x + b y (n doubles): numerics/solvers.py:278-279 under-relaxation */
TP_API int tp_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream);
/* After a solve, in one pass over n values: d = x - u, u_prev = u, u = x (the step
 * increment for the projected guess and the state update; no reference counterpart) */
TP_API int tp_advance_state(int64_t n, const double* x, double* u, double* u_prev, double* d,
                            void* stream);
/* The same with n_hist (1..8) increment buffers shifted in place, newest first:
 * hist[k] = hist[k-1], hist[0] = x - u (fixed pointers: replayable in a CUDA graph);
 * ring2 (NULL or n_hist buffers, e.g. the increments' stiffness images) is shifted the
 * same way with its slot 0 left unchanged */
TP_API int tp_advance_history(int64_t n, const double* x, double* u, double* u_prev,
                              int n_hist, double* const* hist, double* const* ring2,
                              void* stream);

/* (n, S) row-major columns -> (n, ld) interleaved, padding columns zero, and back.
 * Plumbing for host arrays of S species (no reference counterpart). */
TP_API int tp_pack_columns(int64_t n, int S, int ld, const double* src, double* dst,
                           void* stream);
TP_API int tp_unpack_columns(int64_t n, int S, int ld, const double* src, double* dst,
                             void* stream);

/* ------------------------------------------------------------------ operators */
/* gpu/ceed_operators.py:87-108, 247-353 as intended, on S interleaved columns:
 * y[:, s] = sum_e [diff_scale[s] De_e K_e + (inv_dt + alpha_e + shift[s]) M_e] x_e[:, s]
 * recomputing the P1 gradients of every cell from coords4 in FP64.  legacy != 0 weights
 * the stiffness by 4 (the reference QFunction omits wdetJ, :101-104) instead of |detJ|/6.
 * fp32 != 0: x, y float (geometry still FP64).  diff_scale/shift: host, S values, or NULL.
 * y is overwritten. */
TP_API int tp_matfree_apply(const tp_mesh* m, int S, int ld, int fp32, const double* De_cell,
                     const double* alpha_cell, const double* diff_scale, const double* shift,
                     double inv_dt, int lumped, int legacy, const void* x, void* y,
                     void* stream);

/* Multi-column CSR operator: y[:, s] = dscale[s] (K x)[:, s] + cscale[s] (M x)[:, s]
 * + diag[:, s] .* x[:, s], with K and M sharing the CSR pattern (M may be NULL).
 * val32/val64 hold the same matrix in FP32/FP64 (inner and outer operator of the
 * mixed-precision solve).  Rows with bc_mask != 0 are identity rows. */
typedef struct tp_csr_op {
  int64_t n_rows;
  int32_t S;            /* columns in use, 1..4                                 */
  int32_t ld;           /* interleave stride: 1, 2 or 4                         */
  const int32_t* indptr;
  const int32_t* indices;
  const double* K64;    /* (nnz) */
  const float* K32;     /* (nnz) or NULL when the solve is FP64 only            */
  const double* M64;    /* (nnz) or NULL */
  const float* M32;
  const double* diag64; /* (n_rows, ld) or NULL */
  const float* diag32;
  const uint8_t* bc_mask; /* (n_rows) or NULL */
  double dscale[TP_MAX_COLS];
  double cscale[TP_MAX_COLS];
  /* independent systems solved together (block-diagonal union), rows contiguous:
     sys_row_ptr (n_systems + 1, host); n_systems = 1 for a single mesh */
  int32_t n_systems;
  const int64_t* sys_row_ptr;
} tp_csr_op;

/* [sync] Matrix-free Jacobi-PCG (numerics/solvers.py:172-203, 375-404: the reference's
 * PETSc KSP around the CeedDiffusionMassOp MatShell): solves A x = b for S interleaved
 * columns, A the operator of tp_matfree_apply (same arguments), every product recomputing
 * the P1 gradients from coords4; nothing is assembled.  FP64.  bc_mask (or NULL): those
 * rows are identity rows (x = b there).  rtol (host, S values): stops each lane when its
 * recurrence residual ||r||_2 <= rtol ||b||_2, then confirms it on ||b - A x||_2 (reported
 * per lane in res).  x: initial guess in, solution out.  workspace: 256-byte aligned,
 * tp_mfcg_workspace_bytes(n_verts, ld) bytes. */
typedef struct tp_mfcg_result {
  int32_t status, iterations;
  int32_t lane_status[4], lane_iters[4];
  double lane_rnorm[4], lane_bnorm[4];
} tp_mfcg_result;
TP_API size_t tp_mfcg_workspace_bytes(int64_t n_verts, int ld);
TP_API int tp_mfcg_solve(const tp_mesh* m, int S, int ld, const double* De_cell,
                         const double* alpha_cell, const double* diff_scale,
                         const double* shift, double inv_dt, int lumped, int legacy,
                         const uint8_t* bc_mask, const double* b, double* x,
                         const double* rtol, int max_it, void* workspace,
                         size_t workspace_bytes, tp_mfcg_result* res, void* stream);

/* y = A x with the FP64 (fp32 = 0) or FP32 (fp32 = 1) values of op */
TP_API int tp_csr_apply(const tp_csr_op* op, int fp32, const void* x, void* y, void* stream);

/* y1 = D K x1 and y2 = D K (x1 - x2) with the FP64 values K64 of op (D = op->dscale; no
 * mass, diagonal or identity rows) in one pass: the stiffness images of u^n and of the
 * last increment that the learned initial guess reads (no reference counterpart). */
TP_API int tp_csr_images(const tp_csr_op* op, const double* x1, const double* x2, double* y1,
                         double* y2, void* stream);

/* The initial guess projected in the energy norm (no reference counterpart; the learned
 * guess's last stage).  op: the stiffness D K (K64, dscale, S, ld); A = D K + diag (diag
 * (n_rows, ld); identity rows where bc_mask); opU = D K U (tp_csr_images).  With n_dirs
 * (0..6) directions dirs[k] ((n_rows, ld) device arrays: increments of past steps, the
 * network's correction), writes
 *   x = U + sum_k c_k dirs[k]   (free rows),   x = b   (Dirichlet rows, columns < S),
 * c per column solving the Galerkin system G c = h, G_kl = d_k . A d_l,
 * h_k = d_k . (b - A U) over the free rows (directions taken as zero on Dirichlet rows;
 * a direction numerically in the span of the earlier ones gets c_k = 0): the minimum of
 * the A-norm of the error over U + span{d_k}, so never above U in that norm.
 * imgs: NULL, or n_dirs pointers with D K dirs[k] where already computed (tp_csr_images'
 * second output, kept from earlier steps while K is unchanged) and NULL where the kernel
 * gathers it; used only without Dirichlet rows.  Deterministic.  work: device scratch of
 * tp_guess_project_workspace_doubles() doubles. */
TP_API size_t tp_guess_project_workspace_doubles(void);
TP_API int tp_guess_project(const tp_csr_op* op, const double* diag, const uint8_t* bc_mask,
                            const double* b, const double* U, const double* opU, int n_dirs,
                            const double* const* dirs, const double* const* imgs, double* x,
                            double* work, void* stream);

/* ------------------------------------------------------------------ Krylov solve */
/* Jacobi-preconditioned CG on every (system, column) lane at once, captured in a CUDA
 * graph whose device-side while loop runs until every lane converges or max_it.
 * Replaces KSP(gmres, restart 50) + PC(bjacobi) of numerics/solvers.py:322-335, 369 on
 * the symmetric free block (Dirichlet rows are identity rows; the preconditioner is zero
 * there).  Stopping rule per lane: ||b - A x||_2 <= rtol ||b||_2 in FP64.
 * inner_fp32 = 1: the iteration (operator, vectors) runs in FP32 and FP64 reliable
 * updates (x += x_inner, r = b - A x recomputed with the FP64 operator) happen whenever
 * the FP32 residual falls below `delta` times its value at the last update, or below the
 * tolerance; convergence is only ever declared on the FP64 residual.  Dot products and
 * norms accumulate in FP64 in both modes. */
typedef struct tp_cg_config {
  int32_t max_it;
  int32_t inner_fp32;
  double delta;          /* reliable-update ratio (FP32 inner); <= 0 -> 0.1         */
  int32_t group;         /* threads per CSR row: 1, 2, 4, 8 (autotuned)             */
  int32_t block;         /* threads per block: 128 or 256                           */
  int32_t rows_per_tile; /* rows per reduction tile (multiple of block/group)        */
  int32_t use_graph_loop;/* 1: conditional-node while loop; 0: host loop            */
} tp_cg_config;

typedef struct tp_cg_result {
  int32_t status;        /* TP_OK if every lane converged                            */
  int32_t iterations;    /* iterations of the longest lane                           */
  int32_t n_reliable;    /* FP64 residual recomputations                             */
  int32_t n_lanes;
} tp_cg_result;

typedef struct tp_cg_handle tp_cg_handle;

/* bytes of device workspace a handle needs */
TP_API size_t tp_cg_workspace_bytes(const tp_csr_op* op, const tp_cg_config* cfg);

/* Build a solver for fixed buffers: b (n_rows, ld) FP64 right-hand sides, x (n_rows, ld)
 * FP64 initial guess in / solution out, rtol (n_systems * S lanes, device doubles,
 * lane = system * S + column).  The op arrays, b, x, rtol and workspace must stay valid
 * and unmoved for the handle's lifetime; their contents may change between runs. */
TP_API int tp_cg_create(const tp_csr_op* op, const tp_cg_config* cfg, const double* b, double* x,
                 const double* rtol, void* workspace, size_t workspace_bytes, void* stream,
                 tp_cg_handle** out);

/* enqueue one solve (recomputes the Jacobi diagonal from the current values) */
TP_API int tp_cg_run(tp_cg_handle* h, void* stream);

/* [sync] summary of the last run, plus per-lane arrays (host, n_lanes each, any NULL) */
TP_API int tp_cg_result_get(tp_cg_handle* h, tp_cg_result* res, int32_t* lane_iters,
                     int32_t* lane_status, double* lane_rnorm, double* lane_bnorm,
                     void* stream);

TP_API int tp_cg_destroy(tp_cg_handle* h);

/* time `reps` launches of one inner SpMV+dot with the given config (autotuner support);
 * returns milliseconds per launch through *ms (host). [sync] */
TP_API int tp_cg_time_spmv(tp_cg_handle* h, int reps, float* ms, void* stream);

/* ------------------------------------------------------------------ SELL-32 operator */
/* Sliced ELL with slices of 32 rows: entry k of the 32 rows of slice s sits at
 * slice_ptr[s] + 32 k + lane, so every index/value load of a warp is one 128-byte access.
 * Rows shorter than their slice are padded with their own column and value 0.
 * (No reference counterpart: the device layout of the inner Krylov operator.) */
typedef struct tp_sell {
  int64_t n_rows;
  int64_t n_entries;         /* 32 * sum of slice widths                              */
  const int32_t* slice_ptr;  /* (ceil(n_rows/32) + 1)                                 */
  const int32_t* sell_col;   /* (n_entries)                                           */
  const float* sK32;         /* (n_entries) values of K (FP32) or NULL                */
  const double* sK64;        /* (n_entries) values of K (FP64) or NULL                */
  const float* sM32;         /* optional mass values                                  */
  const double* sM64;
} tp_sell;

/* [sync] SELL-32 pattern of a CSR pattern: slice_ptr always; sell_col and csr2sell
 * (position of each CSR entry, (nnz)) when both are non-NULL.  *n_entries (host)
 * receives the storage size; allocate sell_col and the value arrays to it, zeroed. */
TP_API int tp_sell_build(int64_t n_rows, const int32_t* indptr, const int32_t* indices,
                         int32_t* slice_ptr, int32_t* sell_col, int32_t* csr2sell,
                         int64_t* n_entries, void* stream);

/* values of a CSR matrix into SELL order (padding entries are left untouched) */
TP_API int tp_sell_scatter(int64_t nnz, const int32_t* csr2sell, const double* csr_vals,
                           float* sell32, double* sell64, void* stream);

/* ------------------------------------------------------------------ persistent solve */
/* The Jacobi-PCG of tp_cg_* for ONE system (S <= 4 columns) as a single cooperative
 * kernel: one launch per solve, grid barriers with a bounded wait (TP_ERR_TIMEOUT when a
 * barrier wait exceeds 2 s), the inner operator read in SELL-32 order, the FP64 operator
 * (Jacobi diagonal, initial / reliable-update / final residuals) in CSR.  Same stopping
 * rule and lane results as tp_cg_*.  Reliable updates (FP32 inner): when any lane's
 * recurrence residual has dropped by `delta` (<= 0 -> 0.01) since its last update, every
 * active lane is updated in the same FP64 sweep. */
typedef struct tp_pcg_handle tp_pcg_handle;

TP_API size_t tp_pcg_workspace_bytes(const tp_csr_op* op, int inner_fp32);
/* ctas_per_sm: 1 or 2 resident 512-thread CTAs per SM (0 = 1; 2 only for rows of at most
 * 8 bytes per column set, i.e. 1-2 FP32 or 1 FP64 column) */
TP_API int tp_pcg_create(const tp_csr_op* op, const tp_sell* sell, int max_it, int inner_fp32,
                         double delta, int ctas_per_sm, const double* b, double* x,
                         const double* rtol, void* workspace, size_t workspace_bytes,
                         void* stream, tp_pcg_handle** out);
TP_API int tp_pcg_run(tp_pcg_handle* h, void* stream);
TP_API int tp_pcg_result_get(tp_pcg_handle* h, tp_cg_result* res, int32_t* lane_iters,
                             int32_t* lane_status, double* lane_rnorm, double* lane_bnorm,
                             void* stream);
TP_API int tp_pcg_grid(tp_pcg_handle* h, int* grid, int* block);
/* Engine the handle runs (chosen at create).  *window = 1: the window engine -- the
 * Chronopoulos-Gear form of the same Jacobi-PCG, in which the only vector shared between
 * CTAs is u = D^-1 r; every CTA keeps u of its rows plus its halo (the columns outside its
 * row range that its rows reference) and 16-bit window-local column indices in shared
 * memory (one CTA per SM, at most 65535 window entries per CTA, the tables within the
 * per-block shared-memory limit).  *window = 2: the window engine with the operator
 * values and every per-row vector of the recurrence (p, s, xi, r) in tensor memory and
 * D^-1 in shared memory (FP32 inner iterations, no mass matrix, 2 or 4 columns, at most
 * 2048 rows per CTA, rows of at most 16 entries; DISSOLVE_PCG_CGT=0 at create keeps
 * engine 1).  *window = 3: the pipelined form of the same Jacobi-PCG (Ghysels-Vanroose,
 * one grid barrier per iteration; its FP64 refreshes restart the refreshed lanes) with
 * the same tensor-memory layout, for at most 3 columns (DISSOLVE_PCG_PIPE=0 at create keeps
 * engine 2); it refreshes at least every factor 1e3 of residual reduction whatever
 * `delta` asks for.  *window = 0: the streaming engine (standard recurrences, columns and
 * gathers from global memory).  *smem_bytes: dynamic shared memory per CTA.  The
 * environment variable DISSOLVE_PCG_ENGINE=stream at create forces the streaming
 * engine. */
TP_API int tp_pcg_engine(tp_pcg_handle* h, int* window, size_t* smem_bytes);
/* per-CTA phase times of the next runs: prof (grid * 8 device u64, ns) receives per CTA
 * [A work, A barrier wait, B work, B barrier wait, scalar updates, reliable updates,
 * final, init]; NULL switches it off */
TP_API int tp_pcg_set_profile(tp_pcg_handle* h, unsigned long long* prof);
/* Bound of every grid-barrier wait of the next runs (limit_ns; 0 restores the default of
 * 2 s) and, for tests of the failure path only, missing_arrivals (<= 1024) arrivals that
 * every barrier waits for beyond the grid's own: with missing_arrivals > 0 the first wait
 * runs out after limit_ns, the run ends with TP_ERR_TIMEOUT in its status and every
 * lane status, and the handle stays usable (set 0 again for normal runs).  The failure
 * it stands for is a CTA that never arrives; the caller's contract on any error is the
 * reference's fallback (numerics/solvers.py:264-271: catch, then solve another way). */
TP_API int tp_pcg_set_wait_limit(tp_pcg_handle* h, unsigned long long limit_ns,
                                 unsigned int missing_arrivals);
TP_API int tp_pcg_destroy(tp_pcg_handle* h);

/* ------------------------------------------------------------------ learned guess */
/* Per-vertex MLP predicting the next backward-Euler state as the Krylov initial guess
 * (no reference counterpart).  One network for all species; a row is (vertex, species).
 * Inputs (normalised: (x - mean[f]) * istd[f]): phi, |grad phi|, u^n, u^{n-1},
 * u^n - u^{n-1}, log D_s, k_s, 1; 16 -> 64 -> ReLU -> 64 -> ReLU -> 1, BF16 weights and
 * activations on the tensor cores, FP32 accumulation.  Parameters: one FP32 vector of
 * tp_mlp_param_count() floats [W1 (64x16) | b1 | W2 (64x64) | b2 | w3 (64) | b3]. */
typedef struct tp_mlp_inputs {
  int64_t n_verts;
  int32_t S, ld;
  const double* U;           /* (n_verts, ld) u^n      */
  const double* U_prev;      /* (n_verts, ld) u^{n-1}  */
  const double* phi;         /* (n_verts) or NULL       */
  const double* normgradphi; /* (n_verts) or NULL       */
  const double* opU;         /* (n_verts, ld) stiffness image D_s K u^n, or NULL        */
  const double* opDU;        /* (n_verts, ld) D_s K (u^n - u^{n-1}), or NULL           */
  double logD[4], k[4];      /* per species             */
  double mean[10], istd[10]; /* input normalisation (features 0..9) */
  int32_t base;              /* the guess the network corrects: 0 u^n, 1 2 u^n - u^{n-1},
                                2 none (tp_mlp_predict writes sigma y alone)             */
  int32_t* tc_status;        /* device int32 or NULL: tp_mlp_predict sets it to 0 before its
                                launch (on the stream) and the launch sets it to 1 when a
                                bounded tensor-core wait ran out; the rows of such a tile
                                are then not written (x_out keeps what it held)          */
} tp_mlp_inputs;

TP_API int tp_mlp_param_count(void);
/* x_out[v, s] = B[v, s] + sigma * y(v, s) (the guess, written into a solver's x), with
 * B = U (base 0), 2 U - U_prev (base 1, linear extrapolation) or 0 (base 2: the scaled
 * output alone, the direction tp_guess_project takes), or
 * y_out[v * S + s] = y when x_out is NULL */
TP_API int tp_mlp_predict(const tp_mlp_inputs* in, const float* params, float sigma,
                          double* x_out, float* y_out, void* stream);
/* [sync] *timed_out = 1 if any inference launch of this library since it was loaded gave
 * up waiting for its tensor-core operations (sticky; the per-call word is
 * tp_mlp_inputs.tc_status), else 0 */
TP_API int tp_mlp_tensor_status(int* timed_out, void* stream);
/* Polls of one mbarrier phase before an inference wait gives up (0 restores the default,
 * 2^24, about 0.1 s), for the launches that follow on any thread.  skip_issue != 0 is for
 * tests of the failure path only: the issuing thread then launches no tensor-core
 * operation and commits nothing, so every wait runs out with nothing in flight. */
TP_API int tp_mlp_set_wait_limit(unsigned int polls, int skip_issue);
/* the normalised inputs as BF16 rows of 16 (training set) */
TP_API int tp_mlp_features(const tp_mlp_inputs* in, void* X_bf16, void* stream);
/* training target (U_next - B) / sigma per row, B = U_n (U_prev NULL) or
 * 2 U_n - U_prev (the base of tp_mlp_inputs.base = 1) */
TP_API int tp_mlp_target(int64_t n_verts, int S, int ld, const double* U_n,
                         const double* U_prev, const double* U_next, double sigma, float* T,
                         void* stream);
TP_API size_t tp_mlp_grad_workspace_floats(int grid);
/* one AdamW step on rows [row0, row0 + nrows) of (X, T), loss = mean squared error.
 * grid CTAs write partial gradients into workspace (tp_mlp_grad_workspace_floats(grid)).
 * lr <= 0: gradient only (grad_out, the summed gradient, may be NULL otherwise).
 * loss_out: sum of squared errors (device float) or NULL. */
TP_API int tp_mlp_train_step(const void* X_bf16, const float* T, int64_t row0, int64_t nrows,
                             float* params, float* adam_m, float* adam_v, int step, float lr,
                             float beta1, float beta2, float eps, float weight_decay, int grid,
                             float* workspace, float* grad_out, float* loss_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DISSOLVE_TP_H */
