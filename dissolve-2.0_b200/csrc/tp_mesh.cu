// tp_mesh.cu -- one-time mesh setup on the GPU: per-cell geometry, vertex->cell
// incidence, CSR sparsity pattern, scatter map and the row-local slot map.
//
// The reference builds all of this on the host (gpu/gpu_assembler.py:376-438): numpy
// geometry, a Python set per row for the pattern and a dict over nnz plus a triple loop
// over cells x 16 for the scatter map (tens of seconds at 1.5M cells).  Here every step
// is a kernel; the pattern is produced row-parallel with no sort of the 16 n pairs:
// each row deduplicates the vertices of its incident cells in shared memory.
#include <algorithm>
#include <vector>

#include "tp_common.cuh"

namespace tp {

// ----------------------------------------------------------------- geometry
// J = [x1-x0 | x2-x0 | x3-x0] (columns are edges).  Rows of J^-1 are the cross
// products (e2 x e3, e3 x e1, e1 x e2) / det J.
__global__ void k_cell_geometry(int64_t n, int64_t nv, const int4* __restrict__ cells,
                                const double* __restrict__ coords, double* __restrict__ geo,
                                double* __restrict__ detJ, double* __restrict__ Gflat,
                                double* __restrict__ JinvT, int32_t* __restrict__ flags) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const int vv[4] = {v.x, v.y, v.z, v.w};
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 4; k++) bad |= (vv[k] < 0) || (vv[k] >= nv);
    if (bad) {
      atomicOr(flags, FLAG_INDEX);
      continue;
    }
    double x[4][3];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      x[k][0] = coords[3 * (int64_t)vv[k] + 0];
      x[k][1] = coords[3 * (int64_t)vv[k] + 1];
      x[k][2] = coords[3 * (int64_t)vv[k] + 2];
    }
    double e[3][3];  // e[k] = x[k+1] - x[0]
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int d = 0; d < 3; d++) e[k][d] = x[k + 1][d] - x[0][d];
    double cr[3][3];  // rows of adj(J): e2 x e3, e3 x e1, e1 x e2
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
    if (!(det != 0.0) || !isfinite(det)) {
      atomicOr(flags, FLAG_DEGENERATE);
      continue;
    }
    const double inv = 1.0 / det;
    double Ji[3][3];  // J^-1 rows
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int d = 0; d < 3; d++) Ji[a][d] = cr[a][d] * inv;
    double G[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
        G[a][b] = Ji[a][0] * Ji[b][0] + Ji[a][1] * Ji[b][1] + Ji[a][2] * Ji[b][2];
    const double adet = fabs(det);
    double4* g4 = reinterpret_cast<double4*>(geo + 8 * c);
    g4[0] = make_double4(G[0][0], G[0][1], G[0][2], G[1][1]);
    g4[1] = make_double4(G[1][2], G[2][2], adet, 0.0);
    if (detJ) detJ[c] = adet;
    if (Gflat) {
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) Gflat[9 * c + 3 * a + b] = G[a][b];
    }
    if (JinvT) {
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) JinvT[9 * c + 3 * a + b] = Ji[b][a];
    }
  }
}

__global__ void k_pad_coords(int64_t nv, const double* __restrict__ xyz,
                             double* __restrict__ c4) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    reinterpret_cast<double4*>(c4)[i] =
        make_double4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0);
  }
}

__global__ void k_pack_geometry(int64_t n, const double* __restrict__ detJ,
                                const double* __restrict__ Gflat, double* __restrict__ geo) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double* G = Gflat + 9 * c;
    double4* g4 = reinterpret_cast<double4*>(geo + 8 * c);
    g4[0] = make_double4(G[0], G[1], G[2], G[4]);
    g4[1] = make_double4(G[5], G[8], detJ[c], 0.0);
  }
}

// ----------------------------------------------------------------- scan
// exclusive scan of n int32 counts into n+1 int32 offsets, via int64 block sums
constexpr int SCAN_T = 256, SCAN_I = 8, SCAN_B = SCAN_T * SCAN_I;

__global__ void k_scan_blocksums(int64_t n, const int32_t* __restrict__ in,
                                 int64_t* __restrict__ bsum) {
  __shared__ double sh[SCAN_T / 32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_B;
  double s = 0;
  for (int k = threadIdx.x; k < SCAN_B; k += SCAN_T) {
    const int64_t i = base + k;
    if (i < n) s += (double)in[i];
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) bsum[blockIdx.x] = (int64_t)s;
}

__global__ void k_scan_offsets(int64_t nb, int64_t* __restrict__ bsum) {
  // one block: sequential chunks of SCAN_T with a running carry
  __shared__ int64_t sh[SCAN_T];
  int64_t carry = 0;
  for (int64_t base = 0; base < nb; base += SCAN_T) {
    const int64_t i = base + threadIdx.x;
    int64_t v = (i < nb) ? bsum[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < SCAN_T; o <<= 1) {
      int64_t t = (threadIdx.x >= (unsigned)o) ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    const int64_t incl = sh[threadIdx.x];
    if (i < nb) bsum[i] = carry + incl - v;
    __syncthreads();
    carry += sh[SCAN_T - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void k_scan_apply(int64_t n, const int32_t* __restrict__ in,
                             const int64_t* __restrict__ boff, int32_t* __restrict__ out,
                             int32_t* __restrict__ flags) {
  __shared__ int64_t sh[SCAN_T];
  const int64_t base = (int64_t)blockIdx.x * SCAN_B + (int64_t)threadIdx.x * SCAN_I;
  int64_t loc[SCAN_I];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_I; k++) {
    const int64_t i = base + k;
    loc[k] = s;
    s += (i < n) ? in[i] : 0;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < SCAN_T; o <<= 1) {
    int64_t t = (threadIdx.x >= (unsigned)o) ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  const int64_t off = boff[blockIdx.x] + sh[threadIdx.x] - s;
#pragma unroll
  for (int k = 0; k < SCAN_I; k++) {
    const int64_t i = base + k;
    if (i < n) {
      const int64_t v = off + loc[k];
      if (v > INT32_MAX) atomicOr(flags, FLAG_ROWCAP);
      out[i] = (int32_t)v;
    }
  }
}

__global__ void k_scan_total(int64_t n, int64_t nb, const int64_t* __restrict__ boff,
                             int32_t* __restrict__ out, int32_t* __restrict__ flags) {
  const int64_t t = boff[nb];
  if (t > INT32_MAX) atomicOr(flags, FLAG_ROWCAP);
  out[n] = (int32_t)t;
}

// scratch layout helpers ---------------------------------------------------------
struct Scratch {
  int64_t* bsum;     // blocks + 1
  int32_t* cnt;      // n_verts (counts / cursors)
  int32_t* flags;    // 4
  double* red;       // reduction partials (1024)
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static Scratch carve(void* base, int64_t n_cells, int64_t nv) {
  (void)n_cells;
  char* p = static_cast<char*>(base);
  Scratch s;
  const int64_t nb = (nv + SCAN_B - 1) / SCAN_B + 1;
  s.bsum = reinterpret_cast<int64_t*>(p);
  p += align256(sizeof(int64_t) * (nb + 1));
  s.cnt = reinterpret_cast<int32_t*>(p);
  p += align256(sizeof(int32_t) * (nv + 1));
  s.flags = reinterpret_cast<int32_t*>(p);
  p += align256(sizeof(int32_t) * 4);
  s.red = reinterpret_cast<double*>(p);
  return s;
}

static int exclusive_scan(int64_t n, const int32_t* in, int32_t* out, const Scratch& s,
                          cudaStream_t st) {
  const int64_t nb = (n + SCAN_B - 1) / SCAN_B;
  if (nb > 0) {
    k_scan_blocksums<<<(unsigned)nb, SCAN_T, 0, st>>>(n, in, s.bsum);
    TP_LAUNCH_CHECK();
  }
  k_scan_offsets<<<1, SCAN_T, 0, st>>>(nb, s.bsum);
  TP_LAUNCH_CHECK();
  if (nb > 0) {
    k_scan_apply<<<(unsigned)nb, SCAN_T, 0, st>>>(n, in, s.bsum, out, s.flags);
    TP_LAUNCH_CHECK();
  }
  k_scan_total<<<1, 1, 0, st>>>(n, nb, s.bsum, out, s.flags);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

static int read_flags(const int32_t* flags, cudaStream_t st, int32_t* out) {
  TP_CUDA_TRY(cudaMemcpyAsync(out, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  return TP_OK;
}

// ----------------------------------------------------------------- incidence
__global__ void k_inc_count(int64_t n, int64_t nv, const int4* __restrict__ cells,
                            int32_t* __restrict__ cnt, int32_t* __restrict__ flags) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const int vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (vv[k] < 0 || vv[k] >= nv) {
        atomicOr(flags, FLAG_INDEX);
        continue;
      }
      atomicAdd(&cnt[vv[k]], 1);
    }
  }
}

__global__ void k_inc_fill(int64_t n, const int4* __restrict__ cells,
                           const int32_t* __restrict__ ptr, int32_t* __restrict__ cursor,
                           int32_t* __restrict__ v2c) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int4 v = cells[c];
    const int vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int pos = ptr[vv[k]] + atomicAdd(&cursor[vv[k]], 1);
      v2c[pos] = (int32_t)(c * 4 + k);
    }
  }
}

// per-vertex insertion sort: lists are short (mesh vertex degree)
__global__ void k_inc_sort(int64_t nv, const int32_t* __restrict__ ptr,
                           int32_t* __restrict__ v2c) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int lo = ptr[v], hi = ptr[v + 1];
    for (int i = lo + 1; i < hi; i++) {
      const int32_t key = v2c[i];
      int j = i - 1;
      while (j >= lo && v2c[j] > key) {
        v2c[j + 1] = v2c[j];
        j--;
      }
      v2c[j + 1] = key;
    }
  }
}

__global__ void k_max_i32(int64_t n, const int32_t* __restrict__ ptr,
                          int32_t* __restrict__ out) {
  int32_t m = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    m = max(m, ptr[v + 1] - ptr[v]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ----------------------------------------------------------------- pattern
// One warp per row.  Candidates = the 4 vertices of every incident cell; a candidate is
// kept if no earlier candidate has the same id; its column rank is the number of kept
// candidates with a smaller id.  cap = 4 * max_degree entries of shared memory per warp.
template <bool FILL>
__global__ void k_pattern_rows(int64_t nv, const int32_t* __restrict__ cells,
                               const int32_t* __restrict__ v2c_ptr,
                               const int32_t* __restrict__ v2c, int cap,
                               int32_t* __restrict__ row_cnt, const int32_t* __restrict__ indptr,
                               int32_t* __restrict__ indices) {
  extern __shared__ int32_t smem[];
  const int wpb = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int32_t* buf = smem + (size_t)w * cap * 2;
  int32_t* keep = buf + cap;
  for (int64_t r = (int64_t)blockIdx.x * wpb + w; r < nv; r += (int64_t)gridDim.x * wpb) {
    const int lo = v2c_ptr[r], deg = v2c_ptr[r + 1] - lo, m = 4 * deg;
    for (int k = lane; k < m; k += 32) {
      const int32_t e = v2c[lo + (k >> 2)];
      buf[k] = cells[(int64_t)(e >> 2) * 4 + (k & 3)];
    }
    __syncwarp();
    int cnt = 0;
    for (int k = lane; k < m; k += 32) {
      const int32_t v = buf[k];
      int first = 1;
      for (int j = 0; j < k; j++)
        if (buf[j] == v) {
          first = 0;
          break;
        }
      keep[k] = first;
      cnt += first;
    }
    __syncwarp();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (!FILL) {
      if (lane == 0) row_cnt[r] = cnt;
    } else {
      const int base = indptr[r];
      for (int k = lane; k < m; k += 32) {
        if (!keep[k]) continue;
        const int32_t v = buf[k];
        int rank = 0;
        for (int j = 0; j < m; j++) rank += (keep[j] && buf[j] < v);
        indices[base + rank] = v;
      }
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------- scatter map & slots
__device__ __forceinline__ int find_col(const int32_t* __restrict__ idx, int lo, int hi,
                                        int32_t col) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (idx[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void k_scatter_map(int64_t n, const int32_t* __restrict__ cells,
                              const int32_t* __restrict__ indptr,
                              const int32_t* __restrict__ indices, int32_t* __restrict__ sm) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 4 * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t >> 2;
    const int i = (int)(t & 3);
    const int row = cells[c * 4 + i];
    const int lo = indptr[row], hi = indptr[row + 1];
    int4 out;
    out.x = find_col(indices, lo, hi, cells[c * 4 + 0]);
    out.y = find_col(indices, lo, hi, cells[c * 4 + 1]);
    out.z = find_col(indices, lo, hi, cells[c * 4 + 2]);
    out.w = find_col(indices, lo, hi, cells[c * 4 + 3]);
    reinterpret_cast<int4*>(sm)[t] = out;
  }
}

__global__ void k_inc_slots(int64_t nv, const int32_t* __restrict__ cells,
                            const int32_t* __restrict__ v2c_ptr,
                            const int32_t* __restrict__ v2c, const int32_t* __restrict__ indptr,
                            const int32_t* __restrict__ indices, uint32_t* __restrict__ slots,
                            int32_t* __restrict__ flags) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nv;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int lo = indptr[r], hi = indptr[r + 1];
    if (hi - lo > 255) atomicOr(flags, FLAG_ROWCAP);
    for (int k = v2c_ptr[r]; k < v2c_ptr[r + 1]; k++) {
      const int64_t c = v2c[k] >> 2;
      uint32_t packed = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int32_t col = cells[c * 4 + j];
        const int at = find_col(indices, lo, hi, col);
        int pos = at - lo;
        if (at >= hi || indices[at] != col || pos > 254) {
          atomicOr(flags, FLAG_ROWCAP);  // pattern does not hold the cell: never index by it
          pos = 255;
        }
        packed |= (uint32_t)(pos & 0xff) << (8 * j);
      }
      slots[k] = packed;
    }
  }
}

static int flags_to_status(int32_t f) {
  if (f & FLAG_INDEX) {
    set_error("cell connectivity holds a vertex id outside [0, n_verts)");
    return TP_ERR_INDEX;
  }
  if (f & FLAG_DEGENERATE) {
    set_error("a cell has det J == 0 or non-finite coordinates");
    return TP_ERR_DEGENERATE;
  }
  if (f & FLAG_ROWCAP) {
    set_error("a CSR row exceeds 255 entries or nnz exceeds int32");
    return TP_ERR_CAPACITY;
  }
  if (f & FLAG_BCINDEX) {
    set_error("a Dirichlet dof is outside [0, n_verts)");
    return TP_ERR_INDEX;
  }
  return TP_OK;
}

}  // namespace tp

using namespace tp;

extern "C" int tp_cell_geometry(int64_t n_cells, int64_t n_verts, const int32_t* cells,
                                const double* coords, double* coords4, double* geo,
                                double* detJ, double* Gflat, double* JinvT,
                                int32_t* flags_dev, void* stream) {
  TP_REQUIRE(n_cells >= 0 && n_verts >= 0, "negative size");
  TP_REQUIRE(cells && coords && geo && flags_dev, "null pointer");
  TP_REQUIRE(((uintptr_t)cells & 15) == 0 && ((uintptr_t)geo & 31) == 0,
             "cells must be 16-byte and geo 32-byte aligned");
  cudaStream_t st = as_stream(stream);
  TP_CUDA_TRY(cudaMemsetAsync(flags_dev, 0, sizeof(int32_t), st));
  if (coords4) {
    TP_REQUIRE(((uintptr_t)coords4 & 31) == 0, "coords4 must be 32-byte aligned");
    if (n_verts > 0) {
      k_pad_coords<<<grid_for(n_verts, 256, 65535), 256, 0, st>>>(n_verts, coords, coords4);
      TP_LAUNCH_CHECK();
    }
  }
  if (n_cells > 0) {
    k_cell_geometry<<<grid_for(n_cells, 128, 65535), 128, 0, st>>>(
        n_cells, n_verts, reinterpret_cast<const int4*>(cells), coords, geo, detJ, Gflat, JinvT,
        flags_dev);
    TP_LAUNCH_CHECK();
  }
  int32_t f = 0;
  int rc = read_flags(flags_dev, st, &f);
  if (rc) return rc;
  return flags_to_status(f);
}

extern "C" int tp_pack_geometry(int64_t n_cells, const double* detJ, const double* Gflat,
                                double* geo, void* stream) {
  TP_REQUIRE(detJ && Gflat && geo, "null pointer");
  TP_REQUIRE(((uintptr_t)geo & 31) == 0, "geo must be 32-byte aligned");
  cudaStream_t st = as_stream(stream);
  if (n_cells > 0) {
    k_pack_geometry<<<grid_for(n_cells, 256, 65535), 256, 0, st>>>(n_cells, detJ, Gflat, geo);
    TP_LAUNCH_CHECK();
  }
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  return TP_OK;
}

extern "C" size_t tp_setup_scratch_bytes(int64_t n_cells, int64_t n_verts) {
  (void)n_cells;
  const int64_t nb = (n_verts + SCAN_B - 1) / SCAN_B + 1;
  return align256(sizeof(int64_t) * (nb + 1)) + align256(sizeof(int32_t) * (n_verts + 1)) +
         align256(sizeof(int32_t) * 4) + align256(sizeof(double) * 4096);
}

extern "C" int tp_incidence(int64_t n_cells, int64_t n_verts, const int32_t* cells,
                            int32_t* v2c_ptr, int32_t* v2c, void* scratch,
                            int32_t* max_degree_out, void* stream) {
  TP_REQUIRE(cells && v2c_ptr && v2c && scratch, "null pointer");
  TP_REQUIRE(n_cells * 4 < INT32_MAX, "too many cells for int32 incidence ids");
  cudaStream_t st = as_stream(stream);
  Scratch s = carve(scratch, n_cells, n_verts);
  TP_CUDA_TRY(cudaMemsetAsync(s.flags, 0, sizeof(int32_t) * 4, st));
  TP_CUDA_TRY(cudaMemsetAsync(s.cnt, 0, sizeof(int32_t) * (n_verts + 1), st));
  if (n_cells > 0) {
    k_inc_count<<<grid_for(n_cells, 256, 65535), 256, 0, st>>>(
        n_cells, n_verts, reinterpret_cast<const int4*>(cells), s.cnt, s.flags);
    TP_LAUNCH_CHECK();
  }
  int32_t f = 0;
  int rc = read_flags(s.flags, st, &f);
  if (rc) return rc;
  if (f) return flags_to_status(f);
  rc = exclusive_scan(n_verts, s.cnt, v2c_ptr, s, st);
  if (rc) return rc;
  TP_CUDA_TRY(cudaMemsetAsync(s.cnt, 0, sizeof(int32_t) * (n_verts + 1), st));
  if (n_cells > 0) {
    k_inc_fill<<<grid_for(n_cells, 256, 65535), 256, 0, st>>>(
        n_cells, reinterpret_cast<const int4*>(cells), v2c_ptr, s.cnt, v2c);
    TP_LAUNCH_CHECK();
  }
  if (n_verts > 0) {
    k_inc_sort<<<grid_for(n_verts, 128, 65535), 128, 0, st>>>(n_verts, v2c_ptr, v2c);
    TP_LAUNCH_CHECK();
  }
  TP_CUDA_TRY(cudaMemsetAsync(s.flags + 1, 0, sizeof(int32_t), st));
  if (n_verts > 0) {
    k_max_i32<<<grid_for(n_verts, 256, 1024), 256, 0, st>>>(n_verts, v2c_ptr, s.flags + 1);
    TP_LAUNCH_CHECK();
  }
  int32_t md = 0;
  TP_CUDA_TRY(cudaMemcpyAsync(&md, s.flags + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  if (max_degree_out) *max_degree_out = md;
  return TP_OK;
}

extern "C" int tp_pattern(int64_t n_cells, int64_t n_verts, const int32_t* cells,
                          const int32_t* v2c_ptr, const int32_t* v2c, int32_t max_degree,
                          int32_t* indptr, int32_t* indices, void* scratch, int64_t* nnz_out,
                          int32_t* max_row_len_out, void* stream) {
  (void)n_cells;
  TP_REQUIRE(cells && v2c_ptr && v2c && indptr && scratch, "null pointer");
  TP_REQUIRE(max_degree >= 0, "bad max_degree");
  cudaStream_t st = as_stream(stream);
  Scratch s = carve(scratch, n_cells, n_verts);
  const int cap = 4 * std::max(max_degree, 1);
  const int wpb = 4;
  const size_t smem = sizeof(int32_t) * (size_t)cap * 2 * wpb;
  if (smem > 200 * 1024) {
    set_error("vertex degree %d too large for the pattern kernel", max_degree);
    return TP_ERR_CAPACITY;
  }
  if (smem > 48 * 1024) {
    TP_CUDA_TRY(cudaFuncSetAttribute(k_pattern_rows<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TP_CUDA_TRY(cudaFuncSetAttribute(k_pattern_rows<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  const int grid = grid_for(n_verts, wpb, 1 << 20);
  if (!indices) {
    TP_CUDA_TRY(cudaMemsetAsync(s.flags, 0, sizeof(int32_t) * 4, st));
    if (n_verts > 0) {
      k_pattern_rows<false><<<grid, 32 * wpb, smem, st>>>(n_verts, cells, v2c_ptr, v2c, cap,
                                                         s.cnt, nullptr, nullptr);
      TP_LAUNCH_CHECK();
    }
    int rc = exclusive_scan(n_verts, s.cnt, indptr, s, st);
    if (rc) return rc;
    TP_CUDA_TRY(cudaMemsetAsync(s.flags + 1, 0, sizeof(int32_t), st));
    if (n_verts > 0) {
      k_max_i32<<<grid_for(n_verts, 256, 1024), 256, 0, st>>>(n_verts, indptr, s.flags + 1);
      TP_LAUNCH_CHECK();
    }
    int32_t hdr[2] = {0, 0};
    TP_CUDA_TRY(cudaMemcpyAsync(hdr, s.flags, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    int32_t nnz = 0;
    TP_CUDA_TRY(cudaMemcpyAsync(&nnz, indptr + n_verts, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
    TP_CUDA_TRY(cudaStreamSynchronize(st));
    if (hdr[0]) return flags_to_status(hdr[0]);
    if (nnz_out) *nnz_out = nnz;
    if (max_row_len_out) *max_row_len_out = hdr[1];
    if (hdr[1] > 255) {
      set_error("CSR row of %d entries exceeds the 255-slot limit", hdr[1]);
      return TP_ERR_CAPACITY;
    }
    return TP_OK;
  }
  if (n_verts > 0) {
    k_pattern_rows<true><<<grid, 32 * wpb, smem, st>>>(n_verts, cells, v2c_ptr, v2c, cap,
                                                      nullptr, indptr, indices);
    TP_LAUNCH_CHECK();
  }
  TP_CUDA_TRY(cudaStreamSynchronize(st));
  return TP_OK;
}

extern "C" int tp_scatter_map(int64_t n_cells, const int32_t* cells, const int32_t* indptr,
                              const int32_t* indices, int32_t* scatter_map, void* stream) {
  TP_REQUIRE(cells && indptr && indices && scatter_map, "null pointer");
  TP_REQUIRE(((uintptr_t)scatter_map & 15) == 0, "scatter_map must be 16-byte aligned");
  if (n_cells == 0) return TP_OK;
  k_scatter_map<<<grid_for(4 * n_cells, 256, 65535), 256, 0, as_stream(stream)>>>(
      n_cells, cells, indptr, indices, scatter_map);
  TP_LAUNCH_CHECK();
  return TP_OK;
}

extern "C" int tp_incidence_slots(const tp_mesh* m, uint32_t* slots, int32_t* flags_dev,
                                  void* stream) {
  TP_REQUIRE(m && slots && flags_dev && m->cells && m->v2c_ptr && m->v2c && m->indptr &&
                 m->indices,
             "null pointer");
  cudaStream_t st = as_stream(stream);
  TP_CUDA_TRY(cudaMemsetAsync(flags_dev, 0, sizeof(int32_t), st));
  if (m->n_verts > 0) {
    k_inc_slots<<<grid_for(m->n_verts, 128, 65535), 128, 0, st>>>(
        m->n_verts, m->cells, m->v2c_ptr, m->v2c, m->indptr, m->indices, slots, flags_dev);
    TP_LAUNCH_CHECK();
  }
  int32_t f = 0;
  int rc = read_flags(flags_dev, st, &f);
  if (rc) return rc;
  return flags_to_status(f);
}
