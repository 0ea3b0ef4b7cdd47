// tp_tiles.cu -- row tiles for the tiled assembly and operator kernels (built once).
//
// The row-owned kernels (one thread per CSR row, summing the row's cells in ascending
// order) read each cell record once per incident row: four times, each a 64-byte gather
// of its own.  A tile of R nearby rows touches far fewer distinct cells than it visits
// (2.1x fewer for R = 64 on a jittered Kuhn cube), so a tiled kernel loads the tile's
// distinct cells once, coalesced, computes their element entries into shared memory and
// sums the diagonal of each row and each owned edge from there (tp_tiles.cuh).
//
// Rows are grouped by recursive coordinate bisection (split the longest axis of the
// bounding box at a multiple of R, depth first), which keeps tiles compact on
// unstructured and jittered meshes alike; the depth-first order puts neighbouring tiles
// next to each other in the launch, so cell records shared by them stay in L2.
#include <algorithm>
#include <cstdio>
#include <functional>
#include <thread>
#include <vector>

#include "tp_tiles.cuh"

using namespace tp;

namespace {

struct Range {
  int64_t lo, hi;
};

// tiles of exactly R rows (the last one of a subtree may be smaller), depth first
void rcb(const std::vector<double>& xyz4, int R, std::vector<int32_t>& idx,
         std::vector<int64_t>& starts) {
  std::vector<Range> stack{{0, (int64_t)idx.size()}};
  while (!stack.empty()) {
    const Range r = stack.back();
    stack.pop_back();
    const int64_t n = r.hi - r.lo;
    if (n <= R) {
      if (n > 0) starts.push_back(r.lo);
      continue;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = r.lo; i < r.hi; i++) {
      const double* p = &xyz4[4 * (int64_t)idx[i]];
      for (int a = 0; a < 3; a++) {
        lo[a] = std::min(lo[a], p[a]);
        hi[a] = std::max(hi[a], p[a]);
      }
    }
    int ax = 0;
    for (int a = 1; a < 3; a++)
      if (hi[a] - lo[a] > hi[ax] - lo[ax]) ax = a;
    const int64_t ntiles = (n + R - 1) / R;
    const int64_t left = (ntiles / 2) * R;
    std::nth_element(idx.begin() + r.lo, idx.begin() + r.lo + left, idx.begin() + r.hi,
                     [&](int32_t a, int32_t b) {
                       const double pa = xyz4[4 * (int64_t)a + ax], pb = xyz4[4 * (int64_t)b + ax];
                       return pa < pb || (pa == pb && a < b);
                     });
    stack.push_back({r.lo + left, r.hi});
    stack.push_back({r.lo, r.lo + left});
  }
}

}  // namespace

static inline int tri_host(int i, int j) {
  const int lo = std::min(i, j), hi = std::max(i, j);
  static const int base[4] = {0, 4, 7, 9};
  return base[lo] + (hi - lo);
}

extern "C" int tp_tiles_create(const tp_mesh* m, int rows_per_tile, void* stream,
                               tp_tiles** out) {
  TP_REQUIRE(m && out && m->coords4 && m->v2c_ptr && m->v2c && m->v2c_slots && m->indptr &&
                 m->indices,
             "tiles need coords4, incidence, slots and the CSR pattern");
  TP_REQUIRE(rows_per_tile >= 32 && rows_per_tile <= 256 && rows_per_tile % 32 == 0,
             "rows_per_tile must be a multiple of 32 in [32, 256]");
  *out = nullptr;
  const int R = rows_per_tile;
  const int64_t nv = m->n_verts, n4 = 4 * m->n_cells, nnz = m->nnz;
  cudaStream_t st = as_stream(stream);
  std::vector<double> xyz(4 * (size_t)nv);
  std::vector<int32_t> vptr(nv + 1), v2c(n4), indptr(nv + 1), indices(nnz);
  std::vector<uint32_t> slots(n4);
  auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
  };
  TP_CUDA_TRY(d2h(xyz.data(), m->coords4, sizeof(double) * 4 * nv));
  TP_CUDA_TRY(d2h(vptr.data(), m->v2c_ptr, sizeof(int32_t) * (nv + 1)));
  TP_CUDA_TRY(d2h(indptr.data(), m->indptr, sizeof(int32_t) * (nv + 1)));
  TP_CUDA_TRY(d2h(v2c.data(), m->v2c, sizeof(int32_t) * n4));
  TP_CUDA_TRY(d2h(slots.data(), m->v2c_slots, sizeof(uint32_t) * n4));
  TP_CUDA_TRY(d2h(indices.data(), m->indices, sizeof(int32_t) * nnz));
  TP_CUDA_TRY(cudaStreamSynchronize(st));

  std::vector<int32_t> idx(nv);
  for (int64_t i = 0; i < nv; i++) idx[i] = (int32_t)i;
  std::vector<int64_t> starts;
  rcb(xyz, R, idx, starts);
  const int nt = (int)starts.size();
  auto pos_in_row = [&](int32_t row, int32_t col) -> int32_t {
    const auto b = indices.begin() + indptr[row], e = indices.begin() + indptr[row + 1];
    const auto it = std::lower_bound(b, e, col);
    return (it != e && *it == col) ? (int32_t)(it - indices.begin()) : -1;
  };
  std::vector<int32_t> rows((size_t)nt * R, -1), dpos((size_t)nt * R, -1);
  std::vector<int32_t> cell_ptr(nt + 1, 0), dterm_ptr(nt + 1, 0), edge_ptr(nt + 1, 0),
      eterm_ptr(nt + 1, 0);
  // Tiles are independent: contiguous tile ranges are built on host threads into local
  // buffers (per-tile sizes in the *_ptr slots), then concatenated in tile order, so the
  // tables are the same whatever the thread count.
  struct Local {
    std::vector<int32_t> cells;
    std::vector<uint16_t> dterms, eterms;
    std::vector<int2> edges, edge_rv;
    int max_cells = 0, max_edges = 0, rc = TP_OK;
    char msg[160] = {0};
  };
  auto build_range = [&](int t0, int t1, Local& L) {
    std::vector<int32_t> tc;
    std::vector<std::vector<uint16_t>> eterm_lists;  // per owned edge of the tile
    std::vector<int32_t> slot_edge(256);
    auto fail = [&](int rc, const char* msg) {
      L.rc = rc;
      snprintf(L.msg, sizeof(L.msg), "%s", msg);
    };
    for (int t = t0; t < t1; t++) {
      const int64_t b = starts[t], e = (t + 1 < nt) ? starts[t + 1] : nv;
      // rows of the tile ascending (writes then walk the CSR forward)
      std::sort(idx.begin() + b, idx.begin() + e);
      tc.clear();
      int kmax = 0;
      for (int64_t i = b; i < e; i++) {
        const int32_t r = idx[i];
        rows[(size_t)t * R + (i - b)] = r;
        dpos[(size_t)t * R + (i - b)] = pos_in_row(r, r);
        kmax = std::max(kmax, vptr[r + 1] - vptr[r]);
        for (int k = vptr[r]; k < vptr[r + 1]; k++) tc.push_back(v2c[k] >> 2);
      }
      std::sort(tc.begin(), tc.end());
      tc.erase(std::unique(tc.begin(), tc.end()), tc.end());
      if (tc.size() >= (1u << TILE_LOC_BITS)) {
        char m[160];
        snprintf(m, sizeof(m), "tile %d touches %zu cells (at most %d)", t, tc.size(),
                 (1 << TILE_LOC_BITS) - 1);
        return fail(TP_ERR_CAPACITY, m);
      }
      L.max_cells = std::max(L.max_cells, (int)tc.size());
      L.cells.insert(L.cells.end(), tc.begin(), tc.end());
      cell_ptr[t + 1] = (int32_t)tc.size();
      // diagonal terms [row][k]; owned edges and their terms
      const int KD = (kmax + 7) & ~7;
      const size_t dbase = L.dterms.size();
      L.dterms.resize(dbase + (size_t)KD * R, TILE_TERM_NONE);
      eterm_lists.clear();
      const size_t ebase = L.edges.size();
      for (int64_t i = b; i < e; i++) {
        const int32_t r = idx[i];
        const int32_t p0 = indptr[r], len = indptr[r + 1] - p0;
        if (len > 256) {
          char m[160];
          snprintf(m, sizeof(m), "row %d has %d entries (tiles support 256)", r, len);
          return fail(TP_ERR_CAPACITY, m);
        }
        std::fill(slot_edge.begin(), slot_edge.begin() + len, -1);
        for (int k = vptr[r]; k < vptr[r + 1]; k++) {
          const int32_t c = v2c[k] >> 2;
          const int li = v2c[k] & 3;
          const uint16_t loc = (uint16_t)(std::lower_bound(tc.begin(), tc.end(), c) - tc.begin());
          L.dterms[dbase + (size_t)(i - b) * KD + (k - vptr[r])] =
              (uint16_t)(loc | (li << TILE_LOC_BITS));
          for (int j = 0; j < 4; j++) {
            if (j == li) continue;
            const int sl = (slots[k] >> (8 * j)) & 0xff;
            if (sl >= len) {
              char m[160];
              snprintf(m, sizeof(m), "incidence slot %d outside row %d", sl, r);
              return fail(TP_ERR_INDEX, m);
            }
            const int32_t v = indices[p0 + sl];
            if (v < r) continue;  // owned by v's tile
            if (slot_edge[sl] < 0) {
              slot_edge[sl] = (int32_t)eterm_lists.size();
              eterm_lists.emplace_back();
              const int32_t q = pos_in_row(v, r);
              if (q < 0) {
                char m[160];
                snprintf(m, sizeof(m), "pattern is not symmetric at (%d, %d)", r, v);
                return fail(TP_ERR_INDEX, m);
              }
              L.edges.push_back(make_int2(p0 + sl, q));
              L.edge_rv.push_back(make_int2(r, v));
            }
            eterm_lists[slot_edge[sl]].push_back(
                (uint16_t)(loc | (tri_host(li, j) << TILE_LOC_BITS)));
          }
        }
      }
      dterm_ptr[t + 1] = (int32_t)(L.dterms.size() - dbase);
      const int ne = (int)(L.edges.size() - ebase);
      L.max_edges = std::max(L.max_edges, ne);
      edge_ptr[t + 1] = ne;
      size_t ke = 0;
      for (const auto& l : eterm_lists) ke = std::max(ke, l.size());
      const size_t KE = (ke + 7) & ~(size_t)7;
      const size_t tbase = L.eterms.size();
      L.eterms.resize(tbase + KE * (size_t)ne, TILE_TERM_NONE);
      for (int q = 0; q < ne; q++)
        for (size_t k = 0; k < eterm_lists[q].size(); k++)
          L.eterms[tbase + (size_t)q * KE + k] = eterm_lists[q][k];
      eterm_ptr[t + 1] = (int32_t)(KE * (size_t)ne);
    }
  };
  const int nthreads =
      (int)std::max(1u, std::min(16u, std::min((unsigned)std::max(nt / 64, 1),
                                               std::thread::hardware_concurrency())));
  std::vector<Local> locals(nthreads);
  {
    std::vector<std::thread> pool;
    for (int k = 0; k < nthreads; k++) {
      const int t0 = (int)((int64_t)nt * k / nthreads), t1 = (int)((int64_t)nt * (k + 1) / nthreads);
      pool.emplace_back(build_range, t0, t1, std::ref(locals[k]));
    }
    for (auto& th : pool) th.join();
  }
  std::vector<int32_t> cells;
  std::vector<uint16_t> dterms, eterms;
  std::vector<int2> edges, edge_rv;
  int max_cells = 0, max_edges = 0;
  for (auto& L : locals) {
    if (L.rc != TP_OK) {
      set_error("%s", L.msg);
      return L.rc;
    }
    cells.insert(cells.end(), L.cells.begin(), L.cells.end());
    dterms.insert(dterms.end(), L.dterms.begin(), L.dterms.end());
    eterms.insert(eterms.end(), L.eterms.begin(), L.eterms.end());
    edges.insert(edges.end(), L.edges.begin(), L.edges.end());
    edge_rv.insert(edge_rv.end(), L.edge_rv.begin(), L.edge_rv.end());
    max_cells = std::max(max_cells, L.max_cells);
    max_edges = std::max(max_edges, L.max_edges);
  }
  if (eterms.size() > (size_t)INT32_MAX || dterms.size() > (size_t)INT32_MAX ||
      cells.size() > (size_t)INT32_MAX) {
    set_error("tile terms exceed int32 offsets");
    return TP_ERR_CAPACITY;
  }
  // per-tile sizes -> offsets
  for (int t = 0; t < nt; t++) {
    cell_ptr[t + 1] += cell_ptr[t];
    dterm_ptr[t + 1] += dterm_ptr[t];
    edge_ptr[t + 1] += edge_ptr[t];
    eterm_ptr[t + 1] += eterm_ptr[t];
  }

  tp_tiles* h = new tp_tiles();
  auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  struct Part {
    const void* src;
    size_t bytes;
  };
  const Part parts[] = {
      {rows.data(), sizeof(int32_t) * rows.size()},
      {dpos.data(), sizeof(int32_t) * dpos.size()},
      {cell_ptr.data(), sizeof(int32_t) * cell_ptr.size()},
      {cells.data(), sizeof(int32_t) * cells.size()},
      {dterm_ptr.data(), sizeof(int32_t) * dterm_ptr.size()},
      {dterms.data(), sizeof(uint16_t) * dterms.size()},
      {edge_ptr.data(), sizeof(int32_t) * edge_ptr.size()},
      {edges.data(), sizeof(int2) * edges.size()},
      {edge_rv.data(), sizeof(int2) * edge_rv.size()},
      {eterm_ptr.data(), sizeof(int32_t) * eterm_ptr.size()},
      {eterms.data(), sizeof(uint16_t) * eterms.size()},
  };
  constexpr int NP = sizeof(parts) / sizeof(parts[0]);
  for (const Part& q : parts) h->bytes += a256(std::max<size_t>(q.bytes, 1));
  cudaError_t err = cudaMalloc(&h->dmem, h->bytes);
  if (err != cudaSuccess) {
    set_error("tiles: cudaMalloc of %zu bytes failed: %s", h->bytes, cudaGetErrorString(err));
    h->dmem = nullptr;
    delete h;
    return TP_ERR_CUDA;
  }
  void* dst[NP];
  char* p = static_cast<char*>(h->dmem);
  for (int i = 0; i < NP && err == cudaSuccess; i++) {
    dst[i] = p;
    if (parts[i].bytes)
      err = cudaMemcpyAsync(p, parts[i].src, parts[i].bytes, cudaMemcpyHostToDevice, st);
    p += a256(std::max<size_t>(parts[i].bytes, 1));
  }
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) {
    delete h;
    set_error("tiles upload failed: %s", cudaGetErrorString(err));
    return TP_ERR_CUDA;
  }
  TileView& v = h->v;
  v.R = R;
  v.n_tiles = nt;
  v.max_cells = max_cells;
  v.max_edges = max_edges;
  v.rows = static_cast<const int32_t*>(dst[0]);
  v.diag_pos = static_cast<const int32_t*>(dst[1]);
  v.cell_ptr = static_cast<const int32_t*>(dst[2]);
  v.cells = static_cast<const int32_t*>(dst[3]);
  v.dterm_ptr = static_cast<const int32_t*>(dst[4]);
  v.dterms = static_cast<const uint16_t*>(dst[5]);
  v.edge_ptr = static_cast<const int32_t*>(dst[6]);
  v.edge_pos = static_cast<const int2*>(dst[7]);
  v.edge_rv = static_cast<const int2*>(dst[8]);
  v.eterm_ptr = static_cast<const int32_t*>(dst[9]);
  v.eterms = static_cast<const uint16_t*>(dst[10]);
  h->n_terms = (int64_t)dterms.size() + (int64_t)eterms.size();
  *out = h;
  return TP_OK;
}

extern "C" int tp_tiles_info(const tp_tiles* t, int32_t* n_tiles, int32_t* rows_per_tile,
                             int32_t* max_cells, int64_t* n_entries, size_t* device_bytes) {
  TP_REQUIRE(t, "null tiles");
  if (n_tiles) *n_tiles = t->v.n_tiles;
  if (rows_per_tile) *rows_per_tile = t->v.R;
  if (max_cells) *max_cells = t->v.max_cells;
  if (n_entries) *n_entries = t->n_terms;
  if (device_bytes) *device_bytes = t->bytes;
  return TP_OK;
}

extern "C" int tp_tiles_destroy(tp_tiles* t) {
  delete t;
  return TP_OK;
}
