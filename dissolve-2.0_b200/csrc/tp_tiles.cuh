// tp_tiles.cuh -- row tiles of a mesh, as the tiled kernels see them.
//
// A tile is a group of R nearby rows (vertices).  Its cells are the distinct cells the
// rows touch, ascending.  Every CSR value of a P1 operator is an ordered sum over cells:
// the diagonal (r, r) over the cells of r, an off-diagonal (r, v) over the cells holding
// the edge r-v.  Within a cell the entries are symmetric bit for bit, so (r, v) and (v, r)
// are the same sum: each edge is summed once, by the tile that owns it (the tile of its
// lower endpoint), and written to both positions.  The tables list, per tile row, its
// cells as (position in the tile's cell list, the row's local vertex), and per owned
// edge its cells as (position, upper-triangle index of the edge in the cell's 4x4 block),
// in ascending cell order; each row's and each edge's terms are contiguous and padded to
// a multiple of 8, so a thread reads 8 terms with one 16-byte load and a warp's loads of
// consecutive rows or edges are one contiguous range.
#pragma once
#include "tp_common.cuh"

namespace tp {

constexpr uint16_t TILE_TERM_NONE = 0xFFFFu;  // padding after a row's or edge's last term
constexpr int TILE_LOC_BITS = 12;             // cell position in the tile: < 4096

struct TileView {
  int R, n_tiles, max_cells, max_edges;
  const int32_t* rows;       // (n_tiles * R) row ids, -1 where a tile has fewer rows
  const int32_t* diag_pos;   // (n_tiles * R) CSR position of (r, r)
  const int32_t* cell_ptr;   // (n_tiles + 1)
  const int32_t* cells;      // distinct cells of each tile, ascending
  const int32_t* dterm_ptr;  // (n_tiles + 1) offsets of the diagonal terms (R rows x KD)
  const uint16_t* dterms;    // [row][k]: loc | li << 12, KD a multiple of 8 per tile
  const int32_t* edge_ptr;   // (n_tiles + 1) first owned edge of each tile
  const int2* edge_pos;      // CSR positions of (r, v) and (v, r), r the lower endpoint
  const int2* edge_rv;       // (r, v)
  const int32_t* eterm_ptr;  // (n_tiles + 1) offsets of the edge terms (edges x KE)
  const uint16_t* eterms;    // [edge][k]: loc | tri_index << 12, KE a multiple of 8
};

}  // namespace tp

struct tp_tiles {
  tp::TileView v;
  void* dmem = nullptr;
  size_t bytes = 0;
  int64_t n_terms = 0;
  ~tp_tiles() {
    if (dmem) cudaFree(dmem);
  }
};
