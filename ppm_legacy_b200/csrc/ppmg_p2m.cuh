// ppmg_p2m.cuh -- launch interface of the particle -> mesh tile gather.
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

enum P2MPrec {
  P2M_FP64 = 0,   // FP64 weights and sums
  P2M_MIXED = 1,  // FP32 weights/products, compensated FP32 sums, FP64 field
  P2M_FP32 = 2,   // single-precision API: FP32 throughout
};

// The 0-based node range org .. org+ext-1 per axis that a 3D tile grid
// covers: the unique nodes 0 .. N-1 of a periodic axis (org 0, ext N), the
// whole written box -g .. N+g of a cut axis (an axis along which the local
// subdomain is one interval of several: no periodic images, cell layers
// outside 0 .. N-1 hold none of its particles).
struct TileSpan {
  int org[3], ext[3];
};
TileSpan cell_span(const int N[3]);

struct P2MParams {
  int N[3];            // cells per axis
  int TZ;              // tile depth along the sweep axis (z in 3D, y in 2D)
  int cap;             // staging capacity (particles per chunk)
  int c0;              // first component written by this launch
  const int* start;    // cell offsets into the sorted particle order
  const void* rec;     // Vec4 (fx, fy, fz, cell) per sorted particle
  const void* us;      // Vec4 strengths (4 components of one chunk)
  int64_t ps;          // plane stride of rec / us in 16-byte units (set by launch_p2m)
  void* field;         // field_up base (element (1, lb...))
  FieldDesc fd;
  // 3D work items (xy tile, z0, z1), filled by launch_p2m
  const int4* items;
  const int* nitems;
  int item_cap;
  // cut axes (open[a]: the subdomain is one interval of several along a)
  // and the node range the work items cover (cell_span(N) without cuts)
  int open[3];
  TileSpan span;
};

// Device scratch launch_p2m needs (work items, per-layer counts); sp: the
// node range the items cover (nullptr: cell_span(N)).
size_t p2m_scratch_bytes(int dim, const int N[3], const TileSpan* sp = nullptr);

// Work items of the 3D tile kernels: (xy tile of kTileX x kTileY cells,
// z0, z1) with z ranges split so every item holds a similar particle count.
struct TileItems {
  const int4* items;
  const int* nitems;  // device count
  int cap;            // grid size to launch (items beyond *nitems exit)
};
size_t tile_items_bytes(const int N[3], const TileSpan* sp = nullptr);
// The items a previous make_tile_items left in `scratch`.
TileItems tile_items_view(void* scratch, const int N[3], const TileSpan* sp = nullptr);
// Items over the xy tiles and z planes of the span sp (nullptr: the cells
// 0 .. N-1); nodes outside the cells count no particles.
// tdx x tdy: the tile of the kernel that uses them (kTileX x kTileY for the
// tile gathers).
cudaError_t make_tile_items(const int* start, const int N[3], int64_t nvalid, void* scratch,
                            TileItems& out, cudaStream_t st, const TileSpan* sp = nullptr,
                            int tdx = kTileX, int tdy = kTileY);

// Whether launch_p2m runs the 3D row gather (whose items are not the tile
// gathers' items that M2P and the adjoint can reuse).
bool p2m_row_gather(int dim, P2MPrec prec);

// Tile depth (nodes along the sweep axis per CTA) of the 2D gather.
int p2m_tile_depth(int dim, const int N[3]);

// Launch the gather for all components (chunks of 4) of a P2M / remesh.
// stored_weights: P.rec holds FP64 1D weights per sorted particle
// (wx[S], wy[S][, wz[S]]) from comp_weights instead of offset records.
cudaError_t launch_p2m(const P2MParams& P, int dim, int kernel, P2MPrec prec, int lda,
                       int64_t nvalid, bool stored_weights, void* scratch, cudaStream_t st);

}  // namespace ppmg
