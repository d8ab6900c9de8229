// ppmg_map.cuh -- particle routing between z-slab subdomains (ppmg_map.cu).
#pragma once

#include "ppmg_common.cuh"
#include "ppmg_sort.cuh"

namespace ppmg {

// Boxes a particle is routed into: the local slab (0), the slab below (1)
// and the slab above (2), all spanning [lo, hi) in x and y; a class whose
// z range is empty takes no particle.  Bounds in both precisions, compared
// in the positions' own.
struct RouteParams {
  double lo[2], hi[2], zlo[3], zhi[3];
  float lof[2], hif[2], zlof[3], zhif[3];
};

int route_blocks(int64_t np);

// dest (np bytes), bc and off (4 * route_blocks(np) ints) are scratch; perm
// (np ints) receives the particle ids grouped by class 0..3, each class in
// ascending id.
template <class T>
cudaError_t launch_route(const RouteParams& R, const T* xp, int64_t ldxp, int64_t np,
                         unsigned char* dest, int* bc, int* off, int* perm, Workspace& ws,
                         cudaStream_t st);

// Global routing (ppm_map_part_global): every particle to the subdomain
// that contains it among all nsubs (<= kMaxGlobalSubs), subdomain s spanning
// [min_sub, max_sub) on every axis (R.box).  Class nsubs: in no subdomain.  perm (np ints) receives the ids grouped by class 0..nsubs,
// each class in ascending id; off (device, (nsubs + 1) * route_blocks(np))
// ends holding the exclusive class-major offsets, so class c starts at
// off[c * nblk].
constexpr int kMaxGlobalSubs = 255;
struct GlobalRouteParams {
  int nsubs;
  const double* box;  // device [6][nsubs]: min_sub x, y, z, then max_sub x, y, z
};
template <class T>
cudaError_t launch_route_global(const GlobalRouteParams& R, const T* xp, int64_t ldxp,
                                int64_t np, unsigned char* dest, int* bc, int* off, int* perm,
                                Workspace& ws, cudaStream_t st);

// dst(0:lda-1, j) = src(0:lda-1, perm[j]) for j < n.
template <class T>
cudaError_t launch_gather_cols(const T* src, int64_t lds, int lda, const int* perm, int64_t n,
                               T* dst, int64_t ldd, cudaStream_t st);

}  // namespace ppmg
