// ppmg_halo.cuh -- blocks of the ghost exchange between z-slab subdomains.
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

// One exchange of the local slab: blocks towards / from the slab above
// (index 0) and below (index 1), as element offsets into field_up.
struct HaloPlan {
  int64_t count;       // elements per block
  int send_peer[2], send_tag[2];
  int64_t send_off[2];
  int recv_peer[2], recv_tag[2];
  int64_t recv_off[2];
};

// Builds the plan from the geometry (istart, nnodes: [nsubs][3], 1-based
// global node offsets and counts; Nmz global nodes along z).  Returns 0, or
// a message describing the argument that is wrong.
const char* halo_plan(int nsubs, const int* istart, const int* nnodes, int Nmz, int isub,
                      int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int gz, bool put,
                      HaloPlan& out);

// dst[i] += src[i] for i < n (the pop with add of a received block).
template <class T>
cudaError_t launch_plane_add(T* dst, const T* src, int64_t n, cudaStream_t st);

}  // namespace ppmg
