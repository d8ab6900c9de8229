// ppmg_halo.cuh -- blocks of the ghost exchange between z-slab subdomains.
#pragma once

#include <vector>

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

// Whether the subdomains (istart, nnodes: [nsubs][3], 1-based) form a
// cartesian decomposition of the mesh of Nm nodes per axis: along every axis
// either all of them span the mesh or all are cut, the intervals tile
// 1 .. Nm (each starting on the previous one's last node), and every
// combination of the axes' intervals is one subdomain.  0, or why not.
const char* check_cartesian(int nsubs, const int* istart, const int* nnodes, const int Nm[3]);

// The neighbours of subdomain isub in a cartesian decomposition (sorted,
// isub excluded): the subdomains whose interval along every axis equals
// isub's or touches it, across the periodic faces too (the subdomains whose
// boxes share a face, an edge or a corner with isub's: the neighbour list
// ppm_map_part_partial sends to).
void cart_neighbours(int nsubs, const int* istart, const int* nnodes, const int Nm[3], int isub,
                     std::vector<int>& out);

// The exchange of any cartesian decomposition (cuts along one, two or three
// axes): blocks are boxes of the local field, in its 1-based local node
// indices (inclusive), for every neighbouring subdomain and periodic shift.
struct HaloBox {
  int peer, tag;
  int64_t lo[3], hi[3];
};
// Builds the boxes of subdomain isub (istart, nnodes: [nsubs][3]; Nm: global
// nodes per axis; g: ghost widths).  Returns 0, or a message describing the
// argument that is wrong.
const char* halo_boxes(int nsubs, const int* istart, const int* nnodes, const int Nm[3],
                       int isub, const int g[3], bool put, std::vector<HaloBox>& sends,
                       std::vector<HaloBox>& recvs);

// Pack the boxes of field (ldf rows per node, element strides s[3], lower
// bounds lb[3]) into buf, or unpack buf into them (add: the put's pop with
// add; else a copy); each box travels as all ldf rows of its nodes, x
// fastest.  tab: device table of 8 int64 per box (lo[3], ext[3], the box's
// first index in the launch's index space -- the boxes back to back in table
// order, tot elements in all -- and its offset in buf), nbox boxes.  The
// boxes of one launch must not overlap unless every one only reads field.
template <class T>
cudaError_t launch_box_copy(T* field, int64_t ldf, const int64_t s[3], const int lb[3],
                            const int64_t* tab, int nbox, int64_t tot, T* buf, int mode,
                            cudaStream_t st);
constexpr int kBoxPack = 0, kBoxCopy = 1, kBoxAdd = 2;

// dst[i] += src[i] for i < n (the pop with add of a received block).
template <class T>
cudaError_t launch_plane_add(T* dst, const T* src, int64_t n, cudaStream_t st);

}  // namespace ppmg
