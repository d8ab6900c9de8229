// ppmg_sort.cuh -- device counting sort of particles into mesh cells.
//
// Replaces the two-pass particle -> sub assignment of the reference
// (ppm_interp_p2m.f:496-750) and the ranking of ppm_util_rank3d.f:353-533:
// every particle gets a cell key, cells are counted, scanned, and the
// particle ids are scattered into cell order with ascending id inside each
// cell (the reference's stable fill order, ppm_util_rank3d.f:525-533).
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

// A growable device buffer.  A `fixed` buffer is a view of memory it does not
// own (p and bytes set by its user): ensure() never reallocates it, it only
// reports whether the request fits, and release() leaves the memory alone.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool fixed = false;
  cudaError_t ensure(size_t n);
  void release();
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

// Scratch of one handle (device memory, grown on demand, reused).
struct Workspace {
  DevBuf key, slot, idx, count, start, bsum, rec, us, err, big, tiles;
  DevBuf key2, idx2, rec2, hist, gaps;  // radix sort: second key/id set, record rows, histograms
  DevBuf h_xp, h_up, h_field, h_aux;  // device mirrors for host-pointer calls
  DevBuf w1d;                          // comp_weights state: sorted 1D weights
  int* h_err_pinned = nullptr;         // pinned host copy of the error word
  ~Workspace();
};

// How particle positions turn into cell keys.
enum KeyMode {
  KEY_INTERP_CHECKED = 0,  // P2M / comp_weights: x in [min_sub, max_sub) required
  KEY_INTERP_WRAP = 1,     // M2P / adjoint: any finite x, periodic wrap
};

// Key computation parameters (one subdomain).  An axis is periodic within the
// subdomain unless open[a]: the subdomain is then one slab of a larger
// domain along a, its neighbours hold the rest, and positions outside it
// are invalid in every mode.
struct KeyParams {
  int dim;
  int N[3];
  double min[3], max[3];
  double dxi[3];
  float minf[3], maxf[3], dxif[3];
  int mode;
  int open[3];
};

// Counting sort of Np particles into the Nx*Ny*Nz cells.  On return
// (stream-ordered): ws.idx holds particle ids in cell order (ascending inside
// a cell), ws.start[0..ncell] the cell offsets (start[ncell] = number of
// valid particles), ws.key the cell of every particle (-1 if invalid).
// T is the position type (double or float).
// Invalid particles increment *err_counter (device, not reset here); when
// zout is given their rows zout(0:nz-1, p) are zeroed (M2P output).  When
// hash is given it receives the position fingerprint of position_hash.
template <class T>
cudaError_t bin_sort(const KeyParams& kp, const T* xp, int64_t ldxp, int64_t np,
                     int64_t ncell, Workspace& ws, int* err_counter, cudaStream_t st,
                     T* zout = nullptr, int64_t ldz = 0, int nz = 0,
                     unsigned long long* hash = nullptr);

// 64-bit fingerprint of the first `dim` coordinates of xp(ldxp, np) into
// *hash (device): sum over particles of a mixed hash of (index, coordinates).
template <class T>
cudaError_t position_hash(const T* xp, int64_t ldxp, int64_t np, int dim,
                          unsigned long long* hash, cudaStream_t st);

// Exclusive scan of n ints (in may alias out).
cudaError_t scan_exclusive(const int* in, int* out, int64_t n, Workspace& ws,
                           cudaStream_t st);

// Pack sorted particle records: rec[s] = (fx, fy, fz, cell) of particle idx[s]
// in CT precision, us chunk ch (vector offset ch*np) [s] = up(4ch..4ch+3,
// idx[s]) (when up != null); both in the plane layout of load_vec (stride np).
// Positions s < *d_nvalid (the sorted count, start[ncell]) are packed.
template <class T, class CT>
cudaError_t pack_records(const KeyParams& kp, const T* xp, int64_t ldxp, const T* up,
                         int64_t ldup, int lda, int64_t np, const int* d_nvalid,
                         Workspace& ws, cudaStream_t st);

// Stable LSD radix sort of the particles by cell (the order of bin_sort:
// ascending id inside a cell) of (key, id) pairs, followed by one gather of
// the packed records and strengths into the sorted order.  On
// return (stream-ordered), for sorted positions s < np:
//   ws.key[s]  cell of the particle (ncell for an invalid one; those sort last)
//   ws.idx[s]  particle id
//   ws.rec     (fx, fy, fz, cell) in CT precision, as pack_records
//   ws.us      up(4ch..4ch+3, id) in CT precision (when up != null), chunk ch
//              at vector offset ch*np
// (rec and us in the 16-byte plane layout of load_vec, plane stride np) and
// ws.start[0..ncell] the cell offsets (start[ncell] = valid count).
// Invalid particles increment *err_counter; zout / hash as for bin_sort.
// *wait_flag is set if a bulk copy of the sort never completes (the sort is
// then incomplete and must not be used).
template <class T, class CT>
cudaError_t radix_sort_records(const KeyParams& kp, const T* xp, int64_t ldxp, const T* up,
                               int64_t ldup, int lda, int64_t np, int64_t ncell,
                               Workspace& ws, int* err_counter, int* wait_flag, cudaStream_t st,
                               T* zout = nullptr, int64_t ldz = 0, int nz = 0,
                               unsigned long long* hash = nullptr);

// Clist ranking (ppm_util_rank{2,3}d): keys from FLOOR((x-xmin)*rdx)+Ngl with
// the reference's upper-boundary corrections; -1 outside the mesh.  The
// number of particles inside is counted in ws.err[0].
struct ClistParams {
  int dim;
  int Nm[3];
  int Ngl[6];
  int Nt[3];
  double xmin[3], xmax[3], rd[3];  // double positions
  float xminf[3], xmaxf[3], rdf[3];  // float positions (ppm_util_rank3d_s)
};
template <class T>
cudaError_t clist_sort(const ClistParams& cp, const T* xp, int64_t ldxp, int64_t np,
                       int64_t nbox, Workspace& ws, cudaStream_t st);

}  // namespace ppmg
