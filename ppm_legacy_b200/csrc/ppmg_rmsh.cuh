// ppmg_rmsh.cuh -- remeshing helpers and periodic ghost get/put.
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

// Stored 1D weights per sorted particle: dim x S values of the routine's
// kind, padded to a multiple of 16 bytes (one or more whole 16-byte units).
inline int weight_stride(int dim, int S, int tsize) {
  return (dim * S * tsize + 15) / 16 * 16 / tsize;
}

// ppm_rmsh_comp_weights (T = double: _d, float: _s): 1D weights per sorted particle.
template <class T>
struct CWParams {
  int dim, S;
  int wstride;          // weight_stride(dim, S, sizeof(T))
  int64_t nvalid;       // grid bound (Np); sorted count is *d_nvalid
  const int* d_nvalid;
  const int* idx;
  const T* xp;
  int64_t ldxp;
  T min_phys[3];
  T dxiq[3];  // FP32 mesh spacing (ppm_rmsh_comp_weights.f:146-147)
  int istart[3];
  T* w;       // out: nvalid x wstride
};

// ppm_rmsh_create_part (T = double: _d, float: _s).
template <class T>
struct CPParams {
  int dim, lda, lda2;
  int nn[3];        // nodes visited per axis
  const T* field;
  FieldDesc fd;
  const T* field_wp;
  FieldDesc fdw;
  const T* cw;  // cutoff weights or nullptr
  T cut0, cut1;
  T h[3], min_sub[3];
  T* up;
  T* xp;
  T* wp;
};

struct GhostParams {
  int dim, lda;
  int N[3];         // cells (Nm-1)
  int lo[3], hi[3]; // box 1-g .. Nm+g
  FieldDesc fd;
};

template <class T>
cudaError_t launch_comp_weights(const CWParams<T>& P, cudaStream_t st);
template <class T>
cudaError_t launch_weights_to_user(const T* w, const int* idx, int64_t nvalid,
                                   const int* d_nvalid, int wstride, int S, int axis, T* out,
                                   cudaStream_t st);
template <class T>
cudaError_t launch_cp_flag(const CPParams<T>& P, int* flag, cudaStream_t st);
template <class T>
cudaError_t launch_cp_fill(const CPParams<T>& P, const int* flag, const int* pos,
                           cudaStream_t st);
template <class T>
cudaError_t launch_ghost(const GhostParams& P, int maptype, T* field, T* tmp,
                         cudaStream_t st);
cudaError_t launch_plus_one(const int* in, int* out, int64_t n, cudaStream_t st);

}  // namespace ppmg
