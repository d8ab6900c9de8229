// ppmg_rmsh.cuh -- remeshing helpers and periodic ghost get/put.
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

// ppm_rmsh_comp_weights: 1D weights per sorted particle.
struct CWParams {
  int dim, S;
  int64_t nvalid;       // grid bound (Np); sorted count is *d_nvalid
  const int* d_nvalid;
  const int* idx;
  const double* xp;
  int64_t ldxp;
  double min_phys[3];
  double dxiq[3];  // FP32 mesh spacing widened (ppm_rmsh_comp_weights.f:146-147)
  int istart[3];
  double* w;       // out: nvalid x dim x S
};

// ppm_rmsh_create_part.
struct CPParams {
  int dim, lda, lda2;
  int nn[3];        // nodes visited per axis
  const double* field;
  FieldDesc fd;
  const double* field_wp;
  FieldDesc fdw;
  const double* cw;  // cutoff weights or nullptr
  double cut0, cut1;
  double h[3], min_sub[3];
  double* up;
  double* xp;
  double* wp;
};

struct GhostParams {
  int dim, lda;
  int N[3];         // cells (Nm-1)
  int lo[3], hi[3]; // box 1-g .. Nm+g
  FieldDesc fd;
};

cudaError_t launch_comp_weights(const CWParams& P, cudaStream_t st);
cudaError_t launch_weights_to_user(const double* w, const int* idx, int64_t nvalid,
                                   const int* d_nvalid, int dim, int S, int axis, double* out,
                                   cudaStream_t st);
cudaError_t launch_cp_flag(const CPParams& P, int* flag, cudaStream_t st);
cudaError_t launch_cp_fill(const CPParams& P, const int* flag, const int* pos,
                           cudaStream_t st);
template <class T>
cudaError_t launch_ghost(const GhostParams& P, int maptype, T* field, T* tmp,
                         cudaStream_t st);
cudaError_t launch_plus_one(const int* in, int* out, int64_t n, cudaStream_t st);

}  // namespace ppmg
