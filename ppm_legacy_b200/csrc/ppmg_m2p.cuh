// ppmg_m2p.cuh -- launch interface of the mesh -> particle gather and adjoint.
#pragma once

#include "ppmg_common.cuh"

namespace ppmg {

enum M2PPrec {
  M2P_FP64 = 0,   // FP64, no contraction: the reference's arithmetic
  M2P_MIXED = 1,  // FP32 weights and sums from FP64 offsets, FP64 in/out
  M2P_FP32 = 2,   // single-precision API
};

struct M2PParams {
  int N[3];
  int64_t nvalid;      // grid bound (Np); the sorted count is *d_nvalid
  const int* d_nvalid;
  const int* idx;     // sorted position -> particle id
  const void* rec;    // Vec4 (fx, fy, fz, cell) per sorted particle, planes nvalid apart
  const void* field;  // field_up base (element (1, lb...))
  FieldDesc fd;
  void* up;           // output up(ldup, Np) (adjoint: dw)
  int64_t ldup;
  int lda;
  int c0;             // first component of this launch (tile kernel)
  int open[3];        // cut axes: nodes read without periodic wrap (ghosts included)
  // 3D tile kernel: cell offsets and work items
  const int* start;
  const int4* items;
  const int* nitems;
  int item_cap;
  // adjoint only
  const double* upin;
  int64_t ldupin;
  double* dx;
  int64_t lddx;
  double dxi[3];
};

cudaError_t launch_m2p(const M2PParams& P, int dim, int kernel, M2PPrec prec, cudaStream_t st);
cudaError_t launch_adjoint(const M2PParams& P, int kernel, M2PPrec prec, cudaStream_t st);

}  // namespace ppmg
