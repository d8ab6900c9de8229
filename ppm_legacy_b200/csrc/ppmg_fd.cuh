// ppmg_fd.cuh -- FFT Poisson solver on one periodic subdomain (ppmg_fd.cu).
#pragma once

#include <cufft.h>

#include "ppmg_common.cuh"
#include "ppmg_sort.cuh"

namespace ppmg {

// cuFFT plans of a handle's mesh, kept between calls.
struct FFTPlans {
  cufftHandle fwd = 0, inv = 0;
  int prec = -1;  // 0 FP64, 1 FP32
  int n[3] = {0, 0, 0};
  void release();
};

// lap(phi) = omega for components 0..lda-1 of field_up (described by fd,
// its box the written one): omega on the unique nodes 1..N, phi written to
// every position of the box.  Returns 1 on a cuFFT failure, else 0 (a CUDA
// error in ce).
template <class T>
int fd_poisson(FFTPlans& plans, Workspace& ws, const int N[3], const double len[3], T* field,
               const FieldDesc& fd, int lda, cudaStream_t st, cudaError_t& ce);

}  // namespace ppmg
