// ppmg_fd.cuh -- FFT Poisson solver on one periodic subdomain (ppmg_fd.cu).
#pragma once

#include <cufft.h>

#include <functional>

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

// The slab form of the solver (ppm_fdsolver_solve_slab, ppm/src/
// ppm_fdsolver_solve_3d.f:18-21: FFTs on xy slabs, then on z pencils).  The
// domain is cut into P z-slabs, slab q holding the unique planes
// z0[q] .. z0[q]+nz[q]-1 (0-based, global) of an N[0] x N[1] x N[2] mesh.
struct SlabSolve {
  int P = 0, me = 0;
  int N[3] = {0, 0, 0};
  double len[3] = {1.0, 1.0, 1.0};
  const int* z0 = nullptr;
  const int* nz = nullptr;
};

// Plans and buffers of a handle's slab solve, kept between calls.
struct SlabFFTPlans {
  cufftHandle xy_fwd = 0, xy_inv = 0, zc = 0;
  int prec = -1, nx = 0, ny = 0, nzl = 0, nzg = 0, nyl = 0;
  void release();
};

// One exchange of device blocks with the other slabs (the caller's transport;
// nonzero: it failed).
using BlockExchange = std::function<int(int nsend, const ppmg_halo_block* sends, int nrecv,
                                        const ppmg_halo_block* recvs)>;

// lap(phi) = omega on the slab decomposition: omega on the local slab's
// unique nodes (planes 1 .. nz[me] of field_up), phi written there and at
// every x, y image of those planes; the z ghost planes and the shared upper
// plane are left to a ghost get.  The pencils split the ky modes over the P
// slabs (N[1] >= P).  Returns 1 on a cuFFT failure, 2 on a transport failure,
// else 0 (a CUDA error in ce).
template <class T>
int fd_poisson_slab(SlabFFTPlans& plans, Workspace& ws, const SlabSolve& sl, T* field,
                    const FieldDesc& fd, int lda, cudaStream_t st, const BlockExchange& xchg,
                    cudaError_t& ce);

}  // namespace ppmg
