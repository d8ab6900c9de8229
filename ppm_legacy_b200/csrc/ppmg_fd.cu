// ppmg_fd.cu -- FFT Poisson solver on the periodic mesh of one subdomain:
// the spectral step of ppm_fdsolver_poisson_3d (ppm/src/ppm_fdsolver_poisson_3d.f:
// 60-82: every mode of the transformed field times -1/|k|^2, the zero mode
// set to 0, k_a = 2 pi / L_a times the wave number folded to |.| <= N_a/2)
// between a forward and a backward transform (ppm_fdsolver_solve_3d.f:822-
// 1170 with FFTW; cuFFT here), and the 1/(Nx Ny Nz) of the inverse
// (ppm_fdsolver_solve_3d.f:1383).  The result solves lap(phi) = omega.
#include <cuda_runtime.h>

#include "ppmg_fd.cuh"

namespace ppmg {

namespace {

int blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

// Unique nodes 1..N of component c of field_up into r[z][y][x] (x fastest).
template <class T>
__global__ void k_fd_pack(const T* __restrict__ field, FieldDesc fd, int c, int N0, int N1,
                          int N2, T* __restrict__ r) {
  const int64_t n = (int64_t)N0 * N1 * N2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % N0), y = (int)((q / N0) % N1), z = (int)(q / ((int64_t)N0 * N1));
    const int64_t o = (int64_t)(x + 1 - fd.lb[0]) * fd.s[0] + (int64_t)(y + 1 - fd.lb[1]) * fd.s[1] +
                      (int64_t)(z + 1 - fd.lb[2]) * fd.s[2] + c;
    r[q] = field[o];
  }
}

// Spectrum C[z][y][x'] (x' <= N0/2, the half spectrum of the real-to-complex
// axis) times -1/|k|^2 / (N0 N1 N2); the zero mode becomes 0.
template <class T, class C>
__global__ void k_fd_spectral(C* __restrict__ spec, int N0, int N1, int N2, T kx0, T ky0, T kz0,
                              T inv_n) {
  const int H = N0 / 2 + 1;
  const int64_t n = (int64_t)H * N1 * N2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % H), y = (int)((q / H) % N1), z = (int)(q / ((int64_t)H * N1));
    const int yf = y >= N1 / 2 + 1 ? N1 - y : y;  // the reference's fold (sign irrelevant)
    const int zf = z >= N2 / 2 + 1 ? N2 - z : z;
    C v = spec[q];
    if (x == 0 && y == 0 && z == 0) {
      v.x = T(0);
      v.y = T(0);
    } else {
      const T kx = kx0 * (T)x, ky = ky0 * (T)yf, kz = kz0 * (T)zf;
      const T f = -inv_n / (kx * kx + ky * ky + kz * kz);
      v.x *= f;
      v.y *= f;
    }
    spec[q] = v;
  }
}

// r[z][y][x] into component c of every position of the box (real nodes and
// their periodic images).
template <class T>
__global__ void k_fd_unpack(const T* __restrict__ r, int N0, int N1, int N2, T* __restrict__ field,
                            FieldDesc fd, int c) {
  const int e0 = fd.box_hi[0] - fd.box_lo[0] + 1, e1 = fd.box_hi[1] - fd.box_lo[1] + 1,
            e2 = fd.box_hi[2] - fd.box_lo[2] + 1;
  const int64_t n = (int64_t)e0 * e1 * e2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = fd.box_lo[0] + (int)(q % e0);
    const int j = fd.box_lo[1] + (int)((q / e0) % e1);
    const int k = fd.box_lo[2] + (int)(q / ((int64_t)e0 * e1));
    const int x = wrap_index(i - 1, N0), y = wrap_index(j - 1, N1), z = wrap_index(k - 1, N2);
    const int64_t o = (int64_t)(i - fd.lb[0]) * fd.s[0] + (int64_t)(j - fd.lb[1]) * fd.s[1] +
                      (int64_t)(k - fd.lb[2]) * fd.s[2] + c;
    field[o] = r[(int64_t)x + (int64_t)N0 * (y + (int64_t)N1 * z)];
  }
}

template <class T>
struct FFTTypes;
template <>
struct FFTTypes<double> {
  using C = cufftDoubleComplex;
  static constexpr cufftType fwd = CUFFT_D2Z, inv = CUFFT_Z2D;
  static cufftResult exec_fwd(cufftHandle p, double* in, C* out) { return cufftExecD2Z(p, in, out); }
  static cufftResult exec_inv(cufftHandle p, C* in, double* out) { return cufftExecZ2D(p, in, out); }
};
template <>
struct FFTTypes<float> {
  using C = cufftComplex;
  static constexpr cufftType fwd = CUFFT_R2C, inv = CUFFT_C2R;
  static cufftResult exec_fwd(cufftHandle p, float* in, C* out) { return cufftExecR2C(p, in, out); }
  static cufftResult exec_inv(cufftHandle p, C* in, float* out) { return cufftExecC2R(p, in, out); }
};

}  // namespace

void FFTPlans::release() {
  if (fwd) cufftDestroy(fwd);
  if (inv) cufftDestroy(inv);
  fwd = inv = 0;
  prec = -1;
}

template <class T>
int fd_poisson(FFTPlans& plans, Workspace& ws, const int N[3], const double len[3], T* field,
               const FieldDesc& fd, int lda, cudaStream_t st, cudaError_t& ce) {
  using F = FFTTypes<T>;
  using C = typename F::C;
  ce = cudaSuccess;
  const int prec = sizeof(T) == 8 ? 0 : 1;
  if (plans.prec != prec || plans.n[0] != N[0] || plans.n[1] != N[1] || plans.n[2] != N[2]) {
    plans.release();
    // cuFFT sizes slowest first: (z, y, x), x the real-to-complex axis
    if (cufftPlan3d(&plans.fwd, N[2], N[1], N[0], F::fwd) != CUFFT_SUCCESS ||
        cufftPlan3d(&plans.inv, N[2], N[1], N[0], F::inv) != CUFFT_SUCCESS) {
      plans.release();
      return 1;
    }
    plans.prec = prec;
    for (int a = 0; a < 3; ++a) plans.n[a] = N[a];
  }
  if (cufftSetStream(plans.fwd, st) != CUFFT_SUCCESS ||
      cufftSetStream(plans.inv, st) != CUFFT_SUCCESS)
    return 1;
  const int64_t nr = (int64_t)N[0] * N[1] * N[2];
  const int64_t nc = (int64_t)(N[0] / 2 + 1) * N[1] * N[2];
  if ((ce = ws.rec.ensure(sizeof(T) * (size_t)nr)) || (ce = ws.us.ensure(sizeof(C) * (size_t)nc)))
    return 0;
  T* r = ws.rec.as<T>();
  C* spec = ws.us.as<C>();
  const double two_pi = 6.283185307179586476925286766559;
  const T kx0 = (T)(two_pi / len[0]), ky0 = (T)(two_pi / len[1]), kz0 = (T)(two_pi / len[2]);
  const T inv_n = (T)(1.0 / (double)nr);
  for (int c = 0; c < lda; ++c) {
    k_fd_pack<T><<<blocks(nr), 256, 0, st>>>(field, fd, c, N[0], N[1], N[2], r);
    if (F::exec_fwd(plans.fwd, r, spec) != CUFFT_SUCCESS) return 1;
    k_fd_spectral<T, C><<<blocks(nc), 256, 0, st>>>(spec, N[0], N[1], N[2], kx0, ky0, kz0, inv_n);
    if (F::exec_inv(plans.inv, spec, r) != CUFFT_SUCCESS) return 1;
    const int64_t nb = (int64_t)(fd.box_hi[0] - fd.box_lo[0] + 1) *
                       (fd.box_hi[1] - fd.box_lo[1] + 1) * (fd.box_hi[2] - fd.box_lo[2] + 1);
    k_fd_unpack<T><<<blocks(nb), 256, 0, st>>>(r, N[0], N[1], N[2], field, fd, c);
    count_launch(3);
    if ((ce = cudaGetLastError())) return 0;
  }
  return 0;
}

template int fd_poisson<double>(FFTPlans&, Workspace&, const int*, const double*, double*,
                                const FieldDesc&, int, cudaStream_t, cudaError_t&);
template int fd_poisson<float>(FFTPlans&, Workspace&, const int*, const double*, float*,
                               const FieldDesc&, int, cudaStream_t, cudaError_t&);

}  // namespace ppmg
