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

// ---- slab form: the ky modes split over the P slabs for the z pencils ----
// Rows ky of slab q: y0 .. y0+ny-1, the first Ny % P slabs one row more.
__host__ __device__ inline void y_split(int Ny, int P, int q, int& y0, int& ny) {
  const int b = Ny / P, r = Ny % P;
  ny = b + (q < r ? 1 : 0);
  y0 = q * b + (q < r ? q : r);
}
__device__ inline int y_owner(int ky, int Ny, int P) {
  const int b = Ny / P, r = Ny % P;
  return ky < r * (b + 1) ? ky / (b + 1) : r + (ky - r * (b + 1)) / b;
}

// spec[z][ky][kx] (nzl planes of the slab's xy transforms) to the pencils:
// the rows of this slab straight into T[z0 + z][ky - y0][kx], the rows of
// slab q into its send block (blocks of the other slabs in slab order).
template <class C>
__global__ void k_y_pack(const C* __restrict__ spec, int H, int Ny, int nzl, int P, int me,
                         int z0me, int nylme, const int64_t* __restrict__ soff,
                         C* __restrict__ send, C* __restrict__ pen) {
  const int64_t n = (int64_t)H * Ny * nzl;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(q % H), ky = (int)((q / H) % Ny), z = (int)(q / ((int64_t)H * Ny));
    const int o = y_owner(ky, Ny, P);
    int y0, ny;
    y_split(Ny, P, o, y0, ny);
    if (o == me)
      pen[((int64_t)(z0me + z) * nylme + (ky - y0)) * H + kx] = spec[q];
    else
      send[soff[o] + ((int64_t)z * ny + (ky - y0)) * H + kx] = spec[q];
  }
}

// The way back: spec[z][ky][kx] from this slab's pencils or the block that
// slab q returned (blocks in slab order at roff).
template <class C>
__global__ void k_y_unpack(C* __restrict__ spec, int H, int Ny, int nzl, int P, int me,
                           int z0me, int nylme, const int64_t* __restrict__ roff,
                           const C* __restrict__ recv, const C* __restrict__ pen) {
  const int64_t n = (int64_t)H * Ny * nzl;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(q % H), ky = (int)((q / H) % Ny), z = (int)(q / ((int64_t)H * Ny));
    const int o = y_owner(ky, Ny, P);
    int y0, ny;
    y_split(Ny, P, o, y0, ny);
    spec[q] = o == me ? pen[((int64_t)(z0me + z) * nylme + (ky - y0)) * H + kx]
                      : recv[roff[o] + ((int64_t)z * ny + (ky - y0)) * H + kx];
  }
}

// The spectral step on the pencils T[kz][ky - y0][kx] of this slab (global
// wave numbers; the 1/(Nx Ny Nz) of the inverse folded in), as k_fd_spectral.
template <class T, class C>
__global__ void k_fd_spectral_pencil(C* __restrict__ pen, int H, int nyl, int y0, int N1, int N2,
                                     T kx0, T ky0, T kz0, T inv_n) {
  const int64_t n = (int64_t)H * nyl * N2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % H), yl = (int)((q / H) % nyl), z = (int)(q / ((int64_t)H * nyl));
    const int y = y0 + yl;
    const int yf = y >= N1 / 2 + 1 ? N1 - y : y;
    const int zf = z >= N2 / 2 + 1 ? N2 - z : z;
    C v = pen[q];
    if (x == 0 && y == 0 && z == 0) {
      v.x = T(0);
      v.y = T(0);
    } else {
      const T kx = kx0 * (T)x, ky = ky0 * (T)yf, kz = kz0 * (T)zf;
      const T f = -inv_n / (kx * kx + ky * ky + kz * kz);
      v.x *= f;
      v.y *= f;
    }
    pen[q] = v;
  }
}

// r[z][y][x] (the slab's planes 1..nzl) into component c of those planes of
// field_up and of every x, y image inside the box.
template <class T>
__global__ void k_fd_unpack_slab(const T* __restrict__ r, int N0, int N1, int nzl,
                                 T* __restrict__ field, FieldDesc fd, int c) {
  const int e0 = fd.box_hi[0] - fd.box_lo[0] + 1, e1 = fd.box_hi[1] - fd.box_lo[1] + 1;
  const int64_t n = (int64_t)e0 * e1 * nzl;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = fd.box_lo[0] + (int)(q % e0);
    const int j = fd.box_lo[1] + (int)((q / e0) % e1);
    const int z = (int)(q / ((int64_t)e0 * e1));  // plane z + 1
    const int x = wrap_index(i - 1, N0), y = wrap_index(j - 1, N1);
    const int64_t o = (int64_t)(i - fd.lb[0]) * fd.s[0] + (int64_t)(j - fd.lb[1]) * fd.s[1] +
                      (int64_t)(z + 1 - fd.lb[2]) * fd.s[2] + c;
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

namespace {
template <class T>
struct C2C;
template <>
struct C2C<double> {
  static constexpr cufftType type = CUFFT_Z2Z;
  static cufftResult exec(cufftHandle p, cufftDoubleComplex* d, int dir) {
    return cufftExecZ2Z(p, d, d, dir);
  }
};
template <>
struct C2C<float> {
  static constexpr cufftType type = CUFFT_C2C;
  static cufftResult exec(cufftHandle p, cufftComplex* d, int dir) {
    return cufftExecC2C(p, d, d, dir);
  }
};
}  // namespace

void SlabFFTPlans::release() {
  if (xy_fwd) cufftDestroy(xy_fwd);
  if (xy_inv) cufftDestroy(xy_inv);
  if (zc) cufftDestroy(zc);
  xy_fwd = xy_inv = zc = 0;
  prec = -1;
}

template <class T>
int fd_poisson_slab(SlabFFTPlans& plans, Workspace& ws, const SlabSolve& sl, T* field,
                    const FieldDesc& fd, int lda, cudaStream_t st, const BlockExchange& xchg,
                    cudaError_t& ce) {
  using F = FFTTypes<T>;
  using C = typename F::C;
  ce = cudaSuccess;
  const int Nx = sl.N[0], Ny = sl.N[1], Nz = sl.N[2], P = sl.P, me = sl.me;
  const int H = Nx / 2 + 1;
  const int nzl = sl.nz[me], z0me = sl.z0[me];
  int y0me, nyl;
  y_split(Ny, P, me, y0me, nyl);
  const int prec = sizeof(T) == 8 ? 0 : 1;
  if (plans.prec != prec || plans.nx != Nx || plans.ny != Ny || plans.nzl != nzl ||
      plans.nzg != Nz || plans.nyl != nyl) {
    plans.release();
    int n2[2] = {Ny, Nx};  // slowest first; x the real-to-complex axis
    int nz1[1] = {Nz};
    const int col = nyl * H;  // z pencils: stride between planes of T
    if (cufftPlanMany(&plans.xy_fwd, 2, n2, nullptr, 1, Ny * Nx, nullptr, 1, Ny * H, F::fwd,
                      nzl) != CUFFT_SUCCESS ||
        cufftPlanMany(&plans.xy_inv, 2, n2, nullptr, 1, Ny * H, nullptr, 1, Ny * Nx, F::inv,
                      nzl) != CUFFT_SUCCESS ||
        cufftPlanMany(&plans.zc, 1, nz1, nz1, col, 1, nz1, col, 1, C2C<T>::type, col) !=
            CUFFT_SUCCESS) {
      plans.release();
      return 1;
    }
    plans.prec = prec;
    plans.nx = Nx;
    plans.ny = Ny;
    plans.nzl = nzl;
    plans.nzg = Nz;
    plans.nyl = nyl;
  }
  if (cufftSetStream(plans.xy_fwd, st) != CUFFT_SUCCESS ||
      cufftSetStream(plans.xy_inv, st) != CUFFT_SUCCESS ||
      cufftSetStream(plans.zc, st) != CUFFT_SUCCESS)
    return 1;
  // block offsets (in complex elements) of the other slabs' rows in the
  // send buffer (forward) and in the receive buffer (backward): the same
  std::vector<int64_t> off(P, 0);
  int64_t tot = 0;
  for (int q = 0; q < P; ++q) {
    int y0, ny;
    y_split(Ny, P, q, y0, ny);
    off[q] = tot;
    if (q != me) tot += (int64_t)nzl * ny * H;
  }
  const int64_t nr = (int64_t)Nx * Ny * nzl;
  const int64_t nspec = (int64_t)H * Ny * nzl;
  const int64_t npen = (int64_t)H * nyl * Nz;
  if ((ce = ws.rec.ensure(sizeof(T) * (size_t)nr)) ||
      (ce = ws.us.ensure(sizeof(C) * (size_t)nspec)) ||
      (ce = ws.rec2.ensure(sizeof(C) * (size_t)npen)) ||
      (ce = ws.big.ensure(sizeof(C) * (size_t)(tot > 0 ? tot : 1))) ||
      (ce = ws.h_aux.ensure(sizeof(C) * (size_t)(tot > 0 ? tot : 1))) ||
      (ce = ws.count.ensure(sizeof(int64_t) * (size_t)P)))
    return 0;
  T* r = ws.rec.as<T>();
  C* spec = ws.us.as<C>();
  C* pen = ws.rec2.as<C>();
  C* sendb = ws.big.as<C>();
  C* recvb = ws.h_aux.as<C>();
  int64_t* doff = ws.count.as<int64_t>();
  if ((ce = cudaMemcpyAsync(doff, off.data(), sizeof(int64_t) * P, cudaMemcpyHostToDevice, st)))
    return 0;
  const double two_pi = 6.283185307179586476925286766559;
  const T kx0 = (T)(two_pi / sl.len[0]), ky0 = (T)(two_pi / sl.len[1]),
          kz0 = (T)(two_pi / sl.len[2]);
  const T inv_n = (T)(1.0 / ((double)Nx * Ny * Nz));
  std::vector<ppmg_halo_block> sends, recvs;
  for (int c = 0; c < lda; ++c) {
    const int tag_f = 40 + 2 * c, tag_b = 41 + 2 * c;
    k_fd_pack<T><<<blocks(nr), 256, 0, st>>>(field, fd, c, Nx, Ny, nzl, r);
    if (F::exec_fwd(plans.xy_fwd, r, spec) != CUFFT_SUCCESS) return 1;
    k_y_pack<C><<<blocks(nspec), 256, 0, st>>>(spec, H, Ny, nzl, P, me, z0me, nyl, doff, sendb,
                                               pen);
    count_launch(2);
    if ((ce = cudaGetLastError())) return 0;
    sends.clear();
    recvs.clear();
    for (int q = 0; q < P; ++q) {
      if (q == me) continue;
      int y0, ny;
      y_split(Ny, P, q, y0, ny);
      sends.push_back({q, tag_f, sendb + off[q], (int64_t)(sizeof(C) * nzl * ny * H)});
      recvs.push_back({q, tag_f, pen + (int64_t)sl.z0[q] * nyl * H,
                       (int64_t)(sizeof(C) * (size_t)sl.nz[q] * nyl * H)});
    }
    if (xchg((int)sends.size(), sends.data(), (int)recvs.size(), recvs.data())) return 2;
    if (C2C<T>::exec(plans.zc, pen, CUFFT_FORWARD) != CUFFT_SUCCESS) return 1;
    k_fd_spectral_pencil<T, C><<<blocks(npen), 256, 0, st>>>(pen, H, nyl, y0me, Ny, Nz, kx0, ky0,
                                                             kz0, inv_n);
    count_launch();
    if ((ce = cudaGetLastError())) return 0;
    if (C2C<T>::exec(plans.zc, pen, CUFFT_INVERSE) != CUFFT_SUCCESS) return 1;
    sends.clear();
    recvs.clear();
    for (int q = 0; q < P; ++q) {
      if (q == me) continue;
      int y0, ny;
      y_split(Ny, P, q, y0, ny);
      sends.push_back({q, tag_b, pen + (int64_t)sl.z0[q] * nyl * H,
                       (int64_t)(sizeof(C) * (size_t)sl.nz[q] * nyl * H)});
      recvs.push_back({q, tag_b, recvb + off[q], (int64_t)(sizeof(C) * nzl * ny * H)});
    }
    if (xchg((int)sends.size(), sends.data(), (int)recvs.size(), recvs.data())) return 2;
    k_y_unpack<C><<<blocks(nspec), 256, 0, st>>>(spec, H, Ny, nzl, P, me, z0me, nyl, doff, recvb,
                                                 pen);
    count_launch();
    if ((ce = cudaGetLastError())) return 0;
    if (F::exec_inv(plans.xy_inv, spec, r) != CUFFT_SUCCESS) return 1;
    const int64_t nb = (int64_t)(fd.box_hi[0] - fd.box_lo[0] + 1) *
                       (fd.box_hi[1] - fd.box_lo[1] + 1) * nzl;
    k_fd_unpack_slab<T><<<blocks(nb), 256, 0, st>>>(r, Nx, Ny, nzl, field, fd, c);
    count_launch();
    if ((ce = cudaGetLastError())) return 0;
  }
  return 0;
}

template int fd_poisson_slab<double>(SlabFFTPlans&, Workspace&, const SlabSolve&, double*,
                                     const FieldDesc&, int, cudaStream_t, const BlockExchange&,
                                     cudaError_t&);
template int fd_poisson_slab<float>(SlabFFTPlans&, Workspace&, const SlabSolve&, float*,
                                    const FieldDesc&, int, cudaStream_t, const BlockExchange&,
                                    cudaError_t&);

template int fd_poisson<double>(FFTPlans&, Workspace&, const int*, const double*, double*,
                                const FieldDesc&, int, cudaStream_t, cudaError_t&);
template int fd_poisson<float>(FFTPlans&, Workspace&, const int*, const double*, float*,
                               const FieldDesc&, int, cudaStream_t, cudaError_t&);

}  // namespace ppmg
