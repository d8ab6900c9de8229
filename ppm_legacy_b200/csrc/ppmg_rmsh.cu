// ppmg_rmsh.cu -- remeshing helpers (comp_weights, create_part), the periodic
// ghost get/put of one subdomain, and small conversion kernels.
#include <cuda_runtime.h>

#include "ppmg_rmsh.cuh"

namespace ppmg {

namespace {

int nblocks(int64_t n, int t = 256) {
  int64_t b = (n + t - 1) / t;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

// ---------------------------------------------------------------------------
// ppm_rmsh_comp_weights.f:851-996 per sorted particle: with
// xi = (x - min_phys)*dxi (dxi from the FP32 mesh spacing, Q1) and
// ip = INT(xi) + 2 - istart, the weights of nodes ip-1..ip+2 (M'4) or ip..ip+1
// (bsp2) at distances |ii - 2 + istart - xi|, tested with <= as the reference.
// Stored as (w_axis0[S], w_axis1[S], [w_axis2[S]]) per sorted particle.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T mp4_le(T x) {
  if (x <= T(2)) {
    if (x <= T(1)) return rsub(T(1), rmul(rmul(x, x), rsub(T(2.5), rmul(T(1.5), x))));
    return radd(T(2), rmul(radd(T(-4), rmul(rsub(T(2.5), rmul(T(0.5), x)), x)), x));
  }
  return T(0);
}

template <class T>
__global__ void k_comp_weights(CWParams<T> P) {
  const int S = P.S;
  const int64_t nv = min(P.nvalid, (int64_t)*P.d_nvalid);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nv;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = P.idx[s];
    const T* x = P.xp + p * P.ldxp;
    T* w = P.w + s * (int64_t)P.wstride;
    for (int a = 0; a < P.dim; ++a) {
      const T xi = rmul(rsub(x[a], P.min_phys[a]), P.dxiq[a]);
      const int ip = (int)xi + 2 - P.istart[a];
      const int lo = S == 4 ? ip - 1 : ip;
      for (int t = 0; t < S; ++t) {
        const int ii = lo + t;
        const T xd = fabs(rsub((T)(ii - 2 + P.istart[a]), xi));
        T v;
        if (S == 4) {
          v = mp4_le<T>(xd);
        } else {
          v = xd <= T(1) ? rsub(T(1), xd) : T(0);
        }
        w[a * S + t] = v;
      }
    }
  }
}

// Sorted weights -> the reference's user layout wx(1:2ks, 1:1, 1-ks:Np+ks)
// for one axis, indexed by the particle's list position (= id + 1).
template <class T>
__global__ void k_weights_to_user(const T* __restrict__ w, const int* __restrict__ idx,
                                  int64_t nvalid, const int* __restrict__ d_nvalid, int wstride,
                                  int S, int axis, T* __restrict__ out) {
  const int ks = S / 2;
  const int64_t nv = min(nvalid, (int64_t)*d_nvalid);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nv;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx[s];
    for (int t = 0; t < S; ++t)
      out[(int64_t)t + (int64_t)S * (p + ks)] = w[s * wstride + axis * S + t];
  }
}

// ---------------------------------------------------------------------------
// ppm_rmsh_create_part.f:427-681.  Nodes i=1..nn(0), j, k (periodic axes
// exclude node Nm) in Fortran order; flag[q] = 1 when the strength lies
// strictly inside the band.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t node_off(const FieldDesc& fd, int dim, int i, int j,
                                           int k) {
  int64_t o = (int64_t)(i - fd.lb[0]) * fd.s[0] + (int64_t)(j - fd.lb[1]) * fd.s[1];
  if (dim == 3) o += (int64_t)(k - fd.lb[2]) * fd.s[2];
  return o;
}

template <class T>
__global__ void k_cp_flag(CPParams<T> P, int* __restrict__ flag) {
  const int64_t nq = (int64_t)P.nn[0] * P.nn[1] * P.nn[2];
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % P.nn[0]) + 1;
    const int j = (int)((q / P.nn[0]) % P.nn[1]) + 1;
    const int k = (int)(q / ((int64_t)P.nn[0] * P.nn[1])) + 1;
    const T* f = P.field + node_off(P.fd, P.dim, i, j, k);
    T str;
    if (P.lda == 1 && P.cw == nullptr) {
      str = fabs(f[0]);
    } else {
      T sum = T(0);
      for (int a = 0; a < P.lda; ++a) {
        T v = f[a];
        if (P.cw) v = rmul(v, P.cw[a]);
        sum = radd(sum, rmul(v, v));
      }
      str = sqrt(sum);
    }
    flag[q] = (str > P.cut0 && str < P.cut1) ? 1 : 0;
  }
}

template <class T>
__global__ void k_cp_fill(CPParams<T> P, const int* __restrict__ flag,
                          const int* __restrict__ pos) {
  const int64_t nq = (int64_t)P.nn[0] * P.nn[1] * P.nn[2];
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq;
       q += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[q]) continue;
    const int64_t o = pos[q];
    const int i = (int)(q % P.nn[0]) + 1;
    const int j = (int)((q / P.nn[0]) % P.nn[1]) + 1;
    const int k = (int)(q / ((int64_t)P.nn[0] * P.nn[1])) + 1;
    const int64_t off = node_off(P.fd, P.dim, i, j, k);
    for (int a = 0; a < P.lda; ++a) P.up[o * P.lda + a] = P.field[off + a];
    if (P.wp && P.field_wp) {
      const int64_t ow = node_off(P.fdw, P.dim, i, j, k);
      for (int a = 0; a < P.lda2; ++a) P.wp[o * P.lda2 + a] = P.field_wp[ow + a];
    }
    if (P.xp) {
      const int idx[3] = {i, j, k};
      for (int a = 0; a < P.dim; ++a)
        P.xp[o * P.dim + a] = radd(rmul((T)(idx[a] - 1), P.h[a]), P.min_sub[a]);
    }
  }
}

// ---------------------------------------------------------------------------
// Periodic ghost get / put for one subdomain (ppm_map_field_ghost_get/put.f
// with the blocks of ppm_map_field_ghost_init.f:234-447 for nsubs = 1).
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_ghost_get(GhostParams P, T* __restrict__ F) {
  const int64_t ex = P.hi[0] - P.lo[0] + 1, ey = P.hi[1] - P.lo[1] + 1;
  const int64_t ez = P.dim == 3 ? P.hi[2] - P.lo[2] + 1 : 1;
  const int64_t n = ex * ey * ez;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % ex) + P.lo[0];
    const int j = (int)((q / ex) % ey) + P.lo[1];
    const int k = P.dim == 3 ? (int)(q / (ex * ey)) + P.lo[2] : 0;
    const bool real = i >= 1 && i <= P.N[0] && j >= 1 && j <= P.N[1] &&
                      (P.dim == 2 || (k >= 1 && k <= P.N[2]));
    if (real) continue;
    const int si = wrap_index(i - 1, P.N[0]) + 1;
    const int sj = wrap_index(j - 1, P.N[1]) + 1;
    const int sk = P.dim == 3 ? wrap_index(k - 1, P.N[2]) + 1 : 0;
    T* dst = F + node_off(P.fd, P.dim, i, j, k);
    const T* src = F + node_off(P.fd, P.dim, si, sj, sk);
    for (int a = 0; a < P.lda; ++a) dst[a] = src[a];
  }
}

// put, pass 1: tmp = sum over the periodic images (shifts -1, 0, +1 per
// periodic axis, as the reference's shift list) of every real node 1..Nm
template <class T>
__global__ void k_ghost_put_sum(GhostParams P, const T* __restrict__ F, T* __restrict__ tmp) {
  const int nmx = P.N[0] + 1, nmy = P.N[1] + 1, nmz = P.dim == 3 ? P.N[2] + 1 : 1;
  const int64_t n = (int64_t)nmx * nmy * nmz;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nmx) + 1;
    const int j = (int)((q / nmx) % nmy) + 1;
    const int k = P.dim == 3 ? (int)(q / ((int64_t)nmx * nmy)) + 1 : 0;
    for (int a = 0; a < P.lda; ++a) {
      T acc = F[node_off(P.fd, P.dim, i, j, k) + a];
      const int kmax = P.dim == 3 ? 1 : 0;
      for (int dk = -kmax; dk <= kmax; ++dk)
        for (int dj = -1; dj <= 1; ++dj)
          for (int di = -1; di <= 1; ++di) {
            if (di == 0 && dj == 0 && dk == 0) continue;
            const int ti = i + di * P.N[0], tj = j + dj * P.N[1];
            const int tk = P.dim == 3 ? k + dk * P.N[2] : 0;
            if (ti < P.lo[0] || ti > P.hi[0] || tj < P.lo[1] || tj > P.hi[1]) continue;
            if (P.dim == 3 && (tk < P.lo[2] || tk > P.hi[2])) continue;
            acc = acc + F[node_off(P.fd, P.dim, ti, tj, tk) + a];
          }
      tmp[q * P.lda + a] = acc;
    }
  }
}

template <class T>
__global__ void k_ghost_put_store(GhostParams P, const T* __restrict__ tmp, T* __restrict__ F) {
  const int nmx = P.N[0] + 1, nmy = P.N[1] + 1, nmz = P.dim == 3 ? P.N[2] + 1 : 1;
  const int64_t n = (int64_t)nmx * nmy * nmz;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nmx) + 1;
    const int j = (int)((q / nmx) % nmy) + 1;
    const int k = P.dim == 3 ? (int)(q / ((int64_t)nmx * nmy)) + 1 : 0;
    for (int a = 0; a < P.lda; ++a) F[node_off(P.fd, P.dim, i, j, k) + a] = tmp[q * P.lda + a];
  }
}

__global__ void k_plus_one(const int* __restrict__ in, int* __restrict__ out, int64_t n) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    out[q] = in[q] + 1;
}

}  // namespace

template <class T>
cudaError_t launch_comp_weights(const CWParams<T>& P, cudaStream_t st) {
  if (P.nvalid <= 0) return cudaSuccess;
  k_comp_weights<T><<<nblocks(P.nvalid), 256, 0, st>>>(P);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_weights_to_user(const T* w, const int* idx, int64_t nvalid,
                                   const int* d_nvalid, int wstride, int S, int axis, T* out,
                                   cudaStream_t st) {
  if (nvalid <= 0) return cudaSuccess;
  k_weights_to_user<T><<<nblocks(nvalid), 256, 0, st>>>(w, idx, nvalid, d_nvalid, wstride, S,
                                                        axis, out);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_cp_flag(const CPParams<T>& P, int* flag, cudaStream_t st) {
  const int64_t nq = (int64_t)P.nn[0] * P.nn[1] * P.nn[2];
  k_cp_flag<T><<<nblocks(nq), 256, 0, st>>>(P, flag);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_cp_fill(const CPParams<T>& P, const int* flag, const int* pos,
                           cudaStream_t st) {
  const int64_t nq = (int64_t)P.nn[0] * P.nn[1] * P.nn[2];
  k_cp_fill<T><<<nblocks(nq), 256, 0, st>>>(P, flag, pos);
  count_launch();
  return cudaGetLastError();
}

#define PPMG_RMSH_INST(T)                                                                     \
  template cudaError_t launch_comp_weights<T>(const CWParams<T>&, cudaStream_t);              \
  template cudaError_t launch_weights_to_user<T>(const T*, const int*, int64_t, const int*,   \
                                                 int, int, int, T*, cudaStream_t);            \
  template cudaError_t launch_cp_flag<T>(const CPParams<T>&, int*, cudaStream_t);             \
  template cudaError_t launch_cp_fill<T>(const CPParams<T>&, const int*, const int*,          \
                                         cudaStream_t);
PPMG_RMSH_INST(double)
PPMG_RMSH_INST(float)
#undef PPMG_RMSH_INST

template <class T>
cudaError_t launch_ghost(const GhostParams& P, int maptype, T* field, T* tmp,
                         cudaStream_t st) {
  if (maptype == kMapGhostGet) {
    const int64_t n = (int64_t)(P.hi[0] - P.lo[0] + 1) * (P.hi[1] - P.lo[1] + 1) *
                      (P.dim == 3 ? P.hi[2] - P.lo[2] + 1 : 1);
    k_ghost_get<T><<<nblocks(n), 256, 0, st>>>(P, field);
    count_launch();
  } else {
    const int64_t n = (int64_t)(P.N[0] + 1) * (P.N[1] + 1) * (P.dim == 3 ? P.N[2] + 1 : 1);
    k_ghost_put_sum<T><<<nblocks(n), 256, 0, st>>>(P, field, tmp);
    k_ghost_put_store<T><<<nblocks(n), 256, 0, st>>>(P, tmp, field);
    count_launch(2);
  }
  return cudaGetLastError();
}
template cudaError_t launch_ghost<double>(const GhostParams&, int, double*, double*,
                                          cudaStream_t);
template cudaError_t launch_ghost<float>(const GhostParams&, int, float*, float*, cudaStream_t);

cudaError_t launch_plus_one(const int* in, int* out, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_plus_one<<<nblocks(n), 256, 0, st>>>(in, out, n);
  count_launch();
  return cudaGetLastError();
}

}  // namespace ppmg
