// ppmg_m2p.cu -- mesh -> particle gather (ppm_interp_m2p.f:777-4105) and the
// adjoint of P2M.
//
// Particles are visited in cell order (ppmg_sort.cu), so neighbouring
// threads read overlapping stencils and the field is served from L1/L2.
// Each thread forms its 1D weights from the sorted FP64/FP32 offsets and sums
// the S^d nodes per component in the reference's term order (x outermost,
// z innermost).  The FP64 form evaluates every product and sum without
// contraction, in the reference's association, so it reproduces the
// reference's M2P to the last bit for the same weights.  Periodic wrap
// replaces the client's ghost get: only real nodes 1..Nm-1 are read.
#include <cuda_runtime.h>

#include "ppmg_m2p.cuh"

namespace ppmg {

namespace {

template <int S, class CT, bool EXACT>
__device__ __forceinline__ void m2p_weights(CT f, CT w[S]) {
  if constexpr (S == 4) {
    if constexpr (EXACT)
      mp4_weights_exact<CT>(f, w);
    else
      mp4_weights_fast<CT>(f, w);
  } else {
    bsp2_weights_exact<CT>(f, w);
  }
}

// 2D M'4 in the reference's |x| branching form (ppm_interp_m2p.f:829-845):
// w(ii) for ii = -1..2 at x = |f - ii|.
template <class CT, bool EXACT>
__device__ __forceinline__ void mp4_weights_abs(CT f, CT w[4]) {
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const CT x = fabs(rsub(f, CT(t - 1)));
    if constexpr (EXACT) {
      w[t] = x < CT(1) ? rsub(CT(1), rmul(rmul(x, x), rsub(CT(2.5), rmul(CT(1.5), x))))
                       : radd(CT(2), rmul(radd(CT(-4), rmul(rsub(CT(2.5), rmul(CT(0.5), x)), x)), x));
    } else {
      w[t] = x < CT(1) ? CT(1) - (x * x) * (CT(2.5) - CT(1.5) * x)
                       : CT(2) + (CT(-4) + (CT(2.5) - CT(0.5) * x) * x) * x;
    }
  }
}

template <class CT, bool EXACT>
__device__ __forceinline__ CT mul(CT a, CT b) {
  if constexpr (EXACT) return rmul(a, b); else return a * b;
}

template <class CT, bool EXACT>
__device__ __forceinline__ CT fma_acc(CT acc, CT w, CT v) {
  if constexpr (EXACT) return radd(acc, rmul(w, v)); else return fma(w, v, acc);
}

template <int S, class CT, bool EXACT, class FT>
__global__ void __launch_bounds__(256) k_m2p3d(M2PParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nvalid || s >= (int64_t)*P.d_nvalid) return;
  const V r = static_cast<const V*>(P.rec)[s];
  int cell;
  if constexpr (sizeof(CT) == 4) cell = __float_as_int(r.w); else cell = (int)r.w;
  const int cx = cell % P.N[0];
  const int cy = (cell / P.N[0]) % P.N[1];
  const int cz = cell / (P.N[0] * P.N[1]);
  CT wx[S], wy[S], wz[S];
  m2p_weights<S, CT, EXACT>(r.x, wx);
  m2p_weights<S, CT, EXACT>(r.y, wy);
  m2p_weights<S, CT, EXACT>(r.z, wz);
  int64_t ox[S], oy[S], oz[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    ox[i] = (int64_t)(wrap_index(cx - (HL - 1) + i, P.N[0]) + 1 - P.fd.lb[0]) * P.fd.s[0];
    oy[i] = (int64_t)(wrap_index(cy - (HL - 1) + i, P.N[1]) + 1 - P.fd.lb[1]) * P.fd.s[1];
    oz[i] = (int64_t)(wrap_index(cz - (HL - 1) + i, P.N[2]) + 1 - P.fd.lb[2]) * P.fd.s[2];
  }
  const FT* F = static_cast<const FT*>(P.field);
  FT* up = static_cast<FT*>(P.up) + (int64_t)P.idx[s] * P.ldup;
  for (int a = 0; a < P.lda; ++a) {
    CT acc = CT(0);
#pragma unroll 1
    for (int i = 0; i < S; ++i)
#pragma unroll
      for (int j = 0; j < S; ++j) {
        const CT wij = mul<CT, EXACT>(wx[i], wy[j]);
        const int64_t oij = ox[i] + oy[j] + a;
#pragma unroll
        for (int k = 0; k < S; ++k) {
          const CT v = (CT)__ldg(F + oij + oz[k]);
          acc = fma_acc<CT, EXACT>(acc, mul<CT, EXACT>(wij, wz[k]), v);
        }
      }
    up[a] = (FT)acc;
  }
}

template <int S, class CT, bool EXACT, class FT>
__global__ void __launch_bounds__(256) k_m2p2d(M2PParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nvalid || s >= (int64_t)*P.d_nvalid) return;
  const V r = static_cast<const V*>(P.rec)[s];
  int cell;
  if constexpr (sizeof(CT) == 4) cell = __float_as_int(r.w); else cell = (int)r.w;
  const int cx = cell % P.N[0];
  const int cy = cell / P.N[0];
  CT wx[S], wy[S];
  if constexpr (S == 4) {
    mp4_weights_abs<CT, EXACT>(r.x, wx);
    mp4_weights_abs<CT, EXACT>(r.y, wy);
  } else {
    bsp2_weights_exact<CT>(r.x, wx);
    bsp2_weights_exact<CT>(r.y, wy);
  }
  int64_t ox[S], oy[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    ox[i] = (int64_t)(wrap_index(cx - (HL - 1) + i, P.N[0]) + 1 - P.fd.lb[0]) * P.fd.s[0];
    oy[i] = (int64_t)(wrap_index(cy - (HL - 1) + i, P.N[1]) + 1 - P.fd.lb[1]) * P.fd.s[1];
  }
  const FT* F = static_cast<const FT*>(P.field);
  FT* up = static_cast<FT*>(P.up) + (int64_t)P.idx[s] * P.ldup;
  for (int a = 0; a < P.lda; ++a) {
    CT acc = CT(0);
    if constexpr (S == 4) {
      // reference order: jj outer, ii inner (ppm_interp_m2p.f:829-848)
#pragma unroll
      for (int j = 0; j < S; ++j)
#pragma unroll
        for (int i = 0; i < S; ++i)
          acc = fma_acc<CT, EXACT>(acc, mul<CT, EXACT>(wx[i], wy[j]),
                                   (CT)__ldg(F + ox[i] + oy[j] + a));
    } else {
      // bsp2: i outer, j inner (ppm_interp_m2p.f:3290-3297)
#pragma unroll
      for (int i = 0; i < S; ++i)
#pragma unroll
        for (int j = 0; j < S; ++j)
          acc = fma_acc<CT, EXACT>(acc, mul<CT, EXACT>(wx[i], wy[j]),
                                   (CT)__ldg(F + ox[i] + oy[j] + a));
    }
    up[a] = (FT)acc;
  }
}

// Adjoint of P2M (3D): dw = M2P(r) with P2M's weights, dx = sum_a u_a grad.
template <int S, class CT>
__global__ void __launch_bounds__(256) k_adjoint3d(M2PParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nvalid || s >= (int64_t)*P.d_nvalid) return;
  const V r = static_cast<const V*>(P.rec)[s];
  int cell;
  if constexpr (sizeof(CT) == 4) cell = __float_as_int(r.w); else cell = (int)r.w;
  const int cx = cell % P.N[0];
  const int cy = (cell / P.N[0]) % P.N[1];
  const int cz = cell / (P.N[0] * P.N[1]);
  const CT f[3] = {r.x, r.y, r.z};
  CT w[3][S], dw[3][S];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if constexpr (S == 4) {
      mp4_weights_fast<CT>(f[a], w[a]);
      mp4_dweights<CT>(f[a], dw[a]);
    } else {
      w[a][0] = CT(1) - f[a];
      w[a][1] = f[a];
      dw[a][0] = CT(-1);
      dw[a][1] = CT(1);
    }
#pragma unroll
    for (int i = 0; i < S; ++i) dw[a][i] *= (CT)P.dxi[a];
  }
  int64_t ox[S], oy[S], oz[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    ox[i] = (int64_t)(wrap_index(cx - (HL - 1) + i, P.N[0]) + 1 - P.fd.lb[0]) * P.fd.s[0];
    oy[i] = (int64_t)(wrap_index(cy - (HL - 1) + i, P.N[1]) + 1 - P.fd.lb[1]) * P.fd.s[1];
    oz[i] = (int64_t)(wrap_index(cz - (HL - 1) + i, P.N[2]) + 1 - P.fd.lb[2]) * P.fd.s[2];
  }
  const double* F = static_cast<const double*>(P.field);
  const int64_t p = P.idx[s];
  double* out = static_cast<double*>(P.up) + p * P.ldup;
  const double* u = P.upin + p * P.ldupin;
  CT g[3] = {CT(0), CT(0), CT(0)};
  for (int a = 0; a < P.lda; ++a) {
    CT acc = CT(0), gx = CT(0), gy = CT(0), gz = CT(0);
#pragma unroll 1
    for (int i = 0; i < S; ++i)
#pragma unroll
      for (int j = 0; j < S; ++j) {
        const CT wij = w[0][i] * w[1][j];
        const CT dxij = dw[0][i] * w[1][j];
        const CT dyij = w[0][i] * dw[1][j];
#pragma unroll
        for (int k = 0; k < S; ++k) {
          const CT v = (CT)__ldg(F + ox[i] + oy[j] + oz[k] + a);
          acc += wij * w[2][k] * v;
          gx += dxij * w[2][k] * v;
          gy += dyij * w[2][k] * v;
          gz += wij * dw[2][k] * v;
        }
      }
    out[a] = (double)acc;
    const CT ua = (CT)u[a];
    g[0] += ua * gx;
    g[1] += ua * gy;
    g[2] += ua * gz;
  }
  double* dx = P.dx + p * P.lddx;
  dx[0] = (double)g[0];
  dx[1] = (double)g[1];
  dx[2] = (double)g[2];
}

int blocks_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_m2p(const M2PParams& P, int dim, int kernel, M2PPrec prec, cudaStream_t st) {
  if (P.nvalid <= 0) return cudaSuccess;
  const int nb = blocks_for(P.nvalid);
  if (dim == 3) {
    if (kernel == kKernelMp4) {
      switch (prec) {
        case M2P_FP64: k_m2p3d<4, double, true, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_MIXED: k_m2p3d<4, float, false, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_FP32: k_m2p3d<4, float, false, float><<<nb, 256, 0, st>>>(P); break;
      }
    } else {
      switch (prec) {
        case M2P_FP64: k_m2p3d<2, double, true, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_MIXED: k_m2p3d<2, float, false, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_FP32: k_m2p3d<2, float, false, float><<<nb, 256, 0, st>>>(P); break;
      }
    }
  } else {
    if (kernel == kKernelMp4) {
      switch (prec) {
        case M2P_FP64: k_m2p2d<4, double, true, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_MIXED: k_m2p2d<4, float, false, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_FP32: k_m2p2d<4, float, false, float><<<nb, 256, 0, st>>>(P); break;
      }
    } else {
      switch (prec) {
        case M2P_FP64: k_m2p2d<2, double, true, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_MIXED: k_m2p2d<2, float, false, double><<<nb, 256, 0, st>>>(P); break;
        case M2P_FP32: k_m2p2d<2, float, false, float><<<nb, 256, 0, st>>>(P); break;
      }
    }
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_adjoint(const M2PParams& P, int kernel, M2PPrec prec, cudaStream_t st) {
  if (P.nvalid <= 0) return cudaSuccess;
  const int nb = blocks_for(P.nvalid);
  if (kernel == kKernelMp4) {
    if (prec == M2P_FP64) k_adjoint3d<4, double><<<nb, 256, 0, st>>>(P);
    else k_adjoint3d<4, float><<<nb, 256, 0, st>>>(P);
  } else {
    if (prec == M2P_FP64) k_adjoint3d<2, double><<<nb, 256, 0, st>>>(P);
    else k_adjoint3d<2, float><<<nb, 256, 0, st>>>(P);
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace ppmg
