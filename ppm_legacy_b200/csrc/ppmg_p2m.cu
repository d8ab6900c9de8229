// ppmg_p2m.cu -- deterministic particle -> mesh gather (replaces the scatter
// loops of ppm_interp_p2m.f:783-3663 and ppm_rmsh_remesh.f:614-868, and the
// ghost put cycle that follows them, ppm_interp_p2m.f:3665-3718).
//
// Design: particles are sorted by cell (ppmg_sort.cu).  A CTA owns a tile of
// 16 x 16 node columns and sweeps it in z.  For each cell layer it stages
// the particles of the (16+S-1)^2 cells whose stencils reach the tile into
// shared memory (1D weights computed once per staged particle), then each
// thread adds the contributions of the S x S cells around its column into a
// register window of S nodes.  A node is complete once the sweep has passed
// the last layer that reaches it; it is then written to field_up at its real
// position and at every periodic image inside the 1-g:Nm+g box (the fused
// ghost put/get).  Every node is produced by exactly one thread, in a fixed
// order: results are bitwise reproducible and need no atomics.
#include <cuda_runtime.h>

#include "ppmg_p2m.cuh"

namespace ppmg {

namespace {

constexpr int kTile = 16;
constexpr int kThreads = kTile * kTile;

template <class CT>
__device__ __forceinline__ void two_sum_fold(CT& hi, CT& lo, CT p) {
  CT s = hi + p;
  CT bp = s - hi;
  CT e = (hi - (s - bp)) + (p - bp);
  hi = s;
  lo = lo + e;
}

template <int S, class CT>
__device__ __forceinline__ void weights(CT f, CT w[S]) {
  if constexpr (S == 4) {
    if constexpr (sizeof(CT) == 8)
      mp4_weights_exact<CT>(f, w);
    else
      mp4_weights_fast<CT>(f, w);
  } else {
    bsp2_weights_exact<CT>(f, w);
  }
}

// Write one finished node value (components c0..c0+LC-1) to every image of
// unique node (x, y, z) inside the written box.
template <int DIM, class OT, int LC>
__device__ __forceinline__ void emit_node(const P2MParams& P, int x, int y, int z,
                                          const double v[LC]) {
  OT* F = static_cast<OT*>(P.field);
  const int n[3] = {x, y, z};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    // 1-based images n+1+t*N within [box_lo, box_hi]
    const int N = P.N[a];
    int tlo = (P.fd.box_lo[a] - n[a] - 1 + 64 * N) / N - 64;  // ceil for negatives
    if (n[a] + 1 + tlo * N < P.fd.box_lo[a]) ++tlo;
    int thi = (P.fd.box_hi[a] - n[a] - 1 + 64 * N) / N - 64;  // floor
    lo[a] = tlo;
    hi[a] = thi;
  }
  if (DIM == 2) {
    lo[2] = hi[2] = 0;
  }
  for (int tk = lo[2]; tk <= hi[2]; ++tk) {
    const int64_t oz =
        DIM == 3 ? (int64_t)(n[2] + 1 + tk * P.N[2] - P.fd.lb[2]) * P.fd.s[2] : 0;
    for (int tj = lo[1]; tj <= hi[1]; ++tj) {
      const int64_t oy = (int64_t)(n[1] + 1 + tj * P.N[1] - P.fd.lb[1]) * P.fd.s[1];
      for (int ti = lo[0]; ti <= hi[0]; ++ti) {
        const int64_t o = (int64_t)(n[0] + 1 + ti * P.N[0] - P.fd.lb[0]) * P.fd.s[0] + oy +
                          oz + P.c0;
#pragma unroll
        for (int a = 0; a < LC; ++a) F[o + a] = (OT)v[a];
      }
    }
  }
}

// --------------------------------------------------------------------------
// 3D tile gather.
// S: stencil width (4 = M'4, 2 = bsp2).  CT: arithmetic type.  COMP:
// compensated FP32 accumulation (per-layer partial sums folded into a
// (hi, lo) pair with an error-free TwoSum).  OT: field type.  LC: components
// handled by this launch (<= 4).
// --------------------------------------------------------------------------
template <int S, class CT, bool COMP, class OT, int LC, bool WST>
__global__ void __launch_bounds__(kThreads) k_p2m3d(P2MParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  constexpr int HH = S / 2 - 1;
  constexpr int WX = kTile + S - 1;
  constexpr int NSC = WX * WX;
  constexpr int PS = ((3 * S + 4) + 3) / 4 * 4;  // per-particle stride in CT
  constexpr int OFF_U = S;                        // [wz(S) | u(4) | wx(S) | wy(S)]
  constexpr int OFF_WX = S + 4;
  constexpr int OFF_WY = 2 * S + 4;

  extern __shared__ __align__(16) unsigned char smem[];
  int* sc = reinterpret_cast<int*>(smem);  // NSC + 1 prefix offsets
  int* sb = sc + NSC + 1;                  // NSC global starts
  size_t off = (size_t)(2 * NSC + 1) * sizeof(int);
  off = (off + 15) & ~(size_t)15;
  CT* sw = reinterpret_cast<CT*>(smem + off);
  unsigned char* sqx = reinterpret_cast<unsigned char*>(sw + (size_t)P.cap * PS);

  const int tid = threadIdx.x;
  const int tx = tid % kTile, ty = tid / kTile;
  const int tiles_x = (P.N[0] + kTile - 1) / kTile;
  const int X0 = (blockIdx.x % tiles_x) * kTile;
  const int Y0 = (blockIdx.x / tiles_x) * kTile;
  const int Z0 = blockIdx.y * P.TZ;
  const int Z1 = min(Z0 + P.TZ, P.N[2]);
  const int x = X0 + tx, y = Y0 + ty;
  const bool active = x < P.N[0] && y < P.N[1];
  const V* rec = static_cast<const V*>(P.rec);
  const V* us = static_cast<const V*>(P.us);

  CT acc[S][LC];  // plain window (or per-layer partials when COMP)
  CT hi[S][LC], lo[S][LC];
#pragma unroll
  for (int k = 0; k < S; ++k)
#pragma unroll
    for (int a = 0; a < LC; ++a) acc[k][a] = hi[k][a] = lo[k][a] = CT(0);

  for (int cz = Z0 - HL; cz <= Z1 - 1 + HH; ++cz) {
    const int czw = wrap_index(cz, P.N[2]);
    // 1. particle counts of the staged cells
    for (int q = tid; q < NSC; q += kThreads) {
      const int r = q / WX, qx = q % WX;
      const int cx = wrap_index(X0 - HL + qx, P.N[0]);
      const int cy = wrap_index(Y0 - HL + r, P.N[1]);
      const int64_t c = (int64_t)cx + (int64_t)P.N[0] * (cy + (int64_t)P.N[1] * czw);
      const int b = P.start[c];
      sb[q] = b;
      sc[q] = P.start[c + 1] - b;
    }
    __syncthreads();
    // 2. exclusive scan of the counts (two per thread, NSC <= 2*kThreads)
    {
      const int i0 = 2 * tid, i1 = 2 * tid + 1;
      const int v0 = i0 < NSC ? sc[i0] : 0;
      const int v1 = i1 < NSC ? sc[i1] : 0;
      int v = v0 + v1;
      // warp inclusive scan
      const int lane = tid & 31, wid = tid >> 5;
      int inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      __shared__ int wsum[kThreads / 32 + 1];
      if (lane == 31) wsum[wid] = inc;
      __syncthreads();
      if (tid == 0) {
        int run = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
          int t = wsum[w];
          wsum[w] = run;
          run += t;
        }
        wsum[kThreads / 32] = run;
      }
      __syncthreads();
      const int ex = inc - v + wsum[wid];
      if (i0 < NSC) sc[i0] = ex;
      if (i1 < NSC) sc[i1] = ex + v0;
      if (tid == 0) sc[NSC] = wsum[kThreads / 32];
      __syncthreads();
    }
    const int total = sc[NSC];
    for (int cb = 0; cb < total; cb += P.cap) {
      const int n = min(P.cap, total - cb);
      // 3. stage particles [cb, cb+n) of the layer's staged cells
      for (int i = tid; i < n; i += kThreads) {
        const int pos = cb + i;
        int lo_q = 0, hi_q = NSC;  // largest q with sc[q] <= pos
        while (hi_q - lo_q > 1) {
          const int mid = (lo_q + hi_q) >> 1;
          if (sc[mid] <= pos) lo_q = mid; else hi_q = mid;
        }
        const int64_t s = (int64_t)sb[lo_q] + (pos - sc[lo_q]);
        const V u = us[s];
        CT w[3][S];
        if constexpr (WST) {
          // remesh: the 1D weights of ppm_rmsh_comp_weights, stored per
          // sorted particle as (wx[S], wy[S], wz[S]) in FP64
          const double* ws = static_cast<const double*>(P.rec) + s * (3 * S);
#pragma unroll
          for (int k = 0; k < S; ++k) {
            w[0][k] = (CT)ws[k];
            w[1][k] = (CT)ws[S + k];
            w[2][k] = (CT)ws[2 * S + k];
          }
        } else {
          const V r = rec[s];
          weights<S, CT>(r.x, w[0]);
          weights<S, CT>(r.y, w[1]);
          weights<S, CT>(r.z, w[2]);
        }
        CT* d = sw + (size_t)i * PS;
#pragma unroll
        for (int k = 0; k < S; ++k) {
          d[k] = w[2][k];
          d[OFF_WX + k] = w[0][k];
          d[OFF_WY + k] = w[1][k];
        }
        d[OFF_U + 0] = u.x;
        d[OFF_U + 1] = u.y;
        d[OFF_U + 2] = u.z;
        d[OFF_U + 3] = u.w;
        sqx[i] = (unsigned char)(lo_q % WX);
      }
      __syncthreads();
      // 4. accumulate the S x S cells around this thread's column
      if (active) {
#pragma unroll
        for (int dy = 0; dy < S; ++dy) {
          const int row = ty + dy;
          const int pb = max(sc[row * WX + tx], cb);
          const int pe = min(sc[row * WX + tx + S], cb + n);
          for (int pos = pb; pos < pe; ++pos) {
            const int i = pos - cb;
            const CT* d = sw + (size_t)i * PS;
            const int wi = tx - (int)sqx[i] + S - 1;
            const CT c = d[OFF_WX + wi] * d[OFF_WY + S - 1 - dy];
            CT wz[S], uu[4];
            if constexpr (S == 4 && sizeof(CT) == 4) {
              const float4 a = *reinterpret_cast<const float4*>(d);
              wz[0] = a.x; wz[1] = a.y; wz[2] = a.z; wz[3] = a.w;
            } else {
#pragma unroll
              for (int k = 0; k < S; ++k) wz[k] = d[k];
            }
            if constexpr (sizeof(CT) == 4) {
              const float4 b = *reinterpret_cast<const float4*>(d + OFF_U);
              uu[0] = b.x; uu[1] = b.y; uu[2] = b.z; uu[3] = b.w;
            } else {
#pragma unroll
              for (int a = 0; a < 4; ++a) uu[a] = d[OFF_U + a];
            }
#pragma unroll
            for (int a = 0; a < LC; ++a) {
              const CT cu = c * uu[a];
#pragma unroll
              for (int k = 0; k < S; ++k) acc[k][a] += cu * wz[k];
            }
          }
        }
      }
      __syncthreads();
    }
    // 5. node zc = cz - (HL-1) is complete: fold, emit, shift the window
    const int zc = cz - (HL - 1);
    if constexpr (COMP) {
#pragma unroll
      for (int k = 0; k < S; ++k)
#pragma unroll
        for (int a = 0; a < LC; ++a) {
          two_sum_fold<CT>(hi[k][a], lo[k][a], acc[k][a]);
          acc[k][a] = CT(0);
        }
    }
    if (active && zc >= Z0 && zc < Z1) {
      double v[LC];
#pragma unroll
      for (int a = 0; a < LC; ++a)
        v[a] = COMP ? (double)hi[0][a] + (double)lo[0][a] : (double)acc[0][a];
      emit_node<3, OT, LC>(P, x, y, zc, v);
    }
#pragma unroll
    for (int k = 0; k < S - 1; ++k)
#pragma unroll
      for (int a = 0; a < LC; ++a) {
        if constexpr (COMP) {
          hi[k][a] = hi[k + 1][a];
          lo[k][a] = lo[k + 1][a];
        } else {
          acc[k][a] = acc[k + 1][a];
        }
      }
#pragma unroll
    for (int a = 0; a < LC; ++a) {
      if constexpr (COMP) {
        hi[S - 1][a] = CT(0);
        lo[S - 1][a] = CT(0);
      } else {
        acc[S - 1][a] = CT(0);
      }
    }
  }
}

// --------------------------------------------------------------------------
// 2D tile gather: a CTA owns 128 node columns along x and sweeps y.
// (The reference's 2D P2M supports M'4 only, ppm_interp_p2m.f:3657-3662.)
// --------------------------------------------------------------------------
constexpr int kTile2 = 128;

template <int S, class CT, bool COMP, class OT, int LC, bool WST>
__global__ void __launch_bounds__(kTile2) k_p2m2d(P2MParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  constexpr int HH = S / 2 - 1;
  constexpr int WX = kTile2 + S - 1;
  constexpr int PS = ((2 * S + 4) + 3) / 4 * 4;  // [wy(S) | u(4) | wx(S)]
  constexpr int OFF_U = S;
  constexpr int OFF_WX = S + 4;

  extern __shared__ __align__(16) unsigned char smem[];
  int* sc = reinterpret_cast<int*>(smem);  // WX + 1
  int* sb = sc + WX + 1;
  size_t off = (size_t)(2 * WX + 1) * sizeof(int);
  off = (off + 15) & ~(size_t)15;
  CT* sw = reinterpret_cast<CT*>(smem + off);
  unsigned char* sqx = reinterpret_cast<unsigned char*>(sw + (size_t)P.cap * PS);

  const int tid = threadIdx.x;
  const int X0 = blockIdx.x * kTile2;
  const int Y0 = blockIdx.y * P.TZ;
  const int Y1 = min(Y0 + P.TZ, P.N[1]);
  const int x = X0 + tid;
  const bool active = x < P.N[0];
  const V* rec = static_cast<const V*>(P.rec);
  const V* us = static_cast<const V*>(P.us);

  CT acc[S][LC], hi[S][LC], lo[S][LC];
#pragma unroll
  for (int k = 0; k < S; ++k)
#pragma unroll
    for (int a = 0; a < LC; ++a) acc[k][a] = hi[k][a] = lo[k][a] = CT(0);

  for (int cy = Y0 - HL; cy <= Y1 - 1 + HH; ++cy) {
    const int cyw = wrap_index(cy, P.N[1]);
    if (tid == 0) {
      int run = 0;
      for (int q = 0; q < WX; ++q) {
        const int cx = wrap_index(X0 - HL + q, P.N[0]);
        const int64_t c = (int64_t)cx + (int64_t)P.N[0] * cyw;
        const int b = P.start[c];
        sb[q] = b;
        sc[q] = run;
        run += P.start[c + 1] - b;
      }
      sc[WX] = run;
    }
    __syncthreads();
    const int total = sc[WX];
    for (int cb = 0; cb < total; cb += P.cap) {
      const int n = min(P.cap, total - cb);
      for (int i = tid; i < n; i += kTile2) {
        const int pos = cb + i;
        int lo_q = 0, hi_q = WX;
        while (hi_q - lo_q > 1) {
          const int mid = (lo_q + hi_q) >> 1;
          if (sc[mid] <= pos) lo_q = mid; else hi_q = mid;
        }
        const int64_t s = (int64_t)sb[lo_q] + (pos - sc[lo_q]);
        const V u = us[s];
        CT w[2][S];
        if constexpr (WST) {
          const double* ws = static_cast<const double*>(P.rec) + s * (2 * S);
#pragma unroll
          for (int k = 0; k < S; ++k) {
            w[0][k] = (CT)ws[k];
            w[1][k] = (CT)ws[S + k];
          }
        } else {
          const V r = rec[s];
          weights<S, CT>(r.x, w[0]);
          weights<S, CT>(r.y, w[1]);
        }
        CT* d = sw + (size_t)i * PS;
#pragma unroll
        for (int k = 0; k < S; ++k) {
          d[k] = w[1][k];
          d[OFF_WX + k] = w[0][k];
        }
        d[OFF_U + 0] = u.x;
        d[OFF_U + 1] = u.y;
        d[OFF_U + 2] = u.z;
        d[OFF_U + 3] = u.w;
        sqx[i] = (unsigned char)lo_q;
      }
      __syncthreads();
      if (active) {
        const int pb = max(sc[tid], cb);
        const int pe = min(sc[tid + S], cb + n);
        for (int pos = pb; pos < pe; ++pos) {
          const int i = pos - cb;
          const CT* d = sw + (size_t)i * PS;
          const CT c = d[OFF_WX + tid - (int)sqx[i] + S - 1];
#pragma unroll
          for (int a = 0; a < LC; ++a) {
            const CT cu = c * d[OFF_U + a];
#pragma unroll
            for (int k = 0; k < S; ++k) acc[k][a] += cu * d[k];
          }
        }
      }
      __syncthreads();
    }
    const int yc = cy - (HL - 1);
    if constexpr (COMP) {
#pragma unroll
      for (int k = 0; k < S; ++k)
#pragma unroll
        for (int a = 0; a < LC; ++a) {
          two_sum_fold<CT>(hi[k][a], lo[k][a], acc[k][a]);
          acc[k][a] = CT(0);
        }
    }
    if (active && yc >= Y0 && yc < Y1) {
      double v[LC];
#pragma unroll
      for (int a = 0; a < LC; ++a)
        v[a] = COMP ? (double)hi[0][a] + (double)lo[0][a] : (double)acc[0][a];
      emit_node<2, OT, LC>(P, x, yc, 0, v);
    }
#pragma unroll
    for (int k = 0; k < S - 1; ++k)
#pragma unroll
      for (int a = 0; a < LC; ++a) {
        if constexpr (COMP) {
          hi[k][a] = hi[k + 1][a];
          lo[k][a] = lo[k + 1][a];
        } else {
          acc[k][a] = acc[k + 1][a];
        }
      }
#pragma unroll
    for (int a = 0; a < LC; ++a) {
      if constexpr (COMP) {
        hi[S - 1][a] = CT(0);
        lo[S - 1][a] = CT(0);
      } else {
        acc[S - 1][a] = CT(0);
      }
    }
  }
}

template <int S, class CT, bool COMP, class OT, int LC, bool WST>
cudaError_t launch_lc(const P2MParams& P, int dim, cudaStream_t st) {
  if (dim == 3) {
    constexpr int WX = kTile + S - 1;
    constexpr int NSC = WX * WX;
    constexpr int PS = ((3 * S + 4) + 3) / 4 * 4;
    size_t off = ((size_t)(2 * NSC + 1) * sizeof(int) + 15) & ~(size_t)15;
    size_t smem = off + (size_t)P.cap * PS * sizeof(CT) + (size_t)P.cap;
    auto kern = k_p2m3d<S, CT, COMP, OT, LC, WST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int tiles_x = (P.N[0] + kTile - 1) / kTile;
    const int tiles_y = (P.N[1] + kTile - 1) / kTile;
    const int tiles_z = (P.N[2] + P.TZ - 1) / P.TZ;
    dim3 grid(tiles_x * tiles_y, tiles_z);
    kern<<<grid, kThreads, smem, st>>>(P);
  } else {
    constexpr int WX = kTile2 + S - 1;
    constexpr int PS = ((2 * S + 4) + 3) / 4 * 4;
    size_t off = ((size_t)(2 * WX + 1) * sizeof(int) + 15) & ~(size_t)15;
    size_t smem = off + (size_t)P.cap * PS * sizeof(CT) + (size_t)P.cap;
    auto kern = k_p2m2d<S, CT, COMP, OT, LC, WST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((P.N[0] + kTile2 - 1) / kTile2, (P.N[1] + P.TZ - 1) / P.TZ);
    kern<<<grid, kTile2, smem, st>>>(P);
  }
  count_launch();
  return cudaGetLastError();
}

template <int S, class CT, bool COMP, class OT, bool WST>
cudaError_t launch_s(const P2MParams& P, int dim, int lc, cudaStream_t st) {
  switch (lc) {
    case 1: return launch_lc<S, CT, COMP, OT, 1, WST>(P, dim, st);
    case 2: return launch_lc<S, CT, COMP, OT, 2, WST>(P, dim, st);
    case 3: return launch_lc<S, CT, COMP, OT, 3, WST>(P, dim, st);
    default: return launch_lc<S, CT, COMP, OT, 4, WST>(P, dim, st);
  }
}

template <int S, class CT, bool COMP, class OT>
cudaError_t launch_w(const P2MParams& P, int dim, int lc, bool wst, cudaStream_t st) {
  return wst ? launch_s<S, CT, COMP, OT, true>(P, dim, lc, st)
             : launch_s<S, CT, COMP, OT, false>(P, dim, lc, st);
}

}  // namespace

int p2m_tile_depth(int dim, const int N[3]) {
  if (dim == 2) {
    const int tx = (N[0] + kTile2 - 1) / kTile2;
    int want = (148 * 8 + tx - 1) / tx;  // ~8 CTAs per SM in total
    int tz = (N[1] + want - 1) / want;
    return tz < 8 ? (N[1] < 8 ? N[1] : 8) : tz;
  }
  const int txy = ((N[0] + kTile - 1) / kTile) * ((N[1] + kTile - 1) / kTile);
  int want = (148 * 3 * 8 + txy - 1) / txy;  // ~8 waves of 3 CTAs per SM
  int tz = (N[2] + want - 1) / want;
  if (tz < 8) tz = 8;
  if (tz > 64) tz = 64;
  if (tz > N[2]) tz = N[2];
  return tz;
}

cudaError_t launch_p2m(const P2MParams& P0, int dim, int kernel, P2MPrec prec, int lda,
                       int64_t nvalid, bool stored_weights, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  const int nchunk = (lda + 3) / 4;
  for (int ch = 0; ch < nchunk; ++ch) {
    P2MParams P = P0;
    const int lc = lda - 4 * ch < 4 ? lda - 4 * ch : 4;
    P.c0 = 4 * ch;
    const size_t vsz = prec == P2M_FP64 ? sizeof(double4) : sizeof(float4);
    P.us = static_cast<const char*>(P0.us) + (size_t)ch * (size_t)nvalid * vsz;
    if (kernel == kKernelMp4) {
      switch (prec) {
        case P2M_FP64: e = launch_w<4, double, false, double>(P, dim, lc, stored_weights, st); break;
        case P2M_MIXED: e = launch_w<4, float, true, double>(P, dim, lc, stored_weights, st); break;
        case P2M_FP32: e = launch_w<4, float, false, float>(P, dim, lc, stored_weights, st); break;
      }
    } else {
      switch (prec) {
        case P2M_FP64: e = launch_w<2, double, false, double>(P, dim, lc, stored_weights, st); break;
        case P2M_MIXED: e = launch_w<2, float, true, double>(P, dim, lc, stored_weights, st); break;
        case P2M_FP32: e = launch_w<2, float, false, float>(P, dim, lc, stored_weights, st); break;
      }
    }
    if (e != cudaSuccess) return e;
  }
  return e;
}

}  // namespace ppmg
