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

// 0-based node of stencil node n along axis a: periodic wrap, or (a cut
// axis) the node itself, ghost nodes included
__device__ __forceinline__ int node_at(const M2PParams& P, int a, int n) {
  return P.open[a] ? n : wrap_index(n, P.N[a]);
}

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

// dW/dx of the 1D weights times the inverse mesh spacing (adjoint of P2M).
template <int S, class CT>
__device__ __forceinline__ void adj_dweights(CT f, CT dxi, CT d[S]) {
  if constexpr (S == 4) {
    mp4_dweights<CT>(f, d);
  } else {
    d[0] = CT(-1);
    d[1] = CT(1);
  }
#pragma unroll
  for (int i = 0; i < S; ++i) d[i] *= dxi;
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
  const V r = load_vec(static_cast<const V*>(P.rec), s, P.nvalid);
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
    ox[i] = (int64_t)(node_at(P, 0, cx - (HL - 1) + i) + 1 - P.fd.lb[0]) * P.fd.s[0];
    oy[i] = (int64_t)(node_at(P, 1, cy - (HL - 1) + i) + 1 - P.fd.lb[1]) * P.fd.s[1];
    oz[i] = (int64_t)(node_at(P, 2, cz - (HL - 1) + i) + 1 - P.fd.lb[2]) * P.fd.s[2];
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
  const V r = load_vec(static_cast<const V*>(P.rec), s, P.nvalid);
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
  const V r = load_vec(static_cast<const V*>(P.rec), s, P.nvalid);
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
    ox[i] = (int64_t)(node_at(P, 0, cx - (HL - 1) + i) + 1 - P.fd.lb[0]) * P.fd.s[0];
    oy[i] = (int64_t)(node_at(P, 1, cy - (HL - 1) + i) + 1 - P.fd.lb[1]) * P.fd.s[1];
    oz[i] = (int64_t)(node_at(P, 2, cz - (HL - 1) + i) + 1 - P.fd.lb[2]) * P.fd.s[2];
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

// --------------------------------------------------------------------------
// 3D tile gather (M2P).  A CTA owns the particles of a work item's cells
// (kTileX x kTileY cells over [Z0, Z1)).  The nodes their stencils read are
// staged in shared memory as a ring of S node planes along z: per node column
// (x, y) the S ring slots x LC components are contiguous, so a particle reads
// each of its S x S columns with LC*S/4 vector loads and consecutive
// particles (consecutive cells) hit disjoint banks.  One new plane is loaded
// per cell layer; particles of the layer are spread over all threads.
// EXACT (FP64 form): the terms are summed per component in the reference's
// order (x outer, z inner) with the reference's association, no contraction.
// ADJ (adjoint of P2M): the ring holds the adjoint field r; every particle
// gets dw(a) = sum_n W r(a) and dx(d) = sum_a u(a) sum_n d_d W r(a), the
// derivative weights scaled by the inverse mesh spacing (all LC = lda
// components in one launch).
// --------------------------------------------------------------------------
// One particle's LC results to up(c0:c0+LC-1, p).  Rows land at random
// addresses, so every store is a separate L2 request: three FP64 values go
// as one 16-byte and one 8-byte store (the row starts 8 or 16 bytes past a
// 16-byte boundary; which of the two pairs is aligned follows from it).
template <class FT, class CT, int LC>
__device__ __forceinline__ void store_row(FT* out, const CT* acc) {
  if constexpr (sizeof(FT) == 8 && LC == 3) {
    double* o = reinterpret_cast<double*>(out);
    if ((reinterpret_cast<uintptr_t>(out) & 15) == 0) {
      __stcs(reinterpret_cast<double2*>(o), make_double2((double)acc[0], (double)acc[1]));
      __stcs(o + 2, (double)acc[2]);
    } else {
      __stcs(o, (double)acc[0]);
      __stcs(reinterpret_cast<double2*>(o + 1), make_double2((double)acc[1], (double)acc[2]));
    }
  } else {
#pragma unroll
    for (int a = 0; a < LC; ++a) out[a] = (FT)acc[a];
  }
}

// Cell layers gathered per step of the z sweep (one barrier per step) and
// the node-plane ring that takes: the S + LPS - 1 planes the step reads and
// the LPS planes being filled for the next step.  Two layers per step for
// FP32 rings (at ~1 particle per cell a layer gives each thread only ~2
// particles between barriers); one for FP64 rings, whose gather is
// arithmetic-bound.
template <int S, class CT, int LC>
constexpr int m2p_layers() {
  return sizeof(CT) == 4 ? 2 : 1;
}

template <int S, class CT, int LC>
constexpr size_t m2p_ring_bytes() {
  return (size_t)(kTileX + S - 1) * (kTileY + S - 1) * (S + 2 * m2p_layers<S, CT, LC>() - 1) *
         LC * sizeof(CT);
}

// OPEN: a subdomain cut along some axis (P.open), compiled apart so that
// the periodic gather keeps its column and plane loads unconditional.
template <int S, class CT, bool EXACT, class FT, int LC, bool ADJ = false, bool OPEN = false>
__global__ void __launch_bounds__(256) k_m2p3d_tile(M2PParams P) {
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  constexpr int WX = kTileX + S - 1;
  constexpr int WY = kTileY + S - 1;
  constexpr int NCOL = WX * WY;
  constexpr int LPS = m2p_layers<S, CT, LC>();  // cell layers per step
  constexpr int R = S + 2 * LPS - 1;           // ring slots
  constexpr int CS = R * LC;                   // CT values per node column
  constexpr int PER = (NCOL + 255) / 256;      // columns per thread when loading a plane
  static_assert(16 * LPS <= 32, "row tables are loaded by the first warp");

  if ((int)blockIdx.x >= *P.nitems) return;
  const int4 it = P.items[blockIdx.x];
  const int tiles_x = (P.N[0] + kTileX - 1) / kTileX;
  const int X0 = (it.x % tiles_x) * kTileX;
  const int Y0 = (it.x / tiles_x) * kTileY;
  const int Z0 = it.y, Z1 = it.z;
  const int XW = min(kTileX, P.N[0] - X0);  // cells of the tile inside the mesh
  const int YW = min(kTileY, P.N[1] - Y0);

  extern __shared__ __align__(16) unsigned char smem[];
  CT* ring = reinterpret_cast<CT*>(smem);  // [NCOL][R][LC]
  // row tables of the step's LPS layers and of the next step's (double buffered)
  __shared__ int rbeg[2 * LPS][kTileY], rpre[2 * LPS][kTileY + 1];

  const int tid = threadIdx.x;
  const FT* F = static_cast<const FT*>(P.field);

  // global offset of node column q of plane z (component c0)
  auto col_off = [&](int q, int64_t oz) {
    const int r = q / WX, qx = q - r * WX;
    int xw = X0 - (HL - 1) + qx, yw = Y0 - (HL - 1) + r;
    if (!OPEN || !P.open[0]) xw = wrap_index(xw, P.N[0]);
    if (!OPEN || !P.open[1]) yw = wrap_index(yw, P.N[1]);
    return (int64_t)(xw + 1 - P.fd.lb[0]) * P.fd.s[0] +
           (int64_t)(yw + 1 - P.fd.lb[1]) * P.fd.s[1] + oz + P.c0;
  };
  auto plane_oz = [&](int z) {
    return (int64_t)((OPEN && P.open[2] ? z : wrap_index(z, P.N[2])) + 1 - P.fd.lb[2]) *
           P.fd.s[2];
  };
  // along a cut axis only the nodes the cells 0 .. N-1 reach are read (the
  // columns of a tile past the last cell, and a step past the last layer,
  // would reach beyond the required box)
  auto in_reach = [&](int a, int n) { return n >= -(HL - 1) && n <= P.N[a] - 1 + HL; };
  auto plane_ok = [&](int z) { return !OPEN || !P.open[2] || in_reach(2, z); };
  auto col_ok = [&](int q) {
    if (!OPEN) return true;
    const int r = q / WX, qx = q - r * WX;
    return (!P.open[0] || in_reach(0, X0 - (HL - 1) + qx)) &&
           (!P.open[1] || in_reach(1, Y0 - (HL - 1) + r));
  };
  // row ranges of cell layers cz .. cz+LPS-1: thread 16 l + r loads row r of
  // layer cz + l
  auto row_load = [&](int cz, int& b, int& n) {
    b = 0;
    n = 0;
    const int l = tid >> 4, r = tid & 15;
    if (tid < 16 * LPS && r < YW && cz + l < Z1) {
      const int64_t c0 =
          (int64_t)X0 + (int64_t)P.N[0] * (Y0 + r + (int64_t)P.N[1] * (cz + l));
      b = P.start[c0];
      n = P.start[c0 + XW] - b;
    }
  };
  // row tables base .. base+LPS-1 from the loaded ranges (inclusive scan per
  // group of 16 lanes)
  auto row_store = [&](int base, int b, int n) {
    if (tid < 32) {
      const int l = tid >> 4, r = tid & 15;
      int inc = n;
#pragma unroll
      for (int o = 1; o < kTileY; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o, 16);
        if (r >= o) inc += t;
      }
      if (l < LPS) {
        rbeg[base + l][r] = b;
        rpre[base + l][r + 1] = inc;
        if (r == 0) rpre[base + l][0] = 0;
      }
    }
  };

  // prologue: planes Z0-(HL-1) .. Z0+LPS-1+HL (the planes of the first
  // step's layers) and their rows
  for (int z = Z0 - (HL - 1); z <= Z0 + LPS - 1 + HL; ++z) {
    if (!plane_ok(z)) continue;
    const int slot = wrap_index(z, R);
    const int64_t oz = plane_oz(z);
    for (int q = tid; q < NCOL; q += 256) {
      CT* d = ring + (size_t)q * CS + slot * LC;
      if (!col_ok(q)) {
#pragma unroll
        for (int a = 0; a < LC; ++a) d[a] = CT(0);
        continue;
      }
      const int64_t o = col_off(q, oz);
#pragma unroll
      for (int a = 0; a < LC; ++a) d[a] = (CT)__ldg(F + o + a);
    }
  }
  {
    int b, n;
    row_load(Z0, b, n);
    row_store(0, b, n);
  }
  __syncthreads();

  FT* up = static_cast<FT*>(P.up);
  const V* rec = static_cast<const V*>(P.rec);

  for (int cz = Z0, step = 0; cz < Z1; cz += LPS, ++step) {
    const int cb = (step & 1) * LPS;  // row tables of this step's layers
    // prefetch the next step's new planes and rows into registers
    const bool more = cz + LPS < Z1;
    CT pre[LPS][PER][LC];
    if (more) {
#pragma unroll
      for (int l = 0; l < LPS; ++l) {
        const int64_t oz = plane_oz(cz + LPS + HL + l);
        const bool ok = plane_ok(cz + LPS + HL + l);
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          const int q = tid + 256 * k;
          if constexpr (OPEN) {
#pragma unroll
            for (int a = 0; a < LC; ++a) pre[l][k][a] = CT(0);
          }
          if (q < NCOL && ok && col_ok(q)) {
            const int64_t o = col_off(q, oz);
#pragma unroll
            for (int a = 0; a < LC; ++a) pre[l][k][a] = (CT)__ldg(F + o + a);
          }
        }
      }
    }
    int nb, nn;
    row_load(cz + LPS, nb, nn);

    // the step's particles: layer 0's rows, then layer 1's
    const int n0 = rpre[cb][kTileY];
    const int ntot = n0 + (LPS > 1 ? rpre[cb + LPS - 1][kTileY] : 0);
    // software-pipelined particle loop: the next record is loaded while the
    // current particle is gathered
    auto locate = [&](int i, int& r, int& l) {
      l = (LPS > 1 && i >= n0) ? 1 : 0;
      const int j = i - (l ? n0 : 0);
      const int tb = cb + l;
      // the last row starting at or before j (row starts are non-decreasing):
      // binary lifting over rows 0 .. kTileY-1
      static_assert(kTileY == 16, "four lifting steps");
      r = 0;
#pragma unroll
      for (int step = kTileY / 2; step > 0; step >>= 1)
        if (rpre[tb][r + step] <= j) r += step;
      return (int64_t)rbeg[tb][r] + (j - rpre[tb][r]);
    };
    int rcur = 0, idcur = 0, lcur = 0;
    int64_t scur = 0;
    V rvcur;
    if (tid < ntot) {
      scur = locate(tid, rcur, lcur);
      rvcur = load_vec(rec, scur, P.nvalid);
      idcur = P.idx[scur];
    }
    for (int i = tid; i < ntot; i += 256) {
      int rnext = 0, idnext = 0, lnext = 0;
      int64_t snext = 0;
      V rvnext;
      if (i + 256 < ntot) {
        snext = locate(i + 256, rnext, lnext);
        rvnext = load_vec(rec, snext, P.nvalid);
        idnext = P.idx[snext];
      }
      {
        // ring slots of the S planes of this particle's layer
        int slot_k[S];
        {
          const int s0 = wrap_index(cz + lcur - (HL - 1), R);
#pragma unroll
          for (int k = 0; k < S; ++k) slot_k[k] = s0 + k < R ? s0 + k : s0 + k - R;
        }
        int cell;
        if constexpr (sizeof(CT) == 4) cell = __float_as_int(rvcur.w); else cell = (int)rvcur.w;
        const int qx0 = cell % P.N[0] - X0;  // local column of the first stencil node
        const int qy0 = rcur;                // row of the cell inside the tile
        CT wx[S], wy[S], wz[S];
        m2p_weights<S, CT, EXACT>(rvcur.x, wx);
        m2p_weights<S, CT, EXACT>(rvcur.y, wy);
        m2p_weights<S, CT, EXACT>(rvcur.z, wz);
        FT* out = up + (int64_t)idcur * P.ldup + P.c0;
        if constexpr (ADJ) {
          // strengths of the particle (needed once its gradient sums are done)
          CT ua[LC];
#pragma unroll
          for (int a = 0; a < LC; ++a) ua[a] = (CT)__ldg(P.upin + (int64_t)idcur * P.ldupin + a);
          CT dx[S], dy[S], dz[S];
          adj_dweights<S, CT>(rvcur.x, (CT)P.dxi[0], dx);
          adj_dweights<S, CT>(rvcur.y, (CT)P.dxi[1], dy);
          adj_dweights<S, CT>(rvcur.z, (CT)P.dxi[2], dz);
          CT acc[LC], ga[LC][3];
#pragma unroll
          for (int a = 0; a < LC; ++a) acc[a] = ga[a][0] = ga[a][1] = ga[a][2] = CT(0);
#pragma unroll
          for (int ii = 0; ii < S; ++ii)
#pragma unroll
            for (int jj = 0; jj < S; ++jj) {
              const CT wij = wx[ii] * wy[jj];
              const CT dxij = dx[ii] * wy[jj];
              const CT dyij = wx[ii] * dy[jj];
              const CT* col = ring + (size_t)((qy0 + jj) * WX + qx0 + ii) * CS;
#pragma unroll
              for (int a = 0; a < LC; ++a) {
                CT part = CT(0), dpart = CT(0);
#pragma unroll
                for (int k = 0; k < S; ++k) {
                  const CT v = col[slot_k[k] * LC + a];
                  part = fma(wz[k], v, part);
                  dpart = fma(dz[k], v, dpart);
                }
                acc[a] = fma(wij, part, acc[a]);
                ga[a][0] = fma(dxij, part, ga[a][0]);
                ga[a][1] = fma(dyij, part, ga[a][1]);
                ga[a][2] = fma(wij, dpart, ga[a][2]);
              }
            }
          CT g[3] = {CT(0), CT(0), CT(0)};
#pragma unroll
          for (int a = 0; a < LC; ++a) {
#pragma unroll
            for (int d = 0; d < 3; ++d) g[d] = fma(ua[a], ga[a][d], g[d]);
          }
          store_row<FT, CT, LC>(out, acc);
          store_row<double, CT, 3>(P.dx + (int64_t)idcur * P.lddx, g);
        } else if constexpr (EXACT) {
          CT res[LC];
#pragma unroll
          for (int a = 0; a < LC; ++a) {
            CT acc = CT(0);
#pragma unroll 1
            for (int ii = 0; ii < S; ++ii)
#pragma unroll
              for (int jj = 0; jj < S; ++jj) {
                const CT wij = rmul(wx[ii], wy[jj]);
                const CT* col = ring + (size_t)((qy0 + jj) * WX + qx0 + ii) * CS + a;
#pragma unroll
                for (int kk = 0; kk < S; ++kk)
                  acc = radd(acc, rmul(rmul(wij, wz[kk]), col[slot_k[kk] * LC]));
              }
            res[a] = acc;
          }
          store_row<FT, CT, LC>(out, res);
        } else {
          CT acc[LC];
#pragma unroll
          for (int a = 0; a < LC; ++a) acc[a] = CT(0);
#pragma unroll
          for (int ii = 0; ii < S; ++ii)
#pragma unroll
            for (int jj = 0; jj < S; ++jj) {
              const CT wij = wx[ii] * wy[jj];
              const CT* col = ring + (size_t)((qy0 + jj) * WX + qx0 + ii) * CS;
#pragma unroll
              for (int a = 0; a < LC; ++a) {
                CT part = CT(0);
#pragma unroll
                for (int k = 0; k < S; ++k) part = fma(wz[k], col[slot_k[k] * LC + a], part);
                acc[a] = fma(wij, part, acc[a]);
              }
            }
          store_row<FT, CT, LC>(out, acc);
        }
      }
      rcur = rnext;
      scur = snext;
      rvcur = rvnext;
      idcur = idnext;
      lcur = lnext;
    }
    // publish the prefetched planes (their slots are not read by this step)
    // and rows
    if (more) {
#pragma unroll
      for (int l = 0; l < LPS; ++l) {
        const int slot = wrap_index(cz + LPS + HL + l, R);
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          const int q = tid + 256 * k;
          if (q < NCOL) {
            CT* d = ring + (size_t)q * CS + slot * LC;
#pragma unroll
            for (int a = 0; a < LC; ++a) d[a] = pre[l][k][a];
          }
        }
      }
    }
    row_store(cb ^ LPS, nb, nn);
    __syncthreads();
  }
}

template <int S, class CT, bool EXACT, class FT>
cudaError_t launch_tile_lc(const M2PParams& P, int lc, cudaStream_t st) {
  auto go = [&](auto kern, auto kern_oz, size_t smem) {
    auto k = P.open[0] || P.open[1] || P.open[2] ? kern_oz : kern;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e) return e;
    k<<<P.item_cap, 256, smem, st>>>(P);
    return cudaGetLastError();
  };
  switch (lc) {
    case 1: return go(k_m2p3d_tile<S, CT, EXACT, FT, 1>, k_m2p3d_tile<S, CT, EXACT, FT, 1, false, true>,
                      m2p_ring_bytes<S, CT, 1>());
    case 2: return go(k_m2p3d_tile<S, CT, EXACT, FT, 2>, k_m2p3d_tile<S, CT, EXACT, FT, 2, false, true>,
                      m2p_ring_bytes<S, CT, 2>());
    case 3: return go(k_m2p3d_tile<S, CT, EXACT, FT, 3>, k_m2p3d_tile<S, CT, EXACT, FT, 3, false, true>,
                      m2p_ring_bytes<S, CT, 3>());
    default: return go(k_m2p3d_tile<S, CT, EXACT, FT, 4>, k_m2p3d_tile<S, CT, EXACT, FT, 4, false, true>,
                       m2p_ring_bytes<S, CT, 4>());
  }
}

int blocks_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_m2p(const M2PParams& P0, int dim, int kernel, M2PPrec prec, cudaStream_t st) {
  if (P0.nvalid <= 0) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  if (dim == 3) {
    // tiled gather: one launch per chunk of up to 4 components
    TimingScope timed(kTimeM2P, st);
    for (int c0 = 0; c0 < P0.lda; c0 += 4) {
      M2PParams P = P0;
      P.c0 = c0;
      const int lc = P0.lda - c0 < 4 ? P0.lda - c0 : 4;
      if (kernel == kKernelMp4) {
        switch (prec) {
          case M2P_FP64: e = launch_tile_lc<4, double, true, double>(P, lc, st); break;
          case M2P_MIXED: e = launch_tile_lc<4, float, false, double>(P, lc, st); break;
          case M2P_FP32: e = launch_tile_lc<4, float, false, float>(P, lc, st); break;
        }
      } else {
        switch (prec) {
          case M2P_FP64: e = launch_tile_lc<2, double, true, double>(P, lc, st); break;
          case M2P_MIXED: e = launch_tile_lc<2, float, false, double>(P, lc, st); break;
          case M2P_FP32: e = launch_tile_lc<2, float, false, float>(P, lc, st); break;
        }
      }
      count_launch();
      if (e) return e;
    }
    return e;
  }
  const M2PParams& P = P0;
  const int nb = blocks_for(P.nvalid);
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
  count_launch();
  return cudaGetLastError();
}

template <int S, class CT, int LC>
cudaError_t launch_adjoint_tile(const M2PParams& P, cudaStream_t st) {
  auto kern = P.open[0] || P.open[1] || P.open[2]
                  ? k_m2p3d_tile<S, CT, false, double, LC, true, true>
                  : k_m2p3d_tile<S, CT, false, double, LC, true>;
  const size_t smem = m2p_ring_bytes<S, CT, LC>();
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  kern<<<P.item_cap, 256, smem, st>>>(P);
  count_launch();
  return cudaGetLastError();
}

template <int S, class CT>
cudaError_t adjoint_tile_lc(const M2PParams& P, cudaStream_t st) {
  switch (P.lda) {
    case 1: return launch_adjoint_tile<S, CT, 1>(P, st);
    case 2: return launch_adjoint_tile<S, CT, 2>(P, st);
    case 3: return launch_adjoint_tile<S, CT, 3>(P, st);
    default: return launch_adjoint_tile<S, CT, 4>(P, st);
  }
}

cudaError_t launch_adjoint(const M2PParams& P, int kernel, M2PPrec prec, cudaStream_t st) {
  if (P.nvalid <= 0) return cudaSuccess;
  if (P.items && P.lda <= 4) {
    // tiled gather over the work items of the cell order
    if (kernel == kKernelMp4)
      return prec == M2P_FP64 ? adjoint_tile_lc<4, double>(P, st) : adjoint_tile_lc<4, float>(P, st);
    return prec == M2P_FP64 ? adjoint_tile_lc<2, double>(P, st) : adjoint_tile_lc<2, float>(P, st);
  }
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
