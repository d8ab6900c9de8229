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

#include <type_traits>

#include "ppmg_p2m.cuh"

namespace ppmg {

namespace {


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
// The periodic images n+1+t*N (1-based) of unique node n along axis a that
// lie in the written box: t = lo .. hi (0 .. 0 when the node has none).
__device__ __forceinline__ void axis_images(const P2MParams& P, int a, int n, int& lo,
                                            int& hi) {
  const int N = P.N[a];
  if (P.open[a]) {
    // no periodic images along a cut axis: the node itself
    lo = hi = 0;
  } else if (P.fd.box_lo[a] > 1 - N && P.fd.box_hi[a] < 2 * N + 1) {
    // ghost layers narrower than the mesh: t in {-1, 0, 1}
    lo = n + 1 - N >= P.fd.box_lo[a] ? -1 : 0;
    hi = n + 1 + N <= P.fd.box_hi[a] ? 1 : 0;
  } else {
    int tlo = (P.fd.box_lo[a] - n - 1 + 64 * N) / N - 64;  // ceil for negatives
    if (n + 1 + tlo * N < P.fd.box_lo[a]) ++tlo;
    lo = tlo;
    hi = (P.fd.box_hi[a] - n - 1 + 64 * N) / N - 64;  // floor
  }
}

template <int DIM, class OT, int LC>
__device__ __forceinline__ void emit_node(const P2MParams& P, int x, int y, int z,
                                          const double v[LC]) {
  OT* F = static_cast<OT*>(P.field);
  const int n[3] = {x, y, z};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < DIM; ++a) axis_images(P, a, n[a], lo[a], hi[a]);
  if (DIM == 2) {
    lo[2] = hi[2] = 0;
  }
  if ((lo[0] | hi[0] | lo[1] | hi[1] | lo[2] | hi[2]) == 0) {
    // the common case: the node has no image inside the box
    const int64_t o = (int64_t)(n[0] + 1 - P.fd.lb[0]) * P.fd.s[0] +
                      (int64_t)(n[1] + 1 - P.fd.lb[1]) * P.fd.s[1] +
                      (DIM == 3 ? (int64_t)(n[2] + 1 - P.fd.lb[2]) * P.fd.s[2] : 0) + P.c0;
#pragma unroll
    for (int a = 0; a < LC; ++a) F[o + a] = (OT)v[a];
    return;
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
// A CTA of 16 x 16 threads owns 32 x 16 node columns (two adjacent columns
// per thread) over a z-range [Z0, Z1) given by its work item, and sweeps the
// cell layers that reach it.  The particles of the (32+S-1) x (16+S-1) cells
// of a layer whose stencils reach the tile are processed in units of at most
// `cap` particles (one unit per layer unless the layer is dense).  Units are
// software-pipelined: while unit u is accumulated, the records and strengths
// of unit u+1 stream into a raw shared-memory buffer with cp.async; unit u+1
// then gets its 1D weights computed once per particle into structure-of-
// arrays slots (wx, wy, wz, u: one 16-byte vector each).  A thread visits the
// S+1 cells of each of its S rows; the x-weight index of each of its two
// columns follows from the staged cell column, so every visit costs 3 vector
// loads + 1 scalar load for two columns.
// Dense layers are cut into units that give every cell with particles left
// an equal share (cap / active cells, the remainder one more for the first
// cells), so every thread has work in every unit.
// S: stencil width (4 = M'4, 2 = bsp2).  CT: arithmetic type.  COMP:
// compensated FP32 accumulation (per-unit partial sums folded into a
// (hi, lo) pair with an error-free TwoSum).  OT: field type.  LC: components
// handled by this launch (<= 4).  WST: 1D weights come from comp_weights.
// --------------------------------------------------------------------------
constexpr int kTX = 16, kTY = 16;
static_assert(kTileX == 2 * kTX && kTileY == kTY, "tile shape");

template <class CT>
__device__ __forceinline__ CT vget(const typename Vec4<CT>::type& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(smem_dst)),
               "l"(gmem_src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(smem_dst)),
               "l"(gmem_src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// Every cp.async of this thread complete, the ones not yet committed to a
// group included (cp.async.wait_all commits them first).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Exclusive scan over n <= 3*256 cell values v(q) (thread t owns cells 3t ..
// 3t+2) by a CTA of 8 warps; writes out[0..n] (out[n] = total) and returns
// the total through the smem scalar red[0] (visible to all on return).  A
// thread may read its own cells' out[] at once; the others', and the next
// scan, only after a barrier of the caller.
template <class F>
__device__ __forceinline__ void scan_cells(int n, F val, int* out, int* wsum, int* red) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int q0 = 3 * tid;
  const int v0 = q0 < n ? val(q0) : 0;
  const int v1 = q0 + 1 < n ? val(q0 + 1) : 0;
  const int v2 = q0 + 2 < n ? val(q0 + 2) : 0;
  const int s = v0 + v1 + v2;
  int inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    // the 8 warp totals: exclusive offsets by a shuffle scan in warp 0
    const int w = lane < 8 ? wsum[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < 8) wsum[lane] = wi - w;
    if (lane == 7) red[0] = wi;
  }
  __syncthreads();
  const int ex = inc - s + wsum[wid];
  if (q0 < n) out[q0] = ex;
  if (q0 + 1 < n) out[q0 + 1] = ex + v0;
  if (q0 + 2 < n) out[q0 + 2] = ex + v0 + v1;
  if (tid == 0) out[n] = red[0];
}

// Shared memory of k_p2m3d for `cap` staging slots.
// 16-byte units of one staged particle's record part: its packed record, or
// (stored weights) 3 x S weights of the field's type padded to 16 bytes
template <int S, class CT, class OT, bool WST>
constexpr int p2m_rec_units() {
  return WST ? (3 * S * (int)sizeof(OT) + 15) / 16 : (int)sizeof(typename Vec4<CT>::type) / 16;
}

template <int S, class CT, class OT, bool WST>
constexpr size_t p2m3d_smem(int cap) {
  using V = typename Vec4<CT>::type;
  constexpr int NSC = (kTileX + S - 1) * (kTileY + S - 1);
  constexpr int IU = p2m_rec_units<S, CT, OT, WST>() + (int)sizeof(V) / 16;
  return (size_t)cap * (3 * sizeof(V) + (S + 2) * sizeof(CT) + 16 * IU + 2) +
         sizeof(int) * (size_t)(8 * NSC + 2);
}

// The FP64 form's gather (the compensated FP32 form runs in k_p2m3g).
template <int S, class CT, bool COMP, class OT, int LC, bool WST>
__global__ void __launch_bounds__(kTX * kTY, 2) k_p2m3d(P2MParams P) {
  static_assert(!COMP, "plain sums only");
  using V = typename Vec4<CT>::type;
  constexpr int HL = S / 2;
  constexpr int HH = S / 2 - 1;
  constexpr int WX = kTileX + S - 1;
  constexpr int WY = kTileY + S - 1;
  constexpr int NSC = WX * WY;
  constexpr int NT = kTX * kTY;
  constexpr int PERC = (NSC + NT - 1) / NT;  // staged cells per thread (count loads)
  constexpr int RU = p2m_rec_units<S, CT, OT, WST>();  // 16-byte units: record part
  constexpr int UU = (int)sizeof(V) / 16;                          // strengths part
  constexpr int IU = RU + UU;
  static_assert(NSC <= 3 * NT, "staged cells exceed the scan width");

  if ((int)blockIdx.x >= *P.nitems) return;
  const int4 it = P.items[blockIdx.x];
  const int tiles_x = (P.span.ext[0] + kTileX - 1) / kTileX;
  const int X0 = P.span.org[0] + (it.x % tiles_x) * kTileX;
  const int Y0 = P.span.org[1] + (it.x / tiles_x) * kTileY;
  const int XE = P.span.org[0] + P.span.ext[0], YE = P.span.org[1] + P.span.ext[1];
  const int Z0 = it.y, Z1 = it.z;
  const int cap = P.cap;

  constexpr int PXN = S + 2;  // x-weights per slot, zero-padded: [0, w0 .. w(S-1), 0]
  extern __shared__ __align__(16) unsigned char smem[];
  V* sWY = reinterpret_cast<V*>(smem);
  V* sWZ = sWY + cap;
  V* sU = sWZ + cap;
  CT* sPX = reinterpret_cast<CT*>(sU + cap);           // [cap][PXN]
  uint4* raw = reinterpret_cast<uint4*>(sPX + (size_t)cap * PXN);  // [cap][IU] next unit
  int* cnt = reinterpret_cast<int*>(raw + (size_t)cap * IU);  // layer: particles per cell
  int* done = cnt + NSC;                                // layer: particles already in units
  int* cbase = done + NSC;                              // layer: first sorted particle per cell
  int* ubase = cbase + NSC;                             // unit being issued: its first particle per cell
  int* offU = ubase + NSC;                              // [2][NSC + 1] unit offsets per cell
  int* nxb = offU + 2 * (NSC + 1);                      // next layer: cell ranges in flight
  int* nxe = nxb + NSC;
  unsigned char* sQ = reinterpret_cast<unsigned char*>(nxe + NSC);  // [2][cap]
  __shared__ int wsum[16];
  __shared__ int red[2];

  const int tid = threadIdx.x;
  const int tx = tid % kTX, ty = tid / kTX;
  const int x0 = X0 + 2 * tx, y = Y0 + ty;
  const bool act0 = x0 < XE && y < YE;
  const bool act1 = x0 + 1 < XE && y < YE;
  const uint4* grec = static_cast<const uint4*>(P.rec);
  const uint4* gus = static_cast<const uint4*>(P.us);

  CT acc[2][S][LC];  // the node window of the thread's two columns
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int k = 0; k < S; ++k)
#pragma unroll
      for (int a = 0; a < LC; ++a) acc[e][k][a] = CT(0);

  // cell ranges of the staged cells of layer cz: copied asynchronously into
  // nxb / nxe (each thread its own cells), published a unit or more later
  auto load_counts = [&](int cz) {
    // along a cut axis the cells outside 0 .. N-1 hold no particles of
    // this subdomain
    const bool empty = P.open[2] && (cz < 0 || cz >= P.N[2]);
    const int czw = empty ? 0 : wrap_index(cz, P.N[2]);
#pragma unroll
    for (int k = 0; k < PERC; ++k) {
      const int q = tid + NT * k;
      if (q >= NSC) continue;
      const int r = q / WX, qx = q - r * WX;
      const int ux = X0 - HL + qx, uy = Y0 - HL + r;
      const bool out = (P.open[0] && (ux < 0 || ux >= P.N[0])) ||
                       (P.open[1] && (uy < 0 || uy >= P.N[1]));
      if (!empty && !out) {
        const int cx = wrap_index(ux, P.N[0]);
        const int cy = wrap_index(uy, P.N[1]);
        const int64_t c = (int64_t)cx + (int64_t)P.N[0] * (cy + (int64_t)P.N[1] * czw);
        cp_async4(nxb + q, P.start + c);
        cp_async4(nxe + q, P.start + c + 1);
      } else {
        nxb[q] = nxe[q] = 0;
      }
    }
  };
  // (the values are read and stored before the next load_counts of the
  // same cells is issued: the copy cannot overtake the read)
  auto publish = [&]() {
#pragma unroll
    for (int k = 0; k < PERC; ++k) {
      const int q = tid + NT * k;
      if (q < NSC) {
        const int b = nxb[q], e = nxe[q];
        cbase[q] = b;
        cnt[q] = e - b;
        done[q] = 0;
      }
    }
  };
  // Plans the next unit of the published layer into offU[ob]: returns its
  // particle count; `left` (particles of the layer not yet in a unit) is
  // updated.  Thread t plans cells 3t .. 3t+2.
  int left = 0;
  auto plan = [&](int ob, bool first) -> int {
    int* off = offU + ob * (NSC + 1);
    if (first) {
      scan_cells(NSC, [&](int q) { return cnt[q]; }, off, wsum, red);
      left = red[0];
      if (left <= cap) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const int q = 3 * tid + i;
          if (q < NSC) {
            ubase[q] = cbase[q];
            done[q] = cnt[q];
          }
        }
        const int n = left;
        left = 0;
        __syncthreads();
        return n;
      }
    }
    // cells with particles left share the unit equally
    scan_cells(NSC, [&](int q) { return cnt[q] > done[q] ? 1 : 0; }, off, wsum, red);
    const int A = max(red[0], 1);
    const int k = cap / A, rem = cap - A * k;
    auto take_of = [&](int q) {
      const int l = q < NSC ? cnt[q] - done[q] : 0;
      return l > 0 ? min(l, k + (off[q] < rem ? 1 : 0)) : 0;
    };
    const int t0 = take_of(3 * tid), t1 = take_of(3 * tid + 1), t2 = take_of(3 * tid + 2);
    __syncthreads();  // the active ranks in off are read
    scan_cells(NSC, [&](int q) { const int i = q - 3 * tid; return i == 0 ? t0 : (i == 1 ? t1 : t2); },
               off, wsum, red);
    const int n = red[0];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int q = 3 * tid + i;
      if (q < NSC) {
        ubase[q] = cbase[q] + done[q];
        done[q] += i == 0 ? t0 : (i == 1 ? t1 : t2);
      }
    }
    left -= n;
    __syncthreads();
    return n;
  };
  // cp.async of the planned unit's records and strengths into raw; the
  // staged column of every slot goes to sQ[ob].  Thread t issues its cells.
  auto issue = [&](int ob) {
    const int* off = offU + ob * (NSC + 1);
    unsigned char* q8 = sQ + ob * cap;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int q = 3 * tid + i;
      if (q < NSC) {
        const int o0 = off[q], o1 = off[q + 1];
        const int64_t g0 = ubase[q];
        for (int o = o0; o < o1; ++o) {
          const int64_t s = g0 + (o - o0);
          uint4* d = raw + (size_t)o * IU;
#pragma unroll
          for (int t = 0; t < RU; ++t) {
            if constexpr (WST)
              cp_async16(d + t, grec + s * RU + t);
            else
              cp_async16(d + t, grec + t * P.ps + s);
          }
#pragma unroll
          for (int t = 0; t < UU; ++t) cp_async16(d + RU + t, gus + t * P.ps + s);
          q8[o] = (unsigned char)(q % WX);
        }
      }
    }
    cp_async_commit();
  };

  // prologue: layer Z0 - HL published, its first unit in flight, the next
  // layer's cell ranges in registers
  int cz = Z0 - HL;
  const int zlast = Z1 - 1 + HH;
  load_counts(cz);
  cp_async_wait_all();
  publish();
  if (cz < zlast) load_counts(cz + 1);
  __syncthreads();
  int n_cur = plan(0, true);
  bool last_cur = left == 0;  // the unit in flight completes its layer
  issue(0);

  for (int u = 0;; ++u) {
    const int ub = u & 1;
    cp_async_wait_all();
    __syncthreads();
    // 1. weights of unit u: raw -> structure-of-arrays slots
    for (int i = tid; i < n_cur; i += NT) {
      const uint4* r = raw + (size_t)i * IU;
      CT w[3][S];
      if constexpr (WST) {
        const OT* wsrc = reinterpret_cast<const OT*>(r);
#pragma unroll
        for (int k = 0; k < S; ++k) {
          w[0][k] = (CT)wsrc[k];
          w[1][k] = (CT)wsrc[S + k];
          w[2][k] = (CT)wsrc[2 * S + k];
        }
      } else {
        const V rv = *reinterpret_cast<const V*>(r);
        weights<S, CT>(rv.x, w[0]);
        weights<S, CT>(rv.y, w[1]);
        weights<S, CT>(rv.z, w[2]);
      }
      V b, c;
      b.x = w[1][0]; b.y = w[1][1]; b.z = S > 2 ? w[1][S > 2 ? 2 : 0] : CT(0); b.w = S > 3 ? w[1][S > 3 ? 3 : 0] : CT(0);
      c.x = w[2][0]; c.y = w[2][1]; c.z = S > 2 ? w[2][S > 2 ? 2 : 0] : CT(0); c.w = S > 3 ? w[2][S > 3 ? 3 : 0] : CT(0);
      CT* px = sPX + (size_t)i * PXN;
      px[0] = CT(0);
#pragma unroll
      for (int k = 0; k < S; ++k) px[1 + k] = w[0][k];
      px[S + 1] = CT(0);
      sWY[i] = b;
      sWZ[i] = c;
      sU[i] = *reinterpret_cast<const V*>(r + RU);
    }
    __syncthreads();
    // 2. plan and issue unit u+1 (the next layer's first unit when unit u
    //    completes its layer); its loads fly while unit u is accumulated
    const int cz_u = cz;
    const bool last_u = last_cur;
    const int n_u = n_cur;
    bool more = true;
    if (last_u) {
      if (cz < zlast) {
        ++cz;
        publish();
        if (cz < zlast) load_counts(cz + 1);
        __syncthreads();
        n_cur = plan(ub ^ 1, true);
      } else {
        more = false;
      }
    } else {
      n_cur = plan(ub ^ 1, false);
    }
    if (more) {
      last_cur = left == 0;
      issue(ub ^ 1);
    }
    // 3. accumulate unit u: per row, the particles of cells 2tx..2tx+S (one range)
    if (act0 && n_u > 0) {
      const int* off = offU + ub * (NSC + 1);
      const unsigned char* q8 = sQ + ub * cap;
#pragma unroll
      for (int dy = 0; dy < S; ++dy) {
        const int row = (ty + dy) * WX + 2 * tx;
        const int p0 = off[row], p1 = off[row + S + 1];
        for (int p = p0; p < p1; ++p) {
          const int d = (int)q8[p] - 2 * tx;  // cell offset 0..S inside the window
          const CT* px = sPX + (size_t)p * PXN;
          const V wz = sWZ[p];
          const V uv = sU[p];
          const CT wy = vget<CT>(sWY[p], S - 1 - dy);
          // x-weights of the two columns: nodes S-1-d and S-d of the stencil
          const CT w0 = px[S - d], w1 = px[S + 1 - d];
          const CT c0 = w0 * wy, c1 = w1 * wy;
          const CT wzv[4] = {wz.x, wz.y, wz.z, wz.w};
          const CT uu[4] = {uv.x, uv.y, uv.z, uv.w};
#pragma unroll
          for (int a = 0; a < LC; ++a) {
            const CT cu0 = c0 * uu[a], cu1 = c1 * uu[a];
#pragma unroll
            for (int k = 0; k < S; ++k) {
              acc[0][k][a] += cu0 * wzv[k];
              acc[1][k][a] += cu1 * wzv[k];
            }
          }
        }
      }
    }
    // 4. layer complete: node zc = cz_u - (HL-1) of both columns is final: emit, shift
    if (last_u) {
      const int zc = cz_u - (HL - 1);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if ((e == 0 ? act0 : act1) && zc >= Z0 && zc < Z1) {
          double v[LC];
#pragma unroll
          for (int a = 0; a < LC; ++a) v[a] = (double)acc[e][0][a];
          emit_node<3, OT, LC>(P, x0 + e, y, zc, v);
        }
#pragma unroll
        for (int k = 0; k < S - 1; ++k)
#pragma unroll
          for (int a = 0; a < LC; ++a) acc[e][k][a] = acc[e][k + 1][a];
#pragma unroll
        for (int a = 0; a < LC; ++a) acc[e][S - 1][a] = CT(0);
      }
    }
    if (!more) break;
  }
}

// --------------------------------------------------------------------------
// 3D row gather (FP32 arithmetic: the mixed form and the single-precision
// API).
// A CTA of kGW warps owns the kGW x-nodes X0 .. X0+kGW-1 and the 33-S node
// rows Y0 .. Y0+32-S over a z-range [Z0, Z1) of its work item.  Warp w owns
// x-node X0 + w; lane L owns cell row Y0 - HL + L (L = 0 .. 31).  For each
// cell layer the particles of the (kGW+S-1) x 32 cells whose stencils reach
// the tile are staged in shared memory (1D weights once per staged
// particle); thread (w, L) then visits the particles of the S cells
// X0-HL+w .. X0-HL+w+S-1 of its row -- exactly the particles whose
// x-stencils reach node X0 + w -- and adds each one's contribution to the
// S node rows (j) and S node planes (k) of its yz-stencil into registers
// G[j][k][a]: one visit per (particle, x-node), S*S*LC FMAs each.
// The node of row Y0 + L is the sum of G[S-1-d] over lanes L + d
// (d = 0 .. S-1), taken by warp shuffles in a fixed order; lanes L >= 33-S
// only supply rows.  G's planes form a z-window like the node window of
// k_p2m3d: when the sweep leaves layer cz, plane cz-HL+1 is complete and is
// written (with its periodic images); the window then shifts.
// Compensation (COMP): G holds plain FP32 partials.  Once a lane of a warp
// has added more than kFoldTerms particles since the warp's last fold, the
// warp sums all of G's planes over its rows and folds them into the
// per-node (hi, lo) window with an error-free TwoSum, then clears G; a node
// is written as hi + lo + the partial of its plane, in FP64.  Every node is
// produced by one thread in a fixed order: the results are deterministic.
// S: stencil width (4 = M'4, 2 = bsp2).  OT: field type.  LC: components of
// this launch (<= 4).  WST: 1D weights come from comp_weights.
// --------------------------------------------------------------------------
constexpr int kGW = 8;          // warps per CTA = x-nodes per tile
constexpr int kFoldTerms = 48;  // plain FP32 terms per G entry before a fold

template <int S>
constexpr int g_rows() {
  return 33 - S;  // node rows per tile
}


// 16-byte planes per staged particle of the row gather after wx and wz:
// the products wy(j) u(a) (S*LC values), or, when those take more than two
// planes, wy and u themselves (each visit then forms the products wy(j) u(a)
// again: S*LC/2 more packed multiplies, one 16-byte shared load fewer for
// lda 3; the accumulation is bound by its shared wavefronts rather than its
// multiplies)
template <int S, int LC>
constexpr bool g_raw_u() {
  return S * LC > 8;
}
template <int S, int LC>
constexpr int g_wyu_units() {
  return g_raw_u<S, LC>() ? 2 : (S * LC + 3) / 4;
}
template <int S, class OT, int LC, bool WST>
constexpr size_t p2m3g_smem(int cap) {
  constexpr int NSC = (kGW + S - 1) * 32;
  constexpr int IU = p2m_rec_units<S, float, OT, WST>() + 1;
  // per slot: the weight planes and the raw next unit; per thread and unit
  // buffer: the S-1 inner boundaries of its accumulation window
  return (size_t)cap * (16 * (2 + g_wyu_units<S, LC>()) + 16 * IU) +
         sizeof(int) * (size_t)(6 * NSC) +
         sizeof(unsigned short) * (size_t)(2 * (S - 1) * kGW * 32);
}
// staging slots of the row gather: as many as fit in ~110 KB (two CTAs per
// SM), a multiple of 16
template <int S, class OT, int LC, bool WST>
constexpr int p2m3g_cap() {
  int cap = 2048;
  while (cap > 64 && p2m3g_smem<S, OT, LC, WST>(cap) > (size_t)110 * 1024) cap -= 16;
  return cap;
}

template <int S, bool COMP, class OT, int LC, bool WST>
__global__ void __launch_bounds__(kGW * 32, 2) k_p2m3g(P2MParams P) {
  constexpr int HL = S / 2;
  constexpr int HH = S / 2 - 1;
  constexpr int TYN = g_rows<S>();
  constexpr int WX = kGW + S - 1;  // staged columns
  constexpr int NSC = WX * 32;     // staged cells (32 rows)
  constexpr int NT = kGW * 32;
  constexpr int PERC = (NSC + NT - 1) / NT;
  constexpr int RU = p2m_rec_units<S, float, OT, WST>();
  constexpr int IU = RU + 1;
  static_assert(S <= 4 && LC <= 4, "stencil / components");

  if ((int)blockIdx.x >= *P.nitems) return;
  const int4 it = P.items[blockIdx.x];
  const int tiles_x = (P.span.ext[0] + kGW - 1) / kGW;
  const int X0 = P.span.org[0] + (it.x % tiles_x) * kGW;
  const int Y0 = P.span.org[1] + (it.x / tiles_x) * TYN;
  const int XE = P.span.org[0] + P.span.ext[0], YE = P.span.org[1] + P.span.ext[1];
  const int Z0 = it.y, Z1 = it.z;
  constexpr int cap = p2m3g_cap<S, OT, LC, WST>();
  constexpr int UW = g_wyu_units<S, LC>();

  extern __shared__ __align__(16) unsigned char smem[];
  float4* sWX = reinterpret_cast<float4*>(smem);
  float4* sWZ = sWX + cap;
  float4* sWYU = sWZ + cap;  // [UW][cap]: wy(j) u(a) at a * S + j, or wy and u
  constexpr bool RAWU = g_raw_u<S, LC>();
  uint4* raw = reinterpret_cast<uint4*>(sWYU + UW * cap);  // [cap][IU] next unit
  // cell ranges of a layer, [layer parity][NSC]: loaded one layer ahead
  int* nxb = reinterpret_cast<int*>(raw + (size_t)cap * IU);
  int* nxe = nxb + 2 * NSC;
  // [unit parity][NSC]: particles of each cell taken by the units before
  // (read by the plan of a unit) and with it (written by that plan)
  int* dn = nxe + 2 * NSC;
  // [2][S-1][NT]: inner cell boundaries of each lane's accumulation window
  unsigned short* sB = reinterpret_cast<unsigned short*>(dn + 2 * NSC);
  const float* sWXf = reinterpret_cast<const float*>(sWX);

  const int tid = threadIdx.x;
  const int w = tid >> 5, L = tid & 31;
  const int nx = X0 + w, ny = Y0 + L;
  const bool owner = L < TYN && nx < XE && ny < YE;
  const uint4* grec = static_cast<const uint4*>(P.rec);
  const uint4* gus = static_cast<const uint4*>(P.us);

  // G: plain FP32 partials, node rows j in pairs (j = 2J: .x, 2J + 1: .y);
  // (hi, lo): the compensated sums of the node planes; the planes form a
  // ring (slot = node plane mod S)
  float2 G[S / 2][S][LC];
  float hi[S][LC], lo[S][LC];
#pragma unroll
  for (int j = 0; j < S / 2; ++j)
#pragma unroll
    for (int k = 0; k < S; ++k)
#pragma unroll
      for (int a = 0; a < LC; ++a) G[j][k][a] = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < S; ++k)
#pragma unroll
    for (int a = 0; a < LC; ++a) hi[k][a] = lo[k][a] = 0.f;
  int nterm = 0;  // particles added to G since the warp's last fold

  // the staged cells of this thread (q = tid + NT k): their xy offset in
  // the cell numbering, -1 for cells outside the subdomain along a cut axis
  int64_t cxy[PERC];
#pragma unroll
  for (int k = 0; k < PERC; ++k) {
    const int q = tid + NT * k;
    const int r = q / WX, qx = q - r * WX;
    const int ux = X0 - HL + qx, uy = Y0 - HL + r;
    const bool out = q >= NSC || (P.open[0] && (ux < 0 || ux >= P.N[0])) ||
                     (P.open[1] && (uy < 0 || uy >= P.N[1]));
    cxy[k] = out ? -1 : (int64_t)wrap_index(ux, P.N[0]) +
                            (int64_t)P.N[0] * wrap_index(uy, P.N[1]);
  }
  const int64_t plane_cells = (int64_t)P.N[0] * P.N[1];
  // this thread's node column: its offset in field_up when it has no
  // periodic image along x or y (else every image is found per node)
  bool col_img = true;
  int64_t col_off = 0;
  if (owner) {
    int l0, h0, l1, h1;
    axis_images(P, 0, nx, l0, h0);
    axis_images(P, 1, ny, l1, h1);
    col_img = (l0 | h0 | l1 | h1) != 0;
    col_off = (int64_t)(nx + 1 - P.fd.lb[0]) * P.fd.s[0] +
              (int64_t)(ny + 1 - P.fd.lb[1]) * P.fd.s[1] + P.c0;
  }

  auto load_counts = [&](int cz) {
    const bool empty = P.open[2] && (cz < 0 || cz >= P.N[2]);
    const int64_t zoff = empty ? 0 : plane_cells * wrap_index(cz, P.N[2]);
    int* b = nxb + (cz & 1) * NSC;
    int* e = nxe + (cz & 1) * NSC;
#pragma unroll
    for (int k = 0; k < PERC; ++k) {
      const int q = tid + NT * k;
      if (q >= NSC) continue;
      if (!empty && cxy[k] >= 0) {
        const int* src = P.start + zoff + cxy[k];
        cp_async4(b + q, src);
        cp_async4(e + q, src + 1);
      } else {
        b[q] = e[q] = 0;
      }
    }
  };
  // Plan of a unit, without block barriers.  Unit slots follow the staged
  // cells in row-major order, so lane L of every warp walks row L's cell
  // ranges, and warp scans over the 32 rows give the row bases: every warp
  // computes the same plan.  Lane (w, L) keeps its accumulation window's
  // offsets (cells w .. w+S of its row) in registers and shared memory and
  // copies the particles of cells w and w + kGW of its row.
  // A layer's first unit takes all of its particles when they fit `cap`
  // (O(1) row offsets when the staged columns need no periodic wrap, since
  // the row's cells are then consecutive keys).  Else every unit gives each
  // cell with particles left an equal share of `cap` (the first `rem` such
  // cells one more), the taken counts kept per cell in dn.
  int p0c = 0, p1c = 0;  // window offsets of the planned unit (this lane)
  int left = 0;          // particles of the layer not yet in a unit
  // the staged columns X0-HL .. X0-HL+WX-1 need no periodic wrap along x
  const bool row_contig = X0 - HL >= 0 && X0 - HL + WX <= P.N[0];
  auto copy_cell = [&](int o0, int n, int64_t g0) {
    for (int i = 0; i < n; ++i) {
      const int o = o0 + i;
      const int64_t sp = g0 + i;
      uint4* d = raw + (size_t)o * IU;
#pragma unroll
      for (int t = 0; t < RU; ++t) {
        if constexpr (WST)
          cp_async16(d + t, grec + sp * RU + t);
        else
          cp_async16(d + t, grec + t * P.ps + sp);
      }
      cp_async16(d + RU, gus + sp);
    }
  };
  // the row offsets (run: the row's total) become unit offsets, the window
  // is published, and the owned cells are copied
  auto finish_plan = [&](int ob, int run, int ow, int ows, const int* oin, int o1, int n1,
                         int64_t b1, int o2, int n2, int64_t b2) -> int {
    int inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (L >= o) inc += t;
    }
    const int n = __shfl_sync(0xffffffffu, inc, 31);
    const int base = inc - run;
    p0c = base + ow;
    p1c = base + ows;
#pragma unroll
    for (int k = 0; k < S - 1; ++k)
      sB[(ob * (S - 1) + k) * NT + tid] = (unsigned short)(base + oin[k]);
    copy_cell(base + o1, n1, b1);
    if (w + kGW < WX) copy_cell(base + o2, n2, b2);
    cp_async_commit();
    return n;
  };
  auto plan_unit = [&](int par, int ob, bool first) -> int {
    const int* b = nxb + par * NSC + L * WX;
    const int* e = nxe + par * NSC + L * WX;
    int oin[S - 1];  // inner window boundaries (cells w+1 .. w+S-1), within the row
#pragma unroll
    for (int k = 0; k < S - 1; ++k) oin[k] = 0;
    if (first) {
      int run = 0, ow = 0, ows = 0, o1 = 0, n1 = 0, b1 = 0, o2 = 0, n2 = 0, b2 = 0;
      if (row_contig) {
        const int r0 = b[0];
        run = e[WX - 1] - r0;
        b1 = b[w];
        n1 = e[w] - b1;
        ow = o1 = b1 - r0;
        ows = w + S < WX ? b[w + S] - r0 : run;
#pragma unroll
        for (int k = 0; k < S - 1; ++k) oin[k] = b[w + 1 + k] - r0;
        if (w + kGW < WX) {
          b2 = b[w + kGW];
          n2 = e[w + kGW] - b2;
          o2 = b2 - r0;
        }
      } else {
#pragma unroll
        for (int qx = 0; qx < WX; ++qx) {
          const int bb = b[qx], cc = e[qx] - bb;
          if (qx == w) {
            ow = o1 = run;
            n1 = cc;
            b1 = bb;
          }
          if (qx == w + S) ows = run;
#pragma unroll
          for (int k = 0; k < S - 1; ++k)
            if (qx == w + 1 + k) oin[k] = run;
          if (qx == w + kGW) {
            o2 = run;
            n2 = cc;
            b2 = bb;
          }
          run += cc;
        }
        if (w + S == WX) ows = run;
      }
      const int total = __reduce_add_sync(0xffffffffu, run);
      if (total <= cap) {
        left = 0;
        return finish_plan(ob, run, ow, ows, oin, o1, n1, b1, o2, n2, b2);
      }
    }
    // equal shares: dn[ob] holds the counts taken before (none on the
    // layer's first unit), dn[ob ^ 1] gets the counts after this unit
    const int* dc = dn + ob * NSC + L * WX;
    int* dx = dn + (ob ^ 1) * NSC + L * WX;
    int rl = 0, ra = 0;
#pragma unroll
    for (int qx = 0; qx < WX; ++qx) {
      const int l = e[qx] - b[qx] - (first ? 0 : dc[qx]);
      rl += l;
      ra += l > 0 ? 1 : 0;
    }
    const int tot = __reduce_add_sync(0xffffffffu, rl);
    const int A = max(__reduce_add_sync(0xffffffffu, ra), 1);
    const int kk = cap / A, rem = cap - A * kk;
    int rk = ra;  // rank of the row's first cell with particles left: exclusive scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, rk, o);
      if (L >= o) rk += t;
    }
    rk -= ra;
    int run = 0, ow = 0, ows = 0, o1 = 0, n1 = 0, o2 = 0, n2 = 0;
    int64_t b1 = 0, b2 = 0;
#pragma unroll
    for (int qx = 0; qx < WX; ++qx) {
      const int d = first ? 0 : dc[qx];
      const int l = e[qx] - b[qx] - d;
      const int t = l > 0 ? min(l, kk + (rk < rem ? 1 : 0)) : 0;
      rk += l > 0 ? 1 : 0;
      if (qx == w) {
        ow = o1 = run;
        n1 = t;
        b1 = (int64_t)b[qx] + d;
      }
      if (qx == w + S) ows = run;
#pragma unroll
      for (int k = 0; k < S - 1; ++k)
        if (qx == w + 1 + k) oin[k] = run;
      if (qx == w + kGW) {
        o2 = run;
        n2 = t;
        b2 = (int64_t)b[qx] + d;
      }
      if (qx == w || qx == w + kGW) dx[qx] = d + t;
      run += t;
    }
    if (w + S == WX) ows = run;
    const int n = finish_plan(ob, run, ow, ows, oin, o1, n1, b1, o2, n2, b2);
    left = tot - n;
    return n;
  };
  // the sum over the warp's rows of ring slot k, component a of G for the
  // node row of this lane (lanes L .. L+S-1 contribute, nearest first)
  auto g_at = [&](int j, int k, int a) -> float {
    return (j & 1) ? G[j >> 1][k][a].y : G[j >> 1][k][a].x;
  };
  auto row_sum = [&](int k, int a) -> float {
    float s = g_at(S - 1, k, a);
#pragma unroll
    for (int d = 1; d < S; ++d) s += __shfl_down_sync(0xffffffffu, g_at(S - 1 - d, k, a), d);
    return s;
  };

  int cz = Z0 - HL;
  const int zlast = Z1 - 1 + HH;
  // ring slot of the node plane cz - HL + 1 (the first plane of layer cz)
  int ph = wrap_index(cz - HL + 1, S);
  load_counts(cz);
  cp_async_wait_all();
  __syncthreads();
  if (cz < zlast) load_counts(cz + 1);
  int n_cur = plan_unit(cz & 1, 0, true);
  bool last_cur = left == 0;

  for (int u = 0;; ++u) {
    const int ub = u & 1;
    cp_async_wait_all();
    __syncthreads();
    // 1. weights of unit u: raw -> structure-of-arrays slots
    for (int i = tid; i < n_cur; i += NT) {
      const uint4* r = raw + (size_t)i * IU;
      float wv[3][4];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int k = 0; k < 4; ++k) wv[d][k] = 0.f;
      if constexpr (WST) {
        const OT* wsrc = reinterpret_cast<const OT*>(r);
#pragma unroll
        for (int k = 0; k < S; ++k) {
          wv[0][k] = (float)wsrc[k];
          wv[1][k] = (float)wsrc[S + k];
          wv[2][k] = (float)wsrc[2 * S + k];
        }
      } else {
        const float4 rv = *reinterpret_cast<const float4*>(r);
        weights<S, float>(rv.x, wv[0]);
        weights<S, float>(rv.y, wv[1]);
        weights<S, float>(rv.z, wv[2]);
      }
      sWX[i] = make_float4(wv[0][0], wv[0][1], wv[0][2], wv[0][3]);
      sWZ[i] = make_float4(wv[2][0], wv[2][1], wv[2][2], wv[2][3]);
      const float4 u4 = *reinterpret_cast<const float4*>(r + RU);
      if constexpr (RAWU) {
        sWYU[i] = make_float4(wv[1][0], wv[1][1], wv[1][2], wv[1][3]);
        sWYU[cap + i] = u4;
      } else {
        const float uu[4] = {u4.x, u4.y, u4.z, u4.w};
        float f[4 * UW];
#pragma unroll
        for (int t = 0; t < 4 * UW; ++t) f[t] = 0.f;
#pragma unroll
        for (int aa = 0; aa < LC; ++aa)
#pragma unroll
          for (int j = 0; j < S; ++j) f[aa * S + j] = wv[1][j] * uu[aa];
#pragma unroll
        for (int t = 0; t < UW; ++t)
          sWYU[t * cap + i] = make_float4(f[4 * t], f[4 * t + 1], f[4 * t + 2], f[4 * t + 3]);
      }
    }
    __syncthreads();
    // 2. plan and issue unit u+1 (the next layer's first unit when unit u
    //    completes its layer)
    const int cz_u = cz;
    const bool last_u = last_cur;
    const int n_u = n_cur;
    const int p0u = p0c, p1u = p1c;
    bool more = true;
    if (last_u) {
      if (cz < zlast) {
        ++cz;
        // the ranges of layer cz + 1 go to the buffer layer cz - 1 used
        if (cz < zlast) load_counts(cz + 1);
        n_cur = plan_unit(cz & 1, ub ^ 1, true);
      } else {
        more = false;
      }
    } else {
      n_cur = plan_unit(cz & 1, ub ^ 1, false);
    }
    if (more) last_cur = left == 0;
    // 3.-5. with the ring phase a compile-time constant
    auto body = [&](auto phc) {
      constexpr int PH = decltype(phc)::value;
      // 3. accumulate unit u: the particles of cells w .. w+S-1 of row L
      if (n_u > 0) {
        const int p0 = p0u, p1 = p1u;
        // the window's inner cell boundaries: a particle of cell w + m
        // (m boundaries at or below it) takes x-weight S-1-m for node X0 + w
        int bnd[S - 1];
#pragma unroll
        for (int k = 0; k < S - 1; ++k) bnd[k] = (int)sB[(ub * (S - 1) + k) * NT + tid];
        nterm += p1 - p0;
        for (int p = p0; p < p1; ++p) {
          int ix = S - 1;
#pragma unroll
          for (int k = 0; k < S - 1; ++k) ix -= p >= bnd[k] ? 1 : 0;
          const float wxi = sWXf[4 * p + ix];
          const float4 wz4 = sWZ[p];
          const float wz[4] = {wz4.x, wz4.y, wz4.z, wz4.w};
          if constexpr (RAWU) {
            const float4 wy4 = sWYU[p];
            const float4 u4 = sWYU[cap + p];
            const float uu[4] = {u4.x, u4.y, u4.z, u4.w};
            const float wy[4] = {wy4.x, wy4.y, wy4.z, wy4.w};
            const float2 wx2 = make_float2(wxi, wxi);
            // (wx (wy(2J) u(a)), wx (wy(2J+1) u(a))) times wz(k), packed FP32
            // pairs: the products in the order of the staged form
#pragma unroll
            for (int a = 0; a < LC; ++a) {
              const float2 u2 = make_float2(uu[a], uu[a]);
#pragma unroll
              for (int J = 0; J < S / 2; ++J) {
                const float2 cu =
                    __fmul2_rn(wx2, __fmul2_rn(make_float2(wy[2 * J], wy[2 * J + 1]), u2));
#pragma unroll
                for (int k = 0; k < S; ++k)
                  G[J][(PH + k) % S][a] =
                      __ffma2_rn(cu, make_float2(wz[k], wz[k]), G[J][(PH + k) % S][a]);
              }
            }
          } else {
            float f[4 * UW];
#pragma unroll
            for (int t = 0; t < UW; ++t) {
              const float4 v = sWYU[t * cap + p];
              f[4 * t] = v.x;
              f[4 * t + 1] = v.y;
              f[4 * t + 2] = v.z;
              f[4 * t + 3] = v.w;
            }
            const float2 wx2 = make_float2(wxi, wxi);
            // (wx wy(2J) u(a), wx wy(2J+1) u(a)) times wz(k), packed FP32 pairs
#pragma unroll
            for (int J = 0; J < S / 2; ++J)
#pragma unroll
              for (int a = 0; a < LC; ++a) {
                const float2 cu =
                    __fmul2_rn(wx2, make_float2(f[a * S + 2 * J], f[a * S + 2 * J + 1]));
#pragma unroll
                for (int k = 0; k < S; ++k)
                  G[J][(PH + k) % S][a] =
                      __ffma2_rn(cu, make_float2(wz[k], wz[k]), G[J][(PH + k) % S][a]);
              }
          }
        }
      }
      // 4. fold G into the node ring once a lane has added kFoldTerms
      //    particles since the warp's last fold
      if constexpr (COMP) {
        if (__any_sync(0xffffffffu, nterm > kFoldTerms)) {
#pragma unroll
          for (int k = 0; k < S; ++k)
#pragma unroll
            for (int a = 0; a < LC; ++a) {
              const float s = row_sum(k, a);
              two_sum_fold<float>(hi[k][a], lo[k][a], s);
            }
#pragma unroll
          for (int j = 0; j < S / 2; ++j)
#pragma unroll
            for (int k = 0; k < S; ++k)
#pragma unroll
              for (int a = 0; a < LC; ++a) G[j][k][a] = make_float2(0.f, 0.f);
          nterm = 0;
        }
      }
      // 5. layer complete: node plane zc (slot PH) is final: write it and
      //    clear its slot for plane zc + S
      if (last_u) {
        const int zc = cz_u - (HL - 1);
        float s0[LC];
#pragma unroll
        for (int a = 0; a < LC; ++a) s0[a] = row_sum(PH, a);
        if (owner && zc >= Z0 && zc < Z1) {
          double v[LC];
#pragma unroll
          for (int a = 0; a < LC; ++a)
            v[a] = COMP ? ((double)hi[PH][a] + (double)lo[PH][a]) + (double)s0[a]
                        : (double)s0[a];
          int l2, h2;
          axis_images(P, 2, zc, l2, h2);
          if (!col_img && (l2 | h2) == 0) {
            OT* F = static_cast<OT*>(P.field) + col_off +
                    (int64_t)(zc + 1 - P.fd.lb[2]) * P.fd.s[2];
#pragma unroll
            for (int a = 0; a < LC; ++a) F[a] = (OT)v[a];
          } else {
            emit_node<3, OT, LC>(P, nx, ny, zc, v);
          }
        }
#pragma unroll
        for (int a = 0; a < LC; ++a) {
#pragma unroll
          for (int j = 0; j < S / 2; ++j) G[j][PH][a] = make_float2(0.f, 0.f);
          hi[PH][a] = lo[PH][a] = 0.f;
        }
      }
    };
    if constexpr (S == 4) {
      switch (ph) {
        case 0: body(std::integral_constant<int, 0>{}); break;
        case 1: body(std::integral_constant<int, 1>{}); break;
        case 2: body(std::integral_constant<int, 2>{}); break;
        default: body(std::integral_constant<int, 3>{}); break;
      }
    } else {
      if (ph == 0)
        body(std::integral_constant<int, 0>{});
      else
        body(std::integral_constant<int, 1>{});
    }
    if (last_u) ph = ph + 1 == S ? 0 : ph + 1;
    if (!more) break;
  }
}

// Per (xy tile, cell layer): particles in the tile's own cells of that layer
// (tiles of the span from (ox, oy), ex x ey nodes; cells outside 0 .. N-1
// count none), stored tile-major: lc[tile * N2 + cz] (k_make_items walks a
// tile's layers in one thread).
__global__ void k_layer_counts(const int* __restrict__ start, int N0, int N1, int N2, int ox,
                               int oy, int ex, int ey, int tdx, int tdy, int tiles_x,
                               int ntiles, int* __restrict__ lc) {
  const int64_t n = (int64_t)ntiles * N2;
  // i = cz * ntiles + tile: neighbouring threads take neighbouring tiles of
  // one layer, whose row ends share sectors of start[] (186 -> 83 us at 512^3
  // against layer-fastest threads)
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int tile = (int)(i % ntiles), cz = (int)(i / ntiles);
    const int tx0 = ox + (tile % tiles_x) * tdx, ty0 = oy + (tile / tiles_x) * tdy;
    const int X0 = max(tx0, 0), X1 = min(min(tx0 + tdx, ox + ex), N0);
    const int Y0 = max(ty0, 0), Y1 = min(min(ty0 + tdy, oy + ey), N1);
    int sum = 0;
    for (int y = Y0; y < Y1 && X0 < X1; ++y) {
      const int64_t c0 = (int64_t)X0 + (int64_t)N0 * (y + (int64_t)N1 * cz);
      sum += start[c0 + (X1 - X0)] - start[c0];
    }
    lc[(int64_t)tile * N2 + cz] = sum;
  }
}

// Split every xy tile's z range into work items of about `target` particles
// (at least min_tz and at most max_tz layers; the halo makes short items dear).
// The z planes are zlo .. zlo+ze-1; plane z counts the particles of cell
// layer z (none outside 0 .. N2-1).
__global__ void k_make_items(const int* __restrict__ lc, int N2, int zlo, int ze, int ntiles,
                             int target, int min_tz, int max_tz, int4* __restrict__ items,
                             int* __restrict__ nitems) {
  // one warp per tile: lane l holds layer c0 + l of a chunk of 32 and the
  // chunk's inclusive prefix of the counts; the item ends are the layers the
  // sequential rule below would cut at, found a chunk at a time by ballots
  //   acc: particles since the item's first layer z0, len = ez + 1 - z0;
  //   cut at ez when ez is the last layer, or when (acc >= target and
  //   len >= min_tz, or len >= max_tz) and min_tz layers or more remain
  const int lane = threadIdx.x & 31;
  const int tile = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (tile >= ntiles) return;
  int z0 = 0, carry = 0;  // item start; its particles in the chunks before
  for (int c0 = 0; c0 < ze; c0 += 32) {
    const int ez = c0 + lane;
    const int cz = zlo + ez;
    const int v = (ez < ze && cz >= 0 && cz < N2) ? lc[(int64_t)tile * N2 + cz] : 0;
    int pre = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, pre, o);
      if (lane >= o) pre += t;
    }
    for (;;) {
      // the prefix up to the layer before z0 (or minus the carry when the
      // item began in an earlier chunk)
      const int at = z0 - c0 - 1;
      const int pz = __shfl_sync(0xffffffffu, pre, at >= 0 ? at : 0);
      const int s0 = at >= 0 ? pz : -carry;
      const int acc = pre - s0;
      const int len = ez + 1 - z0;
      const bool want = (acc >= target && len >= min_tz) || len >= max_tz;
      const bool cut = ez >= z0 && ez < ze && (ez == ze - 1 || (want && ze - (ez + 1) >= min_tz));
      const unsigned m = __ballot_sync(0xffffffffu, cut);
      if (m == 0) {
        carry = __shfl_sync(0xffffffffu, acc, 31);  // the item's particles up to the chunk end
        break;
      }
      const int f = __ffs(m) - 1;
      if (lane == f) {
        const int q = atomicAdd(nitems, 1);
        // weight: particles of the item's own cells + a per-layer cost
        items[q] = make_int4(tile, zlo + z0, zlo + ez + 1, acc + 32 * len);
      }
      z0 = c0 + f + 1;
      carry = 0;
      if (z0 >= c0 + 32 || z0 >= ze) break;
    }
  }
}

// Longest items first (a one-CTA bucket sort by log2 weight, heaviest bucket
// first): heavy items of dense regions start in the first wave instead of
// stretching the tail.  Items write disjoint nodes, so the order changes
// only the schedule, never a result.
__global__ void __launch_bounds__(1024) k_order_items(const int4* __restrict__ tmp,
                                                      const int* __restrict__ nitems,
                                                      int4* __restrict__ items) {
  __shared__ int hist[32];
  const int n = *nitems;
  if (threadIdx.x < 32) hist[threadIdx.x] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    atomicAdd(&hist[31 - __clz(max(tmp[i].w, 1))], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int b = 31; b >= 0; --b) {
      const int c = hist[b];
      hist[b] = run;
      run += c;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int4 t = tmp[i];
    items[atomicAdd(&hist[31 - __clz(max(t.w, 1))], 1)] = t;
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
        const V u = load_vec(us, s, P.ps);
        CT w[2][S];
        if constexpr (WST) {
          // stored weights: 2 x S values of the field's type, padded to 16 bytes
          constexpr int WS2 = (2 * S * (int)sizeof(OT) + 15) / 16 * 16 / (int)sizeof(OT);
          const OT* ws = static_cast<const OT*>(P.rec) + s * WS2;
#pragma unroll
          for (int k = 0; k < S; ++k) {
            w[0][k] = (CT)ws[k];
            w[1][k] = (CT)ws[S + k];
          }
        } else {
          const V r = load_vec(rec, s, P.ps);
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
    P2MParams Q = P;
    int cap = 2048;
    size_t smem;
    cudaError_t e;
    if constexpr (std::is_same<CT, float>::value) {
      // row gather (FP32 arithmetic): two CTAs of 8 warps per SM, staging
      // slots in ~110 KB each
      cap = p2m3g_cap<S, OT, LC, WST>();
      Q.cap = cap;
      smem = p2m3g_smem<S, OT, LC, WST>(cap);
      auto kern = k_p2m3g<S, COMP, OT, LC, WST>;
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      kern<<<Q.item_cap, kGW * 32, smem, st>>>(Q);
    } else {
      // tile gather (the FP64 form): staging slots in ~110 KB (2 CTAs / SM)
      while (cap > 64 && p2m3d_smem<S, CT, OT, WST>(cap) > (size_t)110 * 1024) cap -= 16;
      Q.cap = cap;
      smem = p2m3d_smem<S, CT, OT, WST>(cap);
      auto kern = k_p2m3d<S, CT, COMP, OT, LC, WST>;
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      kern<<<Q.item_cap, kTX * kTY, smem, st>>>(Q);
    }
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
  const int tx = (N[0] + kTile2 - 1) / kTile2;
  int want = (148 * 8 + tx - 1) / tx;  // ~8 CTAs per SM in total
  int tz = (N[1] + want - 1) / want;
  (void)dim;
  return tz < 8 ? (N[1] < 8 ? N[1] : 8) : tz;
}

TileSpan cell_span(const int N[3]) {
  TileSpan sp;
  for (int a = 0; a < 3; ++a) {
    sp.org[a] = 0;
    sp.ext[a] = N[a];
  }
  return sp;
}

namespace {
constexpr int kMinTZ = 8, kMaxTZ = 64;
int tiles_xy(const TileSpan& sp, int tdx, int tdy) {
  return ((sp.ext[0] + tdx - 1) / tdx) * ((sp.ext[1] + tdy - 1) / tdy);
}
int item_capacity(const TileSpan& sp, int tdx, int tdy) {
  return tiles_xy(sp, tdx, tdy) * ((sp.ext[2] + kMinTZ - 1) / kMinTZ) + 1;
}
TileSpan span_of(const int N[3], const TileSpan* sp) { return sp ? *sp : cell_span(N); }
size_t items_bytes(const TileSpan& s, int N2, int tdx, int tdy) {
  return 2 * sizeof(int4) * (size_t)item_capacity(s, tdx, tdy) +
         sizeof(int) * (size_t)tiles_xy(s, tdx, tdy) * N2 + 64;
}
}  // namespace

// Layout: items[cap] | nitems (64 bytes) | unordered items[cap] | layer counts
size_t tile_items_bytes(const int N[3], const TileSpan* sp) {
  return items_bytes(span_of(N, sp), N[2], kTileX, kTileY);
}

size_t p2m_scratch_bytes(int dim, const int N[3], const TileSpan* sp) {
  if (dim != 3) return 16;
  // the items of either 3D gather (tile gather or row gather)
  const TileSpan s = span_of(N, sp);
  const size_t a = items_bytes(s, N[2], kTileX, kTileY);
  const size_t b = items_bytes(s, N[2], kGW, g_rows<2>());
  const size_t c = items_bytes(s, N[2], kGW, g_rows<4>());
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

bool p2m_row_gather(int dim, P2MPrec prec) { return dim == 3 && prec != P2M_FP64; }

TileItems tile_items_view(void* scratch, const int N[3], const TileSpan* sp) {
  TileItems t;
  t.cap = item_capacity(span_of(N, sp), kTileX, kTileY);
  t.items = static_cast<const int4*>(scratch);
  t.nitems = reinterpret_cast<const int*>(t.items + t.cap);
  return t;
}

cudaError_t make_tile_items(const int* start, const int N[3], int64_t nvalid, void* scratch,
                            TileItems& out, cudaStream_t st, const TileSpan* sp, int tdx,
                            int tdy) {
  const TileSpan s = span_of(N, sp);
  const int zlo = s.org[2], ze = s.ext[2];
  const int nt = tiles_xy(s, tdx, tdy);
  const int cap_items = item_capacity(s, tdx, tdy);
  int4* items = static_cast<int4*>(scratch);
  int* nitems = reinterpret_cast<int*>(items + cap_items);
  int4* unordered = reinterpret_cast<int4*>(nitems + 16);
  int* lc = reinterpret_cast<int*>(unordered + cap_items);
  cudaError_t e = cudaMemsetAsync(nitems, 0, sizeof(int), st);
  if (e) return e;
  const int64_t nl = (int64_t)nt * N[2];
  const int gl = (int)((nl + 255) / 256 < 148 * 32 ? (nl + 255) / 256 : 148 * 32);
  k_layer_counts<<<gl, 256, 0, st>>>(start, N[0], N[1], N[2], s.org[0], s.org[1], s.ext[0],
                                     s.ext[1], tdx, tdy, (s.ext[0] + tdx - 1) / tdx, nt, lc);
  // the tile gathers: ~16 items per SM (two CTAs per SM), 8-64 layers; the
  // row gather (a dearer per-layer halo): ~8 per SM, 16-128
  const bool rows = tdx == kGW;
  const int64_t tgt64 = nvalid / (rows ? 148 * 8 : 148 * 2 * 8);
  const int target = (int)(tgt64 < 4096 ? 4096 : (tgt64 > (1 << 30) ? (1 << 30) : tgt64));
  k_make_items<<<(nt + 3) / 4, 128, 0, st>>>(lc, N[2], zlo, ze, nt, target,
                                                 rows ? 2 * kMinTZ : kMinTZ,
                                                 rows ? 2 * kMaxTZ : kMaxTZ, unordered, nitems);
  k_order_items<<<1, 1024, 0, st>>>(unordered, nitems, items);
  count_launch(3);
  out.items = items;
  out.nitems = nitems;
  out.cap = cap_items;
  return cudaGetLastError();
}

cudaError_t launch_p2m(const P2MParams& P0, int dim, int kernel, P2MPrec prec, int lda,
                       int64_t nvalid, bool stored_weights, void* scratch, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  P2MParams Pw = P0;
  Pw.ps = nvalid;
  if (dim == 3) {
    // work items: xy tiles split along z into segments of similar particle count
    TileItems ti;
    const bool rows = p2m_row_gather(dim, prec);
    const int tdy = rows ? (kernel == kKernelMp4 ? g_rows<4>() : g_rows<2>()) : kTileY;
    if ((e = make_tile_items(P0.start, P0.N, nvalid, scratch, ti, st, &P0.span,
                             rows ? kGW : kTileX, tdy)))
      return e;
    Pw.items = ti.items;
    Pw.nitems = ti.nitems;
    Pw.item_cap = ti.cap;
  }
  TimingScope timed(dim == 3 ? kTimeP2M : kTimedParts, dim == 3 ? st : nullptr);
  const int nchunk = (lda + 3) / 4;
  for (int ch = 0; ch < nchunk; ++ch) {
    P2MParams P = Pw;
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
