// ppmg_sort_dev.cuh -- device helpers shared by the counting sort and the
// radix sort: cell keys and offsets of particles, position fingerprints and
// block-wide scans.
#pragma once

#include "ppmg_sort.cuh"

namespace ppmg {

template <class T>
struct KeyArith;
template <>
struct KeyArith<double> {
  __device__ static double mn(const KeyParams& k, int a) { return k.min[a]; }
  __device__ static double mx(const KeyParams& k, int a) { return k.max[a]; }
  __device__ static double di(const KeyParams& k, int a) { return k.dxi[a]; }
};
template <>
struct KeyArith<float> {
  __device__ static float mn(const KeyParams& k, int a) { return k.minf[a]; }
  __device__ static float mx(const KeyParams& k, int a) { return k.maxf[a]; }
  __device__ static float di(const KeyParams& k, int a) { return k.dxif[a]; }
};

// Cell of one particle along one axis, and its offset f from the stencil
// origin, as the reference computes them (ppm_interp_p2m.f:800-822):
// xi = (x - min_sub) * dxi, i0 = INT(xi), f = xi - i0.
template <class T>
__device__ __forceinline__ bool cell_axis(const KeyParams& kp, int a, T x, int& cell, T& f) {
  using A = KeyArith<T>;
  const T xi = rmul(rsub(x, A::mn(kp, a)), A::di(kp, a));
  const int n = kp.N[a];
  if (kp.mode == KEY_INTERP_CHECKED || kp.open[a]) {
    // closed-lower / open-upper containment (periodic upper face)
    if (!(x >= A::mn(kp, a) && x < A::mx(kp, a))) return false;
    int i0 = (int)xi;  // xi >= 0 here: INT == FLOOR
    // xi may round up to exactly Nc: on a periodic axis that is cell 0 at
    // offset 0, on an open axis the last cell at offset 1 (the same node
    // weights: only the node at the upper face gets 1)
    if (kp.open[a] && i0 >= n) i0 = n - 1;
    f = rsub(xi, (T)i0);
    cell = i0 >= n ? i0 - n : i0;
    return true;
  }
  // periodic wrap of any finite position
  if (!(fabs((double)xi) < 1.0e9)) return false;
  T fl = floor(xi);
  f = rsub(xi, fl);
  cell = wrap_index((int)fl, n);
  return true;
}

// 64-bit fingerprint of a particle's coordinates (splitmix64 finaliser over
// the coordinate bits and the particle index); summed over particles it
// identifies a position array (accidental equality ~2^-64).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
template <class T>
__device__ __forceinline__ unsigned long long bits64(T v) {
  if constexpr (sizeof(T) == 8) return (unsigned long long)__double_as_longlong((double)v);
  else return (unsigned long long)(unsigned)__float_as_int((float)v);
}
template <class T>
__device__ __forceinline__ unsigned long long particle_hash(const T* x, int dim, int64_t p) {
  unsigned long long h = mix64((unsigned long long)p);
  for (int a = 0; a < dim; ++a) h = mix64(h ^ bits64<T>(x[a]));
  return h;
}
__device__ __forceinline__ void block_add_hash(unsigned long long v, unsigned long long* out) {
  __shared__ unsigned long long part[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) part[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    atomicAdd(out, t);
  }
}

__device__ __forceinline__ int warp_incl_scan(int v) {
  const unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (unsigned)o) v += n;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ int block_excl_scan(int v, int* smem_warp, int& total) {
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  int inc = warp_incl_scan(v);
  if (lane == 31) smem_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? smem_warp[lane] : 0;
    int wi = warp_incl_scan(w);
    if (lane < nw) smem_warp[lane] = wi - w;
    if (lane == nw - 1) smem_warp[32] = wi;
  }
  __syncthreads();
  int excl = inc - v + smem_warp[wid];
  total = smem_warp[32];
  __syncthreads();
  return excl;
}

}  // namespace ppmg
