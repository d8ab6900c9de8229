// ppmg_map.cu -- particle redistribution between z-slab subdomains: the
// routing step of ppm_map_part_partial (ppm/src/ppm_map_part_partial.f:
// 288-420: every particle goes to the neighbouring subdomain that contains
// it, closed-lower / open-upper containment) and the gather that packs
// positions and properties in routed order.  The transfer between the
// slabs' GPUs is the host's (ppm_legacy_b200.halo over torch.distributed).
#include <cuda_runtime.h>

#include "ppmg_map.cuh"

namespace ppmg {

namespace {

constexpr int kRouteThreads = 256;
constexpr int kRouteChunk = 4096;  // items per block, visited in order

// Class of one particle: 0 inside the local slab, 1 in the slab below,
// 2 in the slab above, 3 in none of them.
template <class T>
__device__ __forceinline__ int route_class(const RouteParams& R, const T* x) {
  constexpr bool F = sizeof(T) == 4;
  bool inxy = true;
  for (int a = 0; a < 2; ++a) {
    const T lo = F ? (T)R.lof[a] : (T)R.lo[a], hi = F ? (T)R.hif[a] : (T)R.hi[a];
    inxy = inxy && x[a] >= lo && x[a] < hi;
  }
  if (!inxy) return 3;
  for (int c = 0; c < 3; ++c) {
    const T lo = F ? (T)R.zlof[c] : (T)R.zlo[c], hi = F ? (T)R.zhif[c] : (T)R.zhi[c];
    if (x[2] >= lo && x[2] < hi) return c;
  }
  return 3;
}

// Per block: the class of every item (dest) and the block's count per class
// (bc[c * nblk + b]).
template <class T>
__global__ void __launch_bounds__(kRouteThreads) k_route_count(RouteParams R, const T* xp,
                                                               int64_t ldxp, int64_t np,
                                                               unsigned char* dest, int* bc,
                                                               int nblk) {
  __shared__ int cnt[4];
  if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * kRouteChunk;
  const int64_t b1 = min(np, b0 + kRouteChunk);
  int mine[4] = {0, 0, 0, 0};
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kRouteThreads) {
    const int c = route_class<T>(R, xp + i * ldxp);
    dest[i] = (unsigned char)c;
    ++mine[c];
  }
  for (int c = 0; c < 4; ++c)
    if (mine[c]) atomicAdd(&cnt[c], mine[c]);
  __syncthreads();
  if (threadIdx.x < 4) bc[(int64_t)threadIdx.x * nblk + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter: item i of class c goes to off[c * nblk + b] + (its rank
// among the block's class-c items), visiting the block's items in order in
// rounds of 256 (per-warp ballots, warp totals scanned in shared memory).
__global__ void __launch_bounds__(kRouteThreads) k_route_scatter(const unsigned char* dest,
                                                                 int64_t np, const int* off,
                                                                 int nblk, int* perm) {
  __shared__ int wcnt[4][kRouteThreads / 32];
  __shared__ int run[4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x < 4) run[threadIdx.x] = off[(int64_t)threadIdx.x * nblk + blockIdx.x];
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * kRouteChunk;
  const int64_t b1 = min(np, b0 + kRouteChunk);
  for (int64_t base = b0; base < b1; base += kRouteThreads) {
    const int64_t i = base + threadIdx.x;
    const int c = i < b1 ? (int)dest[i] : -1;
    unsigned m[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      m[k] = __ballot_sync(0xffffffffu, c == k);
      if (lane == 0) wcnt[k][w] = __popc(m[k]);
    }
    __syncthreads();
    if (c >= 0) {
      int before = run[c];
      for (int ww = 0; ww < w; ++ww) before += wcnt[c][ww];
      before += __popc(m[c] & ((1u << lane) - 1u));
      perm[before] = (int)i;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      int t = 0;
      for (int ww = 0; ww < kRouteThreads / 32; ++ww) t += wcnt[threadIdx.x][ww];
      run[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

// Global routing: the class of every item is its subdomain (the reference
// tests the subdomains from the last to the first, ppm_map_part_global.f:355-420;
// the boxes do not overlap, so the first hit is the only one) or nsubs.
template <class T>
__global__ void __launch_bounds__(kRouteThreads) k_groute_count(GlobalRouteParams R,
                                                                const T* xp, int64_t ldxp,
                                                                int64_t np, unsigned char* dest,
                                                                int* bc, int nblk) {
  __shared__ int cnt[kMaxGlobalSubs + 1];
  __shared__ T bl[3][kMaxGlobalSubs], bh[3][kMaxGlobalSubs];
  const int ncls = R.nsubs + 1;
  for (int c = threadIdx.x; c < ncls; c += kRouteThreads) cnt[c] = 0;
  for (int q = threadIdx.x; q < R.nsubs; q += kRouteThreads)
    for (int a = 0; a < 3; ++a) {
      // the positions' own precision, as the reference compares
      bl[a][q] = (T)R.box[a * R.nsubs + q];
      bh[a][q] = (T)R.box[(3 + a) * R.nsubs + q];
    }
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * kRouteChunk;
  const int64_t b1 = min(np, b0 + kRouteChunk);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kRouteThreads) {
    const T* x = xp + i * ldxp;
    const T x0 = x[0], x1 = x[1], x2 = x[2];
    int c = R.nsubs;
    for (int q = R.nsubs - 1; q >= 0; --q)
      if (x0 >= bl[0][q] && x0 < bh[0][q] && x1 >= bl[1][q] && x1 < bh[1][q] &&
          x2 >= bl[2][q] && x2 < bh[2][q]) {
        c = q;
        break;
      }
    dest[i] = (unsigned char)c;
    atomicAdd(&cnt[c], 1);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncls; c += kRouteThreads)
    bc[(int64_t)c * nblk + blockIdx.x] = cnt[c];
}

// Stable scatter into ncls classes: rounds of 256 items in order; lanes of
// one class in a warp are found with __match_any_sync, the warps' counts per
// class are kept in shared memory (zeroed by their writers after use).
__global__ void __launch_bounds__(kRouteThreads) k_groute_scatter(const unsigned char* dest,
                                                                  int64_t np, const int* off,
                                                                  int nblk, int ncls,
                                                                  int* perm) {
  constexpr int W = kRouteThreads / 32;
  __shared__ int wcnt[kMaxGlobalSubs + 1][W];
  __shared__ int run[kMaxGlobalSubs + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c = threadIdx.x; c < ncls; c += kRouteThreads) {
    run[c] = off[(int64_t)c * nblk + blockIdx.x];
    for (int ww = 0; ww < W; ++ww) wcnt[c][ww] = 0;
  }
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * kRouteChunk;
  const int64_t b1 = min(np, b0 + kRouteChunk);
  for (int64_t base = b0; base < b1; base += kRouteThreads) {
    const int64_t i = base + threadIdx.x;
    const int c = i < b1 ? (int)dest[i] : -1;
    const unsigned m = __match_any_sync(0xffffffffu, c);
    const bool leader = lane == __ffs(m) - 1;
    if (c >= 0 && leader) wcnt[c][w] = __popc(m);
    __syncthreads();
    if (c >= 0) {
      int before = run[c];
      for (int ww = 0; ww < w; ++ww) before += wcnt[c][ww];
      before += __popc(m & ((1u << lane) - 1u));
      perm[before] = (int)i;
    }
    __syncthreads();
    if (c >= 0 && leader) {
      atomicAdd(&run[c], wcnt[c][w]);
      wcnt[c][w] = 0;
    }
    __syncthreads();
  }
}

template <class T>
__global__ void k_gather_cols(const T* src, int64_t lds, int lda, const int* perm, int64_t n,
                              T* dst, int64_t ldd) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const T* s = src + (int64_t)perm[j] * lds;
    T* d = dst + j * ldd;
    for (int a = 0; a < lda; ++a) d[a] = s[a];
  }
}

}  // namespace

int route_blocks(int64_t np) { return (int)((np + kRouteChunk - 1) / kRouteChunk); }

template <class T>
cudaError_t launch_route(const RouteParams& R, const T* xp, int64_t ldxp, int64_t np,
                         unsigned char* dest, int* bc, int* off, int* perm, Workspace& ws,
                         cudaStream_t st) {
  if (np <= 0) return cudaSuccess;
  const int nblk = route_blocks(np);
  k_route_count<T><<<nblk, kRouteThreads, 0, st>>>(R, xp, ldxp, np, dest, bc, nblk);
  count_launch();
  cudaError_t e = scan_exclusive(bc, off, (int64_t)4 * nblk, ws, st);
  if (e) return e;
  k_route_scatter<<<nblk, kRouteThreads, 0, st>>>(dest, np, off, nblk, perm);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_route_global(const GlobalRouteParams& R, const T* xp, int64_t ldxp,
                                int64_t np, unsigned char* dest, int* bc, int* off, int* perm,
                                Workspace& ws, cudaStream_t st) {
  if (np <= 0) return cudaSuccess;
  if (R.nsubs < 1 || R.nsubs > kMaxGlobalSubs) return cudaErrorInvalidValue;
  const int nblk = route_blocks(np);
  const int ncls = R.nsubs + 1;
  k_groute_count<T><<<nblk, kRouteThreads, 0, st>>>(R, xp, ldxp, np, dest, bc, nblk);
  count_launch();
  cudaError_t e = scan_exclusive(bc, off, (int64_t)ncls * nblk, ws, st);
  if (e) return e;
  k_groute_scatter<<<nblk, kRouteThreads, 0, st>>>(dest, np, off, nblk, ncls, perm);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_gather_cols(const T* src, int64_t lds, int lda, const int* perm, int64_t n,
                               T* dst, int64_t ldd, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  k_gather_cols<T><<<(int)b, 256, 0, st>>>(src, lds, lda, perm, n, dst, ldd);
  count_launch();
  return cudaGetLastError();
}

template cudaError_t launch_route<double>(const RouteParams&, const double*, int64_t, int64_t,
                                          unsigned char*, int*, int*, int*, Workspace&,
                                          cudaStream_t);
template cudaError_t launch_route<float>(const RouteParams&, const float*, int64_t, int64_t,
                                         unsigned char*, int*, int*, int*, Workspace&,
                                         cudaStream_t);
template cudaError_t launch_route_global<double>(const GlobalRouteParams&, const double*,
                                                 int64_t, int64_t, unsigned char*, int*, int*,
                                                 int*, Workspace&, cudaStream_t);
template cudaError_t launch_route_global<float>(const GlobalRouteParams&, const float*, int64_t,
                                                int64_t, unsigned char*, int*, int*, int*,
                                                Workspace&, cudaStream_t);
template cudaError_t launch_gather_cols<double>(const double*, int64_t, int, const int*, int64_t,
                                                double*, int64_t, cudaStream_t);
template cudaError_t launch_gather_cols<float>(const float*, int64_t, int, const int*, int64_t,
                                               float*, int64_t, cudaStream_t);

}  // namespace ppmg
