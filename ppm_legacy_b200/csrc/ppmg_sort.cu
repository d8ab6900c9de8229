// ppmg_sort.cu -- device counting sort into cell lists (see ppmg_sort.cuh).
#include <cuda_runtime.h>

#include <cmath>

#include "ppmg_sort_dev.cuh"
#include "ppmg_sort.cuh"

namespace ppmg {

cudaError_t DevBuf::ensure(size_t n) {
  if (fixed) return n <= bytes && p != nullptr ? cudaSuccess : cudaErrorMemoryAllocation;
  if (n <= bytes && p != nullptr) return cudaSuccess;
  if (p) {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  size_t want = n < 256 ? 256 : n;
  // grow with headroom so slowly growing particle counts do not reallocate
  want = want + want / 8;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    return e;
  }
  bytes = want;
  return cudaSuccess;
}

void DevBuf::release() {
  if (fixed) return;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

Workspace::~Workspace() {
  DevBuf* all[] = {&key, &slot, &idx, &count, &start, &bsum, &rec, &us, &err,
                   &big, &tiles, &h_xp, &h_up, &h_field, &h_aux, &w1d,
                   &key2, &idx2, &rec2, &hist, &gaps};
  for (DevBuf* b : all) b->release();
  if (h_err_pinned) cudaFreeHost(h_err_pinned);
}

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanRounds = 16;
constexpr int kScanTile = kScanThreads * kScanRounds;
constexpr int kSmallCell = 64;

__global__ void k_scan_reduce(const int* __restrict__ in, int64_t n, int* __restrict__ bsum) {
  __shared__ int sw[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int acc = 0;
#pragma unroll 4
  for (int r = 0; r < kScanRounds; ++r) {
    int64_t i = base + (int64_t)r * kScanThreads + threadIdx.x;
    if (i < n) acc += in[i];
  }
  int tot;
  (void)block_excl_scan(acc, sw, tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_bsum(int* bsum, int nb) {
  __shared__ int sw[33];
  int carry = 0;
  for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
    int i = b0 + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    int tot;
    int ex = block_excl_scan(v, sw, tot);
    if (i < nb) bsum[i] = ex + carry;
    carry += tot;
  }
}

__global__ void k_scan_apply(const int* in, int* out, int64_t n, const int* __restrict__ bsum) {
  __shared__ int sw[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int carry = bsum[blockIdx.x];
  for (int r = 0; r < kScanRounds; ++r) {
    int64_t i = base + (int64_t)r * kScanThreads + threadIdx.x;
    int v = i < n ? in[i] : 0;
    int tot;
    int ex = block_excl_scan(v, sw, tot);
    if (i < n) out[i] = ex + carry;
    carry += tot;
  }
}

template <class T>
__global__ void k_bin(KeyParams kp, const T* __restrict__ xp, int64_t ldxp, int64_t np,
                      int* __restrict__ key, int* __restrict__ slot, int* __restrict__ count,
                      int* __restrict__ err, T* __restrict__ zout, int64_t ldz, int nz,
                      unsigned long long* __restrict__ hash) {
  unsigned long long hacc = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const T* x = xp + p * ldxp;
    int c[3] = {0, 0, 0};
    T f;
    bool ok = true;
    for (int a = 0; a < kp.dim; ++a) ok = ok && cell_axis<T>(kp, a, x[a], c[a], f);
    if (hash) hacc += particle_hash<T>(x, kp.dim, p);
    int k = -1;
    if (ok) {
      k = c[0] + kp.N[0] * (c[1] + kp.N[1] * c[2]);
      slot[p] = atomicAdd(&count[k], 1);
    } else {
      atomicAdd(err, 1);
      if (zout)
        for (int a = 0; a < nz; ++a) zout[p * ldz + a] = T(0);
    }
    key[p] = k;
  }
  if (hash) block_add_hash(hacc, hash);
}

template <class T>
__global__ void k_hash(const T* __restrict__ xp, int64_t ldxp, int64_t np, int dim,
                       unsigned long long* __restrict__ hash) {
  unsigned long long hacc = 0;
  // unrolled: the loads of several particles are in flight at once
#pragma unroll 4
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x)
    hacc += particle_hash<T>(xp + p * ldxp, dim, p);
  block_add_hash(hacc, hash);
}

// The same fingerprint for 3D FP64 positions packed three to a row (ldxp 3)
// at a 16-byte aligned base: each thread reads particles 2q and 2q+1 as
// three 16-byte streaming loads; a last odd particle is read alone.
__global__ void k_hash_xyz_pairs(const double* __restrict__ xp, int64_t np,
                                 unsigned long long* __restrict__ hash) {
  unsigned long long hacc = 0;
  const int64_t npair = np / 2;
  const double2* v = reinterpret_cast<const double2*>(xp);
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npair;
       q += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = __ldcs(v + 3 * q), b = __ldcs(v + 3 * q + 1), c = __ldcs(v + 3 * q + 2);
    const double x0[3] = {a.x, a.y, b.x}, x1[3] = {b.y, c.x, c.y};
    hacc += particle_hash<double>(x0, 3, 2 * q) + particle_hash<double>(x1, 3, 2 * q + 1);
  }
  if ((np & 1) && blockIdx.x == 0 && threadIdx.x == 0)
    hacc += particle_hash<double>(xp + 3 * (np - 1), 3, np - 1);
  block_add_hash(hacc, hash);
}

__global__ void k_scatter(const int* __restrict__ key, const int* __restrict__ slot,
                          const int* __restrict__ start, int64_t np, int* __restrict__ idx) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    int k = key[p];
    if (k >= 0) idx[start[k] + slot[p]] = (int)p;
  }
}

// Sort each cell's ids ascending: insertion sort for small cells, big cells
// are queued for a block-cooperative rank sort.
__global__ void k_segsort_small(const int* __restrict__ start, int64_t ncell, int* idx,
                                int* big, int bigcap) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    int b = start[c], e = start[c + 1];
    int n = e - b;
    if (n <= 1) continue;
    if (n > kSmallCell) {
      int q = atomicAdd(&big[0], 1);
      if (q < bigcap) {
        big[1 + q] = (int)c;
        continue;
      }
      atomicSub(&big[0], 1);  // queue full: sort it here (correct, slower)
    }
    int* a = idx + b;
    for (int i = 1; i < n; ++i) {
      int v = a[i];
      int j = i - 1;
      while (j >= 0 && a[j] > v) {
        a[j + 1] = a[j];
        --j;
      }
      a[j + 1] = v;
    }
  }
}

__global__ void k_segsort_big(const int* __restrict__ start, const int* __restrict__ big,
                              int bigcap, int* idx, int* tmp) {
  const int nbig = min(big[0], bigcap);
  for (int q = blockIdx.x; q < nbig; q += gridDim.x) {
    const int c = big[1 + q];
    const int b = start[c], e = start[c + 1];
    const int n = e - b;
    // ids are distinct: rank = number of smaller ids
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      int v = idx[b + j];
      int r = 0;
      for (int i = 0; i < n; ++i) r += idx[b + i] < v;
      tmp[b + r] = v;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) idx[b + j] = tmp[b + j];
    __syncthreads();
  }
}

int grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

cudaError_t sort_tail(int64_t np, int64_t ncell, Workspace& ws, cudaStream_t st) {
  // count -> start (exclusive scan of ncell+1 entries; count[ncell] == 0)
  cudaError_t e = scan_exclusive(ws.count.as<int>(), ws.start.as<int>(), ncell + 1, ws, st);
  if (e != cudaSuccess) return e;
  k_scatter<<<grid_for(np, 256), 256, 0, st>>>(ws.key.as<int>(), ws.slot.as<int>(),
                                               ws.start.as<int>(), np, ws.idx.as<int>());
  count_launch();
  if ((e = cudaMemsetAsync(ws.big.as<int>(), 0, sizeof(int), st)) != cudaSuccess) return e;
  const int bigcap = (int)(ws.big.bytes / sizeof(int)) - 2;
  k_segsort_small<<<grid_for(ncell, 256), 256, 0, st>>>(ws.start.as<int>(), ncell,
                                                        ws.idx.as<int>(), ws.big.as<int>(),
                                                        bigcap);
  k_segsort_big<<<148, 256, 0, st>>>(ws.start.as<int>(), ws.big.as<int>(), bigcap,
                                     ws.idx.as<int>(), ws.slot.as<int>());
  count_launch(2);
  return cudaGetLastError();
}

}  // namespace

cudaError_t scan_exclusive(const int* in, int* out, int64_t n, Workspace& ws,
                           cudaStream_t st) {
  const int64_t nb64 = (n + kScanTile - 1) / kScanTile;
  const int nb = (int)(nb64 < 1 ? 1 : nb64);
  cudaError_t e = ws.bsum.ensure(sizeof(int) * (size_t)(nb + 1));
  if (e != cudaSuccess) return e;
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, n, ws.bsum.as<int>());
  k_scan_bsum<<<1, 1024, 0, st>>>(ws.bsum.as<int>(), nb);
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, out, n, ws.bsum.as<int>());
  count_launch(3);
  return cudaGetLastError();
}

template <class T>
cudaError_t bin_sort(const KeyParams& kp, const T* xp, int64_t ldxp, int64_t np,
                     int64_t ncell, Workspace& ws, int* err_counter, cudaStream_t st,
                     T* zout, int64_t ldz, int nz, unsigned long long* hash) {
  cudaError_t e;
  const size_t pn = sizeof(int) * (size_t)(np > 0 ? np : 1);
  if ((e = ws.key.ensure(pn)) || (e = ws.slot.ensure(pn)) || (e = ws.idx.ensure(pn)) ||
      (e = ws.count.ensure(sizeof(int) * (size_t)(ncell + 1))) ||
      (e = ws.start.ensure(sizeof(int) * (size_t)(ncell + 1))) ||
      (e = ws.err.ensure(sizeof(int) * 4)) ||
      (e = ws.big.ensure(sizeof(int) * (size_t)(ncell + 1 < 1 << 20 ? ncell + 2 : (1 << 20) + 2))))
    return e;
  if ((e = cudaMemsetAsync(ws.count.p, 0, sizeof(int) * (size_t)(ncell + 1), st))) return e;
  if (hash && (e = cudaMemsetAsync(hash, 0, sizeof(unsigned long long), st))) return e;
  if (np > 0) {
    k_bin<T><<<grid_for(np, 256), 256, 0, st>>>(kp, xp, ldxp, np, ws.key.as<int>(),
                                                ws.slot.as<int>(), ws.count.as<int>(),
                                                err_counter, zout, ldz, nz, hash);
    count_launch();
  }
  return sort_tail(np, ncell, ws, st);
}

template cudaError_t bin_sort<double>(const KeyParams&, const double*, int64_t, int64_t,
                                      int64_t, Workspace&, int*, cudaStream_t, double*,
                                      int64_t, int, unsigned long long*);
template cudaError_t bin_sort<float>(const KeyParams&, const float*, int64_t, int64_t,
                                     int64_t, Workspace&, int*, cudaStream_t, float*, int64_t,
                                     int, unsigned long long*);

template <class T>
cudaError_t position_hash(const T* xp, int64_t ldxp, int64_t np, int dim,
                          unsigned long long* hash, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(hash, 0, sizeof(unsigned long long), st);
  if (e) return e;
  if (np > 0) {
    if (sizeof(T) == 8 && dim == 3 && ldxp == 3 && (reinterpret_cast<uintptr_t>(xp) & 15) == 0)
      k_hash_xyz_pairs<<<grid_for((np + 1) / 2, 256), 256, 0, st>>>(
          reinterpret_cast<const double*>(xp), np, hash);
    else
      k_hash<T><<<grid_for(np, 256), 256, 0, st>>>(xp, ldxp, np, dim, hash);
    count_launch();
  }
  return cudaGetLastError();
}
template cudaError_t position_hash<double>(const double*, int64_t, int64_t, int,
                                           unsigned long long*, cudaStream_t);
template cudaError_t position_hash<float>(const float*, int64_t, int64_t, int,
                                          unsigned long long*, cudaStream_t);

// ---------------------------------------------------------------------------
// Sorted records
// ---------------------------------------------------------------------------
namespace {

template <class T, class CT>
__global__ void k_pack(KeyParams kp, const T* __restrict__ xp, int64_t ldxp,
                       const T* __restrict__ up, int64_t ldup, int lda, int nchunk,
                       int64_t np, const int* __restrict__ d_nvalid,
                       const int* __restrict__ idx,
                       typename Vec4<CT>::type* __restrict__ rec,
                       typename Vec4<CT>::type* __restrict__ us) {
  using V = typename Vec4<CT>::type;
  const int64_t nvalid = min(np, (int64_t)*d_nvalid);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nvalid;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx[s];
    const T* x = xp + p * ldxp;
    int c[3] = {0, 0, 0};
    T f[3] = {T(0), T(0), T(0)};
    for (int a = 0; a < kp.dim; ++a) cell_axis<T>(kp, a, x[a], c[a], f[a]);
    const int cell = c[0] + kp.N[0] * (c[1] + kp.N[1] * c[2]);
    V r;
    r.x = (CT)f[0];
    r.y = (CT)f[1];
    r.z = (CT)f[2];
    if constexpr (sizeof(CT) == 4)
      r.w = __int_as_float(cell);
    else
      r.w = (double)cell;
    store_vec(rec, s, np, r);
    const T* u = up + p * ldup;
    for (int ch = 0; ch < nchunk; ++ch) {
      CT v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int a = ch * 4 + q;
        v[q] = a < lda ? (CT)u[a] : CT(0);
      }
      V w;
      w.x = v[0];
      w.y = v[1];
      w.z = v[2];
      w.w = v[3];
      store_vec(us + (int64_t)ch * np, s, np, w);
    }
  }
}

}  // namespace

template <class T, class CT>
cudaError_t pack_records(const KeyParams& kp, const T* xp, int64_t ldxp, const T* up,
                         int64_t ldup, int lda, int64_t np, const int* d_nvalid,
                         Workspace& ws, cudaStream_t st) {
  using V = typename Vec4<CT>::type;
  const int nchunk = up ? (lda + 3) / 4 : 0;
  cudaError_t e;
  const size_t n = (size_t)(np > 0 ? np : 1);
  if ((e = ws.rec.ensure(sizeof(V) * n))) return e;
  if ((e = ws.us.ensure(sizeof(V) * n * (size_t)(nchunk > 0 ? nchunk : 1)))) return e;
  if (np > 0) {
    k_pack<T, CT><<<grid_for(np, 256), 256, 0, st>>>(kp, xp, ldxp, up, ldup, lda, nchunk, np,
                                                     d_nvalid, ws.idx.as<int>(),
                                                     ws.rec.as<V>(), ws.us.as<V>());
    count_launch();
  }
  return cudaGetLastError();
}

template cudaError_t pack_records<double, double>(const KeyParams&, const double*, int64_t,
                                                  const double*, int64_t, int, int64_t,
                                                  const int*, Workspace&, cudaStream_t);
template cudaError_t pack_records<double, float>(const KeyParams&, const double*, int64_t,
                                                 const double*, int64_t, int, int64_t,
                                                 const int*, Workspace&, cudaStream_t);
template cudaError_t pack_records<float, float>(const KeyParams&, const float*, int64_t,
                                                const float*, int64_t, int, int64_t,
                                                const int*, Workspace&, cudaStream_t);

// ---------------------------------------------------------------------------
// Cell-list ranking, ppm_util_rank3d.f:353-533 / ppm_util_rank2d.f
// ---------------------------------------------------------------------------
namespace {

template <class T>
__global__ void k_clist_bin(ClistParams cp, const T* __restrict__ xp, int64_t ldxp,
                            int64_t np, int* __restrict__ key, int* __restrict__ slot,
                            int* __restrict__ count, int* __restrict__ nin) {
  constexpr bool F = sizeof(T) == 4;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const T* x = xp + p * ldxp;
    int c[3] = {0, 0, 0};
    for (int a = 0; a < cp.dim; ++a) {
      // FLOOR((x - x0) * rdx) + Ngl in REAL(MK): the subtraction first
      // (ppm_util_rank3d.f:353-425)
      const T x0 = F ? (T)cp.xminf[a] : (T)cp.xmin[a];
      const T rd = F ? (T)cp.rdf[a] : (T)cp.rd[a];
      const T xm = F ? (T)cp.xmaxf[a] : (T)cp.xmax[a];
      c[a] = (int)floor(rmul(rsub(x[a], x0), rd)) + cp.Ngl[a];
      if (x[a] >= xm && c[a] < cp.Nm[a] + cp.Ngl[a]) c[a] = cp.Nm[a] + cp.Ngl[a];
    }
    for (int a = 0; a < cp.dim; ++a) {
      const T xm = F ? (T)cp.xmaxf[a] : (T)cp.xmax[a];
      if (x[a] < xm && c[a] >= cp.Nm[a] + cp.Ngl[a]) c[a] = cp.Nm[a] + cp.Ngl[a] - 1;
    }
    bool in = true;
    for (int a = 0; a < cp.dim; ++a) in = in && c[a] >= 0 && c[a] < cp.Nt[a];
    int k = -1;
    if (in) {
      k = c[0] + cp.Nt[0] * (c[1] + (cp.dim == 3 ? cp.Nt[1] * c[2] : 0));
      slot[p] = atomicAdd(&count[k], 1);
      atomicAdd(nin, 1);
    }
    key[p] = k;
  }
}

}  // namespace

template <class T>
cudaError_t clist_sort(const ClistParams& cp, const T* xp, int64_t ldxp, int64_t np,
                       int64_t nbox, Workspace& ws, cudaStream_t st) {
  cudaError_t e;
  const size_t pn = sizeof(int) * (size_t)(np > 0 ? np : 1);
  if ((e = ws.key.ensure(pn)) || (e = ws.slot.ensure(pn)) || (e = ws.idx.ensure(pn)) ||
      (e = ws.count.ensure(sizeof(int) * (size_t)(nbox + 1))) ||
      (e = ws.start.ensure(sizeof(int) * (size_t)(nbox + 1))) ||
      (e = ws.err.ensure(sizeof(int) * 4)) ||
      (e = ws.big.ensure(sizeof(int) * (size_t)(nbox + 1 < 1 << 20 ? nbox + 2 : (1 << 20) + 2))))
    return e;
  if ((e = cudaMemsetAsync(ws.count.p, 0, sizeof(int) * (size_t)(nbox + 1), st))) return e;
  if ((e = cudaMemsetAsync(ws.err.p, 0, sizeof(int) * 4, st))) return e;
  if (np > 0) {
    k_clist_bin<T><<<grid_for(np, 256), 256, 0, st>>>(cp, xp, ldxp, np, ws.key.as<int>(),
                                                      ws.slot.as<int>(), ws.count.as<int>(),
                                                      ws.err.as<int>());
    count_launch();
  }
  return sort_tail(np, nbox, ws, st);
}
template cudaError_t clist_sort<double>(const ClistParams&, const double*, int64_t, int64_t,
                                        int64_t, Workspace&, cudaStream_t);
template cudaError_t clist_sort<float>(const ClistParams&, const float*, int64_t, int64_t,
                                       int64_t, Workspace&, cudaStream_t);

}  // namespace ppmg
