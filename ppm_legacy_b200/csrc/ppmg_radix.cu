// ppmg_radix.cu -- stable LSD radix sort of particles into cell order, with
// their packed records and strengths placed in that order (declared in
// ppmg_sort.cuh).
//
// The counting sort of ppmg_sort.cu scatters particle ids to random cell
// slots and then gathers every particle's position and strengths from random
// addresses; on large unordered particle sets those random accesses, not the
// arithmetic, set its time.  Here every pass reads its input in order and
// writes it grouped by one digit of the cell key: a sub-tile of 4096
// particles is ranked in shared memory and leaves as runs of equal digit, so
// both the reads and the writes are coalesced.  The first count pass builds
// the keys from xp and writes each particle's record and strengths as one
// row of 16-byte units (32 bytes in the mixed form); the passes move only
// (key, id), and one gather then copies every row into the sorted planes.
// A random row read costs DRAM about 128 bytes, yet carrying the 32-64 byte
// payload through every pass cost more than that single random read.
// The sort is stable and starts from particle-id order, so particles of one
// cell end in ascending id -- the fill order of ppm_util_rank3d.f:525-533.
#include <cuda_runtime.h>

#include "ppmg_sort.cuh"
#include "ppmg_sort_dev.cuh"

namespace ppmg {
namespace {

constexpr int kCThreads = 512;                  // count kernel (full occupancy in one wave)
constexpr int kRThreads = 512;                  // move kernel (two CTAs per SM)
constexpr int kRWarps = kRThreads / 32;
constexpr int kRItems = 8;                      // items per thread and sub-tile
constexpr int kRSub = kRThreads * kRItems;      // 4096 items per sub-tile
constexpr int kRWarpItems = kRSub / kRWarps;    // 256 consecutive items per warp
constexpr int kRMaxBits = 9;                    // >= 8 items per digit and sub-tile
constexpr int kRMaxBuckets = 1 << kRMaxBits;
constexpr int kRSlots = kRMaxBuckets + 32;      // + the invalid bucket of the first pass
constexpr int kRDigitsPerThread = (kRMaxBuckets + 1 + kRThreads - 1) / kRThreads;
constexpr int kRGapRun = 64;                    // longer runs of empty cells: k_fill_gaps
constexpr int kRWaitLimit = 1 << 22;            // mbarrier polls before a unit is given up

// Cell key of one particle (ncell when it has no cell) and its offsets.
template <class T>
__device__ __forceinline__ int particle_key(const KeyParams& kp, const T* x, int ncell,
                                            T f[3]) {
  int c[3] = {0, 0, 0};
  f[0] = f[1] = f[2] = T(0);
  bool ok = true;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (a < kp.dim) ok = ok && cell_axis<T>(kp, a, x[a], c[a], f[a]);
  return ok ? c[0] + kp.N[0] * (c[1] + kp.N[1] * c[2]) : ncell;
}

template <class T, class CT>
struct CountArgs {
  using V = typename Vec4<CT>::type;
  KeyParams kp;
  const T* xp;
  int64_t ldxp;
  const T* up;
  int64_t ldup;
  int lda, nchunk;
  int64_t np;
  const int* d_nvalid;  // later passes: items [0, *d_nvalid) are sorted
  int ncell, shift, bits, subs, ntiles;
  const int* key_in;
  int* hist;  // [digit * ntiles + tile]
  // first pass: keys in particle order, and every particle's record and
  // strength units side by side (iu 16-byte units per particle)
  int* key0;
  uint4* aos;
  int iu;
  int* err;
  T* zout;
  int64_t ldz;
  int nz;
  unsigned long long* hash;
  const int* unsorted;  // 0: the first pass found the keys in order (later passes skip)
};

// Digit of a key; in the first pass invalid particles (key ncell) take the
// extra bucket nb, which sorts them behind all valid ones.
template <bool FIRST>
__device__ __forceinline__ int digit_of(int k, int shift, unsigned mask, int nb, int ncell) {
  if (FIRST && k == ncell) return nb;
  return (int)(((unsigned)k >> shift) & mask);
}

template <class T, class CT>
__device__ __forceinline__ typename Vec4<CT>::type make_us(const T* u, int lda, int ch) {
  CT v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int a = ch * 4 + q;
    v[q] = a < lda ? (CT)u[a] : CT(0);
  }
  typename Vec4<CT>::type w;
  w.x = v[0];
  w.y = v[1];
  w.z = v[2];
  w.w = v[3];
  return w;
}

// A float4 / double4 as its 16-byte units (streaming stores: the units are
// read back once, in sorted order, by k_gather_units).
template <class V>
__device__ __forceinline__ void store_units(uint4* dst, const V& v) {
  const uint4* u = reinterpret_cast<const uint4*>(&v);
#pragma unroll
  for (int t = 0; t < (int)(sizeof(V) / 16); ++t) __stcs(dst + t, u[t]);
}

// Digit histogram of each tile (subs sub-tiles of consecutive items).  The
// first pass computes the keys from the positions, writes the keys and each
// particle's record and strength units in particle order, counts invalid
// particles, zeroes their output rows and accumulates the position
// fingerprint.
template <class T, class CT, bool FIRST>
__global__ void __launch_bounds__(kCThreads) k_radix_count(CountArgs<T, CT> A) {
  using V = typename Vec4<CT>::type;
  __shared__ int sh[kRSlots];
  const int nb = 1 << A.bits;
  const int nbk = FIRST ? nb + 1 : nb;
  const unsigned mask = (unsigned)nb - 1u;
  for (int d = threadIdx.x; d < nbk; d += kCThreads) sh[d] = 0;
  __syncthreads();
  if (!FIRST && *A.unsorted == 0) return;  // keys already in order: nothing to count
  const int64_t n = FIRST ? A.np : (int64_t)*A.d_nvalid;
  const int64_t t0 = (int64_t)blockIdx.x * A.subs * kRSub;
  const int64_t t1 = min(n, t0 + (int64_t)A.subs * kRSub);
  unsigned long long hacc = 0;
  for (int64_t i = t0 + threadIdx.x; i < t1; i += kCThreads) {
    int k;
    if constexpr (FIRST) {
      const T* x = A.xp + i * A.ldxp;
      T f[3];
      k = particle_key<T>(A.kp, x, A.ncell, f);
      if (A.hash) hacc += particle_hash<T>(x, A.kp.dim, i);
      if (k == A.ncell) {
        atomicAdd(A.err, 1);
        if (A.zout)
          for (int a = 0; a < A.nz; ++a) A.zout[i * A.ldz + a] = T(0);
      }
      A.key0[i] = k;
      V r;
      r.x = (CT)f[0];
      r.y = (CT)f[1];
      r.z = (CT)f[2];
      if constexpr (sizeof(CT) == 4)
        r.w = __int_as_float(k);
      else
        r.w = (double)k;
      constexpr int RU = (int)(sizeof(V) / 16);
      uint4* row = A.aos + i * A.iu;
      store_units(row, r);
      for (int ch = 0; ch < A.nchunk; ++ch)
        store_units(row + RU * (1 + ch), make_us<T, CT>(A.up + i * A.ldup, A.lda, ch));
    } else {
      k = A.key_in[i];
    }
    atomicAdd(&sh[digit_of<FIRST>(k, A.shift, mask, nb, A.ncell)], 1);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < nbk; d += kCThreads)
    A.hist[(int64_t)d * A.ntiles + blockIdx.x] = sh[d];
  if (FIRST && A.hash) block_add_hash(hacc, A.hash);
}

struct MoveArgs {
  int64_t np;     // items of the first pass
  int* d_nvalid;  // written by the first pass, read by the later ones
  int ncell, shift, bits, subs, ntiles;
  const int* hist;  // exclusive-scanned, [digit * ntiles + tile]
  const int* key_in;
  const int* id_in;  // not read by the first pass (ids = item positions)
  int* key_out;
  int* id_out;
  int* wait_flag;  // set when a bulk copy never completes
  const int* unsorted;  // 0: the first pass found the keys in order (the passes skip)
};

// Shared memory of k_radix_move: two key and two id buffers (kRSub entries
// each), the 16-bit inverse map and per-warp digit counts, the per-digit
// offsets and the mbarriers (~98 KB: two CTAs of 16 warps per SM, so one
// CTA's ranking overlaps the other's barriers and stores).
constexpr size_t kMoveSmem = 4 * sizeof(int) * (size_t)kRSub +
                             sizeof(unsigned short) * (size_t)(kRSub + kRWarps * kRSlots) +
                             sizeof(int) * (size_t)(3 * kRSlots + 64) + 4 * sizeof(uint64_t);

// One stable pass over (key, id) pairs.  Every tile walks its sub-tiles in
// order.  The keys and the ids of a sub-tile arrive by TMA bulk copies issued
// two sub-tiles ahead into double buffers (the first pass reads no ids: they
// are the item positions), each completing on its own mbarrier.  The keys are
// ranked by digit (warp w owns items [kRWarpItems w, kRWarpItems (w+1)),
// ranked round by round with one ballot per digit bit); inv[] maps every
// sorted position of the sub-tile to its item, so keys and ids leave in digit
// runs.
template <bool FIRST>
__global__ void __launch_bounds__(kRThreads, 2) k_radix_move(MoveArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  int* kb = reinterpret_cast<int*>(smem);                             // [2][kRSub] keys
  int* ib = kb + 2 * kRSub;                                           // [2][kRSub] ids
  unsigned short* inv = reinterpret_cast<unsigned short*>(ib + 2 * kRSub);  // [kRSub]
  unsigned short* whist = inv + kRSub;                                // [kRWarps][kRSlots]
  int* run = reinterpret_cast<int*>(whist + kRWarps * kRSlots);       // next output slot per digit
  int* dst = run + kRSlots;                                           // digit start in the sub-tile
  int* tot = dst + kRSlots;                                           // digit count of the sub-tile
  int* sw = tot + kRSlots;                                            // block scan scratch [33]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sw + 64);               // [0,1] keys, [2,3] ids

  const int nb = 1 << A.bits;
  const int nbk = FIRST ? nb + 1 : nb;
  const unsigned mask = (unsigned)nb - 1u;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int w = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  unsigned short* wh = whist + w * kRSlots;
  const int dbits = A.bits + (FIRST ? 1 : 0);  // the first pass has the invalid bucket nb

  const int64_t n = FIRST ? A.np : (int64_t)*A.d_nvalid;
  if (FIRST && blockIdx.x == 0 && tid == 0)
    *A.d_nvalid = A.hist[(int64_t)nb * A.ntiles];  // start of the invalid bucket
  if (*A.unsorted == 0) return;  // keys already in order: k_sorted_finish takes over
  const int64_t t0 = (int64_t)blockIdx.x * A.subs * kRSub;
  if (t0 >= n) return;
  const int nsc = (int)min((int64_t)A.subs, (n - t0 + kRSub - 1) / kRSub);

  for (int d = tid; d < nbk; d += kRThreads) run[d] = A.hist[(int64_t)d * A.ntiles + blockIdx.x];
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) mbar_init(&bar[i]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto sub_n = [&](int sub) { return (int)min((int64_t)kRSub, n - (t0 + (int64_t)sub * kRSub)); };
  // keys (and ids) of sub-tile s into buffer s & 1, rounded up to 16 bytes
  // (the key and id arrays are allocated 16 entries long)
  auto issue = [&](int s) {
    if (s >= nsc) return;
    const int64_t base = t0 + (int64_t)s * kRSub;
    const uint32_t bytes = (uint32_t)((sub_n(s) * 4 + 15) & ~15);
    mbar_expect_tx(&bar[s & 1], bytes);
    bulk_load(kb + (s & 1) * kRSub, A.key_in + base, bytes, &bar[s & 1]);
    if (!FIRST) {
      mbar_expect_tx(&bar[2 + (s & 1)], bytes);
      bulk_load(ib + (s & 1) * kRSub, A.id_in + base, bytes, &bar[2 + (s & 1)]);
    }
  };
  // every thread waits; all give up together (copies still outstanding are
  // waited for once more, with the same bound)
  auto wait_on = [&](uint64_t* br, int use) -> bool {
    const bool ok = mbar_wait(br, (uint32_t)((use >> 1) & 1), kRWaitLimit);
    if (__syncthreads_and(ok)) return true;
    if (tid == 0) atomicExch(A.wait_flag, 1);
    for (int i = 0; i < 4; ++i)
      mbar_wait(&bar[i], 0u, kRWaitLimit), mbar_wait(&bar[i], 1u, kRWaitLimit);
    return false;
  };

  if (tid == 0) {
    issue(0);
    issue(1);
  }
  for (int sub = 0; sub < nsc; ++sub) {
    const int64_t base = t0 + (int64_t)sub * kRSub;
    const int subn = sub_n(sub);
    if (!wait_on(&bar[sub & 1], sub)) return;
    const int* skeys = kb + (sub & 1) * kRSub;
    for (int d = lane; d < nbk; d += 32) wh[d] = 0;
    __syncwarp();
    int key[kRItems], lpos[kRItems];
#pragma unroll
    for (int r = 0; r < kRItems; ++r) {
      const int li = w * kRWarpItems + r * 32 + lane;
      const bool valid = li < subn;
      key[r] = valid ? skeys[li] : 0;
      const int d = valid ? digit_of<FIRST>(key[r], A.shift, mask, nb, A.ncell) : -1;
      // lanes holding the same digit, one ballot per digit bit (a match
      // instruction serialises over the distinct values of the warp)
      unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int b = 0; b <= kRMaxBits; ++b)
        if (b < dbits) {
          const bool bit = (d >> b) & 1;
          const unsigned m = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? m : ~m;
        }
      const int before = valid ? wh[d] : 0;
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) wh[d] = (unsigned short)(before + __popc(peers));
      __syncwarp();
      lpos[r] = valid ? before + __popc(peers & lt) : -1;
    }
    __syncthreads();
    // per digit: exclusive prefix over the warps and the sub-tile total
    for (int d = tid; d < nbk; d += kRThreads) {
      int s = 0;
#pragma unroll
      for (int ww = 0; ww < kRWarps; ++ww) {
        const int c = whist[ww * kRSlots + d];
        whist[ww * kRSlots + d] = (unsigned short)s;
        s += c;
      }
      tot[d] = s;
    }
    __syncthreads();
    {
      // digit starts inside the sub-tile: exclusive scan of tot
      int v[kRDigitsPerThread], sum = 0;
#pragma unroll
      for (int q = 0; q < kRDigitsPerThread; ++q) {
        const int d = tid * kRDigitsPerThread + q;
        v[q] = d < nbk ? tot[d] : 0;
        sum += v[q];
      }
      int tsum;
      int ex = block_excl_scan(sum, sw, tsum);
#pragma unroll
      for (int q = 0; q < kRDigitsPerThread; ++q) {
        const int d = tid * kRDigitsPerThread + q;
        if (d < nbk) dst[d] = ex;
        ex += v[q];
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRItems; ++r)
      if (lpos[r] >= 0) {
        const int d = digit_of<FIRST>(key[r], A.shift, mask, nb, A.ncell);
        inv[lpos[r] + dst[d] + wh[d]] = (unsigned short)(w * kRWarpItems + r * 32 + lane);
      }
    __syncthreads();  // inv[] complete
    // the ids of this sub-tile (later passes) must have landed
    if (!FIRST && !wait_on(&bar[2 + (sub & 1)], sub)) return;
    // keys and ids; thread t takes the sorted positions j = t + kRThreads q
    const int* sids = ib + (sub & 1) * kRSub;
#pragma unroll
    for (int q = 0; q < kRItems; ++q) {
      const int j = tid + q * kRThreads;
      if (j < subn) {
        const int li = inv[j];
        const int kk = skeys[li];
        const int d = digit_of<FIRST>(kk, A.shift, mask, nb, A.ncell);
        const int g = run[d] + (j - dst[d]);
        __stcs(A.key_out + g, kk);
        __stcs(A.id_out + g, FIRST ? (int)(base + li) : sids[li]);
      }
    }
    __syncthreads();
    for (int d = tid; d < nbk; d += kRThreads) run[d] += tot[d];
    if (tid == 0) issue(sub + 2);
  }
}

// start[c] = first sorted position whose key is >= c, for c in [0, ncell]
// (start[ncell] = the valid count): position s writes the cells between the
// previous key and its own; runs of more than kRGapRun empty cells go to a
// list that k_fill_gaps writes.
// Particles that arrive in cell order (those ppm_rmsh_create_part emits, or a
// caller that keeps its particles sorted) need no pass: *unsorted stays 0
// when no key of the first pass exceeds its successor (invalid particles,
// key ncell, then sit at the end already).
// Each thread checks four consecutive keys (one 16-byte load; the key arrays
// are 16-entry padded and 16-byte aligned) and the next group's first key.
__global__ void k_keys_sorted(const int* __restrict__ key, int64_t np, int* unsorted) {
  const int64_t ng = (np + 3) / 4;
  bool bad = false;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < ng;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int4 k = reinterpret_cast<const int4*>(key)[q];
    const int64_t i = 4 * q;
    const int v[4] = {k.x, k.y, k.z, k.w};
#pragma unroll
    for (int j = 0; j < 3; ++j) bad |= i + j + 1 < np && v[j] > v[j + 1];
    if (i + 4 < np) bad |= v[3] > key[i + 4];
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) *unsorted = 1;
}

// The sorted order of keys found in order: the keys as they are, identity ids.
__global__ void k_sorted_finish(const int* __restrict__ unsorted, const int* __restrict__ key0,
                                int64_t np, int* __restrict__ key, int* __restrict__ id) {
  if (*unsorted != 0) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (key != key0) key[i] = key0[i];
    id[i] = (int)i;
  }
}

__global__ void k_cell_starts(const int* __restrict__ key, const int* __restrict__ d_nvalid,
                              int ncell, int* __restrict__ start, int4* __restrict__ gaps,
                              int* __restrict__ ngaps, int gapcap) {
  const int64_t nv = *d_nvalid;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s <= nv;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int kprev = s > 0 ? key[s - 1] : -1;
    const int kcur = s < nv ? key[s] : ncell;
    const int c0 = kprev + 1;
    const int c1 = kcur;
    if (c1 < c0) continue;
    if (c1 - c0 < kRGapRun) {
      for (int c = c0; c <= c1; ++c) start[c] = (int)s;
    } else {
      const int g = atomicAdd(ngaps, 1);
      if (g < gapcap) gaps[g] = make_int4(c0, c1, (int)s, 0);
    }
  }
}

__global__ void k_fill_gaps(const int4* __restrict__ gaps, const int* __restrict__ ngaps,
                            int gapcap, int* __restrict__ start) {
  const int n = min(*ngaps, gapcap);
  for (int g = blockIdx.x; g < n; g += gridDim.x) {
    const int4 q = gaps[g];
    for (int c = q.x + threadIdx.x; c <= q.y; c += blockDim.x) start[c] = q.z;
  }
}

// Payload of the sorted order: sorted position s takes the units of particle
// ids[s] from its row of aos (IU units; in the mixed form with lda <= 4 a
// row is one 32-byte sector) into the planes, units 0 .. ru-1 to rec and the
// rest to us.  The lanes of one particle are adjacent, so a row costs one
// sector request and a warp's stores to a plane are contiguous.  Four units
// per thread are in flight at once (the reads land at random rows).
template <int IU>
__global__ void __launch_bounds__(256) k_gather_units(const int* __restrict__ ids,
                                                      const int* __restrict__ d_nvalid,
                                                      const uint4* __restrict__ aos, int iu_rt,
                                                      int ru, int64_t np, uint4* __restrict__ rec,
                                                      uint4* __restrict__ us) {
  constexpr int kU = 4;
  const int iu = IU > 0 ? IU : iu_rt;
  const int64_t n = (int64_t)*d_nvalid * iu;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g0 < n; g0 += kU * stride) {
    int64_t s[kU];
    int t[kU], id[kU];
#pragma unroll
    for (int k = 0; k < kU; ++k) {
      const int64_t g = g0 + k * stride;
      s[k] = g / iu;
      t[k] = (int)(g - s[k] * iu);
      id[k] = g < n ? __ldcs(ids + s[k]) : 0;
    }
    uint4 v[kU];
#pragma unroll
    for (int k = 0; k < kU; ++k)
      if (g0 + k * stride < n) v[k] = __ldcs(aos + (int64_t)id[k] * iu + t[k]);
#pragma unroll
    for (int k = 0; k < kU; ++k)
      if (g0 + k * stride < n) {
        uint4* dst = t[k] < ru ? rec + (int64_t)t[k] * np : us + (int64_t)(t[k] - ru) * np;
        __stcs(dst + s[k], v[k]);
      }
  }
}

int bit_length(int64_t v) {
  int b = 0;
  while (v > 0) {
    ++b;
    v >>= 1;
  }
  return b;
}

}  // namespace

template <class T, class CT>
cudaError_t radix_sort_records(const KeyParams& kp, const T* xp, int64_t ldxp, const T* up,
                               int64_t ldup, int lda, int64_t np, int64_t ncell,
                               Workspace& ws, int* err_counter, int* wait_flag, cudaStream_t st,
                               T* zout, int64_t ldz, int nz, unsigned long long* hash) {
  using V = typename Vec4<CT>::type;
  constexpr int RU = (int)(sizeof(V) / 16);
  const int nchunk = up ? (lda + 3) / 4 : 0;
  const int IU = RU * (1 + nchunk);  // 16-byte units per particle: record, strengths
  const size_t n = (size_t)(np > 0 ? np : 1);
  const size_t nus = n * (size_t)(nchunk > 0 ? nchunk : 1);
  const size_t nk = n + 16;  // bulk copies of keys round up to 16 bytes
  cudaError_t e;
  if ((e = ws.key.ensure(sizeof(int) * nk)) || (e = ws.key2.ensure(sizeof(int) * nk)) ||
      (e = ws.idx.ensure(sizeof(int) * nk)) || (e = ws.idx2.ensure(sizeof(int) * nk)) ||
      (e = ws.rec.ensure(sizeof(V) * n)) || (e = ws.rec2.ensure(sizeof(uint4) * n * IU)) ||
      (e = ws.us.ensure(sizeof(V) * nus)) ||
      (e = ws.start.ensure(sizeof(int) * (size_t)(ncell + 1))) ||
      (e = ws.err.ensure(sizeof(int) * 8)))
    return e;
  if (hash && (e = cudaMemsetAsync(hash, 0, sizeof(unsigned long long), st))) return e;
  if (np == 0) return cudaMemsetAsync(ws.start.p, 0, sizeof(int) * (size_t)(ncell + 1), st);
  TimingScope timed(kTimeSort, st);

  // digits of the valid keys [0, ncell); the first pass adds an invalid bucket
  const int nbits = ncell > 1 ? bit_length(ncell - 1) : 1;
  const int passes = (nbits + kRMaxBits - 1) / kRMaxBits;
  const int bits = (nbits + passes - 1) / passes;
  const int64_t nsub = (np + kRSub - 1) / kRSub;
  const int64_t want_tiles = 148 * 4;
  const int subs = (int)((nsub + want_tiles - 1) / want_tiles);
  const int ntiles = (int)((nsub + subs - 1) / subs);
  if ((e = ws.hist.ensure(sizeof(int) * (size_t)ntiles * (size_t)((1 << bits) + 1)))) return e;
  if ((e = cudaFuncSetAttribute(k_radix_move<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kMoveSmem)) ||
      (e = cudaFuncSetAttribute(k_radix_move<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kMoveSmem)))
    return e;
  int* d_nvalid = ws.err.as<int>() + 2;
  int* unsorted = ws.err.as<int>() + 4;
  if ((e = cudaMemsetAsync(unsorted, 0, sizeof(int), st))) return e;
  DevBuf* keys[2] = {&ws.key, &ws.key2};
  DevBuf* ids[2] = {&ws.idx, &ws.idx2};
  const int gk = (int)((np + 255) / 256 < 148 * 16 ? (np + 255) / 256 : 148 * 16);
  const int64_t g4 = ((np + 3) / 4 + 255) / 256;
  const int gk4 = (int)(g4 < 148 * 8 ? g4 : 148 * 8);
  for (int p = 0; p < passes; ++p) {
    const int shift = p * bits;
    const int pb = nbits - shift < bits ? nbits - shift : bits;
    const int nbk = p == 0 ? (1 << pb) + 1 : (1 << pb);
    const int out = (passes - 1 - p) & 1;  // the last pass writes set 0
    const int in = out ^ 1;
    CountArgs<T, CT> C{};
    C.kp = kp;
    C.xp = xp;
    C.ldxp = ldxp;
    C.up = up;
    C.ldup = ldup;
    C.lda = lda;
    C.nchunk = nchunk;
    C.np = np;
    C.d_nvalid = d_nvalid;
    C.ncell = (int)ncell;
    C.shift = shift;
    C.bits = pb;
    C.subs = subs;
    C.ntiles = ntiles;
    C.key_in = keys[in]->as<int>();
    C.hist = ws.hist.as<int>();
    C.key0 = keys[in]->as<int>();
    C.aos = ws.rec2.as<uint4>();
    C.iu = IU;
    C.err = err_counter;
    C.zout = zout;
    C.ldz = ldz;
    C.nz = nz;
    C.hash = hash;
    C.unsorted = unsorted;
    if (p == 0) {
      k_radix_count<T, CT, true><<<ntiles, kCThreads, 0, st>>>(C);
      k_keys_sorted<<<gk4, 256, 0, st>>>(keys[in]->as<int>(), np, unsorted);
      count_launch();
    } else {
      k_radix_count<T, CT, false><<<ntiles, kCThreads, 0, st>>>(C);
    }
    count_launch();
    if ((e = scan_exclusive(ws.hist.as<int>(), ws.hist.as<int>(), (int64_t)ntiles * nbk, ws,
                            st)))
      return e;
    MoveArgs M{};
    M.np = np;
    M.d_nvalid = d_nvalid;
    M.ncell = (int)ncell;
    M.shift = shift;
    M.bits = pb;
    M.subs = subs;
    M.ntiles = ntiles;
    M.hist = ws.hist.as<int>();
    M.key_in = keys[in]->as<int>();
    M.id_in = ids[in]->as<int>();
    M.key_out = keys[out]->as<int>();
    M.id_out = ids[out]->as<int>();
    M.wait_flag = wait_flag;
    M.unsorted = unsorted;
    if (p == 0)
      k_radix_move<true><<<ntiles, kRThreads, kMoveSmem, st>>>(M);
    else
      k_radix_move<false><<<ntiles, kRThreads, kMoveSmem, st>>>(M);
    count_launch();
  }
  // keys found in order: set 0 takes them as they are, with identity ids
  {
    const int first_in = ((passes - 1) & 1) ^ 1;  // the set the first pass read its keys into
    k_sorted_finish<<<gk, 256, 0, st>>>(unsorted, keys[first_in]->as<int>(), np,
                                        ws.key.as<int>(), ws.idx.as<int>());
    count_launch();
  }
  // records and strengths into the sorted order (the last pass wrote set 0)
  {
    const int64_t units = np * (int64_t)IU;
    const int64_t gb = (units + 256 * 4 - 1) / (256 * 4);
    const int grid = (int)(gb < 148 * 16 ? gb : 148 * 16);
    uint4* rec = ws.rec.as<uint4>();
    uint4* us = ws.us.as<uint4>();
    const uint4* aos = ws.rec2.as<uint4>();
    const int* sid = ws.idx.as<int>();
    switch (IU) {
      case 1: k_gather_units<1><<<grid, 256, 0, st>>>(sid, d_nvalid, aos, IU, RU, np, rec, us); break;
      case 2: k_gather_units<2><<<grid, 256, 0, st>>>(sid, d_nvalid, aos, IU, RU, np, rec, us); break;
      case 4: k_gather_units<4><<<grid, 256, 0, st>>>(sid, d_nvalid, aos, IU, RU, np, rec, us); break;
      default: k_gather_units<0><<<grid, 256, 0, st>>>(sid, d_nvalid, aos, IU, RU, np, rec, us); break;
    }
    count_launch();
  }
  // cell offsets from the sorted keys
  const int gapcap = (int)((ncell + 1) / (kRGapRun + 1) + 2);
  if ((e = ws.gaps.ensure(sizeof(int4) * (size_t)gapcap))) return e;
  if ((e = cudaMemsetAsync(ws.err.as<int>() + 3, 0, sizeof(int), st))) return e;
  const int64_t gs = (np + 1 + 255) / 256;
  k_cell_starts<<<(int)(gs < 148 * 16 ? gs : 148 * 16), 256, 0, st>>>(
      ws.key.as<int>(), d_nvalid, (int)ncell, ws.start.as<int>(), ws.gaps.as<int4>(),
      ws.err.as<int>() + 3, gapcap);
  k_fill_gaps<<<148 * 2, 256, 0, st>>>(ws.gaps.as<int4>(), ws.err.as<int>() + 3, gapcap,
                                       ws.start.as<int>());
  count_launch(2);
  return cudaGetLastError();
}

#define PPMG_RADIX_INST(T, CT)                                                              \
  template cudaError_t radix_sort_records<T, CT>(const KeyParams&, const T*, int64_t,      \
                                                 const T*, int64_t, int, int64_t, int64_t, \
                                                 Workspace&, int*, int*, cudaStream_t, T*, \
                                                 int64_t, int, unsigned long long*);
PPMG_RADIX_INST(double, double)
PPMG_RADIX_INST(double, float)
PPMG_RADIX_INST(float, float)
#undef PPMG_RADIX_INST

}  // namespace ppmg
