// ppmg_api.cu -- the C-ABI of libppmg (declared in include/ppmg.h): handle
// registry (the geometry state the reference keeps in ppm_module_data*),
// argument validation with the reference's info/errno conventions, and the
// host-pointer (synchronous) and device-pointer (stream-ordered) pipelines.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "ppmg_common.cuh"
#include "ppmg_m2p.cuh"
#include "ppmg_p2m.cuh"
#include "ppmg_rmsh.cuh"
#include "ppmg_map.cuh"
#include "ppmg_fd.cuh"
#include "ppmg_halo.cuh"
#include "ppmg_sort.cuh"

namespace ppmg {

std::atomic<int64_t> g_launches{0};

namespace {

struct ErrState {
  int info = 0;
  int errnum = 0;
  std::string msg;
};
thread_local ErrState t_err;

int initial_precision() {
  const char* e = std::getenv("PPMG_PRECISION");
  if (e && (std::strcmp(e, "mixed") == 0 || std::strcmp(e, "MIXED") == 0))
    return PPMG_PREC_MIXED;
  return PPMG_PREC_FP64;
}
std::atomic<int> g_precision{initial_precision()};

struct Handle {
  int topo_id = 0, mesh_id = 0;
  int dim = 0, nsubs = 0;
  int Nm[3] = {1, 1, 1};
  int bcdef[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> min_sub, max_sub;
  std::vector<int> subs_bc, istart, nnodes;
  // the subdomain this GPU computes on (ppm_isublist of one entry): -1 until
  // ppmg_mesh_set_local_sub when nsubs > 1
  int local_sub = 0;
  // cut axes: the local subdomain is one interval of several along them, not
  // periodic within it; the neighbouring subdomains own its ghost nodes
  bool open[3] = {false, false, false};
  int Nm_global[3] = {1, 1, 1};  // global nodes (Nm becomes the subdomain's)
  bool cut() const { return open[0] || open[1] || open[2]; }
  // slabs along z: the exchange moves whole planes (ppmg_halo_plan)
  bool slab() const { return open[2] && !open[0] && !open[1]; }
  // transport of the ghost exchange with the neighbouring slabs (caller's)
  ppmg_halo_fn halo_fn = nullptr;
  void* halo_ctx = nullptr;
  DevBuf halo_rbuf;                     // blocks received by a put (device)
  DevBuf halo_sbuf;                     // packed blocks to send (box exchange)
  DevBuf halo_tab;                      // box tables of the box exchange
  std::vector<int64_t> halo_tab_host;
  std::vector<unsigned char> halo_host;  // host staging of the host entry points
  Geom g{};
  Workspace ws;       // P2M / M2P / adjoint / ghost / clist scratch
  Workspace ws_rmsh;  // comp_weights -> remesh state (ppm_module_data_rmsh)
  Workspace ws_map;   // particle routing between slabs
  Workspace ws_fd;    // Poisson solver buffers
  FFTPlans fft;       // its cuFFT plans
  SlabFFTPlans fft_slab;  // the slab form's plans (z-slab handles, virtual slabs of cuts)
  DevBuf fd_slab;         // a cut's virtual z-slab of the field (the solve on cuts)
  cudaStream_t stream = nullptr;
  int* d_status = nullptr;  // [0] particles outside the sub, [1] non-finite
  // position fingerprints: [0] of the sort held in ws, [1] of an M2P's xp
  unsigned long long* d_hash = nullptr;
  unsigned long long* h_small = nullptr;  // pinned host copy (hashes + status)
  // The cell order, packed records and work items in `ws` belong to the
  // positions fingerprinted in d_hash[0]; an M2P of the same positions reuses
  // them (same key arithmetic: M2P's FP32 spacing equals P2M's spacing).
  bool sort_cached = false;
  int cache_prec = -1;        // record precision: 0 FP64 (double4), 1 FP32 (float4)
  bool cache_quirk = false;   // the sort's keys used M2P's FP32 mesh spacing
  int64_t cache_np = -1, cache_ldxp = -1;
  // ws.tiles holds work items of the tile gathers (M2P, adjoint) for the
  // cached sort (a P2M by the row gather leaves items of its own shape)
  bool items_m2p = false;
  bool dxi_same_d = false, dxi_same_f = false;
  std::mutex mu;
  // comp_weights state
  bool w_valid = false;
  bool w_single = false;  // the stored weights are FP32 (comp_weights_s)
  int w_kernel = 0;
  int64_t w_np = 0;
  ~Handle() {
    fft.release();
    fft_slab.release();
    if (stream) cudaStreamDestroy(stream);
    if (d_status) cudaFree(d_status);
    if (d_hash) cudaFree(d_hash);
    if (h_small) cudaFreeHost(h_small);
  }
};

// Heap-allocated and never destroyed: handle destructors call into the CUDA
// runtime, which must not happen from static destructors at process exit.
std::mutex g_mu;
std::map<std::pair<int, int>, std::unique_ptr<Handle>>& handles() {
  static auto* m = new std::map<std::pair<int, int>, std::unique_ptr<Handle>>();
  return *m;
}

int fail(int* info, int sev, int errnum, const std::string& msg) {
  set_error(sev, errnum, msg);
  if (info) *info = sev;
  return sev;
}

int cuda_fail(int* info, cudaError_t e, const char* where) {
  const int errnum = e == cudaErrorMemoryAllocation ? kErrAlloc : 602;
  std::string m = std::string(where) + ": CUDA error: " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky launch error of this thread
  return fail(info, kErrorFatal, errnum, m);
}

Handle* find_handle(int topo_id, int mesh_id) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = handles().find({topo_id, mesh_id});
  return it == handles().end() ? nullptr : it->second.get();
}

// Checks shared by every hot-path entry point (the ppm_debug > 0 checks of
// ppm_interp_p2m.f:338-410, always on here).
Handle* get_checked(int topo_id, int mesh_id, int dim, const char* caller, int* info,
                    bool sub_ok = false) {
  Handle* h = find_handle(topo_id, mesh_id);
  if (!h) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid");
    return nullptr;
  }
  if (h->dim != dim) {
    fail(info, kErrorError, kErrArgument,
         std::string(caller) + ": routine dimension does not match the registered mesh");
    return nullptr;
  }
  if (h->local_sub < 0) {
    fail(info, kErrorError, kErrArgument,
         std::string(caller) +
             ": nsubs > 1: select this GPU's subdomain with ppmg_mesh_set_local_sub");
    return nullptr;
  }
  if (h->cut() && !sub_ok) {
    fail(info, kErrorError, kErrArgument,
         std::string(caller) +
             ": a subdomain of several is supported by the 3D P2M, M2P, adjoint, remeshing and "
             "ghost mapping; this routine needs one periodic subdomain per GPU");
    return nullptr;
  }
  for (int f = 0; f < 2 * dim; ++f)
    if (h->bcdef[f] != kBcPeriodic) {
      fail(info, kErrorError, kErrArgument,
           std::string(caller) + ": only periodic boundary conditions are supported");
      return nullptr;
    }
  return h;
}

bool check_kernel(int kernel, const char* caller, int* info) {
  if (kernel != kKernelMp4 && kernel != kKernelBsp2) {
    fail(info, kErrorError, kErrArgument,
         std::string(caller) + ": wrong kernel definition (only M'4 = 2 and bsp2 = 1)");
    return false;
  }
  return true;
}

// field_up(ldf, lb:ub, ...) descriptor; `need_lo/hi` is the index box the
// routine touches.  Returns false (info set) when the allocation is too small.
bool make_fd(const Handle& h, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
             const int need_lo[3], const int need_hi[3], FieldDesc& fd, const char* caller,
             int* info) {
  int64_t s = ldf;
  for (int a = 0; a < 3; ++a) {
    fd.s[a] = 0;
    fd.lb[a] = 0;
    fd.ub[a] = 0;
    fd.box_lo[a] = 0;
    fd.box_hi[a] = 0;
  }
  for (int a = 0; a < h.dim; ++a) {
    if (f_ub[a] < f_lb[a]) {
      fail(info, kErrorError, kErrArgument, std::string(caller) + ": field bounds are empty");
      return false;
    }
    fd.s[a] = s;
    fd.lb[a] = (int)f_lb[a];
    fd.ub[a] = (int)f_ub[a];
    fd.box_lo[a] = need_lo[a];
    fd.box_hi[a] = need_hi[a];
    if (f_lb[a] > need_lo[a] || f_ub[a] < need_hi[a]) {
      fail(info, kErrorError, kErrArgument,
           std::string(caller) + ": field_up bounds do not cover the required index box");
      return false;
    }
    s *= (f_ub[a] - f_lb[a] + 1);
  }
  return true;
}

int64_t field_elems(const Handle& h, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub) {
  int64_t n = ldf;
  for (int a = 0; a < h.dim; ++a) n *= (f_ub[a] - f_lb[a] + 1);
  return n;
}

KeyParams make_kp(const Handle& h, int mode, bool quirk) {
  KeyParams kp{};
  kp.dim = h.dim;
  kp.mode = mode;
  for (int a = 0; a < 3; ++a) {
    kp.N[a] = a < h.dim ? h.g.N[a] : 1;
    kp.min[a] = a < h.dim ? h.g.min_sub[a] : 0.0;
    kp.max[a] = a < h.dim ? h.g.max_sub[a] : 1.0;
    kp.dxi[a] = a < h.dim ? (quirk ? h.g.dxiq_d[a] : h.g.dxi_d[a]) : 1.0;
    kp.minf[a] = (float)kp.min[a];
    kp.maxf[a] = (float)kp.max[a];
    kp.dxif[a] = a < h.dim ? (quirk ? h.g.dxiq_f[a] : h.g.dxi_f[a]) : 1.0f;
    kp.open[a] = h.open[a] ? 1 : 0;
  }
  return kp;
}

const int* d_nvalid_of(const Workspace& ws, int64_t ncell) {
  return ws.start.as<int>() + ncell;
}

template <class T>
constexpr bool is_f32() { return sizeof(T) == 4; }

// Cell-order sort of the interpolation entry points into h.ws: radix sort
// with the records (FP64 or FP32) and, for P2M, the strengths as payload.
template <class T>
cudaError_t sort_interp(Handle& h, const KeyParams& kp, const T* xp, int64_t ldxp, const T* up,
                        int64_t ldup, int lda, int64_t Np, bool fp64_rec, int* err, T* zout,
                        int64_t ldz, int nz, cudaStream_t st) {
  unsigned long long* hash = h.d_hash + 0;
  int* wflag = h.d_status + 2;
  if constexpr (is_f32<T>()) {
    return radix_sort_records<T, float>(kp, xp, ldxp, up, ldup, lda, Np, h.g.ncell, h.ws, err,
                                        wflag, st, zout, ldz, nz, hash);
  } else {
    if (fp64_rec)
      return radix_sort_records<T, double>(kp, xp, ldxp, up, ldup, lda, Np, h.g.ncell, h.ws,
                                           err, wflag, st, zout, ldz, nz, hash);
    return radix_sort_records<T, float>(kp, xp, ldxp, up, ldup, lda, Np, h.g.ncell, h.ws, err,
                                        wflag, st, zout, ldz, nz, hash);
  }
}

// ---------------------------------------------------------------------------
// P2M pipeline (stream-ordered).  Returns 0 or the argument-error info.
// ---------------------------------------------------------------------------
// ghostsize(1:dim) must be >= 0 and small against the mesh (the periodic
// image arithmetic of the fused ghost write assumes g < 16 * Nc).
bool check_ghost(const Handle& h, const int* ghost, const char* caller, int* info) {
  for (int a = 0; a < h.dim; ++a)
    if (ghost[a] < 0 || ghost[a] > 16 * h.g.N[a]) {
      fail(info, kErrorError, kErrArgument,
           std::string(caller) + ": ghostsize must be >= 0 and <= 16 * (Nm - 1)");
      return false;
    }
  return true;
}

template <class T>
int p2m_pipeline(Handle& h, const T* xp, int64_t ldxp, int64_t Np, const T* up, int64_t ldup,
                 int lda, int kernel, const int* ghost, T* field, int64_t ldf,
                 const int64_t* f_lb, const int64_t* f_ub, bool remesh, cudaStream_t st,
                 int* info, const char* caller) {
  if (!check_ghost(h, ghost, caller, info)) return *info;
  int lo[3], hi[3];
  for (int a = 0; a < h.dim; ++a) {
    lo[a] = 1 - ghost[a];
    hi[a] = h.Nm[a] + ghost[a];
    // along a cut axis the stencils reach HL - 1 nodes past the real ones,
    // whose contributions the ghost layers carry to the neighbours
    if (h.open[a] && ghost[a] < (kernel == kKernelMp4 ? 1 : 0))
      return fail(info, kErrorError, kErrArgument,
                  std::string(caller) + ": ghostsize too small for this kernel on a cut axis");
  }
  FieldDesc fd;
  if (!make_fd(h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return *info;
  const P2MPrec prec = is_f32<T>() ? P2M_FP32
                                   : (g_precision.load() == PPMG_PREC_MIXED ? P2M_MIXED
                                                                            : P2M_FP64);
  Workspace& ws = remesh ? h.ws_rmsh : h.ws;
  cudaError_t e;
  if (remesh) {
    // zero the whole allocation (ppm_rmsh_remesh.f:582: field_up = 0)
    e = cudaMemsetAsync(field, 0, sizeof(T) * (size_t)field_elems(h, ldf, f_lb, f_ub), st);
    if (e) return cuda_fail(info, e, caller);
    // records of the comp_weights order (ws_rmsh holds its sort)
    KeyParams kp = make_kp(h, KEY_INTERP_CHECKED, false);
    const int* dnv = d_nvalid_of(ws, h.g.ncell);
    if (prec == P2M_FP64)
      e = pack_records<T, double>(kp, xp, ldxp, up, ldup, lda, Np, dnv, ws, st);
    else
      e = pack_records<T, float>(kp, xp, ldxp, up, ldup, lda, Np, dnv, ws, st);
    if (e) return cuda_fail(info, e, caller);
  } else {
    h.sort_cached = false;
    KeyParams kp = make_kp(h, KEY_INTERP_CHECKED, false);
    e = sort_interp<T>(h, kp, xp, ldxp, up, ldup, lda, Np, prec == P2M_FP64, h.d_status + 0,
                       (T*)nullptr, 0, 0, st);
    if (e) return cuda_fail(info, e, caller);
  }
  P2MParams P{};
  for (int a = 0; a < 3; ++a) P.N[a] = a < h.dim ? h.g.N[a] : 1;
  P.TZ = p2m_tile_depth(h.dim, P.N);
  // staging slots per CTA (4 vectors per particle): ~72 KB for 3D, 2 CTAs / SM
  if (h.dim == 3)
    P.cap = prec == P2M_FP64 ? 544 : 1088;
  else
    P.cap = prec == P2M_FP64 ? 448 : 896;
  P.c0 = 0;
  P.start = ws.start.as<int>();
  P.rec = remesh ? (const void*)ws.w1d.p : ws.rec.p;
  P.us = ws.us.p;
  P.field = field;
  P.fd = fd;
  P.span = cell_span(P.N);
  for (int a = 0; a < h.dim; ++a)
    if (h.open[a]) {
      // a cut axis: every node of the written box 1-g:Nm+g is produced
      // (ghost nodes hold the contributions owed to the neighbours)
      P.open[a] = 1;
      P.span.org[a] = lo[a] - 1;
      P.span.ext[a] = hi[a] - lo[a] + 1;
    }
  if ((e = ws.tiles.ensure(p2m_scratch_bytes(h.dim, P.N, &P.span)))) return cuda_fail(info, e, caller);
  e = launch_p2m(P, h.dim, kernel, prec, lda, Np > 0 ? Np : 1, remesh, ws.tiles.p, st);
  if (e) return cuda_fail(info, e, caller);
  if (!remesh) {
    h.sort_cached = true;
    h.items_m2p = !p2m_row_gather(h.dim, prec);
    h.cache_quirk = false;
    h.cache_prec = prec == P2M_FP64 ? 0 : 1;
    h.cache_np = Np;
    h.cache_ldxp = ldxp;
  }
  return 0;
}

// Whether the cell order held in h.ws can serve an M2P (quirk: keys from
// M2P's FP32 mesh spacing) or a P2M adjoint (P2M's spacing) of these
// positions: same count, layout, record precision and key arithmetic, no
// invalid particle in the sort, and an equal position fingerprint.
// Synchronises the stream once (a 24-byte read-back).
template <class T>
bool can_reuse_sort(Handle& h, const T* xp, int64_t ldxp, int64_t Np, int rec_prec, bool quirk,
                    cudaStream_t st) {
  if (!h.sort_cached || h.cache_np != Np || h.cache_ldxp != ldxp || h.cache_prec != rec_prec)
    return false;
  // keys and offsets agree when both sorts used the same mesh spacing
  if (h.cache_quirk != quirk && !(is_f32<T>() ? h.dxi_same_f : h.dxi_same_d)) return false;
  if (position_hash<T>(xp, ldxp, Np, h.dim, h.d_hash + 1, st)) return false;
  if (cudaMemcpyAsync(h.h_small, h.d_hash, 2 * sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost, st))
    return false;
  if (cudaMemcpyAsync(h.h_small + 2, h.d_status, sizeof(int), cudaMemcpyDeviceToHost, st))
    return false;
  if (cudaStreamSynchronize(st)) return false;
  const int bad = *reinterpret_cast<const int*>(h.h_small + 2);
  return h.h_small[0] == h.h_small[1] && bad == 0;
}

template <class T>
int m2p_pipeline(Handle& h, const T* xp, int64_t ldxp, int64_t Np, T* up, int64_t ldup,
                 int lda, int kernel, const T* field, int64_t ldf, const int64_t* f_lb,
                 const int64_t* f_ub, cudaStream_t st, int* info, const char* caller) {
  int lo[3], hi[3];
  for (int a = 0; a < h.dim; ++a) {
    lo[a] = 1;
    hi[a] = h.g.N[a];
  }
  for (int a = 0; a < h.dim; ++a)
    if (h.open[a]) {
      // a cut axis: the nodes the stencils reach are read, ghost nodes
      // included (filled from the neighbours by a ghost get)
      const int HL = kernel == kKernelMp4 ? 2 : 1;
      lo[a] = 2 - HL;
      hi[a] = h.g.N[a] + HL;
    }
  FieldDesc fd;
  if (!make_fd(h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return *info;
  if (Np == 0) return 0;
  const M2PPrec prec = is_f32<T>() ? M2P_FP32
                                   : (g_precision.load() == PPMG_PREC_MIXED ? M2P_MIXED
                                                                            : M2P_FP64);
  const int rec_prec = prec == M2P_FP64 ? 0 : 1;
  const bool reuse = can_reuse_sort<T>(h, xp, ldxp, Np, rec_prec, true, st);
  cudaError_t e = cudaSuccess;
  KeyParams kp = make_kp(h, KEY_INTERP_WRAP, true);
  if (!reuse) {
    h.sort_cached = false;
    // outside a z-slab: unassigned (405); else only non-finite positions fail
    e = sort_interp<T>(h, kp, xp, ldxp, (const T*)nullptr, 0, 0, Np, prec == M2P_FP64,
                       h.d_status + (h.cut() ? 0 : 1), up, ldup, lda, st);
    if (e) return cuda_fail(info, e, caller);
  }
  const int* dnv = d_nvalid_of(h.ws, h.g.ncell);
  M2PParams P{};
  for (int a = 0; a < 3; ++a) P.N[a] = a < h.dim ? h.g.N[a] : 1;
  P.nvalid = Np;
  P.d_nvalid = dnv;
  P.idx = h.ws.idx.as<int>();
  P.rec = h.ws.rec.p;
  P.field = field;
  P.fd = fd;
  P.up = up;
  P.ldup = ldup;
  P.lda = lda;
  for (int a = 0; a < 3; ++a) P.open[a] = h.open[a] ? 1 : 0;
  if (h.dim == 3) {
    TileItems ti;
    if ((e = h.ws.tiles.ensure(tile_items_bytes(P.N)))) return cuda_fail(info, e, caller);
    // a cut subdomain's P2M items cover its nodes -g .. N+g, not M2P's
    // cells: M2P builds its own (the cell order itself is reused)
    if (reuse && !h.cut() && h.items_m2p) {
      ti = tile_items_view(h.ws.tiles.p, P.N);
    } else if ((e = make_tile_items(h.ws.start.as<int>(), P.N, Np, h.ws.tiles.p, ti, st))) {
      return cuda_fail(info, e, caller);
    } else {
      h.items_m2p = !h.cut();
    }
    P.start = h.ws.start.as<int>();
    P.items = ti.items;
    P.nitems = ti.nitems;
    P.item_cap = ti.cap;
  }
  if (!reuse && h.dim == 3) {
    // the M2P sort (with its items) is now what ws holds
    h.sort_cached = true;
    h.cache_quirk = true;
    h.cache_prec = rec_prec;
    h.cache_np = Np;
    h.cache_ldxp = ldxp;
  }
  e = launch_m2p(P, h.dim, kernel, prec, st);
  if (e) return cuda_fail(info, e, caller);
  return 0;
}

// Device status -> info (synchronises the stream).
int read_status(Handle& h, cudaStream_t st, int* info, const char* caller) {
  int hs[3] = {0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(hs, h.d_status, sizeof(hs), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return cuda_fail(info, e, caller);
  if (hs[0] || hs[1] || hs[2]) {
    e = cudaMemsetAsync(h.d_status, 0, 3 * sizeof(int), st);
    cudaStreamSynchronize(st);
  }
  if (hs[2] > 0) {
    return fail(info, kErrorFatal, 602,
                std::string(caller) + ": a device copy did not complete in time (results invalid)");
  }
  if (hs[0] > 0) {
    return fail(info, kErrorFatal, kErrPartUnass,
                std::string(caller) + ": " + std::to_string(hs[0]) +
                    " particles lie outside the subdomain (unassigned)");
  }
  if (hs[1] > 0) {
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": " + std::to_string(hs[1]) +
                    " particles have non-finite positions");
  }
  if (info) *info = 0;
  return 0;
}

template <class T>
T* mirror(DevBuf& b, const T* host, int64_t n, cudaStream_t st, cudaError_t& e) {
  e = b.ensure(sizeof(T) * (size_t)(n > 0 ? n : 1));
  if (e) return nullptr;
  if (host && n > 0) e = cudaMemcpyAsync(b.p, host, sizeof(T) * (size_t)n,
                                         cudaMemcpyHostToDevice, st);
  return b.as<T>();
}

bool field_is_box(const Handle& h, const int64_t* f_lb, const int64_t* f_ub, const int* ghost) {
  for (int a = 0; a < h.dim; ++a)
    if (f_lb[a] != 1 - ghost[a] || f_ub[a] != h.Nm[a] + ghost[a]) return false;
  return true;
}

template <class T>
int sub_exchange(Handle& h, T* field, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                 const int* ghost, bool put, bool host_transport, cudaStream_t st, int* info,
                 const char* caller);

template <class T>
void p2m_host(const T* xp, int64_t ldxp, int64_t Np, const T* up, int64_t ldup, int lda,
              int topo_id, int mesh_id, int kernel, const int* ghostsize, T* field_up,
              int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info, int dim,
              const char* caller) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": particles must be specified"); return; }
  if (Np > 0 && ldxp < dim) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": leading dimension of xp insufficient"); return; }
  if (lda < 1 || ldup < lda || ldf < lda) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": lda / leading dimensions inconsistent"); return; }
  if (Np >= (int64_t)1 << 31) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": Np must be < 2^31"); return; }
  if (!check_kernel(kernel, caller, info)) return;
  if (dim == 2 && kernel != kKernelMp4) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": Only Mp4 is available in 2D"); return; }
  Handle* h = get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t st = h->stream;
  cudaError_t e;
  const T* dxp = mirror<T>(h->ws.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const T* dup = mirror<T>(h->ws.h_up, up, ldup * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  // the written box is all of field_up in the common case; otherwise bring the
  // untouched surroundings along so the copy back preserves them
  const bool whole = field_is_box(*h, f_lb, f_ub, ghostsize) && ldf == lda;
  T* dfield = mirror<T>(h->ws.h_field, whole ? (const T*)nullptr : field_up, nf, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if (p2m_pipeline<T>(*h, dxp, ldxp, Np, dup, ldup, lda, kernel, ghostsize, dfield, ldf, f_lb,
                      f_ub, false, st, info, caller))
    return;
  // a z-slab ends with the ghost put, as ppm_interp_p2m.f:3665-3718 does
  if (h->cut() && h->halo_fn &&
      sub_exchange<T>(*h, dfield, ldf, f_lb, f_ub, ghostsize, true, true, st, info, caller))
    return;
  e = cudaMemcpyAsync(field_up, dfield, sizeof(T) * (size_t)nf, cudaMemcpyDeviceToHost, st);
  if (e) { cuda_fail(info, e, caller); return; }
  read_status(*h, st, info, caller);
}

template <class T>
void p2m_dev(const T* xp, int64_t ldxp, int64_t Np, const T* up, int64_t ldup, int lda,
             int topo_id, int mesh_id, int kernel, const int* ghostsize, T* field_up,
             int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info, int dim,
             cudaStream_t st, const char* caller) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < dim) || lda < 1 || ldup < lda || ldf < lda ||
      Np >= (int64_t)1 << 31) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": invalid sizes");
    return;
  }
  if (!check_kernel(kernel, caller, info)) return;
  if (dim == 2 && kernel != kKernelMp4) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": Only Mp4 is available in 2D"); return; }
  Handle* h = get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  if (p2m_pipeline<T>(*h, xp, ldxp, Np, up, ldup, lda, kernel, ghostsize, field_up, ldf, f_lb,
                      f_ub, false, st, info, caller))
    return;
  // a z-slab ends with the ghost put, as ppm_interp_p2m.f:3665-3718 does
  if (h->cut() && h->halo_fn)
    sub_exchange<T>(*h, field_up, ldf, f_lb, f_ub, ghostsize, true, false, st, info, caller);
}

template <class T>
void m2p_host(const T* xp, int64_t ldxp, int64_t Np, T* up, int64_t ldup, int lda,
              int topo_id, int mesh_id, int kernel, const int* ghostsize, const T* field_up,
              int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info, int dim,
              const char* caller) {
  (void)ghostsize;
  clear_error();
  if (info) *info = 0;
  if (Np < 0) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": particles must be specified"); return; }
  if (Np > 0 && ldxp < dim) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": leading dimension of xp insufficient"); return; }
  if (lda < 1 || ldup < lda || ldf < lda) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": lda / leading dimensions inconsistent"); return; }
  if (Np >= (int64_t)1 << 31) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": Np must be < 2^31"); return; }
  if (!check_kernel(kernel, caller, info)) return;
  Handle* h = get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t st = h->stream;
  cudaError_t e;
  const T* dxp = mirror<T>(h->ws.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  // up is overwritten column by column; rows beyond lda (ldup > lda) are kept
  T* dup = mirror<T>(h->ws.h_up, ldup == lda ? (const T*)nullptr : (const T*)up, ldup * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  const T* dfield = mirror<T>(h->ws.h_field, field_up, nf, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if (m2p_pipeline<T>(*h, dxp, ldxp, Np, dup, ldup, lda, kernel, dfield, ldf, f_lb, f_ub, st,
                      info, caller))
    return;
  if (Np > 0) {
    e = cudaMemcpyAsync(up, dup, sizeof(T) * (size_t)(ldup * Np), cudaMemcpyDeviceToHost, st);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  read_status(*h, st, info, caller);
}

template <class T>
void m2p_dev(const T* xp, int64_t ldxp, int64_t Np, T* up, int64_t ldup, int lda, int topo_id,
             int mesh_id, int kernel, const int* ghostsize, const T* field_up, int64_t ldf,
             const int64_t* f_lb, const int64_t* f_ub, int* info, int dim, cudaStream_t st,
             const char* caller) {
  (void)ghostsize;
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < dim) || lda < 1 || ldup < lda || ldf < lda ||
      Np >= (int64_t)1 << 31) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": invalid sizes");
    return;
  }
  if (!check_kernel(kernel, caller, info)) return;
  Handle* h = get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  m2p_pipeline<T>(*h, xp, ldxp, Np, up, ldup, lda, kernel, field_up, ldf, f_lb, f_ub, st, info,
                  caller);
}

int adjoint_pipeline(Handle& h, const double* xp, int64_t ldxp, int64_t Np, const double* up,
                     int64_t ldup, int lda, int kernel, const double* r, int64_t ldf,
                     const int64_t* f_lb, const int64_t* f_ub, double* dw, int64_t lddw,
                     double* dx, int64_t lddx, cudaStream_t st, int* info, const char* caller) {
  int lo[3], hi[3];
  for (int a = 0; a < h.dim; ++a) {
    lo[a] = 1;
    hi[a] = h.g.N[a];
  }
  for (int a = 0; a < 3; ++a)
    if (h.open[a]) {
      // a cut axis: r's ghost nodes are read (the adjoint of the put is a get)
      const int HL = kernel == kKernelMp4 ? 2 : 1;
      lo[a] = 2 - HL;
      hi[a] = h.g.N[a] + HL;
    }
  FieldDesc fd;
  if (!make_fd(h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return *info;
  if (Np == 0) return 0;
  const M2PPrec prec = g_precision.load() == PPMG_PREC_MIXED ? M2P_MIXED : M2P_FP64;
  // the transpose of P2M: P2M's stencil (FP64 mesh spacing), periodic wrap;
  // the cell order of a P2M of the same positions serves as is
  cudaError_t e = cudaSuccess;
  const bool reuse = can_reuse_sort<double>(h, xp, ldxp, Np, prec == M2P_FP64 ? 0 : 1, false, st);
  if (!reuse) {
    h.sort_cached = false;  // the work items below describe this sort only
    KeyParams kp = make_kp(h, KEY_INTERP_WRAP, false);
    e = sort_interp<double>(h, kp, xp, ldxp, nullptr, 0, 0, Np, prec == M2P_FP64,
                            h.d_status + (h.cut() ? 0 : 1), dw, lddw, lda, st);
    if (e) return cuda_fail(info, e, caller);
  }
  const int* dnv = d_nvalid_of(h.ws, h.g.ncell);
  M2PParams P{};
  for (int a = 0; a < 3; ++a) P.N[a] = h.g.N[a];
  P.nvalid = Np;
  P.d_nvalid = dnv;
  P.idx = h.ws.idx.as<int>();
  P.rec = h.ws.rec.p;
  P.field = r;
  P.fd = fd;
  P.up = dw;
  P.ldup = lddw;
  P.lda = lda;
  P.upin = up;
  P.ldupin = ldup;
  P.dx = dx;
  P.lddx = lddx;
  for (int a = 0; a < 3; ++a) P.open[a] = h.open[a] ? 1 : 0;
  for (int a = 0; a < 3; ++a) P.dxi[a] = h.g.dxi_d[a];
  if (lda <= 4) {
    TileItems ti;
    if ((e = h.ws.tiles.ensure(tile_items_bytes(P.N)))) return cuda_fail(info, e, caller);
    // a cut subdomain's P2M items cover nodes, not cells: own items
    if (reuse && !h.cut() && h.items_m2p) {
      ti = tile_items_view(h.ws.tiles.p, P.N);
    } else if ((e = make_tile_items(h.ws.start.as<int>(), P.N, Np, h.ws.tiles.p, ti, st))) {
      return cuda_fail(info, e, caller);
    } else {
      h.items_m2p = !h.cut();
    }
    P.start = h.ws.start.as<int>();
    P.items = ti.items;
    P.nitems = ti.nitems;
    P.item_cap = ti.cap;
  }
  e = launch_adjoint(P, kernel, prec, st);
  if (e) return cuda_fail(info, e, caller);
  return 0;
}

template <class T>
int ghost_pipeline(Handle& h, T* field, int64_t ldf, int lda, const int64_t* f_lb,
                   const int64_t* f_ub, const int* ghost, int maptype, cudaStream_t st,
                   int* info, const char* caller) {
  if (maptype != kMapGhostGet && maptype != kMapGhostPut)
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": maptype must be ghost_get (5) or ghost_put (6)");
  if (!check_ghost(h, ghost, caller, info)) return *info;
  int lo[3], hi[3];
  for (int a = 0; a < h.dim; ++a) {
    lo[a] = 1 - ghost[a];
    hi[a] = h.Nm[a] + ghost[a];
  }
  FieldDesc fd;
  if (!make_fd(h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return *info;
  GhostParams P{};
  P.dim = h.dim;
  P.lda = lda;
  for (int a = 0; a < 3; ++a) {
    P.N[a] = a < h.dim ? h.g.N[a] : 1;
    P.lo[a] = a < h.dim ? lo[a] : 0;
    P.hi[a] = a < h.dim ? hi[a] : 0;
  }
  P.fd = fd;
  T* tmp = nullptr;
  if (maptype == kMapGhostPut) {
    int64_t n = lda;
    for (int a = 0; a < h.dim; ++a) n *= h.Nm[a];
    cudaError_t e = h.ws.h_aux.ensure(sizeof(T) * (size_t)n);
    if (e) return cuda_fail(info, e, caller);
    tmp = h.ws.h_aux.as<T>();
  }
  cudaError_t e = launch_ghost<T>(P, maptype, field, tmp, st);
  if (e) return cuda_fail(info, e, caller);
  return 0;
}

// One call of the caller's transport on device blocks.  host_transport (the
// host entry points): the transport sees host staging copies of them.
// Returns the transport's status (a CUDA error of the staging in e).
int run_transport(Handle& h, int ns, const ppmg_halo_block* sends, int nr,
                  const ppmg_halo_block* recvs, bool host_transport, cudaStream_t st,
                  cudaError_t& e) {
  e = cudaSuccess;
  if (!host_transport) return h.halo_fn(h.halo_ctx, ns, sends, nr, recvs, 1, st);
  size_t tot = 0;
  for (int b = 0; b < ns; ++b) tot += (size_t)sends[b].bytes;
  for (int b = 0; b < nr; ++b) tot += (size_t)recvs[b].bytes;
  h.halo_host.resize(tot > 0 ? tot : 1);
  unsigned char* hb = h.halo_host.data();
  std::vector<ppmg_halo_block> hs(sends, sends + ns), hr(recvs, recvs + nr);
  size_t o = 0;
  for (int b = 0; b < ns && !e; ++b) {
    hs[b].buf = hb + o;
    e = cudaMemcpyAsync(hb + o, sends[b].buf, (size_t)sends[b].bytes, cudaMemcpyDeviceToHost, st);
    o += (size_t)sends[b].bytes;
  }
  for (int b = 0; b < nr; ++b) {
    hr[b].buf = hb + o;
    o += (size_t)recvs[b].bytes;
  }
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return 0;
  const int rc = h.halo_fn(h.halo_ctx, ns, hs.data(), nr, hr.data(), 0, nullptr);
  for (int b = 0; b < nr && !rc && !e; ++b)
    e = cudaMemcpyAsync(recvs[b].buf, hr[b].buf, (size_t)recvs[b].bytes, cudaMemcpyHostToDevice,
                        st);
  if (!e) e = cudaStreamSynchronize(st);  // the staging is reused by the next call
  return rc;
}

// The ghost exchange of a z-slab handle with its neighbours through the
// caller's transport, on the device field `field` (the caller's for the `_dev`
// entry points, the mirror of the host entry points).  host_transport: the
// transport sees host staging buffers (host entry points) instead of device
// memory.  put: received blocks are added to the planes they belong to; get:
// they replace the ghost planes.
template <class T>
int slab_exchange(Handle& h, T* field, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                  const int* ghost, bool put, bool host_transport, cudaStream_t st, int* info,
                  const char* caller) {
  if (h.halo_fn == nullptr)
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": z-slab subdomain without a halo transport "
                                      "(ppmg_halo_set_transport)");
  HaloPlan pl;
  const char* why = halo_plan(h.nsubs, h.istart.data(), h.nnodes.data(), h.Nm_global[2],
                              h.local_sub, ldf, f_lb, f_ub, ghost[2], put, pl);
  if (why) return fail(info, kErrorError, kErrArgument, std::string(caller) + ": " + why);
  if (pl.count == 0) return 0;
  const size_t bytes = sizeof(T) * (size_t)pl.count;
  T* rbuf[2];
  cudaError_t e = cudaSuccess;
  if (put) {
    if ((e = h.halo_rbuf.ensure(2 * bytes))) return cuda_fail(info, e, caller);
    rbuf[0] = h.halo_rbuf.as<T>();
    rbuf[1] = rbuf[0] + pl.count;
  } else {  // a get receives straight into the ghost planes (never sent)
    rbuf[0] = field + pl.recv_off[0];
    rbuf[1] = field + pl.recv_off[1];
  }
  ppmg_halo_block sends[2], recvs[2];
  for (int b = 0; b < 2; ++b) {
    sends[b] = {pl.send_peer[b], pl.send_tag[b], field + pl.send_off[b], (int64_t)bytes};
    recvs[b] = {pl.recv_peer[b], pl.recv_tag[b], rbuf[b], (int64_t)bytes};
  }
  const int rc = run_transport(h, 2, sends, 2, recvs, host_transport, st, e);
  if (e) return cuda_fail(info, e, caller);
  if (rc != 0)
    return fail(info, kErrorFatal, 2,
                std::string(caller) + ": the halo transport failed (returned " +
                    std::to_string(rc) + ")");
  if (put)
    for (int b = 0; b < 2 && !e; ++b)
      e = launch_plane_add<T>(field + pl.recv_off[b], rbuf[b], pl.count, st);
  if (e) return cuda_fail(info, e, caller);
  return 0;
}

// The ghost exchange of a subdomain cut along several axes: boxes per
// neighbour and periodic shift (halo_boxes), packed into one send buffer,
// moved by the caller's transport into one receive buffer, then added (put)
// or copied (get) into the field.  The get's boxes are disjoint: one launch
// copies them all.  The put's may overlap (a corner node receives from up
// to 7 neighbours): they are added in waves of disjoint boxes, each box after
// every earlier box it overlaps, so every node sums in the plan's order.
template <class T>
int box_exchange(Handle& h, T* field, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                 const int* ghost, bool put, bool host_transport, cudaStream_t st, int* info,
                 const char* caller) {
  if (h.halo_fn == nullptr)
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": subdomain without a halo transport "
                                      "(ppmg_halo_set_transport)");
  std::vector<HaloBox> sb, rb;
  const char* why = halo_boxes(h.nsubs, h.istart.data(), h.nnodes.data(), h.Nm_global,
                               h.local_sub, ghost, put, sb, rb);
  if (why) return fail(info, kErrorError, kErrArgument, std::string(caller) + ": " + why);
  for (const auto* v : {&sb, &rb})
    for (const HaloBox& b : *v)
      for (int a = 0; a < 3; ++a)
        if (b.lo[a] < f_lb[a] || b.hi[a] > f_ub[a])
          return fail(info, kErrorError, kErrArgument,
                      std::string(caller) + ": field_up bounds do not cover the ghost layers");
  // table rows: lo[3], ext[3], first index of the box in its launch, its
  // offset in the buffer.  Rows: the sends, the receives, then the
  // receives again grouped by the put's waves (a box goes one wave after
  // the last earlier box it overlaps)
  const int ns = (int)sb.size(), nr = (int)rb.size();
  auto overlap = [&](const HaloBox& x, const HaloBox& y) {
    for (int a = 0; a < 3; ++a)
      if (x.hi[a] < y.lo[a] || y.hi[a] < x.lo[a]) return false;
    return true;
  };
  std::vector<int> wave(nr, 0);
  int nw = 0;
  if (put)
    for (int i = 0; i < nr; ++i) {
      for (int j = 0; j < i; ++j)
        if (wave[j] >= wave[i] && overlap(rb[i], rb[j])) wave[i] = wave[j] + 1;
      nw = wave[i] + 1 > nw ? wave[i] + 1 : nw;
    }
  std::vector<int64_t>& tab = h.halo_tab_host;
  tab.assign(8 * (size_t)(ns + 2 * nr), 0);
  std::vector<int64_t> elems(ns + nr);
  int64_t tot[2] = {0, 0};
  auto row = [&](int r, const HaloBox& b, int64_t first, int64_t off) {
    int64_t* t = tab.data() + 8 * (size_t)r;
    for (int a = 0; a < 3; ++a) {
      t[a] = b.lo[a];
      t[3 + a] = b.hi[a] - b.lo[a] + 1;
    }
    t[6] = first;
    t[7] = off;
  };
  for (int i = 0; i < ns + nr; ++i) {
    const HaloBox& b = i < ns ? sb[i] : rb[i - ns];
    int64_t n = ldf;
    for (int a = 0; a < 3; ++a) n *= b.hi[a] - b.lo[a] + 1;
    elems[i] = n;
    int64_t& acc = tot[i < ns ? 0 : 1];
    row(i, b, acc, acc);
    acc += n;
  }
  std::vector<int> wfirst(nw + 1, 0);
  std::vector<int64_t> wtot(nw, 0);
  {
    int r = ns + nr;
    for (int w = 0; w < nw; ++w) {
      wfirst[w] = r;
      for (int i = 0; i < nr; ++i)
        if (wave[i] == w) {
          row(r++, rb[i], wtot[w], tab[8 * (size_t)(ns + i) + 7]);
          wtot[w] += elems[ns + i];
        }
    }
  }
  cudaError_t e = cudaSuccess;
  if ((e = h.halo_tab.ensure(sizeof(int64_t) * tab.size())) ||
      (e = h.halo_sbuf.ensure(sizeof(T) * (size_t)(tot[0] > 0 ? tot[0] : 1))) ||
      (e = h.halo_rbuf.ensure(sizeof(T) * (size_t)(tot[1] > 0 ? tot[1] : 1))))
    return cuda_fail(info, e, caller);
  int64_t* dtab = h.halo_tab.as<int64_t>();
  T* sbuf = h.halo_sbuf.as<T>();
  T* rbuf = h.halo_rbuf.as<T>();
  if ((e = cudaMemcpyAsync(dtab, tab.data(), sizeof(int64_t) * tab.size(),
                           cudaMemcpyHostToDevice, st)))
    return cuda_fail(info, e, caller);
  int64_t s[3];
  int lb[3];
  s[0] = ldf;
  s[1] = ldf * (f_ub[0] - f_lb[0] + 1);
  s[2] = s[1] * (f_ub[1] - f_lb[1] + 1);
  for (int a = 0; a < 3; ++a) lb[a] = (int)f_lb[a];
  if ((e = launch_box_copy<T>(field, ldf, s, lb, dtab, ns, tot[0], sbuf, kBoxPack, st)))
    return cuda_fail(info, e, caller);
  std::vector<ppmg_halo_block> sends(ns), recvs(nr);
  for (int i = 0; i < ns; ++i)
    sends[i] = {sb[i].peer, sb[i].tag, sbuf + tab[8 * (size_t)i + 7],
                (int64_t)sizeof(T) * elems[i]};
  for (int i = 0; i < nr; ++i)
    recvs[i] = {rb[i].peer, rb[i].tag, rbuf + tab[8 * (size_t)(ns + i) + 7],
                (int64_t)sizeof(T) * elems[ns + i]};
  const int rc = run_transport(h, ns, sends.data(), nr, recvs.data(), host_transport, st, e);
  if (e) return cuda_fail(info, e, caller);
  if (rc != 0)
    return fail(info, kErrorFatal, 2,
                std::string(caller) + ": the halo transport failed (returned " +
                    std::to_string(rc) + ")");
  if (!put)
    e = launch_box_copy<T>(field, ldf, s, lb, dtab + 8 * (size_t)ns, nr, tot[1], rbuf,
                           kBoxCopy, st);
  for (int w = 0; w < nw && !e; ++w)
    e = launch_box_copy<T>(field, ldf, s, lb, dtab + 8 * (size_t)wfirst[w],
                           (w + 1 < nw ? wfirst[w + 1] : ns + 2 * nr) - wfirst[w], wtot[w],
                           rbuf, kBoxAdd, st);
  if (e) return cuda_fail(info, e, caller);
  return 0;
}

template <class T>
int sub_exchange(Handle& h, T* field, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                 const int* ghost, bool put, bool host_transport, cudaStream_t st, int* info,
                 const char* caller) {
  return h.slab() ? slab_exchange<T>(h, field, ldf, f_lb, f_ub, ghost, put, host_transport, st,
                                     info, caller)
                  : box_exchange<T>(h, field, ldf, f_lb, f_ub, ghost, put, host_transport, st,
                                    info, caller);
}

template <class T>
void ghost_host(T* field_up, int64_t ldf, int lda, const int64_t* f_lb, const int64_t* f_ub,
                int topo_id, int mesh_id, const int* ghostsize, int maptype, int* info,
                const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  // a z-slab handle maps through its halo transport
  Handle* h = get_checked(topo_id, mesh_id, hh->dim, caller, info, hh->halo_fn != nullptr);
  if (!h) return;
  if (lda < 1 || ldf < lda) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": lda inconsistent"); return; }
  if (h->cut() && maptype != kMapGhostGet && maptype != kMapGhostPut) { fail(info, kErrorError, kErrArgument, std::string(caller) + ": maptype must be ghost_get (5) or ghost_put (6)"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t st = h->stream;
  cudaError_t e;
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  T* dfield = mirror<T>(h->ws.h_field, field_up, nf, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if (h->cut()) {
    if (sub_exchange<T>(*h, dfield, ldf, f_lb, f_ub, ghostsize, maptype == kMapGhostPut, true,
                         st, info, caller))
      return;
  } else if (ghost_pipeline<T>(*h, dfield, ldf, lda, f_lb, f_ub, ghostsize, maptype, st, info,
                               caller)) {
    return;
  }
  e = cudaMemcpyAsync(field_up, dfield, sizeof(T) * (size_t)nf, cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) cuda_fail(info, e, caller);
}

}  // namespace

void set_error(int info, int errnum, const std::string& msg) {
  t_err.info = info;
  t_err.errnum = errnum;
  t_err.msg = msg;
}
void clear_error() {
  t_err.info = 0;
  t_err.errnum = 0;
  t_err.msg.clear();
}

}  // namespace ppmg

using namespace ppmg;

extern "C" {

int ppmg_version(void) { return 10000; }

int ppmg_last_error(int* errnum, char* msg, int msglen) {
  if (errnum) *errnum = t_err.errnum;
  if (msg && msglen > 0) {
    std::strncpy(msg, t_err.msg.c_str(), (size_t)msglen - 1);
    msg[msglen - 1] = '\0';
  }
  return t_err.info;
}

void ppmg_set_precision(int mode, int* info) {
  clear_error();
  if (mode != PPMG_PREC_FP64 && mode != PPMG_PREC_MIXED) {
    fail(info, kErrorError, kErrArgument, "ppmg_set_precision: mode must be 0 or 1");
    return;
  }
  g_precision.store(mode);
  if (info) *info = 0;
}

int ppmg_get_precision(void) { return g_precision.load(); }

int64_t ppmg_launch_count(void) { return g_launches.load(); }

void ppmg_mesh_register(int topo_id, int mesh_id, int dim, const double* min_phys,
                        const double* max_phys, const int* Nm, const int* bcdef, int nsubs,
                        const double* min_sub, const double* max_sub, const int* subs_bc,
                        const int* istart, const int* nnodes, int* info) {
  clear_error();
  if (info) *info = 0;
  if (dim != 2 && dim != 3) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_register: dim must be 2 or 3"); return; }
  if (nsubs < 1) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_register: nsubs must be >= 1"); return; }
  for (int a = 0; a < dim; ++a) {
    if (Nm[a] < 2) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_register: Nm must be >= 2"); return; }
    if (!(max_phys[a] > min_phys[a])) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_register: max_phys must exceed min_phys"); return; }
  }
  int64_t ncell = 1;
  for (int a = 0; a < dim; ++a) ncell *= (int64_t)(Nm[a] - 1);
  if (ncell >= ((int64_t)1 << 31) - 1) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_register: mesh has >= 2^31 cells"); return; }
  auto h = std::make_unique<Handle>();
  h->topo_id = topo_id;
  h->mesh_id = mesh_id;
  h->dim = dim;
  h->nsubs = nsubs;
  for (int a = 0; a < 3; ++a) h->Nm[a] = a < dim ? Nm[a] : 2;
  for (int a = 0; a < 3; ++a) h->Nm_global[a] = h->Nm[a];
  for (int f = 0; f < 6; ++f) h->bcdef[f] = f < 2 * dim ? bcdef[f] : kBcPeriodic;
  h->min_sub.assign(min_sub, min_sub + 3 * nsubs);
  h->max_sub.assign(max_sub, max_sub + 3 * nsubs);
  h->subs_bc.assign(subs_bc, subs_bc + 6 * nsubs);
  h->istart.assign(istart, istart + 3 * nsubs);
  h->nnodes.assign(nnodes, nnodes + 3 * nsubs);
  h->local_sub = nsubs == 1 ? 0 : -1;
  Geom& g = h->g;
  g.dim = dim;
  g.ncell = ncell;
  for (int a = 0; a < 3; ++a) {
    const bool on = a < dim;
    g.N[a] = on ? Nm[a] - 1 : 1;
    g.min_phys[a] = on ? min_phys[a] : 0.0;
    g.max_phys[a] = on ? max_phys[a] : 1.0;
    g.min_sub[a] = on ? min_sub[a] : 0.0;
    g.max_sub[a] = on ? max_sub[a] : 1.0;
    // P2M / remesh: dx = len/Nc, dxi = 1/dx in the routine's kind
    const double len = g.max_phys[a] - g.min_phys[a];
    g.dxi_d[a] = 1.0 / (len / (double)g.N[a]);
    const float lenf = (float)g.max_phys[a] - (float)g.min_phys[a];
    g.dxi_f[a] = 1.0f / (lenf / (float)g.N[a]);
    // M2P / comp_weights: len_phys, dx, dxi are default REAL (FP32)
    const float len32 = (float)len;
    const float dx32 = (float)((double)len32 / (double)g.N[a]);
    g.dxiq_d[a] = (double)(float)(1.0 / (double)dx32);
    g.dxiq_f[a] = 1.0f / (lenf / (float)g.N[a]);
    g.h_d[a] = len / (double)(on ? Nm[a] - 1 : 1);
  }
  h->dxi_same_d = true;
  h->dxi_same_f = true;
  for (int a = 0; a < dim; ++a) {
    h->dxi_same_d = h->dxi_same_d && g.dxi_d[a] == g.dxiq_d[a];
    h->dxi_same_f = h->dxi_same_f && g.dxi_f[a] == g.dxiq_f[a];
  }
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (!e) e = cudaMalloc(&h->d_status, 4 * sizeof(int));
  if (!e) e = cudaMalloc(&h->d_hash, 2 * sizeof(unsigned long long));
  if (!e) e = cudaMallocHost(&h->h_small, 4 * sizeof(unsigned long long));
  if (!e) e = cudaMemset(h->d_status, 0, 4 * sizeof(int));
  if (e) { cuda_fail(info, e, "ppmg_mesh_register"); return; }
  std::lock_guard<std::mutex> lk(g_mu);
  handles()[{topo_id, mesh_id}] = std::move(h);
}

void ppmg_mesh_set_local_sub(int topo_id, int mesh_id, int isub, int* info) {
  const char* caller = "ppmg_mesh_set_local_sub";
  clear_error();
  if (info) *info = 0;
  Handle* h = find_handle(topo_id, mesh_id);
  if (!h) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  if (isub < 0 || isub >= h->nsubs) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": isub out of range"); return; }
  if (h->nsubs > 1) {
    // supported decompositions: cartesian (ppm_param_decomp_cartesian and
    // the pencil / slab cuts, each axis cut into intervals shared by all
    // subdomains), in 3D
    if (h->dim != 3) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": several subdomains are supported in 3D only"); return; }
    if (const char* why = check_cartesian(h->nsubs, h->istart.data(), h->nnodes.data(),
                                          h->Nm_global)) {
      fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": " + why);
      return;
    }
    Geom& g = h->g;
    for (int a = 0; a < 3; ++a) {
      const int n = h->nnodes[3 * isub + a];
      h->open[a] = n != h->Nm_global[a];
      h->Nm[a] = n;
      g.N[a] = n - 1;
      g.min_sub[a] = h->min_sub[3 * isub + a];
      g.max_sub[a] = h->max_sub[3 * isub + a];
    }
    g.ncell = (int64_t)g.N[0] * g.N[1] * g.N[2];
  }
  h->local_sub = isub;
  h->sort_cached = false;
  h->w_valid = false;
}

void ppmg_halo_set_transport(int topo_id, int mesh_id, ppmg_halo_fn fn, void* ctx, int* info) {
  clear_error();
  if (info) *info = 0;
  Handle* h = find_handle(topo_id, mesh_id);
  if (!h) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_halo_set_transport: topo_id/mesh_id is invalid"); return; }
  if (h->nsubs < 2 || h->dim != 3) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_halo_set_transport: the mesh has one subdomain (no neighbours to exchange with)"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  h->halo_fn = fn;
  h->halo_ctx = fn ? ctx : nullptr;
}

void ppmg_halo_plan(int nsubs, const int* istart, const int* nnodes, int Nmz, int isub,
                    int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, const int* ghostsize,
                    int maptype, int64_t* count, int* send_peer, int* send_tag,
                    int64_t* send_off, int* recv_peer, int* recv_tag, int64_t* recv_off,
                    int* info) {
  clear_error();
  if (info) *info = 0;
  if (maptype != kMapGhostGet && maptype != kMapGhostPut) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_halo_plan: maptype must be ghost_get (5) or ghost_put (6)"); return; }
  HaloPlan pl;
  const char* why = halo_plan(nsubs, istart, nnodes, Nmz, isub, ldf, f_lb, f_ub, ghostsize[2],
                              maptype == kMapGhostPut, pl);
  if (why) { fail(info, kErrorError, ppmg::kErrArgument, std::string("ppmg_halo_plan: ") + why); return; }
  *count = pl.count;
  for (int b = 0; b < 2; ++b) {
    send_peer[b] = pl.send_peer[b];
    send_tag[b] = pl.send_tag[b];
    send_off[b] = pl.send_off[b];
    recv_peer[b] = pl.recv_peer[b];
    recv_tag[b] = pl.recv_tag[b];
    recv_off[b] = pl.recv_off[b];
  }
}

void ppmg_halo_plan_boxes(int nsubs, const int* istart, const int* nnodes, const int* Nm,
                          int isub, const int* ghostsize, int maptype, int cap,
                          ppmg_halo_box* sends, int* nsend, ppmg_halo_box* recvs, int* nrecv,
                          int* info) {
  clear_error();
  if (info) *info = 0;
  if (maptype != kMapGhostGet && maptype != kMapGhostPut) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_halo_plan_boxes: maptype must be ghost_get (5) or ghost_put (6)"); return; }
  std::vector<HaloBox> hs, hr;
  const char* why = halo_boxes(nsubs, istart, nnodes, Nm, isub, ghostsize,
                               maptype == kMapGhostPut, hs, hr);
  if (why) { fail(info, kErrorError, ppmg::kErrArgument, std::string("ppmg_halo_plan_boxes: ") + why); return; }
  auto out = [cap](const std::vector<HaloBox>& v, ppmg_halo_box* dst, int* n) {
    *n = (int)v.size();
    for (int i = 0; i < (int)v.size() && i < cap; ++i) {
      dst[i].peer = v[i].peer;
      dst[i].tag = v[i].tag;
      for (int a = 0; a < 3; ++a) {
        dst[i].lo[a] = v[i].lo[a];
        dst[i].hi[a] = v[i].hi[a];
      }
    }
  };
  out(hs, sends, nsend);
  out(hr, recvs, nrecv);
}

void ppmg_mesh_unregister(int topo_id, int mesh_id, int* info) {
  clear_error();
  if (info) *info = 0;
  std::unique_ptr<Handle> h;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = handles().find({topo_id, mesh_id});
    if (it == handles().end()) {
      fail(info, kErrorError, ppmg::kErrArgument, "ppmg_mesh_unregister: unknown handle");
      return;
    }
    h = std::move(it->second);
    handles().erase(it);
  }
  if (h->stream) cudaStreamSynchronize(h->stream);
}

void ppmg_sync_status(int topo_id, int mesh_id, void* stream, int* info) {
  clear_error();
  Handle* h = find_handle(topo_id, mesh_id);
  if (!h) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_sync_status: topo_id/mesh_id is invalid"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  read_status(*h, (cudaStream_t)stream, info, "ppmg_sync_status");
}

// ---- P2M ------------------------------------------------------------------
#define P2M_V_HOST(NAME, R, DIM)                                                             \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, const R* up, int64_t ldup, int lda,     \
            int topo_id, int mesh_id, int kernel, const int* ghostsize, R* field_up,        \
            int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info) {             \
    p2m_host<R>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, \
                ldf, f_lb, f_ub, info, DIM, #NAME);                                        \
  }
#define P2M_S_HOST(NAME, R, DIM)                                                             \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, const R* up, int topo_id, int mesh_id,   \
            int kernel, const int* ghostsize, R* field_up, const int64_t* f_lb,             \
            const int64_t* f_ub, int* info) {                                               \
    p2m_host<R>(xp, ldxp, Np, up, 1, 1, topo_id, mesh_id, kernel, ghostsize, field_up, 1,   \
                f_lb, f_ub, info, DIM, #NAME);                                             \
  }
#define P2M_V_DEV(NAME, R, DIM)                                                              \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, const R* up, int64_t ldup, int lda,     \
            int topo_id, int mesh_id, int kernel, const int* ghostsize, R* field_up,        \
            int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info,              \
            void* stream) {                                                                 \
    p2m_dev<R>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,  \
               ldf, f_lb, f_ub, info, DIM, (cudaStream_t)stream, #NAME);                   \
  }

P2M_V_HOST(ppmg_interp_p2m_dv_3d, double, 3)
P2M_V_HOST(ppmg_interp_p2m_sv_3d, float, 3)
P2M_S_HOST(ppmg_interp_p2m_ds_3d, double, 3)
P2M_S_HOST(ppmg_interp_p2m_ss_3d, float, 3)
P2M_V_HOST(ppmg_interp_p2m_dv_2d, double, 2)
P2M_V_HOST(ppmg_interp_p2m_sv_2d, float, 2)
P2M_S_HOST(ppmg_interp_p2m_ds_2d, double, 2)
P2M_S_HOST(ppmg_interp_p2m_ss_2d, float, 2)
P2M_V_DEV(ppmg_interp_p2m_dv_3d_dev, double, 3)
P2M_V_DEV(ppmg_interp_p2m_sv_3d_dev, float, 3)
P2M_V_DEV(ppmg_interp_p2m_dv_2d_dev, double, 2)
P2M_V_DEV(ppmg_interp_p2m_sv_2d_dev, float, 2)

// ---- M2P ------------------------------------------------------------------
#define M2P_V_HOST(NAME, R, DIM)                                                            \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, R* up, int64_t ldup, int lda,           \
            int topo_id, int mesh_id, int kernel, const int* ghostsize, const R* field_up,  \
            int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info) {             \
    m2p_host<R>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, \
                ldf, f_lb, f_ub, info, DIM, #NAME);                                        \
  }
#define M2P_S_HOST(NAME, R, DIM)                                                            \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, R* up, int topo_id, int mesh_id,         \
            int kernel, const int* ghostsize, const R* field_up, const int64_t* f_lb,       \
            const int64_t* f_ub, int* info) {                                               \
    m2p_host<R>(xp, ldxp, Np, up, 1, 1, topo_id, mesh_id, kernel, ghostsize, field_up, 1,   \
                f_lb, f_ub, info, DIM, #NAME);                                             \
  }
#define M2P_V_DEV(NAME, R, DIM)                                                             \
  void NAME(const R* xp, int64_t ldxp, int64_t Np, R* up, int64_t ldup, int lda,           \
            int topo_id, int mesh_id, int kernel, const int* ghostsize, const R* field_up,  \
            int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info,              \
            void* stream) {                                                                 \
    m2p_dev<R>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,  \
               ldf, f_lb, f_ub, info, DIM, (cudaStream_t)stream, #NAME);                   \
  }

M2P_V_HOST(ppmg_interp_m2p_dv_3d, double, 3)
M2P_V_HOST(ppmg_interp_m2p_sv_3d, float, 3)
M2P_S_HOST(ppmg_interp_m2p_ds_3d, double, 3)
M2P_S_HOST(ppmg_interp_m2p_ss_3d, float, 3)
M2P_V_HOST(ppmg_interp_m2p_dv_2d, double, 2)
M2P_V_HOST(ppmg_interp_m2p_sv_2d, float, 2)
M2P_S_HOST(ppmg_interp_m2p_ds_2d, double, 2)
M2P_S_HOST(ppmg_interp_m2p_ss_2d, float, 2)
M2P_V_DEV(ppmg_interp_m2p_dv_3d_dev, double, 3)
M2P_V_DEV(ppmg_interp_m2p_sv_3d_dev, float, 3)
M2P_V_DEV(ppmg_interp_m2p_dv_2d_dev, double, 2)
M2P_V_DEV(ppmg_interp_m2p_sv_2d_dev, float, 2)

// ---- adjoint ----------------------------------------------------------------
static void adjoint_common(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                           int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                           const double* r_field, int64_t ldf, const int64_t* f_lb,
                           const int64_t* f_ub, double* dw, int64_t lddw, double* dx,
                           int64_t lddx, int* info, bool dev, cudaStream_t ust) {
  const char* caller = dev ? "ppmg_interp_p2m_adjoint_dv_3d_dev" : "ppmg_interp_p2m_adjoint_dv_3d";
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < 3) || lda < 1 || ldup < lda || ldf < lda || lddw < lda ||
      lddx < 3 || Np >= (int64_t)1 << 31) {
    fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes");
    return;
  }
  if (!check_kernel(kernel, caller, info)) return;
  Handle* h = get_checked(topo_id, mesh_id, 3, caller, info, true);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  if (dev) {
    adjoint_pipeline(*h, xp, ldxp, Np, up, ldup, lda, kernel, r_field, ldf, f_lb, f_ub, dw,
                     lddw, dx, lddx, ust, info, caller);
    return;
  }
  cudaStream_t st = h->stream;
  cudaError_t e;
  const double* dxp = mirror<double>(h->ws.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const double* dup = mirror<double>(h->ws.h_up, up, ldup * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  const double* dr = mirror<double>(h->ws.h_field, r_field, nf, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  double* ddw = mirror<double>(h->ws.h_aux, (const double*)nullptr, lddw * Np + lddx * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  double* ddx = ddw + lddw * Np;
  if (adjoint_pipeline(*h, dxp, ldxp, Np, dup, ldup, lda, kernel, dr, ldf, f_lb, f_ub, ddw, lddw,
                       ddx, lddx, st, info, caller))
    return;
  if (Np > 0) {
    e = cudaMemcpyAsync(dw, ddw, sizeof(double) * (size_t)(lddw * Np), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaMemcpyAsync(dx, ddx, sizeof(double) * (size_t)(lddx * Np), cudaMemcpyDeviceToHost, st);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  read_status(*h, st, info, caller);
}

void ppmg_interp_p2m_adjoint_dv_3d(const double* xp, int64_t ldxp, int64_t Np,
                                   const double* up, int64_t ldup, int lda, int topo_id,
                                   int mesh_id, int kernel, const double* r_field,
                                   int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                                   double* dw, int64_t lddw, double* dx, int64_t lddx,
                                   int* info) {
  adjoint_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, r_field, ldf, f_lb, f_ub,
                 dw, lddw, dx, lddx, info, false, nullptr);
}

void ppmg_interp_p2m_adjoint_dv_3d_dev(const double* xp, int64_t ldxp, int64_t Np,
                                       const double* up, int64_t ldup, int lda, int topo_id,
                                       int mesh_id, int kernel, const double* r_field,
                                       int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                                       double* dw, int64_t lddw, double* dx, int64_t lddx,
                                       int* info, void* stream) {
  adjoint_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, r_field, ldf, f_lb, f_ub,
                 dw, lddw, dx, lddx, info, true, (cudaStream_t)stream);
}

// ---- ghost ------------------------------------------------------------------
void ppmg_map_field_ghost_d(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                            const int64_t* f_ub, int topo_id, int mesh_id,
                            const int* ghostsize, int maptype, int* info) {
  ghost_host<double>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, maptype, info,
                     "ppmg_map_field_ghost_d");
}
void ppmg_map_field_ghost_s(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                            const int64_t* f_ub, int topo_id, int mesh_id,
                            const int* ghostsize, int maptype, int* info) {
  ghost_host<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, maptype, info,
                    "ppmg_map_field_ghost_s");
}
extern "C++" {
template <class T>
static void ghost_dev(T* field_up, int64_t ldf, int lda, const int64_t* f_lb, const int64_t* f_ub,
                      int topo_id, int mesh_id, const int* ghostsize, int maptype, int* info,
                      cudaStream_t stream, const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  // a z-slab handle maps through its halo transport
  Handle* h = get_checked(topo_id, mesh_id, hh->dim, caller, info, hh->halo_fn != nullptr);
  if (!h) return;
  if (lda < 1 || ldf < lda) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": lda inconsistent"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  if (h->cut()) {
    if (maptype != kMapGhostGet && maptype != kMapGhostPut) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": maptype must be ghost_get (5) or ghost_put (6)"); return; }
    sub_exchange<T>(*h, field_up, ldf, f_lb, f_ub, ghostsize, maptype == kMapGhostPut, false,
                     stream, info, caller);
    return;
  }
  ghost_pipeline<T>(*h, field_up, ldf, lda, f_lb, f_ub, ghostsize, maptype, stream, info, caller);
}
}  // extern "C++"

void ppmg_map_field_ghost_d_dev(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int maptype, int* info, void* stream) {
  ghost_dev<double>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, maptype, info,
                    (cudaStream_t)stream, "ppmg_map_field_ghost_d_dev");
}
void ppmg_map_field_ghost_s_dev(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int maptype, int* info, void* stream) {
  ghost_dev<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, maptype, info,
                   (cudaStream_t)stream, "ppmg_map_field_ghost_s_dev");
}

// ---- comp_weights / remesh ---------------------------------------------------
}  // extern "C"

namespace ppmg {
namespace {
// comp_weights on device positions dxp; the optional user weight arrays wx
// (reference layout wx(1:2ks, 1, 1-ks:Np+ks)) are device arrays when
// `user_dev`, else host arrays (copied back, synchronising the stream).
// Returns 0 or the failing info.
template <class T>
int comp_weights_core(Handle& h, const T* dxp, int64_t ldxp, int64_t Np, int kernel,
                      T* const wx[3], bool user_dev, cudaStream_t st, int* info,
                      const char* caller) {
  const int dim = h.dim;
  KeyParams kp = make_kp(h, KEY_INTERP_CHECKED, false);
  cudaError_t e = bin_sort<T>(kp, dxp, ldxp, Np, h.g.ncell, h.ws_rmsh, h.d_status + 0, st);
  if (e) return cuda_fail(info, e, caller);
  const int S = kernel == kKernelMp4 ? 4 : 2;
  const int wstride = weight_stride(dim, S, (int)sizeof(T));
  e = h.ws_rmsh.w1d.ensure(sizeof(T) * (size_t)(Np > 0 ? Np : 1) * wstride);
  if (e) return cuda_fail(info, e, caller);
  CWParams<T> P{};
  P.dim = dim;
  P.S = S;
  P.wstride = wstride;
  P.nvalid = Np;
  P.d_nvalid = d_nvalid_of(h.ws_rmsh, h.g.ncell);
  P.idx = h.ws_rmsh.idx.as<int>();
  P.xp = dxp;
  P.ldxp = ldxp;
  for (int a = 0; a < 3; ++a) {
    P.min_phys[a] = (T)h.g.min_phys[a];
    P.dxiq[a] = is_f32<T>() ? (T)h.g.dxiq_f[a] : (T)h.g.dxiq_d[a];
    P.istart[a] = h.istart[3 * h.local_sub + a];  // the local subdomain's first node
  }
  P.w = h.ws_rmsh.w1d.as<T>();
  if ((e = launch_comp_weights<T>(P, st))) return cuda_fail(info, e, caller);
  const int ks = S / 2;
  const int64_t nu = (int64_t)S * (Np + 2 * ks);
  for (int a = 0; a < dim; ++a) {
    if (!wx[a]) continue;
    T* dst = wx[a];
    if (!user_dev) {
      dst = mirror<T>(h.ws_rmsh.h_aux, (const T*)nullptr, nu, st, e);
      if (e) return cuda_fail(info, e, caller);
    }
    e = cudaMemsetAsync(dst, 0, sizeof(T) * (size_t)nu, st);
    if (!e) e = launch_weights_to_user<T>(P.w, P.idx, Np, P.d_nvalid, wstride, S, a, dst, st);
    if (!e && !user_dev)
      e = cudaMemcpyAsync(wx[a], dst, sizeof(T) * (size_t)nu, cudaMemcpyDeviceToHost, st);
    if (!e && !user_dev) e = cudaStreamSynchronize(st);
    if (e) return cuda_fail(info, e, caller);
  }
  h.w_valid = true;
  h.w_single = is_f32<T>();
  h.w_kernel = kernel;
  h.w_np = Np;
  return 0;
}

Handle* comp_weights_checks(int64_t ldxp, int64_t Np, int topo_id, int mesh_id, int kernel,
                            int* info, const char* caller) {
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid");
    return nullptr;
  }
  const int dim = hh->dim;
  if (Np < 0 || (Np > 0 && ldxp < dim) || Np >= (int64_t)1 << 31) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": invalid sizes");
    return nullptr;
  }
  if (!check_kernel(kernel, caller, info)) return nullptr;
  return get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
}
}  // namespace
}  // namespace ppmg

extern "C" {

extern "C++" {
template <class T>
static void comp_weights_entry(const T* xp, int64_t ldxp, int64_t Np, int topo_id, int mesh_id,
                               int kernel, T* wx1, T* wx2, T* wx3, int* info, bool dev,
                               cudaStream_t dstream, const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* h = comp_weights_checks(ldxp, Np, topo_id, mesh_id, kernel, info, caller);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  T* const wx[3] = {wx1, wx2, wx3};
  if (dev) {
    comp_weights_core<T>(*h, xp, ldxp, Np, kernel, wx, true, dstream, info, caller);
    return;
  }
  cudaStream_t st = h->stream;
  cudaError_t e;
  const T* dxp = mirror<T>(h->ws_rmsh.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if (comp_weights_core<T>(*h, dxp, ldxp, Np, kernel, wx, false, st, info, caller)) return;
  read_status(*h, st, info, caller);
}
}  // extern "C++"

void ppmg_rmsh_comp_weights_d(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                              int mesh_id, int kernel, double* wx1, double* wx2,
                              double* wx3, int* info) {
  comp_weights_entry<double>(xp, ldxp, Np, topo_id, mesh_id, kernel, wx1, wx2, wx3, info, false,
                             nullptr, "ppmg_rmsh_comp_weights_d");
}
void ppmg_rmsh_comp_weights_s(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                              int mesh_id, int kernel, float* wx1, float* wx2, float* wx3,
                              int* info) {
  comp_weights_entry<float>(xp, ldxp, Np, topo_id, mesh_id, kernel, wx1, wx2, wx3, info, false,
                            nullptr, "ppmg_rmsh_comp_weights_s");
}
void ppmg_rmsh_comp_weights_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                  int mesh_id, int kernel, double* wx1, double* wx2,
                                  double* wx3, int* info, void* stream) {
  comp_weights_entry<double>(xp, ldxp, Np, topo_id, mesh_id, kernel, wx1, wx2, wx3, info, true,
                             (cudaStream_t)stream, "ppmg_rmsh_comp_weights_d_dev");
}
void ppmg_rmsh_comp_weights_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                  int mesh_id, int kernel, float* wx1, float* wx2, float* wx3,
                                  int* info, void* stream) {
  comp_weights_entry<float>(xp, ldxp, Np, topo_id, mesh_id, kernel, wx1, wx2, wx3, info, true,
                            (cudaStream_t)stream, "ppmg_rmsh_comp_weights_s_dev");
}
extern "C++" {
template <class T>
static void remesh_common(const T* xp, int64_t ldxp, int64_t Np, const T* up,
                          int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                          const int* ghostsize, T* field_up, int64_t ldf,
                          const int64_t* f_lb, const int64_t* f_ub, int* info, int dim,
                          const char* caller, bool dev = false, cudaStream_t dst = nullptr) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < dim) || lda < 1 || ldup < lda || ldf < lda) {
    fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes");
    return;
  }
  if (!check_kernel(kernel, caller, info)) return;
  const int ks = kernel == kKernelMp4 ? 2 : 1;
  for (int a = 0; a < dim; ++a)
    if (ghostsize[a] < ks - 1) {  // ppm_rmsh_remesh.f:340-347
      fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": ghostsize too small for this kernel");
      return;
    }
  Handle* h = get_checked(topo_id, mesh_id, dim, caller, info, dim == 3);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->w_valid || h->w_kernel != kernel || h->w_np != Np || h->w_single != is_f32<T>()) {
    fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": compute weights before remeshing");
    return;
  }
  if (dev) {
    // device arrays on the caller's stream; errors latch for ppmg_sync_status
    if (p2m_pipeline<T>(*h, xp, ldxp, Np, up, ldup, lda, kernel, ghostsize, field_up, ldf, f_lb,
                        f_ub, true, dst, info, caller))
      return;
    // a z-slab ends with the ghost put, as ppm_rmsh_remesh.f:876-924 does
    if (h->cut() && h->halo_fn)
      sub_exchange<T>(*h, field_up, ldf, f_lb, f_ub, ghostsize, true, false, dst, info, caller);
    return;
  }
  cudaStream_t st = h->stream;
  cudaError_t e;
  const T* dxp = mirror<T>(h->ws_rmsh.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const T* dup = mirror<T>(h->ws_rmsh.h_up, up, ldup * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  T* dfield = mirror<T>(h->ws_rmsh.h_field, (const T*)nullptr, nf, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if (p2m_pipeline<T>(*h, dxp, ldxp, Np, dup, ldup, lda, kernel, ghostsize, dfield, ldf,
                           f_lb, f_ub, true, st, info, caller))
    return;
  if (h->cut() && h->halo_fn &&
      sub_exchange<T>(*h, dfield, ldf, f_lb, f_ub, ghostsize, true, true, st, info, caller))
    return;
  e = cudaMemcpyAsync(field_up, dfield, sizeof(T) * (size_t)nf, cudaMemcpyDeviceToHost, st);
  if (e) { cuda_fail(info, e, caller); return; }
  read_status(*h, st, info, caller);
}
}  // extern "C++"

void ppmg_rmsh_remesh_dv_3d(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, double* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info) {
  remesh_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, ldf,
                f_lb, f_ub, info, 3, "ppmg_rmsh_remesh_dv_3d");
}
void ppmg_rmsh_remesh_dv_2d(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, double* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info) {
  remesh_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, ldf,
                f_lb, f_ub, info, 2, "ppmg_rmsh_remesh_dv_2d");
}
void ppmg_rmsh_remesh_dv_3d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                                int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                                const int* ghostsize, double* field_up, int64_t ldf,
                                const int64_t* f_lb, const int64_t* f_ub, int* info,
                                void* stream) {
  remesh_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, ldf,
                f_lb, f_ub, info, 3, "ppmg_rmsh_remesh_dv_3d_dev", true, (cudaStream_t)stream);
}
void ppmg_rmsh_remesh_dv_2d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                                int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                                const int* ghostsize, double* field_up, int64_t ldf,
                                const int64_t* f_lb, const int64_t* f_ub, int* info,
                                void* stream) {
  remesh_common(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up, ldf,
                f_lb, f_ub, info, 2, "ppmg_rmsh_remesh_dv_2d_dev", true, (cudaStream_t)stream);
}
void ppmg_rmsh_remesh_sv_3d(const float* xp, int64_t ldxp, int64_t Np, const float* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, float* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info) {
  remesh_common<float>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,
                       ldf, f_lb, f_ub, info, 3, "ppmg_rmsh_remesh_sv_3d");
}
void ppmg_rmsh_remesh_sv_3d_dev(const float* xp, int64_t ldxp, int64_t Np, const float* up,
                                int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                                const int* ghostsize, float* field_up, int64_t ldf,
                                const int64_t* f_lb, const int64_t* f_ub, int* info,
                                void* stream) {
  remesh_common<float>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,
                       ldf, f_lb, f_ub, info, 3, "ppmg_rmsh_remesh_sv_3d_dev", true,
                       (cudaStream_t)stream);
}
void ppmg_rmsh_remesh_sv_2d(const float* xp, int64_t ldxp, int64_t Np, const float* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, float* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info) {
  remesh_common<float>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,
                       ldf, f_lb, f_ub, info, 2, "ppmg_rmsh_remesh_sv_2d");
}
void ppmg_rmsh_remesh_sv_2d_dev(const float* xp, int64_t ldxp, int64_t Np, const float* up,
                                int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                                const int* ghostsize, float* field_up, int64_t ldf,
                                const int64_t* f_lb, const int64_t* f_ub, int* info,
                                void* stream) {
  remesh_common<float>(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize, field_up,
                       ldf, f_lb, f_ub, info, 2, "ppmg_rmsh_remesh_sv_2d_dev", true,
                       (cudaStream_t)stream);
}

// ---- create_part ---------------------------------------------------------------
extern "C++" {
template <class T>
static void create_part_common(const T* field_up, int64_t ldf, int lda,
                               const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                               int mesh_id, const T* cutoff, const T* cutoff_weights,
                               int resetpos, const T* field_wp, int64_t ldfw, int lda2,
                               int64_t* np, T* up, T* xp, T* wp, int* info,
                               bool dev, cudaStream_t dstream, const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  Handle* h = get_checked(topo_id, mesh_id, hh->dim, caller, info, hh->dim == 3);
  if (!h) return;
  if (lda < 1 || ldf < lda || (field_wp && (lda2 < 1 || ldfw < lda2))) {
    fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": lda / lda2 inconsistent");
    return;
  }
  std::lock_guard<std::mutex> lk(h->mu);
  const int dim = h->dim;
  int lo[3] = {1, 1, 1}, hi[3];
  for (int a = 0; a < dim; ++a) hi[a] = h->g.N[a];
  FieldDesc fd, fdw;
  if (!make_fd(*h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return;
  if (field_wp && !make_fd(*h, ldfw, f_lb, f_ub, lo, hi, fdw, caller, info)) return;
  cudaStream_t st = dev ? dstream : h->stream;
  cudaError_t e = cudaSuccess;
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  const T* dfield = field_up;
  if (!dev) {
    dfield = mirror<T>(h->ws.h_field, field_up, nf, st, e);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  const T* dfw = field_wp;
  if (field_wp && !dev) {
    dfw = mirror<T>(h->ws.h_xp, field_wp, field_elems(*h, ldfw, f_lb, f_ub), st, e);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  const T* dcw = nullptr;
  if (cutoff_weights) {
    dcw = mirror<T>(h->ws.w1d, cutoff_weights, lda, st, e);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  CPParams<T> P{};
  P.dim = dim;
  P.lda = lda;
  P.lda2 = lda2;
  for (int a = 0; a < 3; ++a) {
    // periodic axes, and a z-slab's internal upper face, visit nodes 1..Nm-1
    // (ppm_rmsh_create_part.f:433-453)
    P.nn[a] = a < dim ? h->g.N[a] : 1;
    P.h[a] = (T)h->g.h_d[a];
    P.min_sub[a] = (T)h->g.min_sub[a];
  }
  P.field = dfield;
  P.fd = fd;
  P.field_wp = dfw;
  P.fdw = fdw;
  P.cw = dcw;
  P.cut0 = cutoff[0];
  P.cut1 = cutoff[1];
  const int64_t nq = (int64_t)P.nn[0] * P.nn[1] * P.nn[2];
  if ((e = h->ws.count.ensure(sizeof(int) * (size_t)(nq + 1))) ||
      (e = h->ws.start.ensure(sizeof(int) * (size_t)(nq + 1)))) { cuda_fail(info, e, caller); return; }
  h->sort_cached = false;  // flag / positions reuse the cell-order buffers
  int* flag = h->ws.count.as<int>();
  int* pos = h->ws.start.as<int>();
  if ((e = cudaMemsetAsync(flag + nq, 0, sizeof(int), st))) { cuda_fail(info, e, caller); return; }
  if ((e = launch_cp_flag(P, flag, st))) { cuda_fail(info, e, caller); return; }
  if ((e = scan_exclusive(flag, pos, nq + 1, h->ws, st))) { cuda_fail(info, e, caller); return; }
  int total = 0;
  e = cudaMemcpyAsync(&total, pos + nq, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) { cuda_fail(info, e, caller); return; }
  if (np) *np = total;
  if (!up) return;  // counting call
  if (dev) {
    // device outputs up(lda, np) [, xp(dim, np), wp(lda2, np)]
    P.up = up;
    P.xp = resetpos ? xp : nullptr;
    P.wp = field_wp ? wp : nullptr;
    if ((e = launch_cp_fill(P, flag, pos, st))) cuda_fail(info, e, caller);
    return;
  }
  T* dout = mirror<T>(h->ws.h_aux, (const T*)nullptr,
                                (int64_t)total * (lda + dim + (field_wp ? lda2 : 0)), st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  P.up = dout;
  P.xp = resetpos ? dout + (int64_t)total * lda : nullptr;
  P.wp = field_wp ? dout + (int64_t)total * (lda + dim) : nullptr;
  if ((e = launch_cp_fill(P, flag, pos, st))) { cuda_fail(info, e, caller); return; }
  if (total > 0) {
    e = cudaMemcpyAsync(up, P.up, sizeof(T) * (size_t)total * lda, cudaMemcpyDeviceToHost, st);
    if (!e && resetpos && xp)
      e = cudaMemcpyAsync(xp, P.xp, sizeof(T) * (size_t)total * dim, cudaMemcpyDeviceToHost, st);
    if (!e && field_wp && wp)
      e = cudaMemcpyAsync(wp, P.wp, sizeof(T) * (size_t)total * lda2, cudaMemcpyDeviceToHost, st);
  }
  if (!e) e = cudaStreamSynchronize(st);
  if (e) cuda_fail(info, e, caller);
}
}  // extern "C++"

void ppmg_rmsh_create_part_d(const double* field_up, int64_t ldf, int lda,
                             const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                             int mesh_id, const double* cutoff, const double* cutoff_weights,
                             int resetpos, const double* field_wp, int64_t ldfw, int lda2,
                             int64_t* np, double* up, double* xp, double* wp, int* info) {
  create_part_common(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, cutoff, cutoff_weights,
                     resetpos, field_wp, ldfw, lda2, np, up, xp, wp, info, false, nullptr,
                     "ppmg_rmsh_create_part_d");
}
void ppmg_rmsh_create_part_d_dev(const double* field_up, int64_t ldf, int lda,
                                 const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                                 int mesh_id, const double* cutoff, const double* cutoff_weights,
                                 int resetpos, const double* field_wp, int64_t ldfw, int lda2,
                                 int64_t* np, double* up, double* xp, double* wp, int* info,
                                 void* stream) {
  create_part_common(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, cutoff, cutoff_weights,
                     resetpos, field_wp, ldfw, lda2, np, up, xp, wp, info, true,
                     (cudaStream_t)stream, "ppmg_rmsh_create_part_d_dev");
}
void ppmg_rmsh_create_part_s(const float* field_up, int64_t ldf, int lda,
                             const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                             int mesh_id, const float* cutoff, const float* cutoff_weights,
                             int resetpos, const float* field_wp, int64_t ldfw, int lda2,
                             int64_t* np, float* up, float* xp, float* wp, int* info) {
  create_part_common<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, cutoff,
                            cutoff_weights, resetpos, field_wp, ldfw, lda2, np, up, xp, wp, info,
                            false, nullptr, "ppmg_rmsh_create_part_s");
}
void ppmg_rmsh_create_part_s_dev(const float* field_up, int64_t ldf, int lda,
                                 const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                                 int mesh_id, const float* cutoff, const float* cutoff_weights,
                                 int resetpos, const float* field_wp, int64_t ldfw, int lda2,
                                 int64_t* np, float* up, float* xp, float* wp, int* info,
                                 void* stream) {
  create_part_common<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, cutoff,
                            cutoff_weights, resetpos, field_wp, ldfw, lda2, np, up, xp, wp, info,
                            true, (cudaStream_t)stream, "ppmg_rmsh_create_part_s_dev");
}

// ---- FFT Poisson solver ------------------------------------------------------------
extern "C++" {
// Unique-node boxes moved between two layouts through the caller's transport:
// the send boxes packed from src (node strides ss, lower bounds slb), the
// receive boxes unpacked into dst (dsd, dlb), nc components per node, the
// boxes in each layout's own 1-based node indices.  Blocks to the local
// subdomain are copied on the device (the i-th local send to the i-th local
// receive).  The receive boxes must be disjoint.
template <class T>
int box_transfer(Handle& h, const T* src, const int64_t ss[3], const int slb[3],
                 const std::vector<HaloBox>& sends, T* dst, const int64_t ds[3],
                 const int dlb[3], const std::vector<HaloBox>& recvs, int nc,
                 bool host_transport, cudaStream_t st, int* info, const char* caller) {
  const int ns = (int)sends.size(), nr = (int)recvs.size();
  std::vector<int64_t>& tab = h.halo_tab_host;
  tab.assign(8 * (size_t)(ns + nr), 0);
  std::vector<int64_t> elems(ns + nr);
  int64_t tot[2] = {0, 0};
  for (int i = 0; i < ns + nr; ++i) {
    const HaloBox& b = i < ns ? sends[i] : recvs[i - ns];
    int64_t* t = tab.data() + 8 * (size_t)i;
    int64_t n = nc;
    for (int a = 0; a < 3; ++a) {
      t[a] = b.lo[a];
      t[3 + a] = b.hi[a] - b.lo[a] + 1;
      n *= t[3 + a];
    }
    int64_t& acc = tot[i < ns ? 0 : 1];
    t[6] = acc;
    t[7] = acc;
    elems[i] = n;
    acc += n;
  }
  cudaError_t e = cudaSuccess;
  if ((e = h.halo_tab.ensure(sizeof(int64_t) * (tab.empty() ? 1 : tab.size()))) ||
      (e = h.halo_sbuf.ensure(sizeof(T) * (size_t)(tot[0] > 0 ? tot[0] : 1))) ||
      (e = h.halo_rbuf.ensure(sizeof(T) * (size_t)(tot[1] > 0 ? tot[1] : 1))))
    return cuda_fail(info, e, caller);
  int64_t* dtab = h.halo_tab.as<int64_t>();
  T* sbuf = h.halo_sbuf.as<T>();
  T* rbuf = h.halo_rbuf.as<T>();
  if (!tab.empty() && (e = cudaMemcpyAsync(dtab, tab.data(), sizeof(int64_t) * tab.size(),
                                           cudaMemcpyHostToDevice, st)))
    return cuda_fail(info, e, caller);
  if ((e = launch_box_copy<T>(const_cast<T*>(src), nc, ss, slb, dtab, ns, tot[0], sbuf, kBoxPack,
                              st)))
    return cuda_fail(info, e, caller);
  // blocks to and from other subdomains go through the transport; the local
  // ones pair up in order (the i-th local send is the i-th local receive)
  std::vector<ppmg_halo_block> sb, rb;
  std::vector<int> self_s, self_r;
  for (int i = 0; i < ns; ++i) {
    if (sends[i].peer == h.local_sub) {
      self_s.push_back(i);
      continue;
    }
    sb.push_back({sends[i].peer, sends[i].tag, sbuf + tab[8 * (size_t)i + 7],
                  (int64_t)sizeof(T) * elems[i]});
  }
  for (int i = 0; i < nr; ++i) {
    if (recvs[i].peer == h.local_sub) {
      self_r.push_back(i);
      continue;
    }
    rb.push_back({recvs[i].peer, recvs[i].tag, rbuf + tab[8 * (size_t)(ns + i) + 7],
                  (int64_t)sizeof(T) * elems[ns + i]});
  }
  if (self_s.size() != self_r.size())
    return fail(info, kErrorError, kErrArgument, std::string(caller) + ": inconsistent local blocks");
  for (size_t k = 0; k < self_s.size() && !e; ++k) {
    const int i = self_s[k], j = self_r[k];
    if (elems[i] != elems[ns + j] || sends[i].tag != recvs[j].tag)
      return fail(info, kErrorError, kErrArgument,
                  std::string(caller) + ": inconsistent local blocks");
    e = cudaMemcpyAsync(rbuf + tab[8 * (size_t)(ns + j) + 7], sbuf + tab[8 * (size_t)i + 7],
                        sizeof(T) * (size_t)elems[i], cudaMemcpyDeviceToDevice, st);
  }
  if (e) return cuda_fail(info, e, caller);
  const int rc = run_transport(h, (int)sb.size(), sb.data(), (int)rb.size(), rb.data(),
                               host_transport, st, e);
  if (e) return cuda_fail(info, e, caller);
  if (rc != 0)
    return fail(info, kErrorFatal, 2,
                std::string(caller) + ": the halo transport failed (returned " +
                    std::to_string(rc) + ")");
  if ((e = launch_box_copy<T>(dst, nc, ds, dlb, dtab + 8 * (size_t)ns, nr, tot[1], rbuf, kBoxCopy,
                              st)))
    return cuda_fail(info, e, caller);
  return 0;
}

// The FFT solver on a cut along several axes.  As ppm_fdsolver_solve_3d
// maps the field onto the slab topology it transforms on
// (ppm_fdsolver_map_3d.f), omega's unique nodes go to P virtual z-slabs
// (slab q on subdomain q's process, N2 split evenly), the slab form solves
// there, and phi comes back to every node of each subdomain's
// ghost-extended box (its real nodes, ghost nodes and periodic images), so
// no ghost get follows.  Tags: 200 forward, 300 + shift back.
template <class T>
int poisson_cut(Handle& h, T* field, int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                const int* ghost, int lda, const double len[3], bool host_transport,
                cudaStream_t st, int* info, const char* caller) {
  const int P = h.nsubs, me = h.local_sub;
  int N[3];
  for (int a = 0; a < 3; ++a) N[a] = h.Nm_global[a] - 1;
  if (N[1] < P || N[2] < P)
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": the solve on a cut along several axes needs at least as "
                                      "many y and z cells as subdomains");
  std::vector<int> z0(P), nz(P);
  for (int q = 0; q < P; ++q) {
    z0[q] = (int)((int64_t)N[2] * q / P);
    nz[q] = (int)((int64_t)N[2] * (q + 1) / P) - z0[q];
  }
  // global 1-based node boxes: a subdomain's unique real nodes (the last
  // node of a cut axis is the next subdomain's), its ghost-extended box, a
  // virtual slab's unique nodes
  auto ist = [&](int q, int a) { return (int64_t)h.istart[3 * q + a]; };
  auto nno = [&](int q, int a) { return (int64_t)h.nnodes[3 * q + a]; };
  auto real_u = [&](int q, int a, int64_t& lo, int64_t& hi) {
    lo = h.open[a] ? ist(q, a) : 1;
    hi = h.open[a] ? ist(q, a) + nno(q, a) - 2 : N[a];
  };
  auto gbox = [&](int q, int a, int64_t& lo, int64_t& hi) {
    lo = (h.open[a] ? ist(q, a) : 1) - ghost[a];
    hi = (h.open[a] ? ist(q, a) + nno(q, a) - 1 : N[a] + 1) + ghost[a];
  };
  auto slab_u = [&](int q, int a, int64_t& lo, int64_t& hi) {
    lo = a < 2 ? 1 : z0[q] + 1;
    hi = a < 2 ? N[a] : z0[q] + nz[q];
  };
  auto local_off = [&](int q, int a) { return h.open[a] ? ist(q, a) - 1 : 0; };
  // the slab buffer: lda x N0 x N1 x nz[me], nodes from (1, 1, 1)
  const int64_t sn = (int64_t)lda * N[0] * N[1] * (nz[me] > 0 ? nz[me] : 1);
  cudaError_t e = h.fd_slab.ensure(sizeof(T) * (size_t)sn);
  if (e) return cuda_fail(info, e, caller);
  T* slab = h.fd_slab.as<T>();
  FieldDesc sfd{};
  sfd.s[0] = lda;
  sfd.s[1] = (int64_t)lda * N[0];
  sfd.s[2] = (int64_t)lda * N[0] * N[1];
  const int sub_[3] = {N[0], N[1], nz[me]};
  for (int a = 0; a < 3; ++a) {
    sfd.lb[a] = sfd.box_lo[a] = 1;
    sfd.ub[a] = sfd.box_hi[a] = sub_[a];
  }
  int64_t fs[3];
  int flb[3];
  fs[0] = ldf;
  fs[1] = ldf * (f_ub[0] - f_lb[0] + 1);
  fs[2] = fs[1] * (f_ub[1] - f_lb[1] + 1);
  for (int a = 0; a < 3; ++a) flb[a] = (int)f_lb[a];
  const int slb[3] = {1, 1, 1};
  // forward: R'_me and U_q (one box per pair)
  std::vector<HaloBox> snd, rcv;
  for (int q = 0; q < P; ++q) {
    HaloBox b;
    bool ok = true;
    for (int a = 0; a < 3 && ok; ++a) {
      int64_t rl, rh, ul, uh;
      real_u(me, a, rl, rh);
      slab_u(q, a, ul, uh);
      b.lo[a] = rl > ul ? rl : ul;
      b.hi[a] = rh < uh ? rh : uh;
      ok = b.lo[a] <= b.hi[a];
      b.lo[a] -= local_off(me, a);
      b.hi[a] -= local_off(me, a);
    }
    if (ok) {
      b.peer = q;
      b.tag = 200;
      snd.push_back(b);
    }
    ok = true;
    for (int a = 0; a < 3 && ok; ++a) {
      int64_t rl, rh, ul, uh;
      real_u(q, a, rl, rh);
      slab_u(me, a, ul, uh);
      b.lo[a] = rl > ul ? rl : ul;
      b.hi[a] = rh < uh ? rh : uh;
      ok = b.lo[a] <= b.hi[a];
      if (a == 2) {
        b.lo[a] -= z0[me];
        b.hi[a] -= z0[me];
      }
    }
    if (ok) {
      b.peer = q;
      b.tag = 200;
      rcv.push_back(b);
    }
  }
  for (const HaloBox& b : snd)
    for (int a = 0; a < 3; ++a)
      if (b.lo[a] < f_lb[a] || b.hi[a] > f_ub[a])
        return fail(info, kErrorError, kErrArgument,
                    std::string(caller) + ": field_up bounds do not cover the real nodes");
  if (box_transfer<T>(h, field, fs, flb, snd, slab, sfd.s, slb, rcv, lda, host_transport, st, info,
                      caller))
    return *info;
  // the slab solve
  SlabSolve sl;
  sl.P = P;
  sl.me = me;
  for (int a = 0; a < 3; ++a) {
    sl.N[a] = N[a];
    sl.len[a] = len[a];
  }
  sl.z0 = z0.data();
  sl.nz = nz.data();
  cudaError_t te = cudaSuccess;
  BlockExchange xchg = [&](int ns, const ppmg_halo_block* sb, int nr, const ppmg_halo_block* rb) {
    const int rc = run_transport(h, ns, sb, nr, rb, host_transport, st, te);
    return te ? 1 : rc;
  };
  const int bad = fd_poisson_slab<T>(h.fft_slab, h.ws_fd, sl, slab, sfd, lda, st, xchg, e);
  if (!e) e = te;
  if (bad == 2)
    return fail(info, kErrorFatal, 2, std::string(caller) + ": the halo transport failed");
  if (bad)
    return fail(info, kErrorError, kErrArgument,
                std::string(caller) + ": cuFFT plan or transform failed");
  if (e) return cuda_fail(info, e, caller);
  // back: G_q and (U_me + tN) from the slab, G_me and (U_q + tN) into the field
  snd.clear();
  rcv.clear();
  auto dir = [](const int t[3]) { return (t[0] + 1) + 3 * (t[1] + 1) + 9 * (t[2] + 1); };
  for (int q = 0; q < P; ++q) {
    int t[3];
    for (t[2] = -1; t[2] <= 1; ++t[2])
      for (t[1] = -1; t[1] <= 1; ++t[1])
        for (t[0] = -1; t[0] <= 1; ++t[0]) {
          HaloBox b;
          bool ok = true;
          for (int a = 0; a < 3 && ok; ++a) {  // me sends to q, in my slab's nodes
            int64_t gl, gh, ul, uh;
            gbox(q, a, gl, gh);
            slab_u(me, a, ul, uh);
            ul += (int64_t)t[a] * N[a];
            uh += (int64_t)t[a] * N[a];
            b.lo[a] = gl > ul ? gl : ul;
            b.hi[a] = gh < uh ? gh : uh;
            ok = b.lo[a] <= b.hi[a];
            const int64_t o = (int64_t)t[a] * N[a] + (a == 2 ? z0[me] : 0);
            b.lo[a] -= o;
            b.hi[a] -= o;
          }
          if (ok) {
            b.peer = q;
            b.tag = 300 + dir(t);
            snd.push_back(b);
          }
          ok = true;
          for (int a = 0; a < 3 && ok; ++a) {  // me receives from q, in my field's nodes
            int64_t gl, gh, ul, uh;
            gbox(me, a, gl, gh);
            slab_u(q, a, ul, uh);
            ul += (int64_t)t[a] * N[a];
            uh += (int64_t)t[a] * N[a];
            b.lo[a] = gl > ul ? gl : ul;
            b.hi[a] = gh < uh ? gh : uh;
            ok = b.lo[a] <= b.hi[a];
            b.lo[a] -= local_off(me, a);
            b.hi[a] -= local_off(me, a);
          }
          if (ok) {
            b.peer = q;
            b.tag = 300 + dir(t);
            rcv.push_back(b);
          }
        }
  }
  if (box_transfer<T>(h, slab, sfd.s, slb, snd, field, fs, flb, rcv, lda, host_transport, st, info,
                      caller))
    return *info;
  return 0;
}

template <class T>
static void poisson_common(T* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                           const int64_t* f_ub, int topo_id, int mesh_id, const int* ghostsize,
                           int* info, bool dev, cudaStream_t dstream, const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  // a z-slab solves with the other slabs through its halo transport
  Handle* h = get_checked(topo_id, mesh_id, 3, caller, info, hh->halo_fn != nullptr);
  if (!h) return;
  if (lda < 1 || ldf < lda) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": lda inconsistent"); return; }
  if (!check_ghost(*h, ghostsize, caller, info)) return;
  if (h->slab() && h->g.N[1] < h->nsubs) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": the slab solve needs at least as many y cells as slabs"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = 1 - ghostsize[a];
    hi[a] = h->Nm[a] + ghostsize[a];
  }
  FieldDesc fd;
  if (!make_fd(*h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return;
  cudaStream_t st = dev ? dstream : h->stream;
  cudaError_t e = cudaSuccess;
  const int64_t nf = field_elems(*h, ldf, f_lb, f_ub);
  T* dfield = field_up;
  if (!dev) {
    dfield = mirror<T>(h->ws.h_field, field_up, nf, st, e);
    if (e) { cuda_fail(info, e, caller); return; }
  }
  double len[3];
  for (int a = 0; a < 3; ++a) len[a] = h->g.max_phys[a] - h->g.min_phys[a];
  int bad = 0;
  if (h->slab()) {
    // ppm_fdsolver_solve_slab: xy transforms on the slab, z on the pencils
    std::vector<int> z0(h->nsubs), nz(h->nsubs);
    for (int q = 0; q < h->nsubs; ++q) {
      z0[q] = h->istart[3 * q + 2] - 1;
      nz[q] = h->nnodes[3 * q + 2] - 1;
    }
    SlabSolve sl;
    sl.P = h->nsubs;
    sl.me = h->local_sub;
    sl.N[0] = h->g.N[0];
    sl.N[1] = h->g.N[1];
    sl.N[2] = h->Nm_global[2] - 1;
    for (int a = 0; a < 3; ++a) sl.len[a] = len[a];
    sl.z0 = z0.data();
    sl.nz = nz.data();
    cudaError_t te = cudaSuccess;
    BlockExchange xchg = [&](int ns, const ppmg_halo_block* sb, int nr,
                             const ppmg_halo_block* rb) {
      const int rc = run_transport(*h, ns, sb, nr, rb, !dev, st, te);
      return te ? 1 : rc;
    };
    bad = fd_poisson_slab<T>(h->fft_slab, h->ws_fd, sl, dfield, fd, lda, st, xchg, e);
    if (!e) e = te;
    if (bad == 2) {
      fail(info, kErrorFatal, 2, std::string(caller) + ": the halo transport failed");
      return;
    }
    // the shared upper plane (node nz+1, the slab above's plane 1), then the
    // z ghost planes, from the neighbours
    if (!bad && !e) {
      HaloPlan pl;
      const char* why = halo_plan(h->nsubs, h->istart.data(), h->nnodes.data(), h->Nm_global[2],
                                  h->local_sub, ldf, f_lb, f_ub, 0, true, pl);
      if (why) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": " + why); return; }
      // with g = 0 the put's blocks are single planes: nz+1 up, 1 down; the
      // plane 1 travelling down replaces the lower slab's plane nz+1
      const int64_t plane = pl.count;
      const int nzl = h->g.N[2];
      ppmg_halo_block sb = {pl.send_peer[1], 19, dfield + pl.send_off[1],
                            (int64_t)(sizeof(T) * plane)};
      ppmg_halo_block rb = {pl.recv_peer[1], 19,
                            dfield + (int64_t)(nzl + 1 - f_lb[2]) * plane,
                            (int64_t)(sizeof(T) * plane)};
      const int rc = run_transport(*h, 1, &sb, 1, &rb, !dev, st, e);
      if (e) { cuda_fail(info, e, caller); return; }
      if (rc) { fail(info, kErrorFatal, 2, std::string(caller) + ": the halo transport failed"); return; }
      if (slab_exchange<T>(*h, dfield, ldf, f_lb, f_ub, ghostsize, false, !dev, st, info, caller))
        return;
    }
  } else if (h->cut()) {
    // a cut along several axes: through virtual z-slabs and back
    if (poisson_cut<T>(*h, dfield, ldf, f_lb, f_ub, ghostsize, lda, len, !dev, st, info, caller))
      return;
  } else {
    bad = fd_poisson<T>(h->fft, h->ws_fd, h->g.N, len, dfield, fd, lda, st, e);
  }
  if (bad) {
    fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": cuFFT plan or transform failed");
    return;
  }
  if (e) { cuda_fail(info, e, caller); return; }
  if (!dev) {
    e = cudaMemcpyAsync(field_up, dfield, sizeof(T) * (size_t)nf, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) cuda_fail(info, e, caller);
  }
}
}  // extern "C++"

void ppmg_fdsolver_poisson_3d_d(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int* info) {
  poisson_common<double>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, info, false,
                         nullptr, "ppmg_fdsolver_poisson_3d_d");
}
void ppmg_fdsolver_poisson_3d_s(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int* info) {
  poisson_common<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, info, false,
                        nullptr, "ppmg_fdsolver_poisson_3d_s");
}
void ppmg_fdsolver_poisson_3d_d_dev(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                    const int64_t* f_ub, int topo_id, int mesh_id,
                                    const int* ghostsize, int* info, void* stream) {
  poisson_common<double>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, info, true,
                         (cudaStream_t)stream, "ppmg_fdsolver_poisson_3d_d_dev");
}
void ppmg_fdsolver_poisson_3d_s_dev(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                    const int64_t* f_ub, int topo_id, int mesh_id,
                                    const int* ghostsize, int* info, void* stream) {
  poisson_common<float>(field_up, ldf, lda, f_lb, f_ub, topo_id, mesh_id, ghostsize, info, true,
                        (cudaStream_t)stream, "ppmg_fdsolver_poisson_3d_s_dev");
}

// ---- particle routing between z-slab subdomains -------------------------------------
extern "C++" {
template <class T>
static void route_common(const T* xp, int64_t ldxp, int64_t Np, int topo_id, int mesh_id,
                         int* perm, int64_t* counts, int* info, cudaStream_t st,
                         const char* caller) {
  clear_error();
  if (info) *info = 0;
  Handle* hh = find_handle(topo_id, mesh_id);
  if (!hh) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": topo_id/mesh_id is invalid"); return; }
  Handle* h = get_checked(topo_id, mesh_id, 3, caller, info, true);
  if (!h) return;
  if (Np < 0 || (Np > 0 && ldxp < 3) || Np >= (int64_t)1 << 31) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes"); return; }
  if (h->cut() && !h->slab()) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": routing to the neighbours supports slabs along z only (ppmg_map_part_global_route routes on any decomposition)"); return; }
  std::lock_guard<std::mutex> lk(h->mu);
  // the local slab and its z neighbours (periodic across the domain's z faces)
  RouteParams R{};
  const int s = h->local_sub;
  const double zmin = h->g.min_phys[2], zmax = h->g.max_phys[2];
  auto box = [&](int c, int sub) {
    R.zlo[c] = h->min_sub[3 * sub + 2];
    R.zhi[c] = h->max_sub[3 * sub + 2];
    R.zlof[c] = (float)R.zlo[c];
    R.zhif[c] = (float)R.zhi[c];
  };
  for (int c = 0; c < 3; ++c) R.zlo[c] = R.zhi[c] = 0.0, R.zlof[c] = R.zhif[c] = 0.0f;
  box(0, s);
  if (h->slab()) {
    const double lo = h->min_sub[3 * s + 2], hi = h->max_sub[3 * s + 2];
    for (int q = 0; q < h->nsubs; ++q) {
      if (q == s) continue;
      if (h->max_sub[3 * q + 2] == (lo > zmin ? lo : zmax)) box(1, q);
      if (h->min_sub[3 * q + 2] == (hi < zmax ? hi : zmin)) box(2, q);
    }
  }
  for (int a = 0; a < 2; ++a) {
    R.lo[a] = h->g.min_sub[a];
    R.hi[a] = h->g.max_sub[a];
    R.lof[a] = (float)R.lo[a];
    R.hif[a] = (float)R.hi[a];
  }
  if (counts)
    for (int c = 0; c < 4; ++c) counts[c] = 0;
  if (Np == 0) return;
  const int nblk = route_blocks(Np);
  Workspace& ws = h->ws_map;
  cudaError_t e;
  if ((e = ws.key.ensure((size_t)Np)) || (e = ws.count.ensure(sizeof(int) * 4 * (size_t)nblk)) ||
      (e = ws.start.ensure(sizeof(int) * 4 * (size_t)nblk))) { cuda_fail(info, e, caller); return; }
  if ((e = launch_route<T>(R, xp, ldxp, Np, static_cast<unsigned char*>(ws.key.p),
                           ws.count.as<int>(), ws.start.as<int>(), perm, ws, st))) {
    cuda_fail(info, e, caller);
    return;
  }
  // class starts: off[c * nblk] (c = 1..3); the call returns once they are read
  int st4[4] = {0, 0, 0, 0};
  for (int c = 1; c < 4 && !e; ++c)
    e = cudaMemcpyAsync(st4 + c, ws.start.as<int>() + (size_t)c * nblk, sizeof(int),
                        cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) { cuda_fail(info, e, caller); return; }
  if (counts) {
    counts[0] = st4[1];
    counts[1] = st4[2] - st4[1];
    counts[2] = st4[3] - st4[2];
    counts[3] = Np - st4[3];
  }
  if (Np - st4[3] > 0)
    fail(info, kErrorError, kErrPartUnass,
         std::string(caller) + ": " + std::to_string(Np - st4[3]) +
             " particles lie in no neighbouring subdomain");
}

// ppm_map_part_global on z-slabs: every particle to the slab that contains it
// (ppm_map_part_global.f:355-420).  counts[0..nsubs]: particles per slab, then
// those in none (dropped without an error, ppm_map_part_global.f:437-442).
template <class T>
static void groute_common(const T* xp, int64_t ldxp, int64_t Np, int topo_id, int mesh_id,
                          int* perm, int64_t* counts, int* info, cudaStream_t st,
                          const char* caller, bool partial = false) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < 3) || Np >= (int64_t)1 << 31) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes"); return; }
  Handle* h = get_checked(topo_id, mesh_id, 3, caller, info, true);
  if (!h) return;
  std::lock_guard<std::mutex> lk(h->mu);
  const int ns = h->nsubs;
  if (ns > kMaxGlobalSubs) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": more than 255 subdomains"); return; }
  if (ns > 1 && !h->cut()) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": select the local subdomain first (ppmg_mesh_set_local_sub)"); return; }
  if (counts)
    for (int c = 0; c <= ns; ++c) counts[c] = 0;
  if (Np == 0) return;
  GlobalRouteParams R{};
  R.nsubs = ns;
  const int nblk = route_blocks(Np);
  Workspace& ws = h->ws_map;
  const size_t ncls = (size_t)ns + 1;
  cudaError_t e;
  if ((e = ws.key.ensure((size_t)Np)) || (e = ws.count.ensure(sizeof(int) * ncls * nblk)) ||
      (e = ws.start.ensure(sizeof(int) * ncls * nblk)) ||
      (e = ws.h_aux.ensure(sizeof(double) * 6 * (size_t)ns))) { cuda_fail(info, e, caller); return; }
  // the subdomain boxes, [6][ns]: min_sub x, y, z, then max_sub x, y, z
  std::vector<double> zb(6 * (size_t)ns);
  std::vector<char> reach(ns, 1);
  if (partial) {
    // ppm_map_part_partial: the local subdomain and its neighbours only; the
    // others get empty boxes, so their particles land in no subdomain
    std::vector<int> nb;
    cart_neighbours(ns, h->istart.data(), h->nnodes.data(), h->Nm_global, h->local_sub, nb);
    std::fill(reach.begin(), reach.end(), 0);
    reach[h->local_sub] = 1;
    for (int q : nb) reach[q] = 1;
  }
  for (int q = 0; q < ns; ++q)
    for (int a = 0; a < 3; ++a) {
      zb[a * ns + q] = reach[q] ? h->min_sub[3 * q + a] : 0.0;
      zb[(3 + a) * ns + q] = reach[q] ? h->max_sub[3 * q + a] : 0.0;
    }
  double* dz = ws.h_aux.as<double>();
  if ((e = cudaMemcpyAsync(dz, zb.data(), sizeof(double) * 6 * ns, cudaMemcpyHostToDevice, st))) { cuda_fail(info, e, caller); return; }
  R.box = dz;
  if ((e = launch_route_global<T>(R, xp, ldxp, Np, static_cast<unsigned char*>(ws.key.p),
                                  ws.count.as<int>(), ws.start.as<int>(), perm, ws, st))) {
    cuda_fail(info, e, caller);
    return;
  }
  // class starts off[c * nblk]; the call returns once they are read (zb's
  // staging also lives until then)
  std::vector<int> cs(ncls, 0);
  for (size_t c = 1; c < ncls && !e; ++c)
    e = cudaMemcpyAsync(&cs[c], ws.start.as<int>() + c * nblk, sizeof(int),
                        cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) { cuda_fail(info, e, caller); return; }
  if (counts)
    for (size_t c = 0; c < ncls; ++c)
      counts[c] = (c + 1 < ncls ? cs[c + 1] : (int)Np) - cs[c];
  // ppm_map_part_partial.f:480-485: particles beyond the neighbours are an error
  const int64_t lost = Np - cs[ns];
  if (partial && lost > 0)
    fail(info, kErrorError, kErrPartUnass,
         std::string(caller) + ": " + std::to_string(lost) +
             " particles lie in no neighbouring subdomain (ppm_map_part_global moves them)");
}

template <class T>
static void gather_common(const T* src, int64_t lds, int lda, const int* perm, int64_t n, T* dst,
                          int64_t ldd, int* info, cudaStream_t st, const char* caller) {
  clear_error();
  if (info) *info = 0;
  if (n < 0 || lda < 1 || lds < lda || ldd < lda) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes"); return; }
  cudaError_t e = launch_gather_cols<T>(src, lds, lda, perm, n, dst, ldd, st);
  if (e) cuda_fail(info, e, caller);
}
}  // extern "C++"

void ppmg_map_part_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                               int mesh_id, int* perm, int64_t* counts, int* info,
                               void* stream) {
  route_common<double>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                       "ppmg_map_part_route_d_dev");
}
void ppmg_map_part_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                               int mesh_id, int* perm, int64_t* counts, int* info,
                               void* stream) {
  route_common<float>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                      "ppmg_map_part_route_s_dev");
}
void ppmg_map_part_global_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                      int mesh_id, int* perm, int64_t* counts, int* info,
                                      void* stream) {
  groute_common<double>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                        "ppmg_map_part_global_route_d_dev");
}
void ppmg_map_part_global_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                      int mesh_id, int* perm, int64_t* counts, int* info,
                                      void* stream) {
  groute_common<float>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                       "ppmg_map_part_global_route_s_dev");
}
void ppmg_map_part_partial_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                       int mesh_id, int* perm, int64_t* counts, int* info,
                                       void* stream) {
  groute_common<double>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                        "ppmg_map_part_partial_route_d_dev", true);
}
void ppmg_map_part_partial_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                       int mesh_id, int* perm, int64_t* counts, int* info,
                                       void* stream) {
  groute_common<float>(xp, ldxp, Np, topo_id, mesh_id, perm, counts, info, (cudaStream_t)stream,
                       "ppmg_map_part_partial_route_s_dev", true);
}
void ppmg_halo_neighbours(int nsubs, const int* istart, const int* nnodes, const int* Nm,
                          int isub, int cap, int* neigh, int* nneigh, int* info) {
  clear_error();
  if (info) *info = 0;
  if (isub < 0 || isub >= nsubs) { fail(info, kErrorError, ppmg::kErrArgument, "ppmg_halo_neighbours: isub out of range"); return; }
  if (const char* why = check_cartesian(nsubs, istart, nnodes, Nm)) { fail(info, kErrorError, ppmg::kErrArgument, std::string("ppmg_halo_neighbours: ") + why); return; }
  std::vector<int> nb;
  cart_neighbours(nsubs, istart, nnodes, Nm, isub, nb);
  *nneigh = (int)nb.size();
  for (int i = 0; i < (int)nb.size() && i < cap; ++i) neigh[i] = nb[i];
}
void ppmg_map_part_gather_d_dev(const double* src, int64_t lds, int lda, const int* perm,
                                int64_t n, double* dst, int64_t ldd, int* info, void* stream) {
  gather_common<double>(src, lds, lda, perm, n, dst, ldd, info, (cudaStream_t)stream,
                        "ppmg_map_part_gather_d_dev");
}
void ppmg_map_part_gather_s_dev(const float* src, int64_t lds, int lda, const int* perm,
                                int64_t n, float* dst, int64_t ldd, int* info, void* stream) {
  gather_common<float>(src, lds, lda, perm, n, dst, ldd, info, (cudaStream_t)stream,
                       "ppmg_map_part_gather_s_dev");
}

// ---- cell lists -------------------------------------------------------------------
extern "C++" {
// T: the precision of ppm_util_rank{2,3}d_{s,d} (positions, bounds and the
// cell spacing rdx = REAL(Nm)/(xmax - xmin) in REAL(MK), ppm_util_rank3d.f:353).
template <class T>
static void rank_common(int dim, const T* xp, int64_t ldxp, int64_t Np, const T* xmin,
                        const T* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                        int64_t* icount, int* info, const char* caller, bool dev = false,
                        cudaStream_t dstream = nullptr) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < dim) || Np >= (int64_t)1 << 31) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": invalid sizes"); return; }
  ClistParams cp{};
  cp.dim = dim;
  int64_t nbox = 1;
  for (int a = 0; a < 3; ++a) {
    cp.Nm[a] = a < dim ? Nm[a] : 1;
    cp.Nt[a] = a < dim ? Nm[a] + Ngl[a] + Ngl[dim + a] : 1;
    cp.xmin[a] = a < dim ? (double)xmin[a] : 0.0;
    cp.xmax[a] = a < dim ? (double)xmax[a] : 1.0;
    cp.rd[a] = a < dim ? (double)Nm[a] / ((double)xmax[a] - (double)xmin[a]) : 1.0;
    cp.xminf[a] = a < dim ? (float)xmin[a] : 0.0f;
    cp.xmaxf[a] = a < dim ? (float)xmax[a] : 1.0f;
    cp.rdf[a] = a < dim ? (float)Nm[a] / ((float)xmax[a] - (float)xmin[a]) : 1.0f;
    nbox *= cp.Nt[a];
  }
  for (int a = 0; a < dim; ++a) {
    cp.Ngl[a] = Ngl[a];
    if (Nm[a] <= 0 || !(xmax[a] > xmin[a])) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": Nm must be > 0 and xmax > xmin"); return; }
  }
  if (nbox >= ((int64_t)1 << 31) - 1) { fail(info, kErrorError, ppmg::kErrArgument, std::string(caller) + ": too many boxes"); return; }
  // a private workspace per call: cell lists are independent of any mesh handle
  static std::mutex mu;
  static Workspace& ws = *new Workspace();  // never destroyed (see handles())
  static cudaStream_t st = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  cudaError_t e = cudaSuccess;
  if (!st) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e) { cuda_fail(info, e, caller); return; }
  if (dev) {
    // device positions and lists on the caller's stream; the workspace is
    // shared by every call, so the call returns once its lists are written
    if ((e = clist_sort<T>(cp, xp, ldxp, Np, nbox, ws, dstream)) ||
        (e = launch_plus_one(ws.idx.as<int>(), lpdx, Np, dstream)) ||
        (e = launch_plus_one(ws.start.as<int>(), lhbx, nbox + 1, dstream))) {
      cuda_fail(info, e, caller);
      return;
    }
    int nd = 0;
    e = cudaMemcpyAsync(&nd, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, dstream);
    if (!e) e = cudaStreamSynchronize(dstream);
    if (e) { cuda_fail(info, e, caller); return; }
    if (icount) *icount = nd;
    return;
  }
  const T* dxp = mirror<T>(ws.h_xp, xp, ldxp * Np, st, e);
  if (e) { cuda_fail(info, e, caller); return; }
  if ((e = clist_sort<T>(cp, dxp, ldxp, Np, nbox, ws, st))) { cuda_fail(info, e, caller); return; }
  int nin = 0;
  e = cudaMemcpyAsync(&nin, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!e) e = ws.h_aux.ensure(sizeof(int) * (size_t)(Np + nbox + 2));
  if (e) { cuda_fail(info, e, caller); return; }
  int* dl = ws.h_aux.as<int>();
  int* dh = dl + (Np > 0 ? Np : 1);
  if ((e = launch_plus_one(ws.idx.as<int>(), dl, Np, st)) ||
      (e = launch_plus_one(ws.start.as<int>(), dh, nbox + 1, st))) { cuda_fail(info, e, caller); return; }
  e = cudaStreamSynchronize(st);
  if (!e && nin > 0) e = cudaMemcpy(lpdx, dl, sizeof(int) * (size_t)nin, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(lhbx, dh, sizeof(int) * (size_t)(nbox + 1), cudaMemcpyDeviceToHost);
  if (e) { cuda_fail(info, e, caller); return; }
  if (icount) *icount = nin;
}
}  // extern "C++"

void ppmg_util_rank3d_d(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                        const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info) {
  rank_common(3, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank3d_d");
}
void ppmg_util_rank2d_d(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                        const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info) {
  rank_common(2, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank2d_d");
}
void ppmg_util_rank3d_d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                            const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream) {
  rank_common(3, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank3d_d_dev", true, (cudaStream_t)stream);
}
void ppmg_util_rank2d_d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                            const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream) {
  rank_common(2, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank2d_d_dev", true, (cudaStream_t)stream);
}
void ppmg_util_rank3d_s_dev(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                            const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream) {
  rank_common(3, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank3d_s_dev", true, (cudaStream_t)stream);
}
void ppmg_util_rank2d_s_dev(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                            const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream) {
  rank_common(2, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank2d_s_dev", true, (cudaStream_t)stream);
}
void ppmg_util_rank3d_s(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                        const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info) {
  rank_common(3, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank3d_s");
}
void ppmg_util_rank2d_s(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                        const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info) {
  rank_common(2, xp, ldxp, Np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount, info,
              "ppmg_util_rank2d_s");
}

}  // extern "C"

// ===========================================================================
// Device-time instrumentation (ppmg_kernel_timing).
// ===========================================================================
namespace ppmg {
namespace {
std::atomic<bool> g_timing{false};
struct TimedPair {
  int part;
  cudaEvent_t begin, end;
};
std::mutex g_tmu;
// heap-allocated and never destroyed (no CUDA calls from static destructors)
std::vector<TimedPair>& pending() {
  static auto* v = new std::vector<TimedPair>();
  return *v;
}
std::vector<cudaEvent_t>& spare_events() {
  static auto* v = new std::vector<cudaEvent_t>();
  return *v;
}
cudaEvent_t take_event() {
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    if (!spare_events().empty()) {
      cudaEvent_t ev = spare_events().back();
      spare_events().pop_back();
      return ev;
    }
  }
  cudaEvent_t ev = nullptr;
  if (cudaEventCreate(&ev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return ev;
}
}  // namespace

TimingScope::TimingScope(int part, cudaStream_t st) : part_(part), st_(st) {
  if (part < 0 || part >= kTimedParts || !g_timing.load(std::memory_order_relaxed)) return;
  begin_ = take_event();
  if (begin_ && cudaEventRecord(begin_, st_) != cudaSuccess) {
    cudaGetLastError();
    begin_ = nullptr;
  }
}

TimingScope::~TimingScope() {
  if (!begin_) return;
  cudaEvent_t end = take_event();
  if (!end) return;
  if (cudaEventRecord(end, st_) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  std::lock_guard<std::mutex> lk(g_tmu);
  pending().push_back({part_, begin_, end});
}
}  // namespace ppmg

extern "C" void ppmg_kernel_timing(int enable) { ppmg::g_timing.store(enable != 0); }

extern "C" int ppmg_kernel_timing_read(int part, double* ms, int64_t* launches) {
  using namespace ppmg;
  if (part < 0 || part >= kTimedParts) return kErrorError;
  std::vector<TimedPair> mine;
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    auto& p = pending();
    for (size_t i = 0; i < p.size();) {
      if (p[i].part == part) {
        mine.push_back(p[i]);
        p[i] = p.back();
        p.pop_back();
      } else {
        ++i;
      }
    }
  }
  double total = 0.0;
  for (const TimedPair& t : mine) {
    float el = 0.f;
    if (cudaEventSynchronize(t.end) == cudaSuccess &&
        cudaEventElapsedTime(&el, t.begin, t.end) == cudaSuccess)
      total += el;
    else
      cudaGetLastError();
  }
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    for (const TimedPair& t : mine) {
      spare_events().push_back(t.begin);
      spare_events().push_back(t.end);
    }
  }
  if (ms) *ms = total;
  if (launches) *launches = (int64_t)mine.size();
  return 0;
}

// ===========================================================================
// P2M without allocation (ppmg_interp_p2m_dv_3d_noalloc).
//
// Some callers cannot let this library call cudaMalloc: a simulation that
// hands nearly all of the GPU's memory to its own pool at start-up (a library
// allocation then fails or fragments that pool), and a time-step loop that
// must not stall, since cudaFree -- and cudaMalloc when the driver has to map
// fresh memory -- synchronises the whole device.  This variant of the device
// P2M keeps its sort and tile scratch in one fixed array compiled into the
// library instead of the mesh handle's growable workspace.  The array is
// modest (kNoAllocBytes = 16 MiB) but every GPU that loads the library holds
// it until the process exits.
// ===========================================================================

// The scratch of every noalloc call on a device.  In host code this name is a
// host-side stand-in for the device array, not a device address: the device
// address comes from cudaGetSymbolAddress, once per device.
static constexpr size_t kNoAllocBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char ppmg_noalloc_scratch[kNoAllocBytes];

namespace ppmg {
namespace {

constexpr int64_t kNoAllocMaxParticles = 131072;
constexpr int64_t kNoAllocMaxCells = 262144;
constexpr int kNoAllocMaxLda = 4;
constexpr int kNoAllocMaxDevices = 64;

std::mutex g_noalloc_mu;
void* g_noalloc_base[kNoAllocMaxDevices] = {};
CUcontext g_noalloc_ctx[kNoAllocMaxDevices] = {};

// The calling thread's current CUDA context (the device's primary context for
// runtime-API callers), through the driver entry point the runtime exposes,
// so that the library needs no link-time dependency on libcuda.
CUcontext current_context() {
  static PFN_cuCtxGetCurrent_v4000 get = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
  }();
  CUcontext c = nullptr;
  if (get == nullptr || get(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Device address of the scratch array on the current device.  The first call
// on a device looks it up (which may load this library's device code there).
// The address belongs to the device's context: after a cudaDeviceReset the
// next call finds a new context and looks the address up again.
void* noalloc_scratch(int* info, const char* caller) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { cuda_fail(info, e, caller); return nullptr; }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": device ordinal >= 64");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  // no current context yet (a thread's first CUDA call) also means a lookup,
  // which makes the device's primary context current
  const CUcontext ctx = current_context();
  if (g_noalloc_base[dev] == nullptr || ctx == nullptr || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, ppmg_noalloc_scratch);
    if (e != cudaSuccess) { cuda_fail(info, e, caller); return nullptr; }
    if (p == nullptr) {
      fail(info, kErrorFatal, 602, std::string(caller) + ": scratch array has no device address");
      return nullptr;
    }
    g_noalloc_base[dev] = p;
    g_noalloc_ctx[dev] = current_context();
  }
  return g_noalloc_base[dev];
}

// Carves the sort and tile buffers of one P2M out of the scratch array as
// fixed views (no buffer can grow, so nothing is allocated).  Returns false
// when they do not fit.
bool noalloc_views(Workspace& ws, void* base, int64_t np, int64_t ncell, int lda, bool fp64,
                   const int N[3]) {
  size_t off = 0;
  auto view = [&](DevBuf& b, size_t n) {
    n = (n + 255) & ~size_t(255);
    b.fixed = true;
    b.p = static_cast<unsigned char*>(base) + off;
    b.bytes = n;
    off += n;
  };
  const size_t pn = sizeof(int) * (size_t)(np > 0 ? np : 1);
  view(ws.key, pn);
  view(ws.slot, pn);
  view(ws.idx, pn);
  view(ws.count, sizeof(int) * (size_t)(ncell + 1));
  view(ws.start, sizeof(int) * (size_t)(ncell + 1));
  view(ws.err, sizeof(int) * 4);
  view(ws.big, sizeof(int) * (size_t)(ncell + 2));
  view(ws.bsum, sizeof(int) * (size_t)(ncell / 1024 + 16));  // scan block sums
  const size_t vsz = fp64 ? sizeof(double4) : sizeof(float4);
  const size_t n = (size_t)(np > 0 ? np : 1);
  view(ws.rec, vsz * n);
  view(ws.us, vsz * n * (size_t)((lda + 3) / 4));
  view(ws.tiles, p2m_scratch_bytes(3, N));
  return off <= kNoAllocBytes;
}

void p2m_noalloc(const double* xp, int64_t ldxp, int64_t Np, const double* up, int64_t ldup,
                 int lda, int topo_id, int mesh_id, int kernel, const int* ghost, double* field,
                 int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int* info,
                 cudaStream_t st, const char* caller) {
  clear_error();
  if (info) *info = 0;
  if (Np < 0 || (Np > 0 && ldxp < 3) || lda < 1 || ldup < lda || ldf < lda) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": invalid sizes");
    return;
  }
  if (!check_kernel(kernel, caller, info)) return;
  Handle* h = get_checked(topo_id, mesh_id, 3, caller, info);
  if (!h) return;
  if (Np > kNoAllocMaxParticles || h->g.ncell > kNoAllocMaxCells || lda > kNoAllocMaxLda) {
    fail(info, kErrorError, kErrArgument,
         std::string(caller) + ": beyond the fixed scratch (Np <= 131072, Nx*Ny*Nz <= 262144 "
                               "cells, lda <= 4); use ppmg_interp_p2m_dv_3d_dev");
    return;
  }
  void* base = noalloc_scratch(info, caller);
  if (!base) return;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!check_ghost(*h, ghost, caller, info)) return;
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = 1 - ghost[a];
    hi[a] = h->Nm[a] + ghost[a];
  }
  FieldDesc fd;
  if (!make_fd(*h, ldf, f_lb, f_ub, lo, hi, fd, caller, info)) return;
  const P2MPrec prec = g_precision.load() == PPMG_PREC_MIXED ? P2M_MIXED : P2M_FP64;
  P2MParams P{};
  for (int a = 0; a < 3; ++a) P.N[a] = h->g.N[a];
  Workspace ws;  // fixed views only: its destructor frees nothing
  if (!noalloc_views(ws, base, Np, h->g.ncell, lda, prec == P2M_FP64, P.N)) {
    fail(info, kErrorError, kErrArgument, std::string(caller) + ": beyond the fixed scratch");
    return;
  }
  // Everything that must start at zero (cell counts, the big-cell list, the
  // work-item counter) is cleared on the stream by the sort and item builders;
  // the rest of the array is written before it is read.
  const KeyParams kp = make_kp(*h, KEY_INTERP_CHECKED, false);
  cudaError_t e = bin_sort<double>(kp, xp, ldxp, Np, h->g.ncell, ws, h->d_status + 0, st);
  if (e) { cuda_fail(info, e, caller); return; }
  const int* dnv = d_nvalid_of(ws, h->g.ncell);
  if (prec == P2M_FP64)
    e = pack_records<double, double>(kp, xp, ldxp, up, ldup, lda, Np, dnv, ws, st);
  else
    e = pack_records<double, float>(kp, xp, ldxp, up, ldup, lda, Np, dnv, ws, st);
  if (e) { cuda_fail(info, e, caller); return; }
  P.TZ = p2m_tile_depth(3, P.N);
  P.cap = prec == P2M_FP64 ? 544 : 1088;
  P.c0 = 0;
  P.span = cell_span(P.N);
  P.start = ws.start.as<int>();
  P.rec = ws.rec.p;
  P.us = ws.us.p;
  P.field = field;
  P.fd = fd;
  e = launch_p2m(P, 3, kernel, prec, lda, Np > 0 ? Np : 1, false, ws.tiles.p, st);
  if (e) { cuda_fail(info, e, caller); return; }
}

}  // namespace
}  // namespace ppmg

extern "C" void ppmg_interp_p2m_dv_3d_noalloc(const double* xp, int64_t ldxp, int64_t Np,
                                              const double* up, int64_t ldup, int lda,
                                              int topo_id, int mesh_id, int kernel,
                                              const int* ghostsize, double* field_up,
                                              int64_t ldf, const int64_t* f_lb,
                                              const int64_t* f_ub, int* info, void* stream) {
  ppmg::p2m_noalloc(xp, ldxp, Np, up, ldup, lda, topo_id, mesh_id, kernel, ghostsize,
                    field_up, ldf, f_lb, f_ub, info, (cudaStream_t)stream,
                    "ppmg_interp_p2m_dv_3d_noalloc");
}
