// ppmg_common.cuh -- shared types and device helpers of libppmg.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "../../include/ppmg.h"

namespace ppmg {

// Reference constants (ppm/src/ppm_param.h, ppm/src/ppm_error.h).
constexpr int kKernelBsp2 = 1;
constexpr int kKernelMp4 = 2;
constexpr int kBcPeriodic = 1;
constexpr int kErrorFatal = -1;
constexpr int kErrorError = -2;
constexpr int kErrAlloc = 101;
constexpr int kErrPartUnass = 405;
constexpr int kErrArgument = 503;
constexpr int kMapGhostGet = 5;
constexpr int kMapGhostPut = 6;

// xy tile (in cells / node columns) of the 3D gather kernels
constexpr int kTileX = 32;
constexpr int kTileY = 16;

// Geometry of one registered (topo_id, mesh_id), one subdomain.
struct Geom {
  int dim;
  int N[3];            // cells per axis (Nm - 1)
  double min_phys[3], max_phys[3];
  double min_sub[3], max_sub[3];
  double dxi_d[3];     // 1/(len/Nc) in FP64 (P2M, remesh; ppm_interp_p2m.f:479-489)
  float dxi_f[3];      // the same evaluated in FP32 (single-precision variants)
  double dxiq_d[3];    // FP32 mesh spacing of M2P/comp_weights widened to FP64
  float dxiq_f[3];     // (ppm_interp_m2p.f:221-222,486-489)
  double h_d[3];       // (max_phys-min_phys)/(Nm-1) (ppm_rmsh_create_part.f:340-342)
  int64_t ncell;       // prod N
};

// Spatial layout of field_up(ldf, lb:ub, ...) in elements.
struct FieldDesc {
  int64_t s[3];   // strides of x, y, z
  int lb[3];      // lower bounds (1-based Fortran indices)
  int ub[3];
  int box_lo[3];  // written box: 1-g .. Nm+g
  int box_hi[3];
};

// Per-thread error state (ppmg_last_error).
void set_error(int info, int errnum, const std::string& msg);
void clear_error();

// Kernel launch counter (ppmg_launch_count).
extern std::atomic<int64_t> g_launches;
inline void count_launch(int n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Device-time instrumentation (ppmg_kernel_timing): while enabled, a scope
// brackets the work it encloses on stream `st` with CUDA events; the elapsed
// times accumulate per part until ppmg_kernel_timing_read.
enum TimedPart { kTimeP2M = 0, kTimeM2P = 1, kTimeSort = 2, kTimedParts = 3 };
class TimingScope {
 public:
  TimingScope(int part, cudaStream_t st);
  ~TimingScope();
  TimingScope(const TimingScope&) = delete;
  TimingScope& operator=(const TimingScope&) = delete;

 private:
  int part_;
  cudaStream_t st_;
  cudaEvent_t begin_ = nullptr;
};

// -------------------------------------------------------------------------
// Device helpers
// -------------------------------------------------------------------------
template <class T>
struct Vec4;
template <>
struct Vec4<float> {
  using type = float4;
};
template <>
struct Vec4<double> {
  using type = double4;
};

// Floating ops that never contract into FMA: the FP64 form evaluates the
// reference's expressions operation by operation (gfortran -O2 emits no FMA).
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }

// M'4 1D weights at f in [0,1), in the reference's unrolled Horner forms
// (ppm_interp_p2m.f:800-853): nodes i0-1, i0, i0+1, i0+2 at
// s = f+1, f, f-1, f-2 with x10 = f+1, x11 = x10-1, x12 = x10-2, x13 = x10-3.
template <class T>
__device__ __forceinline__ void mp4_weights_exact(T f, T w[4]) {
  const T x10 = radd(f, T(1));
  const T x11 = rsub(x10, T(1));
  const T x12 = rsub(x10, T(2));
  const T x13 = rsub(x10, T(3));
  w[0] = radd(T(2), rmul(radd(T(-4), rmul(rsub(T(2.5), rmul(T(0.5), x10)), x10)), x10));
  w[1] = radd(T(1), rmul(radd(T(-2.5), rmul(T(1.5), x11)), rmul(x11, x11)));
  w[2] = radd(T(1), rmul(rsub(T(-2.5), rmul(T(1.5), x12)), rmul(x12, x12)));
  w[3] = radd(T(2), rmul(radd(T(4), rmul(radd(T(2.5), rmul(T(0.5), x13)), x13)), x13));
}

// The same polynomials in factored form for the FP32 mixed form.  With
// g = 1 - f the four M'4 pieces factor as
//   W(f+1) = -1/2 g^2 f,        W(f)   = g (1 + f - 3/2 f^2),
//   W(f-1) = f (1 + g - 3/2 g^2), W(f-2) = -1/2 f^2 g,
// products of well-conditioned factors, so every weight carries a few ulp of
// relative error; the Horner forms above lose up to ulp(4) absolute to
// cancellation, which in FP32 is ~1e-6 of the stencil sum.
// The partition-of-unity defect 1 - sum(w) (exact by Sterbenz: the sum is
// within a few ulp of 1) is then added to the largest weight, so the stored
// weights sum to 1 up to a single rounding: the deposited total strength is
// conserved to the rounding of the tensor products.
template <class T>
__device__ __forceinline__ void mp4_weights_fast(T f, T w[4]) {
  const T g = T(1) - f;
  w[0] = T(-0.5) * (g * g) * f;
  w[1] = g * (T(1) + f - T(1.5) * (f * f));
  w[2] = f * (T(1) + g - T(1.5) * (g * g));
  w[3] = T(-0.5) * (f * f) * g;
  const T defect = T(1) - ((w[0] + w[3]) + (w[1] + w[2]));
  if (f < T(0.5))
    w[1] += defect;
  else
    w[2] += defect;
}

// B-spline 2 weights (ppm_interp_p2m.f:3080-3110): a10 = 1 - f, a11 = 1 + (f - 1).
template <class T>
__device__ __forceinline__ void bsp2_weights_exact(T f, T w[2]) {
  w[0] = rsub(T(1), f);
  w[1] = radd(T(1), rsub(f, T(1)));
}

// Derivatives dW/ds of the M'4 pieces at s = f+1, f, f-1, f-2.
template <class T>
__device__ __forceinline__ void mp4_dweights(T f, T d[4]) {
  const T s0 = f + T(1), s1 = f, s2 = f - T(1), s3 = f - T(2);
  d[0] = T(-4) + T(5) * s0 - T(1.5) * s0 * s0;
  d[1] = T(-5) * s1 + T(4.5) * s1 * s1;
  d[2] = T(-5) * s2 - T(4.5) * s2 * s2;
  d[3] = T(4) + T(5) * s3 + T(1.5) * s3 * s3;
}

// Packed per-particle vectors (sorted records and strength chunks) are kept
// as planes of 16-byte units, `ps` units apart: a float4 is one unit, a
// double4 keeps (x, y) in its first plane and (z, w) in its second.  Every
// plane of a range of sorted particles is then one contiguous block.
__device__ __forceinline__ float4 load_vec(const float4* b, int64_t s, int64_t) { return b[s]; }
__device__ __forceinline__ double4 load_vec(const double4* b, int64_t s, int64_t ps) {
  const double2* p = reinterpret_cast<const double2*>(b);
  const double2 a = p[s], c = p[ps + s];
  return make_double4(a.x, a.y, c.x, c.y);
}
__device__ __forceinline__ void store_vec(float4* b, int64_t s, int64_t, float4 v) { b[s] = v; }
__device__ __forceinline__ void store_vec(double4* b, int64_t s, int64_t ps, double4 v) {
  double2* p = reinterpret_cast<double2*>(b);
  p[s] = make_double2(v.x, v.y);
  p[ps + s] = make_double2(v.z, v.w);
}

// mbarriers and one-dimensional TMA bulk copies (global -> this CTA's
// shared memory, completion counted in bytes on an mbarrier).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait for a phase of an mbarrier (false: gave up after `limit` polls).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

}  // namespace ppmg
