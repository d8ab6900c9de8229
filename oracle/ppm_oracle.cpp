// ppm_oracle.cpp -- CPU restatement of the reference's interpolation and
// remeshing loops.  TEST INFRASTRUCTURE ONLY: used by tests/ as the checker
// and by bench.py as the timed CPU baseline; the product never links it.
// Parity: unpinned against reference outputs (no reference tests exist and no
// Fortran compiler is available); pinned by exact-rational golden vectors and
// analytic identities.  Each routine cites the reference lines it follows
// (paths relative to ppm/src/ of PPMLibrary/ppm_legacy).
#include "ppm_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Field view: field(lda, lb0:ub0, lb1:ub1, [lb2:ub2,] nsubs), column-major.
// ---------------------------------------------------------------------------
template <class T>
struct FieldView {
  T* p;
  int lda, dim;
  int lb[3], ub[3];
  int64_t ext[3];
  FieldView(T* base, const orc_field* fl, int d) : p(base), lda(fl->lda), dim(d) {
    for (int a = 0; a < 3; ++a) {
      lb[a] = fl->lb[a];
      ub[a] = fl->ub[a];
      ext[a] = (a < d) ? (int64_t)(ub[a] - lb[a] + 1) : 1;
    }
  }
  bool inside(int i, int j, int k) const {
    if (i < lb[0] || i > ub[0] || j < lb[1] || j > ub[1]) return false;
    if (dim == 3 && (k < lb[2] || k > ub[2])) return false;
    return true;
  }
  int64_t off(int a, int i, int j, int k, int s) const {
    int64_t kk = (dim == 3) ? (int64_t)(k - lb[2]) : 0;
    return (int64_t)a +
           (int64_t)lda * ((int64_t)(i - lb[0]) +
                           ext[0] * ((int64_t)(j - lb[1]) + ext[1] * (kk + ext[2] * s)));
  }
  T& at(int a, int i, int j, int k, int s) const { return p[off(a, i, j, k, s)]; }
};

template <class T>
inline T geomT(double v) { return (T)v; }

// Fortran INT(): truncation toward zero.
template <class T>
inline int fint(T x) { return (int)x; }

// ---------------------------------------------------------------------------
// Particle -> sub assignment, ppm_interp_p2m.f:496-750 (identical loops in
// ppm_interp_m2p.f:494-747 and ppm_rmsh_comp_weights.f:404-655).
// Subs are scanned from the last to the first; a particle is assigned to a
// sub if it lies in its closure and strictly below its upper face, unless
// that face is a non-periodic physical boundary.
// ---------------------------------------------------------------------------
template <class T>
bool in_sub(const orc_geom* g, int isub, const T* x) {
  const int d = g->dim;
  for (int a = 0; a < d; ++a) {
    T lo = geomT<T>(g->min_sub[isub * 3 + a]);
    T hi = geomT<T>(g->max_sub[isub * 3 + a]);
    if (!(x[a] >= lo && x[a] <= hi)) return false;
  }
  for (int a = 0; a < d; ++a) {
    T hi = geomT<T>(g->max_sub[isub * 3 + a]);
    bool upper_closed = (g->subs_bc[isub * 6 + 2 * a + 1] == 1) &&
                        (g->bcdef[2 * a + 1] != ORC_BC_PERIODIC);
    if (!(x[a] < hi || upper_closed)) return false;
  }
  return true;
}

template <class T>
int assign_subs(const orc_geom* g, const T* xp, int ldxp, int np,
                std::vector<std::vector<int>>& lists, int* err) {
  lists.assign(g->nsubs, std::vector<int>());
  std::vector<int> l1(np), l2;
  for (int i = 0; i < np; ++i) l1[i] = i;
  l2.reserve(np);
  for (int idom = g->nsubs - 1; idom >= 0; --idom) {
    l2.clear();
    for (int ip : l1) {
      if (in_sub<T>(g, idom, xp + (int64_t)ip * ldxp))
        lists[idom].push_back(ip);
      else
        l2.push_back(ip);
    }
    l1.swap(l2);
    if (l1.empty()) break;
  }
  if (!l1.empty()) {
    if (err) *err = ORC_ERR_PART_UNASS;
    return ORC_ERROR_FATAL;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// 1D kernel weights in the reference's own expression forms.
// M'4, 3D interp form (ppm_interp_p2m.f:800-853, ppm_interp_m2p.f:905-950):
//   x10 = f + 1, x11 = x10 - 1, x12 = x10 - 2, x13 = x10 - 3.
// ---------------------------------------------------------------------------
template <class T>
inline void mp4_unrolled(T xp1, T a[4]) {
  const T x10 = xp1 + T(1);
  const T x11 = x10 - T(1);
  const T x12 = x10 - T(2);
  const T x13 = x10 - T(3);
  a[0] = T(2) + (T(-4) + (T(2.5) - T(0.5) * x10) * x10) * x10;
  a[1] = T(1) + (T(-2.5) + T(1.5) * x11) * (x11 * x11);
  a[2] = T(1) + (T(-2.5) - T(1.5) * x12) * (x12 * x12);
  a[3] = T(2) + (T(4) + (T(2.5) + T(0.5) * x13) * x13) * x13;
}

// B-spline 2 (ppm_interp_p2m.f:3080-3110): a10 = 1 - x10, a11 = 1 + (x10 - 1).
template <class T>
inline void bsp2_unrolled(T xp1, T a[2]) {
  const T x10 = xp1;
  const T x11 = x10 - T(1);
  a[0] = T(1) - x10;
  a[1] = T(1) + x11;
}

// M'4 in the |x| branching form used by the 2D loops and comp_weights
// (ppm_interp_p2m.f:3600-3620, ppm_rmsh_comp_weights.f:945-951).
template <class T>
inline T mp4_abs_lt(T x) {  // 2D interp: branch on x < 1
  if (x < T(1)) return T(1) - (x * x) * (T(2.5) - T(1.5) * x);
  return T(2) + (T(-4) + (T(2.5) - T(0.5) * x) * x) * x;
}

// Mesh spacing of the routine's own kind (P2M, remesh): dx = len/Nc, dxi = 1/dx.
template <class T>
inline T dxi_mk(const orc_geom* g, int a) {
  T len = geomT<T>(g->max_phys[a]) - geomT<T>(g->min_phys[a]);
  T dx = len / T(g->Nm[a] - 1);
  return T(1) / dx;
}

// FP32 mesh spacing quirk of M2P and comp_weights: len_phys, dx, dxi are
// default REAL (ppm_interp_m2p.f:221-222, 486-489; ppm_rmsh_comp_weights.f:
// 146-147, 395-398).  Returned widened to T.
template <class T>
inline T dxi_real(const orc_geom* g, int a) {
  float len = (float)(geomT<T>(g->max_phys[a]) - geomT<T>(g->min_phys[a]));
  float dx = (float)((T)len / (T)(g->Nm[a] - 1));
  float dxi = (float)(T(1) / (T)dx);
  return (T)dxi;
}

// ---------------------------------------------------------------------------
// P2M deposit for one sub, ppm_interp_p2m.f:758-3663.
// Returns false if a deposit index leaves the field box (the reference would
// write out of bounds, quirk Q10).
// ---------------------------------------------------------------------------
template <class T>
bool p2m_zero_sub(const orc_geom* g, int isub, const int* ghost, const FieldView<T>& F) {
  const int* nn = g->nnodes + isub * 3;
  int k0 = 0, k1 = 0;
  if (g->dim == 3) { k0 = 1 - ghost[2]; k1 = nn[2] + ghost[2]; }
  for (int k = k0; k <= k1; ++k)
    for (int j = 1 - ghost[1]; j <= nn[1] + ghost[1]; ++j)
      for (int i = 1 - ghost[0]; i <= nn[0] + ghost[0]; ++i) {
        if (!F.inside(i, j, k)) return false;
        for (int a = 0; a < F.lda; ++a) F.at(a, i, j, k, isub) = T(0);
      }
  return true;
}

template <class T>
bool p2m_deposit_sub(const orc_geom* g, int isub, const std::vector<int>& list,
                     const T* xp, int ldxp, const T* up, int lda, int kernel,
                     const FieldView<T>& F) {
  const int d = g->dim;
  T dxi[3];
  for (int a = 0; a < d; ++a) dxi[a] = dxi_mk<T>(g, a);
  T ms[3];
  for (int a = 0; a < d; ++a) ms[a] = geomT<T>(g->min_sub[isub * 3 + a]);
  bool ok = true;
  if (d == 3) {
    for (int iq : list) {
      const T* x = xp + (int64_t)iq * ldxp;
      const T* u = up + (int64_t)iq * lda;
      T x0[3];
      for (int a = 0; a < 3; ++a) x0[a] = (x[a] - ms[a]) * dxi[a];
      if (kernel == ORC_KERNEL_MP4) {
        int ip[3];
        T w[3][4];
        for (int a = 0; a < 3; ++a) {
          ip[a] = fint(x0[a]);
          mp4_unrolled<T>(x0[a] - T(ip[a]), w[a]);
        }
        for (int kk = 0; kk < 4; ++kk)
          for (int jj = 0; jj < 4; ++jj)
            for (int ii = 0; ii < 4; ++ii) {
              int i = ip[0] + ii, j = ip[1] + jj, k = ip[2] + kk;
              if (!F.inside(i, j, k)) { ok = false; continue; }
              T wt = w[0][ii] * w[1][jj] * w[2][kk];
              for (int a = 0; a < lda; ++a) {
                T& f = F.at(a, i, j, k, isub);
                f = f + wt * u[a];
              }
            }
      } else {  // bsp2
        int ip[3];
        T w[3][2];
        for (int a = 0; a < 3; ++a) {
          ip[a] = fint(x0[a]) + 1;
          bsp2_unrolled<T>(x0[a] - T(ip[a] - 1), w[a]);
        }
        for (int kk = 0; kk < 2; ++kk)
          for (int jj = 0; jj < 2; ++jj)
            for (int ii = 0; ii < 2; ++ii) {
              int i = ip[0] + ii, j = ip[1] + jj, k = ip[2] + kk;
              if (!F.inside(i, j, k)) { ok = false; continue; }
              T wt = w[0][ii] * w[1][jj] * w[2][kk];
              for (int a = 0; a < lda; ++a) {
                T& f = F.at(a, i, j, k, isub);
                f = f + wt * u[a];
              }
            }
      }
    }
  } else {  // 2D, M'4 only (ppm_interp_p2m.f:3574-3663)
    for (int iq : list) {
      const T* x = xp + (int64_t)iq * ldxp;
      const T* u = up + (int64_t)iq * lda;
      T x01 = (x[0] - ms[0]) * dxi[0];
      T x02 = (x[1] - ms[1]) * dxi[1];
      int ip1 = fint(x01) + 1;
      int ip2 = fint(x02) + 1;
      T xp1 = x01 - std::trunc(x01);
      T xp2 = x02 - std::trunc(x02);
      for (int jj = -1; jj <= 2; ++jj) {
        T wx2 = mp4_abs_lt<T>(std::fabs(xp2 - T(jj)));
        for (int ii = -1; ii <= 2; ++ii) {
          T wx1 = mp4_abs_lt<T>(std::fabs(xp1 - T(ii)));
          int i = ii + ip1, j = jj + ip2;
          if (!F.inside(i, j, 0)) { ok = false; continue; }
          for (int a = 0; a < lda; ++a) {
            T& f = F.at(a, i, j, 0, isub);
            f = f + wx1 * wx2 * u[a];
          }
        }
      }
    }
  }
  return ok;
}

// ---------------------------------------------------------------------------
// Ghost mesh blocks, ppm_map_field_ghost_init.f:234-447 with
// ppm_mesh_block_intersect.f:207-280.  For each sub i: blocks to every other
// sub (unshifted), then for each periodic shift vector the self image and the
// images seen by every other sub.  A block moves the real nodes of `from`
// (global indices start..start+size-1) to `to` at global index + offset.
// ---------------------------------------------------------------------------
struct Block {
  int from, to;
  int start[3], size[3], offset[3];
};

void intersect(const orc_geom* g, int isub, int jsub, const int* off, const int* ghost,
               std::vector<Block>& out) {
  Block b;
  b.from = isub;
  b.to = jsub;
  for (int k = 0; k < 3; ++k) { b.start[k] = 1; b.size[k] = 1; b.offset[k] = 0; }
  for (int k = 0; k < g->dim; ++k) {
    int fromistart = g->istart[isub * 3 + k] + off[k];
    int fromnn = g->nnodes[isub * 3 + k];
    int toistart = g->istart[jsub * 3 + k] - ghost[k];
    int tonn = g->nnodes[jsub * 3 + k] + 2 * ghost[k];
    int bs = std::max(fromistart, toistart);
    int be = std::min(fromistart + fromnn, toistart + tonn);
    int sz = be - bs;
    if (sz < 1) return;
    b.start[k] = bs - off[k];
    b.size[k] = sz;
    b.offset[k] = off[k];
  }
  out.push_back(b);
}

std::vector<Block> ghost_blocks(const orc_geom* g, const int* ghost) {
  std::vector<Block> out;
  const int d = g->dim;
  int op[3] = {0, 0, 0};
  for (int a = 0; a < d; ++a) op[a] = g->Nm[a] - 1;
  for (int i = 0; i < g->nsubs; ++i) {
    int zero[3] = {0, 0, 0};
    for (int j = 0; j < g->nsubs; ++j)
      if (j != i) intersect(g, i, j, zero, ghost, out);
    auto per = [&](int face) {
      return g->bcdef[face] == ORC_BC_PERIODIC && g->subs_bc[i * 6 + face] != 0;
    };
    bool lw = per(0), le = per(1), ls = per(2), ln = per(3);
    bool lb = d > 2 && per(4), lt = d > 2 && per(5);
    std::vector<std::array<int, 3>> ond;
    auto push = [&](int x, int y, int z) { ond.push_back({x, y, z}); };
    if (lw) push(op[0], 0, 0);
    if (le) push(-op[0], 0, 0);
    if (ls) {
      push(0, op[1], 0);
      if (lw) push(op[0], op[1], 0);
      if (le) push(-op[0], op[1], 0);
    }
    if (ln) {
      push(0, -op[1], 0);
      if (lw) push(op[0], -op[1], 0);
      if (le) push(-op[0], -op[1], 0);
    }
    if (d > 2) {
      for (int zs = 0; zs < 2; ++zs) {
        bool lz = zs == 0 ? lb : lt;
        if (!lz) continue;
        int oz = zs == 0 ? op[2] : -op[2];
        push(0, 0, oz);
        if (lw) push(op[0], 0, oz);
        if (le) push(-op[0], 0, oz);
        if (ls) {
          push(0, op[1], oz);
          if (lw) push(op[0], op[1], oz);
          if (le) push(-op[0], op[1], oz);
        }
        if (ln) {
          push(0, -op[1], oz);
          if (lw) push(op[0], -op[1], oz);
          if (le) push(-op[0], -op[1], oz);
        }
      }
    }
    for (auto& o : ond) {
      intersect(g, i, i, o.data(), ghost, out);
      for (int j = 0; j < g->nsubs; ++j)
        if (j != i) intersect(g, i, j, o.data(), ghost, out);
    }
  }
  return out;
}

template <class T>
void ghost_get(const orc_geom* g, const FieldView<T>& F, const int* ghost) {
  // push (pack every block from the pre-get field), then pop (replace).
  std::vector<Block> bl = ghost_blocks(g, ghost);
  std::vector<std::vector<T>> buf(bl.size());
  for (size_t b = 0; b < bl.size(); ++b) {
    const Block& B = bl[b];
    const int* is = g->istart + B.from * 3;
    for (int k = 0; k < B.size[2]; ++k)
      for (int j = 0; j < B.size[1]; ++j)
        for (int i = 0; i < B.size[0]; ++i) {
          int li = B.start[0] + i - is[0] + 1, lj = B.start[1] + j - is[1] + 1;
          int lk = g->dim == 3 ? B.start[2] + k - is[2] + 1 : 0;
          for (int a = 0; a < F.lda; ++a) buf[b].push_back(F.at(a, li, lj, lk, B.from));
        }
  }
  for (size_t b = 0; b < bl.size(); ++b) {
    const Block& B = bl[b];
    const int* it = g->istart + B.to * 3;
    size_t q = 0;
    for (int k = 0; k < B.size[2]; ++k)
      for (int j = 0; j < B.size[1]; ++j)
        for (int i = 0; i < B.size[0]; ++i) {
          int ti = B.start[0] + i + B.offset[0] - it[0] + 1;
          int tj = B.start[1] + j + B.offset[1] - it[1] + 1;
          int tk = g->dim == 3 ? B.start[2] + k + B.offset[2] - it[2] + 1 : 0;
          for (int a = 0; a < F.lda; ++a) F.at(a, ti, tj, tk, B.to) = buf[b][q++];
        }
  }
}

template <class T>
void ghost_put(const orc_geom* g, const FieldView<T>& F, const int* ghost) {
  // reverse of the get: ghost-region values of `to` are packed first, then
  // added onto the real nodes of `from` in block order (pop with add).
  std::vector<Block> bl = ghost_blocks(g, ghost);
  std::vector<std::vector<T>> buf(bl.size());
  for (size_t b = 0; b < bl.size(); ++b) {
    const Block& B = bl[b];
    const int* it = g->istart + B.to * 3;
    for (int k = 0; k < B.size[2]; ++k)
      for (int j = 0; j < B.size[1]; ++j)
        for (int i = 0; i < B.size[0]; ++i) {
          int ti = B.start[0] + i + B.offset[0] - it[0] + 1;
          int tj = B.start[1] + j + B.offset[1] - it[1] + 1;
          int tk = g->dim == 3 ? B.start[2] + k + B.offset[2] - it[2] + 1 : 0;
          for (int a = 0; a < F.lda; ++a) buf[b].push_back(F.at(a, ti, tj, tk, B.to));
        }
  }
  for (size_t b = 0; b < bl.size(); ++b) {
    const Block& B = bl[b];
    const int* is = g->istart + B.from * 3;
    size_t q = 0;
    for (int k = 0; k < B.size[2]; ++k)
      for (int j = 0; j < B.size[1]; ++j)
        for (int i = 0; i < B.size[0]; ++i) {
          int li = B.start[0] + i - is[0] + 1, lj = B.start[1] + j - is[1] + 1;
          int lk = g->dim == 3 ? B.start[2] + k - is[2] + 1 : 0;
          for (int a = 0; a < F.lda; ++a) {
            T& f = F.at(a, li, lj, lk, B.from);
            f = f + buf[b][q++];
          }
        }
  }
}

// ---------------------------------------------------------------------------
// M2P for one sub, ppm_interp_m2p.f:777-4105.  Term order per component:
// x outermost, then y, then z (3D); y outer, x inner (2D M'4); i outer,
// j inner (2D bsp2).
// ---------------------------------------------------------------------------
template <class T>
bool m2p_sub(const orc_geom* g, int isub, const std::vector<int>& list, const T* xp,
             int ldxp, T* up, int lda, int kernel, const FieldView<T>& F) {
  const int d = g->dim;
  T dxi[3];
  for (int a = 0; a < d; ++a) dxi[a] = dxi_real<T>(g, a);
  T ms[3], mp[3];
  for (int a = 0; a < d; ++a) {
    ms[a] = geomT<T>(g->min_sub[isub * 3 + a]);
    mp[a] = geomT<T>(g->min_phys[a]);
  }
  const int* is = g->istart + isub * 3;
  bool ok = true;
  for (int iq : list) {
    const T* x = xp + (int64_t)iq * ldxp;
    T* u = up + (int64_t)iq * lda;
    if (d == 3) {
      T x0[3];
      for (int a = 0; a < 3; ++a) x0[a] = (x[a] - ms[a]) * dxi[a];
      if (kernel == ORC_KERNEL_MP4) {
        int ip[3];
        T w[3][4];
        for (int a = 0; a < 3; ++a) {
          ip[a] = fint(x0[a]);
          mp4_unrolled<T>(x0[a] - T(ip[a]), w[a]);
        }
        for (int c = 0; c < lda; ++c)
          for (int ii = 0; ii < 4; ++ii)
            for (int jj = 0; jj < 4; ++jj)
              for (int kk = 0; kk < 4; ++kk) {
                int i = ip[0] + ii, j = ip[1] + jj, k = ip[2] + kk;
                if (!F.inside(i, j, k)) { ok = false; continue; }
                T wt = w[0][ii] * w[1][jj] * w[2][kk];
                u[c] = u[c] + wt * F.at(c, i, j, k, isub);
              }
      } else {
        int ip[3];
        T w[3][2];
        for (int a = 0; a < 3; ++a) {
          ip[a] = fint(x0[a]) + 1;
          bsp2_unrolled<T>(x0[a] - T(ip[a] - 1), w[a]);
        }
        for (int c = 0; c < lda; ++c)
          for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
              for (int kk = 0; kk < 2; ++kk) {
                int i = ip[0] + ii, j = ip[1] + jj, k = ip[2] + kk;
                if (!F.inside(i, j, k)) { ok = false; continue; }
                T wt = w[0][ii] * w[1][jj] * w[2][kk];
                u[c] = u[c] + wt * F.at(c, i, j, k, isub);
              }
      }
    } else if (kernel == ORC_KERNEL_MP4) {  // 2D M'4: min_phys + istart form
      T x0 = (x[0] - mp[0]) * dxi[0];
      T y0 = (x[1] - mp[1]) * dxi[1];
      int ip1 = fint(x0) + 2 - is[0];
      int ip2 = fint(y0) + 2 - is[1];
      T xp1 = x0 - std::trunc(x0);
      T xp2 = y0 - std::trunc(y0);
      for (int jj = -1; jj <= 2; ++jj) {
        T wx2 = mp4_abs_lt<T>(std::fabs(xp2 - T(jj)));
        for (int ii = -1; ii <= 2; ++ii) {
          T wx1 = mp4_abs_lt<T>(std::fabs(xp1 - T(ii)));
          int i = ii + ip1, j = jj + ip2;
          if (!F.inside(i, j, 0)) { ok = false; continue; }
          for (int c = 0; c < lda; ++c) u[c] = u[c] + wx1 * wx2 * F.at(c, i, j, 0, isub);
        }
      }
    } else {  // 2D bsp2 (min_sub form)
      T x0 = (x[0] - ms[0]) * dxi[0];
      T y0 = (x[1] - ms[1]) * dxi[1];
      int ip[2] = {fint(x0) + 1, fint(y0) + 1};
      T w[2][2];
      bsp2_unrolled<T>(x0 - T(ip[0] - 1), w[0]);
      bsp2_unrolled<T>(y0 - T(ip[1] - 1), w[1]);
      for (int c = 0; c < lda; ++c)
        for (int ii = 0; ii < 2; ++ii)
          for (int jj = 0; jj < 2; ++jj) {
            int i = ip[0] + ii, j = ip[1] + jj;
            if (!F.inside(i, j, 0)) { ok = false; continue; }
            T wt = w[0][ii] * w[1][jj];
            u[c] = u[c] + wt * F.at(c, i, j, 0, isub);
          }
    }
  }
  return ok;
}

template <class T>
int p2m_impl(const orc_geom* g, const T* xp, int ldxp, int np, const T* up, int lda,
             int kernel, const int* ghost, T* field, const orc_field* fl, int* err,
             bool do_put) {
  if (err) *err = 0;
  if (np < 0 || lda < 1 || ldxp < g->dim) { if (err) *err = ORC_ERR_ARGUMENT; return ORC_ERROR_ERROR; }
  if (kernel != ORC_KERNEL_MP4 && !(kernel == ORC_KERNEL_BSP2 && g->dim == 3)) {
    if (err) *err = ORC_ERR_ARGUMENT;
    return ORC_ERROR_ERROR;
  }
  FieldView<T> F(field, fl, g->dim);
  if (F.lda != lda) { if (err) *err = ORC_ERR_ARGUMENT; return ORC_ERROR_ERROR; }
  std::vector<std::vector<int>> lists;
  if (np > 0) {
    int info = assign_subs<T>(g, xp, ldxp, np, lists, err);
    if (info) return info;
  } else {
    lists.assign(g->nsubs, {});
  }
  for (int s = 0; s < g->nsubs; ++s)
    if (!p2m_zero_sub<T>(g, s, ghost, F)) { if (err) *err = ORC_ERR_OUT_OF_FIELD; return ORC_ERROR_ERROR; }
  bool ok = true;
  for (int s = 0; s < g->nsubs; ++s)
    ok = p2m_deposit_sub<T>(g, s, lists[s], xp, ldxp, up, lda, kernel, F) && ok;
  if (!ok) { if (err) *err = ORC_ERR_OUT_OF_FIELD; return ORC_ERROR_ERROR; }
  if (do_put) ghost_put<T>(g, F, ghost);
  return 0;
}

template <class T>
int m2p_impl(const orc_geom* g, const T* xp, int ldxp, int np, T* up, int lda, int kernel,
             const int* ghost, const T* field, const orc_field* fl, int* err) {
  (void)ghost;
  if (err) *err = 0;
  if (np < 0 || lda < 1 || ldxp < g->dim) { if (err) *err = ORC_ERR_ARGUMENT; return ORC_ERROR_ERROR; }
  if (kernel != ORC_KERNEL_MP4 && kernel != ORC_KERNEL_BSP2) {
    if (err) *err = ORC_ERR_ARGUMENT;
    return ORC_ERROR_ERROR;
  }
  FieldView<T> F(const_cast<T*>(field), fl, g->dim);
  std::vector<std::vector<int>> lists;
  if (g->nsubs != 1) {
    int info = assign_subs<T>(g, xp, ldxp, np, lists, err);
    if (info) return info;
  } else {  // one sub: every particle, no containment check (ppm_interp_m2p.f:748-772)
    lists.assign(1, std::vector<int>(np));
    for (int i = 0; i < np; ++i) lists[0][i] = i;
  }
  for (int64_t i = 0; i < (int64_t)np * lda; ++i) up[i] = T(0);
  bool ok = true;
  for (int s = 0; s < g->nsubs; ++s)
    ok = m2p_sub<T>(g, s, lists[s], xp, ldxp, up, lda, kernel, F) && ok;
  if (!ok) { if (err) *err = ORC_ERR_OUT_OF_FIELD; return ORC_ERROR_ERROR; }
  return 0;
}

// comp_weights weight in |x| form with LE tests (ppm_rmsh_comp_weights.f:937-951).
template <class T>
inline T mp4_abs_le(T x) {
  if (x <= T(2)) {
    if (x <= T(1)) return T(1) - (x * x) * (T(2.5) - T(1.5) * x);
    return T(2) + (T(-4) + (T(2.5) - T(0.5) * x) * x) * x;
  }
  return T(0);
}

}  // namespace

// ===========================================================================
// extern "C" entry points
// ===========================================================================
extern "C" {

int orc_assign_d(const orc_geom* g, const double* xp, int ldxp, int np, int* list_out,
                 int* store_info, int* err) {
  std::vector<std::vector<int>> lists;
  if (err) *err = 0;
  int info = assign_subs<double>(g, xp, ldxp, np, lists, err);
  if (info) return info;
  int q = 0;
  for (int s = 0; s < g->nsubs; ++s) {
    store_info[s] = (int)lists[s].size();
    for (int p : lists[s]) list_out[q++] = p;
  }
  return 0;
}

int orc_assign_s(const orc_geom* g, const float* xp, int ldxp, int np, int* list_out,
                 int* store_info, int* err) {
  std::vector<std::vector<int>> lists;
  if (err) *err = 0;
  int info = assign_subs<float>(g, xp, ldxp, np, lists, err);
  if (info) return info;
  int q = 0;
  for (int s = 0; s < g->nsubs; ++s) {
    store_info[s] = (int)lists[s].size();
    for (int p : lists[s]) list_out[q++] = p;
  }
  return 0;
}

int orc_p2m_d(const orc_geom* g, const double* xp, int ldxp, int np, const double* up,
              int lda, int kernel, const int* ghost, double* field, const orc_field* fl,
              int* err) {
  return p2m_impl<double>(g, xp, ldxp, np, up, lda, kernel, ghost, field, fl, err, true);
}
int orc_p2m_s(const orc_geom* g, const float* xp, int ldxp, int np, const float* up,
              int lda, int kernel, const int* ghost, float* field, const orc_field* fl,
              int* err) {
  return p2m_impl<float>(g, xp, ldxp, np, up, lda, kernel, ghost, field, fl, err, true);
}
int orc_p2m_noput_d(const orc_geom* g, const double* xp, int ldxp, int np,
                    const double* up, int lda, int kernel, const int* ghost,
                    double* field, const orc_field* fl, int* err) {
  return p2m_impl<double>(g, xp, ldxp, np, up, lda, kernel, ghost, field, fl, err, false);
}

int orc_m2p_d(const orc_geom* g, const double* xp, int ldxp, int np, double* up, int lda,
              int kernel, const int* ghost, const double* field, const orc_field* fl,
              int* err) {
  return m2p_impl<double>(g, xp, ldxp, np, up, lda, kernel, ghost, field, fl, err);
}
int orc_m2p_s(const orc_geom* g, const float* xp, int ldxp, int np, float* up, int lda,
              int kernel, const int* ghost, const float* field, const orc_field* fl,
              int* err) {
  return m2p_impl<float>(g, xp, ldxp, np, up, lda, kernel, ghost, field, fl, err);
}

int orc_ghost_get_d(const orc_geom* g, double* field, const orc_field* fl, const int* ghost) {
  ghost_get<double>(g, FieldView<double>(field, fl, g->dim), ghost);
  return 0;
}
int orc_ghost_put_d(const orc_geom* g, double* field, const orc_field* fl, const int* ghost) {
  ghost_put<double>(g, FieldView<double>(field, fl, g->dim), ghost);
  return 0;
}
int orc_ghost_get_s(const orc_geom* g, float* field, const orc_field* fl, const int* ghost) {
  ghost_get<float>(g, FieldView<float>(field, fl, g->dim), ghost);
  return 0;
}
int orc_ghost_put_s(const orc_geom* g, float* field, const orc_field* fl, const int* ghost) {
  ghost_put<float>(g, FieldView<float>(field, fl, g->dim), ghost);
  return 0;
}

}  // extern "C"

// ppm_rmsh_comp_weights.f:851-996.  wx(iidec, isub, ip) with bounds
// (1:2ks, 1:nsubs, 1-ks:maxp+ks); ip is the position in the sub's list.
template <class T>
static int comp_weights_impl(const orc_geom* g, const T* xp, int ldxp, int np, int kernel,
                             const int* list, const int* store_info, int maxp, T* wx1, T* wx2,
                             T* wx3) {
  (void)np;
  const int d = g->dim;
  int ks = kernel == ORC_KERNEL_MP4 ? 2 : (kernel == ORC_KERNEL_BSP2 ? 1 : 0);
  if (ks == 0) return ORC_ERROR_ERROR;
  const int nw = 2 * ks;
  const int64_t n3 = (int64_t)maxp + 2 * ks;
  T* wx[3] = {wx1, wx2, wx3};
  for (int a = 0; a < d; ++a)
    std::fill(wx[a], wx[a] + (int64_t)nw * g->nsubs * n3, T(0));
  T dxi[3];
  for (int a = 0; a < d; ++a) dxi[a] = dxi_real<T>(g, a);
  int q = 0;
  for (int s = 0; s < g->nsubs; ++s) {
    const int* is = g->istart + s * 3;
    for (int ip = 1; ip <= store_info[s]; ++ip) {
      const T* x = xp + (int64_t)list[q + ip - 1] * ldxp;
      for (int a = 0; a < d; ++a) {
        const T mn = (T)g->min_phys[a];
        T xi = (x[a] - mn) * dxi[a];
        int ipa = fint(xi) + 2 - is[a];
        int lo = kernel == ORC_KERNEL_MP4 ? ipa - 1 : ipa;
        for (int t = 0; t < nw; ++t) {
          int ii = lo + t;
          T xd = std::fabs((T)(ii - 2 + is[a]) - (x[a] - mn) * dxi[a]);
          T w = T(0);
          if (kernel == ORC_KERNEL_MP4) {
            w = mp4_abs_le<T>(xd);
          } else if (xd <= T(1)) {
            w = T(1) - xd;
          }
          int64_t idx = (int64_t)t + nw * ((int64_t)s + (int64_t)g->nsubs * ((int64_t)ip - (1 - ks)));
          wx[a][idx] = w;
        }
      }
    }
    q += store_info[s];
  }
  return 0;
}

// ppm_rmsh_remesh.f:508-924: zero the whole field, scatter with the stored
// weights over nodes ip-1..ip+2 (M'4) or ip..ip+1 (bsp2), then ghost put.
template <class T>
static int remesh_impl(const orc_geom* g, const T* xp, int ldxp, int np, const T* up, int lda,
                       int kernel, const int* ghost, const int* list, const int* store_info,
                       int maxp, const T* wx1, const T* wx2, const T* wx3, T* field,
                       const orc_field* fl, int* err) {
  (void)np;
  (void)maxp;
  if (err) *err = 0;
  const int d = g->dim;
  int ks = kernel == ORC_KERNEL_MP4 ? 2 : (kernel == ORC_KERNEL_BSP2 ? 1 : 0);
  if (ks == 0) { if (err) *err = ORC_ERR_ARGUMENT; return ORC_ERROR_ERROR; }
  for (int a = 0; a < d; ++a)
    if (ghost[a] < ks - 1) { if (err) *err = ORC_ERR_ARGUMENT; return ORC_ERROR_ERROR; }
  const int nw = 2 * ks;
  FieldView<T> F(field, fl, d);
  int64_t total = (int64_t)F.lda * F.ext[0] * F.ext[1] * F.ext[2] * g->nsubs;
  std::fill(field, field + total, T(0));
  T dxi[3];
  for (int a = 0; a < d; ++a) dxi[a] = dxi_mk<T>(g, a);
  const T* wx[3] = {wx1, wx2, wx3};
  bool ok = true;
  int q = 0;
  for (int s = 0; s < g->nsubs; ++s) {
    const int* is = g->istart + s * 3;
    for (int ip = 1; ip <= store_info[s]; ++ip) {
      int iq = list[q + ip - 1];
      const T* x = xp + (int64_t)iq * ldxp;
      const T* u = up + (int64_t)iq * lda;
      int ipa[3] = {0, 0, 0};
      for (int a = 0; a < d; ++a) ipa[a] = fint((x[a] - (T)g->min_phys[a]) * dxi[a]) + 2 - is[a];
      int lo[3];
      for (int a = 0; a < 3; ++a) lo[a] = kernel == ORC_KERNEL_MP4 ? ipa[a] - 1 : ipa[a];
      auto W = [&](int a, int t) {
        int64_t idx = (int64_t)t + nw * ((int64_t)s + (int64_t)g->nsubs * ((int64_t)ip - (1 - ks)));
        return wx[a][idx];
      };
      int nk = d == 3 ? nw : 1;
      for (int kd = 0; kd < nk; ++kd)
        for (int jd = 0; jd < nw; ++jd)
          for (int id = 0; id < nw; ++id) {
            int i = lo[0] + id, j = lo[1] + jd, k = d == 3 ? lo[2] + kd : 0;
            if (!F.inside(i, j, k)) { ok = false; continue; }
            T w = d == 3 ? W(0, id) * W(1, jd) * W(2, kd) : W(0, id) * W(1, jd);
            for (int c = 0; c < lda; ++c) {
              T& f = F.at(c, i, j, k, s);
              f = f + w * u[c];
            }
          }
    }
    q += store_info[s];
  }
  if (!ok) { if (err) *err = ORC_ERR_OUT_OF_FIELD; return ORC_ERROR_ERROR; }
  ghost_put<T>(g, F, ghost);
  return 0;
}

// ppm_rmsh_create_part.f:427-681: nodes i=1..nnx (nnx = nnodes-1 on periodic
// or interior upper faces), visited k,j,i with i fastest; a node becomes a
// particle when cutoff(1) < strength < cutoff(2).
template <class T>
static int create_part_impl(const orc_geom* g, const T* field, const orc_field* fl,
                            const T* cutoff, const T* cutoff_weights, int resetpos,
                            const T* field_wp, int lda2, int* np_out, T* up_out, T* xp_out,
                            T* wp_out) {
  const int d = g->dim;
  FieldView<T> F(const_cast<T*>(field), fl, d);
  orc_field fl2 = *fl;
  fl2.lda = lda2 > 0 ? lda2 : 1;
  FieldView<T> FW(const_cast<T*>(field_wp), &fl2, d);
  T h[3];
  for (int a = 0; a < d; ++a)
    h[a] = ((T)g->max_phys[a] - (T)g->min_phys[a]) / (T)(g->Nm[a] - 1);
  int inp = 0;
  for (int s = 0; s < g->nsubs; ++s) {
    int nnl[3] = {1, 1, 1};
    for (int a = 0; a < d; ++a) {
      bool closed = g->subs_bc[s * 6 + 2 * a + 1] == 1 && g->bcdef[2 * a + 1] != ORC_BC_PERIODIC;
      nnl[a] = closed ? g->nnodes[s * 3 + a] : g->nnodes[s * 3 + a] - 1;
    }
    for (int k = 1; k <= nnl[2]; ++k)
      for (int j = 1; j <= nnl[1]; ++j)
        for (int i = 1; i <= nnl[0]; ++i) {
          int kk = d == 3 ? k : 0;
          T str;
          if (F.lda == 1 && cutoff_weights == nullptr) {
            str = std::fabs(F.at(0, i, j, kk, s));
          } else {
            T sum = T(0);
            for (int c = 0; c < F.lda; ++c) {
              T v = F.at(c, i, j, kk, s);
              if (cutoff_weights) v = v * cutoff_weights[c];
              sum = sum + v * v;
            }
            str = std::sqrt(sum);
          }
          if (str > cutoff[0] && str < cutoff[1]) {
            if (up_out) {
              for (int c = 0; c < F.lda; ++c) up_out[(int64_t)inp * F.lda + c] = F.at(c, i, j, kk, s);
              if (wp_out && field_wp)
                for (int c = 0; c < fl2.lda; ++c)
                  wp_out[(int64_t)inp * fl2.lda + c] = FW.at(c, i, j, kk, s);
              if (resetpos && xp_out) {
                int idx[3] = {i, j, k};
                for (int a = 0; a < d; ++a)
                  xp_out[(int64_t)inp * d + a] = (T)(idx[a] - 1) * h[a] + (T)g->min_sub[s * 3 + a];
              }
            }
            ++inp;
          }
        }
  }
  *np_out = inp;
  return 0;
}

extern "C" {

// Single- and double-precision instantiations (ppm_kind_single / _double).
int orc_comp_weights_d(const orc_geom* g, const double* xp, int ldxp, int np, int kernel,
                       const int* list, const int* store_info, int maxp, double* wx1,
                       double* wx2, double* wx3) {
  return comp_weights_impl<double>(g, xp, ldxp, np, kernel, list, store_info, maxp, wx1, wx2, wx3);
}
int orc_comp_weights_s(const orc_geom* g, const float* xp, int ldxp, int np, int kernel,
                       const int* list, const int* store_info, int maxp, float* wx1,
                       float* wx2, float* wx3) {
  return comp_weights_impl<float>(g, xp, ldxp, np, kernel, list, store_info, maxp, wx1, wx2, wx3);
}
int orc_remesh_d(const orc_geom* g, const double* xp, int ldxp, int np, const double* up,
                 int lda, int kernel, const int* ghost, const int* list,
                 const int* store_info, int maxp, const double* wx1, const double* wx2,
                 const double* wx3, double* field, const orc_field* fl, int* err) {
  return remesh_impl<double>(g, xp, ldxp, np, up, lda, kernel, ghost, list, store_info, maxp, wx1,
                             wx2, wx3, field, fl, err);
}
int orc_remesh_s(const orc_geom* g, const float* xp, int ldxp, int np, const float* up,
                 int lda, int kernel, const int* ghost, const int* list,
                 const int* store_info, int maxp, const float* wx1, const float* wx2,
                 const float* wx3, float* field, const orc_field* fl, int* err) {
  return remesh_impl<float>(g, xp, ldxp, np, up, lda, kernel, ghost, list, store_info, maxp, wx1,
                            wx2, wx3, field, fl, err);
}
int orc_create_part_d(const orc_geom* g, const double* field, const orc_field* fl,
                      const double* cutoff, const double* cutoff_weights, int resetpos,
                      const double* field_wp, int lda2, int* np_out, double* up_out,
                      double* xp_out, double* wp_out) {
  return create_part_impl<double>(g, field, fl, cutoff, cutoff_weights, resetpos, field_wp, lda2,
                                  np_out, up_out, xp_out, wp_out);
}
int orc_create_part_s(const orc_geom* g, const float* field, const orc_field* fl,
                      const float* cutoff, const float* cutoff_weights, int resetpos,
                      const float* field_wp, int lda2, int* np_out, float* up_out,
                      float* xp_out, float* wp_out) {
  return create_part_impl<float>(g, field, fl, cutoff, cutoff_weights, resetpos, field_wp, lda2,
                                 np_out, up_out, xp_out, wp_out);
}

// ppm_util_rank3d.f:353-533 and ppm_util_rank2d.f (same structure in 2D).
extern "C++" {
// T: the precision of ppm_util_rank3d_s/_d (positions, bounds and spacing in
// REAL(MK), ppm_util_rank3d.f:353-425).
template <class T>
static int rank_impl(int dim, const T* xp, int ldxp, int np, const T* xmin,
                     const T* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                     int* icount_out) {
  int Nmtot[3] = {1, 1, 1};
  for (int a = 0; a < dim; ++a) Nmtot[a] = Nm[a] + Ngl[a] + Ngl[dim + a];
  int64_t nbox = (int64_t)Nmtot[0] * Nmtot[1] * Nmtot[2];
  T rd[3];
  for (int a = 0; a < dim; ++a) rd[a] = (T)Nm[a] / (xmax[a] - xmin[a]);
  std::vector<int64_t> pbox(np);
  std::vector<int> npbx(nbox, 0);
  int icount = 0;
  int64_t n2 = (int64_t)Nmtot[0] * Nmtot[1];
  for (int ip = 0; ip < np; ++ip) {
    const T* x = xp + (int64_t)ip * ldxp;
    int c[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
      c[a] = (int)std::floor((T)((x[a] - xmin[a]) * rd[a])) + Ngl[a];
      if (x[a] >= xmax[a] && c[a] < Nm[a] + Ngl[a]) c[a] = Nm[a] + Ngl[a];
    }
    for (int a = 0; a < dim; ++a)
      if (x[a] < xmax[a] && c[a] >= Nm[a] + Ngl[a]) c[a] = Nm[a] + Ngl[a] - 1;
    bool in = true;
    for (int a = 0; a < dim; ++a) in = in && c[a] >= 0 && c[a] < Nmtot[a];
    if (in) {
      ++icount;
      pbox[ip] = c[0] + 1 + (int64_t)c[1] * Nmtot[0] + (dim == 3 ? (int64_t)c[2] * n2 : 0);
    } else {
      pbox[ip] = -1;
    }
  }
  for (int ip = 0; ip < np; ++ip)
    if (pbox[ip] > 0) npbx[pbox[ip] - 1]++;
  std::vector<int> cbox(nbox);
  cbox[0] = 1;
  lhbx[0] = 1;
  for (int64_t b = 1; b < nbox; ++b) {
    cbox[b] = cbox[b - 1] + npbx[b - 1];
    lhbx[b] = cbox[b];
  }
  lhbx[nbox] = lhbx[nbox - 1] + npbx[nbox - 1];
  for (int ip = 0; ip < np; ++ip)
    if (pbox[ip] > 0) {
      lpdx[cbox[pbox[ip] - 1] - 1] = ip + 1;
      cbox[pbox[ip] - 1]++;
    }
  *icount_out = icount;
  return 0;
}
}  // extern "C++"

int orc_rank3d_d(const double* xp, int ldxp, int np, const double* xmin,
                 const double* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                 int* icount) {
  return rank_impl(3, xp, ldxp, np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount);
}
int orc_rank2d_d(const double* xp, int ldxp, int np, const double* xmin,
                 const double* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                 int* icount) {
  return rank_impl(2, xp, ldxp, np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount);
}
int orc_rank3d_s(const float* xp, int ldxp, int np, const float* xmin, const float* xmax,
                 const int* Nm, const int* Ngl, int* lpdx, int* lhbx, int* icount) {
  return rank_impl(3, xp, ldxp, np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount);
}
int orc_rank2d_s(const float* xp, int ldxp, int np, const float* xmin, const float* xmax,
                 const int* Nm, const int* Ngl, int* lpdx, int* lhbx, int* icount) {
  return rank_impl(2, xp, ldxp, np, xmin, xmax, Nm, Ngl, lpdx, lhbx, icount);
}

// Adjoint of P2M for a single periodic sub (new routine, no reference
// counterpart).  Weights and stencil exactly as ppm_interp_p2m.f:800-853;
// derivatives of the M'4 pieces: W'(s) = -4 + 5s - 1.5s^2 (1<=s<2),
// -5s + 4.5s^2 (0<=s<1), -5s - 4.5s^2 (-1<=s<0), 4 + 5s + 1.5s^2 (-2<=s<-1).
int orc_p2m_adjoint_d(const orc_geom* g, const double* xp, int ldxp, int np,
                      const double* up, int lda, int kernel, const double* field,
                      const orc_field* fl, double* dw, double* dxo) {
  const int d = g->dim;
  FieldView<double> F(const_cast<double*>(field), fl, d);
  double dxi[3];
  int Nc[3] = {1, 1, 1};
  for (int a = 0; a < d; ++a) { dxi[a] = dxi_mk<double>(g, a); Nc[a] = g->Nm[a] - 1; }
  const int ns = kernel == ORC_KERNEL_MP4 ? 4 : 2;
  for (int p = 0; p < np; ++p) {
    const double* x = xp + (int64_t)p * ldxp;
    const double* u = up + (int64_t)p * lda;
    int base[3] = {0, 0, 0};
    double w[3][4] = {{1, 0, 0, 0}, {1, 0, 0, 0}, {1, 0, 0, 0}};
    double dwv[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int a = 0; a < d; ++a) {
      double x0 = (x[a] - g->min_sub[a]) * dxi[a];
      int i0 = fint(x0);
      double f = x0 - (double)i0;
      if (kernel == ORC_KERNEL_MP4) {
        base[a] = i0;  // 1-based index of node at s = f+1
        mp4_unrolled<double>(f, w[a]);
        double s0 = f + 1.0, s1 = (f + 1.0) - 1.0, s2 = (f + 1.0) - 2.0, s3 = (f + 1.0) - 3.0;
        dwv[a][0] = (-4.0 + 5.0 * s0 - 1.5 * s0 * s0) * dxi[a];
        dwv[a][1] = (-5.0 * s1 + 4.5 * s1 * s1) * dxi[a];
        dwv[a][2] = (-5.0 * s2 - 4.5 * s2 * s2) * dxi[a];
        dwv[a][3] = (4.0 + 5.0 * s3 + 1.5 * s3 * s3) * dxi[a];
      } else {
        base[a] = i0 + 1;
        bsp2_unrolled<double>(f, w[a]);
        dwv[a][0] = -1.0 * dxi[a];
        dwv[a][1] = 1.0 * dxi[a];
      }
    }
    double gx[3] = {0, 0, 0};
    for (int c = 0; c < lda; ++c) {
      double acc = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
      int nk = d == 3 ? ns : 1;
      for (int ii = 0; ii < ns; ++ii)
        for (int jj = 0; jj < ns; ++jj)
          for (int kk = 0; kk < nk; ++kk) {
            int idx[3] = {base[0] + ii, base[1] + jj, d == 3 ? base[2] + kk : 0};
            for (int a = 0; a < d; ++a) idx[a] = ((idx[a] - 1) % Nc[a] + Nc[a]) % Nc[a] + 1;
            double r = F.at(c, idx[0], idx[1], d == 3 ? idx[2] : 0, 0);
            double wz = d == 3 ? w[2][kk] : 1.0;
            double dz = d == 3 ? dwv[2][kk] : 0.0;
            acc += w[0][ii] * w[1][jj] * wz * r;
            ax += dwv[0][ii] * w[1][jj] * wz * r;
            ay += w[0][ii] * dwv[1][jj] * wz * r;
            az += w[0][ii] * w[1][jj] * dz * r;
          }
      dw[(int64_t)p * lda + c] = acc;
      gx[0] += u[c] * ax;
      gx[1] += u[c] * ay;
      gx[2] += u[c] * az;
    }
    for (int a = 0; a < d; ++a) dxo[(int64_t)p * d + a] = gx[a];
  }
  return 0;
}

// CPU baseline: one OpenMP thread per sub, owner-computes (the `mpirun -np P`
// emulation).  Each thread runs the reference's single-sub P2M (containment
// pass + zero + deposit) on its particles, the ghost put/get move data between
// subs, then each thread runs the reference M2P on its particles.
int orc_roundtrip_owned_d(const orc_geom* g, const double* xp, int ldxp, int np,
                          const int* owner, const double* up, int lda, int kernel,
                          const int* ghost, double* field, const orc_field* fl,
                          double* up_out, int nthreads) {
  FieldView<double> F(field, fl, g->dim);
  std::vector<std::vector<int>> lists(g->nsubs);
  for (int p = 0; p < np; ++p) lists[owner[p]].push_back(p);
  int bad = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (int s = 0; s < g->nsubs; ++s) {
    for (int p : lists[s])
      if (!in_sub<double>(g, s, xp + (int64_t)p * ldxp)) ++bad;
    if (!p2m_zero_sub<double>(g, s, ghost, F)) ++bad;
    if (!p2m_deposit_sub<double>(g, s, lists[s], xp, ldxp, up, lda, kernel, F)) ++bad;
  }
  if (bad) return ORC_ERROR_FATAL;
  ghost_put<double>(g, F, ghost);
  ghost_get<double>(g, F, ghost);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (int s = 0; s < g->nsubs; ++s) {
    for (int p : lists[s])
      for (int c = 0; c < lda; ++c) up_out[(int64_t)p * lda + c] = 0.0;
    if (!m2p_sub<double>(g, s, lists[s], xp, ldxp, up_out, lda, kernel, F)) ++bad;
  }
  return bad ? ORC_ERROR_FATAL : 0;
}

}  // extern "C"
