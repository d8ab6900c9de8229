// ppmg_halo.cu -- the ghost exchange between subdomains: which nodes travel
// where (the blocks ppm_map_field_ghost_init.f:234-447 builds: whole planes
// for slabs along z, boxes per neighbour and periodic shift for cuts along
// several axes), the packing of boxes and the add of received blocks
// (ppm_map_field_pop_3d.f, pop with add).  The transport that moves the
// blocks is the caller's.
#include "ppmg_halo.cuh"

#include <array>
#include <map>
#include <set>

namespace ppmg {

const char* halo_plan(int nsubs, const int* istart, const int* nnodes, int Nmz, int isub,
                      int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, int gz, bool put,
                      HaloPlan& out) {
  if (nsubs < 2 || isub < 0 || isub >= nsubs) return "isub / nsubs out of range";
  if (gz < 0) return "negative ghost width";
  // the slab's first and last global node along z; its neighbours share them
  // (periodic: the last node of the domain is its first)
  auto z0 = [&](int s) { return istart[3 * s + 2]; };
  auto z1 = [&](int s) { return istart[3 * s + 2] + nnodes[3 * s + 2] - 1; };
  const int lo = z0(isub), hi = z1(isub);
  int below = -1, above = -1, nb = 0, na = 0;
  for (int s = 0; s < nsubs; ++s) {
    if (z1(s) == (lo > 1 ? lo : Nmz)) { below = s; ++nb; }
    if (z0(s) == (hi < Nmz ? hi : 1)) { above = s; ++na; }
  }
  if (nb != 1 || na != 1) return "the subdomains are not a decomposition into z-slabs";
  const int nz = nnodes[3 * isub + 2] - 1;
  if (nz < gz || nz < 1) return "the z ghost width exceeds the slab's cell layers";
  if (f_lb[2] > 1 - gz || f_ub[2] < nz + 1 + gz)
    return "field_up bounds do not cover the z ghost planes 1-g .. Nm+g";
  if (ldf < 1) return "ldf < 1";
  const int64_t plane = ldf * (f_ub[0] - f_lb[0] + 1) * (f_ub[1] - f_lb[1] + 1);
  auto off = [&](int64_t z) { return (z - f_lb[2]) * plane; };
  // index 0: the block sent up / received from below carries TAG_UP;
  // index 1: the block sent down / received from above carries TAG_DOWN
  out.send_peer[0] = above;
  out.send_peer[1] = below;
  out.send_tag[0] = out.recv_tag[0] = PPMG_HALO_TAG_UP;
  out.send_tag[1] = out.recv_tag[1] = PPMG_HALO_TAG_DOWN;
  out.recv_peer[0] = below;
  out.recv_peer[1] = above;
  if (put) {
    out.count = (int64_t)(gz + 1) * plane;
    out.send_off[0] = off(nz + 1);
    out.send_off[1] = off(1 - gz);
    out.recv_off[0] = off(1);
    out.recv_off[1] = off(nz + 1 - gz);
  } else {
    out.count = (int64_t)gz * plane;
    out.send_off[0] = off(nz + 1 - gz);
    out.send_off[1] = off(2);
    out.recv_off[0] = off(1 - gz);
    out.recv_off[1] = off(nz + 2);
  }
  return nullptr;
}

const char* check_cartesian(int nsubs, const int* istart, const int* nnodes, const int Nm[3]) {
  if (nsubs < 1) return "no subdomain";
  std::vector<std::vector<int>> starts(3);
  for (int a = 0; a < 3; ++a) {
    // an axis is cut when the subdomains do not span it; all of them agree
    const bool cut = nnodes[a] != Nm[a];
    std::map<int, int> iv;  // istart -> nnodes of the axis' intervals
    for (int q = 0; q < nsubs; ++q) {
      const int i0 = istart[3 * q + a], n = nnodes[3 * q + a];
      if ((n != Nm[a]) != cut) return "the subdomains are not a cartesian decomposition";
      if (n < 2 || i0 < 1) return "a subdomain has no cell along an axis";
      auto it = iv.find(i0);
      if (it != iv.end() && it->second != n)
        return "the subdomains are not a cartesian decomposition";
      iv[i0] = n;
    }
    // the intervals tile 1 .. Nm, each starting on the last node of the previous
    int next = 1;
    for (auto& kv : iv) {
      if (kv.first != next) return "the subdomains are not a cartesian decomposition";
      next = kv.first + kv.second - 1;
      starts[a].push_back(kv.first);
    }
    if (next != Nm[a]) return "the subdomains do not cover the mesh";
  }
  // every combination of the axes' intervals is one subdomain
  if ((int64_t)starts[0].size() * starts[1].size() * starts[2].size() != nsubs)
    return "the subdomains are not a cartesian decomposition";
  std::set<std::array<int, 3>> seen;
  for (int q = 0; q < nsubs; ++q)
    if (!seen.insert({istart[3 * q], istart[3 * q + 1], istart[3 * q + 2]}).second)
      return "two subdomains share a box";
  return nullptr;
}

void cart_neighbours(int nsubs, const int* istart, const int* nnodes, const int Nm[3], int isub,
                     std::vector<int>& out) {
  out.clear();
  for (int q = 0; q < nsubs; ++q) {
    if (q == isub) continue;
    bool near = true;
    for (int a = 0; a < 3 && near; ++a) {
      const int s0 = istart[3 * isub + a], s1 = s0 + nnodes[3 * isub + a] - 1;
      const int q0 = istart[3 * q + a], q1 = q0 + nnodes[3 * q + a] - 1;
      near = q0 == s0 || q0 == s1 || q1 == s0 || (s1 == Nm[a] && q0 == 1) ||
             (s0 == 1 && q1 == Nm[a]);
    }
    if (near) out.push_back(q);
  }
}

const char* halo_boxes(int nsubs, const int* istart, const int* nnodes, const int Nm[3],
                       int isub, const int g[3], bool put, std::vector<HaloBox>& sends,
                       std::vector<HaloBox>& recvs) {
  sends.clear();
  recvs.clear();
  if (nsubs < 2 || isub < 0 || isub >= nsubs) return "isub / nsubs out of range";
  if (const char* why = check_cartesian(nsubs, istart, nnodes, Nm)) return why;
  bool open[3];
  int64_t N[3];
  for (int a = 0; a < 3; ++a) {
    open[a] = nnodes[3 * isub + a] != Nm[a];
    N[a] = Nm[a] - 1;
    if (g[a] < 0) return "negative ghost width";
    for (int q = 0; q < nsubs; ++q)
      if (open[a] && g[a] > nnodes[3 * q + a] - 1)
        return "a ghost width exceeds a subdomain's cells";
  }
  auto box = [&](int q, int a, bool ghosts, int64_t& lo, int64_t& hi) {
    if (!open[a]) {
      lo = 1 - g[a];
      hi = Nm[a] + g[a];
    } else {
      lo = istart[3 * q + a] - (ghosts ? g[a] : 0);
      hi = istart[3 * q + a] + nnodes[3 * q + a] - 1 + (ghosts ? g[a] : 0);
    }
  };
  // block of one (sender S, receiver Rv, shift t of the receiver's box in
  // the sender's frame) in global node indices of the sender's frame.
  // put: G_S and (R_Rv + tN); get: the part of (G_Rv + tN) and R'_S outside
  // (R_Rv + tN), cut into at most one box per cut axis (the standard
  // decomposition of a box minus a box), k its index.  R'_S is R_S without
  // its last node along every cut axis (that node is the next subdomain's
  // first): every node is then sent by one subdomain only, and the boxes a
  // get receives never overlap.  Non-cut axes span the whole field box
  // (their images are every subdomain's own).
  auto blocks = [&](int S, int Rv, const int t[3], std::vector<std::pair<int, HaloBox>>& out) {
    out.clear();
    int64_t jl[3], jh[3], rl[3], rh[3];
    for (int a = 0; a < 3; ++a) {
      int64_t sl, sh, ql, qh;
      if (put) {
        box(S, a, true, sl, sh);
        box(Rv, a, false, ql, qh);
      } else {
        box(S, a, false, sl, sh);
        if (open[a]) --sh;
        box(Rv, a, true, ql, qh);
      }
      if (open[a]) {
        ql += t[a] * N[a];
        qh += t[a] * N[a];
        jl[a] = sl > ql ? sl : ql;
        jh[a] = sh < qh ? sh : qh;
        if (jl[a] > jh[a]) return;
      } else {
        box(S, a, true, jl[a], jh[a]);
      }
      box(Rv, a, false, rl[a], rh[a]);
      if (open[a]) {
        rl[a] += t[a] * N[a];
        rh[a] += t[a] * N[a];
      }
    }
    HaloBox b;
    if (put) {
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = jl[a];
        b.hi[a] = jh[a];
      }
      out.push_back({0, b});
      return;
    }
    // get: box J minus box R (over the cut axes): for cut axis a in order,
    // [inside R along the earlier cut axes] x [outside R along a] x [J along the rest]
    int k = 0;
    for (int a = 0; a < 3; ++a) {
      if (!open[a]) continue;
      // J_a outside R_a: one interval (R_Rv + tN touches J at one end only)
      int64_t ol, oh;
      if (jl[a] < rl[a]) {
        ol = jl[a];
        oh = (jh[a] < rl[a] - 1 ? jh[a] : rl[a] - 1);
      } else if (jh[a] > rh[a]) {
        ol = (jl[a] > rh[a] + 1 ? jl[a] : rh[a] + 1);
        oh = jh[a];
      } else {
        ++k;
        continue;  // J_a inside R_a: nothing outside along a
      }
      bool empty = false;
      for (int c = 0; c < 3; ++c) {
        if (c < a && open[c]) {  // inside R along the earlier cut axes
          b.lo[c] = jl[c] > rl[c] ? jl[c] : rl[c];
          b.hi[c] = jh[c] < rh[c] ? jh[c] : rh[c];
        } else if (c == a) {
          b.lo[c] = ol;
          b.hi[c] = oh;
        } else {
          b.lo[c] = jl[c];
          b.hi[c] = jh[c];
        }
        if (b.lo[c] > b.hi[c]) empty = true;
      }
      if (!empty) out.push_back({k, b});
      ++k;
    }
  };
  auto dir = [](const int t[3]) { return (t[0] + 1) + 3 * (t[1] + 1) + 9 * (t[2] + 1); };
  std::vector<std::pair<int, HaloBox>> bl;
  const int s = isub;
  for (int q = 0; q < nsubs; ++q) {
    int t[3];
    for (t[2] = -1; t[2] <= 1; ++t[2])
      for (t[1] = -1; t[1] <= 1; ++t[1])
        for (t[0] = -1; t[0] <= 1; ++t[0]) {
          bool ok = true;
          for (int a = 0; a < 3; ++a) ok = ok && (open[a] || t[a] == 0);
          if (!ok || (q == s && t[0] == 0 && t[1] == 0 && t[2] == 0)) continue;
          // s sends to q: blocks in s's frame, q's box shifted by t
          blocks(s, q, t, bl);
          for (auto& kb : bl) {
            HaloBox b = kb.second;
            b.peer = q;
            b.tag = 100 + 3 * dir(t) + kb.first;
            for (int a = 0; a < 3; ++a) {
              const int64_t o = open[a] ? istart[3 * s + a] - 1 : 0;
              b.lo[a] -= o;
              b.hi[a] -= o;
            }
            sends.push_back(b);
          }
          // s receives from q: q's frame, s's box shifted by t; s's frame: minus tN
          blocks(q, s, t, bl);
          for (auto& kb : bl) {
            HaloBox b = kb.second;
            b.peer = q;
            b.tag = 100 + 3 * dir(t) + kb.first;
            for (int a = 0; a < 3; ++a) {
              const int64_t o = open[a] ? istart[3 * s + a] - 1 + t[a] * N[a] : 0;
              b.lo[a] -= o;
              b.hi[a] -= o;
            }
            recvs.push_back(b);
          }
        }
  }
  return nullptr;
}

namespace {

// One thread per element of the launch's boxes (index space: the boxes back
// to back in table order); a box is found by binary search over the rows'
// first indices, and its elements sit in the buffer from the row's offset.
template <class T>
__global__ void k_box_copy(T* __restrict__ field, int64_t ldf, int64_t s0, int64_t s1,
                           int64_t s2, int lb0, int lb1, int lb2,
                           const int64_t* __restrict__ tab, int nbox, int64_t tot,
                           T* __restrict__ buf, int mode) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nbox - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tab[8 * mid + 6] <= i) lo = mid; else hi = mid - 1;
    }
    const int64_t* b = tab + 8 * lo;
    int64_t r = i - b[6];
    const int64_t j = b[7] + r;  // the element's place in the buffer
    const int64_t c = r % ldf;
    r /= ldf;
    const int64_t x = r % b[3];
    r /= b[3];
    const int64_t y = r % b[4];
    const int64_t z = r / b[4];
    const int64_t o = (b[0] + x - lb0) * s0 + (b[1] + y - lb1) * s1 + (b[2] + z - lb2) * s2 + c;
    if (mode == kBoxPack)
      buf[j] = field[o];
    else if (mode == kBoxCopy)
      field[o] = buf[j];
    else
      field[o] += buf[j];
  }
}

template <class T>
__global__ void k_plane_add(T* __restrict__ dst, const T* __restrict__ src, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

}  // namespace

template <class T>
cudaError_t launch_plane_add(T* dst, const T* src, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + 255) / 256;
  const int grid = (int)(blocks < 148 * 16 ? blocks : 148 * 16);
  k_plane_add<T><<<grid, 256, 0, st>>>(dst, src, n);
  count_launch();
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_box_copy(T* field, int64_t ldf, const int64_t s[3], const int lb[3],
                            const int64_t* tab, int nbox, int64_t tot, T* buf, int mode,
                            cudaStream_t st) {
  if (tot <= 0 || nbox <= 0) return cudaSuccess;
  const int64_t blocks = (tot + 255) / 256;
  const int grid = (int)(blocks < 148 * 16 ? blocks : 148 * 16);
  k_box_copy<T><<<grid, 256, 0, st>>>(field, ldf, s[0], s[1], s[2], lb[0], lb[1], lb[2], tab,
                                      nbox, tot, buf, mode);
  count_launch();
  return cudaGetLastError();
}
template cudaError_t launch_box_copy<double>(double*, int64_t, const int64_t*, const int*,
                                             const int64_t*, int, int64_t, double*, int,
                                             cudaStream_t);
template cudaError_t launch_box_copy<float>(float*, int64_t, const int64_t*, const int*,
                                            const int64_t*, int, int64_t, float*, int,
                                            cudaStream_t);

template cudaError_t launch_plane_add<double>(double*, const double*, int64_t, cudaStream_t);
template cudaError_t launch_plane_add<float>(float*, const float*, int64_t, cudaStream_t);

}  // namespace ppmg
