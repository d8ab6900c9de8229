// ppmg_halo.cu -- the ghost exchange between z-slab subdomains: which planes
// travel where (the blocks ppm_map_field_ghost_init.f:234-447 builds for a cut
// along z) and the add of received blocks (ppm_map_field_pop_3d.f, pop with
// add).  The transport that moves the blocks is the caller's.
#include "ppmg_halo.cuh"

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

namespace {

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

template cudaError_t launch_plane_add<double>(double*, const double*, int64_t, cudaStream_t);
template cudaError_t launch_plane_add<float>(float*, const float*, int64_t, cudaStream_t);

}  // namespace ppmg
