/*
 * ppmg.h -- C-ABI of the B200-native particle<->mesh interpolation and
 * remeshing library (libppmg.so).  A drop-in replacement for the hot path of
 * PPM (PPMLibrary/ppm_legacy): ppm_interp_p2m, ppm_interp_m2p,
 * ppm_rmsh_comp_weights, ppm_rmsh_remesh, ppm_rmsh_create_part, the periodic
 * ghost get/put of ppm_map_field_ghost and the cell ranking of
 * ppm_neighlist_clist / ppm_util_rank{2,3}d.
 *
 * Conventions (shared by every entry point):
 *  - Arrays keep the reference's Fortran column-major layout.  `xp` points at
 *    xp(1,1) of xp(ldxp, Np); `up` at up(1,1) of up(ldup, Np) (scalar variants:
 *    up(Np)); `field_up` at the first element of field_up(ldf, lb(1):ub(1),
 *    lb(2):ub(2)[, lb(3):ub(3)], 1:1), i.e. one subdomain, with the spatial
 *    bounds passed in f_lb[dim] / f_ub[dim] (the allocation may be larger than
 *    the 1-g:Nm+g box the routine writes; nothing outside the box is touched).
 *  - Geometry comes from ppmg_mesh_register (the module state that
 *    ppm_topo_mkfield / ppm_mesh_on_subs leave behind in the reference).
 *  - `info` follows the reference: 0 on success, else a severity
 *    (-1 fatal, -2 error; ppm_param.h:372-375) with the reference error number
 *    (ppm_error.h, e.g. 503 ppm_err_argument, 405 ppm_err_part_unass) and a
 *    message retrievable through ppmg_last_error.  The library never aborts
 *    (the reference calls MPI_Abort on fatal errors, ppm_error.f:195-199).
 *  - Plain entry points take HOST pointers, are synchronous and do their own
 *    host<->device copies.  `_dev` twins take DEVICE pointers and a
 *    cudaStream_t (as void*), enqueue asynchronously on that stream and report
 *    data-dependent errors (e.g. particles outside the subdomain) through
 *    ppmg_sync_status.
 *  - Supported: one subdomain per GPU with periodic boundaries on every face,
 *    kernels M'4 (2) and B-spline 2 (1); anything else returns info = -2 with
 *    errno 503 and does no work (no CPU fallback).
 *  - Precision of the double-precision ('d') variants: PPMG_PREC_FP64 computes
 *    weights and sums in FP64; PPMG_PREC_MIXED forms cell offsets in FP64 and
 *    weights/products in FP32 with compensated FP32 accumulation per node.
 *    Single-precision ('s') variants compute in FP32.
 */
#ifndef PPMG_H
#define PPMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPMG_PREC_FP64 0
#define PPMG_PREC_MIXED 1

/* ---- status, configuration ------------------------------------------- */

/* Version of this library (major*10000 + minor*100 + patch). */
int ppmg_version(void);

/* Last error of the calling thread: returns its info, writes errno and a
 * NUL-terminated message (ppm_error.f:90-199 keeps the same triple). */
int ppmg_last_error(int* errnum, char* msg, int msglen);

/* Precision of the 'd' variants (default PPMG_PREC_FP64, or the
 * PPMG_PRECISION environment variable "fp64" / "mixed" at load time). */
void ppmg_set_precision(int mode, int* info);
int ppmg_get_precision(void);

/* Number of CUDA kernels this library launched so far (all threads). */
int64_t ppmg_launch_count(void);

/* ---- geometry (replaces ppm_topo_mkfield / ppm_mesh_on_subs state) -------
 * min_sub/max_sub: [nsubs][3]; subs_bc: [nsubs][6]; istart/nnodes: [nsubs][3]
 * (C row-major = Fortran (3,nsubs) column-major).  Nm: global nodes per axis;
 * bcdef: 2*dim codes (ppm_param.h:333-338). */
void ppmg_mesh_register(int topo_id, int mesh_id, int dim, const double* min_phys,
                        const double* max_phys, const int* Nm, const int* bcdef, int nsubs,
                        const double* min_sub, const double* max_sub, const int* subs_bc,
                        const int* istart, const int* nnodes, int* info);
void ppmg_mesh_unregister(int topo_id, int mesh_id, int* info);
/* The subdomain (0-based isub) this GPU computes on: the one-entry
 * ppm_isublist of the process (ppm/src/ppm_topo_mkfield.f:311-319 builds the
 * reference's per-process sub list).  Required when nsubs > 1.  Supported
 * decompositions: cartesian in 3D (ppm_param_decomp_cartesian and the
 * pencil and slab cuts): every axis is either spanned by all subdomains or
 * cut into intervals that all subdomains share, each interval starting on
 * the previous one's last node.  Along a cut axis the local subdomain is not
 * periodic: the 3D P2M, M2P, P2M adjoint and remeshing (comp_weights,
 * remesh, create_part) compute on it alone, P2M and remesh leave in their
 * ghost layers the contributions owed to the neighbours, M2P and the adjoint
 * read their field's ghost layers, create_part skips the shared upper node
 * of each cut axis; the exchange between the subdomains (the ghost put / get
 * of ppm_map_field_ghost, ppm_map_field_send.f) is the caller's: through a
 * transport registered with ppmg_halo_set_transport (below), or, for slabs
 * along z, ppm_legacy_b200.halo over torch.distributed.  Without a transport
 * the standalone ghost mapping returns info = -2 (errno 503) on a cut
 * subdomain; the allocation-free P2M always does. */
void ppmg_mesh_set_local_sub(int topo_id, int mesh_id, int isub, int* info);

/* ---- ghost exchange between z-slab subdomains ---------------------------
 * The inter-subdomain part of ppm_map_field_ghost (ppm/src/ppm_map_field_ghost.f:392-670,
 * the blocks of ppm_map_field_ghost_init.f:234-447 for a cut along z, moved
 * by ppm_map_field_send.f and added / copied by ppm_map_field_pop_3d.f).
 * z is field_up's slowest axis, so every block is a run of whole node planes
 * (all ldf rows, the field's full x-y extent), contiguous in memory.  With nz
 * the local slab's cell layers (real nodes 1..nz+1, node nz+1 shared with the
 * slab above) and g the z ghost width:
 *   put: planes nz+1..nz+1+g go up, planes 1-g..1 go down; what arrives from
 *        below is added to planes 1..1+g, from above to planes nz+1-g..nz+1
 *        (both copies of a shared plane end with the full sum);
 *   get: planes nz+1-g..nz go up, planes 2..1+g go down; what arrives from
 *        below replaces planes 1-g..0, from above planes nz+2..nz+1+g.
 * Tags name the direction of travel. */
#define PPMG_HALO_TAG_UP 17   /* a block travelling to the slab above */
#define PPMG_HALO_TAG_DOWN 18 /* a block travelling to the slab below */

typedef struct {
  int peer;      /* subdomain (0-based) on the other side */
  int tag;       /* PPMG_HALO_TAG_UP or PPMG_HALO_TAG_DOWN */
  void* buf;     /* the block: `bytes` contiguous bytes */
  int64_t bytes;
} ppmg_halo_block;

/* The caller's transport (MPI, NCCL, ...): move the blocks and return 0, or
 * nonzero on failure.  Each send must reach the receive of the same tag on
 * the peer.  Blocks are device memory (on_device = 1, the calls of the
 * `_dev` entry points; `stream` is the caller's stream, on which the sent
 * blocks are produced and after which the received blocks are read) or host
 * memory (on_device = 0, the host entry points; stream is NULL).  Every
 * subdomain's process calls it with the same exchange in the same order. */
typedef int (*ppmg_halo_fn)(void* ctx, int nsend, const ppmg_halo_block* sends, int nrecv,
                            const ppmg_halo_block* recvs, int on_device, void* stream);

/* Register (fn != NULL) or remove (fn == NULL) the transport of a handle
 * whose local subdomain is one of several.  With a transport,
 * ppmg_map_field_ghost_{d,s}[_dev] on it performs the put or get with the
 * neighbouring subdomains (whole planes for slabs along z, the boxes of
 * ppmg_halo_plan_boxes otherwise), and the 3D P2M and remesh end with the
 * ghost put, as ppm_interp_p2m.f:3665-3718 and ppm_rmsh_remesh.f:876-924
 * end theirs.  A transport that fails gives
 * info = -1, errno 2 (ppm_err_mpi_fail, ppm_error.h:153). */
void ppmg_halo_set_transport(int topo_id, int mesh_id, ppmg_halo_fn fn, void* ctx, int* info);

/* The blocks of one exchange, from the geometry alone (no device, no
 * handle): the slab isub of nsubs z-slabs given as in ppmg_mesh_register
 * (istart, nnodes: [nsubs][3], Nmz: global nodes along z), a field_up(ldf,
 * f_lb:f_ub) and maptype ppm_param_map_ghost_put (6) or _get (5).  Outputs,
 * index 0 = towards / from the slab above, 1 = the slab below:
 *   *count      elements per block (whole planes, ldf rows each);
 *   send_off[b] element offset into field_up of the block sent to
 *               send_peer[b] with tag send_tag[b] (0: UP, 1: DOWN);
 *   recv_off[b] element offset of the planes the block arriving from
 *               recv_peer[b] with tag recv_tag[b] is added to (put) or
 *               copied into (get). */
void ppmg_halo_plan(int nsubs, const int* istart, const int* nnodes, int Nmz, int isub,
                    int64_t ldf, const int64_t* f_lb, const int64_t* f_ub, const int* ghostsize,
                    int maptype, int64_t* count, int* send_peer, int* send_tag,
                    int64_t* send_off, int* recv_peer, int* recv_tag, int64_t* recv_off,
                    int* info);

/* ---- ghost exchange of any cartesian decomposition ------------------------
 * Cuts along x, y and z (the subdomains of ppm_param_decomp_cartesian, each
 * axis cut into intervals shared by all subdomains of the other axes).  A
 * block is a box of the local field in its 1-based node indices, lo..hi
 * inclusive per axis; it travels as all ldf rows of each node, x fastest
 * (ldf * ext0 * ext1 * ext2 elements, ext = hi - lo + 1).  Along a cut axis
 * the local nodes 1..nnodes hold the subdomain's real nodes (the last one
 * shared with the next subdomain); along an uncut axis the box spans the
 * whole field box 1-g..Nm+g.  With G the ghost-extended box of a subdomain
 * and R its real box, in global node indices, and t in {-1, 0, 1} per cut
 * axis (the periodic shift, N cells):
 *   put: subdomain s sends G_s and (R_q + tN) to q, which adds it to its
 *        nodes; every copy of a real node ends with the sum of all copies;
 *   get: s sends (R'_s and (G_q + tN)) minus (R_q + tN) to q, cut into at
 *        most one box per cut axis, which q copies into its ghost nodes;
 *        R'_s is R_s without its last node along each cut axis (the next
 *        subdomain's first), so that no node arrives twice.
 * Tags: 100 + 3 * d + k, d = (t0+1) + 3 (t1+1) + 9 (t2+1) the shift, k the
 * piece; a send and its receive carry the same tag.  Slabs along z (cuts
 * along z only) exchange whole planes instead (ppmg_halo_plan). */
typedef struct {
  int peer;       /* subdomain (0-based) on the other side */
  int tag;
  int64_t lo[3];  /* first node of the box per axis (local, 1-based) */
  int64_t hi[3];  /* last node, inclusive */
} ppmg_halo_box;

/* The boxes of one exchange of subdomain isub (maptype 6 = put, 5 = get)
 * from the geometry alone (istart, nnodes: [nsubs][3] as in
 * ppmg_mesh_register; Nm: global nodes per axis).  *nsend / *nrecv get the
 * box counts; at most `cap` boxes of each list are written (cap = 0 asks for
 * the counts).  Receives are listed in the order they are applied. */
void ppmg_halo_plan_boxes(int nsubs, const int* istart, const int* nnodes, const int* Nm,
                          int isub, const int* ghostsize, int maptype, int cap,
                          ppmg_halo_box* sends, int* nsend, ppmg_halo_box* recvs, int* nrecv,
                          int* info);

/* Wait for all work of the handle's `_dev` calls on `stream` and return the
 * data-dependent status latched since the last call (info/errno as above). */
void ppmg_sync_status(int topo_id, int mesh_id, void* stream, int* info);

/* ---- ppm_interp_p2m  (ppm/src/ppm_interp_p2m.f:127-163) ------------------
 * field_up(1-g:Nm+g) is overwritten: real nodes hold the periodic sum
 * (node Nm equals node 1), ghost layers hold the periodic images of the real
 * nodes (the state a following ghost get would leave). */
#define PPMG_P2M_V_ARGS(R)                                                          \
  const R *xp, int64_t ldxp, int64_t Np, const R *up, int64_t ldup, int lda,       \
      int topo_id, int mesh_id, int kernel, const int *ghostsize, R *field_up,      \
      int64_t ldf, const int64_t *f_lb, const int64_t *f_ub, int *info
#define PPMG_P2M_S_ARGS(R)                                                          \
  const R *xp, int64_t ldxp, int64_t Np, const R *up, int topo_id, int mesh_id,     \
      int kernel, const int *ghostsize, R *field_up, const int64_t *f_lb,           \
      const int64_t *f_ub, int *info

void ppmg_interp_p2m_dv_3d(PPMG_P2M_V_ARGS(double)); /* ppm_interp_p2m.f:159 */
void ppmg_interp_p2m_sv_3d(PPMG_P2M_V_ARGS(float));  /* ppm_interp_p2m.f:156 */
void ppmg_interp_p2m_ds_3d(PPMG_P2M_S_ARGS(double)); /* ppm_interp_p2m.f:151 */
void ppmg_interp_p2m_ss_3d(PPMG_P2M_S_ARGS(float));  /* ppm_interp_p2m.f:148 */
void ppmg_interp_p2m_dv_2d(PPMG_P2M_V_ARGS(double)); /* ppm_interp_p2m.f:141 */
void ppmg_interp_p2m_sv_2d(PPMG_P2M_V_ARGS(float));  /* ppm_interp_p2m.f:138 */
void ppmg_interp_p2m_ds_2d(PPMG_P2M_S_ARGS(double)); /* ppm_interp_p2m.f:133 */
void ppmg_interp_p2m_ss_2d(PPMG_P2M_S_ARGS(float));  /* ppm_interp_p2m.f:130 */
void ppmg_interp_p2m_dv_3d_dev(PPMG_P2M_V_ARGS(double), void* stream);
void ppmg_interp_p2m_sv_3d_dev(PPMG_P2M_V_ARGS(float), void* stream);
void ppmg_interp_p2m_dv_2d_dev(PPMG_P2M_V_ARGS(double), void* stream);
void ppmg_interp_p2m_sv_2d_dev(PPMG_P2M_V_ARGS(float), void* stream);

/* P2M that allocates nothing.  No counterpart in the reference: this entry
 * point exists for callers that cannot let the library call cudaMalloc -- a
 * code that hands nearly all device memory to its own pool at start-up, or a
 * time-step loop that must not stall on the device-wide synchronisation that
 * cudaFree (and cudaMalloc, when new memory is mapped) brings.
 * Same arguments, results and error reporting as ppmg_interp_p2m_dv_3d_dev,
 * but its sort and tile scratch live in one 16 MiB array compiled into the
 * library, which every GPU that loads the library holds until exit.  Limits:
 * Np <= 131072, Nx*Ny*Nz <= 262144 cells, lda <= 4; larger calls return
 * info = -2 (errnum 503) and launch nothing.
 * The first call on a device looks up the array's device address (this may
 * load the library's device code on that device): make it before any stream
 * capture.  The address is kept per device and looked up again when the
 * device's context has changed (after a cudaDeviceReset).  Particles outside
 * the subdomain are reported through ppmg_sync_status as for the _dev entry
 * point (info = -1, errnum 405).  All calls on a device share the array and each overwrites the
 * previous call's contents (what must start at zero is cleared by the call):
 * calls whose GPU work overlaps -- different streams, or different host
 * threads -- race and corrupt each other's results; order them on one stream. */
void ppmg_interp_p2m_dv_3d_noalloc(PPMG_P2M_V_ARGS(double), void* stream);

/* ---- ppm_interp_m2p  (ppm/src/ppm_interp_m2p.f:126-162) ------------------
 * up is overwritten (zeroed, then the gather).  Reads the real nodes 1..Nm-1
 * of field_up with periodic wrap, i.e. the result of the reference's M2P
 * after a ghost get. */
#define PPMG_M2P_V_ARGS(R)                                                          \
  const R *xp, int64_t ldxp, int64_t Np, R *up, int64_t ldup, int lda, int topo_id, \
      int mesh_id, int kernel, const int *ghostsize, const R *field_up, int64_t ldf, \
      const int64_t *f_lb, const int64_t *f_ub, int *info
#define PPMG_M2P_S_ARGS(R)                                                          \
  const R *xp, int64_t ldxp, int64_t Np, R *up, int topo_id, int mesh_id,           \
      int kernel, const int *ghostsize, const R *field_up, const int64_t *f_lb,     \
      const int64_t *f_ub, int *info

void ppmg_interp_m2p_dv_3d(PPMG_M2P_V_ARGS(double)); /* ppm_interp_m2p.f:158 */
void ppmg_interp_m2p_sv_3d(PPMG_M2P_V_ARGS(float));  /* ppm_interp_m2p.f:155 */
void ppmg_interp_m2p_ds_3d(PPMG_M2P_S_ARGS(double)); /* ppm_interp_m2p.f:150 */
void ppmg_interp_m2p_ss_3d(PPMG_M2P_S_ARGS(float));  /* ppm_interp_m2p.f:147 */
void ppmg_interp_m2p_dv_2d(PPMG_M2P_V_ARGS(double)); /* ppm_interp_m2p.f:140 */
void ppmg_interp_m2p_sv_2d(PPMG_M2P_V_ARGS(float));  /* ppm_interp_m2p.f:137 */
void ppmg_interp_m2p_ds_2d(PPMG_M2P_S_ARGS(double)); /* ppm_interp_m2p.f:132 */
void ppmg_interp_m2p_ss_2d(PPMG_M2P_S_ARGS(float));  /* ppm_interp_m2p.f:129 */
void ppmg_interp_m2p_dv_3d_dev(PPMG_M2P_V_ARGS(double), void* stream);
void ppmg_interp_m2p_sv_3d_dev(PPMG_M2P_V_ARGS(float), void* stream);
void ppmg_interp_m2p_dv_2d_dev(PPMG_M2P_V_ARGS(double), void* stream);
void ppmg_interp_m2p_sv_2d_dev(PPMG_M2P_V_ARGS(float), void* stream);

/* ---- adjoint of P2M (no reference counterpart) -----------------------------
 * Given the adjoint field r = dL/dfield (real nodes, periodic), returns
 * dw(lda,Np) = M2P(r) (the exact transpose of P2M) and
 * dx(dim,Np) = sum_a up(a,p) * sum_n grad_x W(xi_p - n) r(a,n).
 * Weights are recomputed (nothing is stored between forward and backward). */
void ppmg_interp_p2m_adjoint_dv_3d(const double* xp, int64_t ldxp, int64_t Np,
                                   const double* up, int64_t ldup, int lda, int topo_id,
                                   int mesh_id, int kernel, const double* r_field,
                                   int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                                   double* dw, int64_t lddw, double* dx, int64_t lddx,
                                   int* info);
void ppmg_interp_p2m_adjoint_dv_3d_dev(const double* xp, int64_t ldxp, int64_t Np,
                                       const double* up, int64_t ldup, int lda, int topo_id,
                                       int mesh_id, int kernel, const double* r_field,
                                       int64_t ldf, const int64_t* f_lb, const int64_t* f_ub,
                                       double* dw, int64_t lddw, double* dx, int64_t lddx,
                                       int* info, void* stream);

/* ---- ppm_map_field_ghost (ppm/src/ppm_map_field_ghost.f:61-89) -----------
 * maptype ppm_param_map_ghost_get (5): ghost and duplicate nodes <- periodic
 * images of the real nodes; ppm_param_map_ghost_put (6): real nodes += their
 * periodic images in the ghost box (node Nm and node 1 both get the sum), the
 * ghost layers are left unchanged -- the reference's init/put/push/send/pop
 * cycle for one periodic subdomain. */
void ppmg_map_field_ghost_d(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                            const int64_t* f_ub, int topo_id, int mesh_id,
                            const int* ghostsize, int maptype, int* info);
void ppmg_map_field_ghost_s(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                            const int64_t* f_ub, int topo_id, int mesh_id,
                            const int* ghostsize, int maptype, int* info);
void ppmg_map_field_ghost_d_dev(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int maptype, int* info, void* stream);
void ppmg_map_field_ghost_s_dev(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int maptype, int* info, void* stream);

/* ---- ppm_rmsh_comp_weights (ppm/src/ppm_rmsh_comp_weights.f:96-103) ------
 * Computes the per-particle 1D weights and keeps them (with the particle
 * list) in the handle, like the reference's module state
 * (ppm_module_data_rmsh.f:47-73).  wx1/wx2/wx3 may be NULL; when given they
 * receive the reference layout wx(1:2ks, 1:1, 1-ks:Np+ks) (ks = 2 for M'4,
 * 1 for bsp2), indexed by the particle's position in the sub list, which for
 * one subdomain is the particle index. */
void ppmg_rmsh_comp_weights_d(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                              int mesh_id, int kernel, double* wx1, double* wx2,
                              double* wx3, int* info);
/* Device twin: xp and the optional wx1/wx2/wx3 are device arrays, work is
 * enqueued on `stream`; errors latch for ppmg_sync_status. */
void ppmg_rmsh_comp_weights_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                  int mesh_id, int kernel, double* wx1, double* wx2,
                                  double* wx3, int* info, void* stream);
/* Single precision (ppm_rmsh_comp_weights_s): weights in FP32; a following
 * remesh must be single precision too. */
void ppmg_rmsh_comp_weights_s(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                              int mesh_id, int kernel, float* wx1, float* wx2, float* wx3,
                              int* info);
void ppmg_rmsh_comp_weights_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                  int mesh_id, int kernel, float* wx1, float* wx2, float* wx3,
                                  int* info, void* stream);

/* ---- ppm_rmsh_remesh (ppm/src/ppm_rmsh_remesh.f:90-124) ------------------
 * Scatter with the weights of the last comp_weights call of this handle;
 * the field box is overwritten as in P2M. */
void ppmg_rmsh_remesh_dv_3d(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, double* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info);
void ppmg_rmsh_remesh_dv_2d(const double* xp, int64_t ldxp, int64_t Np, const double* up,
                            int64_t ldup, int lda, int topo_id, int mesh_id, int kernel,
                            const int* ghostsize, double* field_up, int64_t ldf,
                            const int64_t* f_lb, const int64_t* f_ub, int* info);
/* Device twins (device xp, up, field_up; enqueued on `stream`). */
void ppmg_rmsh_remesh_dv_3d_dev(PPMG_P2M_V_ARGS(double), void* stream);
void ppmg_rmsh_remesh_dv_2d_dev(PPMG_P2M_V_ARGS(double), void* stream);
/* Single precision (ppm_rmsh_remesh.f:94-110 _sv/_ss: lda = 1 for scalars). */
void ppmg_rmsh_remesh_sv_3d(PPMG_P2M_V_ARGS(float));
void ppmg_rmsh_remesh_sv_2d(PPMG_P2M_V_ARGS(float));
void ppmg_rmsh_remesh_sv_3d_dev(PPMG_P2M_V_ARGS(float), void* stream);
void ppmg_rmsh_remesh_sv_2d_dev(PPMG_P2M_V_ARGS(float), void* stream);

/* ---- ppm_rmsh_create_part (ppm/src/ppm_rmsh_create_part.f:90-171) --------
 * Two calls: with up == NULL it only returns the new particle count in *np;
 * then the caller allocates up(lda, np) [, xp(dim, np), wp(lda2, np)] and
 * calls again to fill them.  Nodes are visited k, j, i with i fastest, node
 * Nm excluded on periodic axes; a node becomes a particle when
 * cutoff[0] < strength < cutoff[1], strength = |u|_2 (or |u*cutoff_weights|_2). */
void ppmg_rmsh_create_part_d(const double* field_up, int64_t ldf, int lda,
                             const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                             int mesh_id, const double* cutoff, const double* cutoff_weights,
                             int resetpos, const double* field_wp, int64_t ldfw, int lda2,
                             int64_t* np, double* up, double* xp, double* wp, int* info);
/* Device twin: field_up, field_wp and the outputs up/xp/wp are device
 * arrays (cutoff and cutoff_weights stay host arrays); both calls run on
 * `stream`, and the counting call synchronises it to return *np. */
void ppmg_rmsh_create_part_d_dev(const double* field_up, int64_t ldf, int lda,
                                 const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                                 int mesh_id, const double* cutoff, const double* cutoff_weights,
                                 int resetpos, const double* field_wp, int64_t ldfw, int lda2,
                                 int64_t* np, double* up, double* xp, double* wp, int* info,
                                 void* stream);
/* Single precision (ppm_rmsh_create_part_s*): field, cutoffs and outputs FP32. */
void ppmg_rmsh_create_part_s(const float* field_up, int64_t ldf, int lda,
                             const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                             int mesh_id, const float* cutoff, const float* cutoff_weights,
                             int resetpos, const float* field_wp, int64_t ldfw, int lda2,
                             int64_t* np, float* up, float* xp, float* wp, int* info);
void ppmg_rmsh_create_part_s_dev(const float* field_up, int64_t ldf, int lda,
                                 const int64_t* f_lb, const int64_t* f_ub, int topo_id,
                                 int mesh_id, const float* cutoff, const float* cutoff_weights,
                                 int resetpos, const float* field_wp, int64_t ldfw, int lda2,
                                 int64_t* np, float* up, float* xp, float* wp, int* info,
                                 void* stream);

/* ---- ppm_neighlist_clist / ppm_util_rank3d (ppm/src/ppm_neighlist_clist.f:
 * 371-429, ppm/src/ppm_util_rank3d.f:353-533) ------------------------------
 * Stable counting sort of particles into the cells of a box: lpdx receives
 * the 1-based ids of the particles inside the mesh (ascending id within each
 * cell), lhbx(1:nbox+1) the 1-based first position of each cell; returns the
 * count of particles inside in *icount.  Bit-identical to the reference. */
void ppmg_util_rank3d_d(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                        const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info);
void ppmg_util_rank2d_d(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                        const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info);
/* Single precision (ppm_util_rank3d_s / ppm_util_rank2d_s): positions, bounds
 * and the cell spacing in FP32, as the reference's REAL(4) build. */
void ppmg_util_rank3d_s(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                        const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info);
void ppmg_util_rank2d_s(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                        const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                        int* lhbx, int64_t* icount, int* info);
/* ---- FFT Poisson solver (ppm_fdsolver_solve_3d with the spectral step of
 * ppm/src/ppm_fdsolver_poisson_3d.f:60-82) ----------------------------------
 * Solves lap(phi) = omega on the periodic mesh of one subdomain, component
 * by component, in place: omega is read at the unique nodes 1..Nm-1 of
 * field_up(ldf, f_lb:f_ub), every mode of its transform is multiplied by
 * -1/|k|^2 (k_a = 2 pi / L_a times the wave number folded to |.| <= N_a/2,
 * the zero mode set to 0), and phi is written to every node of the box
 * 1-g:Nm+g (real nodes and their periodic images).  FFTs by cuFFT (the
 * reference uses FFTW).  On a slab along z with a halo transport the slab
 * form solves the whole domain: xy transforms on every slab, an all-to-all
 * to z pencils through the transport, the z transforms and the spectral
 * step, and back; phi then fills the slab's box, its z ghost planes from the
 * neighbours.  On other cartesian cuts (with a transport) omega's unique
 * nodes go to P virtual z-slabs (slab q on subdomain q's process), the slab
 * form solves there, and phi returns to every node of each subdomain's box
 * 1-g:Nm+g, ghosts and images included (ppm_fdsolver_map_3d.f maps the
 * field the same way); this needs at least as many y and z cells as
 * subdomains (else info = -2, errno 503). */
void ppmg_fdsolver_poisson_3d_d(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int* info);
void ppmg_fdsolver_poisson_3d_s(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                const int64_t* f_ub, int topo_id, int mesh_id,
                                const int* ghostsize, int* info);
void ppmg_fdsolver_poisson_3d_d_dev(double* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                    const int64_t* f_ub, int topo_id, int mesh_id,
                                    const int* ghostsize, int* info, void* stream);
void ppmg_fdsolver_poisson_3d_s_dev(float* field_up, int64_t ldf, int lda, const int64_t* f_lb,
                                    const int64_t* f_ub, int topo_id, int mesh_id,
                                    const int* ghostsize, int* info, void* stream);

/* ---- particle redistribution between z-slab subdomains (the routing of
 * ppm_map_part_partial, ppm/src/ppm_map_part_partial.f:288-420) ------------
 * route: every particle of the device array xp goes to the subdomain that
 * contains it among the local slab and its two z neighbours (closed-lower /
 * open-upper boxes; positions are expected inside the domain, the client
 * imposing the periodic bounds first as in PPM).  perm (device, Np ints)
 * receives the particle ids grouped by class: kept, to the slab below, to the
 * slab above, in no neighbour; each class in ascending id.  counts (host, 4)
 * receives the class sizes; the call returns once they are known.  Particles
 * in no neighbour give info = -2, errno 405.  Slabs along z only (other
 * cuts: info = -2, errno 503; the global routing below serves them).
 * gather: dst(0:lda-1, j) = src(0:lda-1, perm[j]) for j < n (device arrays;
 * positions or any particle property). */
void ppmg_map_part_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                               int mesh_id, int* perm, int64_t* counts, int* info, void* stream);
void ppmg_map_part_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                               int mesh_id, int* perm, int64_t* counts, int* info, void* stream);
/* Global routing (ppm_map_part_global, ppm/src/ppm_map_part_global.f:355-420):
 * every particle to the subdomain that contains it among all nsubs (<= 255;
 * closed-lower / open-upper boxes min_sub .. max_sub on every axis; any
 * registered decomposition).  perm receives the particle ids grouped by
 * destination subdomain 0..nsubs-1 and then those in none, each group in
 * ascending id; counts (host, nsubs+1) the group sizes.  Particles in no
 * subdomain are left out of the exchange without an error, as in the
 * reference (ppm_map_part_global.f:437-442). */
/* Partial routing on any cartesian cut (ppm_map_part_partial,
 * ppm/src/ppm_map_part_partial.f:288-420 over the neighbour list): as the
 * global routing below, but only the local subdomain and its neighbours
 * (ppmg_halo_neighbours) are destinations; particles in none of them go to
 * the last group and give info = -2, errno 405 (ppm_map_part_partial.f:
 * 480-485).  On slabs along z the destinations are the slab and its two z
 * neighbours, the classes of ppmg_map_part_route_* in a per-subdomain
 * layout. */
void ppmg_map_part_partial_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                       int mesh_id, int* perm, int64_t* counts, int* info,
                                       void* stream);
void ppmg_map_part_partial_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                       int mesh_id, int* perm, int64_t* counts, int* info,
                                       void* stream);
/* The neighbours of subdomain isub of a cartesian cut, from the geometry
 * alone (ascending, isub excluded): the subdomains whose boxes share a face,
 * an edge or a corner with isub's, across the periodic faces too (the
 * reference's ineighsubs for such a cut).  *nneigh gets their number; at
 * most cap are written. */
void ppmg_halo_neighbours(int nsubs, const int* istart, const int* nnodes, const int* Nm,
                          int isub, int cap, int* neigh, int* nneigh, int* info);
void ppmg_map_part_global_route_d_dev(const double* xp, int64_t ldxp, int64_t Np, int topo_id,
                                      int mesh_id, int* perm, int64_t* counts, int* info,
                                      void* stream);
void ppmg_map_part_global_route_s_dev(const float* xp, int64_t ldxp, int64_t Np, int topo_id,
                                      int mesh_id, int* perm, int64_t* counts, int* info,
                                      void* stream);
void ppmg_map_part_gather_d_dev(const double* src, int64_t lds, int lda, const int* perm,
                                int64_t n, double* dst, int64_t ldd, int* info, void* stream);
void ppmg_map_part_gather_s_dev(const float* src, int64_t lds, int lda, const int* perm,
                                int64_t n, float* dst, int64_t ldd, int* info, void* stream);

/* Device twins: xp, lpdx (Np entries, the first icount valid) and lhbx
 * (nbox+1) are device arrays, the work runs on `stream`; the bounds, Nm and
 * Ngl are host arrays.  The call returns once the lists are complete (the
 * ranking's scratch is shared by all calls), with icount set when given. */
void ppmg_util_rank3d_d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                            const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream);
void ppmg_util_rank2d_d_dev(const double* xp, int64_t ldxp, int64_t Np, const double* xmin,
                            const double* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream);
void ppmg_util_rank3d_s_dev(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                            const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream);
void ppmg_util_rank2d_s_dev(const float* xp, int64_t ldxp, int64_t Np, const float* xmin,
                            const float* xmax, const int* Nm, const int* Ngl, int* lpdx,
                            int* lhbx, int64_t* icount, int* info, void* stream);

/* ---- Instrumentation (no counterpart in the reference) -------------------
 * ppmg_kernel_timing(1) makes the library bracket, on the launching stream,
 * every launch of its 3D P2M gather kernel (part 0), its 3D M2P gather
 * kernel (part 1) and every cell-order sort (part 2, all its kernels) with
 * CUDA events.  ppmg_kernel_timing_read(part, ...) waits for the recorded
 * events and returns the summed device time in ms and the number of timed
 * launches since the last read of that part, then resets them (returns 0, or
 * -2 for an unknown part).  Off by default; enabling it adds two event
 * records per timed launch. */
void ppmg_kernel_timing(int enable);
int ppmg_kernel_timing_read(int part, double* ms, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* PPMG_H */
