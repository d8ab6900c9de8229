/*
 * ppm_oracle.h -- CPU restatement of PPM's particle<->mesh interpolation and
 * remeshing path, used ONLY as test infrastructure (the checker) and as the
 * timed CPU baseline.  Nothing in the product library links or calls it.
 *
 * Parity status: UNPINNED against reference outputs.  The reference
 * (PPM, Fortran 90 + MPI) ships no tests, fixtures or golden vectors, and no
 * Fortran compiler exists on the build or GPU hosts, so the reference itself
 * cannot be run.  This restatement is pinned instead by (i) line-by-line
 * agreement with the reference loops cited per function in ppm_oracle.cpp
 * (same stencil origin, same Horner forms, same term order, the FP32 mesh
 * spacing of M2P/comp_weights), and (ii) known-answer vectors computed in
 * exact rational arithmetic from the kernel definitions
 * (tests/golden/make_golden.py) plus analytic identities (partition of unity,
 * moment reproduction, P2M = transpose(M2P)).
 *
 * Compile with -O2 -ffp-contract=off: the reference build (gfortran -O2,
 * x86-64 baseline) emits no fused multiply-adds.
 *
 * Array conventions follow the Fortran column-major layout exactly:
 *   xp(ldxp, Np), up(lda, Np), field(lda, lb0:ub0, lb1:ub1[, lb2:ub2], nsubs).
 * Scalar (`*s_*`) reference variants are the lda = 1 case of the same memory
 * layout and the same arithmetic.
 */
#ifndef PPM_ORACLE_H
#define PPM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Geometry of one topology + mesh, as PPM's module state holds it
 * (ppm_module_data / ppm_module_data_mesh).  Sub arrays are sub-major:
 * min_sub[isub*3 + d], subs_bc[isub*6 + face], istart[isub*3 + d]. */
typedef struct {
  int dim;
  int nsubs;
  double min_phys[3];
  double max_phys[3];
  int Nm[3];
  int bcdef[6];
  const double* min_sub;
  const double* max_sub;
  const int* subs_bc;
  const int* istart;
  const int* nnodes;
} orc_geom;

/* Field array descriptor: field(lda, lb[0]:ub[0], lb[1]:ub[1], [lb[2]:ub[2],] nsubs) */
typedef struct {
  int lda;
  int lb[3];
  int ub[3];
} orc_field;

/* Reference constants (ppm_param.h:333-338, 372-375, 405-407; ppm_error.h). */
enum {
  ORC_KERNEL_BSP2 = 1,
  ORC_KERNEL_MP4 = 2,
  ORC_KERNEL_M3P6 = 3,
  ORC_BC_PERIODIC = 1,
  ORC_ERROR_FATAL = -1,
  ORC_ERROR_ERROR = -2,
  ORC_ERR_PART_UNASS = 405,
  ORC_ERR_ARGUMENT = 503,
  ORC_ERR_OUT_OF_FIELD = 9001 /* oracle-only: a deposit left the field box */
};

/* Particle -> sub assignment (two passes, ppm_interp_p2m.f:496-750).
 * list_out: concatenation of per-sub lists (ascending particle index, 0-based),
 * store_info: count per sub.  Returns info; errno in *err. */
int orc_assign_d(const orc_geom* g, const double* xp, int ldxp, int np, int* list_out,
                 int* store_info, int* err);
int orc_assign_s(const orc_geom* g, const float* xp, int ldxp, int np, int* list_out,
                 int* store_info, int* err);

/* ppm_interp_p2m (zero, deposit, ghost put). */
int orc_p2m_d(const orc_geom* g, const double* xp, int ldxp, int np, const double* up,
              int lda, int kernel, const int* ghost, double* field, const orc_field* fl,
              int* err);
int orc_p2m_s(const orc_geom* g, const float* xp, int ldxp, int np, const float* up,
              int lda, int kernel, const int* ghost, float* field, const orc_field* fl,
              int* err);
/* P2M deposit only (no ghost put): the field the reference holds before the put. */
int orc_p2m_noput_d(const orc_geom* g, const double* xp, int ldxp, int np,
                    const double* up, int lda, int kernel, const int* ghost,
                    double* field, const orc_field* fl, int* err);

/* ppm_interp_m2p (zero up, gather).  The client ghost get is NOT included. */
int orc_m2p_d(const orc_geom* g, const double* xp, int ldxp, int np, double* up, int lda,
              int kernel, const int* ghost, const double* field, const orc_field* fl,
              int* err);
int orc_m2p_s(const orc_geom* g, const float* xp, int ldxp, int np, float* up, int lda,
              int kernel, const int* ghost, const float* field, const orc_field* fl,
              int* err);

/* ppm_map_field_ghost get / put on all subs of the topology (block
 * intersections + periodic shifts, ppm_map_field_ghost_init.f:234-447). */
int orc_ghost_get_d(const orc_geom* g, double* field, const orc_field* fl, const int* ghost);
int orc_ghost_put_d(const orc_geom* g, double* field, const orc_field* fl, const int* ghost);
int orc_ghost_get_s(const orc_geom* g, float* field, const orc_field* fl, const int* ghost);
int orc_ghost_put_s(const orc_geom* g, float* field, const orc_field* fl, const int* ghost);

/* ppm_rmsh_comp_weights: wx(1:2ks, 1:nsubs, 1-ks:maxp+ks) per axis,
 * column-major; list/store_info as orc_assign. maxp = max(store_info). */
int orc_comp_weights_d(const orc_geom* g, const double* xp, int ldxp, int np, int kernel,
                       const int* list, const int* store_info, int maxp, double* wx1,
                       double* wx2, double* wx3);
int orc_comp_weights_s(const orc_geom* g, const float* xp, int ldxp, int np, int kernel,
                       const int* list, const int* store_info, int maxp, float* wx1,
                       float* wx2, float* wx3);
/* ppm_rmsh_remesh with stored weights (zero field, scatter, ghost put). */
int orc_remesh_d(const orc_geom* g, const double* xp, int ldxp, int np, const double* up,
                 int lda, int kernel, const int* ghost, const int* list,
                 const int* store_info, int maxp, const double* wx1, const double* wx2,
                 const double* wx3, double* field, const orc_field* fl, int* err);
int orc_remesh_s(const orc_geom* g, const float* xp, int ldxp, int np, const float* up,
                 int lda, int kernel, const int* ghost, const int* list,
                 const int* store_info, int maxp, const float* wx1, const float* wx2,
                 const float* wx3, float* field, const orc_field* fl, int* err);

/* ppm_rmsh_create_part.  Pass 1 (count) when up_out == NULL.
 * cutoff_weights may be NULL; field_wp/wp_out/lda2 optional (NULL / 0). */
int orc_create_part_d(const orc_geom* g, const double* field, const orc_field* fl,
                      const double* cutoff, const double* cutoff_weights, int resetpos,
                      const double* field_wp, int lda2, int* np_out, double* up_out,
                      double* xp_out, double* wp_out);
int orc_create_part_s(const orc_geom* g, const float* field, const orc_field* fl,
                      const float* cutoff, const float* cutoff_weights, int resetpos,
                      const float* field_wp, int lda2, int* np_out, float* up_out,
                      float* xp_out, float* wp_out);

/* ppm_util_rank3d / ppm_util_rank2d: stable cell ranking.
 * lpdx: 1-based particle ids (size >= np), lhbx: nbox+1 1-based pointers.
 * Returns the number of particles inside the mesh in *icount. */
int orc_rank3d_d(const double* xp, int ldxp, int np, const double* xmin,
                 const double* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                 int* icount);
int orc_rank2d_d(const double* xp, int ldxp, int np, const double* xmin,
                 const double* xmax, const int* Nm, const int* Ngl, int* lpdx, int* lhbx,
                 int* icount);
/* Single precision (ppm_util_rank3d_s / rank2d_s): positions, bounds and the
 * cell spacing in FP32. */
int orc_rank3d_s(const float* xp, int ldxp, int np, const float* xmin, const float* xmax,
                 const int* Nm, const int* Ngl, int* lpdx, int* lhbx, int* icount);
int orc_rank2d_s(const float* xp, int ldxp, int np, const float* xmin, const float* xmax,
                 const int* Nm, const int* Ngl, int* lpdx, int* lhbx, int* icount);

/* Adjoint of P2M on one periodic sub (no reference counterpart): given the
 * adjoint field r on real nodes, dw(a,p) = sum_n W(xi_p - n) r(a,n) and
 * dx(d,p) = sum_a up(a,p) * sum_n dW/dx_d r(a,n).  FP64. */
int orc_p2m_adjoint_d(const orc_geom* g, const double* xp, int ldxp, int np,
                      const double* up, int lda, int kernel, const double* field,
                      const orc_field* fl, double* dw, double* dx);

/* CPU baseline: emulation of `mpirun -np P` by P OpenMP threads, one sub per
 * thread (cartesian split), each running the reference P2M loops on the
 * particles it owns, then ghost put, ghost get, then M2P.  Particles must be
 * pre-partitioned: owner[p] = sub of particle p. */
int orc_roundtrip_owned_d(const orc_geom* g, const double* xp, int ldxp, int np,
                          const int* owner, const double* up, int lda, int kernel,
                          const int* ghost, double* field, const orc_field* fl,
                          double* up_out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
