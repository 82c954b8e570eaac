/*
 * oracle.h - CPU oracle for the SIMPLE outer iteration of the reference's generic_simple_v1.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the B200 library: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load it.  The product
 * (libanb.so and the anabasis_simple host program) never links or calls it.
 *
 * It restates, in plain serial/OpenMP C++, the reference's algorithm with each function citing
 * the file:line it follows (apps/generic_simple_v1/src/main.cu, "GSV1" below).  Pinning status:
 *   - geometry, LSQ gradient, Rhie-Chow, continuity, non-orthogonal flux, flux correction and
 *     patch forces are checked against the reference's own host functions compiled from
 *     the reference sources by oracle/build_ref.sh (tests/test_oracle_vs_reference.py);
 *   - the linear solves of the reference are HYPRE 3.0.0 (not vendored, not installable here):
 *     the oracle replaces them with deterministic FP64 Krylov solvers run to tight tolerance, so
 *     solver-level parity is unpinned and parity is checked on converged/tightly-solved fields.
 */
#ifndef ANB_ORACLE_H
#define ANB_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_mesh orc_mesh;

typedef struct orc_params {
  double rho, mu, u_relax, p_relax;
  int n_nonorth_corr, n_vel_nonorth_corr, n_pressure_corr;
  int vel_maxit; double vel_tol, vel_rel_tol;
  int p_maxit; double p_tol, p_rel_tol;
  double corr_tol, tol_mass, tol_vel;
  int n_threads;
  int p_use_amg;  /* 1: pressure PCG preconditioned by the oracle's aggregation AMG, else Jacobi */
} orc_params;

typedef struct orc_stats {
  double mass_res, du, dv, dw, dp;
  int its_u, its_v, its_w, its_p_last, its_p_total;
} orc_stats;

/* topology in OpenFOAM order; returns NULL and fills err on failure */
orc_mesh* orc_mesh_create(int n_points, const double* points, int n_faces, const int* face_off,
                          const int* face_pts, int n_internal, const int* owner, const int* neigh,
                          int n_patches, const int* patch_start, const int* patch_size,
                          char* err, int errlen);
void orc_mesh_free(orc_mesh* m);
int orc_mesh_ncells(const orc_mesh* m);
/* sizes: n_points, n_faces, n_internal, n_cells, n_patches, length of the face point list */
void orc_mesh_sizes(const orc_mesh* m, int* s6);
void orc_mesh_patches(const orc_mesh* m, int* patch_start, int* patch_size);
/* topology back in the creation arrays' layout (any pointer may be NULL) */
void orc_mesh_topology(const orc_mesh* m, double* points, int* face_off, int* face_pts, int* owner, int* neigh);

/* Synthetic channel case (channel.cpp): Lx x Ly x Lz box of nx x ny x nz hexes, interior nodes
 * jittered by +-jitter of the local spacing (mt19937_64(seed)), optionally without the obstacle
 * block box = {x0, x1, y0, y1} (NULL: 0.45 0.55 0.15 0.25); patches patch_0_0 walls, patch_1_0
 * inlet, patch_2_0 outlet, patch_3_0 obstacle. */
orc_mesh* orc_channel_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, double jitter,
                             unsigned long long seed, int obstacle, const double* box, char* err, int errlen);

/* Boundary values per patch (apply_bc_specs_to_legacy_face_arrays, velocity_bc_eval.cu:197-290):
 * vkind per patch with 4 parameters each in vpar, pkind per patch with the fixed value in pval.
 * Outputs as orc_set_bc takes them.  Returns 0, or 1 with a message in err. */
#define ORC_VEL_WALL_NOSLIP 0
#define ORC_VEL_ZERO_GRADIENT 1
#define ORC_VEL_UNIFORM 2        /* vpar: ux uy uz */
#define ORC_VEL_PARABOLIC_BOX 3  /* vpar: H Umax coordA coordB; average patch normal */
#define ORC_P_ZERO_GRADIENT 0
#define ORC_P_FIXED_VALUE 1
int orc_eval_bc(const orc_mesh* m, const int* vkind, const double* vpar, const int* pkind, const double* pval,
                int* tu, int* tv, int* tw, int* tp, double* uf, double* vf, double* wf, double* pf, char* err,
                int errlen);
void orc_mesh_geometry(const orc_mesh* m, double* cc, double* vol, double* xf, double* nf, double* sf,
                       double* af, double* max_nonorth);

/* BC: per patch type (1 Dirichlet / 0 Neumann) for u,v,w,p and per-face values (nFaces) */
void orc_set_bc(orc_mesh* m, const int* tu, const int* tv, const int* tw, const int* tp,
                const double* uf, const double* vf, const double* wf, const double* pf);

/* kernel_apply_lsq_gradient on the build_lsq_gradient_operator coefficients (GSV1:1159-1251,
 * 1403-1440), field = 0 u, 1 v, 2 w, 3 p */
void orc_lsq_gradient(const orc_mesh* m, int field, const double* phi, double* gx, double* gy, double* gz);

/* momentum system for old fields (GSV1:2346-2528 and 3350-3405 with it == 1) */
void orc_momentum(const orc_mesh* m, double rho, double mu, double u_relax, const double* u,
                  const double* v, const double* w, const double* p, double* diag, double* a_pn,
                  double* a_np, double* rhs3, double* rau);

/* pressure matrix (GSV1:2532-2551) + Rhie-Chow flux (GSV1:1474-1521) + continuity
 * (GSV1:1523-1536) */
void orc_pressure(const orc_mesh* m, double rho, const double* u, const double* v, const double* w,
                  const double* p, const double* rau, double* diag, double* a_pn, double* phi_star,
                  double* div_star);

/* kernel_pressure_nonorth_flux_and_divergence (GSV1:1538-1593) for p' gradient g (3 x nCells SoA),
 * and kernel_correct_face_fluxes_simple_nonorth (GSV1:1615-1658) on top of it */
void orc_nonorth(const orc_mesh* m, const double* rau, const double* g, double* phi_no, double* div_no);
void orc_flux_correct(const orc_mesh* m, const double* rau, const double* phi_star, const double* pcorr,
                      const double* g, double* phi);

/* nsteps SIMPLE iterations (GSV1:3388-3634).  u,v,w,p in/out, phi out (nFaces).  stats may be
 * NULL (else nsteps entries).  Returns executed steps (early stop on convergence). */
int orc_simple_run(orc_mesh* m, const orc_params* prm, int nsteps, double* u, double* v, double* w,
                   double* p, double* phi, orc_stats* stats);

/* compute_patch_forces_wall_shear (GSV1:2828-2933); out: Fp[3], Fv[3], F[3], area, nFaces,
 * minDn, maxDn, maxUt, maxShear */
void orc_patch_force(const orc_mesh* m, int patch, int normal_sign, double mu, const double* u,
                     const double* v, const double* w, const double* p, double* out11);

/* scalar libraries: libpoisson gradient (gradient.cu:21-83) and the elliptic / transport
 * assemblies (scalar_elliptic.cu:60-136, scalar_transport_library.cu:250-357) in face-coefficient
 * form; bc_type per face: 0 Dirichlet, 1 normal gradient, 2 zero gradient */
void orc_scalar_gradient(const orc_mesh* m, const int* bc_type, const double* bc_value, const double* phi,
                         double* gx, double* gy, double* gz);
void orc_scalar_assemble(const orc_mesh* m, int transport, int upwind, int nonorth, const double* gamma,
                         const double* flux, const double* src, const double* sp, const int* bc_type,
                         const double* bc_value, const double* grad, int ref_cell, double ref_value,
                         double* diag, double* a_pn, double* a_np, double* rhs);

#ifdef __cplusplus
}
#endif
#endif
