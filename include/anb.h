/*
 * anb.h - C ABI of the B200 SIMPLE library (libanb.so).
 *
 * The library replaces, for one GPU, everything the reference's generic_simple_v1 does between
 * "mesh and boundary values are known" and "final fields are known": the 28 face/cell kernels
 * of apps/generic_simple_v1/src/main.cu:1397-1967 and the HYPRE solves it drives
 * (main.cu:1970-2676), orchestrated by the SIMPLE loop of main.cu:3350-3634.  The host program
 * (reader, .case/.bc front end, VTU and summary writers) stays on the CPU side of this ABI.
 *
 * Conventions
 *   - All arrays are host pointers owned by the caller; the library copies in on every call and
 *     writes results into caller-allocated buffers.  The library owns all device memory and one
 *     CUDA stream per context.
 *   - All cell and face arrays use the caller's (OpenFOAM) numbering.  The library renumbers
 *     internally (reverse Cuthill-McKee cells, owner-sorted faces) and maps back on output.
 *   - Every function returns an ANB_* status.  ANB_NOT_CONVERGED is a warning (the reference's
 *     HYPRE error 256: warn and continue); other non-zero values are errors whose text is
 *     available from anb_last_error().  The library never calls exit() or abort().
 *   - A context is not thread-safe; distinct contexts are independent.
 *   - Each call selects the context's device itself and leaves the caller's current device as it
 *     found it.
 *   - Cell fields cross the boundary through a pinned staging buffer of 4 x nCells doubles: the
 *     host threads copy the caller's arrays into it in chunks, each chunk's DMA overlapping the
 *     next copy, and a device kernel permutes between input and layout numbering.
 */
#ifndef ANB_H
#define ANB_H

#ifdef __cplusplus
extern "C" {
#endif

#define ANB_OK 0
#define ANB_NOT_CONVERGED 1
#define ANB_ERR_INVALID 2
#define ANB_ERR_CUDA 3
#define ANB_ERR_MESH 4
#define ANB_ERR_IO 5
#define ANB_ERR_UNSUPPORTED 6
#define ANB_ERR_DIVERGED 7

#define ANB_PRECISION_FP64 0
#define ANB_PRECISION_MIXED 1

typedef struct anb_ctx anb_ctx;

/* polyMesh topology in OpenFOAM order (replaces the Mesh struct, main.cu:61-72). */
typedef struct anb_mesh_desc {
  int n_points;
  const double* points;      /* 3*n_points, xyz interleaved */
  int n_faces;
  const int* face_offsets;   /* n_faces+1, CSR into face_points */
  const int* face_points;
  int n_internal_faces;
  const int* owner;          /* n_faces */
  const int* neighbour;      /* n_internal_faces */
  int n_patches;
  const int* patch_start;    /* n_patches */
  const int* patch_size;     /* n_patches */
} anb_mesh_desc;

/* Solver controls; field meaning and defaults follow Params, main.cu:73-103. */
typedef struct anb_params {
  double rho, mu;
  double u_relax, p_relax;
  int n_nonorth_corr;        /* pressure non-orthogonal correctors (nNonOrthCorr)       */
  int n_vel_nonorth_corr;    /* momentum re-solves (nVelNonOrthCorr)                     */
  int n_pressure_corr;       /* extra pressure passes (nPressureCorr)                    */
  int vel_maxit;
  double vel_tol, vel_rel_tol;
  int p_maxit;
  double p_tol, p_rel_tol;
  double corr_tol;
  int p_amg_rebuild_every;   /* pressure preconditioner rebuild cadence (main.cu:3409)   */
  int p_use_amg;             /* 1: aggregation-AMG preconditioned CG, 0: Jacobi CG       */
  int precision;             /* ANB_PRECISION_FP64 or ANB_PRECISION_MIXED                */
  int device;
  int p_amg_setup_scope;     /* pAmgSetupScope (main.cu:89, 2594-2598): 0 refresh the pressure
                                preconditioner at the rebuild cadence, 1 before every pressure solve */
  int mom_amg;               /* momentum BiCGSTAB preconditioner: 0 Jacobi (the reference's DiagScale,
                                main.cu:2553-2576), 1 aggregation AMG V-cycle on the momentum matrix
                                (FP64 contexts) */
  int mixed_refine;          /* ANB_PRECISION_MIXED only.  0: every linear solve is an FP64 defect
                                correction repeated until the plain method's tolerance is met;
                                1: one FP32 inner solve per system and outer step, to the relative
                                reduction mixed_inner_rtol, the SIMPLE iteration (FP64 assembly
                                residuals, fluxes and continuity) being the refinement loop */
  double mixed_inner_rtol;   /* relative reduction of one FP32 inner solve (default 1e-4) */
} anb_params;

/* Per-outer-iteration monitor values (the stdout line of main.cu:3609-3611). */
typedef struct anb_iter_stats {
  int step;
  int status;                /* ANB_OK or ANB_NOT_CONVERGED for this step's inner solves */
  double mass_res, du_rel, dv_rel, dw_rel, dp_rel;
  int its_u, its_v, its_w;   /* last BiCGSTAB iteration counts                            */
  int its_p_last, its_p_total;
  double iter_seconds;       /* device time of the step (CUDA events)                     */
} anb_iter_stats;

/* Force on a patch (compute_patch_forces_wall_shear, main.cu:2828-2933). */
typedef struct anb_force_report {
  int valid;
  int n_faces;
  double area;
  double Fp[3], Fv[3], F[3];
  double min_wall_distance, max_wall_distance, max_ut, max_shear_mag;
} anb_force_report;

/* Fills the reference defaults (main.cu:73-103). */
void anb_default_params(anb_params* p);

/* Builds the device layout: geometry (main.cu:582-599), RCM renumbering, face coefficients,
 * least-squares gradient operator (main.cu:1159-1251), matrix patterns and the pressure AMG
 * structure.  Replaces build_device_mesh / build_lsq_gradient_operator / init_*_system
 * (main.cu:1072-1251, 2196-2273). */
int anb_create(const anb_mesh_desc* mesh, const anb_params* params, anb_ctx** out);
void anb_destroy(anb_ctx* ctx);
const char* anb_last_error(const anb_ctx* ctx);
/* Wall seconds of anb_create (no counterpart in the reference): t[0] copy-in and topology, t[1]
 * geometry, t[2] device layout (RCM, SELL-32, face coefficients, LSQ moments), t[3] device
 * allocation and upload; t[4..9] the layout's parts (adjacency, LSQ moments, RCM, face order and
 * coefficients, SELL-32 pattern, boundary faces and cell data). */
int anb_setup_times(const anb_ctx* ctx, double t[10]);

/* Cell/face geometry in input numbering (any pointer may be NULL).  cc, xf, nf: 3 per entry. */
int anb_get_geometry(anb_ctx* ctx, double* cc, double* vol, double* xf, double* nf, double* area,
                     double* max_nonorth_deg);
int anb_get_sizes(const anb_ctx* ctx, int* n_cells, int* n_faces, int* n_internal_faces, int* n_patches);

/* Boundary conditions: per patch 1 = Dirichlet, 0 = Neumann (bc_to_int, main.cu:1058) and per
 * face values (nFaces entries, internal entries ignored).  Replaces make_device_bc ×4
 * (main.cu:1107-1114). */
int anb_set_bc(anb_ctx* ctx, const int* type_u, const int* type_v, const int* type_w, const int* type_p,
               const double* u_face, const double* v_face, const double* w_face, const double* p_face);

/* Cell fields (u, v, w, p).  anb_set_state also resets the face flux to zero. */
int anb_set_state(anb_ctx* ctx, const double* u, const double* v, const double* w, const double* p);
int anb_get_state(anb_ctx* ctx, double* u, double* v, double* w, double* p, double* phi);

/* Runs up to nsteps SIMPLE outer iterations (main.cu:3388-3634).  Stops early on
 * convergence (massRes < tol_mass and max(du,dv,dw) < tol_vel) or divergence (massRes not
 * finite or > 1e50, returns ANB_ERR_DIVERGED).  stats (may be NULL) receives one entry per
 * executed step; *steps_done the count.  Returns ANB_NOT_CONVERGED if any inner solve hit
 * its iteration cap. */
int anb_simple_iterate(anb_ctx* ctx, int nsteps, double tol_mass, double tol_vel, anb_iter_stats* stats,
                       int* steps_done);

/* Pressure and wall-shear force integral over one patch on the device (main.cu:2828-2933);
 * patch is the 0-based patch index in input order. */
int anb_patch_force(anb_ctx* ctx, int patch, int normal_sign, anb_force_report* out);

/* Same integral as anb_patch_force, for callers that cannot allocate device memory when they
 * ask for it (an application that owns the whole GPU through its own pool, code running while
 * another component records a CUDA graph, a plugin with a fixed memory budget).  No counterpart
 * in the reference.  The call allocates nothing: its scratch (block partial sums, result,
 * arrival counter) is one file-scope __device__ array of 131,216 bytes.  anb_create places it
 * (and the kernel's code) on the context's device, while allocation is still allowed, and the
 * device keeps it until the process exits.  Limit: one face per thread over the array's 1,024
 * block partials, i.e. patches of at most 262,144 faces (ANB_ERR_INVALID beyond).  Each call
 * clears the counter and result slots on the context's stream before its launch.  All calls
 * share the array: calls that overlap on the GPU (several threads or contexts on one device at
 * once) race and must be serialised by the caller; an overlap that leaves the result unwritten
 * is reported as ANB_ERR_CUDA.  The caller's current device is restored on return. */
int anb_patch_force_nalloc(anb_ctx* ctx, int patch, int normal_sign, anb_force_report* out);

/* ---- scalar libraries (method-of-manufactured-solutions path) --------------------------------
 * Both solves run on the context's mesh and leave its SIMPLE state (U, p, phi) untouched; they
 * reuse the context's matrix storage, so the next SIMPLE step rebuilds its pressure AMG.
 * Face arrays have nFaces entries in input face order and orientation (internal faces first);
 * bc_type/bc_value are read at boundary faces only.  Cell arrays have nCells entries. */
#define ANB_SCALAR_DIRICHLET 0
#define ANB_SCALAR_NEUMANN 1        /* prescribed normal gradient (libpoisson Neumann,
                                       libscalar NeumannGradient) */
#define ANB_SCALAR_ZERO_GRADIENT 2  /* libscalar ZeroGradient (transport only) */
#define ANB_CONVECTION_CENTRAL 0
#define ANB_CONVECTION_UPWIND 1

typedef struct anb_solve_info {
  int iterations;          /* Krylov iterations of the last linear solve */
  int converged;           /* 1 if every linear solve met its tolerance */
  int outer;               /* non-orthogonal outer passes done */
  double final_res_norm;   /* two-norm of the last solve's residual */
  double final_rel_res;    /* final_res_norm / two-norm of its right-hand side */
} anb_solve_info;

/* solve_scalar_elliptic (libpoisson/src/poisson_library.cu:3-47 with the assembly of
 * scalar_elliptic.cu:60-136 and the gradient of gradient.cu:21-83): -div(gamma grad phi) =
 * source with gamma per face (NULL: 1, i.e. solve_poisson), nonorth_corr+1 passes of gradient,
 * assembly and a PCG solve from phi = 0 (one pass when laplacian_nonorth == 0).  The reference
 * solves with HYPRE PCG + BoomerAMG; this library uses its aggregation-AMG PCG at abs_tol
 * (two-norm) / rel_tol.  Errors as the reference: a problem with no Dirichlet face needs
 * use_reference_cell; reference_cell must be a valid cell. */
int anb_scalar_elliptic_solve(anb_ctx* ctx, const double* gamma_face, const double* cell_source,
                              const int* bc_type, const double* bc_value, int laplacian_nonorth,
                              int nonorth_corr, int use_reference_cell, int reference_cell,
                              double reference_value, double abs_tol, double rel_tol, int max_iter,
                              double* phi, anb_solve_info* info);

/* solve_steady_scalar_transport (libscalar/src/scalar_transport_library.cu:475-514 with the
 * assembly of 250-357): div(F phi) - div(gamma grad phi) = Su + Sp phi for a given face flux
 * (NULL: diffusion only), central or upwind convection, nonorth_corr+1 passes when
 * diffusion_nonorth != 0, each a Jacobi-preconditioned BiCGSTAB solve starting from the
 * current phi (x0, or 0 when NULL). */
int anb_scalar_transport_solve(anb_ctx* ctx, const double* face_flux, const double* gamma_face,
                               const double* su, const double* sp, const int* bc_type,
                               const double* bc_value, int convection, int diffusion_nonorth,
                               int nonorth_corr, double abs_tol, double rel_tol, int max_iter,
                               const double* x0, double* phi, anb_solve_info* info);

/* ---- steady sensitivities (no counterpart in the reference) -----------------------------------
 * At a converged SIMPLE state (U, p) the discrete steady residual R(U, p; g, mu) vanishes, with g
 * the Dirichlet velocity values of the boundary faces and mu the viscosity.  For the objective
 * J = dir . F, F the patch force of anb_patch_force, these entry points give dJ/dg and dJ/dmu
 * (discrete adjoint) or dJ along one direction (tangent-linear).  Both solve one linear system
 * with the exact Jacobian of R (hand-written tangent / transposed face-loop kernels) by FGMRES
 * preconditioned with a SIMPLE-type block sweep (momentum BiCGSTAB on A or A^T, pressure AMG-PCG
 * with the forward solver's hierarchy).  Nothing of the iteration history is stored: everything
 * is recomputed from the converged state.  The state should be converged (see
 * anb_steady_residual, anb_newton_solve); FP64 contexts only.  Boundary arrays have 3 x nFaces
 * entries (u | v | w, input face order); only Dirichlet entries are meaningful. */
typedef struct anb_adjoint_info {
  int iterations;          /* FGMRES iterations (Newton: total over the steps) */
  int converged;
  double res_norm;         /* final residual two-norm of the linear system (Newton: of R) */
  double rhs_norm;
  double seconds;          /* wall time of the call */
  int prec_mom_its;        /* preconditioner work: momentum BiCGSTAB iterations (max component) */
  int prec_p_its;          /* and pressure PCG iterations, summed over the applications */
} anb_adjoint_info;

/* Replaces the viscosity of the context (the next iteration and every sensitivity use it). */
int anb_set_viscosity(anb_ctx* ctx, double mu);
/* Steady residual R (4 x nCells: u | v | w | continuity, input cell order; may be NULL) and its
 * two-norms (momentum, continuity) at the current state. */
int anb_steady_residual(anb_ctx* ctx, double* res, double norms[2]);
/* J = dir . F on the patch and its explicit mu-derivative at fixed (U, p). */
int anb_force_objective(anb_ctx* ctx, int patch, int normal_sign, const double dir[3], double* J,
                        double* dJ_dmu_explicit);
/* Newton iterations on R = 0 from the current state (each an FGMRES solve to 1e-3 relative)
 * until |R|_2 <= tol or max_newton steps; used to converge a perturbed state quickly. */
int anb_newton_solve(anb_ctx* ctx, int max_newton, double tol, int lin_max_iter, int* steps,
                     double* res_norm, anb_adjoint_info* info);
/* dJ along (dbc, dmu): solves J_X dX = -R_theta dtheta (FGMRES to 1e-10 relative; the environment
 * variable ANB_ADJ_RTOL, read when a context first uses these entry points, changes it). */
int anb_tangent_linear(anb_ctx* ctx, int patch, int normal_sign, const double dir[3], const double* dbc,
                       double dmu, double* dJ, anb_adjoint_info* info);
/* dJ/dg (3 x nFaces) and dJ/dmu: solves J_X^T lambda = dJ/dX (FGMRES, same tolerance). */
int anb_adjoint_force_grad(anb_ctx* ctx, int patch, int normal_sign, const double dir[3], double* dJ_dbc,
                           double* dJ_dmu, double* J, anb_adjoint_info* info);
/* Jacobian products for tests: dR = J dX + R_g dbc + R_mu dmu (dX 4 x nCells), and
 * out = J^T w with gbc = R_g^T w, gmu = R_mu^T w. */
int anb_debug_jvp(anb_ctx* ctx, const double* dX, const double* dbc, double dmu, double* dR);
int anb_debug_vjp(anb_ctx* ctx, const double* w, double* out, double* gbc, double* gmu);

/* ---- measurement (no counterpart in the reference; used by the benchmark) ------------------
 * Kernel families for anb_profile_select: every launch of the selected family is bracketed by
 * CUDA events on the context's stream and its algorithmic (compulsory) bytes are accumulated. */
#define ANB_KF_NONE 0
#define ANB_KF_GRADIENT 1      /* least-squares gradient            */
#define ANB_KF_MOMENTUM 2      /* momentum assembly                  */
#define ANB_KF_PRESSURE_RC 3   /* pressure matrix + Rhie-Chow flux   */
#define ANB_KF_NONORTH 4       /* non-orthogonal pressure rhs        */
#define ANB_KF_FLUX_FINAL 5    /* flux/velocity correction           */
#define ANB_KF_BICG_SPMV 6     /* BiCGSTAB matrix-vector products    */
#define ANB_KF_PCG_SPMV 7      /* PCG matrix-vector product          */
#define ANB_KF_AMG_RESID0 8    /* V-cycle level 0 down sweep + restriction (ungraphed V-cycles) */
#define ANB_KF_AMG_UP0 9       /* V-cycle level 0 up sweep (ungraphed V-cycles)               */
#define ANB_KF_AMG_COARSE 10   /* V-cycle coarse levels (ungraphed V-cycles)                  */
#define ANB_KF_PCG_UPDATE 11   /* PCG x, r update and residual norm                           */
#define ANB_KF_BICG_VECTOR 12  /* BiCGSTAB vector updates                                     */
#define ANB_KF_MOMENTUM_SOLVE 13 /* whole momentum solve, host polls included                 */
#define ANB_KF_PRESSURE_SOLVE 14 /* whole pressure solve, host polls included                 */
int anb_profile_select(anb_ctx* ctx, int family);
int anb_profile_read(anb_ctx* ctx, long long* launches, double* seconds, double* algo_bytes);
/* Number of kernel launches this process has issued through libanb.so. */
long long anb_launch_count(void);

/* ---- diagnostic entry points (parity tests of single stages) --------------------------------
 * Each runs one stage of the outer iteration on the given host fields (input numbering) and
 * returns its output in input numbering.  Internal-face coefficients are reported per face in
 * the input orientation: a_pn = row owner / column neighbour, a_np = row neighbour / column
 * owner.  Any output pointer may be NULL. */

/* LSQ gradient of phi with the BC set of `field` (0 u, 1 v, 2 w, 3 p): kernel_apply_lsq_gradient,
 * main.cu:1403-1440. */
int anb_debug_gradient(anb_ctx* ctx, int field, const double* phi, double* gx, double* gy, double* gz);

/* Momentum system for old fields (u,v,w,p): assembly + relaxation + rAU
 * (main.cu:2346-2528).  rhs is 3*nCells (u, v, w components). */
int anb_debug_momentum(anb_ctx* ctx, const double* u, const double* v, const double* w, const double* p,
                       double* diag, double* a_pn, double* a_np, double* rhs, double* rau);

/* Pressure matrix from rAU (main.cu:2532-2551) and the Rhie-Chow predicted flux + continuity
 * (main.cu:1474-1536) for velocity (u,v,w) and pressure p. */
int anb_debug_pressure(anb_ctx* ctx, const double* u, const double* v, const double* w, const double* p,
                       const double* rau, double* diag, double* a_pn, double* phi_star, double* div_star);

/* Divergence of the explicit non-orthogonal correction flux (kernel_pressure_nonorth_flux_and_
 * divergence, main.cu:1538-1593) for rAU and the gradient (gx, gy, gz) of the pressure
 * correction; internal faces and the Dirichlet-pressure boundary faces contribute. */
int anb_debug_nonorth(anb_ctx* ctx, const double* rau, const double* gx, const double* gy, const double* gz,
                      double* div_no);

/* Solves the current pressure system A x = b with the configured preconditioned CG to
 * (p_tol, p_rel_tol); x holds the initial guess on entry.  *iters receives the count. */
int anb_debug_pressure_solve(anb_ctx* ctx, const double* b, double* x, int* iters, double* final_res);

#ifdef __cplusplus
}
#endif
#endif /* ANB_H */
