/*
 * efsi.h — C ABI of the B200 implementation of EulerianFSI.jl's four-stage
 * IMEX fractional step (`integrate_step!`).
 *
 * The library owns every device buffer of one simulation context behind an
 * opaque handle.  Host arrays are Julia-style column-major (x index fastest)
 * FP64 matrices:
 *   U            (Nx+1) x Ny      x-face velocity
 *   V            Nx x (Ny+1)      y-face velocity
 *   cell fields  Nx x Ny          phi, resource c, sigma_xx, sigma_yy, sigma_xy,
 *                                 growth target G, correction potential q
 * Host pointers are only read or written during a call and never retained.
 * Every call is synchronous: results are valid on return.  One handle must not
 * be used by two host threads at the same time.
 *
 * Every entry point returns an EFSI_* status.  Non-zero statuses map onto the
 * exception types the reference throws (see the EFSI_* list below); the message
 * text is available from efsi_last_error().
 */
#ifndef EFSI_H
#define EFSI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EFSI_ABI_VERSION 2

#if defined(__GNUC__)
#define EFSI_API __attribute__((visibility("default")))
#else
#define EFSI_API
#endif

/* ---- status codes ------------------------------------------------------- */
#define EFSI_OK            0
#define EFSI_ARG           1  /* Julia ArgumentError (e.g. TimeIntegrationIMEX.jl:1121, Projection.jl:213) */
#define EFSI_DIM           2  /* Julia DimensionMismatch (TimeIntegrationIMEX.jl:500-516)                    */
#define EFSI_SOLVE         3  /* Julia ErrorException from a linear solve (Projection.jl:281, :293)          */
#define EFSI_DOMAIN        4  /* Julia DomainError, non-SPD structure tensor (StructureTensor.jl:491-496)     */
#define EFSI_CUDA          5  /* CUDA runtime failure or no usable device                                    */
#define EFSI_UNSUPPORTED   6  /* valid reference input that the device step does not implement              */

/* ---- boundary conditions (BoundaryConditions.jl:23-46) ------------------- */
#define EFSI_BC_PERIODIC           0
#define EFSI_BC_DIRICHLET          1
#define EFSI_BC_NEUMANN            2
#define EFSI_BC_MIXED              3
#define EFSI_BC_ADVECTIVE_OUTFLOW  4

/* One side of a BoundaryConditionSetup.  Julia boundary data may be a scalar,
 * a vector or a callable (BoundaryConditions.jl:103-136); the host flattens all
 * three into `value[0..n)`, indexed by the reference's 1-based boundary index
 * minus one.  Required lengths per side (left/right, bottom/top):
 *   U: Ny, Nx+1      V: Ny+1, Nx      cell-centred fields: Ny, Nx            */
typedef struct efsi_bc_side {
    int32_t        type;      /* EFSI_BC_*                                              */
    int32_t        n;         /* entries in value / neumann / mask                      */
    const double*  value;     /* Dirichlet or Neumann datum; MIXED Dirichlet datum;
                                 ADVECTIVE_OUTFLOW backflow datum                       */
    const double*  neumann;   /* MIXED only: Neumann datum                              */
    const uint8_t* mask;      /* MIXED only: 1 where the point is Dirichlet             */
} efsi_bc_side;

typedef struct efsi_bc_setup {
    efsi_bc_side left, right, bottom, top;
} efsi_bc_setup;

/* MeshMetrics (MeshGeneration.jl:41-73).  The device step requires uniform
 * spacing in each direction (every configuration of the benchmark suite is
 * uniform); stretched metrics are rejected with EFSI_UNSUPPORTED. */
typedef struct efsi_mesh {
    int32_t Nx, Ny;
    double  Lx, Ly;
    int32_t periodic_x, periodic_y;
    const double *dx_f, *dx_c, *dy_f, *dy_c;                 /* Nx+1, Nx, Ny+1, Ny */
    const double *wL_c2fx, *wR_c2fx, *wB_c2fy, *wT_c2fy;     /* Nx+1, Nx+1, Ny+1, Ny+1 */
    const double *wL_f2cx, *wR_f2cx, *wB_f2cy, *wT_f2cy;     /* Nx, Nx, Ny, Ny */
    const double *dx_west_corner, *dx_east_corner;           /* Nx+1 */
    const double *dy_south_corner, *dy_north_corner;         /* Ny+1 */
} efsi_mesh;

/* ---- model selections (FSIModels, TimeIntegrationIMEX.jl:156-208) -------- */
#define EFSI_GROWTH_NONE            0   /* NoGrowth                          GrowthModels.jl:51   */
#define EFSI_GROWTH_CONSTANT        1   /* ConstantIntrinsicGrowth(rate)     GrowthModels.jl:67   */
#define EFSI_GROWTH_SATURATING      2   /* SaturatingResourceGrowth(rate,K)  GrowthModels.jl:90   */

#define EFSI_GTENSOR_ISOTROPIC      0   /* IsotropicGrowthTensor             GrowthModels.jl:126  */
#define EFSI_GTENSOR_DIRECTIONAL    1   /* DirectionalGrowthTensor(tx,ty)    GrowthModels.jl:150  */

#define EFSI_VISC_NONE              0   /* NoViscosity                 TransportConstitutive.jl:82  */
#define EFSI_VISC_CONSTANT          1   /* ConstantViscosity           TransportConstitutive.jl:89  */
#define EFSI_VISC_HARMONIC          2   /* HarmonicPhaseViscosity      TransportConstitutive.jl:115 */

#define EFSI_DIFF_NONE              0   /* NoDiffusion                 TransportConstitutive.jl:175 */
#define EFSI_DIFF_CONSTANT          1   /* ConstantDiffusivity         TransportConstitutive.jl:178 */
#define EFSI_DIFF_HARMONIC          2   /* HarmonicPhaseDiffusivity    TransportConstitutive.jl:201 */

#define EFSI_CONSUMPTION_NONE       0   /* NoResourceConsumption          TransportConstitutive.jl:250 */
#define EFSI_CONSUMPTION_SATURATING 1   /* SaturatingResourceConsumption  TransportConstitutive.jl:264 */

#define EFSI_RELAX_NONE             0   /* NoRelaxation           StructuralConstitutive.jl:19 */
#define EFSI_RELAX_MAXWELL          1   /* MaxwellRelaxation      StructuralConstitutive.jl:22 */

#define EFSI_ELASTIC_NONE           0   /* NoElasticStress             StructuralConstitutive.jl:38 */
#define EFSI_ELASTIC_LINEAR         1   /* LinearInternalTensorStress  StructuralConstitutive.jl:40 */

#define EFSI_CAP_NONE               0   /* NoCapillarity                                  */
#define EFSI_CAP_DIFFUSE_AREA       1   /* DiffuseAreaCapillarity     Capillarity.jl:21   */

/* phase_field_method; parameters in pf_param[] / pf_option:
 *   UPWIND : NoPhaseFieldRegularization, or LegacySplit(NoInterfaceFlux)    PhaseFieldMethods.jl:33
 *   CDI    : CurrentCDIPhaseField / LegacySplit(ConservativeDiffuseInterfaceFlux)
 *            pf_param = {inverse_peclet, epsilon, delta_normal}             InterfaceRegularization.jl:23
 *   ACDI   : JainACDIPhaseField; pf_param = {gamma, epsilon, psi_floor, delta_normal},
 *            pf_option = dynamic_gamma                                      PhaseFieldMethods.jl:54
 *   UWCDI  : PirozzoliUWCDIPhaseField; pf_param = {alpha, delta_normal},
 *            pf_option = EFSI_NORMALS_*                                     PhaseFieldMethods.jl:97 */
#define EFSI_PF_UPWIND              0
#define EFSI_PF_CDI                 1
#define EFSI_PF_ACDI                2
#define EFSI_PF_UWCDI               3
#define EFSI_NORMALS_STANDARD       0
#define EFSI_NORMALS_YOUNGS         1
#define EFSI_NORMALS_SMOOTHED9      2

#define EFSI_FORCE_NONE             0   /* NoBodyForce                                        */
#define EFSI_FORCE_CONSTANT         1   /* ConstantBodyForce(fx,fy)   TransportConstitutive.jl:318 */
#define EFSI_FORCE_KOLMOGOROV       2   /* KolmogorovBodyForce(A,k;phase) TransportConstitutive.jl:340 */

typedef struct efsi_models {
    int32_t growth_source;        double growth_rate, growth_half_saturation;
    int32_t growth_tensor;        double growth_direction_x, growth_direction_y;
    int32_t viscosity;            double viscosity_fluid, viscosity_structure;
    int32_t diffusivity;          double diffusivity_fluid, diffusivity_structure;
    int32_t resource_consumption; double consumption_rate, consumption_half_saturation;
    int32_t tensor_relaxation;    double relaxation_rate;
    int32_t elastic_stress;       double elastic_coefficient;
    int32_t capillarity;          double capillary_coefficient, capillary_delta_normal;
    int32_t capillary_smoothing_passes;
    int32_t phase_field_method;   double pf_param[4];   int32_t pf_option;
    int32_t body_force;           double body_force_param[3];  /* (fx,fy,-) or (A,k,phase) */
} efsi_models;

/* ---- numerics (IMEXNumerics + LinearSolverOptions, TimeIntegrationIMEX.jl:211-301) */
#define EFSI_EXT_NONE               0   /* NoStructureExtension         StructureTensor.jl:63  */
#define EFSI_EXT_IDENTITY_OUTSIDE   1   /* IdentityOutsideStructure     StructureTensor.jl:73  */
#define EFSI_EXT_GEOMETRIC          2   /* GeometricStructureExtension  StructureTensor.jl:106 */

#define EFSI_PRECISION_FP64         0   /* plain FP64 step                                        */
#define EFSI_PRECISION_MIXED        1   /* FP32 stencil bulk and multigrid, FP64 state, residuals,
                                           inner products, refinement and mass sums               */

/* LinearSolverOptions.velocity_method / resource_method (TimeIntegrationIMEX.jl:211-233).
 * Every implicit system is SPD after symmetric Dirichlet elimination and is solved by
 * preconditioned CG on the device:
 *   DIRECT  the stand-in for `A \ b`: relative residual 1e-13 (against the initial
 *           residual), at most EFSI_LINEAR_HARD_CAP iterations;
 *   GMRES   `reltol` and `maxiter` of the options.
 * After either, the relative residual |A x - b| / max(|b|, eps) decides as in
 * _solve_linear_system! (:602-641): non-finite or above fallback_reltol falls back
 * to the DIRECT iteration (up to EFSI_LINEAR_HARD_CAP more iterations) when
 * direct_fallback is set, and otherwise fails the step with EFSI_SOLVE. */
#define EFSI_LINEAR_DIRECT          0
#define EFSI_LINEAR_GMRES           1
#define EFSI_LINEAR_HARD_CAP        10000
/* Projection solver: AUTO takes the direct fast-diagonalisation solve when the grid
 * allows it (power-of-two sizes, one boundary kind per side of the correction potential)
 * and the multigrid-preconditioned CG otherwise; MULTIGRID always takes the CG.  Both
 * stop on the same relative residual (projection_reltol). */
#define EFSI_PROJECTION_AUTO      0
#define EFSI_PROJECTION_MULTIGRID 1

typedef struct efsi_numerics {
    int32_t structure_extension;  double extension_rate, extension_exponent, extension_cutoff;
    double  projection_reltol;    int32_t projection_maxiter;
    double  stage1_constraint_atol, stage1_constraint_rtol;
    int32_t check_stage1_constraint;
    double  linear_reltol;        int32_t linear_maxiter;    /* options.reltol, options.maxiter */
    int32_t precision;            /* EFSI_PRECISION_*                                          */
    int32_t velocity_method;      /* EFSI_LINEAR_*                                             */
    int32_t resource_method;      /* EFSI_LINEAR_*                                             */
    int32_t direct_fallback;      /* options.direct_fallback                                   */
    double  fallback_reltol;      /* options.fallback_reltol                                   */
    int32_t projection_solver;    /* EFSI_PROJECTION_* (an extension of this library)          */
    int32_t reserved[3];
} efsi_numerics;

typedef struct efsi_config {
    int32_t       abi_version;    /* EFSI_ABI_VERSION */
    efsi_mesh     mesh;
    efsi_bc_setup bc_U, bc_V, bc_correction, bc_phi, bc_resource;
    efsi_bc_setup bc_sigma_xx, bc_sigma_yy, bc_sigma_xy;
    efsi_models   models;
    efsi_numerics numerics;
} efsi_config;

/* StepReport (TimeIntegrationIMEX.jl:318-327). */
typedef struct efsi_step_report {
    double  maximum_projection_constraint_linf;
    double  maximum_growth_trace_error;
    double  minimum_phi;
    double  maximum_phi;
    double  minimum_resource;
    double  minimum_sigma_eigenvalue;
    double  maximum_abs_sigma_determinant_error;
    int64_t non_spd_cells;
} efsi_step_report;

/* ProjectionResult (Projection.jl:31-37) without the correction matrix, which is
 * read with efsi_get_correction(). */
typedef struct efsi_projection_result {
    double linear_relative_residual;
    double constraint_linf;
    double constraint_l2;
    double compatibility_defect;
} efsi_projection_result;

/* Kernel launch sites that efsi_set_timed_site() can bracket with CUDA events. */
#define EFSI_SITE_NONE          (-1)
#define EFSI_SITE_PHASE           0   /* phase-field right-hand side                     */
#define EFSI_SITE_MOMENTUM        1   /* explicit momentum forcing                       */
#define EFSI_SITE_STRUCTURE       2   /* structure-tensor right-hand side                */
#define EFSI_SITE_VISC_APPLY      3   /* viscous operator history I_uv                   */
#define EFSI_SITE_VISC_CG         4   /* viscous CG: one single-reduction iteration      */
#define EFSI_SITE_VISC_INIT       5   /* viscous CG: start vector, residual, A M r0      */
#define EFSI_SITE_PCG_MATVEC      6   /* projection CG: p update + K p + p.Kp            */
#define EFSI_SITE_PCG_UPDATE      7   /* projection CG: x, r update + |r|^2 (no MG levels) */
#define EFSI_SITE_VCYCLE          8   /* CG update fused with one multigrid V-cycle       */
#define EFSI_SITE_PROJ_RHS        9   /* predictor injection + Poisson right-hand side   */
#define EFSI_SITE_PROJ_FINISH    10   /* correction, velocity update, diagnostics        */
#define EFSI_SITE_COMBINE        11   /* stage combination of phi, sigma, c              */
#define EFSI_SITE_VEL_RHS        12   /* viscous predictor right-hand side               */
#define EFSI_SITE_FINALIZE       13   /* state commit + StepReport reductions            */
#define EFSI_SITE_SPECTRAL       14   /* projection direct solve: one refinement pass     */
#define EFSI_SITE_COUNT          15

/* Solver statistics and device timings of the most recent call. */
typedef struct efsi_stats {
    int32_t projection_iterations[4];   /* per stage; [0] = make_velocity_compatible      */
    int32_t velocity_iterations[4];     /* per stage (stages 2..4)                        */
    int32_t resource_iterations[4];
    int64_t kernel_launches;            /* kernels enqueued by the last call              */
    double  device_ms;                  /* CUDA-event time of the last call on the handle's
                                           stream (host<->device copies included)        */
    int64_t site_launches;              /* timed-site launches since efsi_set_timed_site  */
    double  site_ms;                    /* their summed CUDA-event duration               */
    double  site_bytes;                 /* their summed algorithmic bytes (unique reads +
                                           writes once, FP64)                            */
    double  step_bytes;                 /* summed algorithmic bytes of every site launch of
                                           host-driven steps since efsi_set_timed_site    */
} efsi_stats;

/* Driver diagnostics of the cavity benchmarks (run_sugiyama_lid_driven_cavity.jl),
 * computed on the device-resident state so that a time loop needs no state
 * download per step. */
#define EFSI_DIAG_MAX_MODES 8
typedef struct efsi_diag_config {
    double  density;                 /* flow_diagnostics kinetic-energy density        */
    double  elastic_modulus;         /* tensor_cell_diagnostics_2d                      */
    double  sigma_core_cutoff;       /* tensor regions: core phi >= core,               */
    double  sigma_interface_cutoff;  /*   interface in (interface, core),               */
    double  sigma_safety_cutoff;     /*   tail in (safety, interface]                   */
    double  h_interface;             /* effective_interface_cells = width / h_interface */
    int32_t nmax;                    /* boundary Fourier modes, 0..EFSI_DIAG_MAX_MODES  */
    int32_t reserved[3];
} efsi_diag_config;

/* tensor_region_diagnostics (:739-804); NaN fields when the region is empty. */
typedef struct efsi_tensor_region {
    int64_t cells;
    double  area, determinant_min, determinant_max, max_abs_determinant_error,
            mean_abs_determinant_error, lambda_min, lambda_max;
    int64_t non_spd_cells;
    double  max_effective_stress, mean_effective_stress;
} efsi_tensor_region;

typedef struct efsi_diagnostics {
    /* phase_centroid + phase_geometry_diagnostics (:488-507, :615-707); cell
     * centres at ((i+1/2) Lx/Nx, (j+1/2) Ly/Ny) */
    double x_centroid, y_centroid, phase_integral, perimeter_proxy, mixed_layer_measure,
           effective_interface_width, effective_interface_cells, covariance_major,
           covariance_minor, aspect_ratio, orientation_radians, R0;
    double Rc[EFSI_DIAG_MAX_MODES], Rs[EFSI_DIAG_MAX_MODES], amplitudes[EFSI_DIAG_MAX_MODES];
    /* phase_bound_diagnostics (:709-722) */
    double  phi_minimum, phi_maximum, lower_violation, upper_violation;
    int64_t out_of_bounds_cells;
    /* flow_diagnostics (:724-749) */
    double maximum_speed, kinetic_energy, divergence_linf, divergence_l2;
    /* inputs of comparison_timestep_bounds (:852-934): max |U|, max |V| over all faces */
    double max_abs_U, max_abs_V;
    /* tensor_diagnostics_detailed (:806-828): global, core, interface, tail */
    efsi_tensor_region tensor[4];
} efsi_diagnostics;

typedef struct efsi_handle efsi_handle;

/* build_imex_context + allocate_imex_workspace (TimeIntegrationIMEX.jl:468-493,
 * :389-441): validates the configuration (periodicity agreement, :447-466;
 * supported viscous boundaries, Operators.jl:89-105), uploads boundary data and
 * allocates every device buffer on the current CUDA device.  On failure *out is
 * NULL and efsi_last_error(NULL) describes the cause. */
EFSI_API int  efsi_create(const efsi_config* config, efsi_handle** out);
EFSI_API void efsi_destroy(efsi_handle* handle);
/* Message of the last failing call on `handle` (NULL: last failing efsi_create
 * on this thread). */
EFSI_API const char* efsi_last_error(const efsi_handle* handle);

/* Copy a full FSIState (TimeIntegrationIMEX.jl:103-118) to / from the device. */
EFSI_API int efsi_upload_state(efsi_handle* h, const double* U, const double* V, const double* phi,
                      const double* resource, const double* sigma_xx,
                      const double* sigma_yy, const double* sigma_xy);
EFSI_API int efsi_download_state(efsi_handle* h, double* U, double* V, double* phi, double* resource,
                        double* sigma_xx, double* sigma_yy, double* sigma_xy);

/* IMEXWorkspace.correction, the projection warm start (TimeIntegrationIMEX.jl:386). */
EFSI_API int efsi_set_correction(efsi_handle* h, const double* q);
EFSI_API int efsi_get_correction(efsi_handle* h, double* q);

/* make_velocity_compatible! (TimeIntegrationIMEX.jl:1088-1109) on the device state. */
EFSI_API int efsi_make_velocity_compatible(efsi_handle* h, efsi_projection_result* result);

/* integrate_step! (TimeIntegrationIMEX.jl:1152-1256) on the device-resident state. */
EFSI_API int efsi_integrate_step(efsi_handle* h, double t, double dt, efsi_step_report* report);

/* integrate_step! as the drop-in sees it: the host FSIState arrays and the
 * workspace correction (the projection warm start) are uploaded, advanced in place
 * and downloaded (TimeIntegrationIMEX.jl:1152-1256, with the state copies of :1169
 * and :1232-1238 crossing the host/device boundary).  `correction` may be NULL to
 * keep the device-resident warm start. */
EFSI_API int efsi_integrate_step_host(efsi_handle* h, double* U, double* V, double* phi,
                             double* resource, double* sigma_xx, double* sigma_yy,
                             double* sigma_xy, double* correction, double t, double dt,
                             efsi_step_report* report);

/* n consecutive integrate_step! calls on the device-resident state with host
 * sync only at the end; t advances by dts[k].  reports may be NULL or hold n
 * entries.  On an error the state holds the last completed step and the
 * return value says which step failed (efsi_last_error). */
EFSI_API int efsi_step_n(efsi_handle* h, double t0, const double* dts, int32_t n,
                efsi_step_report* reports);

/* Projection.project! (Projection.jl:170-307) of host velocity arrays onto
 * div(v) = target, using the context's correction boundaries and warm start. */
EFSI_API int efsi_project(efsi_handle* h, double* U, double* V, const double* target,
                 efsi_projection_result* result);

/* phase_field_rhs for the context's phase-field method (PhaseFieldMethods.jl:408-475,
 * :652-671, :852-867) with target divergence G. */
EFSI_API int efsi_phase_field_rhs(efsi_handle* h, const double* U, const double* V, const double* phi,
                         const double* G, double* rhs);

/* uwcdi_strang_step (PhaseFieldMethods.jl:810-850): dimensionally split UWCDI
 * transport of phi over dt (half sweep, full sweep in the other direction, half
 * sweep; x first when x_first != 0) for a context whose method is UWCDI. */
EFSI_API int efsi_uwcdi_strang_step(efsi_handle* h, const double* U, const double* V, const double* phi,
                           double dt, int32_t x_first, double* out);

/* structure_tensor_rhs (StructureTensor.jl:377-463) with K_g built from G by the
 * context's growth-tensor model and the context's relaxation/extension. */
EFSI_API int efsi_structure_tensor_rhs(efsi_handle* h, const double* sigma_xx, const double* sigma_yy,
                              const double* sigma_xy, const double* U, const double* V,
                              const double* phi, const double* G,
                              double* rhs_xx, double* rhs_yy, double* rhs_xy);

/* Explicit momentum forcing of one stage (TimeIntegrationIMEX.jl:959-985):
 * -material_convection + body force + capillary force + div(phi tau_e)
 * + growth-viscous force, on the full MAC faces. */
EFSI_API int efsi_momentum_explicit_rhs(efsi_handle* h, double t, const double* U, const double* V,
                               const double* phi, const double* sigma_xx,
                               const double* sigma_yy, const double* sigma_xy,
                               const double* G, double* Fx, double* Fy);

/* apply_operator(build_viscous_operator(...), uv) (Operators.jl:929-1083, :1115)
 * on the compact velocity vector uv = [U(1:Nx,:); V(:,1:Ny)] with viscosity
 * evaluated from phi. */
EFSI_API int efsi_apply_viscous_operator(efsi_handle* h, const double* phi, const double* uv,
                                double* out);

EFSI_API int efsi_get_stats(const efsi_handle* h, efsi_stats* stats);

/* The diagnostics above for the device-resident state (the state after the last
 * efsi_integrate_step / efsi_step_n / efsi_upload_state).  Driver-side reductions of
 * run_sugiyama_lid_driven_cavity.jl:488-828; the phase gradient of the perimeter
 * proxy uses the context's phi boundaries (phase_center_gradient, :600-613). */
EFSI_API int efsi_state_diagnostics(efsi_handle* h, const efsi_diag_config* config, efsi_diagnostics* out);

/* Bracket every launch of one EFSI_SITE_* with CUDA events on the handle's stream
 * (EFSI_SITE_NONE switches timing off) and reset the site accumulators of
 * efsi_stats.  Tracing aid of the benchmark; no reference counterpart. */
EFSI_API int efsi_set_timed_site(efsi_handle* h, int32_t site);

/* ---- differentiation form ------------------------------------------------------
 * A discrete adjoint of integrate_step! (TimeIntegrationIMEX.jl:1152-1256) for the
 * ChainRulesCore.rrule of a run of steps; the reference has no adjoint, so these
 * entry points have no counterpart there.  The adjoint differentiates the ACDI
 * phase field (fixed mobility), constant or no viscosity, linear elastic stress,
 * Maxwell relaxation, every structure extension and body force, on every boundary
 * kind the step accepts; growth, resource transport and capillarity return
 * EFSI_UNSUPPORTED.  Parameters: the elastic coefficient G and the tangential wall
 * velocity data (a moving lid is U top).  Explicit stencils are transposed exactly
 * (upwind and clamp switches are held at the forward branch); the projection and
 * viscous solves are transposed as exact inverses, solved to a relative residual of
 * 1e-13. */
typedef struct efsi_gradient {
    double  elastic_coefficient;  /* dJ/dG of LinearInternalTensorStress(G)                */
    double *U_bottom, *U_top;     /* dJ/d(U wall data), Nx+1 entries each; may be NULL      */
    double *V_left, *V_right;     /* dJ/d(V wall data), Ny+1 entries each; may be NULL      */
} efsi_gradient;

/* efsi_step_n that also keeps the state (and the projection warm start) every `every`
 * steps in device memory (every <= 0: ceil(sqrt(n)), at most 1024), for a following
 * efsi_backward.  The device state advances exactly as with efsi_step_n. */
EFSI_API int efsi_forward_checkpointed(efsi_handle* h, double t0, const double* dts, int32_t n, int32_t every,
                                       efsi_step_report* reports);
/* Reverse sweep over the steps of the last efsi_forward_checkpointed call: given
 * lam = dJ/d(final state) (host arrays; NULL = zero), returns dJ/d(initial state) in
 * grad_* (NULL = not wanted) and the parameter derivatives in *grad (may be NULL).
 * Each segment between checkpoints is recomputed forward once with its stage fields
 * recorded, then swept backwards; the device state is left at the final state. */
EFSI_API int efsi_backward(efsi_handle* h, const double* lam_U, const double* lam_V, const double* lam_phi,
                           const double* lam_sxx, const double* lam_syy, const double* lam_sxy, double* grad_U,
                           double* grad_V, double* grad_phi, double* grad_sxx, double* grad_syy,
                           double* grad_sxy, efsi_gradient* grad);
/* Transposed Jacobian of one stage's explicit tendencies (TimeIntegrationIMEX.jl:944-1071)
 * at the stage fields (U, V full MAC; cell fields): given the adjoints of E_uv and I_uv
 * (compact rows U(0:Nx-1,:), V(:,0:Ny-1), N each), of E_phi and of E_sigma (NULL = zero),
 * writes the adjoints of the six stage fields and of the parameters.  Exposed for
 * dot-product tests of the transposed stencils. */
EFSI_API int efsi_tendencies_adjoint(efsi_handle* h, const double* U, const double* V, const double* phi,
                                     const double* sxx, const double* syy, const double* sxy,
                                     const double* lam_Eu, const double* lam_Ev, const double* lam_Iu,
                                     const double* lam_Iv, const double* lam_Ephi, const double* lam_Exx,
                                     const double* lam_Eyy, const double* lam_Exy, double* out_U, double* out_V,
                                     double* out_phi, double* out_sxx, double* out_syy, double* out_sxy,
                                     efsi_gradient* grad);
/* Transposed efsi_project (Projection.jl:170-307) with respect to its input velocity:
 * lam of the input faces from lam of the projected faces (full MAC arrays). */
EFSI_API int efsi_project_adjoint(efsi_handle* h, const double* lam_U, const double* lam_V, double* lam_U_in,
                                  double* lam_V_in);

/* How efsi_integrate_step / efsi_integrate_step_host / efsi_step_n run a step:
 *   EFSI_STEP_GRAPH  (default) the whole step is one captured CUDA graph whose
 *                    solver loops are device-terminated conditional nodes;
 *   EFSI_STEP_HOST   every kernel is an ordinary launch from the host, the solver
 *                    loops enqueued in batches (for profilers that list launches).
 * Both run the same kernels and give bit-identical states.  No reference
 * counterpart (the reference has no device). */
#define EFSI_STEP_GRAPH 0
#define EFSI_STEP_HOST  1
EFSI_API int efsi_set_step_mode(efsi_handle* h, int32_t mode);

/* Allocation-free check of a MAC velocity against a divergence target: writes
 * out[0] = max |div(U,V) - G| and out[1] = max |G| over the Nx x Ny cells of a
 * uniform grid on [0,Lx] x [0,Ly] (G may be NULL for a zero target; the same
 * quantity as the step's stage-1 check and ProjectionResult.constraint_linf).
 * No counterpart in the reference: it exists for callers that cannot let a library
 * allocate device memory, such as hosts that hand out all GPU memory from their own
 * pool allocator, or loops that cannot absorb the device-wide synchronisation that
 * cudaMalloc/cudaFree may cause.  It needs no handle, calls no allocator, and works
 * directly on the caller's device arrays (U (Nx+1) x Ny, V Nx x (Ny+1), G and out
 * on the current device).
 *  - A cell whose residual (or |G|) is not finite (NaN or Inf anywhere in its
 *    stencil) makes out[0] (or out[1]) +Inf, so a corrupt field never passes.
 *  - Asynchronous: the kernel runs on `stream` (a cudaStream_t; NULL is the legacy
 *    default stream); out is valid once that stream has been synchronised.
 *  - Scratch: a fixed 256 KiB static device array inside the library holds the
 *    reduction partials, so the grid may hold at most 16384 blocks of 32 x 8 cells
 *    (4,194,304 cells, e.g. 2048 x 2048); larger grids return EFSI_ARG.
 *  - All calls on one device share that array: calls that may overlap on the GPU
 *    (on different streams, or from different host threads) race and give wrong
 *    results.  Serialise them.
 *  - The first call on each device looks up the array's device address; make that
 *    first call before beginning any stream capture.
 * Errors return EFSI_ARG / EFSI_CUDA with the message in efsi_last_error(NULL)
 * (per host thread). */
EFSI_API int efsi_divergence_residual_noalloc(int32_t Nx, int32_t Ny, double Lx, double Ly,
                                              const double* U, const double* V, const double* G,
                                              double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EFSI_H */
