/*
 * gale_gpu.h -- C ABI of the B200 (sm_100a) particle-in-cell Q1-P0 Stokes path.
 *
 * One opaque handle owns one regular Cartesian Q1 velocity / P0 pressure mesh, its
 * material-point swarm and every device buffer.  The host passes plain pointers that
 * are valid for the duration of the call only; the library copies in and out.  Every
 * entry point returns an int status (GG_OK == 0, negative on error) and never aborts;
 * gg_last_error() gives the message.  The reference reports the same failures through
 * Journal_Firewall (abort); the host plugin maps a non-zero status back onto it.
 *
 * Conventions shared with the reference (StgFEM / StgDomain / PICellerator):
 *   - element index  e = i + nx*(j + ny*k)            (Grid_Project, StgDomain/Mesh/src/Grid.cxx:254-272)
 *   - node index     n = i + (nx+1)*(j + (ny+1)*k)
 *   - element-local node a has offsets (a&1, (a>>1)&1, (a>>2)&1)
 *                                          (BilinearElementType.cxx:216-245, TrilinearElementType.cxx:257-300)
 *   - nodal vectors are node-major, dim components per node (FeVariable dof layout)
 *   - y (J_AXIS) is the vertical axis; gravity and thermal buoyancy act along it.
 *
 * Not re-entrant per handle.  One CUDA stream per handle.
 */
#ifndef GALE_GPU_H
#define GALE_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define GG_API __attribute__((visibility("default")))
#else
#define GG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------ */
enum {
    GG_OK                 = 0,
    GG_ERR_INVALID        = -1,  /* bad argument or size                              */
    GG_ERR_CUDA           = -2,  /* CUDA runtime error (message in gg_last_error)     */
    GG_ERR_NONFINITE      = -3,  /* NaN/Inf in a solver scalar (isGoodNumber firewall) */
    GG_ERR_NOT_CONVERGED  = -4,  /* iteration cap reached                             */
    GG_ERR_STAGNATED      = -5,  /* learned preconditioner stagnated and no fallback  */
    GG_ERR_OUT_OF_DOMAIN  = -6,  /* a material point lies outside the mesh            */
    GG_ERR_ZERO_FORCE     = -7,  /* momentum force vector is zero                     */
    GG_ERR_STATE          = -8,  /* entry point called before its inputs were set     */
    GG_ERR_NO_DEVICE      = -9,  /* no CUDA device                                    */
    GG_ERR_EMPTY_CELL     = -10  /* an element holds no material point                */
};

/* ---- mesh ---------------------------------------------------------------------- */
typedef struct gg_mesh_desc {
    int32_t dim;          /* 2 or 3                                  */
    int32_t elements[3];  /* elementResI/J/K                         */
    double  min[3];       /* minX/minY/minZ                          */
    double  max[3];       /* maxX/maxY/maxZ                          */
} gg_mesh_desc;

/* ---- velocity boundary conditions (WallVC) -------------------------------------
 * wall order: 0 left (min x), 1 right (max x), 2 bottom (min y), 3 top (max y),
 *             4 back (min z), 5 front (max z).  A node on several walls takes the
 *             value of the last wall in this order that fixes the component.     */
typedef struct gg_velocity_bc {
    uint8_t fixed[6][3];
    double  value[6][3];
} gg_velocity_bc;

/* ---- rheology (Underworld/Rheology) -------------------------------------------- */
enum {
    GG_RHEO_MATERIAL_VISCOSITY = 1, /* MaterialViscosity.cxx:129-149                  */
    GG_RHEO_ARRHENIUS          = 2, /* Arrhenius.cxx:170-220                          */
    GG_RHEO_FRANK_KAMENETSKII  = 3, /* FrankKamenetskii.cxx:143-161                   */
    GG_RHEO_VON_MISES          = 4, /* VonMises.cxx:183-289                           */
    GG_RHEO_DRUCKER_PRAGER     = 5, /* DruckerPrager.cxx:296-490                      */
    GG_RHEO_BYERLEE            = 6  /* Byerlee.cxx:163-187                            */
};

#define GG_MAX_RHEOLOGIES 4
#define GG_MAX_MATERIALS  16

typedef struct gg_rheology {
    int32_t kind;                       /* GG_RHEO_*                                  */
    int32_t strain_weakening;           /* 1: uses the material's StrainWeakening     */
    /* creep laws */
    double eta0;
    double activation_energy;           /* Arrhenius                                  */
    double activation_volume;           /* Arrhenius                                  */
    double reference_temp;              /* Arrhenius                                  */
    double theta;                       /* FrankKamenetskii                           */
    /* yield laws */
    double cohesion;
    double cohesion_after_softening;
    double friction_coefficient;        /* DruckerPrager                              */
    double friction_coefficient_after_softening;
    double minimum_yield_stress;        /* DruckerPrager                              */
    double minimum_viscosity;           /* YieldRheology minimumViscosity             */
    double max_strain_rate;             /* DruckerPrager                              */
    double depth_coefficient;           /* Byerlee                                    */
    int32_t strain_rate_softening;      /* VonMises                                   */
    int32_t pad;
    /* DruckerPrager boundary strength (DruckerPrager.cxx:225-247, 326-361, 448-490):
     * an element in the first or last element layer along a wall whose bit is set in
     * boundary_walls (bit w = wall w of the order above: left, right, bottom, top, back,
     * front) uses these four in place of cohesion / friction_coefficient               */
    double boundary_cohesion;
    double boundary_cohesion_after_softening;
    double boundary_friction_coefficient;
    double boundary_friction_coefficient_after_softening;
    int32_t boundary_walls;
    /* nonzero: the deck attaches a HydrostaticTerm (DruckerPrager.cxx:327-332), which this
     * library does not evaluate; gg_set_materials refuses it with GG_ERR_INVALID        */
    int32_t hydrostatic_term;
} gg_rheology;

typedef struct gg_strain_weakening {    /* StrainWeakening.cxx:250-275                */
    double initial_softening_strain;
    double final_softening_strain;
    double healing_rate;
} gg_strain_weakening;

typedef struct gg_material {
    int32_t n_rheologies;               /* run in order (Rheology_Register.cxx:70-86) */
    int32_t has_strain_weakening;
    gg_rheology rheology[GG_MAX_RHEOLOGIES];
    gg_strain_weakening strain_weakening;
    double density;                     /* BuoyancyForceTerm density                  */
    double alpha;                       /* BuoyancyForceTerm thermal expansivity      */
} gg_material;

/* ---- body force ------------------------------------------------------------------ */
typedef struct gg_body_force {
    double gravity;        /* BuoyancyForceTerm: f += gravity*gHat*rho*N*w*detJ      */
    double g_hat[3];       /* unit direction (normalised by the library)            */
    double rayleigh;       /* ThermalBuoyancyForceTerm: f_y += Ra*T*N*w*detJ (0=off)  */
} gg_body_force;

/* ---- solver configuration ------------------------------------------------------ */
enum {
    GG_PRECISION_FP64  = 0,  /* every operator and vector in FP64                      */
    GG_PRECISION_MIXED = 1   /* FP32 viscosity, moments and inner K applies inside FP64
                                iterative refinement; FP64 Uzawa update, Schur residual,
                                dots and r = b - A x                                     */
};
enum {
    GG_INNER_JACOBI_CG  = 0, /* PETSc -ksp_type cg -pc_type jacobi                     */
    GG_INNER_MG_CG      = 1, /* geometric multigrid V-cycle preconditioned CG          */
    GG_INNER_LEARNED_CG = 2, /* MG + learned coarse correction, flexible CG; falls back
                                to GG_INNER_MG_CG when the residual stagnates          */
    GG_INNER_LEARNED_JACOBI_CG = 3 /* Jacobi + learned coarse correction, flexible CG;
                                the plain Jacobi flexible CG judges and backs it up    */
};

typedef struct gg_uzawa_params {
    double  tolerance;            /* Stokes_SLE_UzawaSolver "tolerance" (1e-5)          */
    int32_t max_iterations;       /* "maxIterations" (1000)                             */
    int32_t min_iterations;       /* "minIterations" (1)                                */
    int32_t use_absolute_tolerance;
    int32_t use_preconditioner;   /* Ĝ = Gᵀ diag(K_e)⁻¹ G pressure preconditioner       */
    int32_t inner;                /* GG_INNER_*                                         */
    int32_t precision;            /* GG_PRECISION_*                                     */
    double  inner_rtol_factor;    /* inner rtol = factor*tolerance (0.1)                */
    int32_t inner_max_iterations; /* per inner solve (PETSc default 10000)              */
    int32_t reuse_pressure;       /* start from the p passed in (Picard, restart)       */
    int32_t recycle_directions;   /* GG_PRECISION_MIXED only: start the inner solve of
                                     K u* = G s from β u*_prev (s = z + β s_prev); the
                                     inner stopping rule stays relative to ‖G s‖        */
    int32_t smoothing_degree;     /* multigrid: Chebyshev degree of the pre- and post-
                                     smoothing on the fine level, 2..4 (0: 2); coarser
                                     levels use min(degree, 2); the role of
                                     PETScMGSolver's downIterations/upIterations
                                     (PETScMGSolver.cxx:182-183)                         */
} gg_uzawa_params;

typedef struct gg_uzawa_stats {
    int32_t outer_iterations;
    int32_t inner_iterations;     /* total inner Krylov iterations (all solves)         */
    int32_t inner_solves;
    int32_t fallbacks;            /* learned → MG fallbacks taken                       */
    double  rel_residual;         /* final Uzawa relResidual                            */
    double  abs_residual;
    double  div_u;                /* |Gᵀu|/|u|                                          */
    double  momentum_residual;    /* |f - K u - G p| / |f|                              */
    double  solve_ms;             /* device time of the solve                           */
    int64_t kernel_launches;      /* launches of this library's kernels in the solve    */
    /* the persistent multigrid flexible-CG launches of the solve (mixed path): count,
     * summed device time (CUDA events on the handle's stream around each launch), FCG
     * iterations, grid barriers per iteration, and the algorithmic bytes of one iteration
     * counting every phase of the V-cycle (vectors, moments, BC masks, coarse inverse)   */
    int32_t fused_launches;
    int32_t fused_iterations;
    double  fused_ms;
    double  fused_bytes_per_iteration;
    int32_t fused_barriers_per_iteration;
    int32_t uzawa_fused;          /* 1: the whole solve ran as one persistent launch (mixed
                                     path, multigrid inner solves): fused_launches is then 1,
                                     fused_ms that launch's device time                   */
} gg_uzawa_stats;

typedef struct gg_picard_params {
    int32_t max_iterations;       /* nonLinearMaxIterations                             */
    int32_t min_iterations;       /* nonLinearMinIterations                             */
    double  tolerance;            /* nonLinearTolerance                                 */
} gg_picard_params;

typedef struct gg_picard_stats {
    int32_t iterations;
    int32_t converged;
    double  residual;             /* ‖u_k − u_{k−1}‖ / ‖u_k‖ at exit                     */
    int32_t outer_iterations;     /* Uzawa iterations over all Picard steps              */
    int32_t inner_iterations;
    double  solve_ms;
} gg_picard_stats;

/* Learned coarse correction (no counterpart in the reference): a 2-layer, 32-channel
 * convolutional network over the nodal grid of one multigrid level, trained on
 * (viscosity, residual, error) pairs the solver generates on the current operator.     */
typedef struct gg_learn_params {
    int32_t level;          /* multigrid level of the network (≤0: level 2 or the coarsest) */
    int32_t n_rhs;          /* right-hand sides used to generate pairs (force + G s_j)     */
    int32_t iters_per_rhs;  /* stationary MG iterates recorded per right-hand side         */
    int32_t epochs;         /* Adam epochs                                                  */
    float   lr;             /* Adam learning rate                                           */
    int32_t seed;
    int32_t base;           /* GG_LEARN_BASE_*: the preconditioner whose leftover error the
                               network learns to correct                                     */
} gg_learn_params;
enum { GG_LEARN_BASE_MULTIGRID = 0, GG_LEARN_BASE_JACOBI = 1 };

typedef struct gg_learn_stats {
    int32_t samples;
    float   loss_first;     /* mean normalised loss of the first / last epoch              */
    float   loss_last;
    double  train_ms;
} gg_learn_stats;

typedef struct gg_handle gg_handle;

/* ---- lifetime -------------------------------------------------------------------
 * Replaces the Stokes_SLE_UzawaSolver object lifetime: _Build
 * (StgFEM/SLE/ProvidedSystems/StokesFlow/src/Stokes_SLE_UzawaSolver.cxx:199-239) and
 * _Destroy (:269-287).                                                               */
GG_API int  gg_create(const gg_mesh_desc* mesh, gg_handle** out);
GG_API int  gg_destroy(gg_handle* h);
GG_API const char* gg_last_error(const gg_handle* h);
GG_API const char* gg_version(void);

/* ---- inputs ---------------------------------------------------------------------- */
/* Velocity BCs: the WallVC/CompositeVC "velocityBCs" of VelocityField (FeVariable_IsBC,
 * StgFEM/Discretisation/src/FeVariable.cxx) as consumed by __StiffnessMatrix_NewAssemble
 * (StgFEM/SLE/SystemSetup/src/StiffnessMatrix.cxx:2091-2143).                          */
GG_API int  gg_set_velocity_bc(gg_handle* h, const gg_velocity_bc* bc);
/* Velocity BCs per node: a VariableCondition whose values come from a condition function
 * evaluated at the nodes by the host (the "func" entries of a WallVC, e.g.
 * StgFEM_StandardConditionFunctions_PartialLid_TopLayer, StgFEM/plugins/
 * StandardConditionFunctions/StandardConditionFunctions.cxx:547-568).  fixed: [nodes],
 * bit c = component c fixed; values: [nodes*dim] node-major, read on fixed components. */
GG_API int  gg_set_velocity_bc_nodes(gg_handle* h, const uint8_t* fixed, const double* values);
/* Material table: RheologyMaterial + its Rheology_Register
 * (Underworld/Rheology/src/Rheology_Register.cxx:70-86), density/alpha of
 * BuoyancyForceTerm (PICellerator/Utils/src/BuoyancyForceTerm.cxx:414-530).           */
GG_API int  gg_set_materials(gg_handle* h, int32_t n_materials, const gg_material* materials);
/* Material points: MaterialPointsSwarm coords (StandardParticle.h:52-80), material
 * index (MaterialPoint.h:48-52) and StrainWeakening postFailureWeakening (nullable).  */
GG_API int  gg_set_points(gg_handle* h, int64_t n_points, const double* coords,
                   const int32_t* material, const double* plastic_strain);
/* Nodal temperature of TemperatureField (nullable: no temperature).                   */
GG_API int  gg_set_temperature(gg_handle* h, const double* nodal_temperature);
GG_API int  gg_set_body_force(gg_handle* h, const gg_body_force* force);

/* ---- point → cell, ξ, weights ------------------------------------------------------
 * Replaces Swarm_UpdateAllParticleOwners (StgDomain/Swarm/src/SwarmClass.cxx:878-992)
 * with Mesh_RegularAlgorithms_SearchElements (StgDomain/Mesh/src/
 * Mesh_RegularAlgorithms.cxx:191-224) as the search, _CoincidentMapper_Map
 * (PICellerator/MaterialPoints/src/CoincidentMapper.cxx:158-240) for ξ and the
 * per-cell tables, and _ConstantWeights_Calculate (PICellerator/Weights/src/
 * ConstantWeights.cxx:178-187).  owning_cell (nullable) receives the element of each
 * point, bit-exact with the reference; points outside the mesh return
 * GG_ERR_OUT_OF_DOMAIN and get cell = element count (ElementCellLayout.cxx:266-275). */
GG_API int  gg_locate(gg_handle* h, uint32_t* owning_cell);

/* No-allocation point location (no counterpart in the reference).  For callers that
 * cannot allocate device memory (a host that owns all memory through its own allocator
 * or a fixed arena, real-time drivers that forbid allocation after start-up): the same
 * bit-exact search, per-element offsets and stable per-element point order as gg_locate,
 * computed on device buffers the caller owns, without a handle and without any
 * allocation.  Inputs/outputs are device pointers: d_coords [n_points*dim], d_cell
 * [n_points] (element count for points outside), d_offsets [elements+1], d_order
 * [n_points] (point indices grouped by element, ascending inside each element; only
 * d_order[0 .. d_offsets[elements]) is written, entries past it keep the caller's
 * contents, one per point outside the mesh).  Limits:
 * at most 1,048,576 elements and 1024 points per element (GG_ERR_INVALID otherwise, with
 * *message set).  The counting-sort scratch is one fixed device array shared by every
 * call on a device: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on each device performs a one-time set-up (the array's device
 * address); make it before any stream capture.  stream: a cudaStream_t (NULL: default).  */
GG_API int  gg_locate_noalloc(const gg_mesh_desc* mesh, int64_t n_points, const double* d_coords,
                              uint32_t* d_cell, int32_t* d_offsets, int32_t* d_order,
                              int64_t* n_outside, void* stream, const char** message);

/* ---- integration weights and population control (A13) ------------------------------
 * GG_WEIGHTS_CONSTANT: the material points are the integration points with
 * w = 2^dim / points-in-element (_ConstantWeights_Calculate, PICellerator/Weights/src/
 * ConstantWeights.cxx:178-187); the default.
 * GG_WEIGHTS_DVC: DVCWeights (PICellerator/Weights/src/DVCWeights.cxx:788-953): each
 * element's [-1,1]^dim is cut into resolution[0]×resolution[1](×resolution[2]) cells, a
 * discrete Voronoi diagram is grown from the element's points, and every integration
 * point moves to the centroid of its region with the region's volume as weight.  gg_locate
 * recomputes them, and every operator build uses them.  Limits: ≤ 1024 grid cells and
 * ≤ 254 points per element (GG_ERR_INVALID otherwise).                                 */
enum { GG_WEIGHTS_CONSTANT = 0, GG_WEIGHTS_DVC = 1 };
typedef struct {
    int32_t mode;
    int32_t resolution[3];   /* DVCWeights resolutionX/Y/Z (reference default 10)          */
} gg_weights;
GG_API int  gg_set_weights(gg_handle* h, const gg_weights* weights);

/* PCDVC population control (PICellerator/Utils/src/PCDVC.cxx:656-1512), run after
 * gg_locate in GG_WEIGHTS_DVC mode: per element, points whose Voronoi volume is above
 * upper_t % of the element are split (the new point, a copy of its parent, sits at the
 * parent region's centroid; at most max_splits per element) and points below lower_t %
 * are deleted (at most max_deletions, decreasing point index first); elements whose
 * points carry more than one material split/delete only when the *_in_interface_cells
 * flags allow it.  Changed elements get a new diagram.  The point set is then rebuilt:
 * the points that survive in their previous order, followed by the new points (element
 * order, then their parents' order), and re-located; gg_point_count / gg_get_points read
 * it back.  The Inflow branch (random re-seeding) is not provided: inflow != 0 returns
 * GG_ERR_INVALID.                                                                         */
typedef struct {
    double  upper_t, lower_t;          /* upperT (25), lowerT (0.6): % of the element volume */
    int32_t max_splits, max_deletions; /* maxSplits (3), maxDeletions (2)                   */
    int32_t split_in_interface_cells;  /* splitInInterfaceCells (0)                         */
    int32_t delete_in_interface_cells; /* deleteInInterfaceCells (0)                        */
    int32_t inflow;                    /* Inflow: must be 0                                 */
} gg_pcdvc_params;
typedef struct {
    int64_t points_before, points_after, splits, deletions;
    double  ms;                        /* device time of the whole call                     */
} gg_pcdvc_stats;
GG_API int  gg_population_control(gg_handle* h, const gg_pcdvc_params* params, gg_pcdvc_stats* stats);
GG_API int  gg_point_count(gg_handle* h, int64_t* n);
/* The current points: coords [n*dim], material [n], plastic strain [n] (each nullable). */
GG_API int  gg_get_points(gg_handle* h, double* coords, int32_t* material, double* plastic_strain);
/* Integration point of every material point (point order): local coordinates xi [n*dim]
 * and weight [n] as the operator build uses them.                                        */
GG_API int  gg_get_integration_points(gg_handle* h, double* xi, double* weight);

/* ---- operator build ---------------------------------------------------------------
 * Replaces the assembleStiffnessMatrix entry point (__StiffnessMatrix_NewAssemble,
 * StiffnessMatrix.cxx:2016-2200) for k_matrix, g_matrix and the Uzawa preconditioner,
 * i.e. _ConstitutiveMatrixCartesian_AssembleElement (Underworld/Rheology/src/
 * ConstitutiveMatrixCartesian.cxx:206-487), _GradientStiffnessMatrixTerm_AssembleElement
 * (StgFEM/Assembly/src/GradientStiffnessMatrixTerm.cxx:161-251) and
 * _UzawaPreconditionerTerm_AssembleElement (StgFEM/SLE/ProvidedSystems/StokesFlow/src/
 * UzawaPreconditionerTerm.cxx:156-239), plus the force vector terms.  Per point runs
 * the rheology chain; per element stores the viscosity moments of the PIC quadrature.
 * previous_solution_exists gates yielding (YieldRheology.cxx:203-204); u and p
 * (nodal velocity, element pressure, nullable when it is 0) are the previous solution
 * the yield laws read.                                                                */
GG_API int  gg_build_operator(gg_handle* h, int32_t precision, int32_t previous_solution_exists,
                       const double* u, const double* p);

/* ---- solve ---------------------------------------------------------------------------
 * Replaces _Stokes_SLE_UzawaSolver_Solve (Stokes_SLE_UzawaSolver.cxx:393-938) with its
 * inner velocity KSP.  u: nodal velocity [nodes*dim] (out; BC dofs carry their values),
 * p: element pressure [elements] (in when reuse_pressure, out).                        */
GG_API int  gg_uzawa_solve(gg_handle* h, const gg_uzawa_params* params, double* u, double* p,
                    gg_uzawa_stats* stats);

/* Replaces SystemLinearEquations_NonLinearExecute (StgFEM/SLE/SystemSetup/src/
 * SystemLinearEquations.cxx:735-920) for the Stokes SLE: operator build + Uzawa per
 * iteration, yielding enabled from the second solve.                                   */
GG_API int  gg_picard(gg_handle* h, const gg_picard_params* picard, const gg_uzawa_params* uzawa,
               double* u, double* p, gg_picard_stats* stats);

/* Batch of independent problems (uneven sizes): for every handle (inputs already set)
 * locate → build → Uzawa, pulled from a shared work queue by `workers` host threads; each
 * handle runs on its own stream so the problems overlap on the GPU.  Gale runs one SLE
 * per job; the batch form has no single reference counterpart (it replaces running
 * _Stokes_SLE_UzawaSolver_Solve once per job).  status[i] gets each problem's status;
 * the return value is the first non-zero status.                                        */
GG_API int  gg_solve_batch(int32_t n, gg_handle* const* handles, const gg_uzawa_params* params,
                           int32_t workers, double* const* u_out, double* const* p_out,
                           gg_uzawa_stats* stats, int32_t* status);

/* ---- advection ---------------------------------------------------------------------
 * Replaces TimeIntegrand_SecondOrder / first order (StgDomain/Utils/src/
 * TimeIntegrand.cxx:265-335, :457-483) with _SwarmAdvector_TimeDeriv
 * (PICellerator/MaterialPoints/src/SwarmAdvector.cxx:261-287) as the derivative, on the
 * handle's points and the velocity of the last solve (or u when non-null).  Points keep
 * their order.  coords_out (nullable) receives the advected coordinates.              */
GG_API int  gg_advect(gg_handle* h, double dt, int32_t order, const double* u, double* coords_out);
/* Stokes_SLE_UpdateDt (StgFEM/SLE/ProvidedSystems/StokesFlow/src/UpdateDt.cxx:53-84):
 * dt = 0.5 * min element separation / max |v| over velocity nodes.                    */
GG_API int  gg_courant_dt(gg_handle* h, const double* u, double* dt);

/* ---- diagnostics and operator access (parity tests, host shims) ---------------------- */
/* Per-point viscosity η of the last operator build, in input point order.             */
GG_API int  gg_get_point_viscosity(gg_handle* h, double* eta);
/* Per-point StrainWeakening increment and yield flag of the last build (nullable).    */
GG_API int  gg_get_point_yield(gg_handle* h, double* increment, uint8_t* yielded);
/* Element moments M_m(e) = Σ_p w_p detJ η_p m(ξ_p) in FP64, [n_moments][elements].    */
GG_API int  gg_get_moments(gg_handle* h, double* moments, int32_t* n_moments);
/* y = K x on free dofs (BC rows and columns removed, as the reduced PETSc matrix).    */
GG_API int  gg_apply_K(gg_handle* h, int32_t precision, const double* x, double* y);
/* y = G p (velocity sized, BC rows zero);  q = Gᵀ u (element sized, BC columns zero). */
GG_API int  gg_apply_G(gg_handle* h, const double* p, double* y);
GG_API int  gg_apply_GT(gg_handle* h, const double* u, double* q);
/* Force vectors after BC elimination: f [nodes*dim], h [elements].                   */
GG_API int  gg_get_rhs(gg_handle* h, double* f, double* hvec);
/* Diagonal of the assembled K [nodes*dim] and of Ĝ [elements].                        */
GG_API int  gg_get_diagonals(gg_handle* h, double* k_diag, double* schur_diag);
/* ---- learned coarse correction (no counterpart in the reference) ----------------------
 * gg_learned_train needs an operator built with GG_PRECISION_MIXED.  Weights are FP32
 * on the host side of the ABI; the device runs them in BF16.  n: parameter count.      */
GG_API int  gg_learned_train(gg_handle* h, const gg_learn_params* params, gg_learn_stats* stats);
GG_API int  gg_learned_weights(gg_handle* h, float* weights, int32_t* n);
GG_API int  gg_learned_set_weights(gg_handle* h, int32_t level, const float* weights, int32_t n);
/* Forward and backward of a batch on the network's grid (gradient check): inputs
 * [batch][1+dim][nodes], targets [batch][dim][nodes]; writes outputs, the gradient of
 * the normalised loss w.r.t. all parameters and the loss.  level must exist in the
 * multigrid hierarchy (≤ 0: the default level).  *grid_nodes is in/out: on entry the
 * node count the caller's buffers hold (checked against the level before any buffer is
 * read; GG_ERR_INVALID on a mismatch), on return the level's node count.              */
GG_API int  gg_learned_eval(gg_handle* h, int32_t level, int32_t batch, const float* inputs,
                            const float* targets, const float* weights, float* outputs,
                            float* gradient, double* loss, int32_t* grid_nodes);

/* Measurement only (no reference counterpart): average device time of one matrix-free
 * K apply over `reps` back-to-back launches on the handle's stream, CUDA events.       */
GG_API int  gg_time_apply(gg_handle* h, int32_t precision, int32_t reps, double* ms_per_launch);

/* Inspection only (no reference counterpart): the multigrid hierarchy's dense coarse
 * solve.  Sets up the hierarchy of the built operator if needed and returns in *n the
 * size of its coarsest level (0: that level has no dense inverse); when the pointers are
 * non-null, fills inverse[n*n] with the FP32 inverse the solver applies and op[n*n] with
 * the FP64 operator it inverts, both row-major, the Dirichlet rows and columns of the
 * operator replaced by the identity.                                                    */
GG_API int  gg_get_coarse_inverse(gg_handle* h, int64_t* n, float* inverse, double* op);

/* Measurement only (no reference counterpart): microseconds per grid barrier of the
 * persistent kernels, `iters` barriers in one cooperative launch of `blocks_per_sm`
 * blocks of 256 threads per SM on the current device (CUDA events, default stream).   */
GG_API int  gg_time_grid_barrier(int32_t blocks_per_sm, int32_t iters, double* us_per_barrier);

/* Test of the failure path (no reference counterpart): one cooperative launch of one block
 * per SM in which block 0 leaves without arriving at the persistent kernels' grid barrier,
 * so every other block's wait runs out after `spin_limit` polls.  Returns GG_ERR_CUDA, the
 * status the persistent solver reports for a barrier that gave up, with the number of
 * blocks that gave up; the context stays usable.                                       */
GG_API int  gg_check_grid_barrier_timeout(int32_t spin_limit, int32_t* blocks_gave_up);

#ifdef __cplusplus
}
#endif
#endif /* GALE_GPU_H */
