/*
 * stokes_gpu_host.c -- C host side of the Stokes_SLE_UzawaSolverGPU plugin (see the header).
 * Plain C99 over the C ABI; no CUDA, no PETSc, no StGermain.
 */
#include "stokes_gpu_host.h"

#include <string.h>

gg_uzawa_params StokesGPU_DefaultParams(void) {
    gg_uzawa_params p;
    memset(&p, 0, sizeof p);
    p.tolerance = 1.0e-5;          /* "tolerance"     */
    p.max_iterations = 1000;       /* "maxIterations" */
    p.min_iterations = 1;          /* "minIterations" */
    p.use_absolute_tolerance = 0;  /* "useAbsoluteTolerance" */
    p.use_preconditioner = 1;      /* "Preconditioner" present */
    p.inner = GG_INNER_JACOBI_CG;
    p.precision = GG_PRECISION_FP64;
    p.inner_rtol_factor = 0.1;     /* inner rtol = 0.1 * tolerance (:591,596) */
    p.inner_max_iterations = 10000;
    p.reuse_pressure = 0;
    return p;
}

static int load(gg_handle** h, const gale_stokes_view* v) {
    int rc;
    if (!*h) {
        rc = gg_create(&v->mesh, h);
        if (rc != GG_OK) return rc;
    }
    if (v->bc_fixed)
        rc = gg_set_velocity_bc_nodes(*h, v->bc_fixed, v->bc_values);
    else
        rc = gg_set_velocity_bc(*h, &v->bc);
    if (rc != GG_OK) return rc;
    if ((rc = gg_set_materials(*h, v->n_materials, v->materials)) != GG_OK) return rc;
    if ((rc = gg_set_body_force(*h, &v->force)) != GG_OK) return rc;
    if ((rc = gg_set_temperature(*h, v->temperature)) != GG_OK) return rc;
    if ((rc = gg_set_points(*h, v->n_points, v->coords, v->material, v->plastic_strain)) != GG_OK) return rc;
    return gg_locate(*h, NULL);
}

int StokesGPU_Solve(gg_handle** h, const gale_stokes_view* v, const gg_uzawa_params* params,
                    double* u_nodal, double* p_element, gg_uzawa_stats* stats) {
    int rc = load(h, v);
    if (rc != GG_OK) return rc;
    rc = gg_build_operator(*h, params->precision, 0, NULL, NULL);
    if (rc != GG_OK) return rc;
    return gg_uzawa_solve(*h, params, u_nodal, p_element, stats);
}

int StokesGPU_SolveNonLinear(gg_handle** h, const gale_stokes_view* v, const gg_picard_params* picard,
                             const gg_uzawa_params* params, double* u_nodal, double* p_element,
                             gg_picard_stats* stats) {
    int rc = load(h, v);
    if (rc != GG_OK) return rc;
    return gg_picard(*h, picard, params, u_nodal, p_element, stats);
}
