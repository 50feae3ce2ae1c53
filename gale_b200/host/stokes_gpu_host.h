/*
 * stokes_gpu_host.h -- the C host side of the Stokes_SLE_UzawaSolverGPU plugin.
 *
 * Gale's solver seam is `void _solve(void* sleSolver, void* sle)`
 * (StgFEM/SLE/SystemSetup/src/SLE_Solver.h:61-62).  Inside a Gale build a small adapter
 * reads the Stokes_SLE (Stokes_SLE.h:63-81: kStiffMat, gStiffMat, uSolnVec, pSolnVec,
 * fForceVec, hForceVec and the swarm / rheology components behind them) into the flat
 * view below and calls StokesGPU_Solve; everything below the view is plain C over the
 * C ABI of include/gale_gpu.h and builds without StGermain.
 */
#ifndef STOKES_GPU_HOST_H
#define STOKES_GPU_HOST_H

#include <stdint.h>

#include "../../include/gale_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gale_stokes_view {
    gg_mesh_desc mesh;               /* CartesianGenerator geometry          */
    gg_velocity_bc bc;               /* velocityBCs WallVC list              */
    int32_t n_materials;
    gg_material materials[GG_MAX_MATERIALS];
    gg_body_force force;             /* BuoyancyForceTerm / ThermalBuoyancy  */
    int64_t n_points;                /* MaterialPointsSwarm                  */
    const double* coords;            /* [n_points*dim]                      */
    const int32_t* material;         /* [n_points]                          */
    const double* plastic_strain;    /* [n_points] or NULL                  */
    const double* temperature;       /* nodal TemperatureField or NULL      */
    /* per-node velocity conditions (VariableCondition_Apply at the nodes, condition
       functions included); when set they replace `bc`                      */
    const uint8_t* bc_fixed;         /* [nodes] bit c: component c fixed    */
    const double* bc_values;         /* [nodes*dim] node-major              */
} gale_stokes_view;

/* Create (or reuse when *h is set) the handle, load the view, locate the points, build
 * the operator and run the Uzawa solve.  Returns a GG_ status; the caller turns a
 * non-zero status into Journal_Firewall as the reference does. */
int StokesGPU_Solve(gg_handle** h, const gale_stokes_view* v, const gg_uzawa_params* params,
                    double* u_nodal, double* p_element, gg_uzawa_stats* stats);

/* Picard form (SystemLinearEquations_NonLinearExecute). */
int StokesGPU_SolveNonLinear(gg_handle** h, const gale_stokes_view* v, const gg_picard_params* picard,
                             const gg_uzawa_params* params, double* u_nodal, double* p_element,
                             gg_picard_stats* stats);

/* Defaults of the Stokes_SLE_UzawaSolver XML keys (Stokes_SLE_UzawaSolver.cxx:251-255). */
gg_uzawa_params StokesGPU_DefaultParams(void);

#ifdef __cplusplus
}
#endif
#endif
