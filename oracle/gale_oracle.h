/*
 * gale_oracle.h -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the particle-in-cell
 * Q1-P0 Stokes path of Gale.  A plain-C FP64 restatement of the reference algorithm,
 * used by tests/ as the checker, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline / --impl reference legs.  Nothing in the gale_b200 product links it.
 *
 * Parity pinning: the element stiffness assembly is pinned against the reference's
 * golden PETSc matrices (Underworld/Rheology/tests/expected/test{MaterialViscosity,
 * Arrhenius,FrankKamenetskii}2D.matrix, ViscousSuite.cxx:30-110) by
 * tests/test_oracle_golden.py.  The inner Krylov iterate path of PETSc is not
 * vendored with the reference and is not pinned; parity is defined on the converged
 * discrete solution.
 */
#ifndef GALE_ORACLE_H
#define GALE_ORACLE_H
#include <stdint.h>
#include "../include/gale_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_problem or_problem;

/* A1: Mesh_RegularAlgorithms_SearchElements (Mesh_RegularAlgorithms.cxx:191-224).
 * Returns the number of points outside the mesh (their cell = element count).      */
int64_t or_locate(const gg_mesh_desc* m, int64_t n, const double* x, uint32_t* cell);
/* A3: _ElementType_ConvertGlobalCoordToElLocal (ElementType.cxx:221-338).           */
void or_local_coords(const gg_mesh_desc* m, int64_t n, const double* x,
                     const uint32_t* cell, double* xi);
/* A2: per-cell point lists as rebuilt by _CoincidentMapper_Map
 * (CoincidentMapper.cxx:190-215): increasing point index within each cell.          */
void or_cell_lists(int64_t n, const uint32_t* cell, int64_t ncell,
                   int64_t* offsets, int64_t* order);

or_problem* or_create(const gg_mesh_desc* m);
void or_destroy(or_problem* P);
int  or_set_threads(int n);
int  or_set_velocity_bc(or_problem* P, const gg_velocity_bc* bc);
int  or_set_velocity_bc_nodes(or_problem* P, const uint8_t* fixed, const double* values);
int  or_set_materials(or_problem* P, int32_t n, const gg_material* mats);
int  or_set_temperature(or_problem* P, const double* T);
int  or_set_body_force(or_problem* P, const gg_body_force* f);
/* Material points: locate, ξ (Newton) and ConstantWeights.                          */
int  or_set_points(or_problem* P, int64_t n, const double* coords, const int32_t* mat,
                   const double* plastic_strain);
/* Integration points given directly (Gauss swarms of the golden-matrix tests).      */
int  or_set_integration_points(or_problem* P, int64_t n, const uint32_t* cell,
                               const double* xi, const double* weight, const int32_t* mat);
/* K, G, Ĝ, f, h (reference element loops).                                          */
int  or_assemble(or_problem* P, int32_t previous_solution_exists, const double* u,
                 const double* p);
/* Global K (BCs kept, no unit diagonal) as dense [ndof][ndof] for small meshes.     */
int  or_dense_K(or_problem* P, double* K);
int  or_apply_K(or_problem* P, const double* x, double* y);
int  or_apply_G(or_problem* P, const double* p, double* y);
int  or_apply_GT(or_problem* P, const double* u, double* q);
int  or_get_rhs(or_problem* P, double* f, double* h);
int  or_get_diagonals(or_problem* P, double* kdiag, double* sdiag);
int  or_point_viscosity(or_problem* P, double* eta);
int  or_point_yield(or_problem* P, double* increment, uint8_t* yielded);
/* M_m(e) in the product's monomial order (see or_monomials).                       */
int  or_moments(or_problem* P, double* moments, int32_t* n_moments);
int  or_monomials(int32_t dim, int32_t* exponents /* [n][3] */);
int  or_uzawa(or_problem* P, const gg_uzawa_params* prm, double* u, double* p,
              gg_uzawa_stats* st);
int  or_picard(or_problem* P, const gg_picard_params* pic, const gg_uzawa_params* prm,
               double* u, double* p, gg_picard_stats* st);
/* Inner solve alone: x = K⁻¹ b by PETSc-style Jacobi CG; returns iterations.        */
int  or_inner_solve(or_problem* P, const double* b, double* x, double rtol, int32_t maxit);
int  or_advect(or_problem* P, double dt, int32_t order, const double* u, double* coords_out);
int  or_courant_dt(or_problem* P, const double* u, double* dt);
/* FeMesh_CoordLocalToGlobal of points xi [n][dim] in elements cell [n].            */
void or_local_to_global(const gg_mesh_desc* m, int64_t n, const uint32_t* cell, const double* xi, double* x);
const char* or_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
