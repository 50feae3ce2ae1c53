/*
 * gale_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see gale_oracle.h).
 *
 * FP64 restatement of Gale's PIC Q1-P0 Stokes path, written from the reference
 * sources cited beside each function.  Compiled with -ffp-contract=off so the
 * point→cell search reproduces the reference's IEEE arithmetic bit for bit.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 */
#include "gale_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static char g_err[512];
const char* or_last_error(void) { return g_err; }
static int fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

int or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ------------------------------------------------------------------ mesh --- */
typedef struct {
    int dim, n[3], nn[3];
    int64_t nel, nnode;
    int nen;
    double min[3], max[3];
} mesh_t;

static void mesh_init(mesh_t* M, const gg_mesh_desc* d) {
    M->dim = d->dim;
    M->nel = 1;
    M->nnode = 1;
    for (int i = 0; i < 3; i++) {
        M->n[i] = i < d->dim ? d->elements[i] : 1;
        M->nn[i] = i < d->dim ? d->elements[i] + 1 : 1;
        M->min[i] = i < d->dim ? d->min[i] : 0.0;
        M->max[i] = i < d->dim ? d->max[i] : 0.0;
    }
    for (int i = 0; i < d->dim; i++) {
        M->nel *= M->n[i];
        M->nnode *= M->nn[i];
    }
    M->nen = 1 << d->dim;
}

/* Vertex coordinate of grid index i along axis d: CartesianGenerator_CalcGeom
 * (StgDomain/Mesh/src/CartesianGenerator.cxx:2178-2215) without contact depth.      */
static double vert_coord(const mesh_t* M, int d, int i) {
    if (i == 0) return M->min[d];
    if (i == M->n[d]) return M->max[d];
    return M->min[d] + ((double)i / (double)M->n[d]) * (M->max[d] - M->min[d]);
}

static void elem_ijk(const mesh_t* M, int64_t e, int* ijk) {
    ijk[0] = (int)(e % M->n[0]);
    int64_t r = e / M->n[0];
    ijk[1] = (int)(r % M->n[1]);
    ijk[2] = (int)(r / M->n[1]);
}

/* Element-local node a → global node (BilinearElementType.cxx:216-245 ordering).    */
static int64_t elem_node(const mesh_t* M, const int* ijk, int a) {
    int i = ijk[0] + (a & 1), j = ijk[1] + ((a >> 1) & 1), k = ijk[2] + ((a >> 2) & 1);
    return i + (int64_t)M->nn[0] * (j + (int64_t)M->nn[1] * k);
}

static void node_xyz(const mesh_t* M, int64_t n, double* x) {
    int i = (int)(n % M->nn[0]);
    int64_t r = n / M->nn[0];
    int j = (int)(r % M->nn[1]);
    int k = (int)(r / M->nn[1]);
    x[0] = vert_coord(M, 0, i);
    x[1] = vert_coord(M, 1, j);
    x[2] = M->dim == 3 ? vert_coord(M, 2, k) : 0.0;
}

/* Shape functions and local derivatives, Q1 (BilinearElementType.cxx:216-245,
 * TrilinearElementType.cxx:257-300).                                                */
static void shape(int dim, const double* xi, double* N) {
    if (dim == 2) {
        N[0] = 0.25 * (1.0 - xi[0]) * (1.0 - xi[1]);
        N[1] = 0.25 * (1.0 + xi[0]) * (1.0 - xi[1]);
        N[3] = 0.25 * (1.0 + xi[0]) * (1.0 + xi[1]);
        N[2] = 0.25 * (1.0 - xi[0]) * (1.0 + xi[1]);
    } else {
        for (int a = 0; a < 8; a++) {
            double s = (a & 1) ? 1.0 : -1.0, t = (a & 2) ? 1.0 : -1.0, r = (a & 4) ? 1.0 : -1.0;
            N[a] = 0.125 * (1.0 + s * xi[0]) * (1.0 + t * xi[1]) * (1.0 + r * xi[2]);
        }
    }
}

static void shape_local_derivs(int dim, const double* xi, double GNi[3][8]) {
    if (dim == 2) {
        GNi[0][0] = -0.25 * (1.0 - xi[1]);
        GNi[0][1] = 0.25 * (1.0 - xi[1]);
        GNi[0][3] = 0.25 * (1.0 + xi[1]);
        GNi[0][2] = -0.25 * (1.0 + xi[1]);
        GNi[1][0] = -0.25 * (1.0 - xi[0]);
        GNi[1][1] = -0.25 * (1.0 + xi[0]);
        GNi[1][3] = 0.25 * (1.0 + xi[0]);
        GNi[1][2] = 0.25 * (1.0 - xi[0]);
    } else {
        for (int a = 0; a < 8; a++) {
            double s = (a & 1) ? 1.0 : -1.0, t = (a & 2) ? 1.0 : -1.0, r = (a & 4) ? 1.0 : -1.0;
            GNi[0][a] = 0.125 * s * (1.0 + t * xi[1]) * (1.0 + r * xi[2]);
            GNi[1][a] = 0.125 * t * (1.0 + s * xi[0]) * (1.0 + r * xi[2]);
            GNi[2][a] = 0.125 * r * (1.0 + s * xi[0]) * (1.0 + t * xi[1]);
        }
    }
}

/* ElementType_ShapeFunctionsGlobalDerivs (ElementType.cxx:339-474): Jacobian from the
 * element's vertices, inverse by cofactors, GNx = J⁻¹ GNi.                           */
static void global_derivs(const mesh_t* M, const int* ijk, const double* xi, double* detJ,
                          double GNx[3][8]) {
    int dim = M->dim, nen = M->nen;
    double GNi[3][8], jac[3][3] = {{0}}, X[8][3];
    shape_local_derivs(dim, xi, GNi);
    for (int a = 0; a < nen; a++) node_xyz(M, elem_node(M, ijk, a), X[a]);
    for (int r = 0; r < dim; r++)
        for (int c = 0; c < dim; c++)
            for (int a = 0; a < nen; a++) jac[r][c] = jac[r][c] + GNi[r][a] * X[a][c];
    double D, inv[3][3];
    if (dim == 2) {
        D = jac[0][0] * jac[1][1] - jac[0][1] * jac[1][0];
        inv[0][0] = jac[1][1] / D;
        inv[1][1] = jac[0][0] / D;
        inv[0][1] = -jac[0][1] / D;
        inv[1][0] = -jac[1][0] / D;
    } else {
        D = jac[0][0] * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]) -
            jac[0][1] * (jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]) +
            jac[0][2] * (jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]);
        double cof[3][3];
        cof[0][0] = jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1];
        cof[1][0] = -(jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]);
        cof[2][0] = jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0];
        cof[0][1] = -(jac[0][1] * jac[2][2] - jac[0][2] * jac[2][1]);
        cof[1][1] = jac[0][0] * jac[2][2] - jac[0][2] * jac[2][0];
        cof[2][1] = -(jac[0][0] * jac[2][1] - jac[0][1] * jac[2][0]);
        cof[0][2] = jac[0][1] * jac[1][2] - jac[0][2] * jac[1][1];
        cof[1][2] = -(jac[0][0] * jac[1][2] - jac[0][2] * jac[1][0]);
        cof[2][2] = jac[0][0] * jac[1][1] - jac[0][1] * jac[1][0];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) inv[r][c] = cof[r][c] / D;
    }
    *detJ = D;
    for (int dx = 0; dx < dim; dx++)
        for (int a = 0; a < nen; a++) {
            double v = 0.0;
            for (int dxi = 0; dxi < dim; dxi++) v = v + GNi[dxi][a] * inv[dx][dxi];
            GNx[dx][a] = v;
        }
}

/* FeMesh_CoordLocalToGlobal (StgFEM/Discretisation/src/FeMesh.cxx:366-400).          */
static void local_to_global(const mesh_t* M, const int* ijk, const double* xi, double* x) {
    double N[8], X[3];
    shape(M->dim, xi, N);
    x[0] = x[1] = x[2] = 0.0;
    for (int a = 0; a < M->nen; a++) {
        node_xyz(M, elem_node(M, ijk, a), X);
        for (int d = 0; d < M->dim; d++) x[d] += N[a] * X[d];
    }
}

/* Global coordinates of local points xi [n][dim] in elements cell [n].               */
void or_local_to_global(const gg_mesh_desc* md, int64_t n, const uint32_t* cell, const double* xi, double* x) {
    mesh_t M;
    mesh_init(&M, md);
    for (int64_t p = 0; p < n; p++) {
        int ijk[3];
        elem_ijk(&M, cell[p], ijk);
        double g[3];
        local_to_global(&M, ijk, xi + p * M.dim, g);
        for (int d = 0; d < M.dim; d++) x[p * M.dim + d] = g[d];
    }
}

/* -------------------------------------------------------------- A1 locate --- */
/* Num_Approx (StGermain/Base/Foundation/src/Numerics.cxx:38-43), ε = 1e-12.         */
static int num_approx(double var, double val) {
    const double eps = 1e-12;
    return (var >= val - eps && var <= val + eps);
}

static int search_element(const mesh_t* M, const double* sep, const double* pt, int64_t* el) {
    int inds[3] = {0, 0, 0};
    for (int d = 0; d < M->dim; d++) {
        if (num_approx(pt[d] - M->max[d], 0.0))
            inds[d] = M->n[d] - 1;
        else if (pt[d] < M->min[d] || pt[d] > M->max[d])
            return 0;
        else {
            double out = (pt[d] - M->min[d]) / sep[d];
            double integer;
            double frac = modf(out, &integer);
            inds[d] = (int)(unsigned)integer;
            if (inds[d] > 0 && num_approx(frac, 0.0)) inds[d]--;
            /* out can round to n only within an ulp of max, which the first
               branch already claims; kept in range for safety */
            if (inds[d] >= M->n[d]) inds[d] = M->n[d] - 1;
        }
    }
    *el = inds[0] + (int64_t)M->n[0] * (inds[1] + (int64_t)M->n[1] * inds[2]);
    return 1;
}

static void mesh_sep(const mesh_t* M, double* sep) {
    for (int d = 0; d < 3; d++) sep[d] = d < M->dim ? (M->max[d] - M->min[d]) / M->n[d] : 1.0;
}

int64_t or_locate(const gg_mesh_desc* md, int64_t n, const double* x, uint32_t* cell) {
    mesh_t M;
    mesh_init(&M, md);
    double sep[3];
    mesh_sep(&M, sep);
    int64_t outside = 0;
#pragma omp parallel for reduction(+ : outside) schedule(static)
    for (int64_t p = 0; p < n; p++) {
        int64_t el;
        if (search_element(&M, sep, x + p * M.dim, &el))
            cell[p] = (uint32_t)el;
        else {
            cell[p] = (uint32_t)M.nel;
            outside++;
        }
    }
    return outside;
}

/* ----------------------------------------------------------- A3 Newton ξ --- */
static void solve_cramer(int dim, double J[3][3], const double* b, double* x) {
    if (dim == 2) {
        double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        x[0] = (b[0] * J[1][1] - J[0][1] * b[1]) / det;
        x[1] = (J[0][0] * b[1] - b[0] * J[1][0]) / det;
        return;
    }
    double det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
                 J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    x[0] = (b[0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
            J[0][1] * (b[1] * J[2][2] - J[1][2] * b[2]) +
            J[0][2] * (b[1] * J[2][1] - J[1][1] * b[2])) / det;
    x[1] = (J[0][0] * (b[1] * J[2][2] - b[2] * J[1][2]) -
            b[0] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
            J[0][2] * (J[1][0] * b[2] - b[1] * J[2][0])) / det;
    x[2] = (J[0][0] * (J[1][1] * b[2] - J[2][1] * b[1]) -
            J[0][1] * (J[1][0] * b[2] - b[1] * J[2][0]) +
            b[0] * (J[1][0] * J[2][1] - J[1][1] * J[2][0])) / det;
}

static void newton_xi(const mesh_t* M, const int* ijk, const double* gx, double* xi) {
    int dim = M->dim, nen = M->nen;
    double X[8][3];
    for (int a = 0; a < nen; a++) node_xyz(M, elem_node(M, ijk, a), X[a]);
    xi[0] = xi[1] = xi[2] = 0.0;
    for (int it = 0; it < 100; it++) {
        double N[8], GNi[3][8], J[3][3] = {{0}}, rhs[3] = {0, 0, 0}, inc[3] = {0, 0, 0};
        shape(dim, xi, N);
        shape_local_derivs(dim, xi, GNi);
        for (int a = 0; a < nen; a++) {
            for (int r = 0; r < dim; r++)
                for (int c = 0; c < dim; c++) J[r][c] += GNi[c][a] * X[a][r];
            for (int r = 0; r < dim; r++) rhs[r] -= N[a] * X[a][r];
        }
        for (int r = 0; r < dim; r++) rhs[r] += gx[r];
        solve_cramer(dim, J, rhs, inc);
        double mx = 0.0;
        for (int r = 0; r < dim; r++) {
            xi[r] += inc[r];
            if (mx < fabs(inc[r])) mx = fabs(inc[r]);
        }
        if (mx < 0.0001) break;
    }
}

void or_local_coords(const gg_mesh_desc* md, int64_t n, const double* x, const uint32_t* cell,
                     double* xi) {
    mesh_t M;
    mesh_init(&M, md);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; p++) {
        int ijk[3];
        double t[3];
        elem_ijk(&M, cell[p], ijk);
        newton_xi(&M, ijk, x + p * M.dim, t);
        for (int d = 0; d < M.dim; d++) xi[p * M.dim + d] = t[d];
    }
}

void or_cell_lists(int64_t n, const uint32_t* cell, int64_t ncell, int64_t* offsets,
                   int64_t* order) {
    memset(offsets, 0, sizeof(int64_t) * (ncell + 1));
    for (int64_t p = 0; p < n; p++)
        if (cell[p] < ncell) offsets[cell[p] + 1]++;
    for (int64_t c = 0; c < ncell; c++) offsets[c + 1] += offsets[c];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (ncell + 1));
    memcpy(fill, offsets, sizeof(int64_t) * (ncell + 1));
    for (int64_t p = 0; p < n; p++)
        if (cell[p] < ncell) order[fill[cell[p]]++] = p;
    free(fill);
}

/* ---------------------------------------------------------------- problem --- */
struct or_problem {
    mesh_t M;
    int64_t ndof;
    uint8_t* bcmask;  /* per node, bit c: component c fixed */
    double* bcval;    /* [nnode*dim]                         */
    int nmat;
    gg_material mats[GG_MAX_MATERIALS];
    double* T;        /* nodal temperature or NULL           */
    gg_body_force force;
    /* points */
    int64_t np;
    double* coords;
    int32_t* mat;
    double* pstrain;
    uint32_t* cell;
    double* xi;
    double* w;
    int64_t* offsets;
    int64_t* order;
    /* per-point outputs */
    double* eta;
    double* incr;
    uint8_t* yielded;
    /* assembled operators */
    int nb;           /* stencil size 9 / 27 */
    double* Kb;       /* [nnode][nb][dim][dim] */
    double* kdiag;    /* [ndof] assembled diagonal */
    double* sdiag;    /* [nel] Ĝ                  */
    double* f;        /* [ndof]                    */
    double* h;        /* [nel]                     */
    double Ge[8][3];  /* constant element G stencil */
    int assembled;
};

or_problem* or_create(const gg_mesh_desc* md) {
    if (!md || (md->dim != 2 && md->dim != 3)) return NULL;
    or_problem* P = (or_problem*)calloc(1, sizeof(or_problem));
    mesh_init(&P->M, md);
    P->ndof = P->M.nnode * P->M.dim;
    P->bcmask = (uint8_t*)calloc(P->M.nnode, 1);
    P->bcval = (double*)calloc(P->ndof, sizeof(double));
    P->nb = P->M.dim == 2 ? 9 : 27;
    P->force.g_hat[1] = -1.0;
    return P;
}

void or_destroy(or_problem* P) {
    if (!P) return;
    free(P->bcmask); free(P->bcval); free(P->T);
    free(P->coords); free(P->mat); free(P->pstrain); free(P->cell); free(P->xi); free(P->w);
    free(P->offsets); free(P->order); free(P->eta); free(P->incr); free(P->yielded);
    free(P->Kb); free(P->kdiag); free(P->sdiag); free(P->f); free(P->h);
    free(P);
}

/* WallVC semantics: walls applied in order, later walls override shared nodes.     */
int or_set_velocity_bc(or_problem* P, const gg_velocity_bc* bc) {
    mesh_t* M = &P->M;
    memset(P->bcmask, 0, M->nnode);
    memset(P->bcval, 0, sizeof(double) * P->ndof);
    for (int64_t n = 0; n < M->nnode; n++) {
        int idx[3] = {(int)(n % M->nn[0]), (int)((n / M->nn[0]) % M->nn[1]),
                      (int)(n / ((int64_t)M->nn[0] * M->nn[1]))};
        for (int wall = 0; wall < 2 * M->dim; wall++) {
            int ax = wall / 2, hi = wall & 1;
            int on = hi ? (idx[ax] == M->n[ax]) : (idx[ax] == 0);
            if (!on) continue;
            for (int c = 0; c < M->dim; c++)
                if (bc->fixed[wall][c]) {
                    P->bcmask[n] |= (uint8_t)(1u << c);
                    P->bcval[n * M->dim + c] = bc->value[wall][c];
                }
        }
    }
    P->assembled = 0;
    return GG_OK;
}

/* Per-node velocity BCs: a VariableCondition whose values come from a condition function
 * evaluated at the nodes (VariableCondition "func" entries, e.g.
 * StgFEM_StandardConditionFunctions_PartialLid_TopLayer, StgFEM/plugins/
 * StandardConditionFunctions/StandardConditionFunctions.cxx:547-568).  fixed[n] bit c:
 * component c fixed; values [nnode*dim], read on fixed components only. */
int or_set_velocity_bc_nodes(or_problem* P, const uint8_t* fixed, const double* values) {
    mesh_t* M = &P->M;
    if (!fixed || !values) return fail(GG_ERR_INVALID, "null BC arrays");
    for (int64_t n = 0; n < M->nnode; n++) {
        P->bcmask[n] = (uint8_t)(fixed[n] & ((1u << M->dim) - 1u));
        for (int c = 0; c < M->dim; c++)
            P->bcval[n * M->dim + c] = (P->bcmask[n] >> c) & 1 ? values[n * M->dim + c] : 0.0;
    }
    P->assembled = 0;
    return GG_OK;
}

int or_set_materials(or_problem* P, int32_t n, const gg_material* mats) {
    if (n < 1 || n > GG_MAX_MATERIALS) return fail(GG_ERR_INVALID, "material count");
    for (int i = 0; i < n; i++)
        for (int k = 0; k < mats[i].n_rheologies && k < GG_MAX_RHEOLOGIES; k++)
            if (mats[i].rheology[k].hydrostatic_term)
                return fail(GG_ERR_INVALID, "DruckerPrager HydrostaticTerm is not supported");
    P->nmat = n;
    memcpy(P->mats, mats, sizeof(gg_material) * n);
    return GG_OK;
}

int or_set_temperature(or_problem* P, const double* T) {
    free(P->T);
    P->T = NULL;
    if (T) {
        P->T = (double*)malloc(sizeof(double) * P->M.nnode);
        memcpy(P->T, T, sizeof(double) * P->M.nnode);
    }
    return GG_OK;
}

int or_set_body_force(or_problem* P, const gg_body_force* f) {
    P->force = *f;
    double nrm = 0.0;
    for (int d = 0; d < P->M.dim; d++) nrm += f->g_hat[d] * f->g_hat[d];
    nrm = sqrt(nrm);
    if (nrm > 0)
        for (int d = 0; d < P->M.dim; d++) P->force.g_hat[d] = f->g_hat[d] / nrm;
    return GG_OK;
}

static void alloc_points(or_problem* P, int64_t n) {
    int dim = P->M.dim;
    free(P->coords); free(P->mat); free(P->pstrain); free(P->cell); free(P->xi); free(P->w);
    free(P->offsets); free(P->order); free(P->eta); free(P->incr); free(P->yielded);
    P->np = n;
    P->coords = (double*)calloc(n * dim + 1, sizeof(double));
    P->mat = (int32_t*)calloc(n + 1, sizeof(int32_t));
    P->pstrain = (double*)calloc(n + 1, sizeof(double));
    P->cell = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    P->xi = (double*)calloc(n * dim + 1, sizeof(double));
    P->w = (double*)calloc(n + 1, sizeof(double));
    P->offsets = (int64_t*)calloc(P->M.nel + 1, sizeof(int64_t));
    P->order = (int64_t*)calloc(n + 1, sizeof(int64_t));
    P->eta = (double*)calloc(n + 1, sizeof(double));
    P->incr = (double*)calloc(n + 1, sizeof(double));
    P->yielded = (uint8_t*)calloc(n + 1, 1);
}

int or_set_points(or_problem* P, int64_t n, const double* coords, const int32_t* mat,
                  const double* pstrain) {
    mesh_t* M = &P->M;
    alloc_points(P, n);
    memcpy(P->coords, coords, sizeof(double) * n * M->dim);
    for (int64_t p = 0; p < n; p++) {
        P->mat[p] = mat ? mat[p] : 0;
        P->pstrain[p] = pstrain ? pstrain[p] : 0.0;
    }
    gg_mesh_desc md = {M->dim, {M->n[0], M->n[1], M->n[2]}, {M->min[0], M->min[1], M->min[2]},
                       {M->max[0], M->max[1], M->max[2]}};
    if (or_locate(&md, n, P->coords, P->cell) != 0)
        return fail(GG_ERR_OUT_OF_DOMAIN, "material point outside the mesh");
    or_local_coords(&md, n, P->coords, P->cell, P->xi);
    or_cell_lists(n, P->cell, M->nel, P->offsets, P->order);
    /* _ConstantWeights_Calculate: w = cellLocalVolume / count, cellLocalVolume = 2^dim
       (WeightsCalculator.cxx:84, ConstantWeights.cxx:178-187)                       */
    for (int64_t e = 0; e < M->nel; e++) {
        int64_t c = P->offsets[e + 1] - P->offsets[e];
        if (c == 0) return fail(GG_ERR_EMPTY_CELL, "element without material points");
        double wt = (double)(1 << M->dim) / (double)c;
        for (int64_t k = P->offsets[e]; k < P->offsets[e + 1]; k++) P->w[P->order[k]] = wt;
    }
    P->assembled = 0;
    return GG_OK;
}

int or_set_integration_points(or_problem* P, int64_t n, const uint32_t* cell, const double* xi,
                              const double* weight, const int32_t* mat) {
    mesh_t* M = &P->M;
    alloc_points(P, n);
    memcpy(P->cell, cell, sizeof(uint32_t) * n);
    memcpy(P->xi, xi, sizeof(double) * n * M->dim);
    memcpy(P->w, weight, sizeof(double) * n);
    for (int64_t p = 0; p < n; p++) {
        int ijk[3];
        P->mat[p] = mat ? mat[p] : 0;
        elem_ijk(M, cell[p], ijk);
        local_to_global(M, ijk, xi + p * M->dim, P->coords + p * M->dim);
    }
    or_cell_lists(n, P->cell, M->nel, P->offsets, P->order);
    P->assembled = 0;
    return GG_OK;
}

/* ------------------------------------------------------------ A4 rheology --- */
static double interp_nodal(const mesh_t* M, const int* ijk, const double* xi, const double* v) {
    double N[8], s = 0.0;
    shape(M->dim, xi, N);
    for (int a = 0; a < M->nen; a++) s += v[elem_node(M, ijk, a)] * N[a];
    return s;
}

/* StrainWeakening_CalcRatio (StrainWeakening.cxx:497-519).                          */
static double sw_ratio(const gg_material* m, const gg_rheology* r, double* ep) {
    if (!m->has_strain_weakening || !r->strain_weakening) return 0.0;
    if (*ep < 0.0) *ep = 0.0;
    const gg_strain_weakening* s = &m->strain_weakening;
    double ratio = (*ep - s->initial_softening_strain) /
                   (s->final_softening_strain - s->initial_softening_strain);
    if (ratio > 1.0) ratio = 1.0;
    if (ratio < 0.0) ratio = 0.0;
    return ratio;
}

/* SymmetricTensor_2ndInvariant (StgDomain/Geometry/src/TensorMath.cxx:431-460) on the
 * reference storage [xx,yy,xy] / [xx,yy,zz,xy,xz,yz].                                */
static double second_invariant(int dim, const double* t) {
    if (dim == 2) return sqrt(0.5 * (t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);
    return sqrt(0.5 * (t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) + t[3] * t[3] + t[4] * t[4] +
                t[5] * t[5]);
}

/* Strain rate at ξ from the nodal velocity (StrainRateField: symmetric part of the
 * velocity gradient, FeVariable_InterpolateDerivatives_WithGNx FeVariable.cxx:1165-1204). */
static void strain_rate(const mesh_t* M, const int* ijk, const double* xi, const double* u,
                        double* sr) {
    double detJ, GNx[3][8], g[3][3] = {{0}};
    int dim = M->dim;
    global_derivs(M, ijk, xi, &detJ, GNx);
    for (int a = 0; a < M->nen; a++) {
        int64_t n = elem_node(M, ijk, a);
        for (int c = 0; c < dim; c++)
            for (int d = 0; d < dim; d++) g[c][d] += GNx[d][a] * u[n * dim + c];
    }
    if (dim == 2) {
        sr[0] = g[0][0];
        sr[1] = g[1][1];
        sr[2] = 0.5 * (g[0][1] + g[1][0]);
    } else {
        sr[0] = g[0][0];
        sr[1] = g[1][1];
        sr[2] = g[2][2];
        sr[3] = 0.5 * (g[0][1] + g[1][0]);
        sr[4] = 0.5 * (g[0][2] + g[2][0]);
        sr[5] = 0.5 * (g[1][2] + g[2][1]);
    }
}

/* RheologyMaterial_RunRheologies → Rheology_Register_RunRheologies
 * (Rheology_Register.cxx:70-86): each law in order modifies the isotropic viscosity.  */
static double run_rheologies(const or_problem* P, int64_t p, int prev, const double* u,
                             const double* pres, double* incr_out, uint8_t* yielded_out) {
    const mesh_t* M = &P->M;
    int dim = M->dim;
    int ijk[3];
    elem_ijk(M, P->cell[p], ijk);
    const double* xi = P->xi + p * dim;
    const gg_material* m = &P->mats[P->mat[p]];
    double eta = 0.0;
    double ep = P->pstrain[p];
    *incr_out = 0.0;
    *yielded_out = 0;
    for (int ri = 0; ri < m->n_rheologies; ri++) {
        const gg_rheology* r = &m->rheology[ri];
        switch (r->kind) {
        case GG_RHEO_MATERIAL_VISCOSITY: /* MaterialViscosity.cxx:139 */
            eta = r->eta0;
            break;
        case GG_RHEO_ARRHENIUS: { /* Arrhenius.cxx:186-219 */
            double T = P->T ? interp_nodal(M, ijk, xi, P->T) : 0.0;
            if (r->activation_volume > (0.0 + 1e-12)) {
                double x[3];
                local_to_global(M, ijk, xi, x);
                double depth = M->max[1] - x[1];
                eta = r->eta0 * exp((r->activation_energy + r->activation_volume * depth) /
                                    (T + r->reference_temp));
            } else {
                eta = r->eta0 * exp(r->activation_energy / (T + r->reference_temp));
            }
            break;
        }
        case GG_RHEO_FRANK_KAMENETSKII: { /* FrankKamenetskii.cxx:156-160 */
            double T = P->T ? interp_nodal(M, ijk, xi, P->T) : 0.0;
            eta = r->eta0 * exp(-r->theta * T);
            break;
        }
        case GG_RHEO_VON_MISES:
        case GG_RHEO_DRUCKER_PRAGER:
        case GG_RHEO_BYERLEE: {
            /* _YieldRheology_ModifyConstitutiveMatrix (YieldRheology.cxx:190-228) */
            if (!prev) break;
            /* indicator: _VonMises_GetYieldIndicator (VonMises.cxx:207-248) */
            double sr[6], st[6];
            strain_rate(M, ijk, xi, u, sr);
            int ns = dim == 2 ? 3 : 6;
            for (int k = 0; k < ns; k++) st[k] = 2.0 * eta * sr[k];
            double trs = 0.0, trsr = 0.0;
            for (int k = 0; k < dim; k++) {
                trs += st[k];
                trsr += sr[k];
            }
            for (int k = 0; k < dim; k++) {
                sr[k] -= trsr / dim;
                st[k] -= trs / dim;
            }
            double sr_ii = second_invariant(dim, sr);
            double ind = second_invariant(dim, st);
            /* criterion */
            double crit;
            double ratio = sw_ratio(m, r, &ep);
            if (r->kind == GG_RHEO_VON_MISES) { /* VonMises.cxx:183-204 */
                crit = r->cohesion * (1.0 - ratio) + r->cohesion_after_softening * ratio;
            } else if (r->kind == GG_RHEO_DRUCKER_PRAGER) { /* DruckerPrager.cxx:296-412 */
                double pressure = pres ? pres[P->cell[p]] : 0.0;
                /* inside_boundary (:341-361): the element touches a flagged wall */
                int bw = r->boundary_walls;
                int inb = ((bw & 1) && ijk[0] == 0) || ((bw & 2) && ijk[0] == M->n[0] - 1) ||
                          ((bw & 4) && ijk[1] == 0) || ((bw & 8) && ijk[1] == M->n[1] - 1) ||
                          (dim == 3 && (((bw & 16) && ijk[2] == 0) || ((bw & 32) && ijk[2] == M->n[2] - 1)));
                /* _DruckerPrager_EffectiveFrictionCoefficient / _EffectiveCohesion (:448-490) */
                double mu = inb ? r->boundary_friction_coefficient * (1.0 - ratio) +
                                      r->boundary_friction_coefficient_after_softening * ratio
                                : r->friction_coefficient * (1.0 - ratio) +
                                      r->friction_coefficient_after_softening * ratio;
                double C = inb ? r->boundary_cohesion * (1.0 - ratio) + r->boundary_cohesion_after_softening * ratio
                               : r->cohesion * (1.0 - ratio) + r->cohesion_after_softening * ratio;
                double factor, fs;
                if (dim == 2) {
                    factor = 1 / sqrt(1 + mu * mu);
                    fs = mu * pressure * factor + C * factor;
                } else {
                    double cphi = 1 / sqrt(1 + mu * mu), sphi = mu * cphi;
                    factor = 2 * cphi / (sqrt(3.0) * (3 - sphi));
                    fs = mu * factor * pressure + C * 3 * factor;
                }
                double mys = r->minimum_yield_stress;
                if (mys == 0.0) mys = C;
                if (fs < mys * factor) fs = mys * factor;
                crit = fs;
            } else { /* Byerlee.cxx:163-187 */
                double x[3];
                local_to_global(M, ijk, xi, x);
                crit = r->cohesion + r->depth_coefficient * (M->max[1] - x[1]);
            }
            /* StrainWeakening_AssignIncrement before HasYielded (YieldRheology.cxx:206-218),
               _StrainWeakening_CalcIncrementIsotropic (StrainWeakening.cxx:470-495) */
            if (m->has_strain_weakening && r->strain_weakening) {
                double beta = 1.0 - crit / ind;
                if (beta < 0.0) beta = 0.0;
                *incr_out = (crit / eta) * (beta / (1.0 - beta) -
                                            m->strain_weakening.healing_rate * ep);
            }
            if (crit < ind) {
                *yielded_out = 1;
                if (r->kind == GG_RHEO_DRUCKER_PRAGER) { /* DruckerPrager.cxx:414-446 */
                    double v;
                    if (r->max_strain_rate > 0 && sr_ii > r->max_strain_rate)
                        v = crit / (2 * r->max_strain_rate);
                    else
                        v = crit / (2 * sr_ii);
                    if (v < r->minimum_viscosity) v = r->minimum_viscosity;
                    eta = v;
                } else if (r->strain_rate_softening) { /* VonMises.cxx:258-263 */
                    eta = 2.0 * crit * crit * eta / (crit * crit + ind * ind);
                } else { /* VonMises.cxx:264-271 */
                    double beta = 1.0 - crit / ind;
                    double corr = -eta * beta;
                    if ((eta + corr) < r->minimum_viscosity) corr = r->minimum_viscosity - eta;
                    eta += corr;
                }
            }
            break;
        }
        default:
            break;
        }
    }
    return eta;
}

/* ------------------------------------------------------- A5/A6 assembly --- */
static int nbr_index(int dim, int di, int dj, int dk) {
    return dim == 2 ? (di + 1) + 3 * (dj + 1) : (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
}

/* Element K over the cell's integration points: the loop of
 * _ConstitutiveMatrixCartesian_AssembleElement (ConstitutiveMatrixCartesian.cxx:363-486)
 * with isotropic D (ConstitutiveMatrixCartesian.cxx:536-556) and D~B (:631-724).
 * Ke[test dof][trial dof].                                                            */
static void element_K(const or_problem* P, int64_t e, double Ke[24][24]) {
    const mesh_t* M = &P->M;
    int dim = M->dim, nen = M->nen, nd = nen * dim;
    int ijk[3];
    elem_ijk(M, e, ijk);
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) Ke[i][j] = 0.0;
    for (int64_t k = P->offsets[e]; k < P->offsets[e + 1]; k++) {
        int64_t p = P->order[k];
        double detJ, GNx[3][8];
        global_derivs(M, ijk, P->xi + p * dim, &detJ, GNx);
        double eta = P->eta[p];
        double c = detJ * P->w[p];
        if (dim == 2) {
            double D00 = 2.0 * eta * c, D11 = 2.0 * eta * c, D22 = eta * c;
            for (int rn = 0; rn < nen; rn++) {
                double dx = GNx[0][rn], dy = GNx[1][rn];
                double DB[3][2] = {{D00 * dx, 0.0}, {0.0, D11 * dy}, {D22 * dy, D22 * dx}};
                for (int cn = 0; cn < nen; cn++) {
                    double bx = GNx[0][cn], by = GNx[1][cn];
                    Ke[cn * 2][rn * 2] += bx * DB[0][0] + by * DB[2][0];
                    Ke[cn * 2][rn * 2 + 1] += bx * DB[0][1] + by * DB[2][1];
                    Ke[cn * 2 + 1][rn * 2] += by * DB[1][0] + bx * DB[2][0];
                    Ke[cn * 2 + 1][rn * 2 + 1] += by * DB[1][1] + bx * DB[2][1];
                }
            }
        } else {
            double Dn = 2.0 * eta * c, Ds = eta * c;
            for (int rn = 0; rn < nen; rn++) {
                double dx = GNx[0][rn], dy = GNx[1][rn], dz = GNx[2][rn];
                double DB[6][3] = {{Dn * dx, 0, 0},  {0, Dn * dy, 0},  {0, 0, Dn * dz},
                                   {Ds * dy, Ds * dx, 0}, {Ds * dz, 0, Ds * dx}, {0, Ds * dz, Ds * dy}};
                for (int cn = 0; cn < nen; cn++) {
                    double bx = GNx[0][cn], by = GNx[1][cn], bz = GNx[2][cn];
                    for (int j = 0; j < 3; j++) {
                        Ke[cn * 3][rn * 3 + j] += bx * DB[0][j] + by * DB[3][j] + bz * DB[4][j];
                        Ke[cn * 3 + 1][rn * 3 + j] += by * DB[1][j] + bx * DB[3][j] + bz * DB[5][j];
                        Ke[cn * 3 + 2][rn * 3 + j] += bz * DB[2][j] + bx * DB[4][j] + by * DB[5][j];
                    }
                }
            }
        }
    }
}

/* Element G on the 2^dim Gauss swarm (GradientStiffnessMatrixTerm.cxx:161-251):
 * G_e[a*dim+d] += w * (-detJ) * GNx[d][a] * 1 (P0 shape function).                  */
static void element_G(const mesh_t* M, double Ge[8][3]) {
    int dim = M->dim;
    int ijk[3] = {0, 0, 0};
    double g = 1.0 / sqrt(3.0);
    for (int a = 0; a < 8; a++)
        for (int d = 0; d < 3; d++) Ge[a][d] = 0.0;
    int ngp = 1 << dim;
    for (int q = 0; q < ngp; q++) {
        double xi[3] = {(q & 1) ? g : -g, (q & 2) ? g : -g, (q & 4) ? g : -g};
        double detJ, GNx[3][8];
        global_derivs(M, ijk, xi, &detJ, GNx);
        for (int a = 0; a < M->nen; a++)
            for (int d = 0; d < dim; d++) Ge[a][d] += 1.0 * (-detJ) * (GNx[d][a] * 1.0);
    }
}

int or_assemble(or_problem* P, int32_t prev, const double* u, const double* pres) {
    mesh_t* M = &P->M;
    int dim = M->dim, nen = M->nen, nd = nen * dim, nb = P->nb;
    if (P->np == 0 || P->nmat == 0) return fail(GG_ERR_STATE, "points/materials not set");
    if (prev && !u) return fail(GG_ERR_INVALID, "previous solution needed");
    for (int64_t p = 0; p < P->np; p++)
        if (P->mat[p] < 0 || P->mat[p] >= P->nmat) return fail(GG_ERR_INVALID, "material index");
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < P->np; p++)
        P->eta[p] = run_rheologies(P, p, prev, u, pres, &P->incr[p], &P->yielded[p]);

    free(P->Kb); free(P->kdiag); free(P->sdiag); free(P->f); free(P->h);
    P->Kb = (double*)calloc((size_t)M->nnode * nb * dim * dim, sizeof(double));
    P->kdiag = (double*)calloc(P->ndof, sizeof(double));
    P->sdiag = (double*)calloc(M->nel, sizeof(double));
    P->f = (double*)calloc(P->ndof, sizeof(double));
    P->h = (double*)calloc(M->nel, sizeof(double));
    element_G(M, P->Ge);
    double g[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) g[d] = P->force.g_hat[d] * P->force.gravity;

    /* 2^dim colours: elements of one colour share no node, so the scatter is race free */
    for (int colour = 0; colour < (1 << dim); colour++) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t e = 0; e < M->nel; e++) {
            int ijk[3];
            elem_ijk(M, e, ijk);
            int col = (ijk[0] & 1) | ((ijk[1] & 1) << 1) | ((ijk[2] & 1) << 2);
            if (col != colour) continue;
            double Ke[24][24], fe[24];
            element_K(P, e, Ke);
            int64_t nodes[8];
            for (int a = 0; a < nen; a++) nodes[a] = elem_node(M, ijk, a);
            /* force terms (BuoyancyForceTerm.cxx:468-530, ThermalBuoyancyForceTerm.cxx:216-235) */
            for (int i = 0; i < nd; i++) fe[i] = 0.0;
            for (int64_t k = P->offsets[e]; k < P->offsets[e + 1]; k++) {
                int64_t p = P->order[k];
                const double* xi = P->xi + p * dim;
                double detJ, GNx[3][8], N[8];
                global_derivs(M, ijk, xi, &detJ, GNx);
                shape(dim, xi, N);
                const gg_material* m = &P->mats[P->mat[p]];
                if (P->force.gravity != 0.0) {
                    double T = (P->T && m->alpha != 0.0) ? interp_nodal(M, ijk, xi, P->T) : 0.0;
                    double rho = m->density * (1.0 - m->alpha * T);
                    double factor = detJ * P->w[p] * 1.0 * rho;
                    for (int a = 0; a < nen; a++)
                        for (int d = 0; d < dim; d++) fe[a * dim + d] += g[d] * factor * N[a];
                }
                if (P->force.rayleigh != 0.0 && P->T) {
                    double T = interp_nodal(M, ijk, xi, P->T);
                    double factor = detJ * P->w[p] * (P->force.rayleigh * T);
                    for (int a = 0; a < nen; a++) fe[a * dim + 1] += factor * N[a];
                }
            }
            /* Dirichlet elimination into the RHS (StiffnessMatrix.cxx:2091-2117) */
            for (int i = 0; i < nd; i++) {
                int a = i / dim, c = i % dim;
                if (P->bcmask[nodes[a]] & (1u << c)) continue;
                double bcv = 0.0;
                for (int j = 0; j < nd; j++) {
                    int b = j / dim, cb = j % dim;
                    if (P->bcmask[nodes[b]] & (1u << cb))
                        bcv -= P->bcval[nodes[b] * dim + cb] * Ke[i][j];
                }
                fe[i] += bcv;
            }
            /* h: transposed RHS of g_matrix (StiffnessMatrix.cxx:2118-2143) */
            double he = 0.0;
            for (int j = 0; j < nd; j++) {
                int b = j / dim, cb = j % dim;
                if (P->bcmask[nodes[b]] & (1u << cb))
                    he -= P->bcval[nodes[b] * dim + cb] * P->Ge[b][cb];
            }
            P->h[e] = he;
            /* Ĝ_e = G_eᵀ diag(K_e)⁻¹ G_e (UzawaPreconditionerTerm.cxx:199-215), all dofs */
            double s = 0.0;
            for (int j = 0; j < nd; j++) s += P->Ge[j / dim][j % dim] * (P->Ge[j / dim][j % dim] / Ke[j][j]);
            P->sdiag[e] = s;
            /* scatter */
            for (int a = 0; a < nen; a++) {
                for (int c = 0; c < dim; c++) {
                    P->f[nodes[a] * dim + c] += fe[a * dim + c];
                    P->kdiag[nodes[a] * dim + c] += Ke[a * dim + c][a * dim + c];
                }
                for (int b = 0; b < nen; b++) {
                    int di = (b & 1) - (a & 1), dj = ((b >> 1) & 1) - ((a >> 1) & 1),
                        dk = ((b >> 2) & 1) - ((a >> 2) & 1);
                    double* blk = P->Kb + ((size_t)nodes[a] * nb + nbr_index(dim, di, dj, dk)) * dim * dim;
                    for (int c = 0; c < dim; c++)
                        for (int cb = 0; cb < dim; cb++) blk[c * dim + cb] += Ke[a * dim + c][b * dim + cb];
                }
            }
        }
    }
    /* BC rows of f are not part of the reduced system */
    for (int64_t n = 0; n < M->nnode; n++)
        for (int c = 0; c < dim; c++)
            if (P->bcmask[n] & (1u << c)) P->f[n * dim + c] = 0.0;
    P->assembled = 1;
    return GG_OK;
}

int or_dense_K(or_problem* P, double* K) {
    mesh_t* M = &P->M;
    int dim = M->dim, nb = P->nb;
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    int64_t nd = P->ndof;
    memset(K, 0, sizeof(double) * nd * nd);
    for (int64_t n = 0; n < M->nnode; n++) {
        int i = (int)(n % M->nn[0]), j = (int)((n / M->nn[0]) % M->nn[1]),
            k = (int)(n / ((int64_t)M->nn[0] * M->nn[1]));
        for (int q = 0; q < nb; q++) {
            int di = q % 3 - 1, dj = (q / 3) % 3 - 1, dk = dim == 3 ? q / 9 - 1 : 0;
            int ii = i + di, jj = j + dj, kk = k + dk;
            if (ii < 0 || jj < 0 || kk < 0 || ii >= M->nn[0] || jj >= M->nn[1] || kk >= M->nn[2]) continue;
            int64_t m = ii + (int64_t)M->nn[0] * (jj + (int64_t)M->nn[1] * kk);
            const double* blk = P->Kb + ((size_t)n * nb + q) * dim * dim;
            for (int c = 0; c < dim; c++)
                for (int cb = 0; cb < dim; cb++) K[(n * dim + c) * nd + m * dim + cb] = blk[c * dim + cb];
        }
    }
    return GG_OK;
}

/* y = K_ff x_f (BC dofs of x ignored, BC rows of y zero).                            */
static void apply_K(const or_problem* P, const double* x, double* y) {
    const mesh_t* M = &P->M;
    int dim = M->dim, nb = P->nb;
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < M->nnode; n++) {
        int i = (int)(n % M->nn[0]), j = (int)((n / M->nn[0]) % M->nn[1]),
            k = (int)(n / ((int64_t)M->nn[0] * M->nn[1]));
        double acc[3] = {0, 0, 0};
        for (int q = 0; q < nb; q++) {
            int di = q % 3 - 1, dj = (q / 3) % 3 - 1, dk = dim == 3 ? q / 9 - 1 : 0;
            int ii = i + di, jj = j + dj, kk = k + dk;
            if (ii < 0 || jj < 0 || kk < 0 || ii >= M->nn[0] || jj >= M->nn[1] || kk >= M->nn[2]) continue;
            int64_t m = ii + (int64_t)M->nn[0] * (jj + (int64_t)M->nn[1] * kk);
            const double* blk = P->Kb + ((size_t)n * nb + q) * dim * dim;
            for (int cb = 0; cb < dim; cb++) {
                if (P->bcmask[m] & (1u << cb)) continue;
                double xv = x[m * dim + cb];
                for (int c = 0; c < dim; c++) acc[c] += blk[c * dim + cb] * xv;
            }
        }
        for (int c = 0; c < dim; c++) y[n * dim + c] = (P->bcmask[n] & (1u << c)) ? 0.0 : acc[c];
    }
}

/* y = G p on free rows; q = Gᵀ u over free columns.                                 */
static void apply_G(const or_problem* P, const double* p, double* y) {
    const mesh_t* M = &P->M;
    int dim = M->dim;
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < M->nnode; n++) {
        int idx[3] = {(int)(n % M->nn[0]), (int)((n / M->nn[0]) % M->nn[1]),
                      (int)(n / ((int64_t)M->nn[0] * M->nn[1]))};
        double acc[3] = {0, 0, 0};
        for (int a = 0; a < M->nen; a++) {
            /* node n is local node a of the element whose lower corner is n - offset(a) */
            int e3[3] = {idx[0] - (a & 1), idx[1] - ((a >> 1) & 1), idx[2] - ((a >> 2) & 1)};
            int ok = 1;
            for (int d = 0; d < 3; d++)
                if (e3[d] < 0 || e3[d] >= M->n[d]) ok = 0;
            if (!ok) continue;
            int64_t e = e3[0] + (int64_t)M->n[0] * (e3[1] + (int64_t)M->n[1] * e3[2]);
            for (int c = 0; c < dim; c++) acc[c] += P->Ge[a][c] * p[e];
        }
        for (int c = 0; c < dim; c++) y[n * dim + c] = (P->bcmask[n] & (1u << c)) ? 0.0 : acc[c];
    }
}

static void apply_GT(const or_problem* P, const double* u, double* q) {
    const mesh_t* M = &P->M;
    int dim = M->dim;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < M->nel; e++) {
        int ijk[3];
        elem_ijk(M, e, ijk);
        double s = 0.0;
        for (int a = 0; a < M->nen; a++) {
            int64_t n = elem_node(M, ijk, a);
            for (int c = 0; c < dim; c++)
                if (!(P->bcmask[n] & (1u << c))) s += P->Ge[a][c] * u[n * dim + c];
        }
        q[e] = s;
    }
}

int or_apply_K(or_problem* P, const double* x, double* y) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    apply_K(P, x, y);
    return GG_OK;
}
int or_apply_G(or_problem* P, const double* p, double* y) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    apply_G(P, p, y);
    return GG_OK;
}
int or_apply_GT(or_problem* P, const double* u, double* q) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    apply_GT(P, u, q);
    return GG_OK;
}
int or_get_rhs(or_problem* P, double* f, double* h) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    if (f) memcpy(f, P->f, sizeof(double) * P->ndof);
    if (h) memcpy(h, P->h, sizeof(double) * P->M.nel);
    return GG_OK;
}
int or_get_diagonals(or_problem* P, double* kdiag, double* sdiag) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    if (kdiag) memcpy(kdiag, P->kdiag, sizeof(double) * P->ndof);
    if (sdiag) memcpy(sdiag, P->sdiag, sizeof(double) * P->M.nel);
    return GG_OK;
}
int or_point_viscosity(or_problem* P, double* eta) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    memcpy(eta, P->eta, sizeof(double) * P->np);
    return GG_OK;
}
int or_point_yield(or_problem* P, double* incr, uint8_t* yielded) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    if (incr) memcpy(incr, P->incr, sizeof(double) * P->np);
    if (yielded) memcpy(yielded, P->yielded, P->np);
    return GG_OK;
}

/* Monomials ξ^a η^b ζ^c of the element moments: every exponent ≤ 2, with the
 * products that Bᵀ D B of a Q1 element can produce.                                 */
int or_monomials(int32_t dim, int32_t* ex) {
    int n = 0;
    if (dim == 2) {
        static const int t[6][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {0, 2}, {1, 1}};
        for (int i = 0; i < 6; i++) {
            if (ex) { ex[3 * i] = t[i][0]; ex[3 * i + 1] = t[i][1]; ex[3 * i + 2] = 0; }
        }
        return 6;
    }
    for (int c = 0; c < 3; c++)
        for (int b = 0; b < 3; b++)
            for (int a = 0; a < 3; a++) {
                int twos = (a == 2) + (b == 2) + (c == 2);
                int zeros = (a == 0) + (b == 0) + (c == 0);
                if (zeros == 0 && twos >= 2) continue;
                if (ex) { ex[3 * n] = a; ex[3 * n + 1] = b; ex[3 * n + 2] = c; }
                n++;
            }
    return n;
}

int or_moments(or_problem* P, double* mom, int32_t* nmom) {
    mesh_t* M = &P->M;
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    int32_t ex[27 * 3];
    int nm = or_monomials(M->dim, ex);
    if (nmom) *nmom = nm;
    if (!mom) return GG_OK;
    double h[3];
    for (int d = 0; d < 3; d++) h[d] = d < M->dim ? (M->max[d] - M->min[d]) / M->n[d] : 2.0;
    double detJ = h[0] * h[1] * h[2] / 8.0;
    if (M->dim == 2) detJ = h[0] * h[1] / 4.0;
    for (int64_t e = 0; e < M->nel; e++) {
        double acc[27] = {0};
        for (int64_t k = P->offsets[e]; k < P->offsets[e + 1]; k++) {
            int64_t p = P->order[k];
            const double* xi = P->xi + p * M->dim;
            double c = P->w[p] * detJ * P->eta[p];
            for (int m = 0; m < nm; m++) {
                double v = c;
                for (int d = 0; d < M->dim; d++)
                    for (int q = 0; q < ex[3 * m + d]; q++) v *= xi[d];
                acc[m] += v;
            }
        }
        for (int m = 0; m < nm; m++) mom[(int64_t)m * M->nel + e] = acc[m];
    }
    return GG_OK;
}

/* ------------------------------------------------------------ solvers --- */
/* Sum of 64 fixed chunks, each summed in index order, then the chunks in order: the
 * same bits for any thread count and on every run (an OpenMP reduction clause combines
 * the threads' partial sums in arrival order).                                       */
static double dot(int64_t n, const double* a, const double* b) {
    enum { kChunks = 64 };
    double part[kChunks];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < kChunks; c++) {
        const int64_t lo = n * c / kChunks, hi = n * (c + 1) / kChunks;
        double s = 0.0;
        for (int64_t i = lo; i < hi; i++) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < kChunks; c++) s += part[c];
    return s;
}

/* PETSc KSPSolve_CG with PCJACOBI, zero initial guess, KSP_NORM_PRECONDITIONED and
 * KSPConvergedDefault (rnorm ≤ max(rtol·rnorm0, 1e-50)).  Returns iterations, or
 * -1 when maxit was reached.                                                        */
static int jacobi_cg(const or_problem* P, const double* b, double* x, double rtol, int maxit,
                     double* work) {
    int64_t nd = P->ndof;
    double *r = work, *z = work + nd, *p = work + 2 * nd, *Ap = work + 3 * nd;
    const double* dg = P->kdiag;
    const uint8_t* bm = P->bcmask;
    int dim = P->M.dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nd; i++) {
        int fixed = bm[i / dim] & (1u << (i % dim));
        x[i] = 0.0;
        r[i] = fixed ? 0.0 : b[i];
        z[i] = fixed ? 0.0 : r[i] / dg[i];
    }
    double rnorm0 = sqrt(dot(nd, z, z));
    double ttol = rtol * rnorm0;
    if (ttol < 1e-50) ttol = 1e-50;
    if (rnorm0 <= ttol) return 0;
    double beta = dot(nd, z, r), betaold = 0.0;
    int it = 0;
    while (it < maxit) {
        if (it == 0) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < nd; i++) p[i] = z[i];
        } else {
            double bb = beta / betaold;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < nd; i++) p[i] = z[i] + bb * p[i];
        }
        betaold = beta;
        apply_K(P, p, Ap);
        double dpi = dot(nd, p, Ap);
        double a = beta / dpi;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < nd; i++) {
            int fixed = bm[i / dim] & (1u << (i % dim));
            x[i] += a * p[i];
            r[i] -= a * Ap[i];
            z[i] = fixed ? 0.0 : r[i] / dg[i];
        }
        double dp = sqrt(dot(nd, z, z));
        it++;
        if (dp <= ttol) return it;
        if (!isfinite(dp)) return -2;
        beta = dot(nd, z, r);
    }
    return -1;
}

int or_inner_solve(or_problem* P, const double* b, double* x, double rtol, int32_t maxit) {
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    double* work = (double*)malloc(sizeof(double) * 4 * P->ndof);
    int it = jacobi_cg(P, b, x, rtol, maxit, work);
    free(work);
    return it;
}

/* _Stokes_SLE_UzawaSolver_Solve (Stokes_SLE_UzawaSolver.cxx:393-938) with the inner
 * velocity KSP = Jacobi CG.  u and p are nodal / element; BC dofs of u get BC values. */
int or_uzawa(or_problem* P, const gg_uzawa_params* prm, double* u, double* p, gg_uzawa_stats* st) {
    mesh_t* M = &P->M;
    if (!P->assembled) return fail(GG_ERR_STATE, "not assembled");
    int64_t nd = P->ndof, ne = M->nel;
    int dim = M->dim;
    double* work = (double*)malloc(sizeof(double) * 4 * nd);
    double* vstar = (double*)calloc(nd, sizeof(double));
    double* ftmp = (double*)calloc(nd, sizeof(double));
    double* uu = (double*)calloc(nd, sizeof(double));
    double* qtmp = (double*)calloc(ne, sizeof(double));
    double* r = (double*)calloc(ne, sizeof(double));
    double* s = (double*)calloc(ne, sizeof(double));
    double* q = (double*)calloc(ne, sizeof(double));
    int rc = GG_OK;
    gg_uzawa_stats S;
    memset(&S, 0, sizeof S);
    int64_t nfree = 0;
    for (int64_t n = 0; n < M->nnode; n++)
        for (int c = 0; c < dim; c++) nfree += !(P->bcmask[n] & (1u << c));
    double scaleq = sqrt((double)ne);
    int maxit = prm->inner_max_iterations > 0 ? prm->inner_max_iterations : 10000;
    if (prm->reuse_pressure && p)
        memcpy(q, p, sizeof(double) * ne);
    double fnorm = sqrt(dot(nd, P->f, P->f));
    if (fnorm / sqrt((double)nfree) <= 1e-99) { rc = fail(GG_ERR_ZERO_FORCE, "zero force vector"); goto done; }
    /* STEP 1: Fhat - h with inner rtol = tolerance (:553-565) */
    {
        int it = jacobi_cg(P, P->f, vstar, prm->tolerance, maxit, work);
        if (it < 0) { rc = fail(GG_ERR_NOT_CONVERGED, "inner solve"); goto done; }
        S.inner_iterations += it; S.inner_solves++;
    }
    apply_GT(P, vstar, qtmp);
    for (int64_t e = 0; e < ne; e++) qtmp[e] -= P->h[e];
    double inner_rtol = prm->inner_rtol_factor * prm->tolerance;
    double rhs_scale = sqrt(dot(ne, qtmp, qtmp)) / scaleq;
    if (!isfinite(rhs_scale)) { rc = fail(GG_ERR_NONFINITE, "uzawaRhsScale"); goto done; }
    /* STEP 3: u0 = K⁻¹(f - G q0), r = Gᵀu0 - h (:616-659) */
    apply_G(P, q, ftmp);
    for (int64_t i = 0; i < nd; i++) ftmp[i] = P->f[i] - ftmp[i];
    {
        int it = jacobi_cg(P, ftmp, uu, inner_rtol, maxit, work);
        if (it < 0) { rc = fail(GG_ERR_NOT_CONVERGED, "inner solve"); goto done; }
        S.inner_iterations += it; S.inner_solves++;
    }
    apply_GT(P, uu, r);
    for (int64_t e = 0; e < ne; e++) r[e] -= P->h[e];
    double zr_prev = 1.0, absres = 0.0, relres = 0.0;
    int k = 0;
    /* A velocity that already meets the constraint to rounding (the boundary velocities
     * admit an exactly representable flow and the inner solve found it): r0 is rounding
     * noise whose constant-pressure component the Schur CG cannot remove, so the
     * reference's loop (:664-837) would iterate on noise until alpha breaks down.  Here
     * the solve ends at once with q0 (no outer iteration, relative residual 0).          */
    {
        double gmax = 0.0;
        for (int a = 0; a < M->nen; a++)
            for (int c = 0; c < dim; c++) gmax = fmax(gmax, fabs(P->Ge[a][c]));
        double floor_r = 64.0 * DBL_EPSILON * (gmax * sqrt((double)M->nen) * sqrt(dot(nd, uu, uu)) + sqrt(dot(ne, P->h, P->h)));
        double r0 = sqrt(dot(ne, r, r));
        if (r0 <= floor_r) {
            S.abs_residual = r0 / scaleq;
            S.rel_residual = 0.0;
            goto summary;
        }
    }
    for (;;) {
        /* 4.1 z = Ĝ⁻¹ r (Ĝ diagonal for P0) */
        for (int64_t e = 0; e < ne; e++) qtmp[e] = prm->use_preconditioner ? r[e] / P->sdiag[e] : r[e];
        double zr = dot(ne, qtmp, r);
        if (k == 0)
            memcpy(s, qtmp, sizeof(double) * ne);
        else {
            double beta = zr / zr_prev;
            for (int64_t e = 0; e < ne; e++) s[e] = beta * s[e] + qtmp[e];
        }
        apply_G(P, s, ftmp);
        int it = jacobi_cg(P, ftmp, vstar, inner_rtol, maxit, work);
        if (it < 0) { rc = fail(GG_ERR_NOT_CONVERGED, "inner solve"); goto done; }
        S.inner_iterations += it; S.inner_solves++;
        apply_GT(P, vstar, qtmp);
        double sq = dot(ne, s, qtmp);
        double alpha = zr / sq;
        if (!isfinite(zr) || !isfinite(sq) || !isfinite(alpha)) { rc = fail(GG_ERR_NONFINITE, "alpha"); goto done; }
        for (int64_t e = 0; e < ne; e++) { q[e] += alpha * s[e]; r[e] -= alpha * qtmp[e]; }
        for (int64_t i = 0; i < nd; i++) uu[i] -= alpha * vstar[i];
        zr_prev = zr;
        absres = sqrt(dot(ne, r, r)) / scaleq;
        relres = absres / rhs_scale;
        if (!isfinite(absres)) { rc = fail(GG_ERR_NONFINITE, "absResidual"); goto done; }
        if (!(k < prm->max_iterations)) { rc = fail(GG_ERR_NOT_CONVERGED, "Uzawa max iterations"); k++; break; }
        k++;
        double chosen = prm->use_absolute_tolerance ? absres : relres;
        if (!((chosen > prm->tolerance) || (k < prm->min_iterations))) break;
    }
    S.outer_iterations = k;
    S.rel_residual = relres;
    S.abs_residual = absres;
summary:
    /* summary norms (:844-877) */
    {
        apply_GT(P, uu, qtmp);
        double un = sqrt(dot(nd, uu, uu));
        S.div_u = sqrt(dot(ne, qtmp, qtmp)) / un;
        apply_G(P, q, vstar);
        apply_K(P, uu, ftmp);
        for (int64_t i = 0; i < nd; i++) ftmp[i] = P->f[i] - (ftmp[i] + vstar[i]);
        S.momentum_residual = sqrt(dot(nd, ftmp, ftmp)) / fnorm;
    }
done:
    for (int64_t n = 0; n < M->nnode; n++)
        for (int c = 0; c < dim; c++)
            u[n * dim + c] = (P->bcmask[n] & (1u << c)) ? P->bcval[n * dim + c] : uu[n * dim + c];
    if (p) memcpy(p, q, sizeof(double) * ne);
    if (st) *st = S;
    free(work); free(vstar); free(ftmp); free(uu); free(qtmp); free(r); free(s); free(q);
    return rc;
}

/* SystemLinearEquations_NonLinearExecute (SystemLinearEquations.cxx:735-920): first
 * solve without yielding, then re-assemble from the last solution and re-solve until
 * ‖u_k − u_{k−1}‖/‖u_k‖ < tolerance; Uzawa restarts from the last pressure.          */
int or_picard(or_problem* P, const gg_picard_params* pic, const gg_uzawa_params* prm, double* u,
              double* p, gg_picard_stats* st) {
    mesh_t* M = &P->M;
    int64_t nd = P->ndof;
    int dim = M->dim;
    gg_uzawa_params up = *prm;
    gg_uzawa_stats us;
    gg_picard_stats S;
    memset(&S, 0, sizeof S);
    double* prev = (double*)malloc(sizeof(double) * nd);
    memset(p, 0, sizeof(double) * M->nel);
    up.reuse_pressure = 1;
    int rc = or_assemble(P, 0, NULL, NULL);
    if (rc == GG_OK) rc = or_uzawa(P, &up, u, p, &us);
    if (rc != GG_OK) goto done;
    S.outer_iterations += us.outer_iterations;
    S.inner_iterations += us.inner_iterations;
    S.iterations = 1;
    for (int it = 1; it < pic->max_iterations; it++) {
        memcpy(prev, u, sizeof(double) * nd);
        rc = or_assemble(P, 1, u, p);
        if (rc == GG_OK) rc = or_uzawa(P, &up, u, p, &us);
        if (rc != GG_OK) goto done;
        S.outer_iterations += us.outer_iterations;
        S.inner_iterations += us.inner_iterations;
        double dn = 0.0, cn = 0.0;
        for (int64_t n = 0; n < M->nnode; n++)
            for (int c = 0; c < dim; c++) {
                if (P->bcmask[n] & (1u << c)) continue; /* solution vector = free dofs */
                double d = prev[n * dim + c] - u[n * dim + c];
                dn += d * d;
                cn += u[n * dim + c] * u[n * dim + c];
            }
        S.residual = sqrt(dn) / sqrt(cn);
        S.iterations = it + 1;
        if (S.residual < pic->tolerance && it >= pic->min_iterations) { S.converged = 1; break; }
    }
done:
    if (st) *st = S;
    free(prev);
    return rc;
}

/* ------------------------------------------------------------ advection --- */
/* _SwarmAdvector_TimeDeriv via FieldVariable_InterpolateValueAt (FeVariable.cxx:703-730,
 * :904-950, :1531-1570): search, Newton ξ, Σ N_a u_a.  Returns 0 outside the mesh.   */
static int velocity_at(const or_problem* P, const double* sep, const double* x, const double* u,
                       double* v) {
    const mesh_t* M = &P->M;
    int64_t e;
    if (!search_element(M, sep, x, &e)) return 0;
    int ijk[3];
    double xi[3], N[8];
    elem_ijk(M, e, ijk);
    newton_xi(M, ijk, x, xi);
    shape(M->dim, xi, N);
    for (int c = 0; c < M->dim; c++) v[c] = 0.0;
    for (int a = 0; a < M->nen; a++) {
        int64_t n = elem_node(M, ijk, a);
        for (int c = 0; c < M->dim; c++) v[c] += u[n * M->dim + c] * N[a];
    }
    for (int c = 0; c < M->dim; c++)
        if (isinf(v[c])) return 0;
    return 1;
}

/* TimeIntegrand_SecondOrder (TimeIntegrand.cxx:265-335) with allowFallbackToFirstOrder
 * (_TimeIntegrand_RewindToStartAndApplyFirstOrderUpdate :457-483); order 1 = Euler.  */
int or_advect(or_problem* P, double dt, int32_t order, const double* u, double* out) {
    mesh_t* M = &P->M;
    int dim = M->dim;
    double sep[3];
    mesh_sep(M, sep);
    int bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
    for (int64_t p = 0; p < P->np; p++) {
        double x0[3], x[3], k1[3], k2[3];
        for (int c = 0; c < dim; c++) x0[c] = P->coords[p * dim + c];
        if (!velocity_at(P, sep, x0, u, k1)) { bad++; continue; }
        if (order == 1) {
            for (int c = 0; c < dim; c++) x[c] = x0[c] + dt * k1[c];
        } else {
            for (int c = 0; c < dim; c++) x[c] = x0[c] + 0.5 * dt * k1[c];
            if (velocity_at(P, sep, x, u, k2)) {
                for (int c = 0; c < dim; c++) x[c] = x0[c] + dt * k2[c];
            } else {
                for (int c = 0; c < dim; c++) x[c] = x0[c] + dt * k1[c];
            }
        }
        for (int c = 0; c < dim; c++) out[p * dim + c] = x[c];
    }
    if (bad) return fail(GG_ERR_OUT_OF_DOMAIN, "point outside the mesh at stage 1");
    return GG_OK;
}

/* Stokes_SLE_UpdateDt (UpdateDt.cxx:53-84): 0.5 * minimum separation / max |v|.     */
int or_courant_dt(or_problem* P, const double* u, double* dt) {
    mesh_t* M = &P->M;
    double minsep = 1e300, vmax = 0.0;
    for (int d = 0; d < M->dim; d++) {
        double s = (M->max[d] - M->min[d]) / M->n[d];
        if (s < minsep) minsep = s;
    }
    for (int64_t n = 0; n < M->nnode; n++) {
        double v2 = 0.0;
        for (int c = 0; c < M->dim; c++) v2 += u[n * M->dim + c] * u[n * M->dim + c];
        if (v2 > vmax) vmax = v2;
    }
    *dt = 0.5 * minsep / sqrt(vmax);
    return GG_OK;
}
