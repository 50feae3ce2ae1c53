/*
 * stokes_gpu_plugin.c -- the StGermain side of the Stokes_SLE_UzawaSolverGPU plugin (see
 * the header).  Inside a Gale tree it builds against the real StGermain, StgDomain, StgFEM,
 * PICellerator, Underworld and PETSc headers; tests/test_c_plugin.py builds it against the
 * declaration stub in tests/c/stub and drives a solve through the function pointer the
 * stub's component register hands back.
 *
 * The solve reads what _Stokes_SLE_UzawaSolver_Solve (Stokes_SLE_UzawaSolver.cxx:393-938)
 * reads from the Stokes SLE and its components -- the velocity FeVariable's mesh and
 * boundary conditions, the material points, the materials and their rheologies, the body
 * force terms -- into the flat view of stokes_gpu_host.h, runs it through the C ABI, and
 * writes u and p back into the velocity / pressure FeVariables and their SolutionVectors,
 * as the reference's solve leaves them.  A non-zero status ends in Journal_Firewall, the
 * reference's failure mode.
 */
#include <stdlib.h>
#include <string.h>

#include "stokes_gpu_plugin.h"

const Type Underworld_StokesGPU_Type = "Underworld_StokesGPU";
const Type Stokes_SLE_UzawaSolverGPU_Type = "Stokes_SLE_UzawaSolverGPU";

/* ---- registration (Plugin.cxx:55,97; Multigrid.cxx:139-143) ------------------------- */
void* _Underworld_StokesGPU_DefaultNew(Name name) {
    SizeT _sizeOfSelf = sizeof(Codelet);
    Type type = Underworld_StokesGPU_Type;
    Stg_Class_DeleteFunction* _delete = _Codelet_Delete;
    Stg_Class_PrintFunction* _print = _Codelet_Print;
    Stg_Class_CopyFunction* _copy = _Codelet_Copy;
    Stg_Component_DefaultConstructorFunction* _defaultConstructor = _Underworld_StokesGPU_DefaultNew;
    Stg_Component_AssignFromXMLFunction* _construct = _Codelet_AssignFromXML;
    Stg_Component_BuildFunction* _build = _Codelet_Build;
    Stg_Component_InitialiseFunction* _initialise = _Codelet_Initialise;
    Stg_Component_ExecuteFunction* _execute = _Codelet_Execute;
    Stg_Component_DestroyFunction* _destroy = _Codelet_Destroy;
    AllocationType nameAllocationType = NON_GLOBAL;
    return _Codelet_New(CODELET_PASSARGS);
}

Index Underworld_StokesGPU_Register(PluginsManager* pluginsManager) {
    /* the solver type an input deck names, as StokesFlow/src/Init.cxx:64-67 adds its own */
    Stg_ComponentRegister_Add(Stg_ComponentRegister_Get_ComponentRegister(), Stokes_SLE_UzawaSolverGPU_Type,
                              (Name) "0", _Stokes_SLE_UzawaSolverGPU_DefaultNew);
    return PluginsManager_Submit(pluginsManager, Underworld_StokesGPU_Type, (Name) "0",
                                 _Underworld_StokesGPU_DefaultNew);
}

/* ---- the component ------------------------------------------------------------------ */
void* _Stokes_SLE_UzawaSolverGPU_DefaultNew(Name name) {
    SizeT _sizeOfSelf = sizeof(Stokes_SLE_UzawaSolverGPU);
    Type type = Stokes_SLE_UzawaSolverGPU_Type;
    Stg_Class_DeleteFunction* _delete = _SLE_Solver_Delete;
    Stg_Class_PrintFunction* _print = _SLE_Solver_Print;
    Stg_Class_CopyFunction* _copy = NULL;
    Stg_Component_DefaultConstructorFunction* _defaultConstructor = _Stokes_SLE_UzawaSolverGPU_DefaultNew;
    Stg_Component_AssignFromXMLFunction* _construct = _Stokes_SLE_UzawaSolverGPU_AssignFromXML;
    Stg_Component_BuildFunction* _build = NULL;
    Stg_Component_InitialiseFunction* _initialise = NULL;
    Stg_Component_ExecuteFunction* _execute = NULL;
    Stg_Component_DestroyFunction* _destroy = _Stokes_SLE_UzawaSolverGPU_Destroy;
    SLE_Solver_SolverSetupFunction* _solverSetup = _Stokes_SLE_UzawaSolverGPU_SolverSetup;
    SLE_Solver_SolveFunction* _solve = _Stokes_SLE_UzawaSolverGPU_Solve;
    SLE_Solver_GetResidualFunc* _getResidual = NULL;
    AllocationType nameAllocationType = NON_GLOBAL;
    Stokes_SLE_UzawaSolverGPU* self = (Stokes_SLE_UzawaSolverGPU*)_SLE_Solver_New(SLE_SOLVER_PASSARGS);
    self->handle = NULL;
    self->params = StokesGPU_DefaultParams();
    return self;
}

static int inner_kind(const char* s) {
    if (!strcmp(s, "mg")) return GG_INNER_MG_CG;
    if (!strcmp(s, "learned")) return GG_INNER_LEARNED_CG;
    if (!strcmp(s, "learned_jacobi")) return GG_INNER_LEARNED_JACOBI_CG;
    return GG_INNER_JACOBI_CG;
}

/* The keys of _Stokes_SLE_UzawaSolver_AssignFromXML (Stokes_SLE_UzawaSolver.cxx:241-264)
 * with its defaults, plus the GPU path's own: innerSolver (jacobi | mg | learned),
 * precision (fp64 | mixed), innerRtolFactor, innerMaxIterations, smoothingDegree. */
void _Stokes_SLE_UzawaSolverGPU_AssignFromXML(void* solver, Stg_ComponentFactory* cf, void* data) {
    Stokes_SLE_UzawaSolverGPU* self = (Stokes_SLE_UzawaSolverGPU*)solver;
    gg_uzawa_params* p = &self->params;
    self->context = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "Context",
                                                        FiniteElementContext, False, data);
    if (!self->context)
        self->context = (FiniteElementContext*)LiveComponentRegister_Get(cf->LCRegister, (Name) "context");
    self->tolerance = Stg_ComponentFactory_GetDouble(cf, self->name, (Dictionary_Entry_Key) "tolerance", 1.0e-5);
    self->maxUzawaIterations =
        Stg_ComponentFactory_GetUnsignedInt(cf, self->name, (Dictionary_Entry_Key) "maxIterations", 1000);
    self->minUzawaIterations =
        Stg_ComponentFactory_GetUnsignedInt(cf, self->name, (Dictionary_Entry_Key) "minIterations", 1);
    self->useAbsoluteTolerance =
        Stg_ComponentFactory_GetBool(cf, self->name, (Dictionary_Entry_Key) "useAbsoluteTolerance", False);
    self->monitor = Stg_ComponentFactory_GetBool(cf, self->name, (Dictionary_Entry_Key) "monitor", False);
    self->preconditioner = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "Preconditioner",
                                                               StiffnessMatrix, False, data);
    p->tolerance = self->tolerance;
    p->max_iterations = (int32_t)self->maxUzawaIterations;
    p->min_iterations = (int32_t)self->minUzawaIterations;
    p->use_absolute_tolerance = self->useAbsoluteTolerance ? 1 : 0;
    p->use_preconditioner = self->preconditioner ? 1 : 0;
    p->inner = inner_kind(Stg_ComponentFactory_GetString(cf, self->name, (Dictionary_Entry_Key) "innerSolver", "jacobi"));
    p->precision = strcmp(Stg_ComponentFactory_GetString(cf, self->name, (Dictionary_Entry_Key) "precision", "fp64"),
                          "mixed")
                       ? GG_PRECISION_FP64
                       : GG_PRECISION_MIXED;
    p->inner_rtol_factor =
        Stg_ComponentFactory_GetDouble(cf, self->name, (Dictionary_Entry_Key) "innerRtolFactor", 0.1);
    p->inner_max_iterations =
        (int32_t)Stg_ComponentFactory_GetUnsignedInt(cf, self->name, (Dictionary_Entry_Key) "innerMaxIterations", 10000);
    p->smoothing_degree =
        (int32_t)Stg_ComponentFactory_GetUnsignedInt(cf, self->name, (Dictionary_Entry_Key) "smoothingDegree", 0);
    p->recycle_directions = p->precision == GG_PRECISION_MIXED;
    self->materialSwarm = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "MaterialPointsSwarm",
                                                              MaterialPointsSwarm, True, data);
    self->buoyancyForceTerm = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "BuoyancyForceTerm",
                                                                  BuoyancyForceTerm, False, data);
    self->thermalBuoyancyForceTerm = Stg_ComponentFactory_ConstructByKey(
        cf, self->name, (Dictionary_Entry_Key) "ThermalBuoyancyForceTerm", ThermalBuoyancyForceTerm, False, data);
    self->temperatureField = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "TemperatureField",
                                                                 FeVariable, False, data);
    self->strainWeakening = Stg_ComponentFactory_ConstructByKey(cf, self->name, (Dictionary_Entry_Key) "StrainWeakening",
                                                                StrainWeakening, False, data);
    self->materials_Register = self->context ? self->context->materials_Register : NULL;
    self->errorStream = Journal_Register(Error_Type, (Name)Stokes_SLE_UzawaSolverGPU_Type);
}

/* The reference builds its KSP objects here (:308-326); the device state is created by
 * the first solve and kept in the handle. */
void _Stokes_SLE_UzawaSolverGPU_SolverSetup(void* solver, void* stokesSLE) {
    (void)solver;
    (void)stokesSLE;
}

void _Stokes_SLE_UzawaSolverGPU_Destroy(void* solver, void* data) {
    Stokes_SLE_UzawaSolverGPU* self = (Stokes_SLE_UzawaSolverGPU*)solver;
    (void)data;
    if (self->handle) gg_destroy(self->handle);
    self->handle = NULL;
}

/* ---- reading the SLE into the view ---------------------------------------------------- */
static void collect_mesh(FeMesh* mesh, gg_mesh_desc* md) {
    Grid** eg = Mesh_GetExtension(mesh, Grid**, "elementGrid");
    memset(md, 0, sizeof *md);
    md->dim = (int32_t)Mesh_GetDimSize(mesh);
    Mesh_GetGlobalCoordRange(mesh, md->min, md->max);
    for (int d = 0; d < 3; d++) md->elements[d] = d < md->dim ? (int32_t)(*eg)->sizes[d] : 1;
}

/* VariableCondition values as FeVariable_IsBC / FeVariable_GetValueAtNode report them,
 * condition functions included (they were applied at the nodes). */
static void collect_bcs(FeVariable* vel, int64_t nnode, int dim, uint8_t* fixed, double* values) {
    double v[3];
    for (int64_t n = 0; n < nnode; n++) {
        FeVariable_GetValueAtNode(vel, (Node_DomainIndex)n, v);
        fixed[n] = 0;
        for (int c = 0; c < dim; c++) {
            values[n * dim + c] = 0.0;
            if (FeVariable_IsBC(vel, (Node_DomainIndex)n, (Dof_Index)c)) {
                fixed[n] |= (uint8_t)(1u << c);
                values[n * dim + c] = v[c];
            }
        }
    }
}

static void yield_common(const VonMises* vm, gg_rheology* r) {
    r->cohesion = vm->cohesion;
    r->cohesion_after_softening = vm->cohesionAfterSoftening;
    r->minimum_viscosity = vm->minVisc;
    r->strain_weakening = vm->strainWeakening ? 1 : 0;
}

/* One gg_rheology per Rheology of the material's register, in register order
 * (Rheology_Register_RunRheologies, Rheology_Register.cxx:70-86); returns 0 or the
 * name of a type this path does not evaluate. */
static const char* collect_rheology(const Rheology* rh, gg_rheology* r) {
    memset(r, 0, sizeof *r);
    if (!strcmp(rh->type, "MaterialViscosity")) {
        r->kind = GG_RHEO_MATERIAL_VISCOSITY;
        r->eta0 = ((const MaterialViscosity*)rh)->eta0;
    } else if (!strcmp(rh->type, "Arrhenius")) {
        const Arrhenius* a = (const Arrhenius*)rh;
        r->kind = GG_RHEO_ARRHENIUS;
        r->eta0 = a->eta0;
        r->activation_energy = a->activationEnergy;
        r->activation_volume = a->activationVolume;
        r->reference_temp = a->referenceTemp;
    } else if (!strcmp(rh->type, "FrankKamenetskii")) {
        const FrankKamenetskii* fk = (const FrankKamenetskii*)rh;
        r->kind = GG_RHEO_FRANK_KAMENETSKII;
        r->eta0 = fk->eta0;
        r->theta = fk->theta;
    } else if (!strcmp(rh->type, "VonMises")) {
        const VonMises* vm = (const VonMises*)rh;
        r->kind = GG_RHEO_VON_MISES;
        yield_common(vm, r);
        r->strain_rate_softening = vm->strainRateSoftening ? 1 : 0;
    } else if (!strcmp(rh->type, "DruckerPrager")) {
        const DruckerPrager* dp = (const DruckerPrager*)rh;
        r->kind = GG_RHEO_DRUCKER_PRAGER;
        yield_common((const VonMises*)dp, r);
        r->friction_coefficient = dp->frictionCoefficient;
        r->friction_coefficient_after_softening = dp->frictionCoefficientAfterSoftening;
        r->minimum_yield_stress = dp->minimumYieldStress;
        r->minimum_viscosity = dp->minimumViscosity;
        r->max_strain_rate = dp->maxStrainRate;
        r->boundary_cohesion = dp->boundaryCohesion;
        r->boundary_cohesion_after_softening = dp->boundaryCohesionAfterSoftening;
        r->boundary_friction_coefficient = dp->boundaryFrictionCoefficient;
        r->boundary_friction_coefficient_after_softening = dp->boundaryFrictionCoefficientAfterSoftening;
        r->boundary_walls = (dp->boundaryLeft ? 1 : 0) | (dp->boundaryRight ? 2 : 0) | (dp->boundaryBottom ? 4 : 0) |
                            (dp->boundaryTop ? 8 : 0) | (dp->boundaryBack ? 16 : 0) | (dp->boundaryFront ? 32 : 0);
        r->hydrostatic_term = dp->hydrostaticTerm ? 1 : 0;
    } else if (!strcmp(rh->type, "Byerlee")) {
        const Byerlee* by = (const Byerlee*)rh;
        r->kind = GG_RHEO_BYERLEE;
        yield_common((const VonMises*)by, r);
        r->depth_coefficient = by->depthCoefficient;
    } else {
        return rh->type;
    }
    return NULL;
}

static const char* collect_materials(Stokes_SLE_UzawaSolverGPU* self, gale_stokes_view* v) {
    Materials_Register* mr = self->materials_Register;
    const Index nm = mr ? Materials_Register_GetCount(mr) : 0;
    if (nm < 1 || nm > GG_MAX_MATERIALS) return "material count";
    v->n_materials = (int32_t)nm;
    for (Index i = 0; i < nm; i++) {
        RheologyMaterial* rm = (RheologyMaterial*)Materials_Register_GetByIndex(mr, i);
        gg_material* m = &v->materials[i];
        memset(m, 0, sizeof *m);
        const Index nr = rm->rheology_Register ? Rheology_Register_GetCount(rm->rheology_Register) : 0;
        if (nr > GG_MAX_RHEOLOGIES) return "rheology count";
        m->n_rheologies = (int32_t)nr;
        for (Index k = 0; k < nr; k++) {
            const char* bad = collect_rheology(Rheology_Register_GetByIndex(rm->rheology_Register, k), &m->rheology[k]);
            if (bad) return bad;
            if (m->rheology[k].strain_weakening && self->strainWeakening) {
                m->has_strain_weakening = 1;
                m->strain_weakening.initial_softening_strain = self->strainWeakening->initialSofteningStrain;
                m->strain_weakening.final_softening_strain = self->strainWeakening->finalSofteningStrain;
                m->strain_weakening.healing_rate = self->strainWeakening->healingRate;
            }
        }
        if (self->buoyancyForceTerm) {  /* BuoyancyForceTerm.cxx: the material extension */
            BuoyancyForceTerm_MaterialExt* ext = (BuoyancyForceTerm_MaterialExt*)ExtensionManager_Get(
                rm->extensionMgr, rm, self->buoyancyForceTerm->materialExtHandle);
            m->density = ext->density;
            m->alpha = ext->alpha;
        }
    }
    return NULL;
}

void _Stokes_SLE_UzawaSolverGPU_Solve(void* solver, void* stokesSLE) {
    Stokes_SLE_UzawaSolverGPU* self = (Stokes_SLE_UzawaSolverGPU*)solver;
    Stokes_SLE* sle = (Stokes_SLE*)stokesSLE;
    FeVariable* vel = sle->uSolnVec->feVariable;
    FeVariable* pres = sle->pSolnVec->feVariable;
    gale_stokes_view v;
    memset(&v, 0, sizeof v);
    collect_mesh(vel->feMesh, &v.mesh);
    const int dim = v.mesh.dim;
    const int64_t nnode = (int64_t)Mesh_GetDomainSize(vel->feMesh, MT_VERTEX);
    int64_t nel = 1;
    for (int d = 0; d < dim; d++) nel *= v.mesh.elements[d];

    uint8_t* fixed = (uint8_t*)malloc((size_t)nnode);
    double* bcv = (double*)malloc(sizeof(double) * (size_t)(nnode * dim));
    collect_bcs(vel, nnode, dim, fixed, bcv);
    v.bc_fixed = fixed;
    v.bc_values = bcv;

    const char* bad = collect_materials(self, &v);
    Journal_Firewall(bad == NULL, self->errorStream, "Error in func '%s' for %s '%s': unsupported %s\n", __func__,
                     self->type, self->name, bad ? bad : "");

    if (self->buoyancyForceTerm) {
        const BuoyancyForceTerm* b = self->buoyancyForceTerm;
        v.force.gravity = b->gravity;
        for (int d = 0; d < 3; d++) v.force.g_hat[d] = b->gHat ? (d < dim ? b->gHat[d] : 0.0) : (d == 1 ? -1.0 : 0.0);
    } else {
        v.force.g_hat[1] = -1.0;
    }
    if (self->thermalBuoyancyForceTerm) v.force.rayleigh = self->thermalBuoyancyForceTerm->rayleighNumber;

    MaterialPointsSwarm* ms = self->materialSwarm;
    v.n_points = ms->particleLocalCount;
    double* coords = (double*)malloc(sizeof(double) * (size_t)(v.n_points * dim));
    int32_t* mat = (int32_t*)malloc(sizeof(int32_t) * (size_t)v.n_points);
    double* ps = self->strainWeakening ? (double*)malloc(sizeof(double) * (size_t)v.n_points) : NULL;
    for (int64_t i = 0; i < v.n_points; i++) {
        MaterialPoint* mp = (MaterialPoint*)Swarm_ParticleAt(ms, (Particle_Index)i);
        for (int d = 0; d < dim; d++) coords[i * dim + d] = mp->coord[d];
        mat[i] = (int32_t)mp->materialIndex;
        if (ps) ps[i] = StrainWeakening_GetPostFailureWeakening(self->strainWeakening, mp);
    }
    v.coords = coords;
    v.material = mat;
    v.plastic_strain = ps;

    double* T = NULL;
    if (self->temperatureField) {
        T = (double*)malloc(sizeof(double) * (size_t)nnode);
        for (int64_t n = 0; n < nnode; n++) FeVariable_GetValueAtNode(self->temperatureField, (Node_DomainIndex)n, &T[n]);
        v.temperature = T;
    }

    double* u = (double*)malloc(sizeof(double) * (size_t)(nnode * dim));
    double* p = (double*)malloc(sizeof(double) * (size_t)nel);
    const int rc = StokesGPU_Solve(&self->handle, &v, &self->params, u, p, &self->stats);
    Journal_Firewall(rc == GG_OK, self->errorStream, "Error in func '%s' for %s '%s': status %d: %s\n", __func__,
                     self->type, self->name, rc, self->handle ? gg_last_error(self->handle) : "no device handle");

    /* the FeVariables take the nodal / element values, their SolutionVectors the free ones */
    for (int64_t n = 0; n < nnode; n++) FeVariable_SetValueAtNode(vel, (Node_DomainIndex)n, &u[n * dim]);
    for (int64_t e = 0; e < nel; e++) FeVariable_SetValueAtNode(pres, (Node_DomainIndex)e, &p[e]);
    SolutionVector_LoadCurrentFeVariableValuesOntoVector(sle->uSolnVec);
    SolutionVector_LoadCurrentFeVariableValuesOntoVector(sle->pSolnVec);

    free(fixed);
    free(bcv);
    free(coords);
    free(mat);
    free(ps);
    free(T);
    free(u);
    free(p);
}
