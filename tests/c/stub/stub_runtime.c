/*
 * stub_runtime.c -- a minimal implementation of the declaration stub (gale_stub.h) over
 * plain arrays: component / plugin registers, a component factory dictionary, a regular
 * mesh, FeVariables with nodal values and BC masks, SolutionVectors as PETSc-like Vecs of
 * the free dofs, a material-point swarm, materials with rheology registers.  It exists so
 * that gale_b200/host/stokes_gpu_plugin.c can be compiled and driven here.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "stub_runtime.h"

const Type Error_Type = "Error";
const Type Info_Type = "Info";

struct Stream {
    const char* name;
};
static struct Stream g_stream = {"stub"};

Stream* Journal_Register(Type type, Name name) {
    (void)type;
    (void)name;
    return &g_stream;
}

/* the reference aborts the job; the stub prints the message and exits with status 3 */
void Journal_Firewall(Bool expression, Stream* stream, const char* fmt, ...) {
    (void)stream;
    if (expression) return;
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "Journal_Firewall: ");
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fflush(stderr);
    exit(3);
}

void Journal_Printf(Stream* stream, const char* fmt, ...) {
    (void)stream;
    va_list ap;
    va_start(ap, fmt);
    vprintf(fmt, ap);
    va_end(ap);
}

/* ---- registers ------------------------------------------------------------------------ */
#define STUB_MAX 64
typedef struct {
    char type[128];
    Stg_Component_DefaultConstructorFunction* fn;
} RegEntry;
struct PluginsManager {
    int n;
    RegEntry e[STUB_MAX];
};
struct Stg_ComponentRegister {
    int n;
    RegEntry e[STUB_MAX];
};
static struct Stg_ComponentRegister g_components;

PluginsManager* StubPluginsManager_New(void) { return (PluginsManager*)calloc(1, sizeof(PluginsManager)); }

Stg_Component_DefaultConstructorFunction* StubPluginsManager_Get(PluginsManager* self, Type type) {
    for (int i = 0; i < self->n; i++)
        if (!strcmp(self->e[i].type, type)) return self->e[i].fn;
    return NULL;
}

Index PluginsManager_Submit(PluginsManager* self, Type codeletType, Name version,
                            Stg_Component_DefaultConstructorFunction* defaultNew) {
    (void)version;
    snprintf(self->e[self->n].type, sizeof self->e[0].type, "%s", codeletType);
    self->e[self->n].fn = defaultNew;
    return (Index)self->n++;
}

Stg_ComponentRegister* Stg_ComponentRegister_Get_ComponentRegister(void) { return &g_components; }

Bool Stg_ComponentRegister_Add(Stg_ComponentRegister* self, Type componentType, Name version,
                               Stg_Component_DefaultConstructorFunction* func) {
    (void)version;
    snprintf(self->e[self->n].type, sizeof self->e[0].type, "%s", componentType);
    self->e[self->n++].fn = func;
    return True;
}

Stg_Component_DefaultConstructorFunction* Stg_ComponentRegister_Get(Stg_ComponentRegister* self, Type componentType,
                                                                    Name version) {
    (void)version;
    for (int i = 0; i < self->n; i++)
        if (!strcmp(self->e[i].type, componentType)) return self->e[i].fn;
    return NULL;
}

struct LiveComponentRegister {
    int n;
    char name[STUB_MAX][64];
    void* obj[STUB_MAX];
};

LiveComponentRegister* StubLiveComponentRegister_New(void) {
    return (LiveComponentRegister*)calloc(1, sizeof(LiveComponentRegister));
}

void StubLiveComponentRegister_Add(LiveComponentRegister* self, const char* name, void* obj) {
    snprintf(self->name[self->n], sizeof self->name[0], "%s", name);
    self->obj[self->n++] = obj;
}

void* LiveComponentRegister_Get(LiveComponentRegister* self, Name name) {
    for (int i = 0; i < self->n; i++)
        if (!strcmp(self->name[i], name)) return self->obj[i];
    return NULL;
}

/* ---- the component factory's dictionary: (component, key) -> text ---------------------- */
static struct {
    int n;
    char comp[STUB_MAX][64], key[STUB_MAX][64], val[STUB_MAX][64];
} g_dict;

void StubDictionary_Set(const char* component, const char* key, const char* value) {
    snprintf(g_dict.comp[g_dict.n], 64, "%s", component);
    snprintf(g_dict.key[g_dict.n], 64, "%s", key);
    snprintf(g_dict.val[g_dict.n], 64, "%s", value);
    g_dict.n++;
}

static const char* lookup(Name component, Dictionary_Entry_Key key) {
    for (int i = 0; i < g_dict.n; i++)
        if (!strcmp(g_dict.comp[i], component) && !strcmp(g_dict.key[i], key)) return g_dict.val[i];
    return NULL;
}

double Stg_ComponentFactory_GetDouble(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                      double defaultVal) {
    (void)cf;
    const char* v = lookup(componentName, key);
    return v ? strtod(v, NULL) : defaultVal;
}

unsigned int Stg_ComponentFactory_GetUnsignedInt(Stg_ComponentFactory* cf, Name componentName,
                                                 Dictionary_Entry_Key key, unsigned int defaultVal) {
    (void)cf;
    const char* v = lookup(componentName, key);
    return v ? (unsigned)strtoul(v, NULL, 10) : defaultVal;
}

Bool Stg_ComponentFactory_GetBool(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                  Bool defaultVal) {
    (void)cf;
    const char* v = lookup(componentName, key);
    if (!v) return defaultVal;
    return v[0] == 't' || v[0] == 'T' || v[0] == '1';
}

char* Stg_ComponentFactory_GetString(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                     const char* defaultVal) {
    (void)cf;
    const char* v = lookup(componentName, key);
    return (char*)(v ? v : defaultVal);
}

void* _Stg_ComponentFactory_ConstructByKey(Stg_ComponentFactory* cf, Name parentName, Dictionary_Entry_Key key,
                                           Type type, Bool isEssential, void* data) {
    (void)data;
    const char* name = lookup(parentName, key);
    void* obj = name ? LiveComponentRegister_Get(cf->LCRegister, (Name)name) : NULL;
    Journal_Firewall(obj != NULL || !isEssential, &g_stream, "component '%s' (%s) for key '%s' of '%s' not found\n",
                     name ? name : "", type, key, parentName);
    return obj;
}

/* ---- constructors ---------------------------------------------------------------------- */
static void init_component(Stg_Component* c, SizeT size, Type type, Stg_Class_DeleteFunction* del,
                           Stg_Class_PrintFunction* print, Stg_Class_CopyFunction* copy,
                           Stg_Component_DefaultConstructorFunction* dc, Stg_Component_AssignFromXMLFunction* construct,
                           Stg_Component_BuildFunction* build, Stg_Component_InitialiseFunction* init,
                           Stg_Component_ExecuteFunction* exec, Stg_Component_DestroyFunction* destroy, Name name,
                           AllocationType nat) {
    c->_sizeOfSelf = size;
    c->type = type;
    c->_delete = del;
    c->_print = print;
    c->_copy = copy;
    c->name = name;
    c->nameAllocationType = nat;
    c->_defaultConstructor = dc;
    c->_assignFromXML = construct;
    c->_build = build;
    c->_initialise = init;
    c->_execute = exec;
    c->_destroy = destroy;
}

void* _Codelet_New(SizeT _sizeOfSelf, Type type, Stg_Class_DeleteFunction* _delete, Stg_Class_PrintFunction* _print,
                   Stg_Class_CopyFunction* _copy, Stg_Component_DefaultConstructorFunction* _defaultConstructor,
                   Stg_Component_AssignFromXMLFunction* _construct, Stg_Component_BuildFunction* _build,
                   Stg_Component_InitialiseFunction* _initialise, Stg_Component_ExecuteFunction* _execute,
                   Stg_Component_DestroyFunction* _destroy, Name name, AllocationType nameAllocationType) {
    Stg_Component* c = (Stg_Component*)calloc(1, _sizeOfSelf);
    init_component(c, _sizeOfSelf, type, _delete, _print, _copy, _defaultConstructor, _construct, _build, _initialise,
                   _execute, _destroy, name, nameAllocationType);
    return c;
}

void _Codelet_Delete(void* codelet) { free(codelet); }
void _Codelet_Print(void* codelet, Stream* stream) { (void)codelet; (void)stream; }
void* _Codelet_Copy(void* codelet, void* dest, Bool deep, Name nameExt, void* ptrMap) {
    (void)codelet; (void)deep; (void)nameExt; (void)ptrMap;
    return dest;
}
void _Codelet_AssignFromXML(void* codelet, Stg_ComponentFactory* cf, void* data) { (void)codelet; (void)cf; (void)data; }
void _Codelet_Build(void* codelet, void* data) { (void)codelet; (void)data; }
void _Codelet_Initialise(void* codelet, void* data) { (void)codelet; (void)data; }
void _Codelet_Execute(void* codelet, void* data) { (void)codelet; (void)data; }
void _Codelet_Destroy(void* codelet, void* data) { (void)codelet; (void)data; }

void* _SLE_Solver_New(SizeT _sizeOfSelf, Type type, Stg_Class_DeleteFunction* _delete,
                      Stg_Class_PrintFunction* _print, Stg_Class_CopyFunction* _copy,
                      Stg_Component_DefaultConstructorFunction* _defaultConstructor,
                      Stg_Component_AssignFromXMLFunction* _construct, Stg_Component_BuildFunction* _build,
                      Stg_Component_InitialiseFunction* _initialise, Stg_Component_ExecuteFunction* _execute,
                      Stg_Component_DestroyFunction* _destroy, SLE_Solver_SolverSetupFunction* _solverSetup,
                      SLE_Solver_SolveFunction* _solve, SLE_Solver_GetResidualFunc* _getResidual, Name name,
                      AllocationType nameAllocationType) {
    SLE_Solver* s = (SLE_Solver*)calloc(1, _sizeOfSelf);
    init_component((Stg_Component*)s, _sizeOfSelf, type, _delete, _print, _copy, _defaultConstructor, _construct,
                   _build, _initialise, _execute, _destroy, name, nameAllocationType);
    s->_solverSetup = _solverSetup;
    s->_solve = _solve;
    s->_getResidual = _getResidual;
    return s;
}

void _SLE_Solver_Delete(void* sleSolver) { free(sleSolver); }
void _SLE_Solver_Print(void* sleSolver, Stream* stream) { (void)sleSolver; (void)stream; }

/* ---- mesh -------------------------------------------------------------------------------- */
unsigned Mesh_GetDimSize(void* mesh) { return ((StubMesh*)mesh)->dim; }

unsigned Mesh_GetDomainSize(void* mesh, MeshTopology_Dim dim) {
    StubMesh* m = (StubMesh*)mesh;
    unsigned n = 1;
    for (unsigned d = 0; d < m->dim; d++) n *= m->sizes[d] + (dim == MT_VERTEX ? 1 : 0);
    return n;
}

void Mesh_GetGlobalCoordRange(void* mesh, double* min, double* max) {
    StubMesh* m = (StubMesh*)mesh;
    for (unsigned d = 0; d < m->dim; d++) {
        min[d] = m->min[d];
        max[d] = m->max[d];
    }
}

void* Mesh_GetExtensionByName(void* mesh, const char* name) {
    StubMesh* m = (StubMesh*)mesh;
    return strcmp(name, "elementGrid") ? NULL : (void*)&m->gridp;
}

/* ---- FeVariables and vectors ----------------------------------------------------------- */
Bool FeVariable_IsBC(void* feVariable, Node_DomainIndex node, Dof_Index dof) {
    StubFeVariable* v = (StubFeVariable*)feVariable;
    return v->bcmask ? ((v->bcmask[node] >> dof) & 1) : False;
}

void FeVariable_GetValueAtNode(void* feVariable, Node_DomainIndex node, double* value) {
    StubFeVariable* v = (StubFeVariable*)feVariable;
    memcpy(value, v->values + (size_t)node * v->base.fieldComponentCount, sizeof(double) * v->base.fieldComponentCount);
}

void FeVariable_SetValueAtNode(void* feVariable, Node_DomainIndex node, double* value) {
    StubFeVariable* v = (StubFeVariable*)feVariable;
    memcpy(v->values + (size_t)node * v->base.fieldComponentCount, value, sizeof(double) * v->base.fieldComponentCount);
}

struct _p_Vec {
    PetscInt n;
    PetscScalar* a;
};

Vec StubVec_New(void) { return (Vec)calloc(1, sizeof(struct _p_Vec)); }

PetscErrorCode VecGetArray(Vec v, PetscScalar** a) {
    *a = v->a;
    return 0;
}
PetscErrorCode VecRestoreArray(Vec v, PetscScalar** a) {
    (void)v;
    *a = NULL;
    return 0;
}
PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n) {
    *n = v->n;
    return 0;
}

/* the free dofs in node order, component within node (FeEquationNumber of a serial run) */
void SolutionVector_LoadCurrentFeVariableValuesOntoVector(void* solutionVector) {
    SolutionVector* sv = (SolutionVector*)solutionVector;
    StubFeVariable* v = (StubFeVariable*)sv->feVariable;
    const unsigned nc = v->base.fieldComponentCount;
    PetscInt n = 0;
    for (unsigned i = 0; i < v->nnodes; i++)
        for (unsigned c = 0; c < nc; c++)
            if (!FeVariable_IsBC(v, i, c)) n++;
    free(sv->vector->a);
    sv->vector->a = (PetscScalar*)malloc(sizeof(PetscScalar) * (size_t)(n ? n : 1));
    sv->vector->n = n;
    n = 0;
    for (unsigned i = 0; i < v->nnodes; i++)
        for (unsigned c = 0; c < nc; c++)
            if (!FeVariable_IsBC(v, i, c)) sv->vector->a[n++] = v->values[(size_t)i * nc + c];
}

/* ---- swarm, materials, rheologies ---------------------------------------------------- */
void* Swarm_ParticleAt(void* swarm, Particle_Index lParticle_I) {
    return &((StubSwarm*)swarm)->points[lParticle_I];
}

struct Materials_Register {
    Index n;
    Material* m[16];
};

Materials_Register* StubMaterials_Register_New(void) { return (Materials_Register*)calloc(1, sizeof(Materials_Register)); }
void StubMaterials_Register_Add(Materials_Register* self, Material* m) { self->m[self->n++] = m; }
Index Materials_Register_GetCount(Materials_Register* self) { return self->n; }
Material* Materials_Register_GetByIndex(Materials_Register* self, Index i) { return self->m[i]; }

/* the stub's extension manager of a material is its buoyancy extension */
void* ExtensionManager_Get(void* extensionManager, void* ptr, Index handle) {
    (void)ptr;
    (void)handle;
    return extensionManager;
}

struct Rheology_Register {
    Index n;
    Rheology* r[8];
};

Rheology_Register* StubRheology_Register_New(void) { return (Rheology_Register*)calloc(1, sizeof(Rheology_Register)); }
void StubRheology_Register_Add(Rheology_Register* self, Rheology* r) { self->r[self->n++] = r; }
Index Rheology_Register_GetCount(Rheology_Register* self) { return self->n; }
Rheology* Rheology_Register_GetByIndex(Rheology_Register* self, Index i) { return self->r[i]; }

double StrainWeakening_GetPostFailureWeakening(void* strainWeakening, void* particle) {
    (void)strainWeakening;
    (void)particle;
    return 0.0;
}
