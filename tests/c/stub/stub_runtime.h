/* stub_runtime.h -- the stub runtime's own objects and constructors (not part of the
 * reference's interface; tests/c/plugin_driver.c builds a model from them). */
#ifndef STUB_RUNTIME_H
#define STUB_RUNTIME_H

#include "gale_stub.h"

typedef struct StubMesh {
    unsigned dim;
    double min[3], max[3];
    unsigned sizes[3];
    Grid grid;
    Grid* gridp;  /* what Mesh_GetExtension(mesh, Grid**, "elementGrid") dereferences */
} StubMesh;

typedef struct StubFeVariable {
    FeVariable base;
    unsigned nnodes;
    double* values;     /* [nnodes][fieldComponentCount] */
    uint8_t* bcmask;    /* [nnodes] bit c: component c fixed, or NULL */
} StubFeVariable;

typedef struct StubSwarm {
    MaterialPointsSwarm base;
    MaterialPoint* points;
} StubSwarm;

PluginsManager* StubPluginsManager_New(void);
Stg_Component_DefaultConstructorFunction* StubPluginsManager_Get(PluginsManager* self, Type type);
LiveComponentRegister* StubLiveComponentRegister_New(void);
void StubLiveComponentRegister_Add(LiveComponentRegister* self, const char* name, void* obj);
void StubDictionary_Set(const char* component, const char* key, const char* value);
Vec StubVec_New(void);
Materials_Register* StubMaterials_Register_New(void);
void StubMaterials_Register_Add(Materials_Register* self, Material* m);
Rheology_Register* StubRheology_Register_New(void);
void StubRheology_Register_Add(Rheology_Register* self, Rheology* r);

#endif
