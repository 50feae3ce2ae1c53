/*
 * gale_stub.h -- a declaration stub of the StGermain / StgDomain / StgFEM / PICellerator /
 * Underworld / PETSc interfaces that gale_b200/host/stokes_gpu_plugin.c touches, so that
 * the plugin compiles and runs here, where none of those libraries exist.  Type, field
 * and function names are the reference's; only the members the plugin reads are declared,
 * and each class keeps its parent's members first, as the reference's __Class macros do.
 * tests/c/stub/stub_runtime.c implements the functions over plain arrays.
 */
#ifndef GALE_STUB_H
#define GALE_STUB_H

#include <stddef.h>
#include <stdint.h>

/* ---- StGermain/Base/Foundation ---------------------------------------------------- */
typedef const char* Type;
typedef char* Name;
typedef const char* Dictionary_Entry_Key;
typedef unsigned int Index;
typedef unsigned int Iteration_Index;
typedef unsigned int Element_LocalIndex;
typedef unsigned int Node_DomainIndex;
typedef unsigned int Dof_Index;
typedef unsigned int Particle_Index;
typedef unsigned int Material_Index;
typedef int Bool;
typedef size_t SizeT;
typedef double Coord[3];
typedef double XYZ[3];
#define True 1
#define False 0
typedef enum { NON_GLOBAL = 0, GLOBAL } AllocationType;

typedef struct Stream Stream;
Stream* Journal_Register(Type type, Name name);
void Journal_Firewall(Bool expression, Stream* stream, const char* fmt, ...);
void Journal_Printf(Stream* stream, const char* fmt, ...);
extern const Type Error_Type;
extern const Type Info_Type;

/* ---- StGermain/Base/Automation ---------------------------------------------------- */
typedef struct Stg_ComponentFactory Stg_ComponentFactory;
typedef struct LiveComponentRegister LiveComponentRegister;
typedef struct Stg_ComponentRegister Stg_ComponentRegister;
typedef struct PluginsManager PluginsManager;

typedef void (Stg_Class_DeleteFunction)(void* self);
typedef void (Stg_Class_PrintFunction)(void* self, Stream* stream);
typedef void* (Stg_Class_CopyFunction)(void* self, void* dest, Bool deep, Name nameExt, void* ptrMap);
typedef void* (Stg_Component_DefaultConstructorFunction)(Name name);
typedef void (Stg_Component_AssignFromXMLFunction)(void* component, Stg_ComponentFactory* cf, void* data);
typedef void (Stg_Component_BuildFunction)(void* component, void* data);
typedef void (Stg_Component_InitialiseFunction)(void* component, void* data);
typedef void (Stg_Component_ExecuteFunction)(void* component, void* data);
typedef void (Stg_Component_DestroyFunction)(void* component, void* data);

#define __Stg_Class \
    SizeT _sizeOfSelf; \
    Type type; \
    Stg_Class_DeleteFunction* _delete; \
    Stg_Class_PrintFunction* _print; \
    Stg_Class_CopyFunction* _copy;
#define __Stg_Object \
    __Stg_Class \
    Name name; \
    AllocationType nameAllocationType;
#define __Stg_Component \
    __Stg_Object \
    Stg_Component_DefaultConstructorFunction* _defaultConstructor; \
    Stg_Component_AssignFromXMLFunction* _assignFromXML; \
    Stg_Component_BuildFunction* _build; \
    Stg_Component_InitialiseFunction* _initialise; \
    Stg_Component_ExecuteFunction* _execute; \
    Stg_Component_DestroyFunction* _destroy;
typedef struct Stg_Component { __Stg_Component } Stg_Component;

struct Stg_ComponentFactory {
    LiveComponentRegister* LCRegister;
};

Index PluginsManager_Submit(PluginsManager* self, Type codeletType, Name version,
                            Stg_Component_DefaultConstructorFunction* defaultNew);
Stg_ComponentRegister* Stg_ComponentRegister_Get_ComponentRegister(void);
Bool Stg_ComponentRegister_Add(Stg_ComponentRegister* self, Type componentType, Name version,
                               Stg_Component_DefaultConstructorFunction* func);
Stg_Component_DefaultConstructorFunction* Stg_ComponentRegister_Get(Stg_ComponentRegister* self,
                                                                    Type componentType, Name version);
void* LiveComponentRegister_Get(LiveComponentRegister* self, Name name);

double Stg_ComponentFactory_GetDouble(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                      double defaultVal);
unsigned int Stg_ComponentFactory_GetUnsignedInt(Stg_ComponentFactory* cf, Name componentName,
                                                 Dictionary_Entry_Key key, unsigned int defaultVal);
Bool Stg_ComponentFactory_GetBool(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                  Bool defaultVal);
char* Stg_ComponentFactory_GetString(Stg_ComponentFactory* cf, Name componentName, Dictionary_Entry_Key key,
                                     const char* defaultVal);
/* the reference's macro casts the constructed component to `type` */
void* _Stg_ComponentFactory_ConstructByKey(Stg_ComponentFactory* cf, Name parentName, Dictionary_Entry_Key key,
                                           Type type, Bool isEssential, void* data);
#define Stg_ComponentFactory_ConstructByKey(cf, parentName, key, type, isEssential, data) \
    ((type*)_Stg_ComponentFactory_ConstructByKey(cf, parentName, key, #type, isEssential, data))

/* ---- StGermain/Base/Extensibility: plugins are Codelets ----------------------------- */
#define __Codelet __Stg_Component
typedef struct Codelet { __Codelet } Codelet;
#define CODELET_PASSARGS \
    _sizeOfSelf, type, _delete, _print, _copy, _defaultConstructor, _construct, _build, _initialise, _execute, \
        _destroy, name, nameAllocationType
void* _Codelet_New(SizeT _sizeOfSelf, Type type, Stg_Class_DeleteFunction* _delete, Stg_Class_PrintFunction* _print,
                   Stg_Class_CopyFunction* _copy, Stg_Component_DefaultConstructorFunction* _defaultConstructor,
                   Stg_Component_AssignFromXMLFunction* _construct, Stg_Component_BuildFunction* _build,
                   Stg_Component_InitialiseFunction* _initialise, Stg_Component_ExecuteFunction* _execute,
                   Stg_Component_DestroyFunction* _destroy, Name name, AllocationType nameAllocationType);
void _Codelet_Delete(void* codelet);
void _Codelet_Print(void* codelet, Stream* stream);
void* _Codelet_Copy(void* codelet, void* dest, Bool deep, Name nameExt, void* ptrMap);
void _Codelet_AssignFromXML(void* codelet, Stg_ComponentFactory* cf, void* data);
void _Codelet_Build(void* codelet, void* data);
void _Codelet_Initialise(void* codelet, void* data);
void _Codelet_Execute(void* codelet, void* data);
void _Codelet_Destroy(void* codelet, void* data);

/* ---- StgDomain: meshes and swarms ------------------------------------------------- */
typedef struct Grid {
    unsigned nDims;
    unsigned* sizes;
} Grid;
typedef enum { MT_VERTEX = 0, MT_EDGE, MT_FACE, MT_VOLUME } MeshTopology_Dim;
typedef struct Mesh Mesh;
unsigned Mesh_GetDimSize(void* mesh);
unsigned Mesh_GetDomainSize(void* mesh, MeshTopology_Dim dim);
void Mesh_GetGlobalCoordRange(void* mesh, double* min, double* max);
void* Mesh_GetExtensionByName(void* mesh, const char* name);
#define Mesh_GetExtension(self, type, name) ((type)Mesh_GetExtensionByName(self, name))

typedef struct MaterialPoint {
    Coord coord;
    Material_Index materialIndex;
} MaterialPoint;

/* ---- StgFEM ----------------------------------------------------------------------- */
typedef struct _p_Vec* Vec;
typedef struct _p_KSP* KSP;
typedef double PetscScalar;
typedef int PetscErrorCode;
typedef int PetscInt;
PetscErrorCode VecGetArray(Vec v, PetscScalar** a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar** a);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n);

typedef Mesh FeMesh;
typedef struct FeVariable {
    __Stg_Component
    FeMesh* feMesh;
    unsigned fieldComponentCount;
} FeVariable;
Bool FeVariable_IsBC(void* feVariable, Node_DomainIndex node, Dof_Index dof);
void FeVariable_GetValueAtNode(void* feVariable, Node_DomainIndex node, double* value);
void FeVariable_SetValueAtNode(void* feVariable, Node_DomainIndex node, double* value);

typedef struct SolutionVector {
    __Stg_Component
    Vec vector;
    FeVariable* feVariable;
} SolutionVector;
void SolutionVector_LoadCurrentFeVariableValuesOntoVector(void* solutionVector);
typedef struct ForceVector {
    __Stg_Component
    Vec vector;
    FeVariable* feVariable;
} ForceVector;
typedef struct StiffnessMatrix StiffnessMatrix;

typedef struct FiniteElementContext {
    __Stg_Component
    Stg_ComponentFactory* CF;
    struct Materials_Register* materials_Register; /* PICelleratorContext */
} FiniteElementContext;

#define __SystemLinearEquations \
    __Stg_Component \
    FiniteElementContext* context;
#define __Stokes_SLE \
    __SystemLinearEquations \
    StiffnessMatrix* kStiffMat; \
    StiffnessMatrix* gStiffMat; \
    StiffnessMatrix* dStiffMat; \
    StiffnessMatrix* cStiffMat; \
    SolutionVector* uSolnVec; \
    SolutionVector* pSolnVec; \
    ForceVector* fForceVec; \
    ForceVector* hForceVec;
typedef struct Stokes_SLE { __Stokes_SLE } Stokes_SLE;

typedef void (SLE_Solver_SolverSetupFunction)(void* sleSolver, void* sle);
typedef void (SLE_Solver_SolveFunction)(void* sleSolver, void* sle);
typedef Vec (SLE_Solver_GetResidualFunc)(void* sleSolver, Index fvIndex);
#define __SLE_Solver \
    __Stg_Component \
    FiniteElementContext* context; \
    void* extensionManager; \
    SLE_Solver_SolverSetupFunction* _solverSetup; \
    SLE_Solver_SolveFunction* _solve; \
    SLE_Solver_GetResidualFunc* _getResidual; \
    Stream* debug; \
    Stream* info; \
    Iteration_Index maxIterations;
typedef struct SLE_Solver { __SLE_Solver } SLE_Solver;
#define SLE_SOLVER_PASSARGS \
    _sizeOfSelf, type, _delete, _print, _copy, _defaultConstructor, _construct, _build, _initialise, _execute, \
        _destroy, _solverSetup, _solve, _getResidual, name, nameAllocationType
void* _SLE_Solver_New(SizeT _sizeOfSelf, Type type, Stg_Class_DeleteFunction* _delete,
                      Stg_Class_PrintFunction* _print, Stg_Class_CopyFunction* _copy,
                      Stg_Component_DefaultConstructorFunction* _defaultConstructor,
                      Stg_Component_AssignFromXMLFunction* _construct, Stg_Component_BuildFunction* _build,
                      Stg_Component_InitialiseFunction* _initialise, Stg_Component_ExecuteFunction* _execute,
                      Stg_Component_DestroyFunction* _destroy, SLE_Solver_SolverSetupFunction* _solverSetup,
                      SLE_Solver_SolveFunction* _solve, SLE_Solver_GetResidualFunc* _getResidual, Name name,
                      AllocationType nameAllocationType);
void _SLE_Solver_Delete(void* sleSolver);
void _SLE_Solver_Print(void* sleSolver, Stream* stream);

#define __Stokes_SLE_UzawaSolver \
    __SLE_Solver \
    KSP velSolver; \
    KSP pcSolver; \
    StiffnessMatrix* preconditioner; \
    Iteration_Index maxUzawaIterations; \
    Iteration_Index minUzawaIterations; \
    double tolerance; \
    Bool useAbsoluteTolerance; \
    Bool monitor;
typedef struct Stokes_SLE_UzawaSolver { __Stokes_SLE_UzawaSolver } Stokes_SLE_UzawaSolver;

/* ---- PICellerator ------------------------------------------------------------------ */
typedef struct MaterialPointsSwarm {
    __Stg_Component
    Particle_Index particleLocalCount;
} MaterialPointsSwarm;
void* Swarm_ParticleAt(void* swarm, Particle_Index lParticle_I);

#define __Material \
    __Stg_Component \
    Index index; \
    void* extensionMgr;
typedef struct Material { __Material } Material;
typedef struct Materials_Register Materials_Register;
Index Materials_Register_GetCount(Materials_Register* self);
Material* Materials_Register_GetByIndex(Materials_Register* self, Index materialIndex);
void* ExtensionManager_Get(void* extensionManager, void* ptr, Index handle);

typedef struct BuoyancyForceTerm_MaterialExt {
    double alpha;
    double density;
} BuoyancyForceTerm_MaterialExt;
typedef struct BuoyancyForceTerm {
    __Stg_Component
    FeVariable* temperatureField;
    double gravity;
    double* gHat;
    Index materialExtHandle;
    void* hydrostaticTerm;
} BuoyancyForceTerm;

/* StgFEM/Assembly/src/ThermalBuoyancyForceTerm.h */
typedef struct ThermalBuoyancyForceTerm {
    __Stg_Component
    FeVariable* temperatureField;
    double rayleighNumber;
} ThermalBuoyancyForceTerm;

/* ---- Underworld/Rheology --------------------------------------------------------- */
#define __Rheology __Stg_Component
typedef struct Rheology { __Rheology } Rheology;
typedef struct Rheology_Register Rheology_Register;
Index Rheology_Register_GetCount(Rheology_Register* self);
Rheology* Rheology_Register_GetByIndex(Rheology_Register* self, Index rheology_I);
#define __RheologyMaterial \
    __Material \
    Rheology_Register* rheology_Register;
typedef struct RheologyMaterial { __RheologyMaterial } RheologyMaterial;

typedef struct MaterialViscosity { __Rheology double eta0; } MaterialViscosity;
typedef struct Arrhenius {
    __Rheology
    FeVariable* temperatureField;
    double eta0, activationEnergy, activationVolume, referenceTemp;
} Arrhenius;
typedef struct FrankKamenetskii {
    __Rheology
    FeVariable* temperatureField;
    double eta0, theta;
} FrankKamenetskii;
typedef struct StrainWeakening {
    __Stg_Component
    double healingRate, initialSofteningStrain, finalSofteningStrain;
} StrainWeakening;
double StrainWeakening_GetPostFailureWeakening(void* strainWeakening, void* particle);
#define __YieldRheology \
    __Rheology \
    StrainWeakening* strainWeakening; \
    double minVisc;
#define __VonMises \
    __YieldRheology \
    FeVariable* strainRateField; \
    double cohesion; \
    double cohesionAfterSoftening; \
    Bool strainRateSoftening;
typedef struct VonMises { __VonMises } VonMises;
typedef struct DruckerPrager {
    __VonMises
    FeVariable* pressureField;
    double frictionCoefficient, frictionCoefficientAfterSoftening;
    double boundaryCohesion, boundaryCohesionAfterSoftening;
    double boundaryFrictionCoefficient, boundaryFrictionCoefficientAfterSoftening;
    Bool boundaryBottom, boundaryTop, boundaryLeft, boundaryRight, boundaryFront, boundaryBack;
    double minimumYieldStress, minimumViscosity, maxStrainRate;
    void* hydrostaticTerm;
} DruckerPrager;
typedef struct Byerlee {
    __VonMises
    FeMesh* mesh;
    double depthCoefficient;
} Byerlee;

#endif
