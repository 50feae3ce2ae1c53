/*
 * stokes_gpu_plugin.h -- the StGermain side of the Stokes_SLE_UzawaSolverGPU plugin.
 *
 * Gale loads plugins by name and calls <Name>_Register(PluginsManager*)
 * (StGermain/Base/Extensibility/src/Plugin.cxx:55,97; pattern of
 * StgFEM/plugins/Multigrid/Multigrid.cxx:139-143).  Underworld_StokesGPU_Register submits
 * the codelet and adds the component type Stokes_SLE_UzawaSolverGPU to the component
 * register, so an input deck selects the GPU path with
 *     <struct name="uzawa"> <param name="Type">Stokes_SLE_UzawaSolverGPU</param> ... </struct>
 * The type is a Stokes_SLE_UzawaSolver (StgFEM/SLE/ProvidedSystems/StokesFlow/src/
 * Stokes_SLE_UzawaSolver.h) whose _solverSetup / _solve (SLE_Solver.h:61-62) run the
 * solve through the C ABI of include/gale_gpu.h.
 */
#ifndef STOKES_GPU_PLUGIN_H
#define STOKES_GPU_PLUGIN_H

#include <StGermain/StGermain.h>
#include <StgDomain/StgDomain.h>
#include <StgFEM/StgFEM.h>
#include <PICellerator/PICellerator.h>
#include <Underworld/Underworld.h>

#include "stokes_gpu_host.h"

extern const Type Underworld_StokesGPU_Type;
extern const Type Stokes_SLE_UzawaSolverGPU_Type;

#define __Stokes_SLE_UzawaSolverGPU \
    __Stokes_SLE_UzawaSolver \
    gg_handle* handle;                       /* device state, reused across solves */ \
    gg_uzawa_params params; \
    gg_uzawa_stats stats; \
    MaterialPointsSwarm* materialSwarm; \
    Materials_Register* materials_Register; \
    BuoyancyForceTerm* buoyancyForceTerm;    /* NULL: no density body force */ \
    ThermalBuoyancyForceTerm* thermalBuoyancyForceTerm; /* NULL: no Ra·T force */ \
    FeVariable* temperatureField;            /* NULL: no temperature */ \
    StrainWeakening* strainWeakening;        /* NULL: no plastic strain */ \
    Stream* errorStream;

typedef struct Stokes_SLE_UzawaSolverGPU { __Stokes_SLE_UzawaSolverGPU } Stokes_SLE_UzawaSolverGPU;

Index Underworld_StokesGPU_Register(PluginsManager* pluginsManager);
void* _Underworld_StokesGPU_DefaultNew(Name name);

void* _Stokes_SLE_UzawaSolverGPU_DefaultNew(Name name);
void _Stokes_SLE_UzawaSolverGPU_AssignFromXML(void* solver, Stg_ComponentFactory* cf, void* data);
void _Stokes_SLE_UzawaSolverGPU_SolverSetup(void* solver, void* stokesSLE);
void _Stokes_SLE_UzawaSolverGPU_Solve(void* solver, void* stokesSLE);
void _Stokes_SLE_UzawaSolverGPU_Destroy(void* solver, void* data);

#endif
