/* plugin_driver.c -- drives gale_b200/host/stokes_gpu_plugin.c the way Gale would, on the
 * declaration stub of tests/c/stub: loads the plugin through Underworld_StokesGPU_Register,
 * takes the Stokes_SLE_UzawaSolverGPU constructor back from the component register, builds
 * the solver from a component-factory dictionary, and runs _solverSetup and _solve through
 * the SLE_Solver function pointers on a 2D sinker (read from a binary file, as
 * tests/c/stokes_driver.c does).  Writes the velocity and pressure FeVariables' values.
 * Used by tests/test_c_plugin.py. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../gale_b200/host/stokes_gpu_plugin.h"
#include "stub/stub_runtime.h"

static void* slurp(FILE* f, size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (bytes && fread(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "short read\n");
        exit(2);
    }
    return p;
}

static RheologyMaterial* material(const char* name, double eta0, BuoyancyForceTerm_MaterialExt* ext) {
    RheologyMaterial* m = (RheologyMaterial*)calloc(1, sizeof(RheologyMaterial));
    MaterialViscosity* mv = (MaterialViscosity*)calloc(1, sizeof(MaterialViscosity));
    mv->type = "MaterialViscosity";
    mv->name = (Name)name;
    mv->eta0 = eta0;
    m->type = "RheologyMaterial";
    m->rheology_Register = StubRheology_Register_New();
    StubRheology_Register_Add(m->rheology_Register, (Rheology*)mv);
    m->extensionMgr = ext;
    return m;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t n;
    int64_t np;
    if (fread(&n, 4, 1, f) != 1 || fread(&np, 8, 1, f) != 1) return 2;
    double* coords = (double*)slurp(f, sizeof(double) * 2 * (size_t)np);
    int32_t* mat = (int32_t*)slurp(f, sizeof(int32_t) * (size_t)np);
    fclose(f);

    /* the model: unit square, n × n Q1-P0, free slip, two materials */
    StubMesh mesh;
    memset(&mesh, 0, sizeof mesh);
    mesh.dim = 2;
    mesh.max[0] = mesh.max[1] = 1.0;
    mesh.sizes[0] = mesh.sizes[1] = (unsigned)n;
    mesh.grid.nDims = 2;
    mesh.grid.sizes = mesh.sizes;
    mesh.gridp = &mesh.grid;
    const unsigned nnode = (unsigned)((n + 1) * (n + 1)), nel = (unsigned)(n * n);
    StubFeVariable vel, pres;
    memset(&vel, 0, sizeof vel);
    memset(&pres, 0, sizeof pres);
    vel.base.feMesh = (FeMesh*)&mesh;
    vel.base.fieldComponentCount = 2;
    vel.nnodes = nnode;
    vel.values = (double*)calloc((size_t)nnode * 2, sizeof(double));
    vel.bcmask = (uint8_t*)calloc(nnode, 1);
    for (unsigned i = 0; i < nnode; i++) {  /* velocityBCs.freeslip.xml */
        const unsigned ix = i % (unsigned)(n + 1), iy = i / (unsigned)(n + 1);
        if (ix == 0 || ix == (unsigned)n) vel.bcmask[i] |= 1;
        if (iy == 0 || iy == (unsigned)n) vel.bcmask[i] |= 2;
    }
    pres.base.feMesh = (FeMesh*)&mesh;
    pres.base.fieldComponentCount = 1;
    pres.nnodes = nel;
    pres.values = (double*)calloc(nel, sizeof(double));
    SolutionVector usv, psv;
    memset(&usv, 0, sizeof usv);
    memset(&psv, 0, sizeof psv);
    usv.vector = StubVec_New();
    usv.feVariable = (FeVariable*)&vel;
    psv.vector = StubVec_New();
    psv.feVariable = (FeVariable*)&pres;

    BuoyancyForceTerm_MaterialExt ext0 = {0.0, 1.0}, ext1 = {0.0, 1.01};
    Materials_Register* mr = StubMaterials_Register_New();
    StubMaterials_Register_Add(mr, (Material*)material("matrixViscosity", 1.0, &ext0));
    StubMaterials_Register_Add(mr, (Material*)material("inclusionViscosity", 100.0, &ext1));
    double gHat[3] = {0.0, -1.0, 0.0};
    BuoyancyForceTerm bft;
    memset(&bft, 0, sizeof bft);
    bft.type = "BuoyancyForceTerm";
    bft.gravity = 1.0;
    bft.gHat = gHat;
    StubSwarm swarm;
    memset(&swarm, 0, sizeof swarm);
    swarm.base.particleLocalCount = (Particle_Index)np;
    swarm.points = (MaterialPoint*)calloc((size_t)np, sizeof(MaterialPoint));
    for (int64_t i = 0; i < np; i++) {
        swarm.points[i].coord[0] = coords[2 * i];
        swarm.points[i].coord[1] = coords[2 * i + 1];
        swarm.points[i].materialIndex = (Material_Index)mat[i];
    }
    int preconditioner_stand_in = 0;

    Stg_ComponentFactory cf;
    cf.LCRegister = StubLiveComponentRegister_New();
    FiniteElementContext context;
    memset(&context, 0, sizeof context);
    context.CF = &cf;
    context.materials_Register = mr;
    StubLiveComponentRegister_Add(cf.LCRegister, "context", &context);
    StubLiveComponentRegister_Add(cf.LCRegister, "materialSwarm", &swarm);
    StubLiveComponentRegister_Add(cf.LCRegister, "buoyancyForceTerm", &bft);
    StubLiveComponentRegister_Add(cf.LCRegister, "preconditioner", &preconditioner_stand_in);
    /* the deck's <struct name="uzawa"> */
    StubDictionary_Set("uzawa", "Context", "context");
    StubDictionary_Set("uzawa", "tolerance", "1e-5");
    StubDictionary_Set("uzawa", "maxIterations", "1000");
    StubDictionary_Set("uzawa", "Preconditioner", "preconditioner");
    StubDictionary_Set("uzawa", "MaterialPointsSwarm", "materialSwarm");
    StubDictionary_Set("uzawa", "BuoyancyForceTerm", "buoyancyForceTerm");

    Stokes_SLE sle;
    memset(&sle, 0, sizeof sle);
    sle.context = &context;
    sle.uSolnVec = &usv;
    sle.pSolnVec = &psv;

    /* plugin load: <Name>_Register, then the component type a deck selects */
    PluginsManager* pm = StubPluginsManager_New();
    Underworld_StokesGPU_Register(pm);
    Stg_Component_DefaultConstructorFunction* codeletNew = StubPluginsManager_Get(pm, Underworld_StokesGPU_Type);
    Stg_Component* codelet = codeletNew ? (Stg_Component*)codeletNew((Name) "StokesGPU") : NULL;
    Stg_Component_DefaultConstructorFunction* solverNew = Stg_ComponentRegister_Get(
        Stg_ComponentRegister_Get_ComponentRegister(), "Stokes_SLE_UzawaSolverGPU", (Name) "0");
    if (!codelet || !solverNew) {
        fprintf(stderr, "plugin registration failed\n");
        return 1;
    }
    printf("plugin %s solver-type registered\n", codelet->type);
    fflush(stdout);
    SLE_Solver* solver = (SLE_Solver*)solverNew((Name) "uzawa");
    solver->_assignFromXML(solver, &cf, NULL);
    solver->_solverSetup(solver, &sle);
    solver->_solve(solver, &sle);

    Stokes_SLE_UzawaSolverGPU* gs = (Stokes_SLE_UzawaSolverGPU*)solver;
    PetscInt nu = 0, npv = 0;
    VecGetLocalSize(usv.vector, &nu);
    VecGetLocalSize(psv.vector, &npv);
    printf("outer %d inner %d rel_residual %.3e free_u %d p %d\n", gs->stats.outer_iterations,
           gs->stats.inner_iterations, gs->stats.rel_residual, (int)nu, (int)npv);
    FILE* o = fopen(argv[2], "wb");
    fwrite(vel.values, sizeof(double), (size_t)nnode * 2, o);
    fwrite(pres.values, sizeof(double), nel, o);
    PetscScalar* ua = NULL;
    VecGetArray(usv.vector, &ua);
    fwrite(ua, sizeof(double), (size_t)nu, o);
    VecRestoreArray(usv.vector, &ua);
    fclose(o);
    solver->_destroy(solver, NULL);
    return 0;
}
