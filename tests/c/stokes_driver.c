/* C host driver: reads a sinker problem (binary), solves it through the plugin's C host
 * side (gale_b200/host/stokes_gpu_host.c) and writes u, p.  Used by tests/test_c_host.py. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../gale_b200/host/stokes_gpu_host.h"

static void* slurp(FILE* f, size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (bytes && fread(p, 1, bytes, f) != bytes) { fprintf(stderr, "short read\n"); exit(2); }
    return p;
}

int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]); return 2; }
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    gale_stokes_view v;
    memset(&v, 0, sizeof v);
    int32_t n;
    if (fread(&n, 4, 1, f) != 1) return 2;
    v.mesh.dim = 2;
    v.mesh.elements[0] = v.mesh.elements[1] = n;
    v.mesh.elements[2] = 1;
    v.mesh.max[0] = v.mesh.max[1] = 1.0;
    if (fread(&v.n_points, 8, 1, f) != 1) return 2;
    v.coords = (const double*)slurp(f, sizeof(double) * 2 * v.n_points);
    v.material = (const int32_t*)slurp(f, sizeof(int32_t) * v.n_points);
    fclose(f);
    /* free slip: vx on left/right, vy on bottom/top (velocityBCs.freeslip.xml) */
    v.bc.fixed[0][0] = v.bc.fixed[1][0] = 1;
    v.bc.fixed[2][1] = v.bc.fixed[3][1] = 1;
    v.n_materials = 2;
    v.materials[0].n_rheologies = 1;
    v.materials[0].rheology[0].kind = GG_RHEO_MATERIAL_VISCOSITY;
    v.materials[0].rheology[0].eta0 = 1.0;
    v.materials[0].density = 1.0;
    v.materials[1] = v.materials[0];
    v.materials[1].rheology[0].eta0 = 100.0;
    v.materials[1].density = 1.01;
    v.force.gravity = 1.0;
    v.force.g_hat[1] = -1.0;

    gg_uzawa_params prm = StokesGPU_DefaultParams();
    gg_uzawa_stats st;
    int64_t nnode = (int64_t)(n + 1) * (n + 1), nel = (int64_t)n * n;
    double* u = calloc(nnode * 2, sizeof(double));
    double* p = calloc(nel, sizeof(double));
    gg_handle* h = NULL;
    int rc = StokesGPU_Solve(&h, &v, &prm, u, p, &st);
    if (rc != GG_OK) {
        fprintf(stderr, "StokesGPU_Solve: %d %s\n", rc, h ? gg_last_error(h) : "");
        return 1;
    }
    printf("outer %d inner %d rel_residual %.3e\n", st.outer_iterations, st.inner_iterations, st.rel_residual);
    FILE* o = fopen(argv[2], "wb");
    fwrite(u, sizeof(double), nnode * 2, o);
    fwrite(p, sizeof(double), nel, o);
    fclose(o);
    gg_destroy(h);
    return 0;
}
