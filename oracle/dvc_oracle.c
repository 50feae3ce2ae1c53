/* dvc_oracle.c -- TEST INFRASTRUCTURE ONLY (never part of the product path).
 *
 * FP64 C restatement of the discrete-Voronoi integration weights and the population
 * control of one element, for the parity tests of gale_b200/csrc/gg_dvc.cu:
 *   _DVCWeights_ConstructGrid / _ConstructGrid2D   DVCWeights.cxx:525-620
 *   _DVCWeights_CreateVoronoi / 2D                 DVCWeights.cxx:693-786
 *   _DVCWeights_ClaimCells / 2D                    DVCWeights.cxx:260-398
 *   _DVCWeights_UpdateBchain / 2D                  DVCWeights.cxx:420-522
 *   _DVCWeights_DistanceTest / 2D                  DVCWeights.cxx:629-634
 *   _DVCWeights_GetCentroids / 2D                  DVCWeights.cxx:202-258
 *   _PCDVC_Calculate3D / 2D (Inflow = False)       PCDVC.cxx:656-1090, 1092-1512
 *   Swarm_RemoveParticleFromCell                   SwarmClass.cxx:976-992
 * (all paths relative to the reference's PICellerator/ and StgDomain/ trees).
 *
 * The element grid keeps the reference's cell numbering (x fastest, then y, then z) and
 * the neighbour order S, N, E, W, U, D of the boundary update.  Cell centres are formed by
 * the same repeated additions as the reference's grid constructor.  The arithmetic is
 * plain double with -ffp-contract=off, like the reference's x86-64 build.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dvc_oracle.h"

/* cell centres along one axis: X = x0 − d/2, then X += d before each cell */
static void centres(int n, double lo, double hi, double* c) {
    const double D = hi - lo;
    const double d = D / n;
    double X = lo - d / 2.0;
    for (int i = 0; i < n; i++) {
        X = X + d;
        c[i] = X;
    }
}

static double dist_test(int dim, const double* c0, const double* p1, const double* p2) {
    double v = (p1[0] + p2[0] - c0[0] - c0[0]) * (p1[0] - p2[0]) + (p1[1] + p2[1] - c0[1] - c0[1]) * (p1[1] - p2[1]);
    if (dim == 3) v = v + (p1[2] + p2[2] - c0[2] - c0[2]) * (p1[2] - p2[2]);
    return v;
}

typedef struct {
    int* claimed;  /* cells claimed in the last pass */
    int nclaimed;
    int* bound;    /* boundary cells to contest in the next pass */
    int nbound;
} chain_t;

int od_dvc_cell(int32_t dim, const int32_t* res, int32_t nump, const double* xi, double* cent, int32_t* count) {
    if (dim != 2 && dim != 3) return -1;
    if (nump < 1) return -2;
    const int nx = res[0], ny = res[1], nz = dim == 3 ? res[2] : 1;
    const int ncell = nx * ny * nz;
    double cx[64], cy[64], cz[64];
    if (nx > 64 || ny > 64 || nz > 64) return -3;
    centres(nx, -1.0, 1.0, cx);
    centres(ny, -1.0, 1.0, cy);
    if (dim == 3) centres(nz, -1.0, 1.0, cz);
    const double dx = (1.0 - -1.0) / nx, dy = (1.0 - -1.0) / ny, dz = dim == 3 ? (1.0 - -1.0) / nz : 1.0;
    int* owner = (int*)malloc(sizeof(int) * ncell);
    char* done = (char*)calloc(ncell, 1);
    chain_t* ch = (chain_t*)calloc(nump, sizeof(chain_t));
    for (int c = 0; c < ncell; c++) owner[c] = -1;
    for (int i = 0; i < nump; i++) {
        ch[i].claimed = (int*)malloc(sizeof(int) * (ncell + 1));
        ch[i].bound = (int*)malloc(sizeof(int) * (6 * ncell + 1));
    }
    /* boundary update: neighbours S, N, E, W, U, D of the cells just claimed that the point
       does not own, each once */
#define UPDATE_BCHAIN(I)                                                                     \
    do {                                                                                     \
        chain_t* b = &ch[I];                                                                 \
        b->nbound = 0;                                                                       \
        for (int q = 0; q < b->nclaimed; q++) {                                              \
            const int c0 = b->claimed[q];                                                    \
            const int ci = c0 % nx, cj = (c0 / nx) % ny, ck = c0 / (nx * ny);               \
            int nb[6];                                                                       \
            nb[0] = cj > 0 ? c0 - nx : -2;                                                   \
            nb[1] = cj < ny - 1 ? c0 + nx : -2;                                              \
            nb[2] = ci < nx - 1 ? c0 + 1 : -2;                                               \
            nb[3] = ci > 0 ? c0 - 1 : -2;                                                    \
            nb[4] = (dim == 3 && ck < nz - 1) ? c0 + nx * ny : -2;                           \
            nb[5] = (dim == 3 && ck > 0) ? c0 - nx * ny : -2;                                \
            for (int k = 0; k < (dim == 3 ? 6 : 4); k++) {                                   \
                const int c1 = nb[k];                                                        \
                if (c1 != -2 && owner[c1] != (I) && !done[c1]) {                             \
                    b->bound[b->nbound++] = c1;                                              \
                    done[c1] = 1;                                                            \
                }                                                                            \
            }                                                                                \
        }                                                                                    \
        for (int q = 0; q < b->nbound; q++) done[b->bound[q]] = 0;                           \
    } while (0)

    for (int i = 0; i < nump; i++) {
        const double* p = xi + (int64_t)i * dim;
        int k = (int)((p[0] - -1.0) / dx);
        int j = (int)((p[1] - -1.0) / dy);
        int l = dim == 3 ? (int)((p[2] - -1.0) / dz) : 0;
        if (k == nx) k--;
        if (j == ny) j--;
        if (dim == 3 && l == nz) l--;
        const int c = k + j * nx + l * nx * ny;
        owner[c] = i;
        ch[i].claimed[0] = c;
        ch[i].nclaimed = 1;
        UPDATE_BCHAIN(i);
    }
    int claimed = 1;
    while (claimed != 0) {
        claimed = 0;
        for (int i = 0; i < nump; i++) {
            chain_t* b = &ch[i];
            b->nclaimed = 0;
            for (int q = 0; q < b->nbound; q++) {
                const int c = b->bound[q];
                if (owner[c] == -1) {
                    b->claimed[b->nclaimed++] = c;
                    owner[c] = i;
                } else if (owner[c] != i) {
                    const int ci = c % nx, cj = (c / nx) % ny, ck = c / (nx * ny);
                    const double c0[3] = {cx[ci], cy[cj], dim == 3 ? cz[ck] : 0.0};
                    const double* p1 = xi + (int64_t)owner[c] * dim;
                    const double* p2 = xi + (int64_t)i * dim;
                    if (dist_test(dim, c0, p1, p2) > 0.0) {
                        b->claimed[b->nclaimed++] = c;
                        owner[c] = i;
                    }
                }
            }
            claimed += b->nclaimed;
            UPDATE_BCHAIN(i);
        }
    }
#undef UPDATE_BCHAIN
    /* centroids: cell centres summed in cell order */
    for (int i = 0; i < nump; i++) {
        count[i] = 0;
        for (int d = 0; d < dim; d++) cent[(int64_t)i * dim + d] = 0.0;
    }
    int rc = 0;
    for (int c = 0; c < ncell; c++) {
        const int p = owner[c];
        if (p < 0) {
            rc = -4;
            continue;
        }
        const int ci = c % nx, cj = (c / nx) % ny, ck = c / (nx * ny);
        cent[(int64_t)p * dim + 0] += cx[ci];
        cent[(int64_t)p * dim + 1] += cy[cj];
        if (dim == 3) cent[(int64_t)p * dim + 2] += cz[ck];
        count[p]++;
    }
    for (int i = 0; i < nump; i++)
        if (count[i] != 0)
            for (int d = 0; d < dim; d++) cent[(int64_t)i * dim + d] /= count[i];
    for (int i = 0; i < nump; i++) {
        free(ch[i].claimed);
        free(ch[i].bound);
    }
    free(ch);
    free(done);
    free(owner);
    return rc;
}

double od_dvc_cell_volume(int32_t dim, const int32_t* res) {
    const double dx = (1.0 - -1.0) / res[0], dy = (1.0 - -1.0) / res[1];
    if (dim == 2) return dx * dy;
    const double dz = (1.0 - -1.0) / res[2];
    return dx * dy * dz;
}

int od_pcdvc_cell(int32_t dim, const int32_t* res, const od_pcdvc_params* prm, int32_t nump, const double* xi,
                  const int32_t* mat, const int64_t* index, int32_t* out_src, double* out_xi, double* out_cent,
                  double* out_w, int32_t* n_out, int32_t* n_split, int32_t* n_delete) {
    const double da = od_dvc_cell_volume(dim, res);
    double* cent = (double*)malloc(sizeof(double) * (size_t)(nump + prm->max_splits + 1) * dim);
    int32_t* cnt = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nump + prm->max_splits + 1));
    int rc = od_dvc_cell(dim, res, nump, xi, cent, cnt);
    if (rc) {
        free(cent);
        free(cnt);
        return rc;
    }
    const double vol = dim == 3 ? 8.0 : 4.0;
    const double maxW = prm->upper_t * vol / 100.0, minW = prm->lower_t * vol / 100.0;
    int maxDeletions = prm->max_deletions, maxSplits = prm->max_splits;
    for (int i = 0; i < nump; i++)
        if (mat[i] != mat[0]) {
            if (!prm->delete_in_interface_cells) maxDeletions = 0;
            if (!prm->split_in_interface_cells) maxSplits = 0;
            break;
        }
    /* split list in list order; delete list sorted by decreasing swarm index */
    int* split = (int*)malloc(sizeof(int) * nump);
    int* del = (int*)malloc(sizeof(int) * nump);
    int ns = 0, nd = 0;
    for (int i = 0; i < nump; i++) {
        const double w = cnt[i] * da;
        if (w > maxW) split[ns++] = i;
        if (w < minW) del[nd++] = i;
    }
    for (int a = 1; a < nd; a++)  /* insertion sort, decreasing index */
        for (int b = a; b > 0 && index[del[b - 1]] < index[del[b]]; b--) {
            const int t = del[b];
            del[b] = del[b - 1];
            del[b - 1] = t;
        }
    if (maxDeletions > nump - 4) maxDeletions = nump / 2;
    const int nsplit = maxSplits > ns ? ns : maxSplits;
    const int ndel = maxDeletions > nd ? nd : maxDeletions;
    /* the element's list after the splits (appended) and the deletions (swap with last) */
    const int cap = nump + nsplit;
    int32_t* list = (int32_t*)malloc(sizeof(int32_t) * cap);   /* ≥ 0: input slot; < 0: −1 − split number */
    double* lxi = (double*)malloc(sizeof(double) * (size_t)cap * dim);
    int m = 0;
    for (int i = 0; i < nump; i++) {
        list[m] = i;
        memcpy(lxi + (size_t)m * dim, xi + (size_t)i * dim, sizeof(double) * dim);
        m++;
    }
    for (int s = 0; s < nsplit; s++) {
        list[m] = -1 - s;
        memcpy(lxi + (size_t)m * dim, cent + (size_t)split[s] * dim, sizeof(double) * dim);
        m++;
    }
    for (int q = 0; q < ndel; q++) {
        int pos = -1;
        for (int k = 0; k < m; k++)
            if (list[k] == del[q]) pos = k;
        list[pos] = list[m - 1];
        memcpy(lxi + (size_t)pos * dim, lxi + (size_t)(m - 1) * dim, sizeof(double) * dim);
        m--;
    }
    if (nsplit || ndel) {
        /* the reference stops the run when fewer than 3 points are left (PCDVC.cxx:1049) */
        rc = m < 3 ? -5 : od_dvc_cell(dim, res, m, lxi, cent, cnt);
        if (rc) m = 0;
    }
    for (int k = 0; k < m; k++) {
        out_src[k] = list[k] >= 0 ? list[k] : -1 - split[-1 - list[k]];
        memcpy(out_xi + (size_t)k * dim, lxi + (size_t)k * dim, sizeof(double) * dim);
        memcpy(out_cent + (size_t)k * dim, cent + (size_t)k * dim, sizeof(double) * dim);
        out_w[k] = cnt[k] * da;
    }
    *n_out = m;
    *n_split = nsplit;
    *n_delete = ndel;
    free(lxi);
    free(list);
    free(del);
    free(split);
    free(cnt);
    free(cent);
    return rc;
}
