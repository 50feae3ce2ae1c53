/* dvc_oracle.h -- TEST INFRASTRUCTURE ONLY: discrete-Voronoi weights and population
 * control of one element (see dvc_oracle.c for the reference functions restated).      */
#ifndef DVC_ORACLE_H
#define DVC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double upper_t, lower_t;          /* PCDVC upperT / lowerT (% of the element volume) */
    int32_t max_splits, max_deletions;
    int32_t split_in_interface_cells, delete_in_interface_cells;
} od_pcdvc_params;

/* Voronoi regions on the res[0]×res[1](×res[2]) grid of the element [-1,1]^dim grown from
 * the nump points xi [nump][dim] (element-list order): centroids [nump][dim] and the
 * number of grid cells each point owns (weight = count × cell volume).  0, or < 0 when a
 * grid cell stays unowned or the arguments are out of range.                            */
int od_dvc_cell(int32_t dim, const int32_t* res, int32_t nump, const double* xi, double* cent, int32_t* count);
double od_dvc_cell_volume(int32_t dim, const int32_t* res);

/* Population control of one element without the Inflow branch.  In: the element's points
 * in list order (xi, material, swarm index).  Out (capacity nump + max_splits): the
 * element's list afterwards -- out_src ≥ 0: input slot kept; < 0: a new point split from
 * input slot −1 − out_src, at out_xi (its parent's centroid) -- with each point's
 * centroid and weight from the final Voronoi diagram.                                   */
int od_pcdvc_cell(int32_t dim, const int32_t* res, const od_pcdvc_params* prm, int32_t nump, const double* xi,
                  const int32_t* mat, const int64_t* index, int32_t* out_src, double* out_xi, double* out_cent,
                  double* out_w, int32_t* n_out, int32_t* n_split, int32_t* n_delete);

#ifdef __cplusplus
}
#endif
#endif
