// gg_kernels.cuh -- declarations shared by the .cu translation units and the inline
// device helpers of the regular Q1 mesh.
#pragma once

#include "gg_handle.h"
#include "gg_internal.cuh"

namespace gg {

int num_sms();
int grid_for(int64_t n, int block);
// Record a message for gg_last_error and return the status code (gg_api.cu).
int set_error(Handle& H, int code, const std::string& msg);

// Vertex coordinate, CartesianGenerator_CalcGeom (StgDomain/Mesh/src/
// CartesianGenerator.cxx:2178-2215), with explicit roundings (no FMA contraction).
__device__ __forceinline__ double vert_coord_d(const MeshK& mk, int d, int i) {
    if (i == 0) return mk.min[d];
    if (i == mk.n[d]) return mk.max[d];
    return __dadd_rn(mk.min[d], __dmul_rn(__ddiv_rn((double)i, (double)mk.n[d]),
                                          __dsub_rn(mk.max[d], mk.min[d])));
}

__device__ __forceinline__ void elem_ijk(const MeshK& mk, int64_t e, int* ijk) {
    ijk[0] = (int)(e % mk.n[0]);
    const int64_t r = e / mk.n[0];
    ijk[1] = (int)(r % mk.n[1]);
    ijk[2] = (int)(r / mk.n[1]);
}

template <int DIM>
__device__ __forceinline__ int64_t elem_node(const MeshK& mk, const int* ijk, int a) {
    const int i = ijk[0] + (a & 1), j = ijk[1] + ((a >> 1) & 1);
    const int k = DIM == 3 ? ijk[2] + ((a >> 2) & 1) : 0;
    return i + (int64_t)mk.nn[0] * (j + (int64_t)mk.nn[1] * k);
}

// ---- host drivers ------------------------------------------------------------------
int64_t locate_and_sort(Handle& H);
// out = exclusive prefix sum of in[0..n) on the device; *total_host = the sum.
void exclusive_scan_i32(Handle& H, const int32_t* in, int32_t* out, int64_t n, DBuf& tmp, int32_t* total_host);
// DVCWeights of the located points (prm = nullptr) or PCDVC population control with the
// rebuilt and re-located point set (gg_dvc.cu).  GG_OK or a status (message set).
int dvc_update(Handle& H, const gg_pcdvc_params* prm, gg_pcdvc_stats* stats);

// Per-point rheology + moments + force + diagonals.  precision GG_PRECISION_FP64 fills
// mom64/kdiag64/sdiag/f/eta; GG_PRECISION_MIXED additionally fills mom32/kdiag32 with
// the FP32 rheology and FP32 element sums.  Returns 0 or a GG_ERR code.
int build_operator(Handle& H, int precision, int prev, const double* d_prev_u,
                   const double* d_prev_p);

// y = K x on one level (level mesh mk, moments mom, bc mask); y is accumulated and must
// be zero on entry; BC rows of y are left untouched (zero).  FP64 sums every node's
// element terms in a fixed order (one launch per element parity class: the same bits on
// every run); FP32 accumulates with atomics in arrival order.
// energy (nullable): per-block partials of Σ_e x_eᵀ K_e x_e.
template <typename R>
void apply_K(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y,
             cudaStream_t st);
void apply_G(const Handle& H, const double* p, double* y, cudaStream_t st);
void apply_GT(const Handle& H, const double* u, double* q, cudaStream_t st);

// Krylov / Uzawa (gg_solve.cu)
// Sizes the reduction scratch and clears its counters (before the first Krylov kernel).
void prepare_krylov_scratch(Handle& H);
int uzawa_solve(Handle& H, const gg_uzawa_params& prm, gg_uzawa_stats& st);
int inner_solve(Handle& H, const gg_uzawa_params& prm, const double* b, double* x,
                double rtol, int maxit, int* iters, bool warm = false);
void release_graphs(Handle& H);

// Multigrid (gg_mg.cu): hierarchy for the current build; z = M⁻¹ b on level l.
// Chebyshev–Jacobi smoother of degree `degree` on [0.1, 1.1]·λ_max(D⁻¹A):
// x₀ = D⁻¹r/θ, then d_k = c1[k] d_{k−1} + c2[k] D⁻¹ r_k.
struct ChebCoef {
    float inv_theta;
    float c1[8], c2[8];
};
ChebCoef cheb_coef(double lmax_est, int degree);
// Chebyshev degree of level l's smoother (the configured degree on the fine level)
int level_degree(const Handle& H, size_t l);
int mg_setup(Handle& H);
int coarse_inverse_copy(Handle& H, int64_t* n, float* inv, double* op);
void vcycle(Handle& H, size_t l, const float* b, float* x, const int32_t* done);
void mg_restrict(Handle& H, size_t l, const float* fine, float* coarse, const int32_t* done);
void mg_prolong_add(Handle& H, size_t l, const float* coarse, float* fine, const int32_t* done);
// x = K32⁻¹ b by the multigrid flexible CG (FP32, ‖r‖ ≤ rtol‖b‖)
int fcg_mg_solve(Handle& H, const float* b, float* x, double rtol, int maxit, int* iters);
// The same solve as one persistent cooperative kernel (gg_fused.cu); returns 1 when the
// hierarchy does not fit it (no dense coarse level, > 8 levels, degree outside 2..4).
int run_fcg_fused(Handle& H, const float* b, float* x, double rtol, int maxit, int* iters);
bool fused_fcg_enabled();
// The mixed-path Uzawa solve (multigrid inner solves) as one cooperative launch; 1 when it
// does not apply (the caller runs the host-driven loop), else the solve's status with S's
// iteration counts, residuals and launch figures filled and H.fail_where set on failure.
int run_uzawa_fused(Handle& H, const gg_uzawa_params& prm, gg_uzawa_stats& S);
bool fused_uzawa_enabled();
// µs per grid barrier of the persistent kernels (measurement, gg_fused.cu)
int time_grid_barrier(int blocks_per_sm, int iters, double* us);
// the grid barrier's give-up path with a short limit (block 0 never arrives)
int check_barrier_timeout(int spin_limit, int* gave_up);

// Learned coarse correction (gg_learned.cu)
bool learned_ready(Handle& H);
int learned_base(Handle& H);  // GG_LEARN_BASE_* of the current weights, −1 without a network
void jacobi_precond(Handle& H, const float* r, float* z, const int32_t* done);
void learned_prepare(Handle& H);
void learned_correction(Handle& H, const float* r, float* z, const int32_t* done);
int learned_set_level(Handle& H, int level);
int64_t learned_param_count(Handle& H);
void learned_set_weights(Handle& H, const float* w);
void learned_get_weights(Handle& H, float* w);
int learned_eval(Handle& H, int B, const float* xin, const float* tgt, const float* w, float* y, float* grad,
                 double* loss);
int learned_train(Handle& H, const gg_learn_params& P, gg_learn_stats& st);

// prev_u = u + BC values, prev_p = q (gg_api2.cu)
void store_solution(Handle& H);
// store_solution, then the nodal velocity with its boundary values and the element
// pressure to host arrays (gg_api.cu)
void download_solution(Handle& H, double* u, double* p);

// Batched CTA solver (gg_cta.cu): one CTA per problem, one launch for the batch.
bool cta_batch_supported(const gg_uzawa_params& prm);
int cta_batch_solve(std::vector<Handle*>& hs, const gg_uzawa_params& prm, double* const* u_out,
                    double* const* p_out, gg_uzawa_stats* stats, int32_t* status);

// Advection (gg_advect.cu)
int advect(Handle& H, double dt, int order, const double* d_u, double* d_out);

}  // namespace gg
