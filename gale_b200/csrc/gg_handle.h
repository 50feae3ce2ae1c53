// gg_handle.h -- host-side state of one Stokes problem (opaque gg_handle of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "gg_internal.cuh"

namespace gg {

// Device scalars of one Krylov solve (written and read by kernels only).
struct KrylovScalars {
    double rz, rz_old, pAp, alpha, beta;
    double rnorm, rnorm0, ttol;
    double partial_pad[8];
    int32_t done, iterations, failed, maxit;
};

// Device memory of the handle buffers (gg_alloc.cu): pooled up to 4 MB, cudaMalloc above.
void* dev_alloc(size_t bytes, int* dev_out);
void dev_free(void* p, size_t bytes, int dev);

// A device buffer with RAII.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int dev = -1;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) dev_free(p, bytes, dev);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t nbytes) {
        if (nbytes <= bytes && p) return;
        release();
        size_t b = nbytes ? nbytes : 16;
        p = dev_alloc(b, &dev);
        bytes = b;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// One multigrid level (level 0 = the fine mesh).
struct MGLevel {
    MeshK mk{};
    int64_t nnode = 0, nel = 0, ndof = 0;
    DBuf own_mom64, own_mom32, own_bcmask;   // coarse levels own their operator
    DBuf invdiag;                            // FP32 inverse Jacobi diagonal (0 on BC dofs)
    const double* mom64 = nullptr;           // effective pointers (level 0: the fine operator)
    const float* mom32 = nullptr;
    const uint8_t* bcmask = nullptr;
    DBuf x, b, r, d, t;                      // FP32 work vectors [dim*nnode]
    double lambda_max = 0.0;
};

struct Handle {
    gg_mesh_desc desc{};
    MeshK mk{};
    int dim = 0, nm = 0;
    int64_t nel = 0, nnode = 0, ndof = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::string fail_where;  // stage at which the last Uzawa solve stopped early

    // mesh-level data
    DBuf bcmask, bcval, T;
    bool has_T = false, has_bc = false;
    int64_t nfree = 0;  // velocity dofs without a Dirichlet condition
    gg_body_force force{};
    int n_materials = 0;
    std::vector<gg_material> materials;
    std::vector<gg_material> h_materials;  // staging copy for the async upload
    DBuf d_materials;

    // points
    int64_t np = 0, np_in = 0;
    DBuf coords, mat_in, ps_in, cell, perm, cell_s, xi_s, mat_s, ps_s, eta_s, incr_s, yld_s;
    DBuf offsets, fill, scan_tmp, flag;
    bool located = false;
    // integration weights (gg_dvc.cu): with GG_WEIGHTS_DVC, xi_s holds the Voronoi
    // centroids and w_s the volumes of the sorted points once dvc_valid; xi_pts keeps
    // the material points' own ξ, from which the diagrams grow
    gg_weights weights{GG_WEIGHTS_CONSTANT, {10, 10, 10}};
    bool dvc_valid = false;
    DBuf w_s, xi_pts, dvc_cent, dvc_keep, dvc_err, dvc_nsplit, dvc_ndel, dvc_parent, dvc_new, dvc_scan, dvc_scan2;

    // operator
    DBuf mom64, mom32, kdiag64, kdiag32, sdiag, hvec, f;
    DBuf kcorner, fcorner;  // per-element corner terms of the diagonal / force (build scratch)
    bool built = false;
    int built_precision = -1;
    DBuf prev_u, prev_p;  // previous solution read by the yield laws (SoA / element)

    // solver work
    DBuf u, vstar, ftmp, ub, q, qtmp, r, s;           // FP64
    DBuf cg_b, cg_r, cg_z, cg_p, cg_Ap, cg_x;        // FP64 CG
    DBuf r32, cgr32, z32, p32, Ap32, e32;             // FP32 inner CG
    DBuf scal, red;                                   // KrylovScalars, reduction scratch
    KrylovScalars* h_scal = nullptr;                  // pinned mirror
    std::vector<std::unique_ptr<MGLevel>> mg;
    bool mg_ready = false;
    int64_t build_gen = 0;  // incremented by every operator build (graphs bake in its scalars)
    int64_t mg_gen = -1;    // build generation the hierarchy was set up for
    DBuf coarse_inv;        // dense inverse of the coarsest operator (FP32, [n][ld])
    DBuf mg_part, mg_dense; // power-iteration partials; FP64 columns of the coarsest operator
    int64_t coarse_n = 0;   // 0: no dense coarse solve (Chebyshev on the coarsest level)
    int64_t coarse_ld = 0;  // row stride of coarse_inv (coarse_n rounded up to 4)
    int mg_degree = 2;      // Chebyshev degree of the smoother
    int build_shape[2] = {-1, -1};  // autotuned CTA shape of the FP64 / FP32 moment build
    // persistent multigrid FCG (gg_fused.cu): level table for the current hierarchy
    DBuf fused_tab, fused_part, fused_bar, fused_out;
    std::vector<unsigned char> fused_host;
    int64_t fused_gen = -2;  // mg_gen the table was written for
    const float* fused_r = nullptr;  // FCG residual / preconditioned vector baked into it
    const float* fused_z = nullptr;
    const float* fused_x = nullptr;  // the launch's solution and right-hand side (alignment)
    const float* fused_b = nullptr;
    int fused_phases = 0;            // grid barriers per iteration
    // the batched CTA solver's own hierarchy (gg_cta.cu): level buffers and λ_max per level
    std::vector<std::unique_ptr<MGLevel>> cta_levels;
    DBuf cta_lam;
    double fused_bytes_it = 0.0;     // algorithmic bytes of one iteration (every phase)
    // measurement of the persistent launches of the current Uzawa solve (events around
    // each cooperative launch on the handle's stream)
    cudaEvent_t evf0 = nullptr, evf1 = nullptr;
    int fused_launches_acc = 0, fused_its_acc = 0;
    double fused_ms_acc = 0.0;
    // dofs per block of the persistent kernel's grid: 256 for a problem solved alone; 1024
    // when gg_solve_batch runs it beside others (fewer blocks per problem, more problems
    // resident at once: 512 sinkers 94 -> 107 solves/s, a lone 256x64 problem 10 % slower)
    int fused_dofs_per_block = 256;
    // the multigrid refinement sweeps of this Uzawa solve aim at 1e-5 instead of 1e-4 once an
    // inner solve has needed more than two sweeps (set in inner_solve, reset per Uzawa solve)
    bool tight_sweeps = false;
    // learned coarse correction (gg_learned.cu)
    std::shared_ptr<struct LearnedState> learned;
    bool nn_ready = false;
    bool nn_enabled = true;    // cleared after repeated stagnation (fallback to multigrid)
    int fallbacks = 0;         // learned → multigrid fallbacks taken in the current solve
    int calib_mg = 0, calib_nn = 0;  // FCG iterations of the calibration solves (learned vs MG)
    int nn_verdict = -1;       // judge's verdict on the current weights: -1 not judged, 0 off, 1 on
    int nn_level = 2;       // hierarchy level the network acts on
    DBuf mg_xs, mg_xk, mg_xt;  // FP32 fine-level scratch of the training data generator

    // CUDA graphs keyed by solver variant
    std::map<std::string, cudaGraphExec_t> graphs;
    std::map<std::string, int64_t> graph_nodes;  // kernel nodes per captured graph
    double last_solve_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    // last solution (for advection and Picard)
    bool have_solution = false;
    int32_t max_material = 0;       // largest material index of the points
    mutable int64_t kernel_launches = 0;    // launches of this library's kernels (graph nodes counted)
    int64_t launches_at_build = 0;          // counter value when the last build started
    int64_t stats_gen = -1;                 // build generation the last solve statistics covered
    DBuf picard_prev, picard_part;
};

}  // namespace gg

// The opaque handle of the C ABI.
struct gg_handle {
    gg::Handle H;
};
