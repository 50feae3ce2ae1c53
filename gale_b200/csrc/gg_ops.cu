// gg_ops.cu -- matrix-free K, G and Gᵀ on sm_100a.
//
// K apply (replaces MatMult with the assembled k_matrix of __StiffnessMatrix_NewAssemble,
// StgFEM/SLE/SystemSetup/src/StiffnessMatrix.cxx:2016-2200).  One thread per element, a
// block per tile of 32×4×2 elements (32×8 in 2D), x fastest:
//   1. gather the 2^dim nodal values per component (coalesced along x),
//   2. Walsh–Hadamard transform → modal coefficients m[c][S] = Σ_a Π_{d∈S} s_d(a) u_a,c,
//   3. velocity gradient ∂u_c/∂x_d = κ_d Σ_{T⊆others(d)} m[c][{d}∪T] ξ^T,
//   4. stress σ = 2ε̇ (viscosity is inside the moments), projected on the test basis
//      through the element moments M[U+T] = Σ_p c_p ξ_p^{U+T},
//   5. inverse transform → y_e, scattered with atomics (BC rows skipped).
// The same pass returns x_eᵀ K_e x_e, so Σ_e gives pᵀKp for CG without a second pass.
// Bandwidth-bound (nodal vectors + n_mom moments per element); no tensor cores.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {

template <int DIM, typename R, bool kEnergy>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 2 : 1)
k_apply_K(MeshK mk, const R* __restrict__ mom, const uint8_t* __restrict__ bcmask,
          const R* __restrict__ x, R* __restrict__ y, double* __restrict__ energy_part,
          const int32_t* __restrict__ done) {
    if (done && *done) return;
    double en = apply_tiles<DIM, R, 0, kEnergy>(mk, mom, bcmask, x, y, blockIdx.x, gridDim.x);
    if (kEnergy) {
        en = block_sum(en);
        if (threadIdx.x == 0) energy_part[blockIdx.x] = en;
    }
}

// The FP32 apply without the energy: 128-thread blocks (32 × 2 × 2 elements in 3D, 32 × 4
// in 2D), four per SM.  Blocks half the size start and finish at staggered times, so one
// block's gathers overlap another's arithmetic more than with 256-thread blocks (64³:
// 12.3 µs against 13.1 µs per launch).
template <int DIM>
__global__ void __launch_bounds__(128, 4)
k_apply_K_small(MeshK mk, const float* __restrict__ mom, const uint8_t* __restrict__ bcmask,
                const float* __restrict__ x, float* __restrict__ y, const int32_t* __restrict__ done) {
    if (done && *done) return;
    apply_tiles<DIM, float, 0, false, DIM == 3 ? 2 : 4, DIM == 3 ? 2 : 1>(mk, mom, bcmask, x, y, blockIdx.x, gridDim.x);
}

// One parity class of the FP64 apply (see apply_tiles_class): 2^dim launches in class
// order make y = K x the same bits on every run.
template <int DIM>
__global__ void __launch_bounds__(256, 1)
k_apply_K_class(MeshK mk, const double* __restrict__ mom, const uint8_t* __restrict__ bcmask,
                const double* __restrict__ x, double* __restrict__ y, const int32_t* __restrict__ done, int color) {
    if (done && *done) return;
    apply_tiles_class<DIM, double, 0, false>(mk, mom, bcmask, x, y, blockIdx.x, gridDim.x, color);
}

int class_grid(const MeshK& mk, int color) {
    const int64_t t = mk.dim == 3 ? class_tiles<3>(mk, color, ApplyTile<3>::X, ApplyTile<3>::Y, ApplyTile<3>::Z)
                                  : class_tiles<2>(mk, color, ApplyTile<2>::X, ApplyTile<2>::Y, ApplyTile<2>::Z);
    const int64_t cap = 8 * (int64_t)num_sms();
    return (int)(t < 1 ? 1 : (t < cap ? t : cap));
}

template <typename R>
void apply_K_ex(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y,
                double* energy_part, int grid, cudaStream_t st, const int32_t* done) {
    if constexpr (sizeof(R) == 8) {
        // FP64: fixed summation order, one launch per parity class.  No caller asks the
        // FP64 apply for element energies (the FP64 CG has its own class kernels).
        if (energy_part) throw CudaError(cudaErrorInvalidValue, "apply_K_ex<double> with energy", __FILE__, __LINE__);
        const int ncls = 1 << mk.dim;
        for (int c = 0; c < ncls; c++) {
            if (mk.dim == 3)
                k_apply_K_class<3><<<class_grid(mk, c), 256, 0, st>>>(mk, mom, bcmask, x, y, done, c);
            else
                k_apply_K_class<2><<<class_grid(mk, c), 256, 0, st>>>(mk, mom, bcmask, x, y, done, c);
        }
    } else {
        // FP32 (multigrid, learned correction): atomics in arrival order
        if (!energy_part) {
            int64_t g = (mk.nel + 127) / 128;
            const int64_t cap = 16 * (int64_t)num_sms();
            g = g < cap ? g : cap;
            if (mk.dim == 3) k_apply_K_small<3><<<(int)g, 128, 0, st>>>(mk, mom, bcmask, x, y, done);
            else k_apply_K_small<2><<<(int)g, 128, 0, st>>>(mk, mom, bcmask, x, y, done);
            return;
        }
        if (mk.dim == 2) k_apply_K<2, R, true><<<grid, 256, 0, st>>>(mk, mom, bcmask, x, y, energy_part, done);
        else k_apply_K<3, R, true><<<grid, 256, 0, st>>>(mk, mom, bcmask, x, y, energy_part, done);
    }
}
template void apply_K_ex<double>(const MeshK&, const double*, const uint8_t*, const double*, double*,
                                 double*, int, cudaStream_t, const int32_t*);
template void apply_K_ex<float>(const MeshK&, const float*, const uint8_t*, const float*, float*,
                                double*, int, cudaStream_t, const int32_t*);

template <typename R>
void apply_K(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y, cudaStream_t st) {
    apply_K_ex<R>(mk, mom, bcmask, x, y, nullptr, apply_grid(mk.nel), st, nullptr);
    GG_CUDA(cudaGetLastError());
}
template void apply_K<double>(const MeshK&, const double*, const uint8_t*, const double*, double*,
                              cudaStream_t);
template void apply_K<float>(const MeshK&, const float*, const uint8_t*, const float*, float*,
                             cudaStream_t);

int apply_grid(int64_t nel) {
    int64_t g = (nel + 255) / 256;
    const int cap = num_sms() * 8;
    return (int)(g < cap ? (g < 1 ? 1 : g) : cap);
}

// ---- G p (P0 pressure → velocity force): node-centric gather, BC rows zero ----------
template <int DIM, typename R>
__global__ void k_apply_G(MeshK mk, const uint8_t* __restrict__ bcmask, const R* __restrict__ p,
                          R* __restrict__ y, R beta) {
    const int64_t nnode = mk.nnode;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nnode;
         n += (int64_t)gridDim.x * blockDim.x) {
        R acc[DIM];
        g_node<DIM, R, false>(mk, p, n, acc);
        const uint8_t bm = bcmask[n];
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            R* yp = &y[(int64_t)c * nnode + n];
            *yp = ((bm >> c) & 1) ? R(0) : (beta == R(0) ? acc[c] : beta * (*yp) + acc[c]);
        }
    }
}

// ---- Gᵀ u (velocity → element): element-centric, all columns --------------------------
template <int DIM, typename R>
__global__ void k_apply_GT(MeshK mk, const R* __restrict__ u, R* __restrict__ q) {
    const int64_t nel = mk.nel;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel;
         e += (int64_t)gridDim.x * blockDim.x)
        q[e] = gt_elem<DIM, R, false>(mk, u, e);
}

void apply_G(const Handle& H, const double* p, double* y, cudaStream_t st) {
    const int g = grid_for(H.nnode, 256);
    if (H.dim == 2)
        k_apply_G<2, double><<<g, 256, 0, st>>>(H.mk, H.bcmask.as<uint8_t>(), p, y, 0.0);
    else
        k_apply_G<3, double><<<g, 256, 0, st>>>(H.mk, H.bcmask.as<uint8_t>(), p, y, 0.0);
    GG_CUDA(cudaGetLastError());
    H.kernel_launches++;
}

void apply_GT(const Handle& H, const double* u, double* q, cudaStream_t st) {
    const int g = grid_for(H.nel, 256);
    if (H.dim == 2)
        k_apply_GT<2, double><<<g, 256, 0, st>>>(H.mk, u, q);
    else
        k_apply_GT<3, double><<<g, 256, 0, st>>>(H.mk, u, q);
    GG_CUDA(cudaGetLastError());
    H.kernel_launches++;
}

}  // namespace gg
