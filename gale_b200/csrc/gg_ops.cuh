// gg_ops.cuh -- the matrix-free element kernel and reduction helpers shared by
// gg_ops.cu / gg_solve.cu / gg_mg.cu.
#pragma once

#include "gg_internal.cuh"

namespace gg {

// Block-wide sum (any blockDim multiple of 32, ≤ 1024); result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double s_part[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s_part[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? s_part[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

int apply_grid(int64_t nel);

template <typename R>
void apply_K_ex(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y,
                double* energy_part, int grid, cudaStream_t st, const int32_t* done);

// Global node index of element-local node a (int32: every mesh here has < 2^31 nodes).
template <int DIM>
__device__ __forceinline__ int32_t local_node(int32_t n0, int32_t nn0, int32_t nn01, int a) {
    return n0 + (a & 1) + ((a >> 1) & 1) * nn0 + (DIM == 3 ? ((a >> 2) & 1) * nn01 : 0);
}

// y += K_e x_e for element e, scattered with atomics to the non-BC rows; returns the
// element energy x_eᵀ K_e x_e.
//
//   m[c][S] = Σ_a Π_{d∈S} s_d(a) x_{a,c}                 (Walsh–Hadamard, in place)
//   ∂x_c/∂x_d (ξ) = κ_d Σ_{T⊆others(d)} m[c][{d}∪T] ξ^T
//   Q[c][S] = Σ_{d∈S} κ_d Σ_p c_p ξ_p^{S\{d}} σ_cd(ξ_p)   via the moments M[U+T]
//   y_{a,c} = Σ_S Π_{d∈S} s_d(a) Q[c][S]                 (transposed transform)
//   energy  = Σ_c Σ_S m[c][S] Q[c][S]
// with σ_cc = 2 ∂x_c/∂x_c, σ_cd = ∂x_c/∂x_d + ∂x_d/∂x_c (D0 of ConstitutiveMatrixCartesian,
// viscosity and w·detJ inside the moments).  One output component is finished and
// scattered before the next is formed, which keeps the live register set to the moments,
// the modal coefficients and one component's Q.
template <int DIM, typename R>
__device__ __forceinline__ double element_apply_scatter(const MeshK& mk, const R* __restrict__ mom,
                                                        const uint8_t* __restrict__ bcmask,
                                                        const R* __restrict__ x, R* __restrict__ y,
                                                        int64_t e) {
    constexpr int NS = 1 << DIM;
    constexpr int NM = n_moments<DIM>();
    const int32_t nn0 = mk.nn[0], nn01 = mk.nn[0] * mk.nn[1];
    const int32_t nnode = (int32_t)mk.nnode;
    const int64_t nel = mk.nel;
    const int32_t i = (int32_t)(e % mk.n[0]);
    const int32_t r = (int32_t)(e / mk.n[0]);
    const int32_t j = r % mk.n[1], k = r / mk.n[1];
    const int32_t n0 = i + nn0 * (j + mk.nn[1] * k);

    R m[DIM][NS];
#pragma unroll
    for (int a = 0; a < NS; a++) {
        const int32_t n = local_node<DIM>(n0, nn0, nn01, a);
#pragma unroll
        for (int c = 0; c < DIM; c++) m[c][a] = x[(int64_t)c * nnode + n];
    }
    R M[NM];
#pragma unroll
    for (int q = 0; q < NM; q++) M[q] = mom[(int64_t)q * nel + e];
    R kap[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) kap[d] = (R)mk.kappa[d];

#pragma unroll
    for (int c = 0; c < DIM; c++)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int a = 0; a < NS; a++)
                if (!((a >> d) & 1)) {
                    const R lo = m[c][a], hi = m[c][a | (1 << d)];
                    m[c][a] = lo + hi;
                    m[c][a | (1 << d)] = hi - lo;
                }

    double energy = 0.0;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        R Q[NS];
#pragma unroll
        for (int S = 0; S < NS; S++) Q[S] = R(0);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int U = 0; U < NS; U++) {
                if ((U >> d) & 1) continue;
                R acc = R(0);
#pragma unroll
                for (int T = 0; T < NS; T++) {
                    const int e0 = ((U >> 0) & 1) + ((T >> 0) & 1);
                    const int e1 = ((U >> 1) & 1) + ((T >> 1) & 1);
                    const int e2 = DIM == 3 ? ((U >> 2) & 1) + ((T >> 2) & 1) : 0;
                    if (c == d) {
                        if (!((T >> c) & 1))
                            acc += (R(2) * kap[c] * m[c][T | (1 << c)]) * M[mom_slot<DIM>(e0, e1, e2)];
                    } else {
                        if (!((T >> d) & 1)) acc += (kap[d] * m[c][T | (1 << d)]) * M[mom_slot<DIM>(e0, e1, e2)];
                        if (!((T >> c) & 1)) acc += (kap[c] * m[d][T | (1 << c)]) * M[mom_slot<DIM>(e0, e1, e2)];
                    }
                }
                Q[U | (1 << d)] += kap[d] * acc;
            }
#pragma unroll
        for (int S = 1; S < NS; S++) energy += (double)m[c][S] * (double)Q[S];
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int a = 0; a < NS; a++)
                if (!((a >> d) & 1)) {
                    const R q0 = Q[a], q1 = Q[a | (1 << d)];
                    Q[a] = q0 - q1;
                    Q[a | (1 << d)] = q0 + q1;
                }
#pragma unroll
        for (int a = 0; a < NS; a++) {
            const int32_t n = local_node<DIM>(n0, nn0, nn01, a);
            if (!((bcmask[n] >> c) & 1)) atomicAdd(&y[(int64_t)c * nnode + n], Q[a]);
        }
    }
    return energy;
}

}  // namespace gg
