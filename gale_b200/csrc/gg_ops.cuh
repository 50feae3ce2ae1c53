// gg_ops.cuh -- reduction helpers and operator launchers shared by gg_ops.cu/gg_solve.cu.
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

// y_e = K_e u_e of one element from its moments (see gg_ops.cu for the derivation).
template <int DIM, typename R>
__device__ __forceinline__ void element_apply_dev(const MeshK& mk, const R* __restrict__ mom, int64_t nel,
                                              int64_t e, const R (&u)[1 << DIM][DIM], R (&y)[1 << DIM][DIM]) {
    constexpr int NS = 1 << DIM;
    constexpr int NM = n_moments<DIM>();
    R M[NM];
#pragma unroll
    for (int m = 0; m < NM; m++) M[m] = mom[(int64_t)m * nel + e];
    R kap[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) kap[d] = (R)mk.kappa[d];

    // forward transform per component
    R m[DIM][NS];
#pragma unroll
    for (int c = 0; c < DIM; c++) {
#pragma unroll
        for (int a = 0; a < NS; a++) m[c][a] = u[a][c];
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int a = 0; a < NS; a++)
                if (!((a >> d) & 1)) {
                    const R lo = m[c][a], hi = m[c][a | (1 << d)];
                    m[c][a] = lo + hi;
                    m[c][a | (1 << d)] = hi - lo;
                }
    }
    // Q[c][S] = Σ_{d∈S} κ_d P[c][d][S\{d}]
    R Q[DIM][NS];
#pragma unroll
    for (int c = 0; c < DIM; c++)
#pragma unroll
        for (int S = 0; S < NS; S++) Q[c][S] = R(0);
#pragma unroll
    for (int c = 0; c < DIM; c++)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int U = 0; U < NS; U++) {
                if ((U >> d) & 1) continue;
                R acc = R(0);
                if (c == d) {
                    // σ_cc = 2 ∂u_c/∂x_c
#pragma unroll
                    for (int Tm = 0; Tm < NS; Tm++) {
                        if ((Tm >> c) & 1) continue;
                        const int e0 = ((U >> 0) & 1) + ((Tm >> 0) & 1);
                        const int e1 = ((U >> 1) & 1) + ((Tm >> 1) & 1);
                        const int e2 = DIM == 3 ? ((U >> 2) & 1) + ((Tm >> 2) & 1) : 0;
                        acc += (R(2) * kap[c] * m[c][Tm | (1 << c)]) * M[mom_slot<DIM>(e0, e1, e2)];
                    }
                } else {
                    // σ_cd = ∂u_c/∂x_d + ∂u_d/∂x_c
#pragma unroll
                    for (int Tm = 0; Tm < NS; Tm++) {
                        if (!((Tm >> d) & 1)) {
                            const int e0 = ((U >> 0) & 1) + ((Tm >> 0) & 1);
                            const int e1 = ((U >> 1) & 1) + ((Tm >> 1) & 1);
                            const int e2 = DIM == 3 ? ((U >> 2) & 1) + ((Tm >> 2) & 1) : 0;
                            acc += (kap[d] * m[c][Tm | (1 << d)]) * M[mom_slot<DIM>(e0, e1, e2)];
                        }
                        if (!((Tm >> c) & 1)) {
                            const int e0 = ((U >> 0) & 1) + ((Tm >> 0) & 1);
                            const int e1 = ((U >> 1) & 1) + ((Tm >> 1) & 1);
                            const int e2 = DIM == 3 ? ((U >> 2) & 1) + ((Tm >> 2) & 1) : 0;
                            acc += (kap[c] * m[d][Tm | (1 << c)]) * M[mom_slot<DIM>(e0, e1, e2)];
                        }
                    }
                }
                Q[c][U | (1 << d)] += kap[d] * acc;
            }
    // inverse transform: y_a = Σ_S Π_{d∈S} s_d(a) Q[S]
#pragma unroll
    for (int c = 0; c < DIM; c++) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int a = 0; a < NS; a++)
                if (!((a >> d) & 1)) {
                    const R q0 = Q[c][a], q1 = Q[c][a | (1 << d)];
                    Q[c][a] = q0 - q1;
                    Q[c][a | (1 << d)] = q0 + q1;
                }
#pragma unroll
        for (int a = 0; a < NS; a++) y[a][c] = Q[c][a];
    }
}


template <typename R>
void apply_K_ex(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y,
                double* energy_part, int grid, cudaStream_t st);

}  // namespace gg
