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
// grid of one parity-class launch of the FP64 apply (apply_tiles_class)
int class_grid(const MeshK& mk, int color);

template <typename R>
void apply_K_ex(const MeshK& mk, const R* mom, const uint8_t* bcmask, const R* x, R* y,
                double* energy_part, int grid, cudaStream_t st, const int32_t* done);

// Global node index of element-local node a (int32: every mesh here has < 2^31 nodes).
template <int DIM>
__device__ __forceinline__ int32_t local_node(int32_t n0, int32_t nn0, int32_t nn01, int a) {
    return n0 + (a & 1) + ((a >> 1) & 1) * nn0 + (DIM == 3 ? ((a >> 2) & 1) * nn01 : 0);
}

// y += K_e x_e for element e = (i, j, k), one atomic per element node and component
// (BC rows skipped); returns the element energy x_eᵀ K_e x_e when kEnergy (else 0).
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
// The kernel is bound by instruction issue, not by bytes (the moments and vectors of a
// 64³ level sit in L2), so the element index arrives as (i, j, k) without divisions,
// node addresses are row bases plus the next word, the BC bits of the 2^dim nodes are
// read once, and the monomials shared by ∂x_c/∂x_d and ∂x_d/∂x_c take one product.
// kLoad selects how x is read: 0 plain (may use the read-only path), 1 through L2 only
// (ld.global.cg), 2 cached weak loads (ld.global.ca).  A persistent kernel that wrote x in
// an earlier phase of the same launch must not use 0: the non-coherent path is only valid
// for data that no thread writes during the kernel.
// The arithmetic and scatter of one element, given its gathered nodal values m[c][a]
// (corner a = (dx, dy, dz) bits) and moments M; `fixed` holds bit 8q + 4dx + c for the
// Dirichlet components of the corners of row q.  Shared by every loader of the apply.
// c_only ≥ 0 forms and scatters output component c_only alone (the transform and the
// velocity gradients still use every component).
template <int DIM, typename R, bool kEnergy>
__device__ __forceinline__ double element_compute_scatter(const MeshK& mk, R (&m)[DIM][1 << DIM],
                                                          const R (&M)[n_moments<DIM>()], uint32_t fixed,
                                                          R* __restrict__ y, int32_t n0, int c_only = -1) {
    constexpr int NS = 1 << DIM;
    constexpr int NR = NS / 2;
    const int64_t nnode = mk.nnode;
    const int32_t nn0 = mk.nn[0], nn01 = mk.nn[0] * mk.nn[1];
    int32_t rowoff[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) rowoff[q] = (q & 1) * nn0 + (DIM == 3 ? ((q >> 1) & 1) * nn01 : 0);
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
    // velocity-gradient coefficients with κ folded in: g[c][d][T] = κ_d m[c][{d}∪T]
    R g[DIM][DIM][NS];
#pragma unroll
    for (int c = 0; c < DIM; c++)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int T = 0; T < NS; T++) g[c][d][T] = ((T >> d) & 1) ? R(0) : kap[d] * m[c][T | (1 << d)];

    double energy = 0.0;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (c_only >= 0 && c != c_only) continue;
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
                    const bool td = !((T >> d) & 1), tc = !((T >> c) & 1);
                    if (c == d) {
                        if (tc) acc += g[c][c][T] * M[mom_slot<DIM>(e0, e1, e2)];
                    } else if (td && tc) {
                        // monomials of both ∂x_c/∂x_d and ∂x_d/∂x_c: one product
                        acc += (g[c][d][T] + g[d][c][T]) * M[mom_slot<DIM>(e0, e1, e2)];
                    } else if (td) {
                        acc += g[c][d][T] * M[mom_slot<DIM>(e0, e1, e2)];
                    } else if (tc) {
                        acc += g[d][c][T] * M[mom_slot<DIM>(e0, e1, e2)];
                    }
                }
                // σ_cc carries the factor 2 of D0
                Q[U | (1 << d)] += (c == d ? R(2) * kap[d] : kap[d]) * acc;
            }
        if (kEnergy) {
#pragma unroll
            for (int S = 1; S < NS; S++) energy += (double)m[c][S] * (double)Q[S];
        }
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
        for (int q = 0; q < NR; q++) {
            R* yr = y + c * nnode + n0 + rowoff[q];
            if (!((fixed >> (8 * q + c)) & 1)) atomicAdd(yr, Q[2 * q]);
            if (!((fixed >> (8 * q + 4 + c)) & 1)) atomicAdd(yr + 1, Q[2 * q + 1]);
        }
    }
    return energy;
}

// kAxpy: the nodal values are x + beta·x2, formed at the gather (a flexible-CG direction
// p = z + βp applied without storing it first; an FP64 iterate plus its FP32 correction).
template <int DIM, typename R, int kLoad = 0, bool kEnergy = true, bool kAxpy = false, typename X2 = R>
__device__ __forceinline__ double element_apply_scatter(const MeshK& mk, const R* __restrict__ mom,
                                                        const uint8_t* __restrict__ bcmask,
                                                        const R* __restrict__ x, R* __restrict__ y, int i, int j,
                                                        int k, int32_t e, int c_only = -1,
                                                        const X2* __restrict__ x2 = nullptr, R beta = R(0)) {
    constexpr int NS = 1 << DIM;
    constexpr int NM = n_moments<DIM>();
    const int64_t nnode = mk.nnode, nel = mk.nel;
    const int32_t nn0 = mk.nn[0], nn01 = mk.nn[0] * mk.nn[1];
    const int32_t n0 = i + nn0 * j + (DIM == 3 ? nn01 * k : 0);
    // corner a = (dx, dy, dz) bits; the NS/2 rows (dy, dz) start at n0 + rowoff, the x+1
    // corner is the next word of the row
    constexpr int NR = NS / 2;
    int32_t rowoff[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) rowoff[q] = (q & 1) * nn0 + (DIM == 3 ? ((q >> 1) & 1) * nn01 : 0);
    uint32_t fixed = 0;  // bit 4a + c: component c of corner a has a Dirichlet condition
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const uint8_t* br = bcmask + n0 + rowoff[q];
        fixed |= ((uint32_t)br[0] | ((uint32_t)br[1] << 4)) << (8 * q);
    }

    R m[DIM][NS];
#pragma unroll
    for (int c = 0; c < DIM; c++) {
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const R* xr = x + c * nnode + n0 + rowoff[q];
            m[c][2 * q] = kLoad == 1 ? __ldcg(xr) : kLoad == 2 ? __ldca(xr) : xr[0];
            m[c][2 * q + 1] = kLoad == 1 ? __ldcg(xr + 1) : kLoad == 2 ? __ldca(xr + 1) : xr[1];
            if constexpr (kAxpy) {
                const X2* pr = x2 + c * nnode + n0 + rowoff[q];
                m[c][2 * q] = m[c][2 * q] + beta * (R)(kLoad == 1 ? __ldcg(pr) : kLoad == 2 ? __ldca(pr) : pr[0]);
                m[c][2 * q + 1] = m[c][2 * q + 1] +
                                  beta * (R)(kLoad == 1 ? __ldcg(pr + 1) : kLoad == 2 ? __ldca(pr + 1) : pr[1]);
            }
        }
    }
    R M[NM];
    const R* Me = mom + e;
#pragma unroll
    for (int q = 0; q < NM; q++) M[q] = Me[q * nel];
    return element_compute_scatter<DIM, R, kEnergy>(mk, m, M, fixed, y, n0, c_only);
}

// Element tiles of one 256-thread block: 32 × 4 × 2 elements in 3D, 32 × 8 in 2D, x fastest
// (a warp is one row of 32 elements: coalesced moment loads, no index divisions).
template <int DIM>
struct ApplyTile;
template <>
struct ApplyTile<3> {
    static constexpr int X = 32, Y = 4, Z = 2;
};
template <>
struct ApplyTile<2> {
    static constexpr int X = 32, Y = 8, Z = 1;
};

// y += K x over the element tiles tile0, tile0 + tstride, … (blockDim.x must be 256).
// Returns this thread's Σ x_eᵀ K_e x_e when kEnergy.
template <int DIM, typename R, int kLoad = 0, bool kEnergy = true, int TY = ApplyTile<DIM>::Y,
          int TZ = ApplyTile<DIM>::Z, bool kAxpy = false, typename X2 = R>
__device__ __forceinline__ double apply_tiles(const MeshK& mk, const R* __restrict__ mom,
                                              const uint8_t* __restrict__ bcmask, const R* __restrict__ x,
                                              R* __restrict__ y, int64_t tile0, int64_t tstride,
                                              const X2* __restrict__ x2 = nullptr, R beta = R(0)) {
    constexpr int TX = ApplyTile<DIM>::X;
    const int ntx = (mk.n[0] + TX - 1) / TX, nty = (mk.n[1] + TY - 1) / TY;
    const int ntz = DIM == 3 ? (mk.n[2] + TZ - 1) / TZ : 1;
    const int32_t ntiles = ntx * nty * ntz;
    const int tx = threadIdx.x % TX, ty = (threadIdx.x / TX) % TY, tz = threadIdx.x / (TX * TY);
    double en = 0.0;
    for (int32_t tile = (int32_t)tile0; tile < ntiles; tile += (int32_t)tstride) {
        const int rr = tile / ntx;
        const int i = (tile - rr * ntx) * TX + tx, j = (rr % nty) * TY + ty, k = (rr / nty) * TZ + tz;
        if (i < mk.n[0] && j < mk.n[1] && (DIM == 2 || k < mk.n[2]))
            en += element_apply_scatter<DIM, R, kLoad, kEnergy, kAxpy, X2>(mk, mom, bcmask, x, y, i, j, k,
                                                                       i + mk.n[0] * (j + mk.n[1] * k), -1, x2,
                                                                       beta);
    }
    return en;
}

// y += K x with DIM threads per element: work item w = c·nel + e forms and scatters output
// component c of element e.  For levels with fewer elements than a third of the grid's
// threads, where one thread per element leaves most of the grid idle and the apply's time
// is one element's dependency chain: the split shortens that chain to about a third.
template <int DIM, typename R, int kLoad>
__device__ __forceinline__ void apply_split(const MeshK& mk, const R* __restrict__ mom,
                                            const uint8_t* __restrict__ bcmask, const R* __restrict__ x,
                                            R* __restrict__ y, int64_t w0, int64_t wstride) {
    const int32_t nel = (int32_t)mk.nel;
    for (int32_t w = (int32_t)w0; w < DIM * nel; w += (int32_t)wstride) {
        const int c = w / nel;
        const int32_t e = w - c * nel;
        const int32_t i = e % mk.n[0], r = e / mk.n[0];
        const int32_t j = r % mk.n[1], k = DIM == 3 ? r / mk.n[1] : 0;
        element_apply_scatter<DIM, R, kLoad, false>(mk, mom, bcmask, x, y, i, j, k, e, c);
    }
}

// (G p) at node n, component by component, before the BC rows are zeroed: the gather of
// the 2^dim elements around the node in element-corner order a = 0 … 2^dim−1,
// G_e[a][c] = Σ_gauss w (−detJ) ∂N_a/∂x_c (GradientStiffnessMatrixTerm.cxx:213-246).
// kCoherent reads p through L2 only (p written earlier in the same launch).
template <int DIM, typename R, bool kCoherent>
__device__ __forceinline__ void g_node(const MeshK& mk, const R* __restrict__ p, int64_t n, R (&acc)[DIM]) {
    const int i = (int)(n % mk.nn[0]);
    const int j = (int)((n / mk.nn[0]) % mk.nn[1]);
    const int k = DIM == 3 ? (int)(n / ((int64_t)mk.nn[0] * mk.nn[1])) : 0;
#pragma unroll
    for (int c = 0; c < DIM; c++) acc[c] = R(0);
#pragma unroll
    for (int a = 0; a < (1 << DIM); a++) {
        const int ei = i - (a & 1), ej = j - ((a >> 1) & 1), ek = DIM == 3 ? k - ((a >> 2) & 1) : 0;
        if (ei < 0 || ej < 0 || ek < 0 || ei >= mk.n[0] || ej >= mk.n[1] || ek >= mk.n[2]) continue;
        const R* pe = &p[ei + (int64_t)mk.n[0] * (ej + (int64_t)mk.n[1] * ek)];
        const R pv = kCoherent ? __ldcg(pe) : *pe;
#pragma unroll
        for (int c = 0; c < DIM; c++) acc[c] += (R)mk.Ge[a][c] * pv;
    }
}

// (Gᵀ u) of element e: Σ over corners a and components c of G_e[a][c] u_{a,c}
template <int DIM, typename R, bool kCoherent>
__device__ __forceinline__ R gt_elem(const MeshK& mk, const R* __restrict__ u, int64_t e) {
    const int64_t nnode = mk.nnode;
    const int i0 = (int)(e % mk.n[0]);
    const int64_t rr = e / mk.n[0];
    const int j0 = (int)(rr % mk.n[1]), k0 = DIM == 3 ? (int)(rr / mk.n[1]) : 0;
    R s = R(0);
#pragma unroll
    for (int a = 0; a < (1 << DIM); a++) {
        const int64_t n = (i0 + (a & 1)) + (int64_t)mk.nn[0] * ((j0 + ((a >> 1) & 1)) +
                                                            (int64_t)mk.nn[1] * (DIM == 3 ? k0 + ((a >> 2) & 1) : 0));
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            const R* up = &u[(int64_t)c * nnode + n];
            s += (R)mk.Ge[a][c] * (kCoherent ? __ldcg(up) : *up);
        }
    }
    return s;
}

// The FP64 apply is summed in a fixed order: elements are split into the 2^dim parity
// classes color = (i&1) | (j&1)<<1 | (k&1)<<2, and one launch scatters one class.  Two
// elements of the same class share no node, so every atomic of a launch lands on a node
// no other thread of that launch touches, and each node receives its element terms in
// class order 0, 1, …, 2^dim−1: y = ((0 + y_0) + y_1) + …, the same bits on every run.
// The tile is taken in class coordinates (element i = 2·ci + (color&1), …), so a warp
// still covers one x-row of 32 elements of its class.
template <int DIM>
__host__ __device__ __forceinline__ int class_extent(const MeshK& mk, int d, int color) {
    return (mk.n[d] - ((color >> d) & 1) + 1) >> 1;
}

template <int DIM>
inline int64_t class_tiles(const MeshK& mk, int color, int TX, int TY, int TZ) {
    const int c0 = class_extent<DIM>(mk, 0, color), c1 = class_extent<DIM>(mk, 1, color);
    const int c2 = DIM == 3 ? class_extent<DIM>(mk, 2, color) : 1;
    return (int64_t)((c0 + TX - 1) / TX) * ((c1 + TY - 1) / TY) * ((c2 + TZ - 1) / TZ);
}

template <int DIM, typename R, int kLoad = 0, bool kEnergy = true, int TY = ApplyTile<DIM>::Y,
          int TZ = ApplyTile<DIM>::Z>
__device__ __forceinline__ double apply_tiles_class(const MeshK& mk, const R* __restrict__ mom,
                                                    const uint8_t* __restrict__ bcmask, const R* __restrict__ x,
                                                    R* __restrict__ y, int64_t tile0, int64_t tstride, int color) {
    constexpr int TX = ApplyTile<DIM>::X;
    const int px = color & 1, py = (color >> 1) & 1, pz = DIM == 3 ? (color >> 2) & 1 : 0;
    const int c0 = class_extent<DIM>(mk, 0, color), c1 = class_extent<DIM>(mk, 1, color);
    const int c2 = DIM == 3 ? class_extent<DIM>(mk, 2, color) : 1;
    const int ntx = (c0 + TX - 1) / TX, nty = (c1 + TY - 1) / TY, ntz = (c2 + TZ - 1) / TZ;
    const int32_t ntiles = ntx * nty * ntz;
    const int tx = threadIdx.x % TX, ty = (threadIdx.x / TX) % TY, tz = threadIdx.x / (TX * TY);
    double en = 0.0;
    for (int32_t tile = (int32_t)tile0; tile < ntiles; tile += (int32_t)tstride) {
        const int rr = tile / ntx;
        const int ci = (tile - rr * ntx) * TX + tx, cj = (rr % nty) * TY + ty, ck = (rr / nty) * TZ + tz;
        if (ci < c0 && cj < c1 && ck < c2) {
            const int i = 2 * ci + px, j = 2 * cj + py, k = DIM == 3 ? 2 * ck + pz : 0;
            en += element_apply_scatter<DIM, R, kLoad, kEnergy>(mk, mom, bcmask, x, y, i, j, k,
                                                                i + mk.n[0] * (j + mk.n[1] * k));
        }
    }
    return en;
}

}  // namespace gg
