// gg_fused.cu -- the multigrid-preconditioned flexible CG of the inner velocity solve as
// ONE persistent kernel on sm_100a.
//
// The graph-captured solver (run_fcg in gg_solve.cu around vcycle in gg_mg.cu) issues
// about a hundred kernels per iteration, and on the coarse levels each does a few
// microseconds of work, so kernel boundaries set the pace.  Here one cooperative launch
// runs a whole FP32 solve.  The phases of an iteration are:
//   V-cycle (smoothing, restriction, dense coarse solve, prolongation on every level, the
//   dot products fused into the last smoothing step) → fine apply of the direction →
//   update (+ the next level-0 Chebyshev start)
// Each phase boundary is a grid barrier instead of a kernel boundary.  The host writes the
// phase list of one iteration (a "program" for the level hierarchy at hand) into a table
// in device memory; the kernel copies it to shared memory and runs it with one switch, so
// each phase body, the element apply above all, is compiled once.  Neighbouring phases
// are fused:
//   * the update with the level-0 Chebyshev start;
//   * the last smoothing step with the FCG dot products (and the zeroing of Ap);
//   * the restriction with the coarse Chebyshev start;
//   * the direction p = z + βp with the apply of it (formed at the element gather) and
//     with the update (which stores it), so it has no phase of its own.
// The per-phase arithmetic is that of the separate kernels, so the iterates are those of
// run_fcg up to the order of FP32 atomic sums.
//
// Grid barrier: an arrival counter in device memory; thread 0 of each block polls it with
// an iteration limit.  When the limit expires it raises an error word; every block then
// leaves at its next barrier, and the host reads the error word and returns GG_ERR_CUDA.
// The launch is cooperative, so the driver either makes every block co-resident or
// refuses the launch.
// Global reductions: each block writes one FP64 partial; after the barrier every block
// sums all partials in block order.  Every block then holds the same value and takes the
// same branch without a second barrier.
// Vectors written inside the launch are never read through the non-coherent (read-only)
// path.  Reads that touch each value once go through L2 only (__ldcg); reads that reuse
// values across threads of an SM (the apply's nodal gathers, the restriction's and
// prolongation's neighbour reads) are cached weak loads through L1 (__ldca).  Those vectors
// are written only in earlier phases, and the grid barrier's release/acquire pair, followed
// by the block barrier, orders every such write before every later load of the grid.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <cstring>
#include <cstdint>
#include <type_traits>
#include <mutex>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_grid.cuh"
#include "gg_ops.cuh"

namespace gg {

namespace {

constexpr int kFusedMaxLevels = 8;
constexpr int kFusedBlock = 256;

struct FusedLevel {
    MeshK mk;
    const float* mom;
    const uint8_t* bc;
    const float* invd;
    float* b;
    float* x;
    float* r;
    float* d;
    float* t;
    float inv_theta;
    float c1[4], c2[4];
};

// Phase types of the program.  Level 0's x and b are the FCG's z and r.
enum : uint8_t {
    PH_APPLY = 0,      // t_l += A_l d_l (flag 0) or A_l x_l (flag 1)
    PH_STEP = 1,       // Chebyshev step k on level l
    PH_STEP_DOTS = 2,  // the last level-0 step, with the partials of r·z and z·Ap
    PH_RESTRICT = 3,   // b_{l+1} = Pᵀ(r − t)_l, Chebyshev start on l+1 when flag
    PH_DENSE = 4,      // x_l = A_l⁻¹ b_l (coarsest level)
    PH_PROLONG = 5,    // x_l += P x_{l+1}, t_l = 0
    PH_RESTART = 6,    // post-smoothing start on level l
    PH_APPLY_P = 8,    // FCG: Ap = K p for p = z + βp formed at the gather, partials of pᵀAp
    PH_UPDATE = 9,     // FCG: p = z + βp, x += αp, r −= αAp, ‖r‖² partials, level-0 start
};

struct FusedPhase {
    uint8_t type, level, k, flag;
};

constexpr int kMaxPhases = 128;

struct FusedTable {
    int nlevels;   // levels 0..nlevels-1; the last one is solved by the dense inverse
    int nphase;    // phases of one iteration
    int coarse_n;
    int vec4;      // every vector of the table and the launch is 16-byte aligned
    const float* coarse_inv;  // [coarse_n][coarse_ld], 16-byte aligned rows
    int coarse_ld;
    int pad2;
    FusedLevel lv[kFusedMaxLevels];
    FusedPhase ph[kMaxPhases];
};

constexpr int kTabWords = (int)((sizeof(FusedTable) + 15) / 16);

__device__ __forceinline__ void put_partial(double v, double* slot) {
    v = block_sum(v);
    if (threadIdx.x == 0) __stcg(&slot[blockIdx.x], v);
}

// Σ of the per-block partials in block order; identical in every block.
__device__ __noinline__ double all_sum(const double* slot) {
    __shared__ double s_val;
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += __ldcg(&slot[b]);
    v = block_sum(v);
    if (threadIdx.x == 0) s_val = v;
    __syncthreads();
    v = s_val;
    __syncthreads();
    return v;
}

// Two block sums in one pass (thread 0 writes both partials).
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double s_a[32], s_b[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        s_a[wid] = a;
        s_b[wid] = b;
    }
    __syncthreads();
    if (wid == 0) {
        a = lane < (int)(blockDim.x >> 5) ? s_a[lane] : 0.0;
        b = lane < (int)(blockDim.x >> 5) ? s_b[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

__device__ __forceinline__ void put_partial2(double a, double b, double* slot_a, double* slot_b) {
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        __stcg(&slot_a[blockIdx.x], a);
        __stcg(&slot_b[blockIdx.x], b);
    }
}

// all_sum of two partial arrays at once
__device__ __noinline__ void all_sum2(const double* slot_a, const double* slot_b, double& a, double& b) {
    __shared__ double s_val[2];
    a = 0.0;
    b = 0.0;
    for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) {
        a += __ldcg(&slot_a[q]);
        b += __ldcg(&slot_b[q]);
    }
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        s_val[0] = a;
        s_val[1] = b;
    }
    __syncthreads();
    a = s_val[0];
    b = s_val[1];
    __syncthreads();
}

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * (int64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

// t += A v on level L; returns this thread's Σ v_eᵀ A_e v_e when kEnergy.  Element tiles
// block-strided; a level with at most one work item per grid thread at DIM threads per
// element (16³ and below on the 296-block grid) takes the component-split apply instead
// (kEnergy is only asked on level 0).  Measured per phase on creep 64³: the 16³ and 8³
// applies 4.4 → 3.7 and 4.3 → 3.1 µs; the 32³ level (1.3 items per thread) was slower
// split, 5.0 → 5.6 µs.
// kAxpy: the applied vector is v + beta·v2, formed at the element gather.
template <int DIM, bool kEnergy, bool kAxpy = false>
__device__ __forceinline__ double phase_apply(const FusedLevel& L, const float* v, float* t,
                                              const float* v2 = nullptr, float beta = 0.f) {
    if (!kEnergy && !kAxpy && (int64_t)DIM * L.mk.nel <= gstride()) {
        apply_split<DIM, float, 1>(L.mk, L.mom, L.bc, v, t, gtid(), gstride());
        return 0.0;
    }
    return apply_tiles<DIM, float, 1, kEnergy, ApplyTile<DIM>::Y, ApplyTile<DIM>::Z, kAxpy>(
        L.mk, L.mom, L.bc, v, t, blockIdx.x, gridDim.x, v2, beta);
}

// Node-wise phases work on slices of W consecutive FP32 elements: W = 4 moves slice v
// (elements 4v … 4v+3) as one float4, W = 1 element v.  Every load of a slice is
// independent, so a float4 slice keeps four elements' loads in flight where a scalar
// grid-stride loop waited for each element's L2 round trip in turn.  (Batching several
// slices per thread turn was measured slower: the batch's registers spill beside the
// kernel's 128.)
template <int W>
__device__ __forceinline__ void ld_cg(const float* p, int64_t v, float (&o)[W]) {
    if constexpr (W == 4) {
        const float4 q = __ldcg(reinterpret_cast<const float4*>(p) + v);
        o[0] = q.x;
        o[1] = q.y;
        o[2] = q.z;
        o[3] = q.w;
    } else {
        o[0] = __ldcg(p + v);
    }
}

// data no thread writes during the launch (the inverse diagonals)
template <int W>
__device__ __forceinline__ void ld_ro(const float* p, int64_t v, float (&o)[W]) {
    if constexpr (W == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p) + v);
        o[0] = q.x;
        o[1] = q.y;
        o[2] = q.z;
        o[3] = q.w;
    } else {
        o[0] = __ldg(p + v);
    }
}

template <int W>
__device__ __forceinline__ void st(float* p, int64_t v, const float (&o)[W]) {
    if constexpr (W == 4)
        reinterpret_cast<float4*>(p)[v] = make_float4(o[0], o[1], o[2], o[3]);
    else
        p[v] = o[0];
}

// body(width, v) over the n elements of a level vector: float4 slices when `vec`, then the
// n mod 4 tail one element at a time
template <class Body>
__device__ __forceinline__ void for_slices(int64_t n, bool vec, Body body) {
    const int64_t n4 = vec ? n >> 2 : 0;
    for (int64_t v = gtid(); v < n4; v += gstride()) body(std::integral_constant<int, 4>(), v);
    for (int64_t i = 4 * n4 + gtid(); i < n; i += gstride()) body(std::integral_constant<int, 1>(), i);
}

// r −= t, d = c1 d + c2 D⁻¹ r, x += d, t = 0
template <int DIM>
__device__ __forceinline__ void phase_cheb_step(const FusedLevel& L, int k, bool vec) {
    const float c1 = L.c1[k], c2 = L.c2[k];
    for_slices((int64_t)DIM * L.mk.nnode, vec, [&](auto w, int64_t v) {
        constexpr int W = decltype(w)::value;
        float r[W], t[W], d[W], iv[W], x[W], z0[W];
        ld_cg<W>(L.r, v, r);
        ld_cg<W>(L.t, v, t);
        ld_cg<W>(L.d, v, d);
        ld_ro<W>(L.invd, v, iv);
        ld_cg<W>(L.x, v, x);
#pragma unroll
        for (int e = 0; e < W; e++) {
            r[e] = r[e] - t[e];
            d[e] = c1 * d[e] + c2 * iv[e] * r[e];
            x[e] = x[e] + d[e];
            z0[e] = 0.f;
        }
        st<W>(L.r, v, r);
        st<W>(L.d, v, d);
        st<W>(L.x, v, x);
        st<W>(L.t, v, z0);
    });
}

// the same step on level 0, finishing z, with the FCG partial sums r·z and z·Ap; Ap is
// zeroed once read (the direction's apply accumulates into it)
template <int DIM>
__device__ __forceinline__ void phase_cheb_step_dots(const FusedLevel& L, int k, float* Ap, double& rz,
                                                     double& zap, bool vec) {
    const float c1 = L.c1[k], c2 = L.c2[k];
    for_slices((int64_t)DIM * L.mk.nnode, vec, [&](auto w, int64_t v) {
        constexpr int W = decltype(w)::value;
        float r[W], t[W], d[W], iv[W], z[W], rf[W], ap[W], z0[W];
        ld_cg<W>(L.r, v, r);
        ld_cg<W>(L.t, v, t);
        ld_cg<W>(L.d, v, d);
        ld_ro<W>(L.invd, v, iv);
        ld_cg<W>(L.x, v, z);
        ld_cg<W>(L.b, v, rf);
        ld_cg<W>(Ap, v, ap);
#pragma unroll
        for (int e = 0; e < W; e++) {
            r[e] = r[e] - t[e];
            d[e] = c1 * d[e] + c2 * iv[e] * r[e];
            z[e] = z[e] + d[e];
            z0[e] = 0.f;
            rz += (double)rf[e] * (double)z[e];
            zap += (double)z[e] * (double)ap[e];
        }
        st<W>(L.r, v, r);
        st<W>(L.d, v, d);
        st<W>(L.x, v, z);
        st<W>(L.t, v, z0);
        st<W>(Ap, v, z0);
    });
}

// post-smoothing start from x: r = b − t (t = A x), d = D⁻¹r/θ, x += d, t = 0
template <int DIM>
__device__ __forceinline__ void phase_restart(const FusedLevel& L, bool vec) {
    const float th = L.inv_theta;
    for_slices((int64_t)DIM * L.mk.nnode, vec, [&](auto w, int64_t v) {
        constexpr int W = decltype(w)::value;
        float b[W], t[W], iv[W], x[W], r[W], d[W], z0[W];
        ld_cg<W>(L.b, v, b);
        ld_cg<W>(L.t, v, t);
        ld_ro<W>(L.invd, v, iv);
        ld_cg<W>(L.x, v, x);
#pragma unroll
        for (int e = 0; e < W; e++) {
            r[e] = b[e] - t[e];
            d[e] = th * iv[e] * r[e];
            x[e] = x[e] + d[e];
            z0[e] = 0.f;
        }
        st<W>(L.r, v, r);
        st<W>(L.d, v, d);
        st<W>(L.x, v, x);
        st<W>(L.t, v, z0);
    });
}

// b_C = Pᵀ (r − t)_L (zero on coarse BC dofs); when C is smoothed, its Chebyshev start:
// r = b, d = D⁻¹b/θ, x = d, t = 0.  One thread per coarse node.  Node counts are below 2^31
// on every level: 32-bit index arithmetic.  Neighbours past the mesh edge are read at the
// clamped (valid) index with weight 0, so every load of a node is unconditional and all of
// them can be in flight at once.
template <int DIM>
__device__ __forceinline__ void phase_restrict(const FusedLevel& L, const FusedLevel& C, bool start) {
    const MeshK& fk = L.mk;
    const MeshK& ck = C.mk;
    const int32_t cnode = (int32_t)ck.nnode;
    for (int32_t N = (int32_t)gtid(); N < cnode; N += (int32_t)gstride()) {
        const int32_t I = N % ck.nn[0], rr = N / ck.nn[0];
        const int32_t J = rr % ck.nn[1], K = DIM == 3 ? rr / ck.nn[1] : 0;
        float acc[DIM];
#pragma unroll
        for (int c = 0; c < DIM; c++) acc[c] = 0.f;
#pragma unroll
        for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); dz++)
#pragma unroll
            for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int i = 2 * I + dx, j = 2 * J + dy, k = 2 * K + dz;
                    const bool in = i >= 0 && j >= 0 && k >= 0 && i < fk.nn[0] && j < fk.nn[1] && k < fk.nn[2];
                    const float w = in ? (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f) : 0.f;
                    const int32_t n = min(max(i, 0), fk.nn[0] - 1) +
                                      fk.nn[0] * (min(max(j, 0), fk.nn[1] - 1) +
                                                  fk.nn[1] * (DIM == 3 ? min(max(k, 0), fk.nn[2] - 1) : 0));
#pragma unroll
                    for (int c = 0; c < DIM; c++) {
                        const int64_t q = (int64_t)c * fk.nnode + n;
                        acc[c] += w * (__ldcg(&L.r[q]) - __ldcg(&L.t[q]));
                    }
                }
        const uint8_t bm = C.bc[N];
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            const int64_t q = (int64_t)c * ck.nnode + N;
            const float bv = ((bm >> c) & 1) ? 0.f : acc[c];
            C.b[q] = bv;
            if (start) {
                const float dv = C.inv_theta * C.invd[q] * bv;
                C.r[q] = bv;
                C.d[q] = dv;
                C.x[q] = dv;
                C.t[q] = 0.f;
            }
        }
    }
}

// The same restriction with one warp per coarse node: lane q < 3^dim loads fine neighbour q,
// the warp sums the weighted values with a butterfly (fixed order).  A thread per coarse
// node issues its 27 neighbours' loads one after another, which on the small levels (a few
// hundred coarse nodes, a few warps busy) made each restriction ≈10 µs of latency.
template <int DIM>
__device__ __forceinline__ void phase_restrict_warp(const FusedLevel& L, const FusedLevel& C, bool start) {
    const MeshK& fk = L.mk;
    const MeshK& ck = C.mk;
    const int lane = threadIdx.x & 31;
    constexpr int NQ = DIM == 3 ? 27 : 9;
    const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = DIM == 3 ? lane / 9 - 1 : 0;
    const float w = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
    for (int64_t N = gtid() >> 5; N < ck.nnode; N += gstride() >> 5) {
        const int I = (int)(N % ck.nn[0]);
        const int64_t rr = N / ck.nn[0];
        const int J = (int)(rr % ck.nn[1]), K = DIM == 3 ? (int)(rr / ck.nn[1]) : 0;
        float acc[DIM];
#pragma unroll
        for (int c = 0; c < DIM; c++) acc[c] = 0.f;
        const int i = 2 * I + dx, j = 2 * J + dy, k = 2 * K + dz;
        if (lane < NQ && i >= 0 && j >= 0 && k >= 0 && i < fk.nn[0] && j < fk.nn[1] && k < fk.nn[2]) {
            const int64_t n = i + (int64_t)fk.nn[0] * (j + (int64_t)fk.nn[1] * k);
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const int64_t q = (int64_t)c * fk.nnode + n;
                acc[c] = w * (__ldcg(&L.r[q]) - __ldcg(&L.t[q]));
            }
        }
#pragma unroll
        for (int c = 0; c < DIM; c++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        if (lane < DIM) {
            const int c = lane;
            const uint8_t bm = C.bc[N];
            const int64_t q = (int64_t)c * ck.nnode + N;
            const float bv = ((bm >> c) & 1) ? 0.f : acc[c];
            C.b[q] = bv;
            if (start) {
                const float dv = C.inv_theta * C.invd[q] * bv;
                C.r[q] = bv;
                C.d[q] = dv;
                C.x[q] = dv;
                C.t[q] = 0.f;
            }
        }
    }
}

// x_L += P x_C (fine BC dofs untouched), t_L = 0.  Each thread takes kProlongBatch fine
// nodes per turn (n, n + stride, …) and issues all their coarse-corner loads before any
// update, so one L2 round trip covers the batch.  A corner of weight 0 is the low corner
// again (hi = lo), so every load is valid and unconditional.  32-bit index arithmetic.
// The phase reads and writes each fine x value once, so no other thread reads it meanwhile.
constexpr int kProlongBatch = 2;

template <int DIM>
__device__ __forceinline__ void phase_prolong(const FusedLevel& L, const FusedLevel& C) {
    float* xl = L.x;
    const MeshK& fk = L.mk;
    const MeshK& ck = C.mk;
    const int32_t fnode = (int32_t)fk.nnode, stride = (int32_t)gstride();
    for (int32_t n0 = (int32_t)gtid(); n0 < fnode; n0 += kProlongBatch * stride) {
        float acc[kProlongBatch][DIM], xv[kProlongBatch][DIM];
#pragma unroll
        for (int bt = 0; bt < kProlongBatch; bt++) {
            const int32_t n = n0 + bt * stride;
            if (n >= fnode) break;
#pragma unroll
            for (int c = 0; c < DIM; c++) xv[bt][c] = __ldcg(&xl[(int64_t)c * fk.nnode + n]);
            const int32_t i = n % fk.nn[0], rr = n / fk.nn[0];
            const int32_t j = rr % fk.nn[1], k = DIM == 3 ? rr / fk.nn[1] : 0;
            const int idx[3] = {i, j, k};
            int lo[3], hi[3];
            float wl[3], wh[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (d >= DIM || (idx[d] & 1) == 0) {
                    lo[d] = hi[d] = idx[d] >> 1;
                    wl[d] = 1.f;
                    wh[d] = 0.f;
                } else {
                    lo[d] = idx[d] >> 1;
                    hi[d] = lo[d] + 1;
                    wl[d] = wh[d] = 0.5f;
                }
            }
#pragma unroll
            for (int c = 0; c < DIM; c++) acc[bt][c] = 0.f;
#pragma unroll
            for (int q = 0; q < (1 << DIM); q++) {
                const int I = (q & 1) ? hi[0] : lo[0], J = (q & 2) ? hi[1] : lo[1], K = (q & 4) ? hi[2] : lo[2];
                const float w = ((q & 1) ? wh[0] : wl[0]) * ((q & 2) ? wh[1] : wl[1]) *
                                (DIM == 3 ? ((q & 4) ? wh[2] : wl[2]) : 1.f);
                const int32_t N = I + ck.nn[0] * (J + ck.nn[1] * K);
#pragma unroll
                for (int c = 0; c < DIM; c++) acc[bt][c] += w * __ldca(&C.x[(int64_t)c * ck.nnode + N]);
            }
        }
#pragma unroll
        for (int bt = 0; bt < kProlongBatch; bt++) {
            const int32_t n = n0 + bt * stride;
            if (n >= fnode) break;
            const uint8_t bm = L.bc[n];
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const int64_t q = (int64_t)c * fk.nnode + n;
                if (!((bm >> c) & 1)) xl[q] = xv[bt][c] + acc[bt][c];
                L.t[q] = 0.f;
            }
        }
    }
}

// x = A⁻¹ b on the coarsest level: one warp per row of the dense FP32 inverse, the row
// (padded to ld, a multiple of 4) and b read as float4 into four partial sums;
// b was written by the restriction before the phase's barrier and is reused by every row,
// so it is read through L1 (cached weak loads, ordered after that barrier's acquire)
__device__ __forceinline__ void phase_dense(int n, int ld, const float* A, const float* b, float* x) {
    const int lane = threadIdx.x & 31;
    const int n4 = n >> 2;
    const float4* b4 = reinterpret_cast<const float4*>(b);
    for (int64_t row = gtid() >> 5; row < n; row += gstride() >> 5) {
        const float4* a4 = reinterpret_cast<const float4*>(A + row * ld);
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        for (int k = lane; k < n4; k += 32) {
            const float4 av = __ldg(&a4[k]);
            const float4 bv = __ldca(&b4[k]);
            s0 += av.x * bv.x;
            s1 += av.y * bv.y;
            s2 += av.z * bv.z;
            s3 += av.w * bv.w;
        }
        for (int k = 4 * n4 + lane; k < n; k += 32) s0 += __ldg(&A[row * ld + k]) * __ldca(&b[k]);
        float s = (s0 + s1) + (s2 + s3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = s;
    }
}

// x = 0, r = b (BC rows zero), p = Ap = 0 (update = false); or p = z + βp, x += αp,
// r −= αAp (update = true); then the level-0 Chebyshev start on r.  Returns this
// thread's Σ r².
template <int DIM>
__device__ __forceinline__ double phase_update_start(const FusedLevel& L0, bool update, float alpha, float beta,
                                                     const float* b, const double* b64, float* x, float* p,
                                                     float* Ap, bool vec) {
    const int64_t nnode = L0.mk.nnode, n = (int64_t)DIM * nnode;
    float* r = L0.b;
    float* z = L0.x;
    double acc = 0.0;
    if (update) {
        const float th = L0.inv_theta;
        for_slices(n, vec, [&](auto w, int64_t v) {
            constexpr int W = decltype(w)::value;
            float xv[W], pv[W], rv[W], ap[W], iv[W], d[W], z0[W], zv[W];
            ld_cg<W>(x, v, xv);
            ld_cg<W>(p, v, pv);
            ld_cg<W>(r, v, rv);
            ld_cg<W>(Ap, v, ap);
            ld_ro<W>(L0.invd, v, iv);
            ld_cg<W>(z, v, zv);
#pragma unroll
            for (int e = 0; e < W; e++) {
                pv[e] = zv[e] + beta * pv[e];  // the direction the apply formed: p = z + βp
                xv[e] = xv[e] + alpha * pv[e];
                rv[e] = rv[e] - alpha * ap[e];  // BC rows of Ap are zero
                acc += (double)rv[e] * (double)rv[e];
                d[e] = th * iv[e] * rv[e];
                z0[e] = 0.f;
            }
            st<W>(x, v, xv);
            st<W>(p, v, pv);
            st<W>(r, v, rv);
            st<W>(L0.r, v, rv);
            st<W>(L0.d, v, d);
            st<W>(z, v, d);
            st<W>(L0.t, v, z0);
        });
        return acc;
    }
    for (int64_t i = gtid(); i < n; i += gstride()) {
        float rv;
        if (update) {
            x[i] = __ldcg(&x[i]) + alpha * __ldcg(&p[i]);
            rv = __ldcg(&r[i]) - alpha * __ldcg(&Ap[i]);  // BC rows of Ap are zero
        } else {
            const int c = (int)(i / nnode);
            const bool fixed = (L0.bc[i - (int64_t)c * nnode] >> c) & 1;
            rv = fixed ? 0.f : (b64 ? (float)__ldcg(&b64[i]) : __ldcg(&b[i]));
            x[i] = 0.f;
            p[i] = 0.f;
            Ap[i] = 0.f;
        }
        r[i] = rv;
        acc += (double)rv * (double)rv;
        const float dv = L0.inv_theta * L0.invd[i] * rv;
        L0.r[i] = rv;
        L0.d[i] = dv;
        z[i] = dv;
        L0.t[i] = 0.f;
    }
    return acc;
}

// Outcome of one flexible-CG solve (identical in every block).
struct FcgResult {
    double rnorm0, rnorm, ttol, rz, pAp;
    int iterations;
    int failed;  // 0 converged, 1 iteration cap, 2 non-finite residual, 3 pᵀAp ≤ 0
};

// The start of a flexible-CG solve for dof i of level 0 with right-hand side value rv
// (0 on Dirichlet rows): x = p = Ap = 0, r = rv and the level-0 Chebyshev start — what
// phase_update_start does when update = false.  For a caller that folds the start into a
// phase of its own; the caller also writes Σ rv² per block into part[0, gridDim.x).
__device__ __forceinline__ void fcg_start_dof(const FusedLevel& L0, int64_t i, float rv, float* x, float* p,
                                              float* Ap) {
    x[i] = 0.f;
    p[i] = 0.f;
    Ap[i] = 0.f;
    L0.b[i] = rv;
    const float dv = L0.inv_theta * L0.invd[i] * rv;
    L0.r[i] = rv;
    L0.d[i] = dv;
    L0.x[i] = dv;
    L0.t[i] = 0.f;
}

// The whole solve of K32 x = b to ‖r‖ ≤ rtol‖b‖ from x = 0, within a launch whose barrier
// count is `epoch`; b is FP32, or FP64 (b64 non-null: rounded to FP32 as it is read).
// prestarted: the caller has made the start (fcg_start_dof for every dof, the Σ r²
// partials in part[0, gridDim.x)) in a phase that ended with a grid barrier.
// Uses part[0, 4·gridDim.x).  Returns false if a barrier gave up.
template <int DIM>
__device__ __forceinline__ bool fcg_body(const FusedTable& T, const float* b, const double* b64, float* x, float* p,
                                         float* Ap, double rtol, int maxit, double* part, GridBarrier* gb,
                                         unsigned int& epoch, FcgResult& res, bool prestarted = false) {
    const FusedLevel& L0 = T.lv[0];
    const int64_t n = (int64_t)DIM * L0.mk.nnode;
    const int G = gridDim.x;
    double* p_rr = part;
    double* p_rz = part + G;
    double* p_zap = part + 2 * G;
    double* p_pap = part + 3 * G;
    const bool vec = T.vec4 != 0;
    if (!prestarted) {
        put_partial(phase_update_start<DIM>(L0, false, 0.f, 0.f, b, b64, x, p, Ap, vec), p_rr);
        if (!grid_barrier(gb, &epoch)) return false;
    }
    const double rnorm0 = sqrt(all_sum(p_rr));
    const double tt = rtol * rnorm0;
    const double ttol = tt < 1e-30 ? 1e-30 : tt;
    double rn = rnorm0, rz = 0.0, pAp = 1.0;
    float alpha = 0.f, beta = 0.f;
    int it = 0, failed = 0;
    bool done = rnorm0 <= ttol;
    while (!done) {
        for (int q = 0; q < T.nphase && !done; q++) {
            const FusedPhase P = T.ph[q];
            const FusedLevel& L = T.lv[P.level];
            switch (P.type) {
                case PH_APPLY:
                    phase_apply<DIM, false>(L, P.flag ? L.x : L.d, L.t);
                    break;
                case PH_APPLY_P:  // Ap = K(z + βp), with the partials of pᵀAp
                    put_partial(phase_apply<DIM, true, true>(L0, L0.x, Ap, p, beta), p_pap);
                    break;
                case PH_STEP:
                    phase_cheb_step<DIM>(L, P.k, vec);
                    break;
                case PH_STEP_DOTS: {
                    double rzp = 0.0, zap = 0.0;
                    phase_cheb_step_dots<DIM>(L, P.k, Ap, rzp, zap, vec);
                    put_partial2(rzp, zap, p_rz, p_zap);
                    break;
                }
                case PH_RESTRICT:
                    // a warp per coarse node where the grid's warps outnumber a quarter of
                    // the coarse nodes (every level below the first coarse one)
                    if ((gstride() >> 5) * 4 >= T.lv[P.level + 1].mk.nnode)
                        phase_restrict_warp<DIM>(L, T.lv[P.level + 1], P.flag != 0);
                    else
                        phase_restrict<DIM>(L, T.lv[P.level + 1], P.flag != 0);
                    break;
                case PH_DENSE:
                    phase_dense(T.coarse_n, T.coarse_ld, T.coarse_inv, L.b, L.x);
                    break;
                case PH_PROLONG:
                    phase_prolong<DIM>(L, T.lv[P.level + 1]);
                    break;
                case PH_RESTART:
                    phase_restart<DIM>(L, vec);
                    break;
                case PH_UPDATE:
                    put_partial(phase_update_start<DIM>(L0, true, alpha, beta, b, b64, x, p, Ap, vec), p_rr);
                    break;
                default:
                    break;
            }
            if (!grid_barrier(gb, &epoch)) return false;
            // scalars after the phases that end in a reduction (same value in every block)
            if (P.type == PH_STEP_DOTS) {
                double zap;
                all_sum2(p_rz, p_zap, rz, zap);
                // truncated flexible CG (Notay 2000): β = −(z·Ap)/(pᵀAp), p = z on the first step
                beta = it == 0 ? 0.f : (float)(-zap / pAp);
            } else if (P.type == PH_APPLY_P) {
                pAp = all_sum(p_pap);
                if (!(pAp > 0.0) || isinf(pAp)) {
                    failed = 3;
                    done = true;
                } else {
                    alpha = (float)(rz / pAp);
                }
            } else if (P.type == PH_UPDATE) {
                rn = sqrt(all_sum(p_rr));
                it++;
                if (!(rn == rn) || isinf(rn)) {
                    failed = 2;
                    done = true;
                } else if (rn <= ttol) {
                    done = true;
                } else if (it >= maxit) {
                    failed = 1;
                    done = true;
                }
            }
        }
    }
    res.rnorm0 = rnorm0;
    res.rnorm = rn;
    res.ttol = ttol;
    res.rz = rz;
    res.pAp = pAp;
    res.iterations = it;
    res.failed = failed;
    return true;
}

template <int DIM>
__global__ void __launch_bounds__(kFusedBlock, 2)
k_fcg_fused(const int4* __restrict__ tab, const float* __restrict__ b, float* x, float* p, float* Ap, double rtol,
            int maxit, KrylovScalars* ks, double* part, GridBarrier* gb) {
    __shared__ int4 s_tab[kTabWords];
    for (int i = threadIdx.x; i < kTabWords; i += blockDim.x) s_tab[i] = tab[i];
    __syncthreads();
    const FusedTable& T = *reinterpret_cast<const FusedTable*>(s_tab);
    unsigned int epoch = 0;
    FcgResult res;
    // a barrier that gave up is reported by the barrier's own error word (read by the host)
    if (fcg_body<DIM>(T, b, nullptr, x, p, Ap, rtol, maxit, part, gb, epoch, res) && blockIdx.x == 0 &&
        threadIdx.x == 0) {
        ks->rnorm0 = res.rnorm0;
        ks->rnorm = res.rnorm;
        ks->ttol = res.ttol;
        ks->rz = res.rz;
        ks->pAp = res.pAp;
        ks->iterations = res.iterations;
        ks->failed = res.failed;
        ks->maxit = maxit;
        ks->done = 1;
    }
}

// ---- the whole Uzawa solve as one launch ---------------------------------------------
// Stokes_SLE_UzawaSolver_Solve (StgFEM/SLE/ProvidedSystems/StokesFlow/src/
// Stokes_SLE_UzawaSolver.cxx:393-938) on the mixed path: the outer conjugate-gradient loop
// on the pressure, and each inner velocity solve as FP64 defect correction around the
// multigrid flexible CG above (fcg_body).  The steps and stopping rules are those of
// uzawa_solve / inner_solve in gg_solve.cu, which the host runs one kernel at a time
// with a device-to-host read after every reduction; here every reduction is a grid
// barrier and every block takes the same branches on the same values, so the solve
// returns to the host once.  The FP64 K apply sums each node's element terms in parity-
// class order (one phase per class) as apply_K<double> does.

// Where a solve stopped early: the step whose status it returns.
enum : int {
    UZ_NONE = 0,
    UZ_FIRST_INNER = 1,  // K u* = f
    UZ_RHS = 2,          // ‖Gᵀu* − h‖ not finite
    UZ_VELOCITY = 3,     // K u = f − G p
    UZ_INNER_DIR = 4,    // K u* = G s
    UZ_STEP = 5,         // z·r, s·Gᵀu*, α not finite
    UZ_RESIDUAL = 6,     // ‖r‖ not finite
    UZ_LIMIT = 7,        // outer iteration limit
};

struct UzawaFusedOut {
    int status;            // GG_OK or a GG_ERR code
    int where;             // UZ_*
    int outer_iterations;
    int inner_iterations;  // flexible-CG iterations of all inner solves
    int inner_solves;
    int sweeps;            // FP32 flexible-CG solves (defect-correction sweeps)
    int pad[2];
    double rel_residual, abs_residual;
};

struct UzawaFusedArgs {
    const double* mom64;
    const double* kdiag;  // FP64 diagonal of K (the inner stopping norm ‖D⁻¹r‖)
    const double* sdiag;  // Ĝ, the pressure preconditioner's diagonal
    const double* f;
    const double* hv;
    double *u, *vstar, *ftmp, *q, *qtmp, *r, *s, *r64;
    double* acc64;  // FP64 apply accumulator (zero between sweeps)
    float *e32, *p32, *Ap32;
    double tolerance, inner_rtol, scaleq;
    double floor_u, floor_h;  // the exact-flow test: ‖r0‖ ≤ floor_u ‖u‖ + floor_h ‖h‖
    int max_iterations, min_iterations, use_abs, use_precond, recycle, inner_maxit, sweep_cap;
    int pad;
    UzawaFusedOut* out;
    double* part;  // 8 · gridDim.x doubles
    GridBarrier* gb;
};

// acc64 += K (x + e): the FP64 iterate plus the sweep's FP32 correction, added at the
// element gather (x itself is updated in the defect phase that follows), all elements in
// one phase with FP64 atomics (arrival order).  Summed in element parity-class order
// instead (one phase per class, as the plain FP64 path does), the FP64 applies of the
// creep 64³ solve (136 outer, 692 flexible-CG iterations) took 30.6 ms against 11.5 ms;
// the mixed path's iterates already depend on the FP32 atomics' order.  acc64 is zero on
// entry.  False if a barrier gave up.
template <int DIM>
__device__ __forceinline__ bool uz_apply_K64(const FusedTable& T, const UzawaFusedArgs& A, const double* x,
                                             unsigned int& epoch) {
    const FusedLevel& L0 = T.lv[0];
    apply_tiles<DIM, double, 1, false, ApplyTile<DIM>::Y, ApplyTile<DIM>::Z, true, float>(
        L0.mk, A.mom64, L0.bc, x, A.acc64, blockIdx.x, gridDim.x, A.e32, 1.0);
    return grid_barrier(A.gb, &epoch);
}

// The defect phase after a sweep: r64 = b − acc64 on free rows (0 on Dirichlet rows),
// acc64 = 0 for the next apply, x += e; and, speculatively, the next sweep's flexible-CG
// start on that defect (fcg_start_dof; it is simply overwritten if the solve has
// converged).  Returns ‖D⁻¹ r64‖ (every block the same value); the Σ r² partials of the
// start are in part[0, gridDim.x).  *ok = false if the barrier gave up.
template <int DIM>
__device__ __forceinline__ double uz_defect_start(const FusedTable& T, const UzawaFusedArgs& A, const double* b,
                                                  double* x, unsigned int& epoch, bool* ok) {
    const FusedLevel& L0 = T.lv[0];
    const int64_t nnode = L0.mk.nnode;
    double* P = A.part + 4 * gridDim.x;
    double acc = 0.0, acc32 = 0.0;
    for (int64_t n = gtid(); n < nnode; n += gstride()) {
        const uint8_t bm = L0.bc[n];
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            const int64_t i = (int64_t)c * nnode + n;
            double rv = 0.0;
            if (!((bm >> c) & 1)) {
                rv = __ldcg(&b[i]) - __ldcg(&A.acc64[i]);
                const double zv = rv / A.kdiag[i];
                acc += zv * zv;
            }
            A.r64[i] = rv;
            A.acc64[i] = 0.0;
            x[i] = __ldcg(&x[i]) + (double)__ldcg(&A.e32[i]);
            const float r32 = (float)rv;
            fcg_start_dof(L0, i, r32, A.e32, A.p32, A.Ap32);
            acc32 += (double)r32 * (double)r32;
        }
    }
    put_partial2(acc, acc32, P, A.part);
    *ok = grid_barrier(A.gb, &epoch);
    return *ok ? sqrt(all_sum(P)) : 0.0;
}

constexpr int kUzBarrierFail = -1;

// K x = b to ‖D⁻¹(b − Kx)‖ ≤ rtol ‖D⁻¹b‖ (inner_solve's mixed branch): FP32 multigrid
// flexible-CG sweeps on the FP64 defect, each followed by the FP64 defect of x + e.
// warm: start from x, whose defect b − Kx the caller has already put in r64 (else
// x = 0).  Each phase that ends with a defect also makes the next sweep's start, so a
// sweep costs its FCG iterations plus two phases (the FP64 apply and the defect).
// prestarted: the caller's last phase (which ended with a grid barrier) already did the
// first phase below (x, r64, acc64, the first sweep's start and the three partial sums).
// Returns GG_OK / GG_ERR_NOT_CONVERGED / GG_ERR_NONFINITE, or kUzBarrierFail.
template <int DIM>
__device__ __forceinline__ int uz_inner(const FusedTable& T, const UzawaFusedArgs& A, const double* b, double* x,
                                        double rtol, bool warm, bool& tight, unsigned int& epoch, int& its,
                                        int& sweeps, bool prestarted) {
    const FusedLevel& L0 = T.lv[0];
    const int64_t nnode = L0.mk.nnode;
    double* P = A.part + 4 * gridDim.x;
    double* P1 = A.part + 5 * gridDim.x;
    // x = 0 and r = b on free rows (the defect of x = 0), or the warm start's defect as
    // given; acc64 = 0; the first sweep's start on r; the partials of ‖D⁻¹b‖, ‖D⁻¹r‖ and
    // the start's Σ r²
    if (!prestarted) {
        double acc = 0.0, acc_r = 0.0, acc32 = 0.0;
        for (int64_t n = gtid(); n < nnode; n += gstride()) {
            const uint8_t bm = L0.bc[n];
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const int64_t i = (int64_t)c * nnode + n;
                const bool fixed = (bm >> c) & 1;
                const double bv = fixed ? 0.0 : __ldcg(&b[i]);
                double rv = bv;
                if (warm) rv = fixed ? 0.0 : __ldcg(&A.r64[i]);
                if (!fixed) {
                    const double zv = bv / A.kdiag[i];
                    acc += zv * zv;
                    const double zr = rv / A.kdiag[i];
                    acc_r += zr * zr;
                }
                if (!warm) {
                    x[i] = 0.0;
                    A.r64[i] = bv;
                }
                A.acc64[i] = 0.0;
                const float r32 = (float)rv;
                fcg_start_dof(L0, i, r32, A.e32, A.p32, A.Ap32);
                acc32 += (double)r32 * (double)r32;
            }
        }
        put_partial2(acc, acc_r, P, P1);
        put_partial(acc32, A.part);
        if (!grid_barrier(A.gb, &epoch)) return kUzBarrierFail;
    }
    double b2, r2;
    all_sum2(P, P1, b2, r2);
    const double rnorm0 = sqrt(b2);
    double ttol = rtol * rnorm0;
    if (ttol < 1e-50) ttol = 1e-50;
    double rn_cur = rnorm0;
    if (warm) {
        const double rn = sqrt(r2);
        if (!(rn == rn)) return GG_ERR_NONFINITE;
        if (rn <= ttol) return GG_OK;
        rn_cur = rn;
    } else if (rnorm0 <= ttol) {
        return GG_OK;
    }
    int total = 0;
    int rc = GG_ERR_NOT_CONVERGED;
    for (int sweep = 0; sweep < 50; sweep++) {
        const double inner_rtol = tight ? 1e-5 : 1e-4;
        const double srtol = fmax(inner_rtol, fmin(0.5, ttol / rn_cur));
        FcgResult res;
        if (!fcg_body<DIM>(T, nullptr, A.r64, A.e32, A.p32, A.Ap32, srtol, A.sweep_cap, A.part, A.gb, epoch, res,
                           true))
            return kUzBarrierFail;
        total += res.iterations;
        sweeps++;
        if (res.failed >= 2) {
            rc = GG_ERR_NONFINITE;
            break;
        }
        if (!uz_apply_K64<DIM>(T, A, x, epoch)) return kUzBarrierFail;
        bool ok = true;
        const double rn = uz_defect_start<DIM>(T, A, b, x, epoch, &ok);
        if (!ok) return kUzBarrierFail;
        if (!(rn == rn)) {
            rc = GG_ERR_NONFINITE;
            break;
        }
        if (sweep >= 2) tight = true;
        if (rn <= ttol) {
            rc = GG_OK;
            break;
        }
        rn_cur = rn;
        if (total >= A.inner_maxit) break;
    }
    its += total;
    return rc;
}

// The solve is written around ONE call of the inner solve (stage 1: K u* = f; stage 2:
// K u = f − G p; stage 3: K u* = G s, once per outer iteration), so the flexible CG is
// inlined once and keeps the kernel's registers.
template <int DIM>
__device__ __forceinline__ bool uzawa_body(const FusedTable& T, const UzawaFusedArgs& A, UzawaFusedOut& o) {
    const FusedLevel& L0 = T.lv[0];
    const MeshK& mk = L0.mk;
    const int64_t nnode = mk.nnode, nel = mk.nel;
    const int G = gridDim.x;
    double* P0 = A.part + 4 * G;
    double* P1 = A.part + 5 * G;
    double* P2 = A.part + 6 * G;
    unsigned int epoch = 0;
    bool tight = false;
    o.status = GG_OK;
    o.where = UZ_NONE;
    o.outer_iterations = 0;
    o.inner_iterations = 0;
    o.inner_solves = 0;
    o.sweeps = 0;
    o.rel_residual = 0.0;
    o.abs_residual = 0.0;
    int it = 0, stage = 1;
    double rhs_scale = 0.0, absres = 0.0, relres = 0.0, zr = 0.0, zr_prev = 1.0;
    bool exact = false;
    // the inner solve of the current stage
    const double* ib = A.f;  // STEP 1 (:553-565)
    double* ix = A.vstar;
    double irtol = A.tolerance;
    bool iwarm = false, ipre = false;
    for (;;) {
        o.inner_solves++;
        const int rc = uz_inner<DIM>(T, A, ib, ix, irtol, iwarm, tight, epoch, o.inner_iterations, o.sweeps, ipre);
        if (rc == kUzBarrierFail) return false;
        if (rc != GG_OK) {
            o.status = rc;
            o.where = stage == 1 ? UZ_FIRST_INNER : stage == 2 ? UZ_VELOCITY : UZ_INNER_DIR;
            o.outer_iterations = it;
            return true;
        }
        if (stage == 1) {
            // Gᵀu* − h and its norm
            double acc = 0.0;
            for (int64_t e = gtid(); e < nel; e += gstride()) {
                const double qv = -__ldcg(&A.hv[e]) + gt_elem<DIM, double, true>(mk, A.vstar, e);
                A.qtmp[e] = qv;
                acc += qv * qv;
            }
            put_partial(acc, P0);
            if (!grid_barrier(A.gb, &epoch)) return false;
            rhs_scale = sqrt(all_sum(P0)) / A.scaleq;
            if (!isfinite(rhs_scale)) {
                o.status = GG_ERR_NONFINITE;
                o.where = UZ_RHS;
                return true;
            }
            // STEP 3 (:616-659): K u = f − G p
            for (int64_t n = gtid(); n < nnode; n += gstride()) {
                double g[DIM];
                g_node<DIM, double, true>(mk, A.q, n, g);
                const uint8_t bm = L0.bc[n];
#pragma unroll
                for (int c = 0; c < DIM; c++) {
                    const int64_t i = (int64_t)c * nnode + n;
                    A.ftmp[i] = A.f[i] - (((bm >> c) & 1) ? 0.0 : g[c]);
                }
            }
            if (!grid_barrier(A.gb, &epoch)) return false;
            stage = 2;
            ib = A.ftmp;
            ix = A.u;
            irtol = A.inner_rtol;
            continue;
        }
        if (stage == 2) {
            // r = Gᵀu − h, and the exact-flow test: a velocity that meets the constraint
            // to rounding ends the solve with the current pressure (no outer iteration)
            double rr = 0.0, hh = 0.0, uu = 0.0;
            for (int64_t e = gtid(); e < nel; e += gstride()) {
                const double hvv = __ldcg(&A.hv[e]);
                const double rv = -hvv + gt_elem<DIM, double, true>(mk, A.u, e);
                A.r[e] = rv;
                rr += rv * rv;
                hh += hvv * hvv;
            }
            for (int64_t i = gtid(); i < (int64_t)DIM * nnode; i += gstride()) {
                const double uv = __ldcg(&A.u[i]);
                uu += uv * uv;
            }
            put_partial2(rr, hh, P0, P1);
            put_partial(uu, P2);
            if (!grid_barrier(A.gb, &epoch)) return false;
            double r0, h2;
            all_sum2(P0, P1, r0, h2);
            r0 = sqrt(r0);
            if (r0 <= A.floor_u * sqrt(all_sum(P2)) + A.floor_h * sqrt(h2)) {
                exact = true;
                absres = r0 / A.scaleq;
                break;
            }
        } else {
            // STEP 4 (:664-837), after K u* = G s: Gᵀu*, s·Gᵀu*, α
            double acc = 0.0;
            for (int64_t e = gtid(); e < nel; e += gstride()) {
                const double qv = gt_elem<DIM, double, true>(mk, A.vstar, e);
                A.qtmp[e] = qv;
                acc += __ldcg(&A.s[e]) * qv;
            }
            put_partial(acc, P0);
            if (!grid_barrier(A.gb, &epoch)) return false;
            const double sq = all_sum(P0);
            const double alpha = zr / sq;
            if (!isfinite(zr) || !isfinite(sq) || !isfinite(alpha)) {
                o.status = GG_ERR_NONFINITE;
                o.where = UZ_STEP;
                o.outer_iterations = it;
                return true;
            }
            // p += α s, r −= α Gᵀu*, u −= α u*; ‖r‖
            acc = 0.0;
            for (int64_t e = gtid(); e < nel; e += gstride()) {
                A.q[e] = alpha * __ldcg(&A.s[e]) + __ldcg(&A.q[e]);
                const double rv = -alpha * __ldcg(&A.qtmp[e]) + __ldcg(&A.r[e]);
                A.r[e] = rv;
                acc += rv * rv;
            }
            for (int64_t i = gtid(); i < (int64_t)DIM * nnode; i += gstride())
                A.u[i] = -alpha * __ldcg(&A.vstar[i]) + __ldcg(&A.u[i]);
            put_partial(acc, P0);
            if (!grid_barrier(A.gb, &epoch)) return false;
            zr_prev = zr;
            absres = sqrt(all_sum(P0)) / A.scaleq;
            relres = absres / rhs_scale;
            if (!isfinite(absres)) {
                o.status = GG_ERR_NONFINITE;
                o.where = UZ_RESIDUAL;
                o.outer_iterations = it;
                return true;
            }
            if (!(it < A.max_iterations)) {
                it++;
                o.status = GG_ERR_NOT_CONVERGED;
                o.where = UZ_LIMIT;
                break;
            }
            it++;
            const double chosen = A.use_abs ? absres : relres;
            if (!((chosen > A.tolerance) || (it < A.min_iterations))) break;
        }
        // the next conjugate direction: z = Ĝ⁻¹ r (or r), z·r
        double acc = 0.0;
        for (int64_t e = gtid(); e < nel; e += gstride()) {
            const double rv = __ldcg(&A.r[e]);
            const double z = A.use_precond ? rv / A.sdiag[e] : rv;
            A.qtmp[e] = z;
            acc += z * rv;
        }
        put_partial(acc, P0);
        if (!grid_barrier(A.gb, &epoch)) return false;
        zr = all_sum(P0);
        const double beta = zr / zr_prev;
        // s = z (first step) or z + β s
        for (int64_t e = gtid(); e < nel; e += gstride()) {
            const double z = __ldcg(&A.qtmp[e]);
            A.s[e] = it == 0 ? z : z + beta * __ldcg(&A.s[e]);
        }
        if (!grid_barrier(A.gb, &epoch)) return false;
        // G s, and the recycled start β u*_prev of K u* = G s with its defect: the previous
        // inner solve ended with r = G s_prev − K u*_prev (its last FP64 defect, still in
        // r64, ftmp still G s_prev), so G s − K(β u*_prev) = G s − β (G s_prev − r) without
        // an apply (free rows; 0 on Dirichlet rows).  The same pass makes the inner solve's
        // first phase (uz_inner, prestarted): acc64 = 0, the first sweep's start and the
        // partial sums of ‖D⁻¹G s‖, ‖D⁻¹r‖ and the start's Σ r².
        const bool warm = A.recycle && it > 0;
        double acc_b = 0.0, acc_r = 0.0, acc32 = 0.0;
        for (int64_t n = gtid(); n < nnode; n += gstride()) {
            double g[DIM];
            g_node<DIM, double, true>(mk, A.s, n, g);
            const uint8_t bm = L0.bc[n];
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const int64_t i = (int64_t)c * nnode + n;
                const bool fixed = (bm >> c) & 1;
                const double gs = fixed ? 0.0 : g[c];
                double rv = gs;
                if (warm) {
                    A.vstar[i] = beta * __ldcg(&A.vstar[i]);
                    rv = fixed ? 0.0 : gs - beta * (__ldcg(&A.ftmp[i]) - __ldcg(&A.r64[i]));
                } else {
                    A.vstar[i] = 0.0;
                }
                A.r64[i] = rv;
                A.ftmp[i] = gs;
                A.acc64[i] = 0.0;
                if (!fixed) {
                    const double zb = gs / A.kdiag[i], zr = rv / A.kdiag[i];
                    acc_b += zb * zb;
                    acc_r += zr * zr;
                }
                const float r32 = (float)rv;
                fcg_start_dof(L0, i, r32, A.e32, A.p32, A.Ap32);
                acc32 += (double)r32 * (double)r32;
            }
        }
        put_partial2(acc_b, acc_r, P0, P1);
        put_partial(acc32, A.part);
        if (!grid_barrier(A.gb, &epoch)) return false;
        stage = 3;
        ib = A.ftmp;
        ix = A.vstar;
        irtol = A.inner_rtol;
        iwarm = warm;
        ipre = true;
    }
    o.outer_iterations = it;
    o.rel_residual = exact ? 0.0 : relres;
    o.abs_residual = absres;
    return true;
}

template <int DIM>
__global__ void __launch_bounds__(kFusedBlock, 2)
k_uzawa_fused(const int4* __restrict__ tab, const UzawaFusedArgs A) {
    __shared__ int4 s_tab[kTabWords];
    for (int i = threadIdx.x; i < kTabWords; i += blockDim.x) s_tab[i] = tab[i];
    __syncthreads();
    const FusedTable& T = *reinterpret_cast<const FusedTable*>(s_tab);
    UzawaFusedOut o;
    // a barrier that gave up is reported by the barrier's own error word (read by the host)
    if (uzawa_body<DIM>(T, A, o) && blockIdx.x == 0 && threadIdx.x == 0) *A.out = o;
}

// Algorithmic bytes of one iteration of the program: what each phase must read and write
// once (FP32 vectors, moments, BC bytes, the dense coarse inverse), no cache effects.
double program_bytes(const FusedTable& T, const std::vector<FusedPhase>& prog, int nm) {
    auto ndof = [&](int l) { return (double)T.lv[l].mk.dim * (double)T.lv[l].mk.nnode; };
    double b = 0.0;
    for (const FusedPhase& P : prog) {
        const int l = P.level;
        const double n = ndof(l), f = 4.0;
        switch (P.type) {
            case PH_APPLY:  // x in, y out, moments, BC bytes
                b += 2.0 * n * f + (double)T.lv[l].mk.nel * nm * f + (double)T.lv[l].mk.nnode;
                break;
            case PH_APPLY_P:  // + the previous direction read with z
                b += 3.0 * n * f + (double)T.lv[l].mk.nel * nm * f + (double)T.lv[l].mk.nnode;
                break;
            case PH_STEP:  // r, t, d, D⁻¹, x in; r, d, x, t out
                b += 9.0 * n * f;
                break;
            case PH_STEP_DOTS:  // + the FCG residual and Ap in, Ap zeroed
                b += 12.0 * n * f;
                break;
            case PH_RESTRICT:  // fine r, t in; coarse b (and the Chebyshev start) out
                b += 2.0 * n * f + ndof(l + 1) * f * (P.flag ? 6.0 : 1.0) + (double)T.lv[l + 1].mk.nnode;
                break;
            case PH_DENSE:
                b += (double)T.coarse_n * T.coarse_ld * f + 2.0 * T.coarse_n * f;
                break;
            case PH_PROLONG:  // coarse x in; fine x in and out, t out
                b += ndof(l + 1) * f + 3.0 * n * f + (double)T.lv[l].mk.nnode;
                break;
            case PH_RESTART:  // b, t, D⁻¹, x in; r, d, x, t out
                b += 8.0 * n * f;
                break;
            case PH_UPDATE:  // x, p, r, Ap, D⁻¹, z in; x, p, r, level-0 r, d, z, t out
                b += 13.0 * n * f;
                break;
            default:
                break;
        }
    }
    return b;
}

}  // namespace

// `iters` grid barriers in a row (the persistent kernels' barrier, nothing else): the
// cost of one phase boundary.
__global__ void __launch_bounds__(256) k_barrier_loop(int iters, GridBarrier* gb, int* failed) {
    unsigned int epoch = 0;
    for (int i = 0; i < iters; i++)
        if (!grid_barrier(gb, &epoch)) {
            if (threadIdx.x == 0) atomicAdd(failed, 1);
            return;
        }
}

// The barrier's give-up path: block 0 leaves without arriving, so every other block's wait
// runs out after `spin_limit` polls; each records that it gave up and returns.
__global__ void __launch_bounds__(256) k_barrier_abandoned(long long spin_limit, GridBarrier* gb, int* gave_up) {
    unsigned int epoch = 0;
    if (blockIdx.x == 0) return;
    if (!grid_barrier(gb, &epoch, spin_limit) && threadIdx.x == 0) atomicAdd(gave_up, 1);
}

int check_barrier_timeout(int spin_limit, int* gave_up) {
    int per_sm = 0;
    GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_abandoned, 256, 0));
    if (per_sm < 1 || spin_limit < 1) return GG_ERR_INVALID;
    const int grid = num_sms();
    GridBarrier* gb = nullptr;
    int* d_gave = nullptr;
    GG_CUDA(cudaMalloc(&gb, sizeof(GridBarrier)));
    GG_CUDA(cudaMalloc(&d_gave, sizeof(int)));
    GG_CUDA(cudaMemset(gb, 0, sizeof(GridBarrier)));
    GG_CUDA(cudaMemset(d_gave, 0, sizeof(int)));
    long long lim = spin_limit;
    void* args[] = {(void*)&lim, (void*)&gb, (void*)&d_gave};
    GG_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_abandoned, dim3(grid), dim3(256), args, 0, 0));
    GG_CUDA(cudaDeviceSynchronize());
    GG_CUDA(cudaMemcpy(gave_up, d_gave, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(gb);
    cudaFree(d_gave);
    // the status the persistent solver reports for a barrier that gave up
    return *gave_up > 0 ? GG_ERR_CUDA : GG_OK;
}

// Measurement only: microseconds per grid barrier over `iters` barriers of one cooperative
// launch with `blocks_per_sm` blocks of 256 threads per SM (CUDA events).
int time_grid_barrier(int blocks_per_sm, int iters, double* us) {
    int dev = 0, per_sm = 0;
    GG_CUDA(cudaGetDevice(&dev));
    GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_loop, 256, 0));
    if (blocks_per_sm < 1 || blocks_per_sm > per_sm || iters < 1) return GG_ERR_INVALID;
    int grid = blocks_per_sm * num_sms();
    GridBarrier* gb = nullptr;
    int* failed = nullptr;
    GG_CUDA(cudaMalloc(&gb, sizeof(GridBarrier)));
    GG_CUDA(cudaMalloc(&failed, sizeof(int)));
    cudaEvent_t e0, e1;
    GG_CUDA(cudaEventCreate(&e0));
    GG_CUDA(cudaEventCreate(&e1));
    float ms = 0.f;
    int hf = 0;
    for (int rep = 0; rep < 2; rep++) {  // the first launch warms up
        GG_CUDA(cudaMemset(gb, 0, sizeof(GridBarrier)));
        GG_CUDA(cudaMemset(failed, 0, sizeof(int)));
        void* args[] = {(void*)&iters, (void*)&gb, (void*)&failed};
        GG_CUDA(cudaEventRecord(e0, 0));
        GG_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_loop, dim3(grid), dim3(256), args, 0, 0));
        GG_CUDA(cudaEventRecord(e1, 0));
        GG_CUDA(cudaEventSynchronize(e1));
        GG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        GG_CUDA(cudaMemcpy(&hf, failed, sizeof(int), cudaMemcpyDeviceToHost));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(gb);
    cudaFree(failed);
    if (hf) return GG_ERR_CUDA;
    *us = (double)ms * 1e3 / iters;
    return GG_OK;
}

// On unless the environment sets GALE_B200_FUSED_FCG=0, which selects the graph-captured
// kernel sequence (read at every solve, so one process can compare both).
bool fused_fcg_enabled() {
    const char* e = getenv("GALE_B200_FUSED_FCG");
    return !(e && e[0] == '0');
}

// Multigrid FCG in one cooperative launch: x = K32⁻¹ b to ‖r‖ ≤ rtol‖b‖.  Returns
// GG_OK / GG_ERR_NOT_CONVERGED / GG_ERR_NONFINITE / GG_ERR_CUDA, or 1 when the hierarchy
// does not fit this kernel (the caller then runs the graph-captured solver).
// Co-resident blocks of the persistent kernel `fn` on this device (probed once per device
// and kernel slot: DIM for k_fcg_fused, 4 + DIM for k_uzawa_fused; 0 where cooperative
// launches are unavailable).
static int fused_max_blocks(int slot, const void* fn) {
    static std::mutex mu;
    static int blocks[16][8];
    static bool probed[16][8];
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16 || slot < 0 || slot >= 8) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!probed[dev][slot]) {
        int coop = 0, per_sm = 0;
        GG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        if (coop) GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kFusedBlock, 0));
        blocks[dev][slot] = per_sm * num_sms();
        probed[dev][slot] = true;
    }
    return blocks[dev][slot];
}

// The level table of the current hierarchy in device memory, for a flexible CG whose
// solution is x and right-hand side b (level 0 smooths the FCG residual H.cgr32 into
// H.z32).  Rebuilt when the hierarchy or those vectors change.  Returns 1 when the
// hierarchy does not fit the persistent kernels.
static int fused_table(Handle& H, const float* b, float* x) {
    const size_t nl = H.mg.size();
    const int deg = H.mg_degree;
    if (nl < 2 || nl > (size_t)kFusedMaxLevels || !H.coarse_n || deg < 2 || deg > 4) return 1;
    float* r = H.cgr32.as<float>();
    float* z = H.z32.as<float>();
    if (H.fused_gen != H.mg_gen || H.fused_r != r || H.fused_z != z || H.fused_x != x || H.fused_b != b) {
        FusedTable T;
        std::memset(&T, 0, sizeof T);
        T.nlevels = (int)nl;
        T.coarse_n = (int)H.coarse_n;
        T.coarse_inv = H.coarse_inv.as<float>();
        T.coarse_ld = (int)H.coarse_ld;
        for (size_t l = 0; l < nl; l++) {
            const MGLevel& L = *H.mg[l];
            FusedLevel& F = T.lv[l];
            F.mk = L.mk;
            F.mom = L.mom32;
            F.bc = L.bcmask;
            F.invd = L.invdiag.as<float>();
            F.b = l == 0 ? r : L.b.as<float>();  // level 0 smooths the FCG residual into z
            F.x = l == 0 ? z : L.x.as<float>();
            F.r = L.r.as<float>();
            F.d = L.d.as<float>();
            F.t = L.t.as<float>();
            const ChebCoef cc = cheb_coef(L.lambda_max, level_degree(H, l));
            F.inv_theta = cc.inv_theta;
            for (int k = 0; k < 4; k++) {
                F.c1[k] = cc.c1[k];
                F.c2[k] = cc.c2[k];
            }
        }
        // one iteration: the V-cycle after the level-0 start (which PH_UPDATE performs),
        // then direction, apply and update
        std::vector<FusedPhase> prog;
        auto ph = [&](uint8_t type, int level, int k = 0, int flag = 0) {
            prog.push_back(FusedPhase{type, (uint8_t)level, (uint8_t)k, (uint8_t)flag});
        };
        const int ns = (int)nl - 1;  // smoothed levels
        for (int l = 0; l < ns; l++) {
            const int dl = level_degree(H, l);
            for (int k = 1; k < dl; k++) {
                ph(PH_APPLY, l, 0, 0);
                ph(PH_STEP, l, k);
            }
            ph(PH_APPLY, l, 0, 0);
            ph(PH_RESTRICT, l, 0, l + 1 < ns ? 1 : 0);
        }
        ph(PH_DENSE, ns);
        for (int l = ns - 1; l >= 0; l--) {
            ph(PH_PROLONG, l);
            ph(PH_APPLY, l, 0, 1);
            ph(PH_RESTART, l);
            const int dl = level_degree(H, l);
            for (int k = 1; k < dl; k++) {
                ph(PH_APPLY, l, 0, 0);
                ph(l == 0 && k == dl - 1 ? PH_STEP_DOTS : PH_STEP, l, k);
            }
        }
        ph(PH_APPLY_P, 0);
        ph(PH_UPDATE, 0);
        if ((int)prog.size() > kMaxPhases) return 1;
        auto a16 = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
        bool al = a16(r) && a16(z) && a16(x) && a16(H.p32.p) && a16(H.Ap32.p);
        for (size_t l = 0; l < nl; l++) {
            const FusedLevel& F = T.lv[l];
            al = al && a16(F.invd) && a16(F.b) && a16(F.x) && a16(F.r) && a16(F.d) && a16(F.t);
        }
        // the dense phase reads the inverse's rows and the coarsest right-hand side as float4
        if (!a16(T.coarse_inv) || !a16(T.lv[nl - 1].b) || (T.coarse_ld & 3)) return 1;
        T.vec4 = al ? 1 : 0;
        T.nphase = (int)prog.size();
        H.fused_bytes_it = program_bytes(T, prog, H.nm);
        for (size_t q = 0; q < prog.size(); q++) T.ph[q] = prog[q];
        H.fused_host.assign(kTabWords * 16, 0);
        std::memcpy(H.fused_host.data(), &T, sizeof T);
        H.fused_tab.ensure(kTabWords * 16);
        GG_CUDA(cudaMemcpyAsync(H.fused_tab.p, H.fused_host.data(), kTabWords * 16, cudaMemcpyHostToDevice, H.stream));
        H.fused_gen = H.mg_gen;
        H.fused_r = r;
        H.fused_z = z;
        H.fused_x = x;
        H.fused_b = b;
        H.fused_phases = T.nphase;
    }
    return GG_OK;
}

int run_fcg_fused(Handle& H, const float* b, float* x, double rtol, int maxit, int* iters) {
    const int dim = H.dim;
    const int max_blocks =
        fused_max_blocks(dim, dim == 2 ? (const void*)k_fcg_fused<2> : (const void*)k_fcg_fused<3>);
    if (max_blocks <= 0) return 1;
    if (fused_table(H, b, x) != GG_OK) return 1;
    const int64_t n = H.ndof;
    const int64_t per = H.fused_dofs_per_block > 0 ? H.fused_dofs_per_block : kFusedBlock;
    int grid = (int)std::min<int64_t>((int64_t)max_blocks, (n + per - 1) / per);
    if (grid < 1) grid = 1;
    H.fused_part.ensure(sizeof(double) * 4 * grid);
    H.fused_bar.ensure(sizeof(GridBarrier));
    GG_CUDA(cudaMemsetAsync(H.fused_bar.p, 0, sizeof(GridBarrier), H.stream));
    const int4* tab = H.fused_tab.as<int4>();
    float* p = H.p32.as<float>();
    float* Ap = H.Ap32.as<float>();
    KrylovScalars* ks = H.scal.as<KrylovScalars>();
    double* part = H.fused_part.as<double>();
    GridBarrier* gb = H.fused_bar.as<GridBarrier>();
    void* args[] = {(void*)&tab, (void*)&b,      (void*)&x,   (void*)&p,    (void*)&Ap, (void*)&rtol,
                    (void*)&maxit, (void*)&ks, (void*)&part, (void*)&gb};
    const void* fn = dim == 2 ? (const void*)k_fcg_fused<2> : (const void*)k_fcg_fused<3>;
    GG_CUDA(cudaEventRecord(H.evf0, H.stream));
    GG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kFusedBlock), args, 0, H.stream));
    GG_CUDA(cudaEventRecord(H.evf1, H.stream));
    H.kernel_launches += 1;
    GG_CUDA(cudaMemcpyAsync(H.h_scal, ks, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, H.stream));
    int* h_err = &H.h_scal[1].failed;  // pinned scratch word for the barrier's error flag
    GG_CUDA(cudaMemcpyAsync(h_err, &gb->err, sizeof(int), cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    if (*h_err) {
        H.err = "fused multigrid solve: grid barrier timed out";
        return GG_ERR_CUDA;
    }
    *iters = H.h_scal->iterations;
    {
        float ms = 0.f;
        GG_CUDA(cudaEventElapsedTime(&ms, H.evf0, H.evf1));
        H.fused_ms_acc += ms;
        H.fused_launches_acc++;
        H.fused_its_acc += H.h_scal->iterations;
    }
    if (H.h_scal->failed == 1) return GG_ERR_NOT_CONVERGED;
    if (H.h_scal->failed) return GG_ERR_NONFINITE;
    return GG_OK;
}

// On unless the environment sets GALE_B200_FUSED_UZAWA=0, which selects the host-driven
// Uzawa loop (read at every solve).
bool fused_uzawa_enabled() {
    const char* e = getenv("GALE_B200_FUSED_UZAWA");
    return !(e && e[0] == '0');
}

int run_uzawa_fused(Handle& H, const gg_uzawa_params& prm, gg_uzawa_stats& S) {
    const int dim = H.dim;
    const void* fn = dim == 2 ? (const void*)k_uzawa_fused<2> : (const void*)k_uzawa_fused<3>;
    const int max_blocks = fused_max_blocks(4 + dim, fn);
    if (max_blocks <= 0) return 1;
    if (fused_table(H, H.r32.as<float>(), H.e32.as<float>()) != GG_OK) return 1;
    const int64_t per = H.fused_dofs_per_block > 0 ? H.fused_dofs_per_block : kFusedBlock;
    int grid = (int)std::min<int64_t>((int64_t)max_blocks, (H.ndof + per - 1) / per);
    if (grid < 1) grid = 1;
    H.fused_part.ensure(sizeof(double) * 8 * grid);
    H.fused_bar.ensure(sizeof(GridBarrier));
    H.fused_out.ensure(sizeof(UzawaFusedOut));
    GG_CUDA(cudaMemsetAsync(H.fused_bar.p, 0, sizeof(GridBarrier), H.stream));
    GG_CUDA(cudaMemsetAsync(H.fused_out.p, 0, sizeof(UzawaFusedOut), H.stream));
    UzawaFusedArgs A;
    std::memset(&A, 0, sizeof A);
    A.mom64 = H.mom64.as<double>();
    A.kdiag = H.kdiag64.as<double>();
    A.sdiag = H.sdiag.as<double>();
    A.f = H.f.as<double>();
    A.hv = H.hvec.as<double>();
    A.u = H.u.as<double>();
    A.vstar = H.vstar.as<double>();
    A.ftmp = H.ftmp.as<double>();
    A.q = H.q.as<double>();
    A.qtmp = H.qtmp.as<double>();
    A.r = H.r.as<double>();
    A.s = H.s.as<double>();
    A.r64 = H.cg_r.as<double>();
    A.acc64 = H.cg_z.as<double>();
    A.e32 = H.e32.as<float>();
    A.p32 = H.p32.as<float>();
    A.Ap32 = H.Ap32.as<float>();
    A.tolerance = prm.tolerance;
    A.inner_rtol = prm.inner_rtol_factor * prm.tolerance;
    A.scaleq = sqrt((double)H.nel);
    double gmax = 0.0;
    const int nen = 1 << dim;
    for (int a = 0; a < nen; a++)
        for (int c = 0; c < dim; c++) gmax = std::max(gmax, std::fabs(H.mk.Ge[a][c]));
    A.floor_u = 64.0 * 2.220446049250313e-16 * gmax * std::sqrt((double)nen);
    A.floor_h = 64.0 * 2.220446049250313e-16;
    A.max_iterations = prm.max_iterations;
    A.min_iterations = prm.min_iterations;
    A.use_abs = prm.use_absolute_tolerance;
    A.use_precond = prm.use_preconditioner;
    A.recycle = prm.recycle_directions;
    A.inner_maxit = prm.inner_max_iterations > 0 ? prm.inner_max_iterations : 10000;
    A.sweep_cap = std::min(A.inner_maxit, 150);
    A.out = H.fused_out.as<UzawaFusedOut>();
    A.part = H.fused_part.as<double>();
    A.gb = H.fused_bar.as<GridBarrier>();
    const int4* tab = H.fused_tab.as<int4>();
    void* args[] = {(void*)&tab, (void*)&A};
    GG_CUDA(cudaEventRecord(H.evf0, H.stream));
    GG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kFusedBlock), args, 0, H.stream));
    GG_CUDA(cudaEventRecord(H.evf1, H.stream));
    H.kernel_launches += 1;
    UzawaFusedOut o;
    GridBarrier gb;
    GG_CUDA(cudaMemcpyAsync(&o, A.out, sizeof o, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaMemcpyAsync(&gb, A.gb, sizeof gb, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    if (gb.err) {
        H.err = "fused Uzawa solve: grid barrier timed out";
        return GG_ERR_CUDA;
    }
    float ms = 0.f;
    GG_CUDA(cudaEventElapsedTime(&ms, H.evf0, H.evf1));
    S.outer_iterations = o.outer_iterations;
    S.inner_iterations += o.inner_iterations;  // after any learned-correction calibration
    S.inner_solves += o.inner_solves;
    S.rel_residual = o.rel_residual;
    S.abs_residual = o.abs_residual;
    S.fused_launches = 1;
    S.fused_iterations = o.inner_iterations;
    S.fused_ms = ms;
    S.fused_bytes_per_iteration = H.fused_bytes_it;
    S.fused_barriers_per_iteration = H.fused_phases;
    S.uzawa_fused = 1;
    H.fail_where.clear();
    static const char* kWhere[] = {"",
                                   "first inner solve (K u* = f)",
                                   "pressure right-hand side",
                                   "velocity solve K u = f - G p",
                                   "inner solve K u* = G s",
                                   "conjugate-direction step",
                                   "pressure residual",
                                   "outer iteration limit reached"};
    if (o.where > 0 && o.where < 8) {
        H.fail_where = kWhere[o.where];
        if (o.where != 7)
            H.fail_where += " at outer iteration " + std::to_string(o.outer_iterations) + " (" +
                            std::to_string(o.inner_iterations) + " inner iterations so far)";
    }
    return o.status;
}

}  // namespace gg
