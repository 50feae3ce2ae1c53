// gg_advect.cu -- material point advection on sm_100a.
//
// TimeIntegrand_SecondOrder (StgDomain/Utils/src/TimeIntegrand.cxx:265-335) and the Euler
// update, with _SwarmAdvector_TimeDeriv (PICellerator/MaterialPoints/src/SwarmAdvector.cxx:
// 261-287) as the derivative: locate (the bit-exact search of gg_points.cu), local
// coordinate, Q1 interpolation of the nodal velocity.  A corrector position outside the
// mesh falls back to the first-order update from the start position
// (_TimeIntegrand_RewindToStartAndApplyFirstOrderUpdate, :457-483); a predictor outside
// the mesh is an error (the reference's Journal_Firewall).  Position updates use explicit
// roundings (no FMA contraction), as the x86-64 reference build computes them.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {

namespace {

template <int DIM>
__device__ bool velocity_at(const MeshK& mk, const double* x, const double* __restrict__ u, double* v) {
    int inds[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double dmax = __dsub_rn(x[d], mk.max[d]);
        if (dmax >= -1e-12 && dmax <= 1e-12) {
            inds[d] = mk.n[d] - 1;
        } else if (x[d] < mk.min[d] || x[d] > mk.max[d]) {
            return false;
        } else {
            const double out = __ddiv_rn(__dsub_rn(x[d], mk.min[d]), mk.sep[d]);
            const double ip = trunc(out);
            const double frac = __dsub_rn(out, ip);
            int i = (int)ip;
            if (i > 0 && frac >= -1e-12 && frac <= 1e-12) i--;
            if (i >= mk.n[d]) i = mk.n[d] - 1;
            inds[d] = i;
        }
    }
    double xi[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double lo = vert_coord_d(mk, d, inds[d]), hi = vert_coord_d(mk, d, inds[d] + 1);
        xi[d] = __ddiv_rn(__dsub_rn(x[d], __dmul_rn(0.5, __dadd_rn(lo, hi))), __dmul_rn(0.5, __dsub_rn(hi, lo)));
    }
#pragma unroll
    for (int c = 0; c < DIM; c++) v[c] = 0.0;
#pragma unroll
    for (int a = 0; a < (1 << DIM); a++) {
        double N = (DIM == 2) ? 0.25 : 0.125;
#pragma unroll
        for (int d = 0; d < DIM; d++) N *= 1.0 + (((a >> d) & 1) ? xi[d] : -xi[d]);
        const int64_t n = elem_node<DIM>(mk, inds, a);
#pragma unroll
        for (int c = 0; c < DIM; c++) v[c] += u[(int64_t)c * mk.nnode + n] * N;
    }
#pragma unroll
    for (int c = 0; c < DIM; c++)
        if (isinf(v[c])) return false;
    return true;
}

template <int DIM>
__global__ void k_advect(MeshK mk, int64_t np, double dt, int order, const double* __restrict__ u,
                         double* __restrict__ coords, int32_t* __restrict__ flag) {
    const double hdt = __dmul_rn(0.5, dt);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        double x0[3], x[3], k1[3], k2[3];
#pragma unroll
        for (int c = 0; c < DIM; c++) x0[c] = coords[p * DIM + c];
        if (!velocity_at<DIM>(mk, x0, u, k1)) {
            atomicAdd(flag, 1);
            continue;
        }
        if (order == 1) {
#pragma unroll
            for (int c = 0; c < DIM; c++) x[c] = __dadd_rn(x0[c], __dmul_rn(dt, k1[c]));
        } else {
#pragma unroll
            for (int c = 0; c < DIM; c++) x[c] = __dadd_rn(x0[c], __dmul_rn(hdt, k1[c]));
            if (velocity_at<DIM>(mk, x, u, k2)) {
#pragma unroll
                for (int c = 0; c < DIM; c++) x[c] = __dadd_rn(x0[c], __dmul_rn(dt, k2[c]));
            } else {
#pragma unroll
                for (int c = 0; c < DIM; c++) x[c] = __dadd_rn(x0[c], __dmul_rn(dt, k1[c]));
            }
        }
#pragma unroll
        for (int c = 0; c < DIM; c++) coords[p * DIM + c] = x[c];
    }
}

}  // namespace

int advect(Handle& H, double dt, int order, const double* d_u, double* d_out) {
    (void)d_out;
    H.flag.ensure(sizeof(int32_t) * 4);
    GG_CUDA(cudaMemsetAsync(H.flag.p, 0, sizeof(int32_t) * 4, H.stream));
    const int g = grid_for(H.np, 256);
    if (H.dim == 2)
        k_advect<2><<<g, 256, 0, H.stream>>>(H.mk, H.np, dt, order, d_u, H.coords.as<double>(), H.flag.as<int32_t>());
    else
        k_advect<3><<<g, 256, 0, H.stream>>>(H.mk, H.np, dt, order, d_u, H.coords.as<double>(), H.flag.as<int32_t>());
    GG_CUDA(cudaGetLastError());
    int32_t bad = 0;
    GG_CUDA(cudaMemcpyAsync(&bad, H.flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    H.located = false;
    H.built = false;
    return bad ? GG_ERR_OUT_OF_DOMAIN : GG_OK;
}

}  // namespace gg
