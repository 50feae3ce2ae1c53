// gg_points.cu -- material point → element mapping on sm_100a.
//
//  k_locate        bit-exact Mesh_RegularAlgorithms_SearchElements
//                  (StgDomain/Mesh/src/Mesh_RegularAlgorithms.cxx:191-224) + per-element
//                  histogram
//  k_scan_*        exclusive scan of the histogram → CSR offsets
//  k_scatter       counting-sort scatter (arbitrary order inside an element)
//  k_segsort       per-element rank sort by input index, which restores the order that
//                  _CoincidentMapper_Map (PICellerator/MaterialPoints/src/
//                  CoincidentMapper.cxx:190-215) rebuilds: increasing point index
//  k_gather_points ξ (closed form of the Newton step of ElementType.cxx:221-338 on an
//                  axis-aligned element), material, plastic strain in sorted order
//
// All integer work; HBM-bound.  Every kernel is grid-stride and sized from the SM count.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {

__global__ void k_locate(MeshK mk, int64_t np, const double* __restrict__ x,
                         uint32_t* __restrict__ cell, int32_t* __restrict__ count,
                         int32_t* __restrict__ flag) {
    const int dim = mk.dim;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        int inds[3] = {0, 0, 0};
        bool inside = true;
        for (int d = 0; d < dim; d++) {
            const double v = x[p * dim + d];
            const double dmax = __dsub_rn(v, mk.max[d]);
            if (dmax >= -1e-12 && dmax <= 1e-12) {          // Num_Approx(x - max, 0)
                inds[d] = mk.n[d] - 1;
            } else if (v < mk.min[d] || v > mk.max[d]) {
                inside = false;
            } else {
                const double out = __ddiv_rn(__dsub_rn(v, mk.min[d]), mk.sep[d]);
                const double ip = trunc(out);               // modf: integral part
                const double frac = __dsub_rn(out, ip);     // exact fractional part
                int i = (int)ip;
                if (i > 0 && frac >= -1e-12 && frac <= 1e-12) i--;  // lower element wins
                if (i >= mk.n[d]) i = mk.n[d] - 1;
                inds[d] = i;
            }
        }
        if (inside) {
            const int64_t e = inds[0] + (int64_t)mk.n[0] * (inds[1] + (int64_t)mk.n[1] * inds[2]);
            cell[p] = (uint32_t)e;
            atomicAdd(&count[e], 1);
        } else {
            cell[p] = (uint32_t)mk.nel;
            atomicAdd(flag, 1);
        }
    }
}

// ---- exclusive scan, 3 phases (1024 items per block) -------------------------------
__global__ void k_scan_blocks(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ out,
                              int32_t* __restrict__ block_sums) {
    __shared__ int32_t warp_tot[32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t v = i < n ? in[i] : 0;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        int32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_tot[lane] = wi - w;  // exclusive prefix of warp totals
        if (lane == 31) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    if (i < n) out[i] = incl - v + warp_tot[wid];
}

__global__ void k_scan_sums(int32_t* __restrict__ sums, int64_t nblocks, int32_t* __restrict__ total) {
    // one block: sequential carry over chunks of blockDim
    __shared__ int32_t warp_tot[32];
    __shared__ int32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t base = 0; base < nblocks; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int32_t v = i < nblocks ? sums[i] : 0;
        int32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int32_t w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
            int32_t wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            warp_tot[lane] = wi - w;
        }
        __syncthreads();
        const int32_t c = carry;
        if (i < nblocks) sums[i] = c + incl - v + warp_tot[wid];
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c + incl + warp_tot[wid];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ sums,
                           const int32_t* __restrict__ total) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
    if (i == 0) out[n] = *total;
}

__global__ void k_scatter(int64_t np, int64_t nel, const uint32_t* __restrict__ cell,
                          const int32_t* __restrict__ offsets, int32_t* __restrict__ fill,
                          int32_t* __restrict__ unsorted) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t e = cell[p];
        if (e < (uint32_t)nel) unsorted[offsets[e] + atomicAdd(&fill[e], 1)] = (int32_t)p;
    }
}

// One warp per element: rank each point index by the number of smaller indices in the
// element's segment (indices are distinct), which sorts the segment ascending.
__global__ void k_segsort(int64_t nel, const int32_t* __restrict__ offsets,
                          const int32_t* __restrict__ unsorted, int32_t* __restrict__ perm) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e = warp; e < nel; e += nwarps) {
        const int32_t b = offsets[e], n = offsets[e + 1] - b;
        if (n <= 32) {
            const int32_t v = lane < n ? unsorted[b + lane] : INT32_MAX;
            int rank = 0;
            for (int j = 0; j < n; j++) rank += (__shfl_sync(0xffffffffu, v, j) < v);
            if (lane < n) perm[b + rank] = v;
        } else {
            for (int k = lane; k < n; k += 32) {
                const int32_t v = unsorted[b + k];
                int rank = 0;
                for (int j = 0; j < n; j++) rank += (unsorted[b + j] < v);
                perm[b + rank] = v;
            }
        }
    }
}

__global__ void k_gather_points(MeshK mk, int64_t np_in, const int32_t* __restrict__ perm,
                                const uint32_t* __restrict__ cell, const double* __restrict__ x,
                                const int32_t* __restrict__ mat_in, const double* __restrict__ ps_in,
                                int32_t* __restrict__ cell_s, double* __restrict__ xi_s,
                                int32_t* __restrict__ mat_s, double* __restrict__ ps_s) {
    const int dim = mk.dim;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np_in;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[i];
        const uint32_t e = cell[p];
        cell_s[i] = (int32_t)e;
        mat_s[i] = mat_in[p];
        ps_s[i] = ps_in[p];
        int idx[3];
        idx[0] = (int)(e % (uint32_t)mk.n[0]);
        idx[1] = (int)((e / (uint32_t)mk.n[0]) % (uint32_t)mk.n[1]);
        idx[2] = (int)(e / ((uint32_t)mk.n[0] * (uint32_t)mk.n[1]));
        for (int d = 0; d < dim; d++) {
            const double lo = vert_coord_d(mk, d, idx[d]), hi = vert_coord_d(mk, d, idx[d] + 1);
            // Newton from ξ=0 on an affine element: J = (hi-lo)/2, rhs = x - (lo+hi)/2
            const double c = __dmul_rn(0.5, __dadd_rn(lo, hi));
            const double J = __dmul_rn(0.5, __dsub_rn(hi, lo));
            xi_s[(int64_t)d * np_in + i] = __ddiv_rn(__dsub_rn(x[(int64_t)p * dim + d], c), J);
        }
    }
}

// ------------------------------------------------------------------ host driver ----
int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    const int cap = num_sms() * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// out = exclusive prefix sum of in[0..n) (device), *total_host = the sum (synchronises).
void exclusive_scan_i32(Handle& H, const int32_t* in, int32_t* out, int64_t n, DBuf& tmp, int32_t* total_host) {
    cudaStream_t st = H.stream;
    const int64_t nblk = (n + 1023) / 1024;
    tmp.ensure(sizeof(int32_t) * (nblk + 2));
    if (n > 0) {
        k_scan_blocks<<<(int)nblk, 1024, 0, st>>>(in, n, out, tmp.as<int32_t>());
        k_scan_sums<<<1, 1024, 0, st>>>(tmp.as<int32_t>(), nblk, tmp.as<int32_t>() + nblk);
        k_scan_add<<<(int)nblk, 1024, 0, st>>>(out, n, tmp.as<int32_t>(), tmp.as<int32_t>() + nblk);
        GG_CUDA(cudaGetLastError());
        GG_CUDA(cudaMemcpyAsync(total_host, tmp.as<int32_t>() + nblk, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    } else {
        *total_host = 0;
    }
    GG_CUDA(cudaStreamSynchronize(st));
}

// Locate + stable counting sort + gather.  Returns number of points outside the mesh.
int64_t locate_and_sort(Handle& H) {
    const int64_t np = H.np, nel = H.nel;
    cudaStream_t st = H.stream;
    H.offsets.ensure(sizeof(int32_t) * (nel + 1));
    H.fill.ensure(sizeof(int32_t) * (nel + 1));
    const int64_t nblk = (nel + 1023) / 1024;
    H.scan_tmp.ensure(sizeof(int32_t) * (nblk + 2));
    H.flag.ensure(sizeof(int32_t) * 4);
    GG_CUDA(cudaMemsetAsync(H.fill.p, 0, sizeof(int32_t) * (nel + 1), st));
    GG_CUDA(cudaMemsetAsync(H.flag.p, 0, sizeof(int32_t) * 4, st));
    k_locate<<<grid_for(np, 256), 256, 0, st>>>(H.mk, np, H.coords.as<double>(), H.cell.as<uint32_t>(),
                                                  H.fill.as<int32_t>(), H.flag.as<int32_t>());
    GG_CUDA(cudaGetLastError());
    k_scan_blocks<<<(int)nblk, 1024, 0, st>>>(H.fill.as<int32_t>(), nel, H.offsets.as<int32_t>(),
                                              H.scan_tmp.as<int32_t>());
    k_scan_sums<<<1, 1024, 0, st>>>(H.scan_tmp.as<int32_t>(), nblk, H.scan_tmp.as<int32_t>() + nblk);
    k_scan_add<<<(int)nblk, 1024, 0, st>>>(H.offsets.as<int32_t>(), nel, H.scan_tmp.as<int32_t>(),
                                           H.scan_tmp.as<int32_t>() + nblk);
    GG_CUDA(cudaGetLastError());
    int32_t outside = 0;
    GG_CUDA(cudaMemcpyAsync(&outside, H.flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GG_CUDA(cudaStreamSynchronize(st));
    GG_CUDA(cudaMemsetAsync(H.fill.p, 0, sizeof(int32_t) * (nel + 1), st));
    k_scatter<<<grid_for(np, 256), 256, 0, st>>>(np, nel, H.cell.as<uint32_t>(), H.offsets.as<int32_t>(),
                                                   H.fill.as<int32_t>(), H.cell_s.as<int32_t>());
    // cell_s doubles as the unsorted permutation until k_gather_points overwrites it
    k_segsort<<<grid_for(nel * 32, 256), 256, 0, st>>>(nel, H.offsets.as<int32_t>(), H.cell_s.as<int32_t>(),
                                                        H.perm.as<int32_t>());
    const int64_t np_in = np - outside;
    k_gather_points<<<grid_for(np_in, 256), 256, 0, st>>>(
        H.mk, np_in, H.perm.as<int32_t>(), H.cell.as<uint32_t>(), H.coords.as<double>(),
        H.mat_in.as<int32_t>(), H.ps_in.as<double>(), H.cell_s.as<int32_t>(), H.xi_s.as<double>(),
        H.mat_s.as<int32_t>(), H.ps_s.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaStreamSynchronize(st));
    return outside;
}

}  // namespace gg
