// gg_noalloc.cu -- point → element location with the per-element point order, for callers
// that cannot allocate device memory.
//
// Who needs it: a host that owns all device memory through its own allocator or a fixed
// arena (a Gale/PETSc process that hands this library pre-sized buffers), real-time or
// embedded drivers that forbid allocation after start-up, and code that must not call
// cudaMalloc/cudaFree because they synchronise the device or fail in restricted contexts.
// gg_locate needs a handle, which allocates; gg_locate_noalloc does the same work — the
// bit-exact element search, the per-element histogram and scan, and the stable order of
// points inside each element — on buffers the caller passes, and keeps the counting-sort
// scratch in one file-scope __device__ array of fixed size.
//
// Limits: meshes of at most kNoAllocMaxElements elements and elements holding at most
// kNoAllocMaxPerElement points (larger inputs are rejected with an error message).
// Every call on a device shares the one scratch array and it keeps the previous call's
// contents; each call clears what must start at zero.  Calls whose work overlaps on the
// GPU (other streams, other host threads) race on the scratch and must be serialised by
// the caller.  The first call on each device looks up the array's device address
// (cudaGetSymbolAddress); make that first call before any stream capture.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {

MeshK make_mesh(const gg_mesh_desc& d);

// kernels of gg_points.cu (same arithmetic as gg_locate)
__global__ void k_locate(MeshK mk, int64_t np, const double* __restrict__ x, uint32_t* __restrict__ cell,
                         int32_t* __restrict__ count, int32_t* __restrict__ flag);
__global__ void k_scan_blocks(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ out,
                              int32_t* __restrict__ block_sums);
__global__ void k_scan_sums(int32_t* __restrict__ sums, int64_t nblocks, int32_t* __restrict__ total);
__global__ void k_scan_add(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ sums,
                           const int32_t* __restrict__ total);
__global__ void k_scatter(int64_t np, int64_t nel, const uint32_t* __restrict__ cell,
                          const int32_t* __restrict__ offsets, int32_t* __restrict__ fill,
                          int32_t* __restrict__ unsorted);

namespace {

constexpr int64_t kNoAllocMaxElements = 1 << 20;  // 1,048,576 elements
constexpr int kNoAllocMaxPerElement = 1024;       // points per element
constexpr int64_t kScanBlocks = (kNoAllocMaxElements + 1023) / 1024;
// layout: [counts: max+1][block sums: kScanBlocks+2][flags: 4]
constexpr int64_t kCountsOff = 0;
constexpr int64_t kSumsOff = kNoAllocMaxElements + 1;
constexpr int64_t kFlagsOff = kSumsOff + kScanBlocks + 2;
constexpr int64_t kScratchWords = kFlagsOff + 4;
constexpr int kMaxDevices = 64;

__device__ __align__(256) int32_t g_noalloc_scratch[kScratchWords];

int32_t* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// One warp per element: sort the element's point indices ascending, in place, through a
// per-warp shared-memory copy (the point indices are distinct).  Flags an element that
// holds more than kNoAllocMaxPerElement points.
__global__ void k_segsort_inplace(int64_t nel, const int32_t* __restrict__ offsets, int32_t* __restrict__ order,
                                  int32_t* __restrict__ flags) {
    constexpr int kWarps = 4;
    __shared__ int32_t seg[kWarps][kNoAllocMaxPerElement];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e = warp; e < nel; e += nwarps) {
        const int32_t b = offsets[e], n = offsets[e + 1] - b;
        if (n > kNoAllocMaxPerElement) {
            if (lane == 0) atomicAdd(&flags[1], 1);
            continue;
        }
        for (int k = lane; k < n; k += 32) seg[wib][k] = order[b + k];
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            const int32_t v = seg[wib][k];
            int rank = 0;
            for (int j = 0; j < n; j++) rank += (seg[wib][j] < v);
            order[b + rank] = v;
        }
        __syncwarp();
    }
}

int grid_of(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g > 148 * 16) g = 148 * 16;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace
}  // namespace gg

extern "C" GG_API int gg_locate_noalloc(const gg_mesh_desc* mesh, int64_t n_points, const double* d_coords,
                                        uint32_t* d_cell, int32_t* d_offsets, int32_t* d_order,
                                        int64_t* n_outside, void* stream, const char** message) {
    using namespace gg;
    const char* dummy;
    const char** msg = message ? message : &dummy;
    *msg = "";
    if (!mesh || !d_coords || !d_cell || !d_offsets || !d_order) {
        *msg = "gg_locate_noalloc: null argument";
        return GG_ERR_INVALID;
    }
    if (mesh->dim != 2 && mesh->dim != 3) {
        *msg = "gg_locate_noalloc: dim must be 2 or 3";
        return GG_ERR_INVALID;
    }
    int64_t nel = 1;
    for (int d = 0; d < mesh->dim; d++) {
        if (mesh->elements[d] < 1 || !(mesh->max[d] > mesh->min[d])) {
            *msg = "gg_locate_noalloc: invalid mesh extent";
            return GG_ERR_INVALID;
        }
        nel *= mesh->elements[d];
    }
    if (nel > kNoAllocMaxElements) {
        *msg = "gg_locate_noalloc: mesh exceeds the 1048576-element scratch of the no-allocation path";
        return GG_ERR_INVALID;
    }
    if (n_points < 1 || n_points >= (int64_t)INT32_MAX) {
        *msg = "gg_locate_noalloc: point count must be in [1, 2^31-1)";
        return GG_ERR_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        *msg = "gg_locate_noalloc: no CUDA device";
        return GG_ERR_NO_DEVICE;
    }
    // an error the caller left pending is not this call's: report it, leave it in place
    // (cudaPeekAtLastError does not clear it) and launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) {
        *msg = "gg_locate_noalloc: a CUDA error was pending before the call";
        return GG_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        *msg = "gg_locate_noalloc: device index beyond 64";
        return GG_ERR_INVALID;
    }
    {
        // set-up, once per device, with that device current: the scratch array's address
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                *msg = "gg_locate_noalloc: cudaGetSymbolAddress failed";
                return GG_ERR_CUDA;
            }
            g_scratch_addr[dev] = static_cast<int32_t*>(p);
        }
    }
    int32_t* scratch = g_scratch_addr[dev];
    int32_t* counts = scratch + kCountsOff;
    int32_t* sums = scratch + kSumsOff;
    int32_t* flags = scratch + kFlagsOff;  // [0] outside points, [1] oversized elements
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const MeshK mk = make_mesh(*mesh);
    const int64_t nblk = (nel + 1023) / 1024;
    // the scratch keeps the previous call's contents: clear the counters and the flags
    if (cudaMemsetAsync(counts, 0, sizeof(int32_t) * (nel + 1), st) != cudaSuccess ||
        cudaMemsetAsync(flags, 0, sizeof(int32_t) * 4, st) != cudaSuccess) {
        *msg = "gg_locate_noalloc: cudaMemsetAsync failed";
        return GG_ERR_CUDA;
    }
    // each launch is checked on its own, so a failure names the kernel that raised it
    auto launched = [&](const char* what) {
        if (cudaGetLastError() == cudaSuccess) return true;
        *msg = what;
        return false;
    };
    k_locate<<<grid_of(n_points, 256), 256, 0, st>>>(mk, n_points, d_coords, d_cell, counts, flags);
    if (!launched("gg_locate_noalloc: launch of the location kernel failed")) return GG_ERR_CUDA;
    k_scan_blocks<<<(int)nblk, 1024, 0, st>>>(counts, nel, d_offsets, sums);
    if (!launched("gg_locate_noalloc: launch of the block scan failed")) return GG_ERR_CUDA;
    k_scan_sums<<<1, 1024, 0, st>>>(sums, nblk, sums + nblk);
    if (!launched("gg_locate_noalloc: launch of the block-sum scan failed")) return GG_ERR_CUDA;
    k_scan_add<<<(int)nblk, 1024, 0, st>>>(d_offsets, nel, sums, sums + nblk);
    if (!launched("gg_locate_noalloc: launch of the scan fix-up failed")) return GG_ERR_CUDA;
    if (cudaMemsetAsync(counts, 0, sizeof(int32_t) * (nel + 1), st) != cudaSuccess) {
        *msg = "gg_locate_noalloc: cudaMemsetAsync failed";
        return GG_ERR_CUDA;
    }
    k_scatter<<<grid_of(n_points, 256), 256, 0, st>>>(n_points, nel, d_cell, d_offsets, counts, d_order);
    if (!launched("gg_locate_noalloc: launch of the scatter failed")) return GG_ERR_CUDA;
    k_segsort_inplace<<<grid_of(nel * 32, 128), 128, 0, st>>>(nel, d_offsets, d_order, flags);
    if (!launched("gg_locate_noalloc: launch of the per-element sort failed")) return GG_ERR_CUDA;
    int32_t hflags[2] = {0, 0};
    if (cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        *msg = "gg_locate_noalloc: CUDA error while reading the flags";
        return GG_ERR_CUDA;
    }
    if (n_outside) *n_outside = hflags[0];
    if (hflags[1]) {
        *msg = "gg_locate_noalloc: an element holds more than 1024 points";
        return GG_ERR_INVALID;
    }
    if (hflags[0]) {
        *msg = "gg_locate_noalloc: material points outside the mesh (cell = element count)";
        return GG_ERR_OUT_OF_DOMAIN;
    }
    return GG_OK;
}
