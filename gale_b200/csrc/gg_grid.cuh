// gg_grid.cuh -- the grid-wide barrier of the persistent cooperative kernels.
#pragma once

#include "gg_internal.cuh"

namespace gg {
namespace {

// a barrier gives up after this many polls (each an L2 round trip): a few seconds, where a
// healthy phase takes microseconds to a millisecond
constexpr long long kBarrierSpinLimit = 1ll << 22;

struct GridBarrier {
    unsigned int arrive;  // arrivals since the launch (zeroed by the host before it)
    unsigned int pad0;
    int err;              // set by a block whose wait gave up
    int pad1;
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All blocks of the grid meet here.  Arrival is a release reduction on a counter that only
// grows (barrier e of the launch completes when it reaches e·gridDim.x, modulo 2^32: the
// counter runs at most gridDim.x ahead of or behind a waiting block's target, so the
// signed difference decides and a launch may pass any number of barriers); waiting is an
// acquire poll of that counter.  The release/acquire pair orders every write of the block
// (made visible to thread 0 by __syncthreads) before every read after the barrier.
// Returns false (uniformly within the block) once any block has given up waiting; the
// caller then leaves the kernel.
__device__ __noinline__ bool grid_barrier(GridBarrier* gb, unsigned int* epoch,
                                          long long spin_limit = kBarrierSpinLimit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int target = (*epoch + 1) * gridDim.x;
        int ok = 1;
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(&gb->arrive), "r"(1u) : "memory");
        long long spins = 0;
        while ((int)(ld_acquire_gpu(&gb->arrive) - target) < 0) {
            if (++spins > spin_limit || ((spins & 1023) == 0 && *(volatile int*)&gb->err)) {
                atomicExch(&gb->err, 1);
                ok = 0;
                break;
            }
        }
        s_ok = ok;
        *epoch = *epoch + 1;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace
}  // namespace gg
