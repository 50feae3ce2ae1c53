// gg_alloc.cu -- the device memory behind every handle buffer (DBuf).
//
// A handle sizes some 70 buffers on its first solve.  Through cudaMalloc those calls
// serialise in the driver: in a batch of 512 small problems driven by 64 host threads they
// took most of the wall time (36 k calls, 536 s summed over the threads, the batch at 53
// solves/s against 96 once every buffer existed).  Buffers of up to 4 MB therefore come from
// per-device pools: power-of-two size classes (256 B … 4 MB) carved from 64 MB chunks, with
// a free list per class, under one mutex per device.  Larger buffers (the fine-level
// moments, points and vectors of big meshes) still use cudaMalloc / cudaFree directly.
// Chunks stay with the process until it exits.
//
// Reuse is as safe as with cudaFree, which synchronises the device: a block goes back on its
// free list only after cudaDeviceSynchronize, so no kernel of any stream still uses it when
// another handle is given it.
#include <mutex>
#include <vector>

#include "gg_handle.h"

namespace gg {

namespace {

constexpr int kMinShift = 8;   // 256 B: every block keeps cudaMalloc's 256-byte alignment
constexpr int kMaxShift = 22;  // 4 MB
constexpr size_t kChunk = size_t(64) << 20;
constexpr int kMaxDevices = 64;

struct DevicePool {
    std::mutex mu;
    std::vector<void*> free_list[kMaxShift + 1];
    char* cur = nullptr;
    size_t left = 0;
};

// Never destroyed: a buffer released while the process exits still finds its pool.
DevicePool& pool(int dev) {
    static DevicePool* pools = new DevicePool[kMaxDevices];
    return pools[dev];
}

int size_class(size_t bytes) {
    int s = kMinShift;
    while ((size_t(1) << s) < bytes) s++;
    return s;
}

}  // namespace

void* dev_alloc(size_t bytes, int* dev_out) {
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    *dev_out = dev;
    if (bytes > (size_t(1) << kMaxShift) || dev < 0 || dev >= kMaxDevices) {
        void* p = nullptr;
        GG_CUDA(cudaMalloc(&p, bytes));
        return p;
    }
    const int s = size_class(bytes);
    const size_t sz = size_t(1) << s;
    DevicePool& P = pool(dev);
    std::lock_guard<std::mutex> lk(P.mu);
    std::vector<void*>& fl = P.free_list[s];
    if (!fl.empty()) {
        void* p = fl.back();
        fl.pop_back();
        return p;
    }
    if (P.left < sz) {  // the rest of the current chunk (< 4 MB) is left unused
        void* c = nullptr;
        GG_CUDA(cudaMalloc(&c, kChunk));
        P.cur = static_cast<char*>(c);
        P.left = kChunk;
    }
    void* p = P.cur;
    P.cur += sz;
    P.left -= sz;
    return p;
}

void dev_free(void* p, size_t bytes, int dev) {
    if (!p) return;
    if (bytes > (size_t(1) << kMaxShift) || dev < 0 || dev >= kMaxDevices) {
        cudaFree(p);
        return;
    }
    int cur = 0;
    const bool switched = cudaGetDevice(&cur) == cudaSuccess && cur != dev;
    if (switched) cudaSetDevice(dev);
    cudaDeviceSynchronize();  // as cudaFree would: no stream of this device still uses p
    if (switched) cudaSetDevice(cur);
    DevicePool& P = pool(dev);
    std::lock_guard<std::mutex> lk(P.mu);
    P.free_list[size_class(bytes)].push_back(p);
}

}  // namespace gg
