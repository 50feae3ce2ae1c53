// gg_internal.cuh -- shared device/host definitions of the sm_100a Stokes path.
//
// Data layout in HBM (one handle = one regular Q1-P0 mesh):
//   nodal vectors      SoA  [dim][nnode]      (component c of node n at c*nnode + n)
//   element moments    SoA  [n_mom][nel]      (moment m of element e at m*nel + e)
//   element scalars         [nel]             (pressure, Schur diagonal, h)
//   material points    sorted by owning element (stable: increasing input index, the
//                      order _CoincidentMapper_Map rebuilds per cell), CSR offsets [nel+1]
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/gale_gpu.h"

#define GG_CUDA(call)                                                               \
    do {                                                                            \
        cudaError_t _e = (call);                                                    \
        if (_e != cudaSuccess) {                                                    \
            throw gg::CudaError(_e, #call, __FILE__, __LINE__);                     \
        }                                                                           \
    } while (0)

namespace gg {

struct CudaError {
    cudaError_t err;
    std::string what;
    CudaError(cudaError_t e, const char* call, const char* file, int line) : err(e) {
        what = std::string(cudaGetErrorString(e)) + " in " + call + " at " + file + ":" +
               std::to_string(line);
    }
};

struct Status {
    int code;
    std::string msg;
};

// Mesh constants passed by value to kernels.
struct MeshK {
    int dim;
    int n[3];       // elements per axis (1 for unused axes)
    int nn[3];      // nodes per axis
    int64_t nel, nnode;
    double min[3], max[3];
    double sep[3];  // (max-min)/n: Mesh_RegularAlgorithms_Update separation
    double h[3];    // element size used by the closed-form shape derivatives
    double detJ;    // Π h/2
    double kappa[3];// 2 / (h_d 2^dim): ∂N/∂x_d = kappa_d * s_d * Π_{e≠d}(1 + s_e ξ_e)
    double Ge[8][3];// element gradient stencil on the 2^dim Gauss swarm
};

constexpr int kMaxMom = 23;

// Moment slot of monomial ξ^a η^b ζ^c (exponents ≤ 2), -1 when not stored.
// 2D order: 1, ξ, η, ξ², η², ξη.  3D order: ascending a + 3b + 9c skipping the four
// monomials with no zero exponent and two or more exponents equal to 2.
__host__ __device__ constexpr int mom_slot2(int a, int b) {
    return (a == 0 && b == 0) ? 0 : (a == 1 && b == 0) ? 1 : (a == 0 && b == 1) ? 2
         : (a == 2 && b == 0) ? 3 : (a == 0 && b == 2) ? 4 : (a == 1 && b == 1) ? 5 : -1;
}
__host__ __device__ constexpr bool mom_kept3(int a, int b, int c) {
    return !((a != 0 && b != 0 && c != 0) && ((a == 2) + (b == 2) + (c == 2) >= 2));
}
__host__ __device__ constexpr int mom_slot3(int a, int b, int c) {
    int idx = a + 3 * b + 9 * c, slot = 0;
    for (int q = 0; q < idx; q++)
        if (mom_kept3(q % 3, (q / 3) % 3, q / 9)) slot++;
    return mom_kept3(a, b, c) ? slot : -1;
}
template <int DIM>
__host__ __device__ constexpr int n_moments() { return DIM == 2 ? 6 : 23; }
template <int DIM>
__host__ __device__ constexpr int mom_slot(int a, int b, int c) {
    return DIM == 2 ? mom_slot2(a, b) : mom_slot3(a, b, c);
}


}  // namespace gg
