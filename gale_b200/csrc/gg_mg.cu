// gg_mg.cu -- geometric multigrid for the inner velocity solve (FP32), sm_100a.
//
// Design reference: Gale's PETScMGSolver + SROpGenerator (StgFEM/SLE/SystemSetup/src/
// PETScMGSolver.cxx:240,513-522,654-704; SROpGenerator.cxx:157-467): geometric levels of
// the regular mesh, a Q1 interpolation between them, smoothed V-cycles as the
// preconditioner of the velocity Krylov solve.  Built B200-first instead of around
// assembled PETSc matrices:
//   * coarse operators are re-discretised from the PIC quadrature itself: the moments
//     of a coarse element are an exact linear re-expansion of its children's moments
//     (ξ_coarse = (ξ_child ± 1)/2), so every level is matrix-free with the same kernel;
//   * smoothing is Chebyshev–Jacobi (eigen-bound from a power iteration), which is a
//     fixed polynomial of D⁻¹A — no inner products inside the V-cycle;
//   * the coarsest level (≤ 3000 dofs) is solved by a dense FP32 inverse (one mat-vec),
//     computed on the device by blocked Gauss–Jordan;
//   * the whole V-cycle is a fixed kernel sequence and is captured into the inner
//     Krylov iteration's CUDA graph; every kernel exits early once the solve is done.
// The V-cycle preconditions a flexible CG (Notay's truncated FCG) so that the learned
// coarse correction (gg_learned.cu) may be added to it.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {

MeshK make_mesh(const gg_mesh_desc& d);

namespace {

constexpr int kMinCoarse = 4;      // coarsen while every axis is even and ≥ 4 elements
// … and the level has more dofs than this.  The dense inverse of the coarsest level is
// rebuilt at every operator build (Picard iterations included) by blocked Gauss–Jordan
// (n³ FP64 multiply-adds); one dense mat-vec then replaces the V-cycle's levels below it,
// each of whose phases is bound by latency, not work (64³: 8³ = 2,187 dofs is the
// coarsest level, and the 8³ and 4³ cycles' ten phases per iteration become one)
constexpr int64_t kDenseStop = 3000;

__device__ __forceinline__ double tcoef(int a, int ap, double o) {
    // ξ_c = (ξ_f + o)/2  ⇒  ξ_c^a = Σ_{a'≤a} T[a][a'] ξ_f^{a'}
    if (a == 0) return ap == 0 ? 1.0 : 0.0;
    if (a == 1) return ap == 0 ? 0.5 * o : (ap == 1 ? 0.5 : 0.0);
    return ap == 0 ? 0.25 : (ap == 1 ? 0.5 * o : 0.25);
}

template <int DIM>
__global__ void k_coarsen_moments(MeshK fk, MeshK ck, const double* __restrict__ mf,
                                  double* __restrict__ mc, float* __restrict__ mc32) {
    constexpr int NM = n_moments<DIM>();
    for (int64_t E = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; E < ck.nel;
         E += (int64_t)gridDim.x * blockDim.x) {
        const int I = (int)(E % ck.n[0]);
        const int64_t rr = E / ck.n[0];
        const int J = (int)(rr % ck.n[1]), K = (int)(rr / ck.n[1]);
        double acc[NM];
#pragma unroll
        for (int q = 0; q < NM; q++) acc[q] = 0.0;
#pragma unroll
        for (int ch = 0; ch < (1 << DIM); ch++) {
            const int dx = ch & 1, dy = (ch >> 1) & 1, dz = DIM == 3 ? (ch >> 2) & 1 : 0;
            const int64_t fe = (2 * I + dx) + (int64_t)fk.n[0] * ((2 * J + dy) + (int64_t)fk.n[1] * (2 * K + dz));
            const double ox = 2.0 * dx - 1.0, oy = 2.0 * dy - 1.0, oz = 2.0 * dz - 1.0;
            double f[NM];
#pragma unroll
            for (int q = 0; q < NM; q++) f[q] = mf[(int64_t)q * fk.nel + fe];
#pragma unroll
            for (int c = 0; c < (DIM == 3 ? 3 : 1); c++)
#pragma unroll
                for (int b = 0; b < 3; b++)
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const int so = mom_slot<DIM>(a, b, c);
                        if (so < 0) continue;
                        double s = 0.0;
#pragma unroll
                        for (int cp = 0; cp <= c; cp++)
#pragma unroll
                            for (int bp = 0; bp <= b; bp++)
#pragma unroll
                                for (int ap = 0; ap <= a; ap++) {
                                    const int si = mom_slot<DIM>(ap, bp, cp);
                                    if (si < 0) continue;
                                    s += tcoef(a, ap, ox) * tcoef(b, bp, oy) * (DIM == 3 ? tcoef(c, cp, oz) : 1.0) * f[si];
                                }
                        acc[so] += s;
                    }
        }
#pragma unroll
        for (int q = 0; q < NM; q++) {
            mc[(int64_t)q * ck.nel + E] = acc[q];
            mc32[(int64_t)q * ck.nel + E] = (float)acc[q];
        }
    }
}

// Jacobi diagonal of a level from its moments (same closed form as the build kernel).
template <int DIM>
__global__ void k_level_diag(MeshK mk, const double* __restrict__ mom, float* __restrict__ diag) {
    constexpr int NM = n_moments<DIM>();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < mk.nel;
         e += (int64_t)gridDim.x * blockDim.x) {
        double M[NM];
#pragma unroll
        for (int q = 0; q < NM; q++) M[q] = mom[(int64_t)q * mk.nel + e];
        int ijk[3];
        elem_ijk(mk, e, ijk);
#pragma unroll
        for (int a = 0; a < (1 << DIM); a++) {
            double S[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double v = 0.0;
#pragma unroll
                for (int k0 = 0; k0 < 3; k0++)
#pragma unroll
                    for (int k1 = 0; k1 < 3; k1++)
#pragma unroll
                        for (int k2 = 0; k2 < 3; k2++) {
                            const int ex[3] = {k0, k1, k2};
                            bool ok = true;
                            double coef = 1.0;
#pragma unroll
                            for (int o = 0; o < 3; o++) {
                                if (o >= DIM || o == d) { if (ex[o] != 0) ok = false; continue; }
                                coef *= ex[o] == 1 ? 2.0 * (((a >> o) & 1) ? 1.0 : -1.0) : 1.0;
                            }
                            if (!ok) continue;
                            v += coef * M[mom_slot<DIM>(k0, k1, k2)];
                        }
                S[d] = v * mk.kappa[d] * mk.kappa[d];
            }
            const double tot = S[0] + S[1] + S[2];
            const int64_t n = elem_node<DIM>(mk, ijk, a);
#pragma unroll
            for (int c = 0; c < DIM; c++) atomicAdd(&diag[(int64_t)c * mk.nnode + n], (float)(tot + S[c]));
        }
    }
}

__global__ void k_invert_diag(int64_t n, int64_t nnode, const uint8_t* __restrict__ bc,
                              const float* __restrict__ diag, float* __restrict__ inv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / nnode);
        inv[i] = ((bc[i - (int64_t)c * nnode] >> c) & 1) ? 0.f : 1.f / diag[i];
    }
}

// coarse node (I,J,K) ↔ fine node (2I,2J,2K): the wall conditions map onto themselves
__global__ void k_coarse_bcmask(MeshK fk, MeshK ck, const uint8_t* __restrict__ bf, uint8_t* __restrict__ bcc) {
    for (int64_t N = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; N < ck.nnode;
         N += (int64_t)gridDim.x * blockDim.x) {
        const int I = (int)(N % ck.nn[0]);
        const int64_t rr = N / ck.nn[0];
        const int J = (int)(rr % ck.nn[1]), K = (int)(rr / ck.nn[1]);
        bcc[N] = bf[2 * I + (int64_t)fk.nn[0] * (2 * J + (int64_t)fk.nn[1] * 2 * K)];
    }
}

// b_c = Pᵀ r_f (full weighting without normalisation), zero on coarse BC dofs
template <int DIM>
__global__ void k_restrict(MeshK fk, MeshK ck, const uint8_t* __restrict__ bcc, const float* __restrict__ rf,
                           float* __restrict__ bcv, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t N = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; N < ck.nnode;
         N += (int64_t)gridDim.x * blockDim.x) {
        const int I = (int)(N % ck.nn[0]);
        const int64_t rr = N / ck.nn[0];
        const int J = (int)(rr % ck.nn[1]), K = DIM == 3 ? (int)(rr / ck.nn[1]) : 0;
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
                    if (i < 0 || j < 0 || k < 0 || i >= fk.nn[0] || j >= fk.nn[1] || k >= fk.nn[2]) continue;
                    const float w = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
                    const int64_t n = i + (int64_t)fk.nn[0] * (j + (int64_t)fk.nn[1] * k);
#pragma unroll
                    for (int c = 0; c < DIM; c++) acc[c] += w * rf[(int64_t)c * fk.nnode + n];
                }
        const uint8_t bm = bcc[N];
#pragma unroll
        for (int c = 0; c < DIM; c++) bcv[(int64_t)c * ck.nnode + N] = ((bm >> c) & 1) ? 0.f : acc[c];
    }
}

// x_f += P x_c (Q1 interpolation), fine BC dofs untouched
template <int DIM>
__global__ void k_prolong_add(MeshK fk, MeshK ck, const uint8_t* __restrict__ bcf, const float* __restrict__ xc,
                              float* __restrict__ xf, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < fk.nnode;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(n % fk.nn[0]);
        const int64_t rr = n / fk.nn[0];
        const int j = (int)(rr % fk.nn[1]), k = DIM == 3 ? (int)(rr / fk.nn[1]) : 0;
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
        float acc[DIM];
#pragma unroll
        for (int c = 0; c < DIM; c++) acc[c] = 0.f;
#pragma unroll
        for (int q = 0; q < (1 << DIM); q++) {
            const int I = (q & 1) ? hi[0] : lo[0], J = (q & 2) ? hi[1] : lo[1], K = (q & 4) ? hi[2] : lo[2];
            const float w = ((q & 1) ? wh[0] : wl[0]) * ((q & 2) ? wh[1] : wl[1]) * (DIM == 3 ? ((q & 4) ? wh[2] : wl[2]) : 1.f);
            if (w == 0.f) continue;
            const int64_t N = I + (int64_t)ck.nn[0] * (J + (int64_t)ck.nn[1] * K);
#pragma unroll
            for (int c = 0; c < DIM; c++) acc[c] += w * xc[(int64_t)c * ck.nnode + N];
        }
        const uint8_t bm = bcf[n];
#pragma unroll
        for (int c = 0; c < DIM; c++)
            if (!((bm >> c) & 1)) xf[(int64_t)c * fk.nnode + n] += acc[c];
    }
}

// ---- Chebyshev–Jacobi smoother vector steps --------------------------------------------
// start from x = 0: r = b, d = D⁻¹r/θ, x = d, t = 0
__global__ void k_cheb_start(int64_t n, const float* __restrict__ b, const float* __restrict__ invd, float inv_theta,
                             float* __restrict__ r, float* __restrict__ d, float* __restrict__ x,
                             float* __restrict__ t, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float rv = b[i];
        const float dv = inv_theta * invd[i] * rv;
        r[i] = rv;
        d[i] = dv;
        x[i] = dv;
        t[i] = 0.f;
    }
}
// post-smoothing start from x: r = b − t (t = A x), d = D⁻¹r/θ, x += d, t = 0
__global__ void k_cheb_restart(int64_t n, const float* __restrict__ b, const float* __restrict__ invd, float inv_theta,
                               float* __restrict__ r, float* __restrict__ d, float* __restrict__ x,
                               float* __restrict__ t, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float rv = b[i] - t[i];
        const float dv = inv_theta * invd[i] * rv;
        r[i] = rv;
        d[i] = dv;
        x[i] += dv;
        t[i] = 0.f;
    }
}
// r −= t (t = A d), d = c1 d + c2 D⁻¹ r, x += d, t = 0
__global__ void k_cheb_step(int64_t n, const float* __restrict__ invd, float c1, float c2, float* __restrict__ r,
                            float* __restrict__ d, float* __restrict__ x, float* __restrict__ t,
                            const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float rv = r[i] - t[i];
        const float dv = c1 * d[i] + c2 * invd[i] * rv;
        r[i] = rv;
        d[i] = dv;
        x[i] += dv;
        t[i] = 0.f;
    }
}
// r −= t, t = 0  (r = b − A x after the last step)
__global__ void k_resid_finish(int64_t n, float* __restrict__ r, float* __restrict__ t, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        r[i] -= t[i];
        t[i] = 0.f;
    }
}

// x = A⁻¹ b on the coarsest level: one warp per row of the dense FP32 inverse (rows
// padded to ld)
__global__ void k_dense_mv(int n, int ld, const float* __restrict__ A, const float* __restrict__ b,
                           float* __restrict__ x, const int32_t* __restrict__ done) {
    if (done && *done) return;
    const int lane = threadIdx.x & 31;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += (gridDim.x * blockDim.x) >> 5) {
        float s = 0.f;
        for (int k = lane; k < n; k += 32) s += A[(int64_t)row * ld + k] * b[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = s;
    }
}

__global__ void k_hash_fill(int64_t n, int64_t nnode, const uint8_t* __restrict__ bc, float* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t h = (uint32_t)i * 2654435761u + 0x9e3779b9u;
        h ^= h >> 15; h *= 0x85ebca6bu; h ^= h >> 13;
        const int c = (int)(i / nnode);
        x[i] = ((bc[i - (int64_t)c * nnode] >> c) & 1) ? 0.f : ((float)(h & 0xffffff) / 16777216.f - 0.5f);
    }
}

// y = D⁻¹ t, partial norms ‖y‖², ‖x‖²; t = 0
__global__ void k_power_step(int64_t n, const float* __restrict__ invd, const float* __restrict__ x,
                             float* __restrict__ t, float* __restrict__ y, double* __restrict__ part) {
    double yy = 0.0, xx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = invd[i] * t[i];
        y[i] = v;
        t[i] = 0.f;
        yy += (double)v * v;
        xx += (double)x[i] * x[i];
    }
    yy = block_sum(yy);
    __syncthreads();
    xx = block_sum(xx);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = yy;
        part[2 * blockIdx.x + 1] = xx;
    }
}

// Σ of the nb block partials in block order (one thread): state[0] = λ = √(‖y‖²/‖x‖²),
// state[1] = 1/‖y‖, state[2] ≠ 0 once a step was degenerate (λ then keeps its last value
// and x is no longer rescaled).
__global__ void k_power_norm(int nb, const double* __restrict__ part, double* __restrict__ state) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double yy = 0, xx = 0;
    for (int b = 0; b < nb; b++) {
        yy += part[2 * b];
        xx += part[2 * b + 1];
    }
    if (state[2] != 0.0 || xx <= 0 || yy <= 0) {
        state[2] = 1.0;
        return;
    }
    state[0] = sqrt(yy / xx);
    state[1] = 1.0 / sqrt(yy);
}

__global__ void k_scale(int64_t n, const double* __restrict__ state, const float* __restrict__ y,
                        float* __restrict__ x) {
    if (state[2] != 0.0) return;
    const float s = (float)state[1];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = s * y[i];
}

int g(int64_t n) { return grid_for(n, 256); }

}  // namespace

// Levels below the fine one smooth with degree ≤ 2: there a phase costs mostly its grid
// barrier, not its arithmetic.  Measured (creep 64³, fine degree 3): 314 → 280 ms per
// solve at 692 against 697 flexible-CG iterations; degree 1 below the fine level needs 957.
constexpr int kCoarseDegree = 2;
int level_degree(const Handle& H, size_t l) {
    const int deg = H.mg_degree;
    if (l == 0) return deg;
    return deg < kCoarseDegree ? deg : kCoarseDegree;
}

ChebCoef cheb_coef(double lmax_est, int degree) {
    const double lmax = 1.1 * lmax_est, lmin = 0.1 * lmax_est;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    ChebCoef cc{};
    cc.inv_theta = (float)(1.0 / theta);
    double rho = 1.0 / sigma;
    for (int k = 1; k < degree && k < 8; k++) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        cc.c1[k] = (float)(rn * rho);
        cc.c2[k] = (float)(2.0 * rn / delta);
        rho = rn;
    }
    return cc;
}

// Enqueue the V-cycle z = M⁻¹ b on level l (b and x are level-l vectors).
void vcycle(Handle& H, size_t l, const float* b, float* x, const int32_t* done) {
    MGLevel& L = *H.mg[l];
    cudaStream_t st = H.stream;
    const int64_t n = L.ndof;
    const int dim = H.dim;
    if (l + 1 == H.mg.size()) {
        if (H.coarse_n) {
            k_dense_mv<<<g((int64_t)H.coarse_n * 32), 256, 0, st>>>((int)H.coarse_n, (int)H.coarse_ld,
                                                                   H.coarse_inv.as<float>(), b, x, done);
            H.kernel_launches++;
            return;
        }
        // no dense solve: a long Chebyshev sweep from zero
        ChebCoef cc = cheb_coef(L.lambda_max, 8);
        k_cheb_start<<<g(n), 256, 0, st>>>(n, b, L.invdiag.as<float>(), cc.inv_theta, L.r.as<float>(), L.d.as<float>(), x,
                                           L.t.as<float>(), done);
        for (int k = 1; k < 8; k++) {
            apply_K_ex<float>(L.mk, L.mom32, L.bcmask, L.d.as<float>(), L.t.as<float>(), nullptr, apply_grid(L.nel), st, done);
            k_cheb_step<<<g(n), 256, 0, st>>>(n, L.invdiag.as<float>(), cc.c1[k], cc.c2[k], L.r.as<float>(), L.d.as<float>(),
                                              x, L.t.as<float>(), done);
        }
        H.kernel_launches += 15;
        return;
    }
    MGLevel& C = *H.mg[l + 1];
    const int deg = level_degree(H, l);
    ChebCoef cc = cheb_coef(L.lambda_max, deg);
    float* r = L.r.as<float>();
    float* d = L.d.as<float>();
    float* t = L.t.as<float>();
    const float* invd = L.invdiag.as<float>();
    const int ga = apply_grid(L.nel);
    // pre-smoothing from zero; the last apply leaves r = b − A x
    k_cheb_start<<<g(n), 256, 0, st>>>(n, b, invd, cc.inv_theta, r, d, x, t, done);
    for (int k = 1; k < deg; k++) {
        apply_K_ex<float>(L.mk, L.mom32, L.bcmask, d, t, nullptr, ga, st, done);
        k_cheb_step<<<g(n), 256, 0, st>>>(n, invd, cc.c1[k], cc.c2[k], r, d, x, t, done);
    }
    apply_K_ex<float>(L.mk, L.mom32, L.bcmask, d, t, nullptr, ga, st, done);
    k_resid_finish<<<g(n), 256, 0, st>>>(n, r, t, done);
    // coarse-grid correction
    if (dim == 2) k_restrict<2><<<g(C.nnode), 256, 0, st>>>(L.mk, C.mk, C.bcmask, r, C.b.as<float>(), done);
    else k_restrict<3><<<g(C.nnode), 256, 0, st>>>(L.mk, C.mk, C.bcmask, r, C.b.as<float>(), done);
    vcycle(H, l + 1, C.b.as<float>(), C.x.as<float>(), done);
    if (dim == 2) k_prolong_add<2><<<g(L.nnode), 256, 0, st>>>(L.mk, C.mk, L.bcmask, C.x.as<float>(), x, done);
    else k_prolong_add<3><<<g(L.nnode), 256, 0, st>>>(L.mk, C.mk, L.bcmask, C.x.as<float>(), x, done);
    // post-smoothing from x
    apply_K_ex<float>(L.mk, L.mom32, L.bcmask, x, t, nullptr, ga, st, done);
    k_cheb_restart<<<g(n), 256, 0, st>>>(n, b, invd, cc.inv_theta, r, d, x, t, done);
    for (int k = 1; k < deg; k++) {
        apply_K_ex<float>(L.mk, L.mom32, L.bcmask, d, t, nullptr, ga, st, done);
        k_cheb_step<<<g(n), 256, 0, st>>>(n, invd, cc.c1[k], cc.c2[k], r, d, x, t, done);
    }
    H.kernel_launches += 6 + 4 * deg;
}

// level l−1 → l restriction and l → l−1 prolongation-add (used by the learned correction)
void mg_restrict(Handle& H, size_t l, const float* fine, float* coarse, const int32_t* done) {
    MGLevel& F = *H.mg[l - 1];
    MGLevel& C = *H.mg[l];
    if (H.dim == 2) k_restrict<2><<<g(C.nnode), 256, 0, H.stream>>>(F.mk, C.mk, C.bcmask, fine, coarse, done);
    else k_restrict<3><<<g(C.nnode), 256, 0, H.stream>>>(F.mk, C.mk, C.bcmask, fine, coarse, done);
    H.kernel_launches++;
}
void mg_prolong_add(Handle& H, size_t l, const float* coarse, float* fine, const int32_t* done) {
    MGLevel& F = *H.mg[l - 1];
    MGLevel& C = *H.mg[l];
    if (H.dim == 2) k_prolong_add<2><<<g(F.nnode), 256, 0, H.stream>>>(F.mk, C.mk, F.bcmask, coarse, fine, done);
    else k_prolong_add<3><<<g(F.nnode), 256, 0, H.stream>>>(F.mk, C.mk, F.bcmask, coarse, fine, done);
    H.kernel_launches++;
}

static double power_lambda(Handle& H, MGLevel& L) {
    cudaStream_t st = H.stream;
    const int64_t n = L.ndof;
    const int nb = 64;
    H.mg_part.ensure(sizeof(double) * (2 * nb + 4));
    double* part = H.mg_part.as<double>();
    double* state = part + 2 * nb;
    float* x = L.x.as<float>();
    float* y = L.d.as<float>();
    float* t = L.t.as<float>();
    k_hash_fill<<<g(n), 256, 0, st>>>(n, L.nnode, L.bcmask, x);
    GG_CUDA(cudaMemsetAsync(t, 0, sizeof(float) * n, st));
    GG_CUDA(cudaMemsetAsync(state, 0, sizeof(double) * 4, st));
    // 12 steps queued without a host round trip; λ is read once at the end
    for (int it = 0; it < 12; it++) {
        apply_K_ex<float>(L.mk, L.mom32, L.bcmask, x, t, nullptr, apply_grid(L.nel), st, nullptr);
        k_power_step<<<nb, 256, 0, st>>>(n, L.invdiag.as<float>(), x, t, y, part);
        k_power_norm<<<1, 32, 0, st>>>(nb, part, state);
        k_scale<<<g(n), 256, 0, st>>>(n, state, y, x);
    }
    H.kernel_launches += 1 + 4 * 12;  // start vector, then 12 × (apply, step, norm, scale)
    double lam = 0.0;
    GG_CUDA(cudaMemcpyAsync(&lam, state, sizeof(double), cudaMemcpyDeviceToHost, st));
    GG_CUDA(cudaStreamSynchronize(st));
    GG_CUDA(cudaGetLastError());
    return lam;
}

// ---- blocked Gauss–Jordan inversion, in place, FP64 ------------------------------------
// For pivot blocks K = [k0, k0 + b) in turn (b ≤ kGjB), with D = W[K,K]:
//   W[i,j] −= W[i,K] D⁻¹ W[K,j]   (i, j ∉ K)      W[K,j] = D⁻¹ W[K,j]   (j ∉ K)
//   W[i,K]  = −W[i,K] D⁻¹         (i ∉ K)         W[K,K] = D⁻¹
// after the last block W holds the inverse.  No pivoting: every leading Schur complement
// of a symmetric positive definite matrix is symmetric positive definite.  The work is a
// rank-b update of the whole matrix per block (n³ multiply-adds in all, on the SMs' FP64
// units from shared-memory tiles); the only sequential part is the b steps inside each
// diagonal block, n steps in all.
constexpr int kGjB = 64;      // pivot block
constexpr int kGjTile = 64;   // output tile of the update (256 threads × 4 × 4)

// W = A as rows (A holds the columns K e_j; K is symmetric up to the order of its FP64
// sums, and the transpose keeps W = K exactly), BC rows and columns replaced by the identity
__global__ void k_bgj_init(int64_t n, int64_t nnode, const uint8_t* __restrict__ bc, const double* __restrict__ A,
                           double* __restrict__ W) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q / n, j = q - i * n;
        const int ci = (int)(i / nnode), cj = (int)(j / nnode);
        const bool fi = (bc[i - ci * nnode] >> ci) & 1, fj = (bc[j - cj * nnode] >> cj) & 1;
        W[q] = (fi || fj) ? (i == j ? 1.0 : 0.0) : A[j * n + i];
    }
}

// D⁻¹ of a pivot block by element-wise Gauss–Jordan steps, the block padded to 64 × 64 with
// the identity (the padded inverse holds D⁻¹ in its top left b × b).  256 threads; thread
// (ty, tx) keeps entries (ty + 16r, tx + 16c), r, c < 4, of the block in a[r][c] for all 64
// steps.  A step needs, besides a thread's own entries, only the pivot row and the pivot
// column: the threads that own row and column p + 1 publish their new values into the other
// half of a double-buffered pair of 64-entry arrays, so each step takes one barrier.  On
// return a[][] holds the padded inverse; the caller writes D⁻¹ out.
__device__ __forceinline__ void gj_block_inverse(double (&a)[4][4], int ty, int tx, double (*s_row)[kGjB],
                                                 double (*s_col)[kGjB]) {
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int i = ty + 16 * r, j = tx + 16 * c;
            if (i == 0) s_row[0][j] = a[r][c];
            if (j == 0) s_col[0][i] = a[r][c];
        }
    __syncthreads();
    for (int p = 0; p < kGjB; p++) {
        const int h = p & 1;
        const double piv = __drcp_rn(s_row[h][p]);
        double dip[4], t[4];
#pragma unroll
        for (int r = 0; r < 4; r++) dip[r] = s_col[h][ty + 16 * r];
#pragma unroll
        for (int c = 0; c < 4; c++) t[c] = s_row[h][tx + 16 * c] * piv;
        // every entry takes the elimination a − a[i][p]·(a[p][j]/a[p][p]); then the pivot
        // row becomes a[p][j]/a[p][p] (1/a[p][p] on the diagonal) and the pivot column
        // −a[i][p]/a[p][p]
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) a[r][c] = a[r][c] - dip[r] * t[c];
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (ty + 16 * r == p) {
#pragma unroll
                for (int c = 0; c < 4; c++) a[r][c] = tx + 16 * c == p ? piv : t[c];
            }
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (tx + 16 * c == p) {
#pragma unroll
                for (int r = 0; r < 4; r++)
                    if (ty + 16 * r != p) a[r][c] = -dip[r] * piv;
            }
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (ty + 16 * r == p + 1) {
#pragma unroll
                for (int c = 0; c < 4; c++) s_row[h ^ 1][tx + 16 * c] = a[r][c];
            }
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (tx + 16 * c == p + 1) {
#pragma unroll
                for (int r = 0; r < 4; r++) s_col[h ^ 1][ty + 16 * r] = a[r][c];
            }
        __syncthreads();
    }
}

__device__ __forceinline__ void gj_store_inverse(const double (&a)[4][4], int ty, int tx, int b,
                                                 double* __restrict__ Dinv) {
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int i = ty + 16 * r, j = tx + 16 * c;
            if (i < b && j < b) Dinv[i * b + j] = a[r][c];
        }
}

// D⁻¹ of the first pivot block (every later one is inverted by the update before it)
__global__ void __launch_bounds__(256) k_bgj_pivot(int64_t n, int64_t k0, int b, const double* __restrict__ W,
                                                   double* __restrict__ Dinv) {
    __shared__ double s_row[2][kGjB], s_col[2][kGjB];
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    double a[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int i = ty + 16 * r, j = tx + 16 * c;
            a[r][c] = (i < b && j < b) ? W[(k0 + i) * n + k0 + j] : (i == j ? 1.0 : 0.0);
        }
    gj_block_inverse(a, ty, tx, s_row, s_col);
    gj_store_inverse(a, ty, tx, b, Dinv);
}

// The pivot block's row panel R[m][j] = (D⁻¹ W[K,:])[m][j] (columns j ∈ K: D⁻¹ itself) and
// a copy of its column panel, stored transposed CT[m][i] = W[i][k0+m], both from W before
// the update.  One CTA of 256 threads per 32 columns (blockIdx.y = 0: the row panel, D⁻¹ and the 64 × 32
// tile of W[K,:] staged in shared memory, 8 outputs a thread, each a sum over l in order)
// or per 32 rows (blockIdx.y = 1: the column panel, transposed through shared memory so
// that both the reads and the writes are coalesced).
constexpr int kGjPanelCols = 32;
__global__ void __launch_bounds__(256) k_bgj_panels(int64_t n, int64_t k0, int b, const double* __restrict__ W,
                                                    const double* __restrict__ Dinv, double* __restrict__ R,
                                                    double* __restrict__ C) {
    __shared__ double sm[kGjB * kGjB + kGjB * kGjPanelCols];  // 48 KB
    const int64_t t0 = (int64_t)blockIdx.x * kGjPanelCols;
    if (blockIdx.y == 0) {
        double* Ds = sm;                // [m][l]
        double* Ws = sm + kGjB * kGjB;  // [l][t]
        for (int q = threadIdx.x; q < kGjB * kGjB; q += blockDim.x) {
            const int m = q / kGjB, l = q % kGjB;
            Ds[q] = m < b && l < b ? Dinv[m * b + l] : 0.0;
        }
        for (int q = threadIdx.x; q < kGjB * kGjPanelCols; q += blockDim.x) {
            const int l = q / kGjPanelCols, t = q % kGjPanelCols;
            Ws[q] = l < b && t0 + t < n ? W[(k0 + l) * n + t0 + t] : 0.0;
        }
        __syncthreads();
        const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int m = ty + 16 * r;
            if (m >= b) continue;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int64_t j = t0 + tx + 16 * c;
                if (j >= n) continue;
                double v;
                if (j >= k0 && j < k0 + b) {
                    v = Ds[m * kGjB + (j - k0)];
                } else {
                    v = 0.0;
                    for (int l = 0; l < b; l++) v += Ds[m * kGjB + l] * Ws[l * kGjPanelCols + tx + 16 * c];
                }
                R[m * n + j] = v;
            }
        }
    } else {
        constexpr int S = kGjPanelCols + 1;
        double* Ts = sm;  // [m][i] with a row stride of 33
        for (int q = threadIdx.x; q < kGjPanelCols * kGjB; q += blockDim.x) {
            const int i = q / kGjB, m = q % kGjB;
            if (m < b && t0 + i < n) Ts[m * S + i] = W[(t0 + i) * n + k0 + m];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < kGjB * kGjPanelCols; q += blockDim.x) {
            const int m = q / kGjPanelCols, i = q % kGjPanelCols;
            if (m < b && t0 + i < n) C[(int64_t)m * n + t0 + i] = Ts[m * S + i];
        }
    }
}

// The rank-b update of one 64 × 64 output tile: rows in K take the row panel, every other
// row W[i,j] (or 0 for j ∈ K) minus C[i,:]·R[:,j].  C (stored transposed) and R tiles are
// staged in shared memory by coalesced loads (64 KB); each thread forms 4 × 4 outputs at a
// stride of 16 rows and columns (a half-warp reads and writes 16 consecutive doubles), its
// 16 old values of W loaded before the multiply-add loop so that their latency hides behind
// it.  The in-place inverse of a symmetric matrix keeps a fixed structure: with P the
// blocks already eliminated and U the rest, W[P,P] and W[U,U] are symmetric and
// W[U,P] = −W[P,U]ᵀ.  So one CTA per tile (I, J) with I ≤ J (tiles are the pivot blocks)
// computes its tile and, for I < J, writes the mirror tile (J, I), transposed through
// shared memory with the sign −1 when exactly one of I, J is in P after this step.  That
// halves the multiply-adds.  When a next pivot block of bn rows follows (it starts at
// k0 + 64, on the tile grid), the CTA that updates its diagonal tile is scheduled first and
// goes on to invert it from its registers (the layout of gj_block_inverse) into Dinv, while
// the others finish the update: the next panels launch finds D⁻¹ ready.
constexpr size_t kGjUpdateSmem = sizeof(double) * 2 * kGjB * kGjTile;
__global__ void __launch_bounds__(256) k_bgj_update(int64_t n, int64_t k0, int b, double* __restrict__ W,
                                                    const double* __restrict__ R, const double* __restrict__ C,
                                                    int bn, double* __restrict__ Dinv) {
    extern __shared__ double s_bgj[];
    __shared__ double s_row[2][kGjB], s_col[2][kGjB];
    double* Cs = s_bgj;                   // [kGjB][kGjTile]
    double* Rs = s_bgj + kGjB * kGjTile;  // [kGjB][kGjTile]
    const int64_t nt = (n + kGjTile - 1) / kGjTile;
    const int64_t kb = k0 / kGjTile;  // this step's pivot block
    // upper-triangle tile t ↔ (I, J), I ≤ J: row I starts at off(I) = I·nt − I(I−1)/2
    auto off = [nt](int64_t I) { return I * nt - I * (I - 1) / 2; };
    const int64_t dn = bn > 0 ? off(kb + 1) : 0;  // the next diagonal tile (kb + 1, kb + 1)
    int64_t tile = blockIdx.x;
    if (tile == 0) tile = dn;
    else if (tile == dn) tile = 0;
    int64_t I = 0;
    while (off(I + 1) <= tile) I++;
    const int64_t J = I + (tile - off(I));
    const int64_t i0 = I * kGjTile, j0 = J * kGjTile;
    for (int q = threadIdx.x; q < kGjB * kGjTile; q += blockDim.x) {
        const int m = q / kGjTile, t = q % kGjTile;
        const bool ok = m < b;
        Cs[q] = ok && i0 + t < n ? C[(int64_t)m * n + i0 + t] : 0.0;
        Rs[q] = ok && j0 + t < n ? R[(int64_t)m * n + j0 + t] : 0.0;
    }
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    double old[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int64_t i = i0 + ty + 16 * r;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int64_t j = j0 + tx + 16 * c;
            const bool keep = i < n && j < n && !(i >= k0 && i < k0 + b) && !(j >= k0 && j < k0 + b);
            old[r][c] = keep ? W[i * n + j] : 0.0;
        }
    }
    __syncthreads();
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
    for (int m = 0; m < b; m++) {
        double cv[4], rv[4];
#pragma unroll
        for (int r = 0; r < 4; r++) cv[r] = Cs[m * kGjTile + ty + 16 * r];
#pragma unroll
        for (int c = 0; c < 4; c++) rv[c] = Rs[m * kGjTile + tx + 16 * c];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[r][c] += cv[r] * rv[c];
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int64_t i = i0 + ty + 16 * r;
        if (i >= n) continue;
        const bool rowK = i >= k0 && i < k0 + b;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int64_t j = j0 + tx + 16 * c;
            if (j >= n) continue;
            const double v = rowK ? R[(i - k0) * n + j] : old[r][c] - acc[r][c];
            W[i * n + j] = v;
            acc[r][c] = v;
        }
    }
    if (I != J) {
        constexpr int S = kGjTile + 1;
        const double sgn = ((I <= kb) != (J <= kb)) ? -1.0 : 1.0;
        double* Ts = s_bgj;  // [j - j0][i - i0]
        __syncthreads();     // every thread is done with the C and R tiles
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) Ts[(tx + 16 * c) * S + ty + 16 * r] = sgn * acc[r][c];
        __syncthreads();
        for (int q = threadIdx.x; q < kGjTile * kGjTile; q += blockDim.x) {
            const int jl = q / kGjTile, il = q % kGjTile;
            const int64_t j = j0 + jl, i = i0 + il;
            if (i < n && j < n) W[j * n + i] = Ts[jl * S + il];
        }
    }
    if (bn > 0 && tile == dn) {
        // this tile is the next pivot block: rows and columns k0 + 64 + [0, bn)
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int i = ty + 16 * r, j = tx + 16 * c;
                if (!(i < bn && j < bn)) acc[r][c] = i == j ? 1.0 : 0.0;
            }
        gj_block_inverse(acc, ty, tx, s_row, s_col);
        gj_store_inverse(acc, ty, tx, bn, Dinv);
    }
}

// the FP32 inverse with rows padded to ld (a multiple of 4) for float4 mat-vecs
__global__ void k_bgj_extract(int64_t n, int64_t ld, const double* __restrict__ W, float* __restrict__ inv) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * ld; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q / ld, j = q - i * ld;
        inv[q] = j < n ? (float)W[i * n + j] : 0.f;
    }
}

// Dense FP32 inverse of the coarsest operator: its columns by unit-vector applies, then
// Gauss–Jordan on the device (n steps of one kernel each).
// Column j of the coarsest operator, A[:, j] = K e_j, from every element that touches dof
// j: one thread per (element, element-local dof), the element arithmetic of the apply on
// the unit vector, scattered into column j (BC rows skipped; columns of BC dofs stay zero).
template <int DIM>
__global__ void k_coarse_columns(MeshK mk, const double* __restrict__ mom, const uint8_t* __restrict__ bc,
                                 double* __restrict__ A) {
    constexpr int NS = 1 << DIM, NR = NS / 2, NM = n_moments<DIM>();
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < mk.nel * NS * DIM;
         q += (int64_t)gridDim.x * blockDim.x) {
    const int32_t e = (int32_t)(q / (NS * DIM));
    const int loc = (int)(q - (int64_t)e * NS * DIM);
    const int ja = loc / DIM, jc = loc - ja * DIM;  // corner and component of the column's dof
    int ijk[3];
    elem_ijk(mk, e, ijk);
    const int32_t nn0 = mk.nn[0], nn01 = mk.nn[0] * mk.nn[1];
    const int32_t n0 = ijk[0] + nn0 * ijk[1] + (DIM == 3 ? nn01 * ijk[2] : 0);
    uint32_t fixed = 0;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const uint8_t* br = bc + n0 + (r & 1) * nn0 + (DIM == 3 ? ((r >> 1) & 1) * nn01 : 0);
        fixed |= ((uint32_t)br[0] | ((uint32_t)br[1] << 4)) << (8 * r);
    }
    // corner ja = (dx, dy, dz) sits in row ja >> 1 at word dx
    if ((fixed >> (8 * (ja >> 1) + 4 * (ja & 1) + jc)) & 1) continue;
    const int32_t node = n0 + (ja & 1) + ((ja >> 1) & 1) * nn0 + (DIM == 3 ? ((ja >> 2) & 1) * nn01 : 0);
    double m[DIM][NS];
#pragma unroll
    for (int c = 0; c < DIM; c++)
#pragma unroll
        for (int a = 0; a < NS; a++) m[c][a] = (c == jc && a == ja) ? 1.0 : 0.0;
    double M[NM];
#pragma unroll
    for (int k = 0; k < NM; k++) M[k] = mom[(int64_t)k * mk.nel + e];
    double* col = A + ((int64_t)jc * mk.nnode + node) * ((int64_t)DIM * mk.nnode);
    element_compute_scatter<DIM, double, false>(mk, m, M, fixed, col, n0);
    }
}

// Dense FP32 inverse of the coarsest operator: its columns by unit-vector applies (FP64),
// then the blocked Gauss–Jordan inversion above (FP64), rounded to FP32 with rows padded
// to a multiple of 4.  Two launches per pivot block of 64 (panels, update with the next
// block's inverse) after one for the first block's inverse: the 8³ level of a 64³ mesh
// (2,187 dofs) takes 35 blocks.
static void coarse_inverse(Handle& H, MGLevel& L) {
    const int64_t n = L.ndof;
    const int64_t ld = (n + 3) & ~(int64_t)3;
    cudaStream_t st = H.stream;
    H.mg_dense.ensure(sizeof(double) * (2 * n * n + 2 * n * kGjB + kGjB * kGjB));
    double* A = H.mg_dense.as<double>();
    double* W = A + n * n;
    double* R = W + n * n;
    double* Cp = R + n * kGjB;
    double* Dinv = Cp + n * kGjB;
    GG_CUDA(cudaMemsetAsync(A, 0, sizeof(double) * n * n, st));
    const int64_t threads = L.nel * (int64_t)(H.dim == 3 ? 24 : 8);
    if (H.dim == 3) k_coarse_columns<3><<<grid_for(threads, 128), 128, 0, st>>>(L.mk, L.mom64, L.bcmask, A);
    else k_coarse_columns<2><<<grid_for(threads, 128), 128, 0, st>>>(L.mk, L.mom64, L.bcmask, A);
    k_bgj_init<<<grid_for(n * n, 256), 256, 0, st>>>(n, L.nnode, L.bcmask, A, W);
    static std::atomic<bool> smem_set[64];
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !smem_set[dev].load()) {
        GG_CUDA(cudaFuncSetAttribute(k_bgj_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGjUpdateSmem));
        smem_set[dev].store(true);
    }
    const int64_t ntile = (n + kGjTile - 1) / kGjTile;
    const unsigned tiles = (unsigned)(ntile * (ntile + 1) / 2);  // I ≤ J
    const dim3 panels((unsigned)((n + kGjPanelCols - 1) / kGjPanelCols), 2);
    int64_t launches = 0;
    k_bgj_pivot<<<1, 256, 0, st>>>(n, 0, (int)std::min<int64_t>(kGjB, n), W, Dinv);
    launches++;
    for (int64_t k0 = 0; k0 < n; k0 += kGjB) {
        const int b = (int)std::min<int64_t>(kGjB, n - k0);
        const int bn = (int)std::max<int64_t>(0, std::min<int64_t>(kGjB, n - k0 - kGjB));
        k_bgj_panels<<<panels, 256, 0, st>>>(n, k0, b, W, Dinv, R, Cp);
        k_bgj_update<<<tiles, 256, kGjUpdateSmem, st>>>(n, k0, b, W, R, Cp, bn, Dinv);
        launches += 2;
    }
    H.coarse_inv.ensure(sizeof(float) * n * ld);
    k_bgj_extract<<<grid_for(n * ld, 256), 256, 0, st>>>(n, ld, W, H.coarse_inv.as<float>());
    GG_CUDA(cudaGetLastError());
    H.kernel_launches += launches + 3;
    GG_CUDA(cudaStreamSynchronize(st));
    H.coarse_n = n;
    H.coarse_ld = ld;
}

// Build (or refresh for a new operator) the hierarchy.  Needs the mixed build (FP32 moments).
// Copies of the coarsest level's dense FP32 inverse (rows of n) and of the FP64 operator it
// inverts (row-major, Dirichlet rows and columns replaced by the identity), for inspection.
int coarse_inverse_copy(Handle& H, int64_t* n, float* inv, double* op) {
    const int rc = mg_setup(H);
    if (rc != GG_OK) return rc;
    *n = H.coarse_n;
    if (!H.coarse_n) return GG_OK;
    const int64_t m = H.coarse_n;
    cudaStream_t st = H.stream;
    if (inv)
        GG_CUDA(cudaMemcpy2DAsync(inv, sizeof(float) * m, H.coarse_inv.p, sizeof(float) * H.coarse_ld,
                                  sizeof(float) * m, m, cudaMemcpyDeviceToHost, st));
    if (op) {
        MGLevel& L = *H.mg.back();
        double* A = H.mg_dense.as<double>();  // the operator's columns, kept after the inversion
        double* W = A + m * m;
        k_bgj_init<<<grid_for(m * m, 256), 256, 0, st>>>(m, L.nnode, L.bcmask, A, W);
        GG_CUDA(cudaGetLastError());
        GG_CUDA(cudaMemcpyAsync(op, W, sizeof(double) * m * m, cudaMemcpyDeviceToHost, st));
    }
    GG_CUDA(cudaStreamSynchronize(st));
    return GG_OK;
}

int mg_setup(Handle& H) {
    if (H.mg_gen == H.build_gen && !H.mg.empty()) return GG_OK;
    cudaStream_t st = H.stream;
    const int dim = H.dim;
    if (H.mg.empty()) {
        auto L0 = std::make_unique<MGLevel>();
        L0->mk = H.mk;
        H.mg.push_back(std::move(L0));
        for (;;) {
            const MeshK& f = H.mg.back()->mk;
            // a level small enough for the dense coarse inverse ends the hierarchy
            if (H.mg.size() > 1 && f.nnode * dim <= kDenseStop) break;
            bool can = true;
            for (int d = 0; d < dim; d++)
                if (f.n[d] % 2 != 0 || f.n[d] < kMinCoarse) can = false;
            if (!can) break;
            gg_mesh_desc cd{};
            cd.dim = dim;
            for (int d = 0; d < dim; d++) {
                cd.elements[d] = f.n[d] / 2;
                cd.min[d] = f.min[d];
                cd.max[d] = f.max[d];
            }
            auto C = std::make_unique<MGLevel>();
            C->mk = make_mesh(cd);
            H.mg.push_back(std::move(C));
        }
        for (size_t l = 0; l < H.mg.size(); l++) {
            MGLevel& L = *H.mg[l];
            L.nnode = L.mk.nnode;
            L.nel = L.mk.nel;
            L.ndof = L.nnode * dim;
            for (DBuf* b : {&L.x, &L.b, &L.r, &L.d, &L.t, &L.invdiag}) b->ensure(sizeof(float) * L.ndof);
            if (l > 0) {
                L.own_mom64.ensure(sizeof(double) * H.nm * L.nel);
                L.own_mom32.ensure(sizeof(float) * H.nm * L.nel);
                L.own_bcmask.ensure(L.nnode);
            }
        }
    }
    // operators
    MGLevel& L0 = *H.mg[0];
    L0.mom64 = H.mom64.as<double>();
    L0.mom32 = H.mom32.as<float>();
    L0.bcmask = H.bcmask.as<uint8_t>();
    k_invert_diag<<<g(L0.ndof), 256, 0, st>>>(L0.ndof, L0.nnode, L0.bcmask, H.kdiag32.as<float>(), L0.invdiag.as<float>());
    for (size_t l = 1; l < H.mg.size(); l++) {
        MGLevel& F = *H.mg[l - 1];
        MGLevel& L = *H.mg[l];
        L.mom64 = L.own_mom64.as<double>();
        L.mom32 = L.own_mom32.as<float>();
        L.bcmask = L.own_bcmask.as<uint8_t>();
        k_coarse_bcmask<<<g(L.nnode), 256, 0, st>>>(F.mk, L.mk, F.bcmask, L.own_bcmask.as<uint8_t>());
        if (dim == 2) k_coarsen_moments<2><<<g(L.nel), 128, 0, st>>>(F.mk, L.mk, F.mom64, L.own_mom64.as<double>(), L.own_mom32.as<float>());
        else k_coarsen_moments<3><<<g(L.nel), 128, 0, st>>>(F.mk, L.mk, F.mom64, L.own_mom64.as<double>(), L.own_mom32.as<float>());
        GG_CUDA(cudaMemsetAsync(L.t.p, 0, sizeof(float) * L.ndof, st));
        if (dim == 2) k_level_diag<2><<<g(L.nel), 128, 0, st>>>(L.mk, L.mom64, L.t.as<float>());
        else k_level_diag<3><<<g(L.nel), 128, 0, st>>>(L.mk, L.mom64, L.t.as<float>());
        k_invert_diag<<<g(L.ndof), 256, 0, st>>>(L.ndof, L.nnode, L.bcmask, L.t.as<float>(), L.invdiag.as<float>());
        GG_CUDA(cudaGetLastError());
    }
    for (auto& L : H.mg) L->lambda_max = power_lambda(H, *L);
    // diag inversion + per coarse level (mask, moments, diag, inversion); power_lambda counts
    // its own launches
    H.kernel_launches += 1 + 4 * (int64_t)(H.mg.size() - 1);
    MGLevel& Lc = *H.mg.back();
    H.coarse_n = 0;
    if (H.mg.size() > 1 && Lc.ndof <= kDenseStop) coarse_inverse(H, Lc);
    GG_CUDA(cudaStreamSynchronize(st));
    H.mg_gen = H.build_gen;
    return GG_OK;
}

}  // namespace gg
